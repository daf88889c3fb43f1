/* acfdtd_b200.h -- C ABI of the sm_100a staggered pressure-velocity leapfrog.
 *
 * One solver handle owns the device state of one rectangular room: the pressure p at cell
 * centres, the three face velocities vx, vy, vz, and up to four ISO 9613-1 relaxation states.
 * Every call returns an int status (ACF_OK on success); acf_last_error() gives a message for
 * the last failure on the calling thread.
 *
 * Interfaces replaced (paths are inside the ac-fdtd project):
 *   acf_create / acf_run      <- struct `acfdtd` + acfdtd_run(acfdtd*, int64_t step_offset)
 *                                (src/ac_fdtd/c/acfdtd.c:56-97, 355-376). The reference borrows
 *                                caller arrays for the duration of one call; here the handle owns
 *                                device buffers and the caller moves state with acf_upload and
 *                                acf_download.
 *   acf_struct_size           <- acfdtd_struct_size (src/ac_fdtd/c/acfdtd.c:99), the ctypes
 *                                mirror check of src/ac_fdtd/c_backend.py:194-200.
 *   acf_is_double             <- acfdtd_is_double (src/ac_fdtd/c/acfdtd.c:101); the precision
 *                                is a per-handle choice here, not a build option.
 *   acf_energy_terms          <- AcousticFDTD.energy (src/ac_fdtd/scheme.py:365-389).
 *
 * Coefficients cross the boundary in FP64 and are rounded once to the solver precision, as
 * the reference casts its FP64 host setup with `dtype.type(...)`/`astype(dtype)`
 * (src/ac_fdtd/scheme.py:135-212).
 *
 * Streams are passed as `void*` (a cudaStream_t, 0 for the legacy default stream) so that FFI
 * callers need no CUDA headers.
 */
#ifndef ACFDTD_B200_H
#define ACFDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACF_ABI_VERSION 1
#define ACF_MAX_RELAXATION 4

/* Status codes. */
enum {
    ACF_OK = 0,
    ACF_ERR_ARGUMENT = 1,    /* a null pointer, a size out of range, an unknown field */
    ACF_ERR_CUDA = 2,        /* a CUDA runtime call failed; see acf_last_error() */
    ACF_ERR_MEMORY = 3,      /* device or pinned host allocation failed */
    ACF_ERR_STATE = 4,       /* call not valid in the handle's current state */
    ACF_ERR_NUMERIC = 5      /* non-finite value detected in the state */
};

/* Fields addressable by acf_upload / acf_download / acf_field_pointer. The relaxation state r
 * is ACF_FIELD_PSI0 + r. Reference shapes (C order, z fastest): p (nx,ny,nz); vx (nx+1,ny,nz);
 * vy (nx,ny+1,nz); vz (nx,ny,nz+1); psi_r (nx,ny,nz) -- src/ac_fdtd/grid.py:125-129. */
enum {
    ACF_FIELD_P = 0,
    ACF_FIELD_VX = 1,
    ACF_FIELD_VY = 2,
    ACF_FIELD_VZ = 3,
    ACF_FIELD_PSI0 = 4
};

typedef struct acf_solver acf_solver;
typedef struct acf_batch acf_batch;
typedef void *acf_stream;

/* Everything the two sweeps need, computed on the host in FP64.
 *
 * Wall coefficients use a shell layout: for each of the six faces in the reference's FACES
 * order ((0,0),(0,1),(1,0),(1,1),(2,0),(2,1); src/ac_fdtd/boundaries.py:73), a row-major
 * (n_b, n_c) array over the two remaining axes in increasing order, holding for every cell on
 * that face the pair (1/(1+a), a/(1+a)) where a is the sum over ALL faces touching the cell
 * (src/ac_fdtd/boundaries.py:167-207). Pair (1, 0) marks a cell with no absorbing face. Pass
 * NULL for all six when every wall is rigid.
 *
 * Layer profiles (src/ac_fdtd/boundaries.py:244-283): cell[a] has n_a entries (cell centres),
 * face[a] has n_a + 1 (faces). Pass NULL for all six when there is no absorbing layer. */
typedef struct acf_config {
    int32_t nx, ny, nz;
    int32_t precision;   /* bytes per element: 4 (float) or 8 (double) */
    int32_t n_relax;     /* 0 .. ACF_MAX_RELAXATION */
    int32_t reserved;
    double vel_coef;     /* dt / (rho dx)                         scheme.py:135 */
    double pres_coef;    /* rho c^2 dt / dx                       scheme.py:136-138 */
    double src_coef;     /* rho c^2 dt                            scheme.py:141 */
    double relax_scale;  /* dt * sum of gains                     scheme.py:189-191 */
    double relax_decay[ACF_MAX_RELAXATION];  /* exp(-dt/tau)         scheme.py:172 */
    double relax_mean[ACF_MAX_RELAXATION];   /* dt * mean weight     scheme.py:176,182 */
    double relax_gain[ACF_MAX_RELAXATION];   /* rho c_r^2 Delta / dx scheme.py:177 */
    const double *wall_shell[6];             /* 2 * n_b * n_c doubles each, or NULL */
    const double *cell[3];                   /* n_a doubles each, or NULL */
    const double *face[3];                   /* n_a + 1 doubles each, or NULL */
} acf_config;

/* Library identity. */
int acf_abi_version(void);
size_t acf_struct_size(void);          /* sizeof(acf_config), for FFI mirror checks */
const char *acf_last_error(void);      /* message of the last failure on this thread */
int acf_device_count(int *count);
/* Make `device` the calling thread's current device in this library's CUDA runtime, so the
 * next acf_create / acf_batch_create place their handle there (a handle keeps its device;
 * every call on it switches to that device and back). Needed by callers with several GPUs in
 * one process: the library links its own runtime, whose current device another runtime's
 * selection need not change. No counterpart in the reference (one CPU pool per process). */
int acf_set_device(int32_t device);

/* Handle lifetime. acf_create allocates zeroed device state on the current device. With the
 * environment variable ACF_INJECT_ALLOC_FAILURE set (non-empty, not "0"), acf_create and
 * acf_batch_create fail with ACF_ERR_MEMORY before allocating, as on an exhausted device: a
 * test hook for callers' error paths. */
int acf_create(const acf_config *config, acf_solver **out);
int acf_destroy(acf_solver *solver);
int acf_is_double(const acf_solver *solver);

/* Sources (src/ac_fdtd/scheme.py:231-244, 360-363). `cell` holds reference flat indices
 * (i*ny + j)*nz + k; `signal` is n rows of `stride` doubles, row s valid for `length[s]`
 * samples. Sample n is added after the damping of step n, in the order given. Replaces the
 * previous set. */
int acf_set_sources(acf_solver *solver, int64_t n, const int64_t *cell, const int64_t *length,
                    const double *signal, int64_t stride);

/* Receivers (src/ac_fdtd/scheme.py:246-262, 294-296): receiver r records p[cell[r]] after
 * every step whose absolute index is >= start_step[r]. Replaces the previous set; recordings of
 * receivers that keep their position in the list are kept. */
int acf_set_receivers(acf_solver *solver, int64_t n, const int64_t *cell,
                      const int64_t *start_step);

/* Copy `n` samples of receiver r, starting at absolute step `first_step`, to `dst` (host or
 * device memory, solver precision). Synchronous. */
int acf_read_recording(acf_solver *solver, int64_t receiver, int64_t first_step, int64_t n,
                       void *dst, acf_stream stream);

/* Move one field between the reference layout (dense C order, solver precision) and the
 * device. `src`/`dst` may be host (pageable or pinned) or device memory. Asynchronous on
 * `stream` for pinned and device memory. */
int acf_upload(acf_solver *solver, int field, const void *src, acf_stream stream);
int acf_download(acf_solver *solver, int field, void *dst, acf_stream stream);

/* Advance n_steps. step_offset is the absolute index of the first step, which selects the
 * source samples (src/ac_fdtd/c/acfdtd.c:358-371). Asynchronous on `stream`. */
int acf_run(acf_solver *solver, int64_t n_steps, int64_t step_offset, acf_stream stream);

/* The two FP64 sums of the pressure-only scheme's conserved energy after its latest step, with
 * u = p^{n+1} and w = p^n: terms[0] = sum (u - w)^2, terms[1] = sum u L w. The energy
 * E = dx^3 / (2 rho c^2) (terms[0] / lam2 - terms[1]) is constant for rigid walls and does not
 * grow with impedance walls (it drops by dx^3/(2 rho c^2) sum a (p^{n+1} - p^{n-1})^2 / lam2 per
 * step); it is the scheme's own quadratic form, not the p-v energy of acf_energy_terms.
 * ACF_ERR_STATE before the scheme's first step. No counterpart in the reference. */
int acf_pressure_only_energy_terms(acf_solver *solver, double terms[2], acf_stream stream);

/* How a single room advances: two sweeps per step over one copy of the state, or one fused
 * sweep that reads the current p and v and writes the next ones to a second copy (4 more
 * fields of memory, (8 + 2R) instead of (12 + 2R) elements moved per cell). Both give
 * bit-identical results. The adjoint's recorded runs use the two sweeps.
 * ACF_SCHEME_FUSED_STAGED is the fused sweep with each CTA's share of every x plane streamed
 * into a shared-memory ring by bulk copies (see acf_set_staging); same memory, same results.
 * No counterpart in the reference (its C loop runs the two sweeps, acfdtd.c:355-376). */
enum { ACF_SCHEME_TWO_SWEEPS = 0, ACF_SCHEME_FUSED = 1, ACF_SCHEME_FUSED_STAGED = 2,
       ACF_SCHEME_PRESSURE_ONLY = 3 };

/* ACF_SCHEME_PRESSURE_ONLY: the second-order wave equation on p alone, for a single room with
 * rigid or impedance walls and no absorbing layer or air absorption (ACF_ERR_STATE otherwise).
 * The reference plans it (its milestone M8, PLAN.md:52-56) and has not built it. With the
 * velocities eliminated, p^{n+1} = fu (2 p^n + lam2 L p^n) - (fu - fp) p^{n-1} - S^{n-1} + S^n
 * (L the rigid-face Laplacian, lam2 = c_p c_v, (fu, fp) the wall pair, S^n the source added
 * after step n): 3 elements moved per cell and step instead of 8 + 2R. The first step after
 * selecting it is the p-v step from the state as it stands (p^n, v^{n-1/2}), so the pressures
 * and recordings equal the p-v scheme's to rounding. From then on the velocities are not kept:
 * acf_download/acf_upload of vx, vy, vz and acf_energy_terms return ACF_ERR_STATE (use
 * acf_pressure_only_energy_terms), as does switching to another scheme before
 * acf_reset_state. Uploading p replaces p^n and keeps p^{n-1}. */
int acf_set_scheme(acf_solver *solver, int32_t scheme);
int acf_get_scheme(const acf_solver *solver);

/* L2 prefetch in the marching kernels: each thread asks L2 for its next x plane's inputs
 * while it computes the current one, so more DRAM reads are in flight than its registers
 * hold. mode -1 (default) enables it when the fields one step streams exceed the device's L2,
 * 0 disables it, 1 enables it. Results never depend on it. acf_get_prefetch returns whether it
 * is in effect (1 or 0; -1 for a null solver). No counterpart in the reference. */
int acf_set_prefetch(acf_solver *solver, int32_t mode);
int acf_get_prefetch(const acf_solver *solver);

/* Steps per launch of the fused scheme in single precision: 1 (the default) or 2, temporal
 * blocking -- one sweep takes each x plane through two steps, reading the state once and writing
 * it once per two steps. Runs then go in units of four steps (two launches, after which the
 * state sits where four single steps leave it) and single steps for the rest; results equal
 * single steps bit for bit. 2 needs one single-precision room with nz a multiple of 4 whose CTAs
 * of one x-plane group fit on the device at once (ACF_ERR_ARGUMENT otherwise), allocates four
 * planes of pressure per group, a counter per CTA and a second copy of the relaxation states,
 * and takes effect while the scheme is ACF_SCHEME_FUSED. acf_get_time_blocking returns the
 * setting (-1 for a null solver). The step after the fused sweep that the reference's C backend
 * names as its next one (c/acfdtd.c:12-14); no counterpart in its API. */
int acf_set_time_blocking(acf_solver *solver, int32_t steps_per_launch);
int acf_get_time_blocking(const acf_solver *solver);

/* Geometry of the staged scheme: y rows per CTA (1..16, each a whole padded z row), ring
 * buffers per CTA (2..8; 0 picks three, or two where three do not fit) and z elements per
 * thread (2 or 4). The x planes per CTA come from acf_set_launch. ACF_ERR_ARGUMENT when the
 * CTA would need more than 256 threads or more shared memory than an SM offers; results never
 * depend on it. Default: 2 rows where 2 rows of 4-element threads fit in 256 threads (else 1),
 * automatic stages, 4 elements. No counterpart in the reference. */
int acf_set_staging(acf_solver *solver, int32_t rows, int32_t stages, int32_t vector);

/* The solver's device status word, then cleared: 0 when nothing was reported; bit 1 when a
 * staged sweep gave up waiting for its copies, or a two-step sweep for its neighbour CTAs'
 * counters; bit 2 when a sweep produced a non-finite
 * pressure (NaN or infinity: every sweep that writes p checks what it writes). Either way the
 * state is not valid. Synchronizes the solver's device. acf_run and acf_batch_run also read
 * the word copied after the previous run, without waiting for the device, and return
 * ACF_ERR_NUMERIC (bit 2) or ACF_ERR_STATE (bit 1) before launching anything. The reference
 * has no such check (its NumPy and C loops run on whatever the state holds). */
int acf_device_status(acf_solver *solver, int32_t *status);
int acf_batch_device_status(acf_batch *batch, int32_t *status);

/* Test hook of the staged and two-step sweeps, for exercising their bounded waits without a
 * fault: every wait gives up after `wait_limit_ns` (0: the built-in two seconds; else 1 ms to
 * two seconds), and with `skip_plane` >= 0 (-1: none) the grid's first CTA withholds something
 * its waiters need. In the staged sweep its producer leaves out the copies of x plane
 * `skip_plane`, so that CTA's consumers wait for data that never arrives, run out of time, raise
 * bit 1 of the status word and return; the producer drains the copies it did issue before the
 * CTA exits. In the two-step sweep it stops publishing its progress from that plane on, so its
 * neighbour CTAs' waits run out, raise bit 1 and stop waiting. No counterpart in the reference. */
int acf_set_wait_test(acf_solver *solver, int64_t wait_limit_ns, int32_t skip_plane);

/* Use CUDA graphs of `steps_per_graph` steps for runs at least that long (0 disables). */
int acf_set_graph(acf_solver *solver, int32_t steps_per_graph);

/* Launch geometry of both sweeps: threads per block (power of two, 32..256) and consecutive
 * x planes each block marches through (1..1024). Results do not depend on it. */
int acf_set_launch(acf_solver *solver, int32_t block_threads, int32_t planes);

/* The seven FP64 sums the reference energy is built from, for the stored (p^n, v^{n-1/2})
 * pair (src/ac_fdtd/scheme.py:365-389): terms[0] = sum p^2; terms[1+a] = sum v_a^2 over all
 * faces; terms[4+a] = sum over interior faces of v_a * (p_hi - p_lo) / dx. Synchronous. */
int acf_energy_terms(acf_solver *solver, double dx, double terms[7], acf_stream stream);
/* The same sums over the x planes [x_begin, x_end) only: their cells (with their y and z
 * faces) and the x faces x_begin .. x_end - 1, plus the far face nx when x_end = nx and
 * far_face is set. The parts of a room cut into x slabs sum to the whole room's terms. */
int acf_energy_terms_planes(acf_solver *solver, double dx, int64_t x_begin, int64_t x_end,
                            int32_t far_face, double terms[7], acf_stream stream);

/* ---- Adjoint (single rooms) ----------------------------------------------------------
 *
 * Gradients of a loss of the receiver signals, by the transposed leapfrog run backward in
 * time. No counterpart in the reference (its solvers are not differentiable). The step is
 * linear in the state, so the backward recursion needs no forward state; parameter gradients
 * read a forward history: the pressure before the step and before the wall closed form on
 * every boundary cell (walls), and D and psi of every cell (air), recomputed segment by segment
 * from full-state checkpoints taken every `checkpoint_every` steps. checkpoint_every = 0 picks
 * it: the whole run when D and psi of every step take at most 60 % of the free device memory
 * -- the recorded run then keeps them and nothing is recomputed -- else ceil(sqrt(max_steps)).
 *
 * acf_adjoint_prepare  allocates the history for runs of up to max_steps steps.
 * acf_forward_record   is acf_run that also writes that history (and the checkpoints). In
 *                      single precision with nz a multiple of 4 and no air gradients it takes one
 *                      lean sweep per step into the second copy of p and v -- allocated on the
 *                      first such call when the scheme has none -- and leaves the state in the
 *                      primary copy; results equal the two-sweep record bit for bit.
 * acf_adjoint_run      takes dL/drec (n_receivers rows of n_steps doubles, host) and returns
 *                      (each optional, host, FP64): dL/dsignal (n_sources rows of n_steps),
 *                      dL/da per boundary cell (acf_adjoint_shell_size entries, shell order of
 *                      the wall coefficients with each cell on the first face it touches), and
 *                      the air sums (dL/dgain_r, dL/dmean_r, dL/ddecay_r for r < n_relax, then
 *                      dL/drelax_scale).
 * acf_adjoint_download returns dL/d of the initial state, field by field.
 * acf_set_coefficients swaps in new coefficients (same grid, precision, relaxation count and
 *                      the same presence of layer and walls) without touching the state. */
enum { ACF_GRAD_WALLS = 1, ACF_GRAD_AIR = 2 };
/* Set every field of the state to zero on the device (a room at rest). Asynchronous. */
int acf_reset_state(acf_solver *solver, acf_stream stream);
int acf_set_coefficients(acf_solver *solver, const acf_config *config);
int acf_adjoint_prepare(acf_solver *solver, int32_t flags, int64_t max_steps,
                        int32_t checkpoint_every);
int64_t acf_adjoint_shell_size(const acf_solver *solver);
/* The checkpoint interval in use (after an automatic choice); -1 for a null solver. */
int32_t acf_adjoint_checkpoint_interval(const acf_solver *solver);
int acf_forward_record(acf_solver *solver, int64_t n_steps, int64_t step_offset,
                       acf_stream stream);
int acf_adjoint_run(acf_solver *solver, const double *grad_rec, double *grad_src,
                    double *grad_shell, double *grad_air, acf_stream stream);
int acf_adjoint_download(acf_solver *solver, int field, void *dst, acf_stream stream);

/* Energy sums without any allocation. No counterpart in the reference.
 *
 * For callers that must not allocate device memory themselves or have the library allocate
 * it: an application that hands this code a fixed device-memory budget from its own pool (an
 * audio plug-in host, a game or simulation engine), or a real-time thread on which
 * cudaMalloc/cudaFree may block or synchronize the device. It computes the same seven sums as
 * acf_energy_terms, but from fields the caller already holds in device memory in the
 * reference's dense C-order layout -- p (nx,ny,nz), vx (nx+1,ny,nz), vy (nx,ny+1,nz),
 * vz (nx,ny,nz+1), `precision` 4 or 8 bytes -- and writes them to `terms_device`, 7 doubles
 * in device memory. It needs no handle and calls no allocator.
 *
 * Its working memory is one static device array of ACF_NOALLOC_MAX_PLANES * 7 doubles
 * (224 KiB), which every GPU that loads this library holds until the process exits. Grids
 * with nx + 1 > ACF_NOALLOC_MAX_PLANES are refused with ACF_ERR_ARGUMENT. The first call on
 * each device looks up that array's device address (with the device current); make that
 * first call before any stream capture. All calls share the one array: calls that overlap on
 * the GPU (two streams, or two host threads) race and must be serialized by the caller. Each
 * call writes every scratch entry it later reads, so nothing is left to clear between calls.
 * Asynchronous on `stream`. */
#define ACF_NOALLOC_MAX_PLANES 4096
int acf_energy_terms_noalloc(const void *p, const void *vx, const void *vy, const void *vz,
                             int32_t nx, int32_t ny, int32_t nz, int32_t precision, double dx,
                             double *terms_device, acf_stream stream);

/* Device address and element strides (z, y, x order reversed: strides[0] is the x stride)
 * of one field in the internal padded layout. */
int acf_field_pointer(acf_solver *solver, int field, void **ptr, int64_t strides[3]);

/* Copy x plane `src_plane` of one field of `src` into x plane `dst_plane` of the same field of
 * `dst` (every field has nx + 1 planes of (ny + 1) padded rows), device to device -- a peer
 * copy when the two solvers live on different GPUs. The rooms must share precision, ny and nz.
 * Asynchronous on `stream`; order it after both solvers' work (the same stream, or a
 * synchronization). The ghost-plane exchange of a room split into x slabs. No counterpart in
 * the reference (its solver is one shared-memory process). */
int acf_copy_plane(acf_solver *dst, int64_t dst_plane, const acf_solver *src, int64_t src_plane,
                   int field, acf_stream stream);

/* The GPU a solver's state lives on (-1 for a null solver). No counterpart in the reference. */
int acf_solver_device(const acf_solver *solver);

/* Advance a room cut into x slabs: parts[q] holds slab q (left to right) with its ghost planes,
 * its own planes being [own_lo[q], own_hi[q]) -- own_lo = 1 where a left neighbour exists else
 * 0, own_hi = nx - 1 where a right neighbour exists else nx. Each step runs every part's
 * velocity sweep, then every part's pressure sweep, which updates its own planes and also stores
 * its first and last own planes of p into the neighbours' ghost planes (peer stores across
 * GPUs; peer access is enabled as needed). The ghost planes must hold the neighbours' p before
 * the first step (acf_copy_plane). With the fused scheme (every part on it, copies in step)
 * each part's step writes its own planes of the next copy and stores its first and last own
 * planes into the neighbours' ghost planes of their next copies: one launch per part across
 * GPUs; on one GPU, in single precision with nz a multiple of 4, one launch per step for up to 8
 * parts, and the steps replay from a CUDA graph. Single rooms of equal scheme, precision, ny and nz. Parts
 * on one GPU run on `stream`; parts on several GPUs on each device's default stream,
 * ordered by events, and `stream` must then be null (ACF_ERR_ARGUMENT otherwise: a stream
 * belongs to one device). Asynchronous. No counterpart in the reference. */
int acf_run_slabs(acf_solver *const *parts, int32_t n_parts, const int32_t *own_lo,
                  const int32_t *own_hi, int64_t n_steps, int64_t step_offset, acf_stream stream);

/* Instrumentation: when enabled, acf_run launches step by step with CUDA events around each
 * sweep and accumulates their device time. */
int acf_profile_enable(acf_solver *solver, int32_t enable);
int acf_profile_read(acf_solver *solver, double *velocity_ms, double *pressure_ms,
                     int64_t *launches);

/* Kernels launched by this handle since creation (sweeps, graph replays counted per kernel). */
int64_t acf_launch_count(const acf_solver *solver);

/* ---- Impulse-response post-processing (FP64, on the device) ----------------------------
 *
 * The steps after the time loop of the reference's room workflow (src/ac_fdtd/room.py:121-176),
 * on receiver signals in device memory: `channels` signals of `n` samples, back to back. Every
 * array argument is a device pointer; each call is asynchronous on `stream` and allocates
 * nothing. Sums are FP64 in another order than NumPy's sequential ones, so results agree with
 * the reference to rounding (about 1e-14 relative), not bit for bit. */

/* Schroeder decay curve in dB, 10 log10 max(I(k)/I(0), 1e-300) floored at `floor_db`, with
 * I(k) the backward integral of the squared signal (src/ac_fdtd/metrics.py:57-69). */
int acf_schroeder_decay(const double *response, int64_t channels, int64_t n, double floor_db,
                        double *decay, acf_stream stream);

/* Seconds per 60 dB of a least-squares line through each decay curve, between the first
 * sample at or below `upper_db` and the first at or below `lower_db` (metrics.py:72-101: T20
 * is (-5, -25), EDT (0, -10)). `seconds` and `failed` hold one value per channel; failed[c] = 1
 * (seconds NaN) where the curve does not reach `lower_db` after `upper_db`, where the reference
 * raises ValueError. */
int acf_decay_fit(const double *decay, int64_t channels, int64_t n, double sample_rate, double upper_db,
                  double lower_db, double *seconds, int32_t *failed, acf_stream stream);

/* Early-to-late energy ratio in dB per channel, split before sample `boundary` (C50 with
 * boundary = round(0.05 fs); metrics.py:104-110). */
int acf_clarity(const double *response, int64_t channels, int64_t n, int64_t boundary, double *db,
                acf_stream stream);

/* The division step of the reference's deconvolution (src/ac_fdtd/sources.py:103-107) on
 * spectra from a real-to-complex FFT (interleaved complex doubles): out = X conj(S) /
 * (|S|^2 + regularisation max|S|^2), zero in bins k with k * bin_hz > max_frequency, for each
 * of `channels` spectra X of `bins` bins and the excitation's spectrum S. `scratch` is one
 * device double. The FFTs themselves are the caller's (a library FFT). */
int acf_spectral_divide(const void *spectra, const void *source, int64_t channels, int64_t bins,
                        double bin_hz, double max_frequency, double regularisation, double *scratch,
                        void *out, acf_stream stream);

/* ---- Batches of rooms/* ---- Batches of rooms -------------------------------------------------------------------
 *
 * Many rooms of different sizes advanced together: each sweep is one persistent launch over a
 * flat tile table covering every room, and runs replay CUDA graphs of both sweeps. No
 * counterpart in the reference, whose solvers hold one room each (src/ac_fdtd/scheme.py:82);
 * per room the arithmetic is exactly that of acf_create/acf_run, so each room's results equal
 * a single-room run bit for bit. All rooms share the precision and the number of relaxation
 * processes, and advance from the same step index. Room-level calls mirror the single-room
 * ones with a room index. */
int acf_batch_create(int32_t n_rooms, const acf_config *configs, acf_batch **out);
int acf_batch_destroy(acf_batch *batch);
int acf_batch_room_count(const acf_batch *batch);
int acf_batch_set_sources(acf_batch *batch, int32_t room, int64_t n, const int64_t *cell,
                          const int64_t *length, const double *signal, int64_t stride);
int acf_batch_set_receivers(acf_batch *batch, int32_t room, int64_t n, const int64_t *cell,
                            const int64_t *start_step);
int acf_batch_read_recording(acf_batch *batch, int32_t room, int64_t receiver,
                             int64_t first_step, int64_t n, void *dst, acf_stream stream);
int acf_batch_upload(acf_batch *batch, int32_t room, int field, const void *src,
                     acf_stream stream);
int acf_batch_download(acf_batch *batch, int32_t room, int field, void *dst, acf_stream stream);
int acf_batch_run(acf_batch *batch, int64_t n_steps, int64_t step_offset, acf_stream stream);
int acf_batch_set_graph(acf_batch *batch, int32_t steps_per_graph);
/* Threads per tile (power of two, 32..256), x planes per tile, and CTAs per SM of a persistent
 * grid striding over the tile table (0: one CTA per tile, scheduled by the hardware). */
int acf_batch_set_launch(acf_batch *batch, int32_t block_threads, int32_t planes,
                         int32_t ctas_per_sm);
/* ACF_SCHEME_TWO_SWEEPS or ACF_SCHEME_FUSED (one sweep per step over the tile table, into a
 * second copy of every room's p and v); bit-identical results. No counterpart in the
 * reference. */
int acf_batch_set_scheme(acf_batch *batch, int32_t scheme);
/* acf_set_prefetch for a batch; the default compares every room's fields together with L2. */
int acf_batch_set_prefetch(acf_batch *batch, int32_t mode);
int acf_batch_energy_terms(acf_batch *batch, int32_t room, double dx, double terms[7],
                           acf_stream stream);
int acf_batch_profile_enable(acf_batch *batch, int32_t enable);
int acf_batch_profile_read(acf_batch *batch, double *velocity_ms, double *pressure_ms,
                           int64_t *launches);
int64_t acf_batch_launch_count(const acf_batch *batch);

/* Adjoint of a batch (wall and source gradients; no counterpart in the reference): as the
 * single-room acf_adjoint_* calls, for every room at once. grad_rec concatenates each room's
 * (n_receivers x n_steps) block in room order; grad_src likewise (n_sources x n_steps); grad_shell
 * concatenates each room's acf_batch_adjoint_shell_size(room) entries. */
int acf_batch_adjoint_prepare(acf_batch *batch, int64_t max_steps);
int64_t acf_batch_adjoint_shell_size(const acf_batch *batch, int32_t room);
int acf_batch_forward_record(acf_batch *batch, int64_t n_steps, int64_t step_offset,
                             acf_stream stream);
int acf_batch_adjoint_run(acf_batch *batch, const double *grad_rec, double *grad_src,
                          double *grad_shell, acf_stream stream);
int acf_batch_reset_state(acf_batch *batch, acf_stream stream);
int acf_batch_set_coefficients(acf_batch *batch, int32_t room, const acf_config *config);

/* Block until all work queued on `stream` is done. */
int acf_synchronize(acf_stream stream);

/* Pinned host memory for fast state transfers. */
int acf_host_alloc(size_t bytes, void **out);
int acf_host_free(void *ptr);

#ifdef __cplusplus
}
#endif

#endif /* ACFDTD_B200_H */
