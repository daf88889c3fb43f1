// acfdtd_b200.cu -- the staggered pressure-velocity leapfrog on sm_100a, behind a C ABI.
//
// One time step is two HBM-bound updates of the grid (ac-fdtd: src/ac_fdtd/scheme.py:285-296,
// src/ac_fdtd/c/acfdtd.c:110-190,342-376):
//
//   (a) velocity: v_a -= c_v (p_hi - p_lo) on interior faces, then the absorbing-layer damping
//       x, y, z in that order on every face (scheme.py:287-290,298-311).
//   (b) pressure: div v, the relaxation states, p -= c_p div, the time-centred wall closed
//       form, the layer damping, the volume sources and the receiver gather, all in the
//       registers of the thread that owns the cell (scheme.py:291-296,313-363).
//
// Arithmetic order follows the NumPy reference operation by operation and the library is
// built with -fmad=false, so no multiply-add is contracted: both precisions reproduce the
// reference's own float64/float32 arithmetic bit for bit.
//
// Layout in HBM: every field of a room uses the same padded geometry, (nx+1) planes of (ny+1)
// rows of pz elements, pz = nz+1 rounded up to a multiple of 8. Element (i,j,k) of any field is
// at (i*(ny+1) + j)*pz + k, so vx's extra plane, vy's extra row and vz's extra face all fit and
// a neighbour on any axis is a constant stride away. Rows start on 32-byte boundaries, which
// keeps every 4-element group of a thread a single aligned vector access.
//
// Three step schemes give the same bits:
//   * two_sweeps: (a) and (b) as two launches, fields updated in place;
//   * fused: one launch per step; each cell computes the updated velocities of its six faces
//     and then its pressure, writing the next p and v into a second copy of the fields
//     (ping-pong), so a cell costs one read and one write of each field;
//   * staged: the fused step with the planes of its inputs brought into a shared-memory ring
//     by the bulk-copy engine (one producer warp, mbarrier waits with a time limit).
//
// Two launch forms share the per-column code:
//   * one room: a 2D grid of (z chunk, y row) threads, each block marching `planes` x planes;
//   * a batch of rooms of different sizes packed in one arena: a persistent grid walks a flat
//     tile table (room, first (row, chunk) pair, plane range); each CTA stages its room's
//     description in shared memory. One launch per sweep covers every room.
//
// The adjoint (transposed) leapfrog for gradients reuses the same layout, launch forms and
// fusion, backward in time.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "acfdtd_b200.h"

namespace {

constexpr int kVec = 4;            // elements per thread along z
constexpr int kRowAlign = 8;       // row pitch granularity, elements
constexpr int kEnergyTerms = 7;

thread_local char g_last_error[512] = "";

int fail(int code, const char *fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, args);
    va_end(args);
    return code;
}

#define ACF_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t err__ = (call);                                                        \
        if (err__ != cudaSuccess)                                                          \
            return fail(ACF_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                      \
                        cudaGetErrorString(err__), __FILE__, __LINE__);                    \
    } while (0)

// ------------------------------------------------------------------------------------------
// Vector access: 4 consecutive elements, one 16-byte access for float, two for double.

template <typename T>
struct Vec4;

template <>
struct Vec4<float> {
    __device__ __forceinline__ static void load(const float *__restrict__ a, float v[4]) {
        const float4 t = *reinterpret_cast<const float4 *>(a);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    __device__ __forceinline__ static void store(float *__restrict__ a, const float v[4]) {
        *reinterpret_cast<float4 *>(a) = make_float4(v[0], v[1], v[2], v[3]);
    }
    // Read-only path: only for arrays no thread writes during the kernel.
    __device__ __forceinline__ static void ldg(const float *__restrict__ a, float v[4]) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(a));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    // Streaming (evict-first) load: data read once, such as the adjoint's history.
    __device__ __forceinline__ static void ldcs(const float *a, float v[4]) {
        const float4 t = __ldcs(reinterpret_cast<const float4 *>(a));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
};

template <>
struct Vec4<double> {
    __device__ __forceinline__ static void load(const double *__restrict__ a, double v[4]) {
        const double2 t0 = *reinterpret_cast<const double2 *>(a);
        const double2 t1 = *reinterpret_cast<const double2 *>(a + 2);
        v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
    }
    __device__ __forceinline__ static void store(double *__restrict__ a, const double v[4]) {
        *reinterpret_cast<double2 *>(a) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2 *>(a + 2) = make_double2(v[2], v[3]);
    }
    __device__ __forceinline__ static void ldg(const double *__restrict__ a, double v[4]) {
        const double2 t0 = __ldg(reinterpret_cast<const double2 *>(a));
        const double2 t1 = __ldg(reinterpret_cast<const double2 *>(a + 2));
        v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
    }
    __device__ __forceinline__ static void ldcs(const double *a, double v[4]) {
        const double2 t0 = __ldcs(reinterpret_cast<const double2 *>(a));
        const double2 t1 = __ldcs(reinterpret_cast<const double2 *>(a + 2));
        v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
    }
};

// Streaming (evict-first) stores of 4 elements, for data written once and read once much later
// -- the adjoint's D/psi history -- so that it does not push the state out of L2.
__device__ __forceinline__ void store_streaming(float *a, const float v[4]) {
    __stcs(reinterpret_cast<float4 *>(a), make_float4(v[0], v[1], v[2], v[3]));
}
__device__ __forceinline__ void store_streaming(double *a, const double v[4]) {
    __stcs(reinterpret_cast<double2 *>(a), make_double2(v[0], v[1]));
    __stcs(reinterpret_cast<double2 *>(a + 2), make_double2(v[2], v[3]));
}

// Ask L2 for the line holding `a` ahead of its load: the request holds no register and no
// shared memory, so a marching thread can have its next plane on the way from DRAM while it
// computes the current one. Only addresses the thread will load later are passed.
template <typename T>
__device__ __forceinline__ void prefetch_l2(const T *a) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

// Bits of a handle's device status word.
constexpr int32_t kStatusWaitTimeout = 1;   // a staged sweep gave up waiting for its copies
constexpr int32_t kStatusNonFinite = 2;     // a sweep produced a NaN or infinite pressure

__device__ __forceinline__ unsigned lane_id() {
    unsigned lane;
    asm("mov.u32 %0, %%laneid;" : "=r"(lane));
    return lane;
}

// Non-finite detector: acc = fma(x, 0, acc) is acc + 0 for every finite x (one rounding, exact)
// and NaN once any x was NaN or infinite; NaN then stays. One fused instruction per value.
template <typename T>
__device__ __forceinline__ T finite_acc(T acc, T x) {
    if constexpr (sizeof(T) == 4) return __fmaf_rn(x, 0.0f, acc);
    else return __fma_rn(x, 0.0, acc);
}

// Raise kStatusNonFinite once per warp whose threads saw a non-finite value.
__device__ __forceinline__ void report_nonfinite(int32_t *status, bool bad) {
    const unsigned mask = __ballot_sync(__activemask(), bad);
    if (bad && status != nullptr && lane_id() == (unsigned)(__ffs(mask) - 1))
        atomicOr(status, kStatusNonFinite);
}

// ------------------------------------------------------------------------------------------
// What the sweeps read about one room. Plain data, identical on host and device.

template <typename T>
struct Room {
    int32_t nx, ny, nz, nchunks;
    int32_t prefetch;              // 1: marching threads ask L2 for their next plane ahead
    int32_t reserved;
    // A slab of a room cut along x: the single-room pressure sweep updates the planes
    // [own_lo, own_hi) only, and also stores p of planes own_lo and own_hi - 1 into the
    // neighbours' ghost planes (null: no neighbour on that side; a peer address when the
    // neighbour lives on another GPU). A whole room: [0, nx), no ghosts.
    int32_t own_lo, own_hi;
    T *ghost_lo, *ghost_hi;
    int64_t pz, plane, field;      // row pitch, plane pitch, elements per field
    T *p, *vx, *vy, *vz, *psi;     // psi: n_relax fields back to back
    T cv, cp, cs, relax_scale;
    T decay[ACF_MAX_RELAXATION], mean[ACF_MAX_RELAXATION], gain[ACF_MAX_RELAXATION];
    const T *cell[3];              // layer profiles at cell centres
    const T *face[3];              // layer profiles at faces
    const T *shell[6];             // wall pairs (1/(1+a), a/(1+a)) per face cell
    int32_t n_src;
    int32_t n_rec;
    const int64_t *src_off;        // padded offsets
    const int64_t *src_len;
    const T *src_sig;
    int64_t src_stride;
    const int64_t *rec_off;        // padded offsets
    const int64_t *rec_start;      // first absolute step recorded
    const int64_t *src_col;        // in-plane offsets (padded offset mod plane): j * pz + k
    const int64_t *rec_col;
    T *rec;
    int64_t rec_stride, rec_origin;
    // Status word of the handle (device memory): the sweeps that write p set kStatusNonFinite
    // in it when a pressure they produced is NaN or infinite. Null: not checked.
    int32_t *status;
};

// Forward history kept for the adjoint: per step, p^n and p-tilde^n -- pressure before the step
// and before the wall closed form -- on every boundary cell (two blocks of shell_total values,
// first every p^n, then every p-tilde^n), and, for a
// segment of steps, the divergence D^n and the relaxation states psi^n before their update.
// Boundary cells are indexed as in the wall shells: the first face of FACES order a cell lies
// on, then row-major over that face's two other axes; face f starts at face_off[f].
template <typename T>
struct History {
    T *shell;                      // steps x 2 x shell_total values, or null
    int64_t shell_total, shell_step0, shell_steps;
    int64_t face_off[6];
    T *fields;                     // slots x (1 + n_relax) fields (padded geometry), or null;
                                   // step n uses slot (n - fields_step0) mod fields_slots
    int64_t fields_step0;
    int32_t fields_slots;
    int32_t reserved;
};

template <typename T>
struct StepParams {
    Room<T> room;
    History<T> hist;
    const int64_t *step_base;      // absolute step of local step 0, in device memory
    int32_t local_step;
    int32_t planes;                // consecutive x planes marched by one block
};

// One unit of work of a batched sweep: up to blockDim.x consecutive (row, chunk) pairs of one
// room, over the x planes [i_begin, i_end).
struct Tile {
    int32_t room, first, count, i_begin, i_end, reserved;
};

template <typename T>
struct BatchParams {
    const Room<T> *rooms;
    const Tile *tiles;
    int32_t n_tiles;
    int32_t local_step;
    const int64_t *step_base;
};

// ------------------------------------------------------------------------------------------
// (a) velocity, one (row j, chunk c) column over the x planes [i_begin, i_end). Each cell owns
// the lower face of each axis; the far boundary faces (x = nx, y = ny, z = nz) are only ever
// damped. Every global load of a plane is issued before its first store, so a thread has all
// of its fields in flight at once (a store may alias a later load, which would otherwise
// serialise them); p of the previous plane stays in registers.

template <typename T, bool LAYER>
__device__ __forceinline__ void velocity_column(const Room<T> &s, int i_begin, int i_end, int j,
                                                int c) {
    const int k0 = c * kVec;
    const T cv = s.cv;
    const int64_t column = (int64_t)j * s.pz + k0;
    T Pm[kVec];  // p at plane i - 1
    if (i_begin > 0) Vec4<T>::ldg(s.p + (int64_t)(i_begin - 1) * s.plane + column, Pm);

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        if (s.prefetch && i + 1 < i_end) {  // the next plane's own-row inputs into L2
            const int64_t next = base + s.plane;
            prefetch_l2(s.p + next);
            prefetch_l2(s.vx + next);
            prefetch_l2(s.vy + next);
            prefetch_l2(s.vz + next);
        }
        // ---- loads
        T P[kVec], Py[kVec], VX[kVec], VY[kVec], VZ[kVec];
        Vec4<T>::ldg(s.p + base, P);
        if (j > 0) Vec4<T>::ldg(s.p + base - s.pz, Py);
        const T below = (k0 > 0) ? __ldg(s.p + base - 1) : T(0);
        Vec4<T>::load(s.vx + base, VX);
        Vec4<T>::load(s.vy + base, VY);
        Vec4<T>::load(s.vz + base, VZ);

        // ---- compute, in the reference's order: gradient update, then x, y, z damping
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            if (k < s.nz) {
                T vx = VX[e], vy = VY[e], vz = VZ[e];
                if (i > 0) vx = vx - cv * (P[e] - Pm[e]);
                if (j > 0) vy = vy - cv * (P[e] - Py[e]);
                if (k > 0) vz = vz - cv * (P[e] - (e == 0 ? below : P[e - 1]));
                if (LAYER) {
                    const T fi_cell = __ldg(s.cell[0] + i), fi_face = __ldg(s.face[0] + i);
                    const T fj_cell = __ldg(s.cell[1] + j), fj_face = __ldg(s.face[1] + j);
                    const T fk_cell = __ldg(s.cell[2] + k), fk_face = __ldg(s.face[2] + k);
                    vx = vx * fi_face;
                    vx = vx * fj_cell;
                    vx = vx * fk_cell;
                    vy = vy * fi_cell;
                    vy = vy * fj_face;
                    vy = vy * fk_cell;
                    vz = vz * fi_cell;
                    vz = vz * fj_cell;
                    vz = vz * fk_face;
                }
                VX[e] = vx;
                VY[e] = vy;
                VZ[e] = vz;
            }
        }

        // ---- stores
        Vec4<T>::store(s.vx + base, VX);
        Vec4<T>::store(s.vy + base, VY);
        Vec4<T>::store(s.vz + base, VZ);
#pragma unroll
        for (int e = 0; e < kVec; e++) Pm[e] = P[e];

        // Far boundary faces (x = nx, y = ny, z = nz): never updated, but the reference damps
        // them with its slabs. Only the threads on those faces do this, after their stores.
        if (LAYER) {
            const T fi_cell = __ldg(s.cell[0] + i);
            const T fj_cell = __ldg(s.cell[1] + j);
            if (i == s.nx - 1) {
                T V[kVec];
                Vec4<T>::load(s.vx + base + s.plane, V);
                const T f = __ldg(s.face[0] + s.nx);
#pragma unroll
                for (int e = 0; e < kVec; e++)
                    if (k0 + e < s.nz) {
                        T v = V[e] * f;
                        v = v * fj_cell;
                        V[e] = v * __ldg(s.cell[2] + k0 + e);
                    }
                Vec4<T>::store(s.vx + base + s.plane, V);
            }
            if (j == s.ny - 1) {
                T V[kVec];
                Vec4<T>::load(s.vy + base + s.pz, V);
                const T f = __ldg(s.face[1] + s.ny);
#pragma unroll
                for (int e = 0; e < kVec; e++)
                    if (k0 + e < s.nz) {
                        T v = V[e] * fi_cell;
                        v = v * f;
                        V[e] = v * __ldg(s.cell[2] + k0 + e);
                    }
                Vec4<T>::store(s.vy + base + s.pz, V);
            }
            if (s.nz - 1 >= k0 && s.nz - 1 < k0 + kVec) {
                T *top = s.vz + (base - k0) + s.nz;
                T v = *top * fi_cell;
                v = v * fj_cell;
                *top = v * __ldg(s.face[2] + s.nz);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// (b) pressure, one column. The velocities are read-only here; p and psi are read and written
// by their owning thread only. vx of the upper face is carried into the next plane's lower face.

// First face (FACES order) that cell (i, j, k) lies on, and its index within that face's
// row-major (b, c) array; -1 for interior cells.
template <typename T>
__device__ __forceinline__ int shell_face(const Room<T> &s, int i, int j, int k, int64_t &idx) {
    if (i == 0) { idx = (int64_t)j * s.nz + k; return 0; }
    if (i == s.nx - 1) { idx = (int64_t)j * s.nz + k; return 1; }
    if (j == 0) { idx = (int64_t)i * s.nz + k; return 2; }
    if (j == s.ny - 1) { idx = (int64_t)i * s.nz + k; return 3; }
    if (k == 0) { idx = (int64_t)i * s.ny + j; return 4; }
    if (k == s.nz - 1) { idx = (int64_t)i * s.ny + j; return 5; }
    return -1;
}

template <typename T>
__device__ __forceinline__ bool wall_pair(const Room<T> &s, int i, int j, int k, T &fu, T &fp) {
    int64_t idx;
    const int f = shell_face(s, i, j, k, idx);
    if (f < 0) return false;
    const T *entry = s.shell[f] + 2 * idx;
    fu = __ldg(entry);
    fp = __ldg(entry + 1);
    return fp != T(0) || fu != T(1);
}

// The wall closed form for the cells of one column chunk at plane i: on an x-face plane or a
// y-face row (both uniform across a warp) every cell is tested; elsewhere only the chunk's
// k = 0 and k = nz - 1 cells can lie on a face -- a z face, the first in FACES order for them --
// so the thread reads just those pairs instead of searching four cells. `apply(e, fu, fp)` is
// called for each cell e (< real) with an absorbing pair.
template <typename T, typename Apply>
__device__ __forceinline__ void column_walls(const Room<T> &s, int i, int j, int k0, int real,
                                             Apply apply) {
    if (i == 0 || i == s.nx - 1 || j == 0 || j == s.ny - 1) {
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            T fu, fp;
            if (e < real && wall_pair(s, i, j, k0 + e, fu, fp)) apply(e, fu, fp);
        }
        return;
    }
    const bool bottom = k0 == 0, top_chunk = k0 + kVec >= s.nz;
    if (!bottom && !top_chunk) return;
    const int64_t at = 2 * ((int64_t)i * s.ny + j);
    if (bottom) {
        const T fu = __ldg(s.shell[4] + at), fp = __ldg(s.shell[4] + at + 1);
        if (fp != T(0) || fu != T(1)) apply(0, fu, fp);
    }
    const int top = s.nz - 1 - k0;
    if (top_chunk && (top > 0 || k0 > 0)) {     // k = nz - 1 is not also k = 0
        const T fu = __ldg(s.shell[5] + at), fp = __ldg(s.shell[5] + at + 1);
        if (fp != T(0) || fu != T(1)) apply(top, fu, fp);
    }
}

// Sources (bit q) and receivers (bit n_src + r) that lie in one (row j, chunk at k0) column,
// found once per column so that the march visits them only at their own plane instead of
// scanning every point at every plane. Beyond 32 points `all` is set and every point is
// scanned, as before.
template <typename T>
__device__ __forceinline__ uint32_t column_points(const Room<T> &s, int j, int k0, bool &all,
                                                 int width = kVec) {
    const int total = s.n_src + s.n_rec;
    all = total > 32;
    uint32_t mask = 0;
    if (all) return 0;
    const int64_t first = (int64_t)j * s.pz + k0;
    for (int q = 0; q < total; q++) {
        const int64_t col = q < s.n_src ? s.src_col[q] : s.rec_col[q - s.n_src];
        if (col >= first && col < first + width) mask |= 1u << q;
    }
    return mask;
}

__device__ __forceinline__ uint32_t source_bits(uint32_t mask, int n_src) {
    return n_src >= 32 ? mask : mask & ((1u << n_src) - 1u);
}

__device__ __forceinline__ uint32_t receiver_bits(uint32_t mask, int n_src) {
    return n_src >= 32 ? 0u : mask >> n_src;
}

// Sources of the column's cell at `base`, after damping, in the order they were added
// (scheme.py:293,360-363).
template <typename T>
__device__ __forceinline__ void add_sources(const Room<T> &s, uint32_t mask, bool all, int64_t base,
                                            int k0, int64_t step, T Pn[kVec]) {
    uint32_t m = all ? 0u : source_bits(mask, s.n_src);
    for (int q = all ? 0 : -1; all ? q < s.n_src : m != 0; q++) {
        if (!all) {
            q = __ffs(m) - 1;
            m &= m - 1;
        }
        const int64_t d = s.src_off[q] - base;
        if (d >= 0 && d < kVec && k0 + d < s.nz && step < s.src_len[q]) {
#pragma unroll
            for (int e = 0; e < kVec; e++)
                if (e == d) Pn[e] = Pn[e] + s.cs * s.src_sig[q * s.src_stride + step];
        }
    }
}

// Receivers of the column read the finished pressure (scheme.py:294-296).
template <typename T>
__device__ __forceinline__ void record_receivers(const Room<T> &s, uint32_t mask, bool all,
                                                 int64_t base, int64_t step, const T Pn[kVec]) {
    uint32_t m = all ? 0u : receiver_bits(mask, s.n_src);
    for (int r = all ? 0 : -1; all ? r < s.n_rec : m != 0; r++) {
        if (!all) {
            r = __ffs(m) - 1;
            m &= m - 1;
        }
        const int64_t d = s.rec_off[r] - base;
        if (d >= 0 && d < kVec && step >= s.rec_start[r]) {
            T v = Pn[0];
#pragma unroll
            for (int e = 1; e < kVec; e++)
                if (e == d) v = Pn[e];
            s.rec[r * s.rec_stride + (step - s.rec_origin)] = v;
        }
    }
}

// Boundary history of one step for the wall gradients: p^n and p before the wall closed form,
// on every boundary cell, in two blocks of shell_total values per step (first p, then the other)
// indexed as the wall shells are -- each cell on the first face of FACES order it lies on, then
// row-major over that face's two other axes. A column on an x-face plane or a y-face row owns
// contiguous entries for its whole chunk; elsewhere only its k = 0 and k = nz - 1 cells are on a
// (z) face.
template <typename T>
__device__ __forceinline__ void record_shell(const Room<T> &s, const History<T> &hist, int i, int j,
                                             int k0, int64_t step, const T P[kVec], const T PT[kVec]) {
    const int64_t slot = step - hist.shell_step0;
    if (slot < 0 || slot >= hist.shell_steps) return;
    T *hp = hist.shell + slot * 2 * hist.shell_total;
    T *ht = hp + hist.shell_total;
    if (i == 0 || i == s.nx - 1 || j == 0 || j == s.ny - 1) {
        const bool x_face = i == 0 || i == s.nx - 1;
        const int f = x_face ? (i == 0 ? 0 : 1) : (j == 0 ? 2 : 3);
        const int64_t at = hist.face_off[f] + (x_face ? (int64_t)j : (int64_t)i) * s.nz + k0;
#pragma unroll
        for (int e = 0; e < kVec; e++)
            if (k0 + e < s.nz) {
                hp[at + e] = P[e];
                ht[at + e] = PT[e];
            }
        return;
    }
    const int64_t at = (int64_t)i * s.ny + j;
    if (k0 == 0) {
        hp[hist.face_off[4] + at] = P[0];
        ht[hist.face_off[4] + at] = PT[0];
    }
    const int top = s.nz - 1 - k0;   // element of k = nz - 1, unless that cell is also k = 0
    if (s.nz > 1 && top >= 0 && top < kVec) {
#pragma unroll
        for (int e = 0; e < kVec; e++)
            if (e == top) {
                hp[hist.face_off[5] + at] = P[e];
                ht[hist.face_off[5] + at] = PT[e];
            }
    }
}

template <typename T, bool LAYER, bool WALLS, int NR, bool REC = false>
__device__ __forceinline__ void pressure_column(const Room<T> &s, int i_begin, int i_end, int j,
                                                int c, int64_t step,
                                                const History<T> *hist = nullptr) {
    const int k0 = c * kVec;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    const bool has_above = k0 + kVec <= s.nz;
    bool all_points = false;
    const uint32_t points = any_point ? column_points(s, j, k0, all_points) : 0u;
    const bool any_mine = points != 0 || all_points;
    // The column touches a wall where its row or its chunk is on the boundary; planes 0 and
    // nx - 1 are boundary planes for every column.
    const bool wall_column = j == 0 || j == s.ny - 1 || k0 == 0 || k0 + kVec >= s.nz;

    T fk[kVec];
    T fj = T(1);
    if (LAYER) {
#pragma unroll
        for (int e = 0; e < kVec; e++) fk[e] = __ldg(s.cell[2] + min(k0 + e, s.nz - 1));
        fj = __ldg(s.cell[1] + j);
    }
    const T cp = s.cp;
    const int64_t column = (int64_t)j * s.pz + k0;
    T XL[kVec];  // vx on the lower x face of the current plane
    Vec4<T>::ldg(s.vx + (int64_t)i_begin * s.plane + column, XL);
    T bad = T(0);   // NaN once a pressure this column produced is not finite

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        if (s.prefetch && i + 1 < i_end) {  // the next plane's own-row inputs into L2
            const int64_t next = base + s.plane;
            prefetch_l2(s.vx + next + s.plane);
            prefetch_l2(s.vy + next);
            prefetch_l2(s.vz + next);
            prefetch_l2(s.p + next);
#pragma unroll
            for (int r = 0; r < NR; r++) prefetch_l2(s.psi + r * s.field + next);
        }
        // ---- loads
        T XH[kVec], YL[kVec], YH[kVec], Z[kVec], P[kVec], S[NR > 0 ? NR : 1][kVec];
        Vec4<T>::ldg(s.vx + base + s.plane, XH);
        Vec4<T>::ldg(s.vy + base, YL);
        Vec4<T>::ldg(s.vy + base + s.pz, YH);
        Vec4<T>::ldg(s.vz + base, Z);
        const T above = has_above ? __ldg(s.vz + base + kVec) : T(0);
        Vec4<T>::load(s.p + base, P);
#pragma unroll
        for (int r = 0; r < NR; r++) Vec4<T>::load(s.psi + r * s.field + base, S[r]);
        const T fi = LAYER ? __ldg(s.cell[0] + i) : T(1);

        // ---- divergence x, then y, then z (scheme.py:317-322)
        T D[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            D[e] = XH[e] - XL[e];
            D[e] = D[e] + (YH[e] - YL[e]);
            D[e] = D[e] + ((e + 1 < kVec ? Z[e + 1] : above) - Z[e]);
        }

        if (REC && hist->fields) {
            const int64_t rel = step - hist->fields_step0;
            const int64_t slot = rel % hist->fields_slots;
            if (rel >= 0) {
                T *h = hist->fields + slot * (1 + NR) * s.field + base;
                store_streaming(h, D);
#pragma unroll
                for (int r = 0; r < NR; r++) store_streaming(h + (1 + r) * s.field, S[r]);
            }
        }

        const bool boundary = wall_column || i == 0 || i == s.nx - 1;
        T Pn[kVec], PT[kVec];   // PT: p before the wall closed form (recorded runs)
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            T pe = P[e];
            PT[e] = T(0);
            if (k < s.nz) {
                // relaxation states (scheme.py:337-358), then p -= c_p div (scheme.py:325-326)
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T target = D[e] * s.gain[r];
                    const T offset = S[r][e] - target;
                    S[r][e] = offset * s.decay[r] + target;
                    pe = pe + offset * s.mean[r];
                }
                if (NR > 0) pe = pe + D[e] * s.relax_scale;
                pe = pe - D[e] * cp;
                if (REC) PT[e] = pe;
                if (WALLS && boundary) {
                    T fu, fp;
                    if (wall_pair(s, i, j, k, fu, fp)) pe = pe * fu - P[e] * fp;
                }
                if (LAYER) {
                    pe = pe * fi;
                    pe = pe * fj;
                    pe = pe * fk[e];
                }
            }
            Pn[e] = pe;
        }

        if (REC && hist->shell && boundary) record_shell(s, *hist, i, j, k0, step, P, PT);
        if (any_mine) add_sources(s, points, all_points, base, k0, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) bad = finite_acc(bad, Pn[e]);

        // ---- stores
        Vec4<T>::store(s.p + base, Pn);
        // A slab's boundary planes also go to the neighbours' ghost planes (same in-plane offset).
        if (s.ghost_lo != nullptr && i == s.own_lo) Vec4<T>::store(s.ghost_lo + column, Pn);
        if (s.ghost_hi != nullptr && i == s.own_hi - 1) Vec4<T>::store(s.ghost_hi + column, Pn);
#pragma unroll
        for (int r = 0; r < NR; r++) Vec4<T>::store(s.psi + r * s.field + base, S[r]);
        if (any_mine) record_receivers(s, points, all_points, base, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) XL[e] = XH[e];
    }
    report_nonfinite(s.status, bad != bad);
}

// ------------------------------------------------------------------------------------------
// (a)+(b) in one sweep. The step reads the current p and v and writes the next ones to a second
// buffer, so a cell can compute the updated velocities of all six of its faces -- its own lower
// faces, which it stores, and its upper faces, which their owners compute identically -- and
// then its pressure. Per cell and step this moves (8 + 2R) elements instead of (12 + 2R); every
// value is produced by the same operations as in the two sweeps, so the results are identical.

template <typename T>
struct FusedParams {
    Room<T> room;                  // p, vx, vy, vz: current state (read); psi updated in place
    T *np, *nvx, *nvy, *nvz;       // next state (written), same geometry
    const int64_t *step_base;
    int32_t local_step;
    int32_t planes;
};

template <typename T, bool LAYER>
__device__ __forceinline__ T damp3(T v, T fa, T fb, T fc) {
    if (LAYER) {
        v = v * fa;
        v = v * fb;
        v = v * fc;
    }
    return v;
}

template <typename T, bool LAYER, bool WALLS, int NR>
__device__ __forceinline__ void fused_column(const FusedParams<T> &f, int i_begin, int i_end, int j,
                                             int c, int64_t step) {
    const Room<T> &s = f.room;
    const int k0 = c * kVec;
    const T cv = s.cv, cp = s.cp;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool has_above = k0 + kVec < s.nz;   // p and vz at k0 + 4 are interior
    bool all_points = false;
    const uint32_t points = any_point ? column_points(s, j, k0, all_points) : 0u;
    const bool any_mine = points != 0 || all_points;
    const bool wall_column = j == 0 || j == s.ny - 1 || k0 == 0 || k0 + kVec >= s.nz;

    // Layer profiles are read where used (L1-resident): holding the z profiles of the chunk
    // across the march would cost registers the load phase needs.
    T fj_cell = T(1), fj_face = T(1), fj1_face = T(1);
    if (LAYER) {
        fj_cell = __ldg(s.cell[1] + j);
        fj_face = __ldg(s.face[1] + j);
        fj1_face = __ldg(s.face[1] + j + 1);
    }

    // Carried from plane to plane: p(i) and the updated vx on face i.
    T P[kVec], XL[kVec];
    T bad = T(0);   // NaN once a pressure this column produced is not finite
    {
        const int64_t base = (int64_t)i_begin * s.plane + column;
        Vec4<T>::ldg(s.p + base, P);
        T V[kVec], Q[kVec];
        Vec4<T>::ldg(s.vx + base, V);
        if (i_begin > 0) Vec4<T>::ldg(s.p + base - s.plane, Q);
        const T fi_face = LAYER ? __ldg(s.face[0] + i_begin) : T(1);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            T v = V[e];
            if (i_begin > 0) v = v - cv * (P[e] - Q[e]);
            XL[e] = damp3<T, LAYER>(v, fi_face, fj_cell,
                                    LAYER ? __ldg(s.cell[2] + min(k0 + e, s.nz - 1)) : T(1));
        }
    }

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        const bool x_inner = i + 1 < s.nx;
        // ---- the next plane's own-row inputs into L2 (its y-neighbour rows are other
        // threads' own rows): the loads of the next iteration then wait on L2, not DRAM.
        if (s.prefetch && i + 1 < i_end) {
            const int64_t next = base + s.plane;
            if (i + 2 < s.nx) prefetch_l2(s.p + next + s.plane);
            prefetch_l2(s.vx + next + s.plane);
            prefetch_l2(s.vy + next);
            prefetch_l2(s.vz + next);
#pragma unroll
            for (int r = 0; r < NR; r++) prefetch_l2(s.psi + r * s.field + next);
        }
        // ---- loads (all read-only: the next state goes to the other buffer)
        T PX[kVec], VXo[kVec], PYm[kVec], PYp[kVec], VY[kVec], VYp[kVec], VZ[kVec], S[NR > 0 ? NR : 1][kVec];
        if (x_inner) Vec4<T>::ldg(s.p + base + s.plane, PX);
        Vec4<T>::ldg(s.vx + base + s.plane, VXo);
        if (j > 0) Vec4<T>::ldg(s.p + base - s.pz, PYm);
        if (j + 1 < s.ny) Vec4<T>::ldg(s.p + base + s.pz, PYp);
        Vec4<T>::ldg(s.vy + base, VY);
        Vec4<T>::ldg(s.vy + base + s.pz, VYp);
        Vec4<T>::ldg(s.vz + base, VZ);
        const T p_below = k0 > 0 ? __ldg(s.p + base - 1) : T(0);
        const T p_above = has_above ? __ldg(s.p + base + kVec) : T(0);
        const T vz_above = k0 + kVec <= s.nz ? __ldg(s.vz + base + kVec) : T(0);
#pragma unroll
        for (int r = 0; r < NR; r++) Vec4<T>::load(s.psi + r * s.field + base, S[r]);
        T fi_cell = T(1), fi1_face = T(1);
        if (LAYER) {
            fi_cell = __ldg(s.cell[0] + i);
            fi1_face = __ldg(s.face[0] + i + 1);
        }

        // ---- updated faces: x upper (carried on), y lower and upper, z lower and upper
        T XH[kVec], YL[kVec], YH[kVec], ZL[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const T fkc = LAYER ? __ldg(s.cell[2] + min(k0 + e, s.nz - 1)) : T(1);
            T v = VXo[e];
            if (x_inner) v = v - cv * (PX[e] - P[e]);
            XH[e] = damp3<T, LAYER>(v, fi1_face, fj_cell, fkc);
            v = VY[e];
            if (j > 0) v = v - cv * (P[e] - PYm[e]);
            YL[e] = damp3<T, LAYER>(v, fi_cell, fj_face, fkc);
            v = VYp[e];
            if (j + 1 < s.ny) v = v - cv * (PYp[e] - P[e]);
            YH[e] = damp3<T, LAYER>(v, fi_cell, fj1_face, fkc);
            const int k = k0 + e;
            v = VZ[e];
            if (k > 0 && k < s.nz) v = v - cv * (P[e] - (e == 0 ? p_below : P[e - 1]));
            ZL[e] = damp3<T, LAYER>(v, fi_cell, fj_cell,
                                    LAYER ? __ldg(s.face[2] + min(k0 + e, s.nz)) : T(1));
        }
        // z face k0 + 4: the next chunk's first lower face, or the top face z = nz.
        T ZH3 = vz_above;
        if (has_above) ZH3 = ZH3 - cv * (p_above - P[kVec - 1]);
        ZH3 = damp3<T, LAYER>(ZH3, fi_cell, fj_cell,
                              LAYER ? __ldg(s.face[2] + min(k0 + kVec, s.nz)) : T(1));

        // ---- pressure, as the pressure sweep computes it
        const bool boundary = wall_column || i == 0 || i == s.nx - 1;
        T Pn[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            T pe = P[e];
            if (k < s.nz) {
                const T zh = e + 1 < kVec ? ZL[e + 1] : ZH3;
                T d = XH[e] - XL[e];
                d = d + (YH[e] - YL[e]);
                d = d + (zh - ZL[e]);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T target = d * s.gain[r];
                    const T offset = S[r][e] - target;
                    S[r][e] = offset * s.decay[r] + target;
                    pe = pe + offset * s.mean[r];
                }
                if (NR > 0) pe = pe + d * s.relax_scale;
                pe = pe - d * cp;
                if (WALLS && boundary) {
                    T fu, fp;
                    if (wall_pair(s, i, j, k, fu, fp)) pe = pe * fu - P[e] * fp;
                }
                if (LAYER) {
                    pe = pe * fi_cell;
                    pe = pe * fj_cell;
                    pe = pe * __ldg(s.cell[2] + k);
                }
            }
            Pn[e] = pe;
        }
        if (any_mine) add_sources(s, points, all_points, base, k0, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) bad = finite_acc(bad, Pn[e]);

        // ---- stores: p, the three lower faces, the far boundary faces, psi in place. A z
        // element k == nz inside this chunk is the top face, already updated in ZL (no
        // gradient, damped by face profile nz); elements past it are padding.
        T ZS[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) ZS[e] = k0 + e <= s.nz ? ZL[e] : VZ[e];
        // A slab's ghost planes get their p from the neighbours' sweeps, never from their own;
        // its boundary planes also go to the neighbours' ghost planes (in their next copies).
        if (i >= s.own_lo && i < s.own_hi) Vec4<T>::store(f.np + base, Pn);
        if (s.ghost_lo != nullptr && i == s.own_lo) Vec4<T>::store(s.ghost_lo + column, Pn);
        if (s.ghost_hi != nullptr && i == s.own_hi - 1) Vec4<T>::store(s.ghost_hi + column, Pn);
        Vec4<T>::store(f.nvx + base, XL);
        Vec4<T>::store(f.nvy + base, YL);
        Vec4<T>::store(f.nvz + base, ZS);
        if (i == s.nx - 1) Vec4<T>::store(f.nvx + base + s.plane, XH);
        if (j == s.ny - 1) Vec4<T>::store(f.nvy + base + s.pz, YH);
        if (k0 + kVec == s.nz) f.nvz[base + kVec] = ZH3;
#pragma unroll
        for (int r = 0; r < NR; r++) Vec4<T>::store(s.psi + r * s.field + base, S[r]);
        if (any_mine) record_receivers(s, points, all_points, base, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            XL[e] = XH[e];
            P[e] = PX[e];
        }
    }
    report_nonfinite(s.status, bad != bad);
}

// Resident blocks of 256 threads the compiler must fit (register budget 65536 / (256 x this)).
// For the fp32 room with a layer: 80 registers, no spills. Timed at 384^3 with the plane
// prefetch, 72 registers (56 bytes of spills) ran 2 % slower and 64 (140 bytes) 19 % slower.
#ifndef ACF_FUSED_MIN_BLOCKS
#define ACF_FUSED_MIN_BLOCKS(T, LAYER, NR) (sizeof(T) == 8 ? 2 : (LAYER || NR >= 4 ? 3 : 4))
#endif

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, ACF_FUSED_MIN_BLOCKS(T, LAYER, NR)) fused_sweep(const FusedParams<T> f) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= f.room.nchunks || j >= f.room.ny) return;
    const bool any_point = (f.room.n_src | f.room.n_rec) != 0;
    const int64_t step = any_point ? (*f.step_base + f.local_step) : 0;
    const int i_begin = blockIdx.z * f.planes;
    fused_column<T, LAYER, WALLS, NR>(f, i_begin, min(f.room.nx, i_begin + f.planes), j, c, step);
}

// ------------------------------------------------------------------------------------------
// The fused step with its inputs staged in shared memory by the bulk-copy engine.
//
// A CTA owns `rows` consecutive y rows (whole padded z rows) over a range of x planes. Rows
// j..j+n of one plane of a field are adjacent in the padded layout, so each field's share of a
// plane is ONE contiguous cp.async.bulk: p over rows j0-1 .. j0+rows (the y halo), vy over
// j0 .. j0+rows, vx, vz and the relaxation states over j0 .. j0+rows-1. One thread issues the
// copies of a plane into a ring of `stages` buffers, each completing its own mbarrier; every
// thread computes plane i from buffers i and i+1 (p and vx of the next plane) while the next
// stages-2 planes are already in flight, so the bytes in flight no longer depend on how many
// registers the arithmetic needs. A thread owns VW = 2 or 4 consecutive z elements of one row:
// shared memory per thread is what bounds the warps an SM holds (the ring takes about 70 bytes
// per thread and stage at VW = 2), so the narrower vector keeps twice as many warps resident
// to hide the arithmetic's latency. The arithmetic is fused_column's, element for element, so
// the results are identical to the two-sweep and fused schemes.
//
// The copies are issued by a producer warp of their own. Consumer warps release a buffer through
// an "empty" mbarrier once they are done with it, and the producer refills it with the plane
// `stages` further on; there is no block-wide barrier in the march, so warps drift apart by up to
// the ring depth instead of waiting for the slowest at every plane.
//
// Every wait is bounded (about two seconds). A warp whose wait runs out raises the room's error
// flag and stops; the producer, before it returns, waits (bounded again) for the copies it has
// issued. The host reports the flag as an error.

constexpr int kStagedBarrierBytes = 128;       // full[8] then empty[8] mbarriers
constexpr int kStagedMaxStages = 8;
constexpr int kStagedMaxConsumers = 256;      // compute threads per CTA; one producer warp more
constexpr uint64_t kWaitLimitNs = 2000000000ull;
constexpr int kWaitLimitIterations = 1 << 21;

template <typename T>
struct StagedParams {
    FusedParams<T> f;
    int32_t rows, stages, vector;   // vector: z elements per thread, 2 or 4
    int32_t block_x;                // compute threads per row (a multiple of 32)
    int64_t stage_elems;            // elements of one ring buffer
    int64_t off_vx, off_vy, off_vz, off_psi;
    int32_t *error;                 // kStatusWaitTimeout is raised here when a wait ran out
    float2 pairs[16];               // single precision: coefficients duplicated into both lanes
    // Test hooks, neutral by default: the time limit of every wait, and one x plane whose copies
    // the producer of the grid's first CTA leaves out (-1: none), so that its consumers' waits
    // run out and the kernel returns with kStatusWaitTimeout raised instead of hanging.
    uint64_t wait_limit_ns;
    int32_t skip_plane;
    int32_t reserved;
};

// Slots of StagedParams::pairs; the Neg slots hold the negated coefficient.
enum { kPairCv = 0, kPairCp = 1, kPairNegRelaxScale = 2, kPairGain = 3, kPairNegDecay = 7, kPairNegMean = 11 };

// Packed single precision (sm_100 f32x2), each lane rounded exactly as the scalar operation it
// replaces. a +- b is the fused a + (+-1) b: the product by +-1 is exact, so the one rounding is
// that of a +- b. The code generator was measured to fuse a packed multiply into a packed add
// that consumes it -- one rounding where the reference has two -- even with contraction
// disabled, and even through a + 1 * b; it was not measured to do so through a - b. So every
// "plus a product" below is written as "minus the product by the negated coefficient", which
// rounds identically (negation is exact and rounding is symmetric in sign), and add2 only ever
// adds values that are not products.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(1.0f, 1.0f), a);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 dup2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 damp2(float2 v, float2 fa, float2 fb, float2 fc) {
    return mul2(mul2(mul2(v, fa), fb), fc);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// One try with a suspend-time hint of a microsecond: true once the phase of `parity` completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: false when the phase completed neither within `limit_ns` (kWaitLimitNs unless
// a test shortened it) nor within kWaitLimitIterations tries.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t start = global_ns();
    for (int it = 0; it < kWaitLimitIterations; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - start > limit_ns) return false;
    }
    return false;
}

// Global -> shared bulk copy (no multicast), completing `bytes` on the mbarrier. Both addresses
// are 16-byte aligned and bytes is a multiple of 16: every copy here starts on a padded row.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

template <typename T>
__device__ __forceinline__ void lds4(const T *a, T v[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(a);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
        const double2 t0 = *reinterpret_cast<const double2 *>(a);
        const double2 t1 = *reinterpret_cast<const double2 *>(a + 2);
        v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
    }
}

// W consecutive elements (W = 2 or 4) of global or shared memory: one 8- or 16-byte access
// for float, one or two 16-byte accesses for double.
template <typename T, int W>
struct VecW;

template <typename T>
struct VecW<T, 4> {
    __device__ __forceinline__ static void ldg(const T *__restrict__ a, T v[4]) { Vec4<T>::ldg(a, v); }
    __device__ __forceinline__ static void ldcs(const T *a, T v[4]) { Vec4<T>::ldcs(a, v); }
    __device__ __forceinline__ static void load(const T *a, T v[4]) { Vec4<T>::load(a, v); }
    __device__ __forceinline__ static void store(T *__restrict__ a, const T v[4]) { Vec4<T>::store(a, v); }
    __device__ __forceinline__ static void lds(const T *a, T v[4]) { lds4<T>(a, v); }
};

template <>
struct VecW<float, 2> {
    __device__ __forceinline__ static void ldg(const float *__restrict__ a, float v[2]) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(a));
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void ldcs(const float *a, float v[2]) {
        const float2 t = __ldcs(reinterpret_cast<const float2 *>(a));
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void load(const float *a, float v[2]) {
        const float2 t = *reinterpret_cast<const float2 *>(a);
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void store(float *__restrict__ a, const float v[2]) {
        *reinterpret_cast<float2 *>(a) = make_float2(v[0], v[1]);
    }
    __device__ __forceinline__ static void lds(const float *a, float v[2]) {
        const float2 t = *reinterpret_cast<const float2 *>(a);
        v[0] = t.x; v[1] = t.y;
    }
};

template <>
struct VecW<double, 2> {
    __device__ __forceinline__ static void ldg(const double *__restrict__ a, double v[2]) {
        const double2 t = __ldg(reinterpret_cast<const double2 *>(a));
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void ldcs(const double *a, double v[2]) {
        const double2 t = __ldcs(reinterpret_cast<const double2 *>(a));
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void load(const double *a, double v[2]) {
        const double2 t = *reinterpret_cast<const double2 *>(a);
        v[0] = t.x; v[1] = t.y;
    }
    __device__ __forceinline__ static void store(double *__restrict__ a, const double v[2]) {
        *reinterpret_cast<double2 *>(a) = make_double2(v[0], v[1]);
    }
    __device__ __forceinline__ static void lds(const double *a, double v[2]) {
        const double2 t = *reinterpret_cast<const double2 *>(a);
        v[0] = t.x; v[1] = t.y;
    }
};

// Sources and receivers inside one CTA's tile, gathered once per launch so that the march
// does not scan every point at every plane. Sorted by index: sources (q < n_src) come first, in
// the order they were added, so several sources in one cell add up in the reference's order and
// receivers read the finished pressure.
constexpr int kStagedPointCap = 32;

struct TilePoint {
    int32_t q;      // source index, or n_src + receiver index
    int32_t i;      // x plane
    int32_t row;    // y row within the tile
    int32_t k;      // z index
};

template <typename T, bool LAYER, bool WALLS, int NR, int VW>
__global__ void __maxnreg__(sizeof(T) == 8 ? (VW == 2 ? 128 : 168) : (VW == 2 ? 80 : 128))
fused_staged_sweep(const StagedParams<T> g) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ TilePoint points[kStagedPointCap];
    __shared__ int n_points;
    const FusedParams<T> &f = g.f;
    const Room<T> &s = f.room;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + kStagedMaxStages;
    T *ring = reinterpret_cast<T *>(smem + kStagedBarrierBytes);

    const int S = g.stages;
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int consumers = g.block_x * g.rows;       // the last warp (tid >= consumers) is the producer
    const bool producer = tid >= consumers;
    const int lane = tid & 31;
    const int j0 = blockIdx.x * g.rows;
    const int i_begin = blockIdx.y * f.planes;
    const int i_end = min(s.nx, i_begin + f.planes);
    // Rows each copy covers. Own rows stop at the last real row; the p halo stops at ny - 1.
    const int n_own = min(g.rows, s.ny - j0);
    const int p_lo = max(j0 - 1, 0);
    const int p_hi = min(j0 + n_own, s.ny - 1);
    const uint32_t row_bytes = (uint32_t)(s.pz * (int64_t)sizeof(T));
    const uint32_t bytes_p = (uint32_t)(p_hi - p_lo + 1) * row_bytes;
    const uint32_t bytes_own = (uint32_t)n_own * row_bytes;
    const uint32_t bytes_vy = (uint32_t)(n_own + 1) * row_bytes;

    // Plane i into buffer `slot`. Plane i_end (<= nx, inside every field's nx + 1 planes) is
    // only read for p and vx, and its relaxation states belong to the next CTA along x.
    const bool skipping = g.skip_plane >= 0 && blockIdx.x == 0 && blockIdx.y == 0;
    auto issue = [&](int i, int slot) {
        if (skipping && i == g.skip_plane) return;   // test hook: this plane never arrives
        T *dst = ring + (int64_t)slot * g.stage_elems;
        const int64_t plane = (int64_t)i * s.plane;
        const int64_t own = plane + (int64_t)j0 * s.pz;
        const bool whole = i < i_end;
        const uint32_t total = bytes_p + bytes_own + (whole ? bytes_vy + bytes_own * (1 + NR) : 0u);
        mbar_arrive_expect_tx(full + slot, total);
        bulk_load(dst + (int64_t)(p_lo - j0 + 1) * s.pz, s.p + plane + (int64_t)p_lo * s.pz, bytes_p,
                  full + slot);
        bulk_load(dst + g.off_vx, s.vx + own, bytes_own, full + slot);
        if (whole) {
            bulk_load(dst + g.off_vy, s.vy + own, bytes_vy, full + slot);
            bulk_load(dst + g.off_vz, s.vz + own, bytes_own, full + slot);
#pragma unroll
            for (int r = 0; r < NR; r++)
                bulk_load(dst + g.off_psi + (int64_t)r * g.rows * s.pz, s.psi + r * s.field + own,
                          bytes_own, full + slot);
        }
    };

    if (tid == 0) {
        for (int q = 0; q < S; q++) {
            mbar_init(full + q, 1);
            mbar_init(empty + q, consumers / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        n_points = 0;
    }
    __syncthreads();
    int issued = i_begin - 1;   // last plane issued (producer lane 0)
    if (tid == consumers) {
        for (int q = 0; q < S && i_begin + q <= i_end; q++) issue(i_begin + q, q);
        issued = min(i_begin + S - 1, i_end);
    }

    // Points of this tile (while the first planes are in flight).
    const bool any_point = (s.n_src | s.n_rec) != 0;
    if (any_point) {
        const int total = s.n_src + s.n_rec;
        for (int q = tid; q < total; q += nthreads) {
            const int64_t off = q < s.n_src ? s.src_off[q] : s.rec_off[q - s.n_src];
            const int pi = (int)(off / s.plane);
            const int64_t rem = off - (int64_t)pi * s.plane;
            const int pj = (int)(rem / s.pz);
            const int pk = (int)(rem - (int64_t)pj * s.pz);
            if (pi >= i_begin && pi < i_end && pj >= j0 && pj < j0 + n_own) {
                const int at = atomicAdd(&n_points, 1);
                if (at < kStagedPointCap) points[at] = TilePoint{q, pi, pj - j0, pk};
            }
        }
        __syncthreads();
        if (tid == 0 && n_points > 1 && n_points <= kStagedPointCap) {
            for (int a = 1; a < n_points; a++) {
                const TilePoint key = points[a];
                int b = a - 1;
                while (b >= 0 && points[b].q > key.q) {
                    points[b + 1] = points[b];
                    b--;
                }
                points[b + 1] = key;
            }
        }
        __syncthreads();
    }
    const int np = any_point ? n_points : 0;
    const bool overflow = np > kStagedPointCap;   // too many: scan every point, as fused_column

    const int c = tid % g.block_x;
    const int ry = tid / g.block_x;
    const int j = j0 + ry;
    const bool active = !producer && c < (s.nz + VW - 1) / VW && j < s.ny;
    const int k0 = c * VW;
    const T cv = s.cv, cp = s.cp;
    const int64_t step = any_point ? (*f.step_base + f.local_step) : 0;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool has_above = k0 + VW < s.nz;
    const bool wall_k = k0 == 0 || k0 + VW >= s.nz;   // the chunk holds k = 0 or k = nz - 1

    // Damping profiles along y and z are fixed for the thread's whole march.
    T fj_cell = T(1), fj_face = T(1), fj1_face = T(1);
    T fkc[VW], fkf[VW + 1];
#pragma unroll
    for (int e = 0; e < VW; e++) fkc[e] = T(1);
#pragma unroll
    for (int e = 0; e <= VW; e++) fkf[e] = T(1);
    T XL[VW];
    if (active) {
        if (LAYER) {
            fj_cell = __ldg(s.cell[1] + j);
            fj_face = __ldg(s.face[1] + j);
            fj1_face = __ldg(s.face[1] + j + 1);
#pragma unroll
            for (int e = 0; e < VW; e++) fkc[e] = __ldg(s.cell[2] + min(k0 + e, s.nz - 1));
#pragma unroll
            for (int e = 0; e <= VW; e++) fkf[e] = __ldg(s.face[2] + min(k0 + e, s.nz));
        }
        // The updated vx on face i_begin, as fused_column starts its march.
        const int64_t base = (int64_t)i_begin * s.plane + column;
        T P0[VW], V[VW], Q[VW];
        VecW<T, VW>::ldg(s.p + base, P0);
        VecW<T, VW>::ldg(s.vx + base, V);
        if (i_begin > 0) VecW<T, VW>::ldg(s.p + base - s.plane, Q);
        const T fi_face = LAYER ? __ldg(s.face[0] + i_begin) : T(1);
#pragma unroll
        for (int e = 0; e < VW; e++) {
            T v = V[e];
            if (i_begin > 0) v = v - cv * (P0[e] - Q[e]);
            XL[e] = damp3<T, LAYER>(v, fi_face, fj_cell, fkc[e]);
        }
    }

    if (producer) {
        // Refill each buffer once every consumer warp has released it.
        if (lane == 0) {
            bool ok = true;
            for (int q = i_begin + S; q <= i_end; q++) {
                const int u = q - i_begin;
                if (!mbar_wait(empty + u % S, (uint32_t)(u / S - 1) & 1u, g.wait_limit_ns)) {
                    ok = false;
                    break;
                }
                issue(q, u % S);
                issued = q;
            }
            if (!ok) {
                atomicOr(g.error, kStatusWaitTimeout);
                // The latest plane issued into each buffer must land before the CTA exits.
                for (int q = max(i_begin, issued - S + 1); q <= issued; q++) {
                    const int u = q - i_begin;
                    mbar_wait(full + u % S, (uint32_t)(u / S) & 1u, g.wait_limit_ns);
                }
            }
        }
        return;
    }

    T bad = T(0);   // NaN once a pressure this thread produced is not finite
    // x damping profiles of the current plane, loaded one plane ahead.
    T fi_cell_next = T(1), fi1_face_next = T(1);
    if (LAYER && active) {
        fi_cell_next = __ldg(s.cell[0] + i_begin);
        fi1_face_next = __ldg(s.face[0] + i_begin + 1);
    }
    for (int i = i_begin; i < i_end; i++) {
        const int u = i - i_begin;
        const int slot = u % S, nslot = (u + 1) % S;
        // Buffer `slot` (plane i) was already waited for as the next plane, except at the start.
        bool ready = u > 0 || mbar_wait(full + slot, 0u, g.wait_limit_ns);
        ready = ready && mbar_wait(full + nslot, (uint32_t)((u + 1) / S) & 1u, g.wait_limit_ns);
        if (!ready) {
            atomicOr(g.error, kStatusWaitTimeout);
            return;
        }
        const T fi_cell_here = fi_cell_next, fi1_face_here = fi1_face_next;
        if (LAYER && active && i + 1 < i_end) {
            fi_cell_next = __ldg(s.cell[0] + i + 1);
            fi1_face_next = __ldg(s.face[0] + i + 2);
        }
        if (active) {
            const T *cur = ring + (int64_t)slot * g.stage_elems;
            const T *nxt = ring + (int64_t)nslot * g.stage_elems;
            const int64_t base = (int64_t)i * s.plane + column;
            const bool x_inner = i + 1 < s.nx;
            const T *prow = cur + (int64_t)(ry + 1) * s.pz + k0;
            const T *vyrow = cur + g.off_vy + (int64_t)ry * s.pz + k0;
            const T *vzrow = cur + g.off_vz + (int64_t)ry * s.pz + k0;
            T P[VW], PX[VW], VXo[VW], PYm[VW], PYp[VW], VY[VW], VYp[VW], VZ[VW];
            T Sg[NR > 0 ? NR : 1][VW];
            VecW<T, VW>::lds(prow, P);
            if (x_inner) VecW<T, VW>::lds(nxt + (int64_t)(ry + 1) * s.pz + k0, PX);
            VecW<T, VW>::lds(nxt + g.off_vx + (int64_t)ry * s.pz + k0, VXo);
            if (j > 0) VecW<T, VW>::lds(prow - s.pz, PYm);
            if (j + 1 < s.ny) VecW<T, VW>::lds(prow + s.pz, PYp);
            VecW<T, VW>::lds(vyrow, VY);
            VecW<T, VW>::lds(vyrow + s.pz, VYp);
            VecW<T, VW>::lds(vzrow, VZ);
            const T p_below = k0 > 0 ? prow[-1] : T(0);
            const T p_above = has_above ? prow[VW] : T(0);
            const T vz_above = k0 + VW <= s.nz ? vzrow[VW] : T(0);
#pragma unroll
            for (int r = 0; r < NR; r++)
                VecW<T, VW>::lds(cur + g.off_psi + ((int64_t)r * g.rows + ry) * s.pz + k0, Sg[r]);
            const T fi_cell = fi_cell_here, fi1_face = fi1_face_here;

            T XH[VW], YL[VW], YH[VW], ZL[VW], Pn[VW], ZH3;
            const bool wall_cell = WALLS && (wall_k || j == 0 || j == s.ny - 1 || i == 0 || i == s.nx - 1);
            if constexpr (sizeof(T) == 4) {
                // Packed single precision: two lanes per instruction, each lane rounded exactly
                // as the scalar operation it replaces, in the same order.
                constexpr int NP = VW / 2;
                const float2 cv2 = g.pairs[kPairCv];
                const float2 fic = dup2(fi_cell), fi1f = dup2(fi1_face);
                const float2 fjc = dup2(fj_cell), fjf = dup2(fj_face), fj1f = dup2(fj1_face);
                float2 P2[NP], XH2[NP], YL2[NP], YH2[NP], ZL2[NP];
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    const int a = 2 * q;
                    P2[q] = make_float2(P[a], P[a + 1]);
                    const float2 fk = make_float2(fkc[a], fkc[a + 1]);
                    float2 v = make_float2(VXo[a], VXo[a + 1]);
                    if (x_inner) v = sub2(v, mul2(cv2, sub2(make_float2(PX[a], PX[a + 1]), P2[q])));
                    XH2[q] = LAYER ? damp2(v, fi1f, fjc, fk) : v;
                    v = make_float2(VY[a], VY[a + 1]);
                    if (j > 0) v = sub2(v, mul2(cv2, sub2(P2[q], make_float2(PYm[a], PYm[a + 1]))));
                    YL2[q] = LAYER ? damp2(v, fic, fjf, fk) : v;
                    v = make_float2(VYp[a], VYp[a + 1]);
                    if (j + 1 < s.ny) v = sub2(v, mul2(cv2, sub2(make_float2(PYp[a], PYp[a + 1]), P2[q])));
                    YH2[q] = LAYER ? damp2(v, fic, fj1f, fk) : v;
                    // z lower faces: lanes with 0 < k < nz take the gradient update
                    const float2 vz = make_float2(VZ[a], VZ[a + 1]);
                    const float2 pm = make_float2(a == 0 ? p_below : P[a - 1], P[a]);
                    v = sub2(vz, mul2(cv2, sub2(P2[q], pm)));
                    if (!(k0 > 0 && k0 + VW <= s.nz)) {
                        if (!(k0 + a > 0 && k0 + a < s.nz)) v.x = vz.x;
                        if (!(k0 + a + 1 < s.nz)) v.y = vz.y;
                    }
                    ZL2[q] = LAYER ? damp2(v, fic, fjc, make_float2(fkf[a], fkf[a + 1])) : v;
                }
                ZH3 = vz_above;
                if (has_above) ZH3 = ZH3 - cv * (p_above - P[VW - 1]);
                ZH3 = damp3<T, LAYER>(ZH3, fi_cell, fj_cell, fkf[VW]);

#pragma unroll
                for (int q = 0; q < NP; q++) {
                    const int a = 2 * q;
                    const float2 xl = make_float2(XL[a], XL[a + 1]);
                    const float2 zh = make_float2(ZL2[q].y, q + 1 < NP ? ZL2[q + 1 < NP ? q + 1 : q].x : ZH3);
                    float2 d = sub2(XH2[q], xl);
                    d = add2(d, sub2(YH2[q], YL2[q]));
                    d = add2(d, sub2(zh, ZL2[q]));
                    float2 pe = P2[q];
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        const float2 old = make_float2(Sg[r][a], Sg[r][a + 1]);
                        const float2 target = mul2(d, g.pairs[kPairGain + r]);
                        const float2 offset = sub2(old, target);
                        // offset * decay + target, pe + offset * mean
                        float2 next = sub2(target, mul2(offset, g.pairs[kPairNegDecay + r]));
                        pe = sub2(pe, mul2(offset, g.pairs[kPairNegMean + r]));
                        if (k0 + a >= s.nz) next.x = old.x;          // padding lanes keep psi
                        if (k0 + a + 1 >= s.nz) next.y = old.y;
                        Sg[r][a] = next.x;
                        Sg[r][a + 1] = next.y;
                    }
                    if (NR > 0) pe = sub2(pe, mul2(d, g.pairs[kPairNegRelaxScale]));   // pe + d * scale
                    pe = sub2(pe, mul2(d, g.pairs[kPairCp]));
                    bad = finite_acc(finite_acc(bad, pe.x), pe.y);
                    if (WALLS && wall_cell) {
                        float fu, fp;
                        if (k0 + a < s.nz && wall_pair(s, i, j, k0 + a, fu, fp)) pe.x = pe.x * fu - P[a] * fp;
                        if (k0 + a + 1 < s.nz && wall_pair(s, i, j, k0 + a + 1, fu, fp))
                            pe.y = pe.y * fu - P[a + 1] * fp;
                    }
                    if (LAYER) pe = mul2(mul2(mul2(pe, fic), fjc), make_float2(fkc[a], fkc[a + 1]));
                    Pn[a] = k0 + a < s.nz ? pe.x : P[a];
                    Pn[a + 1] = k0 + a + 1 < s.nz ? pe.y : P[a + 1];
                    XH[a] = XH2[q].x;
                    XH[a + 1] = XH2[q].y;
                    YL[a] = YL2[q].x;
                    YL[a + 1] = YL2[q].y;
                    YH[a] = YH2[q].x;
                    YH[a + 1] = YH2[q].y;
                    ZL[a] = ZL2[q].x;
                    ZL[a + 1] = ZL2[q].y;
                }
            } else {
    #pragma unroll
                for (int e = 0; e < VW; e++) {
                    T v = VXo[e];
                    if (x_inner) v = v - cv * (PX[e] - P[e]);
                    XH[e] = damp3<T, LAYER>(v, fi1_face, fj_cell, fkc[e]);
                    v = VY[e];
                    if (j > 0) v = v - cv * (P[e] - PYm[e]);
                    YL[e] = damp3<T, LAYER>(v, fi_cell, fj_face, fkc[e]);
                    v = VYp[e];
                    if (j + 1 < s.ny) v = v - cv * (PYp[e] - P[e]);
                    YH[e] = damp3<T, LAYER>(v, fi_cell, fj1_face, fkc[e]);
                    const int k = k0 + e;
                    v = VZ[e];
                    if (k > 0 && k < s.nz) v = v - cv * (P[e] - (e == 0 ? p_below : P[e - 1]));
                    ZL[e] = damp3<T, LAYER>(v, fi_cell, fj_cell, fkf[e]);
                }
                ZH3 = vz_above;
                if (has_above) ZH3 = ZH3 - cv * (p_above - P[VW - 1]);
                ZH3 = damp3<T, LAYER>(ZH3, fi_cell, fj_cell, fkf[VW]);

    #pragma unroll
                for (int e = 0; e < VW; e++) {
                    const int k = k0 + e;
                    T pe = P[e];
                    if (k < s.nz) {
                        const T zh = e + 1 < VW ? ZL[e + 1] : ZH3;
                        T d = XH[e] - XL[e];
                        d = d + (YH[e] - YL[e]);
                        d = d + (zh - ZL[e]);
    #pragma unroll
                        for (int r = 0; r < NR; r++) {
                            const T target = d * s.gain[r];
                            const T offset = Sg[r][e] - target;
                            Sg[r][e] = offset * s.decay[r] + target;
                            pe = pe + offset * s.mean[r];
                        }
                        if (NR > 0) pe = pe + d * s.relax_scale;
                        pe = pe - d * cp;
                        if (WALLS && wall_cell) {
                            T fu, fp;
                            if (wall_pair(s, i, j, k, fu, fp)) pe = pe * fu - P[e] * fp;
                        }
                        if (LAYER) {
                            pe = pe * fi_cell;
                            pe = pe * fj_cell;
                            pe = pe * fkc[e];
                        }
                    }
                    Pn[e] = pe;
                    bad = finite_acc(bad, pe);
                }

            }

            // Sources after damping, then receivers (scheme.py:293-296,360-363).
            if (any_point && !overflow) {
                for (int t = 0; t < np; t++) {
                    const TilePoint pt = points[t];
                    const int d = pt.k - k0;
                    if (pt.i != i || pt.row != ry || d < 0 || d >= VW) continue;
                    if (pt.q < s.n_src) {
                        if (pt.k < s.nz && step < s.src_len[pt.q]) {
                            const T add = s.cs * s.src_sig[pt.q * s.src_stride + step];
#pragma unroll
                            for (int e = 0; e < VW; e++)
                                if (e == d) Pn[e] = Pn[e] + add;
                        }
                    } else {
                        const int r = pt.q - s.n_src;
                        if (step >= s.rec_start[r]) {
                            T v = Pn[0];
#pragma unroll
                            for (int e = 1; e < VW; e++)
                                if (e == d) v = Pn[e];
                            s.rec[r * s.rec_stride + (step - s.rec_origin)] = v;
                        }
                    }
                }
            } else if (any_point) {
                for (int q = 0; q < s.n_src; q++) {
                    const int64_t d = s.src_off[q] - base;
                    if (d >= 0 && d < VW && k0 + d < s.nz && step < s.src_len[q]) {
#pragma unroll
                        for (int e = 0; e < VW; e++)
                            if (e == d) Pn[e] = Pn[e] + s.cs * s.src_sig[q * s.src_stride + step];
                    }
                }
                for (int r = 0; r < s.n_rec; r++) {
                    const int64_t d = s.rec_off[r] - base;
                    if (d >= 0 && d < VW && step >= s.rec_start[r]) {
                        T v = Pn[0];
#pragma unroll
                        for (int e = 1; e < VW; e++)
                            if (e == d) v = Pn[e];
                        s.rec[r * s.rec_stride + (step - s.rec_origin)] = v;
                    }
                }
            }

            T ZS[VW];
#pragma unroll
            for (int e = 0; e < VW; e++) ZS[e] = k0 + e <= s.nz ? ZL[e] : VZ[e];
            VecW<T, VW>::store(f.np + base, Pn);
            VecW<T, VW>::store(f.nvx + base, XL);
            VecW<T, VW>::store(f.nvy + base, YL);
            VecW<T, VW>::store(f.nvz + base, ZS);
            if (i == s.nx - 1) VecW<T, VW>::store(f.nvx + base + s.plane, XH);
            if (j == s.ny - 1) VecW<T, VW>::store(f.nvy + base + s.pz, YH);
            if (k0 + VW == s.nz) f.nvz[base + VW] = ZH3;
#pragma unroll
            for (int r = 0; r < NR; r++) VecW<T, VW>::store(s.psi + r * s.field + base, Sg[r]);
#pragma unroll
            for (int e = 0; e < VW; e++) XL[e] = XH[e];
        }
        // This warp is done with buffer `slot` (plane i).
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + slot);
    }
    report_nonfinite(s.status, bad != bad);
}

// ------------------------------------------------------------------------------------------
// The fused step in single precision, lean in instructions (rooms with nz a multiple of 4).
//
// Bound by HBM only while its warps issue fast enough: fused_column spends about 190
// thread-instructions per cell, so under the power cap's lower SM clock the step slowed with the
// clock. This column performs the same operations with a third of the instructions:
//   * the two-lane f32x2 arithmetic of the staged sweep (same rounding, lane for lane);
//   * damping only by factors that are not exactly 1: a product by 1.0 is the identity, so a
//     thread skips the multiplications of an axis whose profile is 1 at its row, chunk or plane
//     (the middle of a room with a sponge on its x faces damps nothing) and the products it does
//     form keep the x, y, z order -- results are unchanged bit for bit;
//   * z profiles of the chunk held in registers, x profiles loaded once per plane;
//   * with nz a multiple of 4 no chunk holds padding, so the only per-element edge is the k = 0
//     face of the first chunk; every other test is uniform over a plane or a row.

struct LeanParams {
    FusedParams<float> f;
    float2 pairs[16];      // the slots of StagedParams::pairs
};

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// The per-column constants of a lean column: its place, its edges, its sources and receivers and
// the y and z layer factors of its cells and faces.
struct LeanColumn {
    int j, k0, real;
    int64_t column;                 // j * pz + k0
    bool y_lo, y_hi, z_lo, z_hi;
    bool tail;                      // a padding chunk (rows with nz not a multiple of 4)
    bool wall_column, all_points, any_mine, damp_y, damp_z;
    uint32_t points;
    float fj_cell, fj_face, fj1_face, fkf4;
    float2 fkc01, fkc23, fkf01, fkf23;
};

// ALIGNED: nz is a multiple of 4. Otherwise the last chunk of every row holds padding elements
// (k >= nz), which this column leaves as they are, and the top face k = nz, which it damps
// without a gradient update -- exactly as fused_column does -- with per-thread fix-ups that only
// the threads of those chunks take.
template <bool LAYER, bool ALIGNED>
__device__ __forceinline__ LeanColumn lean_setup(const Room<float> &s, int j, int c) {
    LeanColumn col;
    col.j = j;
    col.k0 = c * kVec;
    const int k0 = col.k0;
    col.column = (int64_t)j * s.pz + k0;
    col.y_lo = j > 0;
    col.y_hi = j + 1 < s.ny;
    col.z_lo = k0 > 0;
    col.z_hi = k0 + kVec < s.nz;
    // Padding chunk: `real` elements (1..3) lie inside the room, the next one is the top face.
    col.tail = !ALIGNED && k0 + kVec > s.nz;
    col.real = col.tail ? s.nz - k0 : kVec;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    col.all_points = false;
    col.points = any_point ? column_points(s, j, k0, col.all_points) : 0u;
    col.any_mine = col.points != 0 || col.all_points;
    col.wall_column = !col.y_lo || !col.y_hi || !col.z_lo || !col.z_hi;
    col.fj_cell = col.fj_face = col.fj1_face = col.fkf4 = 1.f;
    col.fkc01 = col.fkc23 = col.fkf01 = col.fkf23 = dup2(1.f);
    col.damp_y = col.damp_z = false;
    if (LAYER) {
        col.fj_cell = __ldg(s.cell[1] + j);
        col.fj_face = __ldg(s.face[1] + j);
        col.fj1_face = __ldg(s.face[1] + j + 1);
        // padding lanes take the last cell's and the top face's factors, as fused_column does
        const int c_last = s.nz - 1, f_last = s.nz;
        auto kc = [&](int e) { return __ldg(s.cell[2] + (ALIGNED ? k0 + e : min(k0 + e, c_last))); };
        auto kf = [&](int e) { return __ldg(s.face[2] + (ALIGNED ? k0 + e : min(k0 + e, f_last))); };
        col.fkc01 = make_float2(kc(0), kc(1));
        col.fkc23 = make_float2(kc(2), kc(3));
        col.fkf01 = make_float2(kf(0), kf(1));
        col.fkf23 = make_float2(kf(2), kf(3));
        col.fkf4 = kf(4);
        col.damp_y = col.fj_cell != 1.f || col.fj_face != 1.f || col.fj1_face != 1.f;
        col.damp_z = col.fkc01.x != 1.f || col.fkc01.y != 1.f || col.fkc23.x != 1.f ||
                     col.fkc23.y != 1.f || col.fkf01.x != 1.f || col.fkf01.y != 1.f ||
                     col.fkf23.x != 1.f || col.fkf23.y != 1.f || col.fkf4 != 1.f;
    }
    return col;
}

// The updated x face below the first plane i of a march: the face's velocity V moved by the
// pressures P (plane i) and Q (plane i - 1, when i > 0), then damped.
template <bool LAYER>
__device__ __forceinline__ void lean_lower_face(const LeanParams &g, const LeanColumn &col, int i,
                                                float4 V, float4 P, float4 Q, float2 &XL01,
                                                float2 &XL23) {
    const Room<float> &s = g.f.room;
    const float2 cv2 = g.pairs[kPairCv];
    XL01 = lo2(V);
    XL23 = hi2(V);
    if (i > 0) {
        XL01 = sub2(XL01, mul2(cv2, sub2(lo2(P), lo2(Q))));
        XL23 = sub2(XL23, mul2(cv2, sub2(hi2(P), hi2(Q))));
    }
    if (LAYER) {
        const float fi_face = __ldg(s.face[0] + i);
        if (fi_face != 1.f) {
            XL01 = mul2(XL01, dup2(fi_face));
            XL23 = mul2(XL23, dup2(fi_face));
        }
        if (col.damp_y) {
            XL01 = mul2(XL01, dup2(col.fj_cell));
            XL23 = mul2(XL23, dup2(col.fj_cell));
        }
        if (col.damp_z) {
            XL01 = mul2(XL01, col.fkc01);
            XL23 = mul2(XL23, col.fkc23);
        }
    }
}

// The state around one chunk at plane i before a step: its pressures P, the pressures next to it
// (x + 1, y -+ 1, z below and above), and the velocities of its faces (x upper, y lower and
// upper, z lower and the one above the chunk).
struct LeanInputs {
    float4 P, PX, PYm, PYp, VXo, VY, VYp, VZ;
    float p_below, p_above, vz_above;
};

// The chunk's updated faces after the step: x upper, y lower and upper, z lower and above.
struct LeanFaces {
    float2 XH01, XH23, YL01, YL23, YH01, YH23, ZL01, ZL23;
    float ZH3;
};

// One step of one chunk at plane i: from the state around it (`in`, the updated lower x face
// XL and the relaxation states S, which it advances in place) to its updated faces and its next
// pressures Pn, with walls, the sponge and the sources of `step`. `bad2` turns NaN once a
// pressure produced is not finite.
template <bool LAYER, bool WALLS, int NR, bool ALIGNED, bool REC = false>
__device__ __forceinline__ void lean_update(const LeanParams &g, const LeanColumn &col, int i,
                                            int64_t base, int64_t step, const LeanInputs &in,
                                            float2 XL01, float2 XL23, float4 (&S)[NR > 0 ? NR : 1],
                                            LeanFaces &o, float (&Pn)[kVec], float2 &bad2,
                                            float *PT = nullptr) {
    const Room<float> &s = g.f.room;
    const bool x_inner = i + 1 < s.nx;
    const float2 cv2 = g.pairs[kPairCv], cp2 = g.pairs[kPairCp];
    const float cv = cv2.x;
    const bool tail = col.tail;
    const int real = col.real;
    float fi_cell = 1.f, fi1_face = 1.f;
    if (LAYER) {
        fi_cell = __ldg(s.cell[0] + i);
        fi1_face = __ldg(s.face[0] + i + 1);
    }

    // ---- updated faces: x upper (carried on), y lower and upper, z lower and upper
    const float4 P = in.P;
    const float2 P01 = lo2(P), P23 = hi2(P);
    float2 XH01 = lo2(in.VXo), XH23 = hi2(in.VXo);
    if (x_inner) {
        XH01 = sub2(XH01, mul2(cv2, sub2(lo2(in.PX), P01)));
        XH23 = sub2(XH23, mul2(cv2, sub2(hi2(in.PX), P23)));
    }
    float2 YL01 = lo2(in.VY), YL23 = hi2(in.VY);
    if (col.y_lo) {
        YL01 = sub2(YL01, mul2(cv2, sub2(P01, lo2(in.PYm))));
        YL23 = sub2(YL23, mul2(cv2, sub2(P23, hi2(in.PYm))));
    }
    float2 YH01 = lo2(in.VYp), YH23 = hi2(in.VYp);
    if (col.y_hi) {
        YH01 = sub2(YH01, mul2(cv2, sub2(lo2(in.PYp), P01)));
        YH23 = sub2(YH23, mul2(cv2, sub2(hi2(in.PYp), P23)));
    }
    const float4 VZ = in.VZ;
    float2 ZL01 = sub2(lo2(VZ), mul2(cv2, sub2(P01, make_float2(in.p_below, P.x))));
    float2 ZL23 = sub2(hi2(VZ), mul2(cv2, sub2(P23, make_float2(P.y, P.z))));
    if (!col.z_lo) ZL01.x = VZ.x;             // face k = 0: a boundary, never updated
    if (tail) {                               // faces k >= nz: the top face and padding
        if (real <= 1) ZL01.y = VZ.y;
        if (real <= 2) ZL23.x = VZ.z;
        ZL23.y = VZ.w;
    }
    float ZH3 = in.vz_above;
    if (col.z_hi) ZH3 = ZH3 - cv * (in.p_above - P.w);
    if (LAYER) {   // x, y, z order; an axis whose factors here are all 1 is skipped
        if (fi_cell != 1.f || fi1_face != 1.f) {
            const float2 a = dup2(fi1_face), b = dup2(fi_cell);
            XH01 = mul2(XH01, a); XH23 = mul2(XH23, a);
            YL01 = mul2(YL01, b); YL23 = mul2(YL23, b);
            YH01 = mul2(YH01, b); YH23 = mul2(YH23, b);
            ZL01 = mul2(ZL01, b); ZL23 = mul2(ZL23, b);
            ZH3 = ZH3 * fi_cell;
        }
        if (col.damp_y) {
            const float2 a = dup2(col.fj_cell), b = dup2(col.fj_face), e = dup2(col.fj1_face);
            XH01 = mul2(XH01, a); XH23 = mul2(XH23, a);
            YL01 = mul2(YL01, b); YL23 = mul2(YL23, b);
            YH01 = mul2(YH01, e); YH23 = mul2(YH23, e);
            ZL01 = mul2(ZL01, a); ZL23 = mul2(ZL23, a);
            ZH3 = ZH3 * col.fj_cell;
        }
        if (col.damp_z) {
            XH01 = mul2(XH01, col.fkc01); XH23 = mul2(XH23, col.fkc23);
            YL01 = mul2(YL01, col.fkc01); YL23 = mul2(YL23, col.fkc23);
            YH01 = mul2(YH01, col.fkc01); YH23 = mul2(YH23, col.fkc23);
            ZL01 = mul2(ZL01, col.fkf01); ZL23 = mul2(ZL23, col.fkf23);
            ZH3 = ZH3 * col.fkf4;
        }
    }

    // ---- pressure, as the pressure sweep computes it
    float2 d01 = sub2(XH01, XL01), d23 = sub2(XH23, XL23);
    d01 = add2(d01, sub2(YH01, YL01));
    d23 = add2(d23, sub2(YH23, YL23));
    d01 = add2(d01, sub2(make_float2(ZL01.y, ZL23.x), ZL01));
    d23 = add2(d23, sub2(make_float2(ZL23.y, ZH3), ZL23));
    float2 pe01 = P01, pe23 = P23;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const float2 t01 = mul2(d01, g.pairs[kPairGain + r]), t23 = mul2(d23, g.pairs[kPairGain + r]);
        const float2 o01 = sub2(lo2(S[r]), t01), o23 = sub2(hi2(S[r]), t23);
        // offset * decay + target, and pe + offset * mean, as minus the negated products
        const float2 n01 = sub2(t01, mul2(o01, g.pairs[kPairNegDecay + r]));
        const float2 n23 = sub2(t23, mul2(o23, g.pairs[kPairNegDecay + r]));
        pe01 = sub2(pe01, mul2(o01, g.pairs[kPairNegMean + r]));
        pe23 = sub2(pe23, mul2(o23, g.pairs[kPairNegMean + r]));
        float4 next = make_float4(n01.x, n01.y, n23.x, n23.y);
        if (tail) {                           // padding lanes keep their state
            if (real <= 1) next.y = S[r].y;
            if (real <= 2) next.z = S[r].z;
            next.w = S[r].w;
        }
        S[r] = next;
    }
    if (NR > 0) {
        pe01 = sub2(pe01, mul2(d01, g.pairs[kPairNegRelaxScale]));
        pe23 = sub2(pe23, mul2(d23, g.pairs[kPairNegRelaxScale]));
    }
    pe01 = sub2(pe01, mul2(d01, cp2));
    pe23 = sub2(pe23, mul2(d23, cp2));
    // Any non-finite p, v or psi reaches pe here; walls, damping and sources are finite.
    bad2 = __ffma2_rn(pe01, dup2(0.f), bad2);
    bad2 = __ffma2_rn(pe23, dup2(0.f), bad2);
    Pn[0] = pe01.x;
    Pn[1] = pe01.y;
    Pn[2] = pe23.x;
    Pn[3] = pe23.y;
    if (REC) {                                // p before the wall closed form, for the history
#pragma unroll
        for (int e = 0; e < kVec; e++) PT[e] = Pn[e];
    }
    if (WALLS && (col.wall_column || i == 0 || i == s.nx - 1)) {
        const float Po[kVec] = {P.x, P.y, P.z, P.w};
        column_walls(s, i, col.j, col.k0, real, [&](int e, float fu, float fp) {
#pragma unroll
            for (int q = 0; q < kVec; q++)
                if (q == e) Pn[q] = Pn[q] * fu - Po[q] * fp;
        });
    }
    if (LAYER) {
        if (fi_cell != 1.f) {
#pragma unroll
            for (int e = 0; e < kVec; e++) Pn[e] = Pn[e] * fi_cell;
        }
        if (col.damp_y) {
#pragma unroll
            for (int e = 0; e < kVec; e++) Pn[e] = Pn[e] * col.fj_cell;
        }
        if (col.damp_z) {
            Pn[0] = Pn[0] * col.fkc01.x;
            Pn[1] = Pn[1] * col.fkc01.y;
            Pn[2] = Pn[2] * col.fkc23.x;
            Pn[3] = Pn[3] * col.fkc23.y;
        }
    }
    if (tail) {                               // padding lanes keep p
        if (real <= 1) Pn[1] = P.y;
        if (real <= 2) Pn[2] = P.z;
        Pn[3] = P.w;
    }
    if (col.any_mine) add_sources(s, col.points, col.all_points, base, col.k0, step, Pn);
    o.XH01 = XH01; o.XH23 = XH23;
    o.YL01 = YL01; o.YL23 = YL23;
    o.YH01 = YH01; o.YH23 = YH23;
    o.ZL01 = ZL01; o.ZL23 = ZL23;
    o.ZH3 = ZH3;
}

// The stores of one chunk's step at plane i: p, the three lower faces, the far boundary faces
// and the relaxation states (to `psi`, n_relax fields of `field` elements). A slab's ghost planes
// get their p from the neighbours' sweeps, never from their own; its boundary planes also go to
// the neighbours' ghost planes (in their next copies).
template <int NR, bool ALIGNED>
__device__ __forceinline__ void lean_store(const LeanParams &g, const LeanColumn &col, int i,
                                           int64_t base, const float (&Pn)[kVec], float2 XL01,
                                           float2 XL23, const LeanFaces &o, float4 VZ,
                                           const float4 (&S)[NR > 0 ? NR : 1], float *psi) {
    const FusedParams<float> &f = g.f;
    const Room<float> &s = f.room;
    const float4 pn4 = make_float4(Pn[0], Pn[1], Pn[2], Pn[3]);
    if (i >= s.own_lo && i < s.own_hi) *reinterpret_cast<float4 *>(f.np + base) = pn4;
    if (s.ghost_lo != nullptr && i == s.own_lo) *reinterpret_cast<float4 *>(s.ghost_lo + col.column) = pn4;
    if (s.ghost_hi != nullptr && i == s.own_hi - 1) *reinterpret_cast<float4 *>(s.ghost_hi + col.column) = pn4;
    *reinterpret_cast<float4 *>(f.nvx + base) = make_float4(XL01.x, XL01.y, XL23.x, XL23.y);
    *reinterpret_cast<float4 *>(f.nvy + base) = make_float4(o.YL01.x, o.YL01.y, o.YL23.x, o.YL23.y);
    float4 ZS = make_float4(o.ZL01.x, o.ZL01.y, o.ZL23.x, o.ZL23.y);
    if (col.tail) {                           // faces past the top one are padding
        if (col.real <= 0) ZS.y = VZ.y;       // (never: real >= 1)
        if (col.real <= 1) ZS.z = VZ.z;
        if (col.real <= 2) ZS.w = VZ.w;
    }
    *reinterpret_cast<float4 *>(f.nvz + base) = ZS;
    if (i + 1 >= s.nx)
        *reinterpret_cast<float4 *>(f.nvx + base + s.plane) = make_float4(o.XH01.x, o.XH01.y, o.XH23.x, o.XH23.y);
    if (!col.y_hi)
        *reinterpret_cast<float4 *>(f.nvy + base + s.pz) = make_float4(o.YH01.x, o.YH01.y, o.YH23.x, o.YH23.y);
    if (!col.z_hi && (ALIGNED || !col.tail)) f.nvz[base + kVec] = o.ZH3;
#pragma unroll
    for (int r = 0; r < NR; r++) *reinterpret_cast<float4 *>(psi + r * s.field + base) = S[r];
}

// REC: also write the boundary history of the wall gradients (record_shell), as
// pressure_sweep_rec does.
template <bool LAYER, bool WALLS, int NR, bool ALIGNED = true, bool REC = false>
__device__ __forceinline__ void lean_column(const LeanParams &g, int i_begin, int i_end, int j, int c,
                                            int64_t step, const History<float> *hist = nullptr) {
    const Room<float> &s = g.f.room;
    const LeanColumn col = lean_setup<LAYER, ALIGNED>(s, j, c);
    const int64_t column = col.column;

    // Carried from plane to plane: p(i) and the updated vx on face i.
    float4 P;
    float2 XL01, XL23;
    float2 bad2 = dup2(0.f);   // NaN once a pressure this column produced is not finite
    {
        const int64_t base = (int64_t)i_begin * s.plane + column;
        P = __ldg(reinterpret_cast<const float4 *>(s.p + base));
        const float4 V = __ldg(reinterpret_cast<const float4 *>(s.vx + base));
        float4 Q = P;
        if (i_begin > 0) Q = __ldg(reinterpret_cast<const float4 *>(s.p + base - s.plane));
        lean_lower_face<LAYER>(g, col, i_begin, V, P, Q, XL01, XL23);
    }

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        const bool x_inner = i + 1 < s.nx;
        if (s.prefetch && i + 1 < i_end) {   // the next plane's own-row inputs into L2
            const int64_t next = base + s.plane;
            if (i + 2 < s.nx) prefetch_l2(s.p + next + s.plane);
            prefetch_l2(s.vx + next + s.plane);
            prefetch_l2(s.vy + next);
            prefetch_l2(s.vz + next);
#pragma unroll
            for (int r = 0; r < NR; r++) prefetch_l2(s.psi + r * s.field + next);
        }
        // ---- loads (all read-only: the next state goes to the other buffer)
        LeanInputs in;
        in.P = P;
        in.PX = in.PYm = in.PYp = P;
        if (x_inner) in.PX = __ldg(reinterpret_cast<const float4 *>(s.p + base + s.plane));
        in.VXo = __ldg(reinterpret_cast<const float4 *>(s.vx + base + s.plane));
        if (col.y_lo) in.PYm = __ldg(reinterpret_cast<const float4 *>(s.p + base - s.pz));
        if (col.y_hi) in.PYp = __ldg(reinterpret_cast<const float4 *>(s.p + base + s.pz));
        in.VY = __ldg(reinterpret_cast<const float4 *>(s.vy + base));
        in.VYp = __ldg(reinterpret_cast<const float4 *>(s.vy + base + s.pz));
        in.VZ = __ldg(reinterpret_cast<const float4 *>(s.vz + base));
        in.p_below = col.z_lo ? __ldg(s.p + base - 1) : 0.f;
        in.p_above = col.z_hi ? __ldg(s.p + base + kVec) : 0.f;
        // face k0 + 4: inside the row when k0 + 4 <= nz (always when ALIGNED)
        in.vz_above = (ALIGNED || !col.tail) ? __ldg(s.vz + base + kVec) : 0.f;
        float4 S[NR > 0 ? NR : 1];
#pragma unroll
        for (int r = 0; r < NR; r++) S[r] = *reinterpret_cast<const float4 *>(s.psi + r * s.field + base);

        LeanFaces o;
        float Pn[kVec], PT[kVec];
        lean_update<LAYER, WALLS, NR, ALIGNED, REC>(g, col, i, base, step, in, XL01, XL23, S, o, Pn,
                                                    bad2, PT);
        lean_store<NR, ALIGNED>(g, col, i, base, Pn, XL01, XL23, o, in.VZ, S, s.psi);
        if (col.any_mine) record_receivers(s, col.points, col.all_points, base, step, Pn);
        if (REC && hist->shell && (col.wall_column || i == 0 || i == s.nx - 1)) {
            const float Po[kVec] = {in.P.x, in.P.y, in.P.z, in.P.w};
            record_shell(s, *hist, i, j, col.k0, step, Po, PT);
        }
        XL01 = o.XH01;
        XL23 = o.XH23;
        P = in.PX;
    }
    report_nonfinite(s.status, bad2.x != bad2.x || bad2.y != bad2.y);
}

// Resident blocks of 256 threads: 80 registers (3 blocks) unless there is neither a layer nor a
// relaxation state (64 registers, 4 blocks); below 80 the relaxation states spill.
#ifndef ACF_LEAN_MIN_BLOCKS
#define ACF_LEAN_MIN_BLOCKS(LAYER, NR) ((LAYER) || (NR) > 0 ? 3 : 4)
#endif

template <bool LAYER, bool WALLS, int NR, bool ALIGNED>
__device__ __forceinline__ void lean_sweep_body(const LeanParams &g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= g.f.room.nchunks || j >= g.f.room.ny) return;
    const bool any_point = (g.f.room.n_src | g.f.room.n_rec) != 0;
    const int64_t step = any_point ? (*g.f.step_base + g.f.local_step) : 0;
    const int i_begin = blockIdx.z * g.f.planes;
    lean_column<LAYER, WALLS, NR, ALIGNED>(g, i_begin, min(g.f.room.nx, i_begin + g.f.planes), j, c, step);
}

template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, ACF_LEAN_MIN_BLOCKS(LAYER, NR)) lean_sweep(const LeanParams g) {
    lean_sweep_body<LAYER, WALLS, NR, true>(g);
}

// Rows with padding: the fix-ups keep a few more values live, so 96 registers (fewer spills).
template <bool LAYER, bool WALLS, int NR>
__global__ void __maxnreg__(96) lean_sweep_padded(const LeanParams g) {
    lean_sweep_body<LAYER, WALLS, NR, false>(g);
}

// The lean step of up to kMaxLeanParts slabs of one room in one launch (slab groups whose parts
// share a GPU): every part's step reads only its own current copy and writes only the next
// copies (its own, and its boundary planes into the neighbours' ghost planes), so the parts of
// one step are independent. blockIdx.z runs over the parts' groups of x planes in turn.
constexpr int kMaxLeanParts = 8;

struct LeanPartsParams {
    LeanParams part[kMaxLeanParts];
    int32_t first_group[kMaxLeanParts + 1];   // part p: blockIdx.z in [first_group[p], first_group[p + 1])
    int32_t n;
};

template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, ACF_LEAN_MIN_BLOCKS(LAYER, NR))
lean_parts_sweep(const __grid_constant__ LeanPartsParams q) {
    int p = 0;
    while (p + 1 < q.n && (int)blockIdx.z >= q.first_group[p + 1]) p++;
    const LeanParams &g = q.part[p];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= g.f.room.nchunks || j >= g.f.room.ny) return;
    const bool any_point = (g.f.room.n_src | g.f.room.n_rec) != 0;
    const int64_t step = any_point ? (*g.f.step_base + g.f.local_step) : 0;
    const int i_begin = ((int)blockIdx.z - q.first_group[p]) * g.f.planes;
    lean_column<LAYER, WALLS, NR, true>(g, i_begin, min(g.f.room.nx, i_begin + g.f.planes), j, c, step);
}

// The recorded forward step of the wall gradients in single precision (rooms with nz a multiple
// of 4): the lean step, also writing the boundary history.
struct LeanRecParams {
    LeanParams g;
    History<float> hist;
};

template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, ACF_LEAN_MIN_BLOCKS(LAYER, NR)) lean_sweep_rec(const LeanRecParams q) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= q.g.f.room.nchunks || j >= q.g.f.room.ny) return;
    const int64_t step = *q.g.f.step_base + q.g.f.local_step;
    const int i_begin = blockIdx.z * q.g.f.planes;
    lean_column<LAYER, WALLS, NR, true, true>(q.g, i_begin, min(q.g.f.room.nx, i_begin + q.g.f.planes), j,
                                              c, step, &q.hist);
}

// ------------------------------------------------------------------------------------------
// Two steps per launch: temporal blocking of the lean column (the step after the fused sweep
// that the reference's C backend names as its next one, c/acfdtd.c:12-14).
//
// One sweep reads the state of step n once and writes the state of step n + 2 once, so a cell
// moves (8 + 2R) elements per two steps instead of per step. Each thread marches its column
// through x and, at plane t, takes the first step at plane t and the second step at plane t - 1.
// The second step needs the first step's pressures of the four neighbouring columns at plane
// t - 1; every other input of it is the thread's own first-step result, kept in registers (the
// updated faces, which every cell computes for all six of its faces), or the relaxation states,
// parked in the output field (the only thread that touches that element is this one).
//
// The neighbours' first-step pressures travel through a ring of kPairRing x planes in global
// memory (L2-resident: four planes of the room per x group). A CTA publishes "first step done
// through plane t" with a release store after a block barrier; before its second step at plane
// t - 1, four threads of warp 0 acquire the four neighbour CTAs' counters (y -+ 1, z -+ 1).
// Counters only grow; the second step at t - 1 waits for plane t - 1 of the neighbours; the ring
// slot written at plane t was last read by the neighbours' second step at t - 4, which precedes
// their publication of plane t - 2, awaited at t - 1. So four slots suffice and no wait depends
// on a later plane. The launch is cooperative (every CTA resident), and every wait is bounded:
// one that runs out raises kStatusWaitTimeout in the room's status word and the thread stops
// waiting; the kernel returns.
//
// The x range is cut into groups of planes, as the lean sweep's is; a group also takes the
// first step at the plane before and the plane after its range (redundantly, without
// publishing it), so that groups never wait on one another. Inputs come only from the read copy
// of p and v and from the input relaxation states, outputs go only to the other copy and the
// output states, so the redundant planes read nothing another group writes.
//
// Every value is produced by the lean column's own update, in the same order: two launches of
// two steps equal four lean steps bit for bit.

constexpr int kPairRing = 4;
constexpr int kPairThreads = 128;

struct PairParams {
    LeanParams g;           // g.f.room: step n (p, v of the read copy; psi: the input states);
                            // g.f.np, nvx, nvy, nvz: the copy that receives step n + 2
    float *psi_out;         // relaxation states after the two steps
    float *ring;            // first-step p: groups x kPairRing planes of the room's geometry
    int32_t *progress;      // one counter per CTA, zero at launch
    uint64_t wait_limit_ns;
    // Test hook, neutral (-1) by default: the first CTA stops publishing from this plane on, so
    // that its neighbours' bounded waits run out and the kernel returns with kStatusWaitTimeout.
    int32_t stop_plane;
    int32_t reserved;
};

__device__ __forceinline__ int32_t load_acquire(const int32_t *p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void store_release(int32_t *p, int32_t v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait for a counter to reach `target`: false when it did not within `limit_ns` nor
// within kWaitLimitIterations polls.
__device__ __forceinline__ bool wait_counter(const int32_t *counter, int32_t target, uint64_t limit_ns) {
    if (load_acquire(counter) >= target) return true;
    const uint64_t start = global_ns();
    for (int it = 0; it < kWaitLimitIterations; it++) {
        __nanosleep(32);
        if (load_acquire(counter) >= target) return true;
        if (global_ns() - start > limit_ns) return false;
    }
    return false;
}

__device__ __forceinline__ float4 f4(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }

template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(kPairThreads, 4) lean_pair_sweep(const PairParams q) {
    const LeanParams &g = q.g;
    const Room<float> &s = g.f.room;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = c < s.nchunks && j < s.ny;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int s0 = blockIdx.z * g.f.planes;              // second step: planes [s0, e0)
    const int e0 = min(s.nx, s0 + g.f.planes);
    const int a_lo = max(0, s0 - 1), a_hi = min(s.nx, e0 + 1);   // first step: [a_lo, a_hi)
    float *ring = q.ring + (int64_t)blockIdx.z * kPairRing * s.plane;
    const int cta = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    int watch = -1;                                      // the neighbour CTA this thread watches
    if (tid == 0 && blockIdx.y > 0) watch = cta - (int)gridDim.x;
    if (tid == 1 && blockIdx.y + 1 < gridDim.y) watch = cta + (int)gridDim.x;
    if (tid == 2 && blockIdx.x > 0) watch = cta - 1;
    if (tid == 3 && blockIdx.x + 1 < gridDim.x) watch = cta + 1;
    bool waiting = watch >= 0;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    const int64_t step = any_point ? (*g.f.step_base + g.f.local_step) : 0;

    LeanColumn col{};
    float4 P = make_float4(0.f, 0.f, 0.f, 0.f);          // p^n at plane t
    float4 PA = P;                                       // p^{n+1} at plane t - 1
    float2 XA01 = dup2(0.f), XA23 = XA01;                // v^{n+1/2} on the x face below plane t
    float2 XB01 = XA01, XB23 = XA01;                     // v^{n+3/2} on the x face below plane t - 1
    LeanFaces A{};                                       // the first step's faces at plane t - 1
    float2 bad2 = dup2(0.f);
    if (active) {
        col = lean_setup<LAYER, true>(s, j, c);
        const int64_t base = (int64_t)a_lo * s.plane + col.column;
        P = __ldg(reinterpret_cast<const float4 *>(s.p + base));
        const float4 V = __ldg(reinterpret_cast<const float4 *>(s.vx + base));
        float4 Q = P;
        if (a_lo > 0) Q = __ldg(reinterpret_cast<const float4 *>(s.p + base - s.plane));
        lean_lower_face<LAYER>(g, col, a_lo, V, P, Q, XA01, XA23);
    }

    for (int t = a_lo; t <= e0; t++) {
        const bool first = t < a_hi, second = t - 1 >= s0;
        // (1) the neighbours' first step through plane t - 1
        if (second && waiting && !wait_counter(q.progress + watch, t, q.wait_limit_ns)) {
            atomicOr(s.status, kStatusWaitTimeout);
            waiting = false;
        }
        // (2) the first step at plane t
        const float2 XO01 = XA01, XO23 = XA23;           // v^{n+1/2} below plane t
        float4 PN = P;                                   // p^{n+1} at plane t
        LeanFaces An{};
        if (active && first) {
            const int64_t base = (int64_t)t * s.plane + col.column;
            const bool x_inner = t + 1 < s.nx;
            if (s.prefetch && t + 1 < a_hi) {
                const int64_t next = base + s.plane;
                if (t + 2 < s.nx) prefetch_l2(s.p + next + s.plane);
                prefetch_l2(s.vx + next + s.plane);
                prefetch_l2(s.vy + next);
                prefetch_l2(s.vz + next);
#pragma unroll
                for (int r = 0; r < NR; r++) prefetch_l2(s.psi + r * s.field + next);
            }
            LeanInputs in;
            in.P = P;
            in.PX = in.PYm = in.PYp = P;
            if (x_inner) in.PX = __ldg(reinterpret_cast<const float4 *>(s.p + base + s.plane));
            in.VXo = __ldg(reinterpret_cast<const float4 *>(s.vx + base + s.plane));
            if (col.y_lo) in.PYm = __ldg(reinterpret_cast<const float4 *>(s.p + base - s.pz));
            if (col.y_hi) in.PYp = __ldg(reinterpret_cast<const float4 *>(s.p + base + s.pz));
            in.VY = __ldg(reinterpret_cast<const float4 *>(s.vy + base));
            in.VYp = __ldg(reinterpret_cast<const float4 *>(s.vy + base + s.pz));
            in.VZ = __ldg(reinterpret_cast<const float4 *>(s.vz + base));
            in.p_below = col.z_lo ? __ldg(s.p + base - 1) : 0.f;
            in.p_above = col.z_hi ? __ldg(s.p + base + kVec) : 0.f;
            in.vz_above = __ldg(s.vz + base + kVec);
            float4 S[NR > 0 ? NR : 1];
#pragma unroll
            for (int r = 0; r < NR; r++) S[r] = __ldg(reinterpret_cast<const float4 *>(s.psi + r * s.field + base));
            float Pn[kVec];
            lean_update<LAYER, WALLS, NR, true>(g, col, t, base, step, in, XA01, XA23, S, An, Pn, bad2);
            PN = make_float4(Pn[0], Pn[1], Pn[2], Pn[3]);
            if (t >= s0 && t < e0) {                     // planes the second step visits
                __stcg(reinterpret_cast<float4 *>(ring + (t % kPairRing) * s.plane + col.column), PN);
#pragma unroll
                for (int r = 0; r < NR; r++)
                    *reinterpret_cast<float4 *>(q.psi_out + r * s.field + base) = S[r];
                if (col.any_mine) record_receivers(s, col.points, col.all_points, base, step, Pn);
            }
            if (t == s0)                                 // the second step's x face below s0
                lean_lower_face<LAYER>(g, col, s0, f4(XO01, XO23), PN, PA, XB01, XB23);
            XA01 = An.XH01;
            XA23 = An.XH23;
            P = in.PX;
        }
        __syncthreads();
        if (tid == 0 && first && !(cta == 0 && q.stop_plane >= 0 && t >= q.stop_plane)) {
            __threadfence();
            store_release(q.progress + cta, t + 1);
        }
        // (3) the second step at plane t - 1
        if (active && second) {
            const int i = t - 1;
            const int64_t base = (int64_t)i * s.plane + col.column;
            const float *slot = ring + (i % kPairRing) * s.plane + col.column;
            LeanInputs in;
            in.P = PA;
            in.PX = i + 1 < s.nx ? PN : PA;
            in.PYm = col.y_lo ? __ldcg(reinterpret_cast<const float4 *>(slot - s.pz)) : PA;
            in.PYp = col.y_hi ? __ldcg(reinterpret_cast<const float4 *>(slot + s.pz)) : PA;
            in.VXo = f4(XO01, XO23);
            in.VY = f4(A.YL01, A.YL23);
            in.VYp = f4(A.YH01, A.YH23);
            in.VZ = f4(A.ZL01, A.ZL23);
            in.p_below = col.z_lo ? __ldcg(slot - 1) : 0.f;
            in.p_above = col.z_hi ? __ldcg(slot + kVec) : 0.f;
            in.vz_above = A.ZH3;
            float4 S[NR > 0 ? NR : 1];
#pragma unroll
            for (int r = 0; r < NR; r++) S[r] = *reinterpret_cast<const float4 *>(q.psi_out + r * s.field + base);
            LeanFaces B;
            float Pn[kVec];
            lean_update<LAYER, WALLS, NR, true>(g, col, i, base, step + 1, in, XB01, XB23, S, B, Pn, bad2);
            lean_store<NR, true>(g, col, i, base, Pn, XB01, XB23, B, in.VZ, S, q.psi_out);
            if (col.any_mine) record_receivers(s, col.points, col.all_points, base, step + 1, Pn);
            XB01 = B.XH01;
            XB23 = B.XH23;
        }
        A = An;
        PA = PN;
    }
    report_nonfinite(s.status, bad2.x != bad2.x || bad2.y != bad2.y);
}

// ------------------------------------------------------------------------------------------
// The pressure-only scheme: the second-order wave equation on p alone, two fields instead of
// 4 + R (the scheme the reference plans as its milestone M8, PLAN.md:52-56, and has not built).
//
// Eliminating v from the staggered pair gives, exactly in real arithmetic, for a room with
// rigid or impedance walls and no sponge or air (a = sum over the cell's absorbing faces of
// c dt xi / (2 dx), a = 0 inside; fu = 1/(1+a), fp = a/(1+a) the wall pair of the p-v scheme):
//
//   p^{n+1} = fu (2 p^n + lam2 L p^n) - (fu - fp) p^{n-1} - S^{n-1} + S^n,   lam2 = c_p c_v
//
// where L p = sum over the cell's interior neighbours of (p_nb - p) (the rigid-face Neumann
// Laplacian: the p-v update never moves a boundary face) and S^n is the volume source added
// after step n. The first step after entering the scheme takes the p-v step itself from
// (p^n, v^{n-1/2}), with the velocities folded in:
//
//   p^{n+1} = fu (p^n - c_p D(v^{n-1/2}) + lam2 L p^n) - fp p^n + S^n
//
// (D the divergence over all faces, as the pressure sweep forms it), so the pressures equal the
// p-v scheme's to rounding from then on; boundary faces keep their velocity in both schemes.
// Per cell and step it reads p^n and p^{n-1} and writes p^{n+1} over p^{n-1}: 3 elements.

template <typename T>
struct PressureOnlyParams {
    Room<T> room;       // geometry, wall pairs, points, status; p, v: the current copy
    const T *cur;       // p^n
    T *next;            // p^{n-1} on entry (not read by the first step), p^{n+1} on exit
    T lam2;             // c_p c_v = (c dt / dx)^2, rounded once from FP64
    const int64_t *step_base;
    int32_t local_step;
    int32_t planes;
};

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c) {
    if constexpr (sizeof(T) == 4) return __fmaf_rn(a, b, c);
    else return __fma_rn(a, b, c);
}

template <typename T, bool WALLS, bool FIRST>
__device__ __forceinline__ void pressure_only_column_simple(const PressureOnlyParams<T> &g, int i_begin,
                                                     int i_end, int j, int c, int64_t step) {
    const Room<T> &s = g.room;
    const int k0 = c * kVec;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool y_lo = j > 0, y_hi = j + 1 < s.ny;
    const bool z_lo = k0 > 0, z_hi = k0 + kVec < s.nz;
    const bool wall_column = !y_lo || !y_hi || !z_lo || k0 + kVec >= s.nz;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    bool all_points = false;
    const uint32_t points = any_point ? column_points(s, j, k0, all_points) : 0u;
    const bool any_mine = points != 0 || all_points;
    const T lam2 = g.lam2, cp = s.cp;
    T bad = T(0);

    T Pm[kVec], P[kVec];
    Vec4<T>::ldg(g.cur + (int64_t)i_begin * s.plane + column, P);
    if (i_begin > 0) Vec4<T>::ldg(g.cur + (int64_t)(i_begin - 1) * s.plane + column, Pm);
    else {
#pragma unroll
        for (int e = 0; e < kVec; e++) Pm[e] = P[e];
    }

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        const bool x_hi = i + 1 < s.nx;
        if (s.prefetch && i + 1 < i_end) {   // the next plane's own-row inputs into L2
            if (i + 2 < s.nx) prefetch_l2(g.cur + base + 2 * s.plane);
            if (!FIRST) prefetch_l2(g.next + base + s.plane);
        }
        T Pp[kVec], Ym[kVec], Yp[kVec], Q[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) Pp[e] = Ym[e] = Yp[e] = Q[e] = P[e];
        if (x_hi) Vec4<T>::ldg(g.cur + base + s.plane, Pp);
        if (y_lo) Vec4<T>::ldg(g.cur + base - s.pz, Ym);
        if (y_hi) Vec4<T>::ldg(g.cur + base + s.pz, Yp);
        const T zb = z_lo ? __ldg(g.cur + base - 1) : P[0];
        const T za = z_hi ? __ldg(g.cur + base + kVec) : P[kVec - 1];
        T D[kVec];
        if constexpr (FIRST) {
            T XL[kVec], XH[kVec], YL[kVec], YH[kVec], Z[kVec];
            Vec4<T>::ldg(s.vx + base, XL);
            Vec4<T>::ldg(s.vx + base + s.plane, XH);
            Vec4<T>::ldg(s.vy + base, YL);
            Vec4<T>::ldg(s.vy + base + s.pz, YH);
            Vec4<T>::ldg(s.vz + base, Z);
            const T above = k0 + kVec <= s.nz ? __ldg(s.vz + base + kVec) : T(0);
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                D[e] = XH[e] - XL[e];
                D[e] = D[e] + (YH[e] - YL[e]);
                D[e] = D[e] + ((e + 1 < kVec ? Z[e + 1] : above) - Z[e]);
            }
        } else {
            Vec4<T>::load(g.next + base, Q);     // p^{n-1}: read, then overwritten by p^{n+1}
        }

        T Pn[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            const T p = P[e];
            if (k >= s.nz) {          // padding
                Pn[e] = p;
                continue;
            }
            const T zm = e == 0 ? zb : P[e - 1];
            const T zp = k + 1 < s.nz ? (e + 1 < kVec ? P[e + 1] : za) : p;
            const T lap = ((Pm[e] - p) + (Pp[e] - p)) + ((Ym[e] - p) + (Yp[e] - p)) + ((zm - p) + (zp - p));
            T fu = T(1), fp = T(0);
            const bool wall = WALLS && (wall_column || i == 0 || i == s.nx - 1) &&
                              wall_pair(s, i, j, k, fu, fp);
            T pn;
            if constexpr (FIRST) {
                const T t = fma_t(lam2, lap, fma_t(-cp, D[e], p));
                pn = wall ? fu * t - fp * p : t;
            } else {
                const T q = fma_t(lam2, lap, p + p);
                pn = wall ? fu * q - (fu - fp) * Q[e] : q - Q[e];
            }
            Pn[e] = pn;
        }
        if (any_mine) {
            // - S^{n-1} (added by the previous step), then + S^n, in the order added
            uint32_t m = all_points ? 0u : source_bits(points, s.n_src);
            for (int q = all_points ? 0 : -1; all_points ? q < s.n_src : m != 0; q++) {
                if (!all_points) {
                    q = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.src_off[q] - base;
                if (d < 0 || d >= kVec || k0 + d >= s.nz) continue;
#pragma unroll
                for (int e = 0; e < kVec; e++) {
                    if (e != d) continue;
                    if (!FIRST && step >= 1 && step - 1 < s.src_len[q])
                        Pn[e] = Pn[e] - s.cs * s.src_sig[q * s.src_stride + step - 1];
                    if (step < s.src_len[q]) Pn[e] = Pn[e] + s.cs * s.src_sig[q * s.src_stride + step];
                }
            }
        }
#pragma unroll
        for (int e = 0; e < kVec; e++) bad = finite_acc(bad, Pn[e]);
        Vec4<T>::store(g.next + base, Pn);
        if (any_mine) record_receivers(s, points, all_points, base, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            Pm[e] = P[e];
            P[e] = Pp[e];
        }
    }
    report_nonfinite(s.status, bad != bad);
}


// The steady-state step, lean in instructions. The Laplacian is formed as the neighbour sum
// minus 6p (a neighbour missing at a rigid face is replaced by p, which is the same Neumann
// operator), and 2 p + lam2 L p as (2 - 6 lam2) p + lam2 (neighbour sum): two fused
// multiply-adds per cell after five additions. The pressures then differ from the p-v scheme's
// by rounding only, like the first form. ALIGNED: nz is a multiple of 4 (no padding lanes).
template <typename T, bool WALLS, bool ALIGNED>
__device__ __forceinline__ void pressure_only_column(const PressureOnlyParams<T> &g, int i_begin,
                                                     int i_end, int j, int c, int64_t step) {
    const Room<T> &s = g.room;
    const T *__restrict__ cur = g.cur;
    T *__restrict__ nxt = g.next;
    const int k0 = c * kVec;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool y_lo = j > 0, y_hi = j + 1 < s.ny;
    const bool z_lo = k0 > 0, z_hi = k0 + kVec < s.nz;
    const bool wall_column = !y_lo || !y_hi || !z_lo || k0 + kVec >= s.nz;
    const int real = ALIGNED ? kVec : min(kVec, s.nz - k0);   // cells of the chunk in the room
    const bool any_point = (s.n_src | s.n_rec) != 0;
    bool all_points = false;
    const uint32_t points = any_point ? column_points(s, j, k0, all_points) : 0u;
    const bool any_mine = points != 0 || all_points;
    const T lam2 = g.lam2, centre = T(2) - T(6) * g.lam2;
    T bad = T(0);

    T Pm[kVec], P[kVec];
    Vec4<T>::ldg(cur + (int64_t)i_begin * s.plane + column, P);
    if (i_begin > 0) Vec4<T>::ldg(cur + (int64_t)(i_begin - 1) * s.plane + column, Pm);
    else {
#pragma unroll
        for (int e = 0; e < kVec; e++) Pm[e] = P[e];
    }

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        if (s.prefetch && i + 1 < i_end) {   // the next plane's own-row inputs into L2
            if (i + 2 < s.nx) prefetch_l2(cur + base + 2 * s.plane);
            prefetch_l2(nxt + base + s.plane);
        }
        T Pp[kVec], Ym[kVec], Yp[kVec], Q[kVec];
        if (i + 1 < s.nx) Vec4<T>::ldg(cur + base + s.plane, Pp);
        else {
#pragma unroll
            for (int e = 0; e < kVec; e++) Pp[e] = P[e];
        }
        if (y_lo) Vec4<T>::ldg(cur + base - s.pz, Ym);
        else {
#pragma unroll
            for (int e = 0; e < kVec; e++) Ym[e] = P[e];
        }
        if (y_hi) Vec4<T>::ldg(cur + base + s.pz, Yp);
        else {
#pragma unroll
            for (int e = 0; e < kVec; e++) Yp[e] = P[e];
        }
        const T zb = z_lo ? __ldg(cur + base - 1) : P[0];
        T za = z_hi ? __ldg(cur + base + kVec) : P[kVec - 1];
        Vec4<T>::load(nxt + base, Q);

        T Pn[kVec];
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            T zp = e + 1 < kVec ? P[e + 1] : za;
            if (!ALIGNED && real < kVec && e + 1 == real) zp = P[e];   // top cell, padded row
            const T zm = e == 0 ? zb : P[e - 1];
            const T sum = ((Pm[e] + Pp[e]) + (Ym[e] + Yp[e])) + (zm + zp);
            Pn[e] = fma_t(lam2, sum, fma_t(centre, P[e], -Q[e]));
        }
        if (WALLS && (wall_column || i == 0 || i == s.nx - 1)) {
            column_walls(s, i, j, k0, real, [&](int e, T fu, T fp) {
#pragma unroll
                for (int q = 0; q < kVec; q++)
                    if (q == e) {
                        const T two_p = Pn[q] + Q[q];      // 2 p + lam2 L p, back from Pn
                        Pn[q] = fu * two_p - (fu - fp) * Q[q];
                    }
            });
        }
        if (!ALIGNED) {
#pragma unroll
            for (int e = 0; e < kVec; e++)
                if (e >= real) Pn[e] = P[e];               // padding lanes keep their value
        }
        if (any_mine) {
            // - S^{n-1} (added by the previous step), then + S^n, in the order added
            uint32_t m = all_points ? 0u : source_bits(points, s.n_src);
            for (int q = all_points ? 0 : -1; all_points ? q < s.n_src : m != 0; q++) {
                if (!all_points) {
                    q = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.src_off[q] - base;
                if (d < 0 || d >= kVec || k0 + d >= s.nz) continue;
#pragma unroll
                for (int e = 0; e < kVec; e++) {
                    if (e != d) continue;
                    if (step >= 1 && step - 1 < s.src_len[q])
                        Pn[e] = Pn[e] - s.cs * s.src_sig[q * s.src_stride + step - 1];
                    if (step < s.src_len[q]) Pn[e] = Pn[e] + s.cs * s.src_sig[q * s.src_stride + step];
                }
            }
        }
#pragma unroll
        for (int e = 0; e < kVec; e++) bad = finite_acc(bad, Pn[e]);
        Vec4<T>::store(nxt + base, Pn);
        if (any_mine) record_receivers(s, points, all_points, base, step, Pn);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            Pm[e] = P[e];
            P[e] = Pp[e];
        }
    }
    report_nonfinite(s.status, bad != bad);
}

// FIRST: the step from the p-v state; otherwise the steady-state step, ALIGNED or padded.
template <typename T, bool WALLS, bool FIRST, bool ALIGNED = false>
__global__ void __launch_bounds__(256) pressure_only_sweep(const PressureOnlyParams<T> g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= g.room.nchunks || j >= g.room.ny) return;
    const bool any_point = (g.room.n_src | g.room.n_rec) != 0;
    const int64_t step = any_point ? (*g.step_base + g.local_step) : 0;
    const int i_begin = blockIdx.z * g.planes;
    if constexpr (FIRST)
        pressure_only_column_simple<T, WALLS, true>(g, i_begin, min(g.room.nx, i_begin + g.planes), j, c, step);
    else
        pressure_only_column<T, WALLS, ALIGNED>(g, i_begin, min(g.room.nx, i_begin + g.planes), j, c, step);
}

// The two sums of the pressure-only scheme's conserved energy after a step, with cur = p^{n+1}
// and prev = p^n: terms 0 and 1 of `partials` hold sum (cur - prev)^2 and sum cur L prev (L the
// Neumann Laplacian of the scheme); the other five are zero. Layout as energy_partials.
template <typename T>
__global__ void __launch_bounds__(256) pressure_only_energy_partials(const Room<T> s, const T *cur,
                                                                     const T *prev, double *partials) {
    double a = 0.0, b = 0.0;
    const int64_t total = (int64_t)s.nx * s.ny * s.nz;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < total;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(n % s.nz);
        const int64_t row = n / s.nz;
        const int j = (int)(row % s.ny);
        const int i = (int)(row / s.ny);
        const int64_t o = (int64_t)i * s.plane + (int64_t)j * s.pz + k;
        const double u = (double)cur[o], v = (double)prev[o];
        a += (u - v) * (u - v);
        double lap = 0.0;
        if (i > 0) lap += (double)prev[o - s.plane] - v;
        if (i + 1 < s.nx) lap += (double)prev[o + s.plane] - v;
        if (j > 0) lap += (double)prev[o - s.pz] - v;
        if (j + 1 < s.ny) lap += (double)prev[o + s.pz] - v;
        if (k > 0) lap += (double)prev[o - 1] - v;
        if (k + 1 < s.nz) lap += (double)prev[o + 1] - v;
        b += u * lap;
    }
    __shared__ double red[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 16; d > 0; d >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, d);
        b += __shfl_down_sync(0xffffffffu, b, d);
    }
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x < kEnergyTerms) {
        double v = 0.0;
        if (threadIdx.x < 2)
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
        partials[blockIdx.x * kEnergyTerms + threadIdx.x] = v;
    }
}

// ------------------------------------------------------------------------------------------
// One room: 2D grid of (chunk, row) threads; blockIdx.z selects a group of `planes` x planes.

template <typename T, bool LAYER>
__global__ void __launch_bounds__(256) velocity_sweep(const StepParams<T> p) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= p.room.nchunks || j >= p.room.ny) return;
    const int i_begin = blockIdx.z * p.planes;
    velocity_column<T, LAYER>(p.room, i_begin, min(p.room.nx, i_begin + p.planes), j, c);
}

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 2 : 4)) pressure_sweep(const StepParams<T> p) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= p.room.nchunks || j >= p.room.ny) return;
    const bool any_point = (p.room.n_src | p.room.n_rec) != 0;
    const int64_t step = any_point ? (*p.step_base + p.local_step) : 0;
    const int first = blockIdx.z * p.planes;
    const int i_begin = max(first, p.room.own_lo);
    const int i_end = min(min(p.room.nx, first + p.planes), p.room.own_hi);
    if (i_begin >= i_end) return;   // planes outside a slab's own range (its ghost planes)
    pressure_column<T, LAYER, WALLS, NR>(p.room, i_begin, i_end, j, c, step);
}

// The same pressure sweep, also writing the forward history the adjoint needs.
template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 2 : 3)) pressure_sweep_rec(const StepParams<T> p) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= p.room.nchunks || j >= p.room.ny) return;
    const int64_t step = *p.step_base + p.local_step;
    const int i_begin = blockIdx.z * p.planes;
    pressure_column<T, LAYER, WALLS, NR, true>(p.room, i_begin, min(p.room.nx, i_begin + p.planes),
                                               j, c, step, &p.hist);
}

// ------------------------------------------------------------------------------------------
// Batches: a persistent grid walks the tile table with a static stride; no CTA waits on any
// other. A CTA copies the description of its tile's room into shared memory when the room
// changes (every thread takes part in the copy and both barriers, so they stay uniform).

template <typename T>
__device__ __forceinline__ void stage_room(const Room<T> *src, Room<T> *dst) {
    static_assert(sizeof(Room<T>) % sizeof(int) == 0, "Room must be a whole number of words");
    const int *from = reinterpret_cast<const int *>(src);
    int *to = reinterpret_cast<int *>(dst);
    for (int w = threadIdx.x; w < (int)(sizeof(Room<T>) / sizeof(int)); w += blockDim.x)
        to[w] = __ldg(from + w);
}

template <typename T, bool LAYER>
__global__ void __launch_bounds__(256) velocity_batch(const BatchParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(Room<T>)];
    Room<T> *room = reinterpret_cast<Room<T> *>(raw);
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_room(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            velocity_column<T, LAYER>(*room, tile.i_begin, tile.i_end, pair / room->nchunks,
                                      pair % room->nchunks);
        }
    }
}

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 2 : 3)) pressure_batch(const BatchParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(Room<T>)];
    Room<T> *room = reinterpret_cast<Room<T> *>(raw);
    const int64_t step = *b.step_base + b.local_step;
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_room(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            pressure_column<T, LAYER, WALLS, NR>(*room, tile.i_begin, tile.i_end,
                                                 pair / room->nchunks, pair % room->nchunks,
                                                 step);
        }
    }
}

// (a)+(b) over a batch: the fused step (fused_column) on the same tile table, each CTA staging
// the fused parameters of its tile's room -- the room description with the current p and v and
// the next copy to write -- for the parity all rooms are at.
template <typename T>
struct FusedBatchParams {
    const FusedParams<T> *rooms;   // one per room, for the current parity
    const Tile *tiles;
    int32_t n_tiles;
    int32_t local_step;
    const int64_t *step_base;
};

// 96 registers (fp32): measured best on 64 uneven rooms against 80 (spills) and 128 (fewer warps).
template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __maxnreg__(sizeof(T) == 8 ? 168 : 96) fused_batch(const FusedBatchParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(FusedParams<T>)];
    FusedParams<T> *room = reinterpret_cast<FusedParams<T> *>(raw);
    static_assert(sizeof(FusedParams<T>) % sizeof(int) == 0, "FusedParams must be a whole number of words");
    const int64_t step = *b.step_base + b.local_step;
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            const int *from = reinterpret_cast<const int *>(b.rooms + tile.room);
            int *to = reinterpret_cast<int *>(raw);
            for (int w = threadIdx.x; w < (int)(sizeof(FusedParams<T>) / sizeof(int)); w += blockDim.x)
                to[w] = __ldg(from + w);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            fused_column<T, LAYER, WALLS, NR>(*room, tile.i_begin, tile.i_end, pair / room->room.nchunks,
                                              pair % room->room.nchunks, step);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Adjoint: the transposed leapfrog, run backward in time (single rooms).
//
// The step is linear in the state x^n = (p^n, v^{n-1/2}, psi^n), so the adjoint recursion
// lambda^n = A^T lambda^{n+1} needs no forward state; only parameter gradients read the forward
// history. With mu the adjoint of the damped, gradient-updated face velocity and lambda_D the
// adjoint of the divergence, the reverse of forward step n is two sweeps mirroring the forward:
//
//   cells: lp  = LP + c_v div_interior(mu^{n+1}) + dL/drec[n] (receiver cells)
//          lp_hat = h lp ; lp_tilde = u lp_hat ; LP <- lp_tilde - q lp_hat        (walls: u, q)
//          lambda_D = (S - c_p) lp_tilde + sum_r G_r ((1 - delta_r) lpsi_r - m_r lp_tilde)
//          LPSI_r <- delta_r lpsi_r + m_r lp_tilde
//          dL/dsignal_s[n] = c_s lp (source cells); dL/da (walls), dL/d(G, m, delta, S) (air)
//   faces: mu_f = g_f (LV_f + lambda_D[lower cell] - lambda_D[upper cell]) -> LV
//
// where u = 1/(1+a), q = a/(1+a), h and g the layer products, S = dt sum G. The gradient of the
// wall closed form p_hat = u p_tilde - q p with respect to a is -u^2 (p_tilde + p).

template <typename T>
struct AdjointParams {
    Room<T> room;                  // coefficients, geometry, profiles, walls, points
    T *lp, *lvx, *lvy, *lvz, *lpsi, *ld;  // adjoint fields (room geometry)
    const double *grad_rec;        // n_rec rows of grad_stride, column = step - grad_step0
    double *grad_src;              // n_src rows of grad_stride
    int64_t grad_stride, grad_step0;
    History<T> hist;
    double *grad_shell;            // FP64 dL/da per boundary cell (shell index)
    double *air_partials;          // per block: G_r (R), m_r (R), delta_r (R), S
    const int64_t *step_base;      // the forward step reversed is *step_base + local_step
    int32_t local_step;
    int32_t planes;
    int32_t air;                   // accumulate air gradients (needs hist.fields)
    // Fused adjoint step only: mu^{n+1} and lambda_D^n go to these (the other copies); lvx..lvz
    // hold mu^{n+2} and ld holds lambda_D^{n+1}.
    T *out_vx, *out_vy, *out_vz, *out_d;
};

// mu on a face: (LV + (lambda_D[lower cell] - lambda_D[upper cell])) g_a g_b g_c, the face
// sweep's arithmetic, with lambda_D = 0 outside the room (x - 0 == x exactly, so the far faces'
// LV + lambda_D[lower] is reproduced bit for bit).
template <typename T, bool LAYER>
__device__ __forceinline__ T adjoint_face(T lv, T d_lower, T d_upper, T ga, T gb, T gc) {
    T m = lv + (d_lower - d_upper);
    if (LAYER) m = ((m * ga) * gb) * gc;
    return m;
}

// One (row j, chunk c) column of the adjoint pressure sweep over planes [i_begin, i_end),
// reversing forward step `step`; air-gradient terms are added to `air_acc`.
//
// FUSED also performs the face sweep of the step after (forward step + 1) first: mu^{n+1} on the
// cell's six faces from mu^{n+2} (lvx..lvz) and lambda_D^{n+1} (ld) -- its own three lower faces
// (stored, with the far boundary faces) and its three upper faces (recomputed exactly as their
// owners compute them) -- and writes lambda_D^n to out_d. Per cell and step this moves (10 + 2R)
// elements instead of the two sweeps' (13 + 2R), with the same results.
template <typename T, bool LAYER, bool WALLS, int NR, bool AIR, bool FUSED = false, int VW = kVec>
__device__ __forceinline__ void adjoint_pressure_column(const AdjointParams<T> &a, int i_begin,
                                                        int i_end, int j, int c, int64_t step,
                                                        T *air_acc) {
    const Room<T> &s = a.room;
    const int k0 = c * VW;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool has_above = k0 + VW <= s.nz;
    const T scp = s.relax_scale - s.cp;
    bool all_points = false;
    const uint32_t points = (s.n_src | s.n_rec) != 0 ? column_points(s, j, k0, all_points, VW) : 0u;
    const bool any_mine = points != 0 || all_points;
    const bool wall_column = j == 0 || j == s.ny - 1 || k0 == 0 || k0 + VW >= s.nz;
    T XL[VW];
    // FUSED: lambda_D^{n+1} of the current cell and of the cell below in x, carried along x
    T Dc[VW], Dm[VW];
    T fj_cell = T(1), fj_face = T(1), fj1_face = T(1);
    if (FUSED) {
        const int64_t b0 = (int64_t)i_begin * s.plane + column;
        VecW<T, VW>::ldg(a.ld + b0, Dc);
#pragma unroll
        for (int e = 0; e < VW; e++) Dm[e] = T(0);
        if (i_begin > 0) VecW<T, VW>::ldg(a.ld + b0 - s.plane, Dm);
        if (LAYER) {
            fj_cell = __ldg(s.cell[1] + j);
            fj_face = __ldg(s.face[1] + j);
            fj1_face = __ldg(s.face[1] + j + 1);
        }
        T V[VW];
        VecW<T, VW>::ldg(a.lvx + b0, V);
        const T fi_face = LAYER ? __ldg(s.face[0] + i_begin) : T(1);
#pragma unroll
        for (int e = 0; e < VW; e++)
            XL[e] = k0 + e < s.nz ? adjoint_face<T, LAYER>(V[e], Dm[e], Dc[e], fi_face, fj_cell,
                                                           LAYER ? __ldg(s.cell[2] + k0 + e) : T(1))
                                  : V[e];
    } else {
        VecW<T, VW>::ldg(a.lvx + (int64_t)i_begin * s.plane + column, XL);
    }
    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        if (s.prefetch && i + 1 < i_end) {  // the next plane's own-row inputs into L2
            const int64_t next = base + s.plane;
            if (FUSED && i + 2 < s.nx) prefetch_l2(a.ld + next + s.plane);
            prefetch_l2(a.lvx + next + s.plane);
            prefetch_l2(a.lvy + next);
            prefetch_l2(a.lvz + next);
            prefetch_l2(a.lp + next);
#pragma unroll
            for (int r = 0; r < NR; r++) prefetch_l2(a.lpsi + r * s.field + next);
            if (AIR && NR > 0) {
                const int64_t slot = (step - a.hist.fields_step0) % a.hist.fields_slots;
                const T *h = a.hist.fields + slot * (1 + NR) * s.field + next;
#pragma unroll
                for (int r = 0; r <= NR; r++) prefetch_l2(h + r * s.field);
            }
        }
        T XH[VW], YL[VW], YH[VW], Z[VW], L[VW], LS[NR > 0 ? NR : 1][VW];
        T above;
        T Dxp[VW];   // FUSED: lambda_D^{n+1} of the next plane
        if (FUSED) {
            T Dy[VW], Dyp[VW], VXp[VW], VY[VW], VYp[VW], VZ[VW];
#pragma unroll
            for (int e = 0; e < VW; e++) {
                Dxp[e] = T(0);
                Dy[e] = T(0);
                Dyp[e] = T(0);
            }
            if (i + 1 < s.nx) VecW<T, VW>::ldg(a.ld + base + s.plane, Dxp);
            if (j > 0) VecW<T, VW>::ldg(a.ld + base - s.pz, Dy);
            if (j + 1 < s.ny) VecW<T, VW>::ldg(a.ld + base + s.pz, Dyp);
            const T d_below = k0 > 0 ? __ldg(a.ld + base - 1) : T(0);
            const T d_above = k0 + VW < s.nz ? __ldg(a.ld + base + VW) : T(0);
            VecW<T, VW>::ldg(a.lvx + base + s.plane, VXp);
            VecW<T, VW>::ldg(a.lvy + base, VY);
            VecW<T, VW>::ldg(a.lvy + base + s.pz, VYp);
            VecW<T, VW>::ldg(a.lvz + base, VZ);
            const T vz_above = has_above ? __ldg(a.lvz + base + VW) : T(0);
            T fi_cell = T(1), fi1_face = T(1);
            if (LAYER) {
                fi_cell = __ldg(s.cell[0] + i);
                fi1_face = __ldg(s.face[0] + i + 1);
            }
#pragma unroll
            for (int e = 0; e < VW; e++) {
                const int k = k0 + e;
                const T gk_cell = LAYER ? __ldg(s.cell[2] + min(k, s.nz - 1)) : T(1);
                if (k < s.nz) {
                    XH[e] = adjoint_face<T, LAYER>(VXp[e], Dc[e], Dxp[e], fi1_face, fj_cell, gk_cell);
                    YL[e] = adjoint_face<T, LAYER>(VY[e], Dy[e], Dc[e], fi_cell, fj_face, gk_cell);
                    YH[e] = adjoint_face<T, LAYER>(VYp[e], Dc[e], Dyp[e], fi_cell, fj1_face, gk_cell);
                } else {
                    XH[e] = VXp[e];
                    YL[e] = VY[e];
                    YH[e] = VYp[e];
                }
                // z face k: between cells k - 1 and k; the top face k = nz has only the lower one
                if (k <= s.nz) {
                    const T lower = k > 0 ? (e == 0 ? d_below : Dc[e - 1]) : T(0);
                    const T upper = k < s.nz ? Dc[e] : T(0);
                    Z[e] = adjoint_face<T, LAYER>(VZ[e], lower, upper, fi_cell, fj_cell,
                                                  LAYER ? __ldg(s.face[2] + k) : T(1));
                } else {
                    Z[e] = VZ[e];
                }
            }
            above = T(0);
            if (has_above)
                above = adjoint_face<T, LAYER>(vz_above, Dc[VW - 1], d_above, fi_cell, fj_cell,
                                               LAYER ? __ldg(s.face[2] + k0 + VW) : T(1));
        } else {
            VecW<T, VW>::ldg(a.lvx + base + s.plane, XH);
            VecW<T, VW>::ldg(a.lvy + base, YL);
            VecW<T, VW>::ldg(a.lvy + base + s.pz, YH);
            VecW<T, VW>::ldg(a.lvz + base, Z);
            above = has_above ? __ldg(a.lvz + base + VW) : T(0);
        }
        VecW<T, VW>::load(a.lp + base, L);
#pragma unroll
        for (int r = 0; r < NR; r++) VecW<T, VW>::load(a.lpsi + r * s.field + base, LS[r]);
        T HD[VW], HS[NR > 0 ? NR : 1][VW];
        constexpr bool air = AIR && NR > 0;
        if (air) {
            const int64_t slot = (step - a.hist.fields_step0) % a.hist.fields_slots;
            const T *h = a.hist.fields + slot * (1 + NR) * s.field + base;
            VecW<T, VW>::ldcs(h, HD);           // read once: streaming
#pragma unroll
            for (int r = 0; r < NR; r++) VecW<T, VW>::ldcs(h + (1 + r) * s.field, HS[r]);
        }
        T fi = T(1), fj = T(1);
        if (LAYER) {
            fi = __ldg(s.cell[0] + i);
            fj = __ldg(s.cell[1] + j);
        }
        // lambda(p^{n+1}): the interior-face divergence of mu^{n+1}, plus dL/drec[n]
        T LPn[VW];
#pragma unroll
        for (int e = 0; e < VW; e++) {
            const int k = k0 + e;
            const T up = e + 1 < VW ? Z[e + 1] : above;
            T dmu = (i + 1 < s.nx ? XH[e] : T(0)) - (i > 0 ? XL[e] : T(0));
            dmu = dmu + ((j + 1 < s.ny ? YH[e] : T(0)) - (j > 0 ? YL[e] : T(0)));
            dmu = dmu + ((k + 1 < s.nz ? up : T(0)) - (k > 0 ? Z[e] : T(0)));
            LPn[e] = L[e] + s.cv * dmu;
        }
        if (any_mine) {
            uint32_t m = all_points ? 0u : receiver_bits(points, s.n_src);
            for (int r = all_points ? 0 : -1; all_points ? r < s.n_rec : m != 0; r++) {
                if (!all_points) {
                    r = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.rec_off[r] - base;
                if (d >= 0 && d < VW && step >= s.rec_start[r]) {
                    const T g = (T)a.grad_rec[r * a.grad_stride + (step - a.grad_step0)];
#pragma unroll
                    for (int e = 0; e < VW; e++)
                        if (e == d) LPn[e] = LPn[e] + g;
                }
            }
            m = all_points ? 0u : source_bits(points, s.n_src);
            for (int q = all_points ? 0 : -1; all_points ? q < s.n_src : m != 0; q++) {
                if (!all_points) {
                    q = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.src_off[q] - base;
                if (d >= 0 && d < VW && step < s.src_len[q]) {
                    T v = LPn[0];
#pragma unroll
                    for (int e = 1; e < VW; e++)
                        if (e == d) v = LPn[e];
                    a.grad_src[q * a.grad_stride + (step - a.grad_step0)] = (double)(s.cs * v);
                }
            }
        }
        const bool boundary = wall_column || i == 0 || i == s.nx - 1;
        T LD[VW];
#pragma unroll
        for (int e = 0; e < VW; e++) {
            const int k = k0 + e;
            LD[e] = T(0);
            if (k >= s.nz) continue;
            const T lp = LPn[e];
            T lph = lp;
            if (LAYER) {
                lph = lph * fi;
                lph = lph * fj;
                lph = lph * __ldg(s.cell[2] + k);
            }
            T lpt = lph, lpart = lph;
            if (WALLS && boundary) {
                int64_t idx;
                const int f = shell_face(s, i, j, k, idx);
                if (f >= 0) {
                    const T *entry = s.shell[f] + 2 * idx;
                    const T u = __ldg(entry), q = __ldg(entry + 1);
                    lpt = u * lph;
                    lpart = lpt - q * lph;
                    if (a.grad_shell) {
                        const T *h = a.hist.shell + (step - a.hist.shell_step0) * 2 * a.hist.shell_total +
                                     a.hist.face_off[f] + idx;
                        const double uu = (double)u;
                        a.grad_shell[a.hist.face_off[f] + idx] +=
                            -(double)lph * uu * uu * ((double)h[a.hist.shell_total] + (double)h[0]);
                    }
                }
            }
            T ld = scp * lpt;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const T lpsi = LS[r][e];
                ld = ld + s.gain[r] * ((T(1) - s.decay[r]) * lpsi - s.mean[r] * lpt);
                LS[r][e] = s.decay[r] * lpsi + s.mean[r] * lpt;
                if (air) {
                    const T d = HD[e];
                    const T off = HS[r][e] - s.gain[r] * d;
                    air_acc[r] += d * ((T(1) - s.decay[r]) * lpsi - s.mean[r] * lpt);
                    air_acc[NR + r] += lpt * off;
                    air_acc[2 * NR + r] += lpsi * off;
                }
            }
            if (air) air_acc[3 * NR] += HD[e] * lpt;
            L[e] = lpart;
            LD[e] = ld;
        }
        VecW<T, VW>::store(a.lp + base, L);
#pragma unroll
        for (int r = 0; r < NR; r++) VecW<T, VW>::store(a.lpsi + r * s.field + base, LS[r]);
        if (FUSED) {
            VecW<T, VW>::store(a.out_d + base, LD);
            VecW<T, VW>::store(a.out_vx + base, XL);
            VecW<T, VW>::store(a.out_vy + base, YL);
            VecW<T, VW>::store(a.out_vz + base, Z);
            if (i == s.nx - 1) VecW<T, VW>::store(a.out_vx + base + s.plane, XH);
            if (j == s.ny - 1) VecW<T, VW>::store(a.out_vy + base + s.pz, YH);
            if (k0 + VW == s.nz) a.out_vz[base + VW] = above;
#pragma unroll
            for (int e = 0; e < VW; e++) {
                Dm[e] = Dc[e];
                Dc[e] = Dxp[e];
            }
        } else {
            VecW<T, VW>::store(a.ld + base, LD);
        }
#pragma unroll
        for (int e = 0; e < VW; e++) XL[e] = XH[e];
    }
}

// VW: z elements per thread (4, or 2 for the air-gradient variants: their per-thread arrays and
// sums otherwise hold the SM to 16 warps, and the step waits on its loads).
template <typename T, bool LAYER, bool WALLS, int NR, bool AIR, int VW = kVec>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? (AIR && VW == kVec ? 1 : 2) : (AIR && VW == kVec ? 2 : 4)))
    adjoint_pressure_sweep(const AdjointParams<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    constexpr int NA = 3 * NR + 1;
    // Per-thread sums over this launch's few cells in the working precision; the block sums
    // and the sums across blocks and steps are FP64.
    T air_acc[NA];
#pragma unroll
    for (int t = 0; t < NA; t++) air_acc[t] = T(0);
    if (c < (a.room.nz + VW - 1) / VW && j < a.room.ny) {
        const int i_begin = blockIdx.z * a.planes;
        adjoint_pressure_column<T, LAYER, WALLS, NR, AIR, false, VW>(a, i_begin, min(a.room.nx, i_begin + a.planes),
                                                                     j, c, *a.step_base + a.local_step, air_acc);
    }
    if (AIR && NR > 0) {  // uniform per launch: every thread reaches the barrier
        __shared__ double red[NA][8];
        const int tid = threadIdx.y * blockDim.x + threadIdx.x;
        const int lane = tid & 31, warp = tid >> 5;
        const int n_warps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
        for (int t = 0; t < NA; t++) {
            double v = (double)air_acc[t];
            for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
            if (lane == 0) red[t][warp] = v;
        }
        __syncthreads();
        if (tid < NA) {
            double v = 0.0;
            for (int w = 0; w < n_warps; w++) v += red[tid][w];
            const int64_t block = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
            a.air_partials[block * NA + tid] += v;
        }
    }
}

// The face sweep of forward step n + 1 and the cell sweep of step n in one launch (FUSED above).
template <typename T, bool LAYER, bool WALLS, int NR, bool AIR, int VW = kVec>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? (AIR && VW == kVec ? 1 : 2) : (AIR && VW == kVec ? 2 : 3)))
    adjoint_fused_sweep(const AdjointParams<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    constexpr int NA = 3 * NR + 1;
    // Per-thread sums over this launch's few cells in the working precision; the block sums
    // and the sums across blocks and steps are FP64.
    T air_acc[NA];
#pragma unroll
    for (int t = 0; t < NA; t++) air_acc[t] = T(0);
    if (c < (a.room.nz + VW - 1) / VW && j < a.room.ny) {
        const int i_begin = blockIdx.z * a.planes;
        adjoint_pressure_column<T, LAYER, WALLS, NR, AIR, true, VW>(a, i_begin, min(a.room.nx, i_begin + a.planes),
                                                                    j, c, *a.step_base + a.local_step, air_acc);
    }
    if (AIR && NR > 0) {  // uniform per launch: every thread reaches the barrier
        __shared__ double red[NA][8];
        const int tid = threadIdx.y * blockDim.x + threadIdx.x;
        const int lane = tid & 31, warp = tid >> 5;
        const int n_warps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
        for (int t = 0; t < NA; t++) {
            double v = (double)air_acc[t];
            for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
            if (lane == 0) red[t][warp] = v;
        }
        __syncthreads();
        if (tid < NA) {
            double v = 0.0;
            for (int w = 0; w < n_warps; w++) v += red[tid][w];
            const int64_t block = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
            a.air_partials[block * NA + tid] += v;
        }
    }
}

// The fused adjoint step in single precision for rooms with nz a multiple of 4 and no air
// gradients: adjoint_pressure_column<float, ..., FUSED> with the lean forward column's packed
// arithmetic -- the same operations in the same order, each lane rounded as the scalar operation
// (sums as a + (+-1) b, "plus a product" as "minus the product by the negated coefficient"),
// layer factors that are exactly 1 skipped -- so its results are the generic column's bit for bit.
// Walls, receivers and sources keep the generic column's scalar code on the cells they touch.

enum {
    kAdjNegCv = 0, kAdjScp = 1,
    kAdjNegGain = 2, kAdjOneMinusDecay = 6, kAdjMean = 10, kAdjNegMean = 14, kAdjDecay = 18
};

struct LeanAdjointParams {
    AdjointParams<float> a;
    float2 k[22];          // the kAdj* slots, each value in both lanes
};

// AIR: also accumulate the air-strength sums of adjoint_pressure_column into `acc` (3R + 1
// two-lane partial sums), from the D/psi history of the reversed step.
template <bool LAYER, bool WALLS, int NR, bool AIR = false>
__device__ __forceinline__ void lean_adjoint_column(const LeanAdjointParams &g, int i_begin, int i_end,
                                                    int j, int c, int64_t step, float2 *acc = nullptr) {
    const AdjointParams<float> &a = g.a;
    const Room<float> &s = a.room;
    const int k0 = c * kVec;
    const int64_t column = (int64_t)j * s.pz + k0;
    const bool y_lo = j > 0, y_hi = j + 1 < s.ny;
    const bool z_lo = k0 > 0, z_hi = k0 + kVec < s.nz;
    bool all_points = false;
    const uint32_t points = (s.n_src | s.n_rec) != 0 ? column_points(s, j, k0, all_points) : 0u;
    const bool any_mine = points != 0 || all_points;
    const bool wall_column = !y_lo || !y_hi || !z_lo || !z_hi;
    const float2 zero2 = dup2(0.f);

    float fj_cell = 1.f, fj_face = 1.f, fj1_face = 1.f, fkf4 = 1.f;
    float2 fkc01 = dup2(1.f), fkc23 = dup2(1.f), fkf01 = dup2(1.f), fkf23 = dup2(1.f);
    bool damp_y = false, damp_z = false;
    if (LAYER) {
        fj_cell = __ldg(s.cell[1] + j);
        fj_face = __ldg(s.face[1] + j);
        fj1_face = __ldg(s.face[1] + j + 1);
        fkc01 = make_float2(__ldg(s.cell[2] + k0), __ldg(s.cell[2] + k0 + 1));
        fkc23 = make_float2(__ldg(s.cell[2] + k0 + 2), __ldg(s.cell[2] + k0 + 3));
        fkf01 = make_float2(__ldg(s.face[2] + k0), __ldg(s.face[2] + k0 + 1));
        fkf23 = make_float2(__ldg(s.face[2] + k0 + 2), __ldg(s.face[2] + k0 + 3));
        fkf4 = __ldg(s.face[2] + k0 + 4);
        damp_y = fj_cell != 1.f || fj_face != 1.f || fj1_face != 1.f;
        damp_z = fkc01.x != 1.f || fkc01.y != 1.f || fkc23.x != 1.f || fkc23.y != 1.f ||
                 fkf01.x != 1.f || fkf01.y != 1.f || fkf23.x != 1.f || fkf23.y != 1.f || fkf4 != 1.f;
    }

    // Carried along x: lambda_D^{n+1} of this plane and mu^{n+1} on its lower x face.
    float4 Dc;
    float2 XL01, XL23;
    {
        const int64_t b0 = (int64_t)i_begin * s.plane + column;
        float4 Dm = make_float4(0.f, 0.f, 0.f, 0.f);
        Dc = __ldg(reinterpret_cast<const float4 *>(a.ld + b0));
        if (i_begin > 0) Dm = __ldg(reinterpret_cast<const float4 *>(a.ld + b0 - s.plane));
        const float4 V = __ldg(reinterpret_cast<const float4 *>(a.lvx + b0));
        XL01 = add2(lo2(V), sub2(lo2(Dm), lo2(Dc)));
        XL23 = add2(hi2(V), sub2(hi2(Dm), hi2(Dc)));
        if (LAYER) {   // (m fi_face) fj_cell gk_cell
            const float fi_face = __ldg(s.face[0] + i_begin);
            if (fi_face != 1.f) { XL01 = mul2(XL01, dup2(fi_face)); XL23 = mul2(XL23, dup2(fi_face)); }
            if (damp_y) { XL01 = mul2(XL01, dup2(fj_cell)); XL23 = mul2(XL23, dup2(fj_cell)); }
            if (damp_z) { XL01 = mul2(XL01, fkc01); XL23 = mul2(XL23, fkc23); }
        }
    }

    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        const bool x_lo = i > 0, x_hi = i + 1 < s.nx;
        if (s.prefetch && i + 1 < i_end) {
            const int64_t next = base + s.plane;
            if (i + 2 < s.nx) prefetch_l2(a.ld + next + s.plane);
            prefetch_l2(a.lvx + next + s.plane);
            prefetch_l2(a.lvy + next);
            prefetch_l2(a.lvz + next);
            prefetch_l2(a.lp + next);
#pragma unroll
            for (int r = 0; r < NR; r++) prefetch_l2(a.lpsi + r * s.field + next);
            if (AIR && NR > 0) {
                const int64_t slot = (step - a.hist.fields_step0) % a.hist.fields_slots;
                const float *h = a.hist.fields + slot * (1 + NR) * s.field + next;
#pragma unroll
                for (int r = 0; r <= NR; r++) prefetch_l2(h + r * s.field);
            }
        }
        // ---- loads
        float4 HD = make_float4(0.f, 0.f, 0.f, 0.f), HS[NR > 0 ? NR : 1];
        if (AIR && NR > 0) {   // D^n and psi^n of the reversed step
            const int64_t slot = (step - a.hist.fields_step0) % a.hist.fields_slots;
            const float *h = a.hist.fields + slot * (1 + NR) * s.field + base;
            HD = __ldcs(reinterpret_cast<const float4 *>(h));         // read once: streaming
#pragma unroll
            for (int r = 0; r < NR; r++) HS[r] = __ldcs(reinterpret_cast<const float4 *>(h + (1 + r) * s.field));
        }
        float4 Dxp = make_float4(0.f, 0.f, 0.f, 0.f), Dy = Dxp, Dyp = Dxp;
        if (x_hi) Dxp = __ldg(reinterpret_cast<const float4 *>(a.ld + base + s.plane));
        if (y_lo) Dy = __ldg(reinterpret_cast<const float4 *>(a.ld + base - s.pz));
        if (y_hi) Dyp = __ldg(reinterpret_cast<const float4 *>(a.ld + base + s.pz));
        const float d_below = z_lo ? __ldg(a.ld + base - 1) : 0.f;
        const float d_above = z_hi ? __ldg(a.ld + base + kVec) : 0.f;
        const float4 VXp = __ldg(reinterpret_cast<const float4 *>(a.lvx + base + s.plane));
        const float4 VY = __ldg(reinterpret_cast<const float4 *>(a.lvy + base));
        const float4 VYp = __ldg(reinterpret_cast<const float4 *>(a.lvy + base + s.pz));
        const float4 VZ = __ldg(reinterpret_cast<const float4 *>(a.lvz + base));
        const float vz_above = __ldg(a.lvz + base + kVec);
        const float4 L = *reinterpret_cast<const float4 *>(a.lp + base);
        float4 LS[NR > 0 ? NR : 1];
#pragma unroll
        for (int r = 0; r < NR; r++) LS[r] = *reinterpret_cast<const float4 *>(a.lpsi + r * s.field + base);
        float fi_cell = 1.f, fi1_face = 1.f;
        if (LAYER) {
            fi_cell = __ldg(s.cell[0] + i);
            fi1_face = __ldg(s.face[0] + i + 1);
        }

        // ---- mu^{n+1} on the six faces: LV + (lambda_D[lower] - lambda_D[upper]), damped
        float2 XH01 = add2(lo2(VXp), sub2(lo2(Dc), lo2(Dxp))), XH23 = add2(hi2(VXp), sub2(hi2(Dc), hi2(Dxp)));
        float2 YL01 = add2(lo2(VY), sub2(lo2(Dy), lo2(Dc))), YL23 = add2(hi2(VY), sub2(hi2(Dy), hi2(Dc)));
        float2 YH01 = add2(lo2(VYp), sub2(lo2(Dc), lo2(Dyp))), YH23 = add2(hi2(VYp), sub2(hi2(Dc), hi2(Dyp)));
        // z face k0 + e lies between cells k0 + e - 1 (below: d_below for e = 0; 0 at k = 0) and k0 + e
        float2 Z01 = add2(lo2(VZ), sub2(make_float2(d_below, Dc.x), lo2(Dc)));
        float2 Z23 = add2(hi2(VZ), sub2(make_float2(Dc.y, Dc.z), hi2(Dc)));
        float above = vz_above + (Dc.w - d_above);
        if (LAYER) {
            if (fi_cell != 1.f || fi1_face != 1.f) {
                const float2 x = dup2(fi1_face), y = dup2(fi_cell);
                XH01 = mul2(XH01, x); XH23 = mul2(XH23, x);
                YL01 = mul2(YL01, y); YL23 = mul2(YL23, y);
                YH01 = mul2(YH01, y); YH23 = mul2(YH23, y);
                Z01 = mul2(Z01, y); Z23 = mul2(Z23, y);
                above = above * fi_cell;
            }
            if (damp_y) {
                const float2 x = dup2(fj_cell), y = dup2(fj_face), z = dup2(fj1_face);
                XH01 = mul2(XH01, x); XH23 = mul2(XH23, x);
                YL01 = mul2(YL01, y); YL23 = mul2(YL23, y);
                YH01 = mul2(YH01, z); YH23 = mul2(YH23, z);
                Z01 = mul2(Z01, x); Z23 = mul2(Z23, x);
                above = above * fj_cell;
            }
            if (damp_z) {
                XH01 = mul2(XH01, fkc01); XH23 = mul2(XH23, fkc23);
                YL01 = mul2(YL01, fkc01); YL23 = mul2(YL23, fkc23);
                YH01 = mul2(YH01, fkc01); YH23 = mul2(YH23, fkc23);
                Z01 = mul2(Z01, fkf01); Z23 = mul2(Z23, fkf23);
                above = above * fkf4;
            }
        }

        // ---- lambda(p^{n+1}) = L + c_v div_interior(mu^{n+1})
        const float2 xh01 = x_hi ? XH01 : zero2, xh23 = x_hi ? XH23 : zero2;
        const float2 xl01 = x_lo ? XL01 : zero2, xl23 = x_lo ? XL23 : zero2;
        const float2 yh01 = y_hi ? YH01 : zero2, yh23 = y_hi ? YH23 : zero2;
        const float2 yl01 = y_lo ? YL01 : zero2, yl23 = y_lo ? YL23 : zero2;
        const float2 zu01 = make_float2(Z01.y, Z23.x);
        const float2 zu23 = make_float2(Z23.y, z_hi ? above : 0.f);     // face k = nz: boundary
        const float2 zl01 = make_float2(z_lo ? Z01.x : 0.f, Z01.y);     // face k = 0: boundary
        float2 d01 = sub2(xh01, xl01), d23 = sub2(xh23, xl23);
        d01 = add2(d01, sub2(yh01, yl01));
        d23 = add2(d23, sub2(yh23, yl23));
        d01 = add2(d01, sub2(zu01, zl01));
        d23 = add2(d23, sub2(zu23, Z23));
        const float2 ncv = g.k[kAdjNegCv];
        float2 P01 = sub2(lo2(L), mul2(ncv, d01)), P23 = sub2(hi2(L), mul2(ncv, d23));
        if (any_mine) {
            float LPn[kVec] = {P01.x, P01.y, P23.x, P23.y};
            uint32_t m = all_points ? 0u : receiver_bits(points, s.n_src);
            for (int r = all_points ? 0 : -1; all_points ? r < s.n_rec : m != 0; r++) {
                if (!all_points) {
                    r = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.rec_off[r] - base;
                if (d >= 0 && d < kVec && step >= s.rec_start[r]) {
                    const float gr = (float)a.grad_rec[r * a.grad_stride + (step - a.grad_step0)];
#pragma unroll
                    for (int e = 0; e < kVec; e++)
                        if (e == d) LPn[e] = LPn[e] + gr;
                }
            }
            m = all_points ? 0u : source_bits(points, s.n_src);
            for (int q = all_points ? 0 : -1; all_points ? q < s.n_src : m != 0; q++) {
                if (!all_points) {
                    q = __ffs(m) - 1;
                    m &= m - 1;
                }
                const int64_t d = s.src_off[q] - base;
                if (d >= 0 && d < kVec && step < s.src_len[q]) {
                    float v = LPn[0];
#pragma unroll
                    for (int e = 1; e < kVec; e++)
                        if (e == d) v = LPn[e];
                    a.grad_src[q * a.grad_stride + (step - a.grad_step0)] = (double)(s.cs * v);
                }
            }
            P01 = make_float2(LPn[0], LPn[1]);
            P23 = make_float2(LPn[2], LPn[3]);
        }

        // ---- the layer, wall and relaxation transposes
        float2 h01 = P01, h23 = P23;             // lp_hat
        if (LAYER) {
            if (fi_cell != 1.f) { h01 = mul2(h01, dup2(fi_cell)); h23 = mul2(h23, dup2(fi_cell)); }
            if (fj_cell != 1.f) { h01 = mul2(h01, dup2(fj_cell)); h23 = mul2(h23, dup2(fj_cell)); }
            if (damp_z) { h01 = mul2(h01, fkc01); h23 = mul2(h23, fkc23); }
        }
        float2 t01 = h01, t23 = h23;             // lp_tilde
        float2 n01 = h01, n23 = h23;             // the new lambda(p)
        if (WALLS && (wall_column || i == 0 || i == s.nx - 1)) {
            float lph[kVec] = {h01.x, h01.y, h23.x, h23.y};
            float lpt[kVec] = {h01.x, h01.y, h23.x, h23.y};
            float lpart[kVec] = {h01.x, h01.y, h23.x, h23.y};
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                int64_t idx;
                const int f = shell_face(s, i, j, k0 + e, idx);
                if (f < 0) continue;
                const float *entry = s.shell[f] + 2 * idx;
                const float u = __ldg(entry), q = __ldg(entry + 1);
                lpt[e] = u * lph[e];
                lpart[e] = lpt[e] - q * lph[e];
                if (a.grad_shell) {
                    const float *hh = a.hist.shell + (step - a.hist.shell_step0) * 2 * a.hist.shell_total +
                                      a.hist.face_off[f] + idx;
                    const double uu = (double)u;
                    a.grad_shell[a.hist.face_off[f] + idx] +=
                        -(double)lph[e] * uu * uu * ((double)hh[a.hist.shell_total] + (double)hh[0]);
                }
            }
            t01 = make_float2(lpt[0], lpt[1]);
            t23 = make_float2(lpt[2], lpt[3]);
            n01 = make_float2(lpart[0], lpart[1]);
            n23 = make_float2(lpart[2], lpart[3]);
        }
        float2 D01 = mul2(g.k[kAdjScp], t01), D23 = mul2(g.k[kAdjScp], t23);   // lambda_D^n
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const float2 p01 = lo2(LS[r]), p23 = hi2(LS[r]);
            // ld + gain ((1 - decay) lpsi - mean lpt); lpsi <- decay lpsi + mean lpt
            const float2 in01 = sub2(mul2(g.k[kAdjOneMinusDecay + r], p01), mul2(g.k[kAdjMean + r], t01));
            const float2 in23 = sub2(mul2(g.k[kAdjOneMinusDecay + r], p23), mul2(g.k[kAdjMean + r], t23));
            D01 = sub2(D01, mul2(g.k[kAdjNegGain + r], in01));
            D23 = sub2(D23, mul2(g.k[kAdjNegGain + r], in23));
            if (AIR) {   // d inner, lpt off, lpsi off with off = psi - gain d
                const float2 d01 = lo2(HD), d23 = hi2(HD);
                const float2 o01 = add2(lo2(HS[r]), mul2(g.k[kAdjNegGain + r], d01));
                const float2 o23 = add2(hi2(HS[r]), mul2(g.k[kAdjNegGain + r], d23));
                acc[r] = add2(add2(acc[r], mul2(d01, in01)), mul2(d23, in23));
                acc[NR + r] = add2(add2(acc[NR + r], mul2(t01, o01)), mul2(t23, o23));
                acc[2 * NR + r] = add2(add2(acc[2 * NR + r], mul2(p01, o01)), mul2(p23, o23));
            }
            const float2 s01 = sub2(mul2(g.k[kAdjDecay + r], p01), mul2(g.k[kAdjNegMean + r], t01));
            const float2 s23 = sub2(mul2(g.k[kAdjDecay + r], p23), mul2(g.k[kAdjNegMean + r], t23));
            LS[r] = make_float4(s01.x, s01.y, s23.x, s23.y);
        }
        if (AIR && NR > 0)
            acc[3 * NR] = add2(add2(acc[3 * NR], mul2(lo2(HD), t01)), mul2(hi2(HD), t23));

        // ---- stores
        *reinterpret_cast<float4 *>(a.lp + base) = make_float4(n01.x, n01.y, n23.x, n23.y);
#pragma unroll
        for (int r = 0; r < NR; r++) *reinterpret_cast<float4 *>(a.lpsi + r * s.field + base) = LS[r];
        *reinterpret_cast<float4 *>(a.out_d + base) = make_float4(D01.x, D01.y, D23.x, D23.y);
        *reinterpret_cast<float4 *>(a.out_vx + base) = make_float4(XL01.x, XL01.y, XL23.x, XL23.y);
        *reinterpret_cast<float4 *>(a.out_vy + base) = make_float4(YL01.x, YL01.y, YL23.x, YL23.y);
        *reinterpret_cast<float4 *>(a.out_vz + base) = make_float4(Z01.x, Z01.y, Z23.x, Z23.y);
        if (!x_hi)
            *reinterpret_cast<float4 *>(a.out_vx + base + s.plane) = make_float4(XH01.x, XH01.y, XH23.x, XH23.y);
        if (!y_hi)
            *reinterpret_cast<float4 *>(a.out_vy + base + s.pz) = make_float4(YH01.x, YH01.y, YH23.x, YH23.y);
        if (!z_hi) a.out_vz[base + kVec] = above;
        Dc = Dxp;
        XL01 = XH01;
        XL23 = XH23;
    }
}

// The same step with the air-strength sums (relaxation states present): per-thread two-lane
// sums over the launch's cells, then FP64 block sums into air_partials, as adjoint_fused_sweep.
template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, 2) lean_adjoint_air_sweep(const LeanAdjointParams g) {
    constexpr int NA = 3 * NR + 1;
    const AdjointParams<float> &a = g.a;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    float2 acc[NA];
#pragma unroll
    for (int t = 0; t < NA; t++) acc[t] = dup2(0.f);
    if (c < a.room.nz / kVec && j < a.room.ny) {
        const int i_begin = blockIdx.z * a.planes;
        lean_adjoint_column<LAYER, WALLS, NR, true>(g, i_begin, min(a.room.nx, i_begin + a.planes), j, c,
                                                    *a.step_base + a.local_step, acc);
    }
    __shared__ double red[NA][8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int n_warps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int t = 0; t < NA; t++) {
        double v = (double)acc[t].x + (double)acc[t].y;
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (lane == 0) red[t][warp] = v;
    }
    __syncthreads();
    if (tid < NA) {
        double v = 0.0;
        for (int w = 0; w < n_warps; w++) v += red[tid][w];
        const int64_t block = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        a.air_partials[block * NA + tid] += v;
    }
}

template <bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, 3) lean_adjoint_sweep(const LeanAdjointParams g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= g.a.room.nz / kVec || j >= g.a.room.ny) return;
    const int i_begin = blockIdx.z * g.a.planes;
    lean_adjoint_column<LAYER, WALLS, NR>(g, i_begin, min(g.a.room.nx, i_begin + g.a.planes), j, c,
                                          *g.a.step_base + g.a.local_step);
}

template <typename T, bool LAYER>
__device__ __forceinline__ void adjoint_velocity_column(const AdjointParams<T> &a, int i_begin,
                                                        int i_end, int j, int c) {
    const Room<T> &s = a.room;
    const int k0 = c * kVec;
    const int64_t column = (int64_t)j * s.pz + k0;
    T Dm[kVec];  // lambda_D at plane i - 1
    if (i_begin > 0) Vec4<T>::ldg(a.ld + (int64_t)(i_begin - 1) * s.plane + column, Dm);
    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + column;
        if (s.prefetch && i + 1 < i_end) {  // the next plane's own-row inputs into L2
            const int64_t next = base + s.plane;
            prefetch_l2(a.ld + next);
            prefetch_l2(a.lvx + next);
            prefetch_l2(a.lvy + next);
            prefetch_l2(a.lvz + next);
        }
        T Dc[kVec], Dy[kVec], VX[kVec], VY[kVec], VZ[kVec];
        Vec4<T>::ldg(a.ld + base, Dc);
        if (j > 0) Vec4<T>::ldg(a.ld + base - s.pz, Dy);
        const T below = k0 > 0 ? __ldg(a.ld + base - 1) : T(0);
        Vec4<T>::load(a.lvx + base, VX);
        Vec4<T>::load(a.lvy + base, VY);
        Vec4<T>::load(a.lvz + base, VZ);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            if (k >= s.nz) continue;
            T mx = VX[e] + ((i > 0 ? Dm[e] : T(0)) - Dc[e]);
            T my = VY[e] + ((j > 0 ? Dy[e] : T(0)) - Dc[e]);
            T mz = VZ[e] + ((k > 0 ? (e == 0 ? below : Dc[e - 1]) : T(0)) - Dc[e]);
            if (LAYER) {
                const T fi_cell = __ldg(s.cell[0] + i), fi_face = __ldg(s.face[0] + i);
                const T fj_cell = __ldg(s.cell[1] + j), fj_face = __ldg(s.face[1] + j);
                const T fk_cell = __ldg(s.cell[2] + k), fk_face = __ldg(s.face[2] + k);
                mx = ((mx * fi_face) * fj_cell) * fk_cell;
                my = ((my * fi_cell) * fj_face) * fk_cell;
                mz = ((mz * fi_cell) * fj_cell) * fk_face;
            }
            VX[e] = mx;
            VY[e] = my;
            VZ[e] = mz;
        }
        Vec4<T>::store(a.lvx + base, VX);
        Vec4<T>::store(a.lvy + base, VY);
        Vec4<T>::store(a.lvz + base, VZ);
        // Far boundary faces: read by the divergence of the last cell, so they carry its lambda_D.
        T fi_cell = T(1), fj_cell = T(1);
        if (LAYER) {
            fi_cell = __ldg(s.cell[0] + i);
            fj_cell = __ldg(s.cell[1] + j);
        }
        if (i == s.nx - 1) {
            T V[kVec];
            Vec4<T>::load(a.lvx + base + s.plane, V);
#pragma unroll
            for (int e = 0; e < kVec; e++)
                if (k0 + e < s.nz) {
                    T m = V[e] + Dc[e];
                    if (LAYER) m = ((m * __ldg(s.face[0] + s.nx)) * fj_cell) * __ldg(s.cell[2] + k0 + e);
                    V[e] = m;
                }
            Vec4<T>::store(a.lvx + base + s.plane, V);
        }
        if (j == s.ny - 1) {
            T V[kVec];
            Vec4<T>::load(a.lvy + base + s.pz, V);
#pragma unroll
            for (int e = 0; e < kVec; e++)
                if (k0 + e < s.nz) {
                    T m = V[e] + Dc[e];
                    if (LAYER) m = ((m * fi_cell) * __ldg(s.face[1] + s.ny)) * __ldg(s.cell[2] + k0 + e);
                    V[e] = m;
                }
            Vec4<T>::store(a.lvy + base + s.pz, V);
        }
        if (s.nz - 1 >= k0 && s.nz - 1 < k0 + kVec) {
            T last = Dc[0];
#pragma unroll
            for (int e = 1; e < kVec; e++)
                if (k0 + e == s.nz - 1) last = Dc[e];
            T *top = a.lvz + (base - k0) + s.nz;
            T m = *top + last;
            if (LAYER) m = ((m * fi_cell) * fj_cell) * __ldg(s.face[2] + s.nz);
            *top = m;
        }
#pragma unroll
        for (int e = 0; e < kVec; e++) Dm[e] = Dc[e];
    }
}

template <typename T, bool LAYER>
__global__ void __launch_bounds__(256) adjoint_velocity_sweep(const AdjointParams<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= a.room.nchunks || j >= a.room.ny) return;
    const int i_begin = blockIdx.z * a.planes;
    adjoint_velocity_column<T, LAYER>(a, i_begin, min(a.room.nx, i_begin + a.planes), j, c);
}

// ---- batches: per-room adjoint descriptions in a device table, staged like Room in the
// forward batch kernels. Walls and sources only (no air terms).

template <typename T>
struct BatchAdjointParams {
    const AdjointParams<T> *rooms;
    const Tile *tiles;
    int32_t n_tiles;
    int32_t local_step;
    const int64_t *step_base;
};

template <typename T>
__device__ __forceinline__ void stage_adjoint(const AdjointParams<T> *src, AdjointParams<T> *dst) {
    static_assert(sizeof(AdjointParams<T>) % sizeof(int) == 0, "whole words");
    const int *from = reinterpret_cast<const int *>(src);
    int *to = reinterpret_cast<int *>(dst);
    for (int w = threadIdx.x; w < (int)(sizeof(AdjointParams<T>) / sizeof(int)); w += blockDim.x)
        to[w] = __ldg(from + w);
}

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 2 : 3)) pressure_batch_rec(const BatchAdjointParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(AdjointParams<T>)];
    AdjointParams<T> *room = reinterpret_cast<AdjointParams<T> *>(raw);
    const int64_t step = *b.step_base + b.local_step;
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_adjoint(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            pressure_column<T, LAYER, WALLS, NR, true>(room->room, tile.i_begin, tile.i_end,
                                                        pair / room->room.nchunks,
                                                        pair % room->room.nchunks, step, &room->hist);
        }
    }
}

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 ? 2 : 3)) adjoint_pressure_batch(const BatchAdjointParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(AdjointParams<T>)];
    AdjointParams<T> *room = reinterpret_cast<AdjointParams<T> *>(raw);
    const int64_t step = *b.step_base + b.local_step;
    T unused[1];
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_adjoint(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            adjoint_pressure_column<T, LAYER, WALLS, NR, false>(*room, tile.i_begin, tile.i_end,
                                                                pair / room->room.nchunks,
                                                                pair % room->room.nchunks, step, unused);
        }
    }
}

// The fused adjoint step (face sweep of forward step n + 1, cell sweep of step n) over a batch:
// each room's parameters name the copy of mu and lambda_D it reads and the one it writes.
template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __maxnreg__(sizeof(T) == 8 ? 168 : 96) adjoint_fused_batch(const BatchAdjointParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(AdjointParams<T>)];
    AdjointParams<T> *room = reinterpret_cast<AdjointParams<T> *>(raw);
    const int64_t step = *b.step_base + b.local_step;
    T unused[1];
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_adjoint(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            adjoint_pressure_column<T, LAYER, WALLS, NR, false, true>(*room, tile.i_begin, tile.i_end,
                                                                      pair / room->room.nchunks,
                                                                      pair % room->room.nchunks, step, unused);
        }
    }
}

template <typename T, bool LAYER>
__global__ void __launch_bounds__(256, 3) adjoint_velocity_batch(const BatchAdjointParams<T> b) {
    __shared__ __align__(16) unsigned char raw[sizeof(AdjointParams<T>)];
    AdjointParams<T> *room = reinterpret_cast<AdjointParams<T> *>(raw);
    int staged = -1;
    for (int t = blockIdx.x; t < b.n_tiles; t += gridDim.x) {
        const Tile tile = b.tiles[t];
        if (tile.room != staged) {
            __syncthreads();
            stage_adjoint(b.rooms + tile.room, room);
            __syncthreads();
            staged = tile.room;
        }
        if ((int)threadIdx.x < tile.count) {
            const int pair = tile.first + threadIdx.x;
            adjoint_velocity_column<T, LAYER>(*room, tile.i_begin, tile.i_end,
                                              pair / room->room.nchunks, pair % room->room.nchunks);
        }
    }
}

// lambda(p^0) = LP + c_v div_interior(mu^0): the gradient with respect to the initial pressure.
template <typename T>
__global__ void __launch_bounds__(256) adjoint_finish(const AdjointParams<T> a) {
    const Room<T> &s = a.room;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= s.nchunks || j >= s.ny) return;
    const int k0 = c * kVec;
    const int i_begin = blockIdx.z * a.planes;
    const int i_end = min(s.nx, i_begin + a.planes);
    for (int i = i_begin; i < i_end; i++) {
        const int64_t base = (int64_t)i * s.plane + (int64_t)j * s.pz + k0;
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            if (k >= s.nz) continue;
            const int64_t o = base + e;
            T dmu = (i + 1 < s.nx ? a.lvx[o + s.plane] : T(0)) - (i > 0 ? a.lvx[o] : T(0));
            dmu = dmu + ((j + 1 < s.ny ? a.lvy[o + s.pz] : T(0)) - (j > 0 ? a.lvy[o] : T(0)));
            dmu = dmu + ((k + 1 < s.nz ? a.lvz[o + 1] : T(0)) - (k > 0 ? a.lvz[o] : T(0)));
            a.lp[o] = a.lp[o] + s.cv * dmu;
        }
    }
}

__global__ void set_step_base(int64_t *base, int64_t value) { *base = value; }
__global__ void bump_step_base(int64_t *base, int64_t by) { *base += by; }

// ------------------------------------------------------------------------------------------
// Energy terms of one room, FP64 accumulation (scheme.py:365-389). Two passes, fixed order:
// block partial sums into a scratch array, then one block sums the partials.
//
// Over the x planes [i0, i1): the cells of those planes with their y and z faces, and the x
// faces i0 .. i_faces - 1 (i_faces = i1, or i1 + 1 to take the far face nx too). The whole
// room is i0 = 0, i1 = nx, i_faces = nx + 1; a slab of a larger room takes its owned planes.
template <typename T>
__global__ void __launch_bounds__(256) energy_partials(const Room<T> s, double inv_dx,
                                                       double *partials, int i0, int i1,
                                                       int i_faces) {
    double acc[kEnergyTerms];
#pragma unroll
    for (int t = 0; t < kEnergyTerms; t++) acc[t] = 0.0;

    const int64_t rows = (int64_t)(i_faces - i0) * (s.ny + 1);
    const int64_t total = rows * (s.nz + 1);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < total;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(n % (s.nz + 1));
        const int64_t row = n / (s.nz + 1);
        const int j = (int)(row % (s.ny + 1));
        const int i = i0 + (int)(row / (s.ny + 1));
        const int64_t o = (int64_t)i * s.plane + (int64_t)j * s.pz + k;
        const bool in_x = i < i1, in_y = j < s.ny, in_z = k < s.nz;
        if (in_x && in_y && in_z) {
            const double p = (double)s.p[o];
            acc[0] += p * p;
        }
        if (in_y && in_z) {  // vx faces 0..nx
            const double v = (double)s.vx[o];
            acc[1] += v * v;
            if (i > 0 && i < s.nx)
                acc[4] += v * (((double)s.p[o] - (double)s.p[o - s.plane]) * inv_dx);
        }
        if (in_x && in_z) {  // vy faces 0..ny
            const double v = (double)s.vy[o];
            acc[2] += v * v;
            if (j > 0 && j < s.ny)
                acc[5] += v * (((double)s.p[o] - (double)s.p[o - s.pz]) * inv_dx);
        }
        if (in_x && in_y) {  // vz faces 0..nz
            const double v = (double)s.vz[o];
            acc[3] += v * v;
            if (k > 0 && k < s.nz) acc[6] += v * (((double)s.p[o] - (double)s.p[o - 1]) * inv_dx);
        }
    }

    __shared__ double red[kEnergyTerms][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kEnergyTerms; t++) {
        double v = acc[t];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (lane == 0) red[t][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kEnergyTerms) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
        partials[blockIdx.x * kEnergyTerms + threadIdx.x] = v;
    }
}

__global__ void energy_finish(const double *partials, int n_blocks, double *out) {
    if (threadIdx.x < kEnergyTerms) {
        double v = 0.0;
        for (int b = 0; b < n_blocks; b++) v += partials[b * kEnergyTerms + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Energy sums without allocation (acf_energy_terms_noalloc). The fields are the caller's, in
// the reference's dense C-order layout; the per-plane partial sums live in a static device
// array instead of a cudaMalloc'd buffer. One block per x plane (planes 0..nx, vx has nx+1)
// writes exactly one slot of 7 partials, so every slot the final pass reads was written by the
// same call and nothing needs clearing between calls.

static __device__ __align__(256) double g_noalloc_scratch[ACF_NOALLOC_MAX_PLANES * kEnergyTerms];

template <typename T>
static __global__ void __launch_bounds__(256) energy_dense_planes(const T *__restrict__ p,
                                                           const T *__restrict__ vx,
                                                           const T *__restrict__ vy,
                                                           const T *__restrict__ vz, int nx,
                                                           int ny, int nz, double inv_dx,
                                                           double *partials) {
    const int i = blockIdx.x;  // plane 0..nx
    double acc[kEnergyTerms];
#pragma unroll
    for (int t = 0; t < kEnergyTerms; t++) acc[t] = 0.0;
    const int64_t per_plane = (int64_t)(ny + 1) * (nz + 1);
    for (int64_t n = threadIdx.x; n < per_plane; n += blockDim.x) {
        const int k = (int)(n % (nz + 1));
        const int j = (int)(n / (nz + 1));
        const bool in_x = i < nx, in_y = j < ny, in_z = k < nz;
        const int64_t c = ((int64_t)i * ny + j) * nz + k;  // p, vx, and the p neighbours
        if (in_x && in_y && in_z) {
            const double v = (double)p[c];
            acc[0] += v * v;
        }
        if (in_y && in_z) {  // vx (nx+1, ny, nz): same index as p
            const double v = (double)vx[c];
            acc[1] += v * v;
            if (i > 0 && i < nx)
                acc[4] += v * (((double)p[c] - (double)p[c - (int64_t)ny * nz]) * inv_dx);
        }
        if (in_x && in_z) {  // vy (nx, ny+1, nz)
            const double v = (double)vy[((int64_t)i * (ny + 1) + j) * nz + k];
            acc[2] += v * v;
            if (j > 0 && j < ny) acc[5] += v * (((double)p[c] - (double)p[c - nz]) * inv_dx);
        }
        if (in_x && in_y) {  // vz (nx, ny, nz+1)
            const double v = (double)vz[((int64_t)i * ny + j) * (nz + 1) + k];
            acc[3] += v * v;
            if (k > 0 && k < nz) acc[6] += v * (((double)p[c] - (double)p[c - 1]) * inv_dx);
        }
    }
    __shared__ double red[kEnergyTerms][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kEnergyTerms; t++) {
        double v = acc[t];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (lane == 0) red[t][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kEnergyTerms) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
        partials[(int64_t)i * kEnergyTerms + threadIdx.x] = v;
    }
}

static constexpr int kNoallocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static double *g_noalloc_address[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once per device. In
// host code the symbol itself is only a host-side stand-in and must never reach a kernel.
static int noalloc_scratch(double **out) {
    int device = 0;
    ACF_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kNoallocMaxDevices)
        return fail(ACF_ERR_ARGUMENT, "device %d beyond the %d devices supported", device, kNoallocMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_address[device]) {
        void *address = nullptr;
        ACF_CUDA(cudaGetSymbolAddress(&address, g_noalloc_scratch));
        if (!address) return fail(ACF_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
        g_noalloc_address[device] = (double *)address;
    }
    *out = g_noalloc_address[device];
    return ACF_OK;
}

// ------------------------------------------------------------------------------------------
// Host side.

namespace {

struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
        if (previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        int now = -1;
        if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous)
            cudaSetDevice(previous);
    }
};

inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Everything the host keeps about one room of a batch.
struct RoomHost {
    int32_t nx = 0, ny = 0, nz = 0, n_relax = 0;
    int64_t pz = 0, plane = 0, field = 0;
    bool has_layer = false, has_walls = false;
    double coef[4] = {0, 0, 0, 0};   // cv, cp, cs, relax_scale
    double decay[ACF_MAX_RELAXATION] = {}, mean[ACF_MAX_RELAXATION] = {},
           gain[ACF_MAX_RELAXATION] = {};
    size_t state_off = 0;            // byte offset of the room's fields in the state arena
    void *second = nullptr;          // p, vx, vy, vz of the fused scheme's other buffer
    int cur = 0;                     // 1 when the current p and v are in `second`
    void *profiles = nullptr;        // cell[3] then face[3], solver precision
    int64_t profile_off[6] = {};
    void *shell = nullptr;           // 6 faces of wall pairs, solver precision
    int64_t shell_off[6] = {};
    // sources
    int64_t n_src = 0, src_stride = 0;
    int64_t *src_off = nullptr, *src_len = nullptr;
    void *src_sig = nullptr;
    // receivers
    int64_t n_rec = 0, rec_capacity = 0, rec_origin = 0;
    bool rec_origin_set = false;
    int64_t *rec_off = nullptr, *rec_start = nullptr;
    void *rec = nullptr;
    std::vector<int64_t> host_rec_start;

    int64_t n_cells() const { return (int64_t)nx * ny * nz; }
    int64_t padded_offset(int64_t flat) const {
        const int64_t k = flat % nz;
        const int64_t j = (flat / nz) % ny;
        const int64_t i = flat / ((int64_t)nz * ny);
        return i * plane + j * pz + k;
    }
};

}  // namespace

struct acf_batch {
    int device = 0;
    int precision = 8;
    int n_relax = 0;                 // the same for every room of a batch
    bool any_layer = false, any_walls = false;
    std::vector<RoomHost> rooms;

    void *state = nullptr;           // every room's fields, one arena
    size_t state_bytes = 0;
    void *room_table = nullptr;      // device array of Room<T>, one per room
    void *fused_table = nullptr;     // fused scheme on a batch: 2 x rooms FusedParams<T>, by parity
    bool room_table_dirty = true;
    Tile *tiles = nullptr;
    int32_t n_tiles = 0;
    int32_t batch_ctas = 0;
    int64_t *step_base = nullptr;    // two int64 in device memory: the step counter, then
                                     // the error flag of the staged sweep (an int32)
    double *energy_scratch = nullptr;
    int energy_blocks = 0;
    int sms = 148;

    // launch geometry (tunable; results never depend on it)
    int block_threads = 256;
    int planes = 4;
    int ctas_per_sm = 4;
    int staged_rows = 2;             // staged scheme: y rows per CTA
    int staged_stages = 0;           // staged scheme: ring buffers per CTA (0: automatic)
    int staged_vector = 4;           // staged scheme: z elements per thread (2 or 4)
    int smem_per_sm = 233472, smem_per_block = 232448;
    int prefetch_mode = -1;          // L2 prefetch of the next plane: -1 by size, 0 off, 1 on
    int64_t l2_bytes = 0;            // the device's L2 size

    // graphs (index: parity of the fused scheme's current buffer at the start of a replay)
    int32_t graph_steps = 0;
    cudaGraphExec_t graph = nullptr, graph_odd = nullptr;
    cudaStream_t capture_stream = nullptr;
    bool graph_dirty = true;

    // profiling
    bool profiling = false;
    double prof_velocity_ms = 0, prof_pressure_ms = 0;
    int64_t prof_launches = 0;
    static constexpr int64_t kRing = 64;
    cudaEvent_t ring[3 * kRing] = {};

    int64_t launches = 0;

    // The device status word (kStatus* bits), copied to pinned host memory after every run so
    // that the next run can report a non-finite state without waiting for the device.
    int32_t *status_host = nullptr;
    cudaEvent_t status_event = nullptr;
    bool status_pending = false;
    // Pressure-only scheme: the next step starts from the p-v state (p^n, v^{n-1/2}); cleared by
    // that step, after which the velocities of either copy are stale.
    bool po_first = true;
    bool po_started = false;
    // Test hooks of the staged sweep (acf_set_wait_test): 0 / -1 leave it as built.
    uint64_t test_wait_limit_ns = 0;
    int32_t test_skip_plane = -1;
    // Steps per launch of the fused single-precision scheme (acf_set_time_blocking): 1, or 2 for
    // the two-step sweep, with its launch and buffers -- the first-step pressure ring, the CTA
    // counters and the second copy of the relaxation states -- allocated when it is selected.
    int32_t time_block = 1;
    dim3 pair_grid, pair_block;
    int32_t pair_planes = 0;
    float *pair_ring = nullptr;
    int32_t *pair_progress = nullptr;
    size_t pair_counters = 0;
    float *psi2 = nullptr;

    // CUDA graphs of the adjoint path: forward record, recompute, adjoint steps
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        int64_t steps = 0;
        void release() {
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    };
    Graph g_record, g_recompute, g_adjoint, g_adjoint_odd;   // adjoint: per starting copy
    bool adj_graphs_dirty = true;

    // adjoint (single rooms)
    struct Adjoint {
        int32_t flags = 0;
        int64_t capacity = 0;        // steps a forward record may hold
        int32_t every = 0;           // checkpoint interval
        int64_t recorded = 0, step0 = 0;
        bool fields_recorded = false;   // the recorded run wrote D and psi of every step itself
        int direct_mode = -1;        // how the last recorded run stepped (graph validity): 0 two
                                     // sweeps, 1 two sweeps writing D and psi, 2 the lean step
        int64_t shell_total = 0;
        int64_t face_off[6] = {};
        void *hist_shell = nullptr;  // capacity x 2 x shell_total values
        void *checkpoints = nullptr; // ceil(capacity / every) room states
        void *scratch = nullptr;     // recompute state
        void *segment = nullptr;     // every x (1 + n_relax) fields
        void *fields = nullptr;      // (5 + n_relax) adjoint fields
        void *fields2 = nullptr;     // the fused adjoint's second copy of mu (3 fields), lambda_D
        double *grad_shell = nullptr;
        double *air_partials = nullptr;
        int64_t air_blocks = 0;
        double *grad_rec = nullptr, *grad_src = nullptr;
        int64_t grad_rows_rec = 0, grad_rows_src = 0;
    } adj;

    // adjoint of a batch of rooms (walls and sources): per-room history and adjoint fields
    struct RoomAdjoint {
        void *hist_shell = nullptr, *fields = nullptr;
        void *fields2 = nullptr;     // second copy of mu (3 fields) and lambda_D for the fused step
        double *grad_shell = nullptr, *grad_rec = nullptr, *grad_src = nullptr;
        int64_t shell_total = 0, face_off[6] = {}, rows_rec = 0, rows_src = 0;
    };
    std::vector<RoomAdjoint> badj;
    int64_t badj_capacity = 0, badj_recorded = 0, badj_step0 = 0;
    void *badj_table = nullptr;      // device array of AdjointParams<T>: 2 per room (the two copies of mu)

    size_t elem() const { return (size_t)precision; }
    int n_fields() const { return 4 + n_relax; }
    size_t room_block_bytes(int r) const { return (size_t)n_fields() * rooms[r].field * elem(); }
    int scheme = ACF_SCHEME_TWO_SWEEPS;
    // one sweep per step into the second copy of p and v (fused, or fused-staged for one room)
    bool fused() const { return scheme == ACF_SCHEME_FUSED || scheme == ACF_SCHEME_FUSED_STAGED; }
    bool pressure_only() const { return scheme == ACF_SCHEME_PRESSURE_ONLY; }
    // Schemes whose step writes the other copy of the state, so that the current one alternates.
    bool alternating() const { return fused() || pressure_only(); }
    int32_t *error_flag() const { return reinterpret_cast<int32_t *>(step_base + 1); }
    char *field_ptr(int r, int f) const {
        const RoomHost &h = rooms[r];
        if (h.cur && f < 4) return (char *)h.second + (size_t)f * h.field * elem();
        return (char *)state + h.state_off + (size_t)f * h.field * elem();
    }
    // p, vx, vy, vz of the buffer that is not current (the fused step's destination)
    char *other_ptr(int r, int f) const {
        const RoomHost &h = rooms[r];
        if (h.cur) return (char *)state + h.state_off + (size_t)f * h.field * elem();
        return (char *)h.second + (size_t)f * h.field * elem();
    }
};

// A single room is a batch of one, launched with the 2D single-room kernels.
struct acf_solver : acf_batch {};

namespace {

// `state` (optional) points at another copy of the room's fields in the same geometry, such as
// the adjoint's recompute buffer.
// Whether the marching kernels ask L2 for each next plane ahead of its loads. Automatically
// when the fields one step streams (every room of the handle; the fused schemes' second copy
// of p and v included) exceed L2: the prefetches then keep more DRAM reads in flight than the
// threads' registers hold, while a room that stays in L2 would only pay for the extra requests.
bool prefetch_planes(const acf_batch *b) {
    if (b->prefetch_mode >= 0) return b->prefetch_mode != 0;
    const double fields = (double)b->n_fields() + (b->scheme != ACF_SCHEME_TWO_SWEEPS ? 4.0 : 0.0);
    double bytes = 0;
    for (const RoomHost &h : b->rooms) bytes += fields * (double)h.field * (double)b->elem();
    return bytes > (double)b->l2_bytes;
}

template <typename T>
Room<T> make_room(const acf_batch *b, int r, const void *state = nullptr) {
    const RoomHost &h = b->rooms[r];
    Room<T> s{};
    s.status = b->error_flag();
    s.nx = h.nx;
    s.ny = h.ny;
    s.nz = h.nz;
    s.nchunks = (int32_t)((h.nz + kVec - 1) / kVec);
    s.prefetch = prefetch_planes(b) ? 1 : 0;
    s.own_lo = 0;
    s.own_hi = h.nx;
    s.pz = h.pz;
    s.plane = h.plane;
    s.field = h.field;
    if (state) {
        T *fields = (T *)state;
        s.p = fields;
        s.vx = fields + h.field;
        s.vy = fields + 2 * h.field;
        s.vz = fields + 3 * h.field;
        s.psi = fields + 4 * h.field;
    } else {
        s.p = (T *)b->field_ptr(r, ACF_FIELD_P);
        s.vx = (T *)b->field_ptr(r, ACF_FIELD_VX);
        s.vy = (T *)b->field_ptr(r, ACF_FIELD_VY);
        s.vz = (T *)b->field_ptr(r, ACF_FIELD_VZ);
        s.psi = (T *)b->field_ptr(r, ACF_FIELD_PSI0);
    }
    s.cv = (T)h.coef[0];
    s.cp = (T)h.coef[1];
    s.cs = (T)h.coef[2];
    s.relax_scale = (T)h.coef[3];
    for (int q = 0; q < ACF_MAX_RELAXATION; q++) {
        s.decay[q] = (T)h.decay[q];
        s.mean[q] = (T)h.mean[q];
        s.gain[q] = (T)h.gain[q];
    }
    for (int a = 0; a < 3; a++) {
        s.cell[a] = h.profiles ? (const T *)h.profiles + h.profile_off[a] : nullptr;
        s.face[a] = h.profiles ? (const T *)h.profiles + h.profile_off[3 + a] : nullptr;
    }
    for (int f = 0; f < 6; f++) s.shell[f] = h.shell ? (const T *)h.shell + h.shell_off[f] : nullptr;
    s.n_src = (int32_t)h.n_src;
    s.src_off = h.src_off;
    s.src_col = h.src_off ? h.src_off + h.n_src : nullptr;
    s.src_len = h.src_len;
    s.src_sig = (const T *)h.src_sig;
    s.src_stride = h.src_stride;
    s.n_rec = (int32_t)h.n_rec;
    s.rec_off = h.rec_off;
    s.rec_col = h.rec_off ? h.rec_off + h.n_rec : nullptr;
    s.rec_start = h.rec_start;
    s.rec = (T *)h.rec;
    s.rec_stride = h.rec_capacity;
    s.rec_origin = h.rec_origin;
    return s;
}

template <typename T>
int upload_room_table(acf_batch *b) {
    std::vector<Room<T>> table(b->rooms.size());
    for (size_t r = 0; r < b->rooms.size(); r++) table[r] = make_room<T>(b, (int)r);
    if (!b->room_table) ACF_CUDA(cudaMalloc(&b->room_table, table.size() * sizeof(Room<T>)));
    ACF_CUDA(cudaMemcpy(b->room_table, table.data(), table.size() * sizeof(Room<T>), cudaMemcpyHostToDevice));
    if (b->scheme == ACF_SCHEME_FUSED) {
        // Both parities: entry [parity * rooms + r] reads the copy that is current at that parity.
        const size_t n = b->rooms.size();
        std::vector<FusedParams<T>> fused(2 * n);
        for (int parity = 0; parity < 2; parity++)
            for (size_t r = 0; r < n; r++) {
                RoomHost &h = b->rooms[r];
                const int saved = h.cur;
                h.cur = parity;
                FusedParams<T> &f = fused[parity * n + r];
                f = FusedParams<T>{};
                f.room = make_room<T>(b, (int)r);
                f.np = (T *)b->other_ptr((int)r, ACF_FIELD_P);
                f.nvx = (T *)b->other_ptr((int)r, ACF_FIELD_VX);
                f.nvy = (T *)b->other_ptr((int)r, ACF_FIELD_VY);
                f.nvz = (T *)b->other_ptr((int)r, ACF_FIELD_VZ);
                h.cur = saved;
            }
        if (!b->fused_table) ACF_CUDA(cudaMalloc(&b->fused_table, fused.size() * sizeof(FusedParams<T>)));
        ACF_CUDA(cudaMemcpy(b->fused_table, fused.data(), fused.size() * sizeof(FusedParams<T>),
                            cudaMemcpyHostToDevice));
    }
    b->room_table_dirty = false;
    return ACF_OK;
}

// Tiles in room order, then plane group, then (row, chunk) block: neighbouring tiles of one
// room run close together, so the y- and x-neighbour rows they share are still in L2.
int build_tiles(acf_batch *b) {
    std::vector<Tile> tiles;
    for (size_t r = 0; r < b->rooms.size(); r++) {
        const RoomHost &h = b->rooms[r];
        const int64_t nchunks = (h.nz + kVec - 1) / kVec;
        const int64_t pairs = (int64_t)h.ny * nchunks;
        for (int i0 = 0; i0 < h.nx; i0 += b->planes)
            for (int64_t first = 0; first < pairs; first += b->block_threads) {
                Tile t{};
                t.room = (int32_t)r;
                t.first = (int32_t)first;
                t.count = (int32_t)std::min<int64_t>(b->block_threads, pairs - first);
                t.i_begin = i0;
                t.i_end = std::min(h.nx, i0 + b->planes);
                tiles.push_back(t);
            }
    }
    if (tiles.size() > (size_t)INT32_MAX) return fail(ACF_ERR_ARGUMENT, "too many tiles");
    cudaFree(b->tiles);
    b->tiles = nullptr;
    ACF_CUDA(cudaMalloc(&b->tiles, std::max<size_t>(1, tiles.size()) * sizeof(Tile)));
    ACF_CUDA(cudaMemcpy(b->tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
    b->n_tiles = (int32_t)tiles.size();
    // ctas_per_sm == 0: one CTA per tile, scheduled by the hardware; otherwise a persistent
    // grid of ctas_per_sm CTAs per SM striding over the table.
    b->batch_ctas = b->ctas_per_sm == 0 ? std::max(1, b->n_tiles)
                                        : std::max(1, std::min(b->n_tiles, b->ctas_per_sm * b->sms));
    return ACF_OK;
}

struct LaunchShape {
    dim3 grid, block;
};

LaunchShape single_shape(const acf_batch *b, int width = kVec) {
    const RoomHost &h = b->rooms[0];
    const int nchunks = (int)((h.nz + width - 1) / width);
    int bx = 1;
    while (bx < nchunks && bx < 32) bx <<= 1;
    int by = std::max(1, std::min<int>(h.ny, b->block_threads / bx));
    LaunchShape L;
    L.block = dim3(bx, by, 1);
    L.grid = dim3((nchunks + bx - 1) / bx, (h.ny + by - 1) / by, (h.nx + b->planes - 1) / b->planes);
    return L;
}

// Template dispatch over the pressure kernels' compile-time features.
template <typename T, template <typename, bool, bool, int> class K, typename P>
void dispatch_pressure(bool layer, bool walls, int nr, const P &params, dim3 grid, dim3 block,
                       cudaStream_t st) {
#define ACF_NR(L, W)                                                                    \
    switch (nr) {                                                                        \
        case 0: K<T, L, W, 0>::launch(params, grid, block, st); break;                  \
        case 1: K<T, L, W, 1>::launch(params, grid, block, st); break;                  \
        case 2: K<T, L, W, 2>::launch(params, grid, block, st); break;                  \
        case 3: K<T, L, W, 3>::launch(params, grid, block, st); break;                  \
        default: K<T, L, W, 4>::launch(params, grid, block, st); break;                 \
    }
    if (layer) {
        if (walls) { ACF_NR(true, true) } else { ACF_NR(true, false) }
    } else {
        if (walls) { ACF_NR(false, true) } else { ACF_NR(false, false) }
    }
#undef ACF_NR
}

template <typename T, bool L, bool W, int NR>
struct SinglePressure {
    static void launch(const StepParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        pressure_sweep<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct BatchPressure {
    static void launch(const BatchParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        pressure_batch<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct FusedStep {
    static void launch(const FusedParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        fused_sweep<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanStep {
    static void launch(const LeanParams &p, dim3 g, dim3 b, cudaStream_t st) {
        lean_sweep<L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanPartsStep {
    static void launch(const LeanPartsParams &p, dim3 g, dim3 b, cudaStream_t st) {
        lean_parts_sweep<L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanStepPadded {
    static void launch(const LeanParams &p, dim3 g, dim3 b, cudaStream_t st) {
        lean_sweep_padded<L, W, NR><<<g, b, 0, st>>>(p);
    }
};


// The packed coefficients of the single-precision kernels: each rounded to float once, the
// negated slots negated after that rounding, so each is exactly minus the scalar's value.
void fill_pairs(float2 *pairs, const RoomHost &h) {
    auto put = [&](int slot, double v) { pairs[slot] = make_float2((float)v, (float)v); };
    auto put_neg = [&](int slot, double v) { pairs[slot] = make_float2(-(float)v, -(float)v); };
    put(kPairCv, h.coef[0]);
    put(kPairCp, h.coef[1]);
    put_neg(kPairNegRelaxScale, h.coef[3]);
    for (int r = 0; r < h.n_relax; r++) {
        put(kPairGain + r, h.gain[r]);
        put_neg(kPairNegDecay + r, h.decay[r]);
        put_neg(kPairNegMean + r, h.mean[r]);
    }
}

template <typename T, bool L, bool W, int NR>
struct BatchFused {
    static void launch(const FusedBatchParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        fused_batch<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

// Ring layout and shared memory of the staged sweep for `rows` y rows per CTA.
struct StagedLayout {
    int64_t stage_elems = 0, off_vx = 0, off_vy = 0, off_vz = 0, off_psi = 0;
    size_t smem(int stages, size_t es) const { return kStagedBarrierBytes + (size_t)stages * stage_elems * es; }
};

inline StagedLayout staged_layout(const RoomHost &h, int rows) {
    StagedLayout L;
    L.off_vx = (int64_t)(rows + 2) * h.pz;             // p: rows + 2 (y halo)
    L.off_vy = L.off_vx + (int64_t)rows * h.pz;        // vx: rows
    L.off_vz = L.off_vy + (int64_t)(rows + 1) * h.pz;  // vy: rows + 1
    L.off_psi = L.off_vz + (int64_t)rows * h.pz;       // vz: rows
    L.stage_elems = L.off_psi + (int64_t)h.n_relax * rows * h.pz;
    return L;
}

inline int staged_block_x(const RoomHost &h, int vector) {
    return (int)round_up((h.nz + vector - 1) / vector, 32);
}

// Ring buffers for (rows, requested): the request if it fits one CTA's shared memory, else 0;
// for 0, three (one plane in flight beyond the two being read) or, if three do not fit, two.
inline int staged_stages(const acf_batch *b, int rows, int requested) {
    const RoomHost &h = b->rooms[0];
    const StagedLayout L = staged_layout(h, rows);
    auto fits = [&](int S) { return L.smem(S, b->elem()) + 1024 <= (size_t)b->smem_per_block; };
    if (requested) return fits(requested) ? requested : 0;
    for (int S = 3; S >= 2; S--)
        if (fits(S)) return S;
    return 0;
}

template <typename T, bool L, bool W, int NR>
struct StagedStep {
    static void launch(const StagedParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        const size_t smem = kStagedBarrierBytes + (size_t)p.stages * p.stage_elems * sizeof(T);
        // Opt in to the largest dynamic shared memory the block can hold beside its static part:
        // a per-device attribute of the kernel, so once on each device (first 64 devices).
        static std::atomic<uint64_t> opted_in{0};
        int device = 0;
        cudaGetDevice(&device);
        const uint64_t bit = device < 64 ? (uint64_t)1 << device : 0;
        if (!bit || !(opted_in.load() & bit)) {
            int optin = 0;
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
            auto opt_in = [optin](const void *kernel) {
                cudaFuncAttributes attr{};
                if (cudaFuncGetAttributes(&attr, kernel) == cudaSuccess)
                    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         optin - (int)attr.sharedSizeBytes);
            };
            opt_in((const void *)fused_staged_sweep<T, L, W, NR, 2>);
            opt_in((const void *)fused_staged_sweep<T, L, W, NR, 4>);
            opted_in.fetch_or(bit);
        }
        if (p.vector == 2) fused_staged_sweep<T, L, W, NR, 2><<<g, b, smem, st>>>(p);
        else fused_staged_sweep<T, L, W, NR, 4><<<g, b, smem, st>>>(p);
    }
};

// The two-step sweep: a cooperative launch, so that every CTA is resident (CTAs wait for their
// neighbours' counters) or the launch fails with an error instead.
template <typename T, bool L, bool W, int NR>
struct PairStep {
    static void launch(const PairParams &p, dim3 g, dim3 b, cudaStream_t st) {
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = b;
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, lean_pair_sweep<L, W, NR>, p);
    }
};

const void *pair_kernel(bool layer, bool walls, int nr) {
#define ACF_PAIR_NR(L, W)                                                  \
    switch (nr) {                                                           \
        case 0: return (const void *)lean_pair_sweep<L, W, 0>;              \
        case 1: return (const void *)lean_pair_sweep<L, W, 1>;              \
        case 2: return (const void *)lean_pair_sweep<L, W, 2>;              \
        case 3: return (const void *)lean_pair_sweep<L, W, 3>;              \
        default: return (const void *)lean_pair_sweep<L, W, 4>;             \
    }
    if (layer) {
        if (walls) { ACF_PAIR_NR(true, true) } else { ACF_PAIR_NR(true, false) }
    } else {
        if (walls) { ACF_PAIR_NR(false, true) } else { ACF_PAIR_NR(false, false) }
    }
#undef ACF_PAIR_NR
}

// Select 1 or 2 steps per launch. Two need one single-precision room with nz a multiple of 4
// whose CTAs (128 threads over 32 chunks and 4 rows, or fewer chunks and more rows) all fit on
// the device at once for one group of x planes; as many groups are used as fit, at least 8
// planes each.
int set_time_blocking(acf_batch *b, int32_t steps) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (steps != 1 && steps != 2) return fail(ACF_ERR_ARGUMENT, "steps per launch must be 1 or 2, got %d", steps);
    if (steps == 1) {
        b->time_block = 1;
        return ACF_OK;
    }
    if (b->precision != 4 || b->rooms.size() != 1)
        return fail(ACF_ERR_ARGUMENT, "two steps per launch need one single-precision room");
    const RoomHost &h = b->rooms[0];
    if (h.nz % kVec != 0)
        return fail(ACF_ERR_ARGUMENT, "two steps per launch need nz to be a multiple of %d, got %d", kVec, h.nz);
    DeviceGuard guard(b->device);
    const int nchunks = h.nz / kVec;
    int bx = 1;
    while (bx < nchunks && bx < 32) bx <<= 1;
    const int by = kPairThreads / bx;
    const int gx = (nchunks + bx - 1) / bx, gy = (h.ny + by - 1) / by;
    int per_sm = 0;
    ACF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_kernel(h.has_layer, h.has_walls, h.n_relax),
                                                           kPairThreads, 0));
    const int64_t resident = (int64_t)per_sm * b->sms, per_group = (int64_t)gx * gy;
    if (per_group > resident)
        return fail(ACF_ERR_ARGUMENT, "two steps per launch: a y-z plane needs %lld CTAs, the device holds %lld",
                    (long long)per_group, (long long)resident);
    int64_t groups = std::min<int64_t>(resident / per_group, std::max<int64_t>(1, h.nx / 8));
    const int planes = (int)((h.nx + groups - 1) / groups);
    groups = (h.nx + planes - 1) / planes;
    const size_t ring_bytes = (size_t)groups * kPairRing * h.plane * sizeof(float);
    const size_t counters = (size_t)(per_group * groups);
    b->time_block = 1;          // until the new buffers are in place
    cudaFree(b->pair_ring);
    cudaFree(b->pair_progress);
    b->pair_ring = nullptr;
    b->pair_progress = nullptr;
    ACF_CUDA(cudaMalloc(&b->pair_ring, ring_bytes));
    ACF_CUDA(cudaMalloc(&b->pair_progress, counters * sizeof(int32_t)));
    if (h.n_relax > 0 && !b->psi2)
        ACF_CUDA(cudaMalloc(&b->psi2, (size_t)h.n_relax * h.field * sizeof(float)));
    b->pair_grid = dim3(gx, gy, (unsigned)groups);
    b->pair_block = dim3(bx, by, 1);
    b->pair_planes = planes;
    b->pair_counters = counters;
    b->time_block = 2;
    return ACF_OK;
}

// Two steps of the fused single-precision scheme in one launch. The relaxation states go from
// the room's own field to the second copy (`back` false) or back; p and v to the other copy.
void launch_pair(acf_batch *b, int32_t local, bool back, cudaStream_t st) {
    RoomHost &h = b->rooms[0];
    PairParams q{};
    LeanParams &g = q.g;
    g.f.room = make_room<float>(b, 0);
    float *own = g.f.room.psi;
    g.f.room.psi = back ? b->psi2 : own;
    q.psi_out = back ? own : b->psi2;
    g.f.np = (float *)b->other_ptr(0, ACF_FIELD_P);
    g.f.nvx = (float *)b->other_ptr(0, ACF_FIELD_VX);
    g.f.nvy = (float *)b->other_ptr(0, ACF_FIELD_VY);
    g.f.nvz = (float *)b->other_ptr(0, ACF_FIELD_VZ);
    g.f.step_base = b->step_base;
    g.f.local_step = local;
    g.f.planes = b->pair_planes;
    fill_pairs(g.pairs, h);
    q.ring = b->pair_ring;
    q.progress = b->pair_progress;
    q.wait_limit_ns = b->test_wait_limit_ns ? b->test_wait_limit_ns : kWaitLimitNs;
    q.stop_plane = b->test_skip_plane;
    cudaMemsetAsync(b->pair_progress, 0, b->pair_counters * sizeof(int32_t), st);
    dispatch_pressure<float, PairStep>(h.has_layer, h.has_walls, h.n_relax, q, b->pair_grid, b->pair_block, st);
    h.cur ^= 1;
    b->launches += 1;
}

// Launch one step; the fused scheme flips the room's current buffer, as the kernel will have
// done by the time anything queued after it runs.
template <typename T>
void launch_step(acf_batch *b, int32_t local, cudaStream_t st, cudaEvent_t *events) {
    if (events) cudaEventRecord(events[0], st);
    if (b->rooms.size() > 1 && b->fused()) {
        // The tile-table launch keeps the generic column: the lean column there measured 82-89
        // Gcell-updates/s on the 64 uneven rooms against 94 (its registers cost warps per SM).
        const dim3 grid(b->batch_ctas), block(b->block_threads);
        FusedBatchParams<T> p{};
        p.rooms = (const FusedParams<T> *)b->fused_table + (b->rooms[0].cur ? b->rooms.size() : 0);
        p.tiles = b->tiles;
        p.n_tiles = b->n_tiles;
        p.local_step = local;
        p.step_base = b->step_base;
        dispatch_pressure<T, BatchFused>(b->any_layer, b->any_walls, b->n_relax, p, grid, block, st);
        for (RoomHost &h : b->rooms) h.cur ^= 1;
        if (events) {
            cudaEventRecord(events[1], st);
            cudaEventRecord(events[2], st);
        }
        return;
    }
    if (b->pressure_only()) {
        RoomHost &h = b->rooms[0];
        PressureOnlyParams<T> g{};
        g.room = make_room<T>(b, 0);
        g.cur = (const T *)b->field_ptr(0, ACF_FIELD_P);
        g.next = (T *)b->other_ptr(0, ACF_FIELD_P);
        g.lam2 = (T)(h.coef[0] * h.coef[1]);
        g.step_base = b->step_base;
        g.local_step = local;
        g.planes = b->planes;
        const LaunchShape L = single_shape(b);
        const bool first = b->po_first;
        b->po_first = false;
        b->po_started = true;
        if (first) {
            if (h.has_walls) pressure_only_sweep<T, true, true><<<L.grid, L.block, 0, st>>>(g);
            else pressure_only_sweep<T, false, true><<<L.grid, L.block, 0, st>>>(g);
        } else if (h.nz % kVec == 0) {
            if (h.has_walls) pressure_only_sweep<T, true, false, true><<<L.grid, L.block, 0, st>>>(g);
            else pressure_only_sweep<T, false, false, true><<<L.grid, L.block, 0, st>>>(g);
        } else {
            if (h.has_walls) pressure_only_sweep<T, true, false, false><<<L.grid, L.block, 0, st>>>(g);
            else pressure_only_sweep<T, false, false, false><<<L.grid, L.block, 0, st>>>(g);
        }
        h.cur ^= 1;
        if (events) {
            cudaEventRecord(events[1], st);
            cudaEventRecord(events[2], st);
        }
        return;
    }
    if (b->fused()) {
        RoomHost &h = b->rooms[0];
        FusedParams<T> f{};
        f.room = make_room<T>(b, 0);
        f.np = (T *)b->other_ptr(0, ACF_FIELD_P);
        f.nvx = (T *)b->other_ptr(0, ACF_FIELD_VX);
        f.nvy = (T *)b->other_ptr(0, ACF_FIELD_VY);
        f.nvz = (T *)b->other_ptr(0, ACF_FIELD_VZ);
        f.step_base = b->step_base;
        f.local_step = local;
        f.planes = b->planes;
        if (b->scheme == ACF_SCHEME_FUSED_STAGED) {
            StagedParams<T> g{};
            g.f = f;
            g.rows = b->staged_rows;
            g.stages = staged_stages(b, b->staged_rows, b->staged_stages);
            g.vector = b->staged_vector;
            const StagedLayout lay = staged_layout(h, b->staged_rows);
            g.stage_elems = lay.stage_elems;
            g.off_vx = lay.off_vx;
            g.off_vy = lay.off_vy;
            g.off_vz = lay.off_vz;
            g.off_psi = lay.off_psi;
            g.error = b->error_flag();
            g.wait_limit_ns = b->test_wait_limit_ns ? b->test_wait_limit_ns : kWaitLimitNs;
            g.skip_plane = b->test_skip_plane;
            if (sizeof(T) == 4) fill_pairs(g.pairs, h);
            g.block_x = staged_block_x(h, b->staged_vector);
            const dim3 block(g.block_x * b->staged_rows + 32);
            const dim3 grid((h.ny + b->staged_rows - 1) / b->staged_rows, (h.nx + b->planes - 1) / b->planes);
            dispatch_pressure<T, StagedStep>(h.has_layer, h.has_walls, h.n_relax, g, grid, block, st);
        } else {
            const LaunchShape L = single_shape(b);
            if constexpr (sizeof(T) == 4) {   // the lean single-precision column
                LeanParams g{};
                g.f = f;
                fill_pairs(g.pairs, h);
                if (h.nz % kVec == 0)
                    dispatch_pressure<float, LeanStep>(h.has_layer, h.has_walls, h.n_relax, g, L.grid, L.block, st);
                else
                    dispatch_pressure<float, LeanStepPadded>(h.has_layer, h.has_walls, h.n_relax, g, L.grid,
                                                             L.block, st);
            } else {
                dispatch_pressure<T, FusedStep>(h.has_layer, h.has_walls, h.n_relax, f, L.grid, L.block, st);
            }
        }
        h.cur ^= 1;
        if (events) {
            cudaEventRecord(events[1], st);
            cudaEventRecord(events[2], st);
        }
        return;
    }
    if (b->rooms.size() == 1) {
        const RoomHost &h = b->rooms[0];
        StepParams<T> p{};
        p.room = make_room<T>(b, 0);
        p.step_base = b->step_base;
        p.local_step = local;
        p.planes = b->planes;
        const LaunchShape L = single_shape(b);
        if (h.has_layer) velocity_sweep<T, true><<<L.grid, L.block, 0, st>>>(p);
        else velocity_sweep<T, false><<<L.grid, L.block, 0, st>>>(p);
        if (events) cudaEventRecord(events[1], st);
        dispatch_pressure<T, SinglePressure>(h.has_layer, h.has_walls, h.n_relax, p, L.grid,
                                             L.block, st);
    } else {
        BatchParams<T> p{};
        p.rooms = (const Room<T> *)b->room_table;
        p.tiles = b->tiles;
        p.n_tiles = b->n_tiles;
        p.local_step = local;
        p.step_base = b->step_base;
        const dim3 grid(b->batch_ctas), block(b->block_threads);
        if (b->any_layer) velocity_batch<T, true><<<grid, block, 0, st>>>(p);
        else velocity_batch<T, false><<<grid, block, 0, st>>>(p);
        if (events) cudaEventRecord(events[1], st);
        dispatch_pressure<T, BatchPressure>(b->any_layer, b->any_walls, b->n_relax, p, grid, block, st);
    }
    if (events) cudaEventRecord(events[2], st);
}

template <typename T>
int run_impl(acf_batch *b, int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    if (b->rooms.size() > 1 && b->room_table_dirty) {
        int rc = upload_room_table<T>(b);
        if (rc) return rc;
    }
    set_step_base<<<1, 1, 0, st>>>(b->step_base, step_offset);
    b->launches += 1;

    if (b->profiling) {
        // Event ring: the host waits on a step's events only when the ring wraps, so the
        // queue stays full while the sweeps are being timed.
        const int64_t R = acf_batch::kRing;
        auto drain = [&](int64_t slot) -> int {
            cudaEvent_t *e = b->ring + 3 * slot;
            ACF_CUDA(cudaEventSynchronize(e[2]));
            float x = 0, y = 0;
            ACF_CUDA(cudaEventElapsedTime(&x, e[0], e[1]));
            ACF_CUDA(cudaEventElapsedTime(&y, e[1], e[2]));
            b->prof_velocity_ms += x;
            b->prof_pressure_ms += y;
            b->prof_launches += 1;
            return ACF_OK;
        };
        for (int64_t t = 0; t < n_steps; t++) {
            const int64_t slot = t % R;
            if (t >= R) {
                int rc = drain(slot);
                if (rc) return rc;
            }
            launch_step<T>(b, 0, st, b->ring + 3 * slot);
            bump_step_base<<<1, 1, 0, st>>>(b->step_base, 1);
            b->launches += b->alternating() ? 2 : 3;
        }
        for (int64_t t = std::max<int64_t>(0, n_steps - R); t < n_steps; t++) {
            int rc = drain(t % R);
            if (rc) return rc;
        }
        ACF_CUDA(cudaGetLastError());
        return ACF_OK;
    }

    if constexpr (sizeof(T) == 4) {
        if (b->time_block == 2 && b->scheme == ACF_SCHEME_FUSED && b->rooms.size() == 1) {
            // Units of four steps (two launches) leave the relaxation states in the room's own
            // field and p, v in the copy that four single steps would; the rest are single steps.
            // A launch covers two full sweeps, so these are not captured in graphs.
            int64_t done = 0;
            for (; done + 4 <= n_steps; done += 4) {
                launch_pair(b, (int32_t)done, false, st);
                launch_pair(b, (int32_t)(done + 2), true, st);
            }
            for (; done < n_steps; done++) {
                launch_step<T>(b, (int32_t)done, st, nullptr);
                b->launches += 1;
            }
            ACF_CUDA(cudaGetLastError());
            return ACF_OK;
        }
    }

    int64_t done = 0;
    if (b->pressure_only() && b->po_first) {
        // The step from the p-v state is not the repeated one: launch it before any graph.
        launch_step<T>(b, 0, st, nullptr);
        bump_step_base<<<1, 1, 0, st>>>(b->step_base, 1);
        b->launches += 2;
        n_steps -= 1;
    }
    const bool fused = b->alternating();
    // A fused graph holds an even number of steps, so a replay leaves the buffers as it found
    // them; one graph is kept per starting buffer.
    const int64_t G = fused ? (b->graph_steps + 1) / 2 * 2 : b->graph_steps;
    const int kernels_per_step = fused ? 1 : 2;
    if (G > 0 && n_steps >= G) {
        if (b->graph_dirty) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            if (b->graph_odd) cudaGraphExecDestroy(b->graph_odd);
            b->graph = b->graph_odd = nullptr;
            b->graph_dirty = false;
        }
        cudaGraphExec_t &exec = (fused && b->rooms[0].cur) ? b->graph_odd : b->graph;
        if (!exec) {
            if (!b->capture_stream)
                ACF_CUDA(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
            ACF_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
            for (int64_t t = 0; t < G; t++) launch_step<T>(b, (int32_t)t, b->capture_stream, nullptr);
            bump_step_base<<<1, 1, 0, b->capture_stream>>>(b->step_base, G);
            cudaGraph_t graph = nullptr;
            ACF_CUDA(cudaStreamEndCapture(b->capture_stream, &graph));
            cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (err != cudaSuccess)
                return fail(ACF_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(err));
        }
        for (; done + G <= n_steps; done += G) {
            ACF_CUDA(cudaGraphLaunch(exec, st));
            b->launches += kernels_per_step * G + 1;
        }
    }
    for (int64_t t = 0; done + t < n_steps; t++) {
        launch_step<T>(b, (int32_t)t, st, nullptr);
        b->launches += kernels_per_step;
    }
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

template <typename T>
int energy_impl(acf_batch *b, int room, double dx, double *terms, cudaStream_t st, int i0, int i1,
                int i_faces) {
    const Room<T> s = make_room<T>(b, room);
    energy_partials<T><<<b->energy_blocks, 256, 0, st>>>(s, 1.0 / dx, b->energy_scratch, i0, i1,
                                                         i_faces);
    energy_finish<<<1, 32, 0, st>>>(b->energy_scratch, b->energy_blocks,
                                    b->energy_scratch + (size_t)b->energy_blocks * kEnergyTerms);
    b->launches += 2;
    ACF_CUDA(cudaGetLastError());
    ACF_CUDA(cudaMemcpyAsync(terms, b->energy_scratch + (size_t)b->energy_blocks * kEnergyTerms,
                             kEnergyTerms * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACF_CUDA(cudaStreamSynchronize(st));
    return ACF_OK;
}

// Reference shape of a field: (nx + [f==VX], ny + [f==VY], nz + [f==VZ]).
void field_shape(const RoomHost &h, int f, int64_t shape[3]) {
    shape[0] = h.nx + (f == ACF_FIELD_VX);
    shape[1] = h.ny + (f == ACF_FIELD_VY);
    shape[2] = h.nz + (f == ACF_FIELD_VZ);
}

int check_room(const acf_batch *b, int room) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (room < 0 || room >= (int)b->rooms.size())
        return fail(ACF_ERR_ARGUMENT, "room %d out of range (0..%d)", room, (int)b->rooms.size() - 1);
    return ACF_OK;
}

int check_field(const acf_batch *b, int room, int f) {
    int rc = check_room(b, room);
    if (rc) return rc;
    if (f < 0 || f >= b->n_fields())
        return fail(ACF_ERR_ARGUMENT, "field %d out of range (0..%d)", f, b->n_fields() - 1);
    return ACF_OK;
}

int copy_field(acf_batch *b, int room, int f, void *host_or_dev, bool upload, cudaStream_t st) {
    const RoomHost &h = b->rooms[room];
    int64_t shape[3];
    field_shape(h, f, shape);
    const size_t es = b->elem();
    cudaMemcpy3DParms p = {};
    cudaPitchedPtr dense = make_cudaPitchedPtr(host_or_dev, (size_t)shape[2] * es, (size_t)shape[2],
                                               (size_t)shape[1]);
    cudaPitchedPtr padded = make_cudaPitchedPtr(b->field_ptr(room, f), (size_t)h.pz * es, (size_t)h.pz,
                                                (size_t)(h.ny + 1));
    p.srcPtr = upload ? dense : padded;
    p.dstPtr = upload ? padded : dense;
    p.extent = make_cudaExtent((size_t)shape[2] * es, (size_t)shape[1], (size_t)shape[0]);
    p.kind = cudaMemcpyDefault;
    ACF_CUDA(cudaMemcpy3DAsync(&p, st));
    return ACF_OK;
}

template <typename T>
void cast_copy(void *dst, const double *src, size_t n) {
    T *d = (T *)dst;
    for (size_t q = 0; q < n; q++) d[q] = (T)src[q];
}

int upload_cast(void **dst, const std::vector<double> &host, size_t es) {
    std::vector<char> cast(std::max<size_t>(1, host.size()) * es, 0);
    if (es == 4) cast_copy<float>(cast.data(), host.data(), host.size());
    else cast_copy<double>(cast.data(), host.data(), host.size());
    ACF_CUDA(cudaMalloc(dst, cast.size()));
    ACF_CUDA(cudaMemcpy(*dst, cast.data(), cast.size(), cudaMemcpyHostToDevice));
    return ACF_OK;
}

void free_room(RoomHost &h) {
    cudaFree(h.second);
    cudaFree(h.profiles);
    cudaFree(h.shell);
    cudaFree(h.src_off);
    cudaFree(h.src_len);
    cudaFree(h.src_sig);
    cudaFree(h.rec_off);
    cudaFree(h.rec_start);
    cudaFree(h.rec);
    h = RoomHost();
}

void free_batch(acf_batch *b) {
    if (!b) return;
    DeviceGuard guard(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->graph_odd) cudaGraphExecDestroy(b->graph_odd);
    b->g_record.release();
    b->g_recompute.release();
    b->g_adjoint.release();
    b->g_adjoint_odd.release();
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    for (auto &e : b->ring)
        if (e) cudaEventDestroy(e);
    if (b->status_event) cudaEventDestroy(b->status_event);
    if (b->status_host) cudaFreeHost(b->status_host);
    for (auto &r : b->rooms) free_room(r);
    cudaFree(b->adj.hist_shell);
    cudaFree(b->adj.checkpoints);
    cudaFree(b->adj.scratch);
    cudaFree(b->adj.segment);
    cudaFree(b->adj.fields);
    cudaFree(b->adj.fields2);
    cudaFree(b->adj.grad_shell);
    cudaFree(b->adj.air_partials);
    cudaFree(b->adj.grad_rec);
    cudaFree(b->adj.grad_src);
    for (auto &ra : b->badj) {
        cudaFree(ra.hist_shell);
        cudaFree(ra.fields);
        cudaFree(ra.fields2);
        cudaFree(ra.grad_shell);
        cudaFree(ra.grad_rec);
        cudaFree(ra.grad_src);
    }
    cudaFree(b->badj_table);
    cudaFree(b->pair_ring);
    cudaFree(b->pair_progress);
    cudaFree(b->psi2);
    cudaFree(b->state);
    cudaFree(b->room_table);
    cudaFree(b->fused_table);
    cudaFree(b->tiles);
    cudaFree(b->step_base);
    cudaFree(b->energy_scratch);
    delete b;
}

int validate_config(const acf_config *cfg, int index) {
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1)
        return fail(ACF_ERR_ARGUMENT, "room %d: cell counts must be >= 1, got (%d, %d, %d)", index, cfg->nx,
                    cfg->ny, cfg->nz);
    if (cfg->precision != 4 && cfg->precision != 8)
        return fail(ACF_ERR_ARGUMENT, "room %d: precision must be 4 or 8 bytes, got %d", index, cfg->precision);
    if (cfg->n_relax < 0 || cfg->n_relax > ACF_MAX_RELAXATION)
        return fail(ACF_ERR_ARGUMENT, "room %d: the kernel holds at most %d relaxation processes, got %d",
                    index, ACF_MAX_RELAXATION, cfg->n_relax);
    const bool layer = cfg->cell[0] != nullptr;
    for (int a = 0; a < 3; a++)
        if ((cfg->cell[a] != nullptr) != layer || (cfg->face[a] != nullptr) != layer)
            return fail(ACF_ERR_ARGUMENT, "room %d: layer profiles must be all given or all NULL", index);
    const bool walls = cfg->wall_shell[0] != nullptr;
    for (int f = 0; f < 6; f++)
        if ((cfg->wall_shell[f] != nullptr) != walls)
            return fail(ACF_ERR_ARGUMENT, "room %d: wall shells must be all given or all NULL", index);
    if ((int64_t)cfg->nx * cfg->ny > INT32_MAX / 2 || (int64_t)cfg->ny * ((cfg->nz + 3) / 4) > INT32_MAX / 2)
        return fail(ACF_ERR_ARGUMENT, "room %d: grid too large", index);
    return ACF_OK;
}

// Allocate and fill every room of a batch (single rooms are batches of one).
int create_batch(int32_t n_rooms, const acf_config *configs, acf_batch *b) {
    if (n_rooms < 1) return fail(ACF_ERR_ARGUMENT, "a batch needs at least one room");
    for (int r = 0; r < n_rooms; r++) {
        int rc = validate_config(configs + r, r);
        if (rc) return rc;
        if (configs[r].precision != configs[0].precision)
            return fail(ACF_ERR_ARGUMENT, "room %d: every room of a batch must have the same precision", r);
        if (configs[r].n_relax != configs[0].n_relax)
            return fail(ACF_ERR_ARGUMENT, "room %d: every room of a batch must have the same number of "
                        "relaxation processes", r);
    }
    ACF_CUDA(cudaGetDevice(&b->device));
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, b->device);
    b->l2_bytes = l2;
    b->precision = configs[0].precision;
    b->n_relax = configs[0].n_relax;
    b->rooms.resize((size_t)n_rooms);
    const size_t es = b->elem();
    size_t offset = 0;
    for (int r = 0; r < n_rooms; r++) {
        const acf_config &c = configs[r];
        RoomHost &h = b->rooms[r];
        h.nx = c.nx;
        h.ny = c.ny;
        h.nz = c.nz;
        h.n_relax = c.n_relax;
        h.pz = round_up((int64_t)c.nz + 1, kRowAlign);
        h.plane = (int64_t)(c.ny + 1) * h.pz;
        h.field = (int64_t)(c.nx + 1) * h.plane;
        h.has_layer = c.cell[0] != nullptr;
        h.has_walls = c.wall_shell[0] != nullptr;
        b->any_layer |= h.has_layer;
        b->any_walls |= h.has_walls;
        h.coef[0] = c.vel_coef;
        h.coef[1] = c.pres_coef;
        h.coef[2] = c.src_coef;
        h.coef[3] = c.relax_scale;
        for (int q = 0; q < ACF_MAX_RELAXATION; q++) {
            h.decay[q] = q < c.n_relax ? c.relax_decay[q] : 0.0;
            h.mean[q] = q < c.n_relax ? c.relax_mean[q] : 0.0;
            h.gain[q] = q < c.n_relax ? c.relax_gain[q] : 0.0;
        }
        h.state_off = offset;
        // One guard row past the last field keeps every vector access of the last row in
        // bounds; rooms start on 256-byte boundaries.
        offset += (size_t)round_up(((int64_t)b->n_fields() * h.field + h.pz) * (int64_t)es, 256);
    }
    b->state_bytes = offset;
    // Test hook: ACF_INJECT_ALLOC_FAILURE set (non-empty, not "0") makes this allocation fail
    // as an exhausted device would, before any device memory is taken.
    if (const char *inject = getenv("ACF_INJECT_ALLOC_FAILURE"); inject && *inject && strcmp(inject, "0") != 0)
        return fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes of state failed (injected by "
                    "ACF_INJECT_ALLOC_FAILURE)", b->state_bytes);
    if (cudaMalloc(&b->state, b->state_bytes) != cudaSuccess)
        return fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes of state failed", b->state_bytes);
    ACF_CUDA(cudaMemset(b->state, 0, b->state_bytes));

    const bool batched = n_rooms > 1;
    for (int r = 0; r < n_rooms; r++) {
        const acf_config &c = configs[r];
        RoomHost &h = b->rooms[r];
        const int64_t n_axis[3] = {c.nx, c.ny, c.nz};
        // In a batch every room carries what any room needs; the neutral values (profiles of
        // one, wall pairs (1, 0)) leave its arithmetic exactly as without the feature.
        if (h.has_layer || (batched && b->any_layer)) {
            std::vector<double> host;
            for (int a = 0; a < 3; a++) {
                h.profile_off[a] = (int64_t)host.size();
                if (h.has_layer) host.insert(host.end(), c.cell[a], c.cell[a] + n_axis[a]);
                else host.insert(host.end(), (size_t)n_axis[a], 1.0);
            }
            for (int a = 0; a < 3; a++) {
                h.profile_off[3 + a] = (int64_t)host.size();
                if (h.has_layer) host.insert(host.end(), c.face[a], c.face[a] + n_axis[a] + 1);
                else host.insert(host.end(), (size_t)n_axis[a] + 1, 1.0);
            }
            int rc = upload_cast(&h.profiles, host, es);
            if (rc) return rc;
        }
        if (h.has_walls || (batched && b->any_walls)) {
            std::vector<double> host;
            for (int f = 0; f < 6; f++) {
                const int axis = f / 2;
                const int64_t nb = axis == 0 ? n_axis[1] : n_axis[0];
                const int64_t nc = axis == 2 ? n_axis[1] : n_axis[2];
                h.shell_off[f] = (int64_t)host.size();
                if (h.has_walls) {
                    host.insert(host.end(), c.wall_shell[f], c.wall_shell[f] + 2 * nb * nc);
                } else {
                    for (int64_t q = 0; q < nb * nc; q++) {
                        host.push_back(1.0);
                        host.push_back(0.0);
                    }
                }
            }
            int rc = upload_cast(&h.shell, host, es);
            if (rc) return rc;
        }
    }

    if (cudaMalloc(&b->step_base, 2 * sizeof(int64_t)) != cudaSuccess)
        return fail(ACF_ERR_MEMORY, "cudaMalloc of step counter failed");
    ACF_CUDA(cudaMemset(b->step_base, 0, 2 * sizeof(int64_t)));
    if (cudaHostAlloc((void **)&b->status_host, sizeof(int32_t), cudaHostAllocDefault) != cudaSuccess)
        return fail(ACF_ERR_MEMORY, "pinned status word allocation failed");
    *b->status_host = 0;
    ACF_CUDA(cudaEventCreateWithFlags(&b->status_event, cudaEventDisableTiming));
    cudaDeviceGetAttribute(&b->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, b->device);
    cudaDeviceGetAttribute(&b->smem_per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    b->energy_blocks = 4 * b->sms;
    const size_t scratch = ((size_t)b->energy_blocks + 1) * kEnergyTerms * sizeof(double);
    if (cudaMalloc(&b->energy_scratch, scratch) != cudaSuccess)
        return fail(ACF_ERR_MEMORY, "cudaMalloc of energy scratch failed");
    for (auto &ev : b->ring) ACF_CUDA(cudaEventCreate(&ev));
    if (batched) {
        // one CTA per tile of 128 (row, chunk) pairs x 8 planes: the best measured schedule on
        // uneven-room batches (persistent grids lose to the hardware scheduler here)
        b->block_threads = 128;
        b->planes = 8;
        b->ctas_per_sm = 0;
    } else {
        b->block_threads = 128;
        // staged scheme: two rows of 4-element threads where they fit in 256 threads (measured
        // best at 384^3), with the automatic ring depth
        const int bx4 = (int)round_up((b->rooms[0].nz + 3) / 4, 32);
        b->staged_rows = 2 * bx4 <= kStagedMaxConsumers ? 2 : 1;
        b->staged_vector = 4;
        b->planes = 4;
        while ((b->rooms[0].nx + b->planes - 1) / b->planes > 65535) b->planes *= 2;
    }
    return batched ? build_tiles(b) : ACF_OK;
}

int set_sources(acf_batch *b, int room, int64_t n, const int64_t *cell, const int64_t *length,
                const double *signal, int64_t stride) {
    int rc = check_room(b, room);
    if (rc) return rc;
    if (n < 0 || n > (1 << 20)) return fail(ACF_ERR_ARGUMENT, "source count %lld out of range", (long long)n);
    if (n > 0 && (!cell || !length || (stride > 0 && !signal) || stride < 0))
        return fail(ACF_ERR_ARGUMENT, "null source arrays");
    RoomHost &h = b->rooms[room];
    DeviceGuard guard(b->device);
    std::vector<int64_t> off((size_t)n), len((size_t)n);
    for (int64_t q = 0; q < n; q++) {
        if (cell[q] < 0 || cell[q] >= h.n_cells())
            return fail(ACF_ERR_ARGUMENT, "source %lld cell %lld outside the grid", (long long)q, (long long)cell[q]);
        if (length[q] < 0 || length[q] > stride)
            return fail(ACF_ERR_ARGUMENT, "source %lld length %lld exceeds stride %lld", (long long)q,
                        (long long)length[q], (long long)stride);
        off[q] = h.padded_offset(cell[q]);
        len[q] = length[q];
    }
    ACF_CUDA(cudaDeviceSynchronize());
    cudaFree(h.src_off);
    cudaFree(h.src_len);
    cudaFree(h.src_sig);
    h.src_off = h.src_len = nullptr;
    h.src_sig = nullptr;
    h.n_src = 0;
    b->graph_dirty = b->adj_graphs_dirty = true;
    b->room_table_dirty = true;
    if (n == 0) return ACF_OK;
    const size_t es = b->elem();
    // padded offsets, then their in-plane offsets
    for (int64_t q = 0; q < n; q++) off.push_back(off[q] % h.plane);
    ACF_CUDA(cudaMalloc(&h.src_off, 2 * n * sizeof(int64_t)));
    ACF_CUDA(cudaMalloc(&h.src_len, n * sizeof(int64_t)));
    ACF_CUDA(cudaMemcpy(h.src_off, off.data(), 2 * n * sizeof(int64_t), cudaMemcpyHostToDevice));
    ACF_CUDA(cudaMemcpy(h.src_len, len.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    std::vector<double> host((size_t)n * (size_t)std::max<int64_t>(stride, 1), 0.0);
    if (stride > 0) std::copy(signal, signal + (size_t)n * stride, host.begin());
    rc = upload_cast(&h.src_sig, host, es);
    if (rc) return rc;
    h.n_src = n;
    h.src_stride = stride;
    return ACF_OK;
}

int set_receivers(acf_batch *b, int room, int64_t n, const int64_t *cell, const int64_t *start_step) {
    int rc = check_room(b, room);
    if (rc) return rc;
    if (n < 0 || n > (1 << 20)) return fail(ACF_ERR_ARGUMENT, "receiver count %lld out of range", (long long)n);
    if (n > 0 && (!cell || !start_step)) return fail(ACF_ERR_ARGUMENT, "null receiver arrays");
    RoomHost &h = b->rooms[room];
    DeviceGuard guard(b->device);
    std::vector<int64_t> off((size_t)n);
    for (int64_t r = 0; r < n; r++) {
        if (cell[r] < 0 || cell[r] >= h.n_cells())
            return fail(ACF_ERR_ARGUMENT, "receiver %lld cell %lld outside the grid", (long long)r, (long long)cell[r]);
        if (start_step[r] < 0) return fail(ACF_ERR_ARGUMENT, "negative start step");
        off[r] = h.padded_offset(cell[r]);
    }
    int64_t origin = h.rec_origin;
    if (n > 0 && !h.rec_origin_set) origin = *std::min_element(start_step, start_step + n);
    for (int64_t r = 0; r < n; r++)
        if (start_step[r] < origin)
            return fail(ACF_ERR_ARGUMENT, "receiver %lld starts before the recording origin", (long long)r);
    ACF_CUDA(cudaDeviceSynchronize());
    if (n > 0 && !h.rec_origin_set) {
        h.rec_origin = origin;
        h.rec_origin_set = true;
    }
    // Keep existing recordings: grow the row count, preserving rows already written.
    const size_t es = b->elem();
    if (n > 0 && h.rec_capacity > 0 && n != h.n_rec) {
        void *grown = nullptr;
        ACF_CUDA(cudaMalloc(&grown, (size_t)n * h.rec_capacity * es));
        ACF_CUDA(cudaMemset(grown, 0, (size_t)n * h.rec_capacity * es));
        const int64_t keep = std::min<int64_t>(n, h.n_rec);
        if (keep > 0 && h.rec)
            ACF_CUDA(cudaMemcpy(grown, h.rec, (size_t)keep * h.rec_capacity * es, cudaMemcpyDeviceToDevice));
        cudaFree(h.rec);
        h.rec = grown;
    }
    cudaFree(h.rec_off);
    cudaFree(h.rec_start);
    h.rec_off = h.rec_start = nullptr;
    h.n_rec = 0;
    b->graph_dirty = b->adj_graphs_dirty = true;
    b->room_table_dirty = true;
    h.host_rec_start.assign(start_step, start_step + n);
    if (n == 0) return ACF_OK;
    for (int64_t r = 0; r < n; r++) off.push_back(off[r] % h.plane);   // then in-plane offsets
    ACF_CUDA(cudaMalloc(&h.rec_off, 2 * n * sizeof(int64_t)));
    ACF_CUDA(cudaMalloc(&h.rec_start, n * sizeof(int64_t)));
    ACF_CUDA(cudaMemcpy(h.rec_off, off.data(), 2 * n * sizeof(int64_t), cudaMemcpyHostToDevice));
    ACF_CUDA(cudaMemcpy(h.rec_start, start_step, n * sizeof(int64_t), cudaMemcpyHostToDevice));
    h.n_rec = n;
    return ACF_OK;
}

int read_recording(acf_batch *b, int room, int64_t r, int64_t first_step, int64_t n, void *dst,
                   acf_stream stream) {
    int rc = check_room(b, room);
    if (rc) return rc;
    RoomHost &h = b->rooms[room];
    if (r < 0 || r >= h.n_rec) return fail(ACF_ERR_ARGUMENT, "receiver %lld out of range", (long long)r);
    if (n < 0 || (n > 0 && !dst)) return fail(ACF_ERR_ARGUMENT, "bad destination");
    if (n == 0) return ACF_OK;
    const int64_t col = first_step - h.rec_origin;
    if (col < 0 || col + n > h.rec_capacity || first_step < h.host_rec_start[(size_t)r])
        return fail(ACF_ERR_ARGUMENT, "steps [%lld, %lld) were not recorded by receiver %lld",
                    (long long)first_step, (long long)(first_step + n), (long long)r);
    DeviceGuard guard(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t es = b->elem();
    ACF_CUDA(cudaMemcpyAsync(dst, (char *)h.rec + ((size_t)r * h.rec_capacity + col) * es, (size_t)n * es,
                             cudaMemcpyDefault, st));
    ACF_CUDA(cudaStreamSynchronize(st));
    return ACF_OK;
}

// Recording capacity for every step a run of [step_offset, step_offset + n_steps) can write.
int ensure_recording(acf_batch *b, int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    for (RoomHost &h : b->rooms) {
        if (h.n_rec == 0) continue;
        const int64_t need = step_offset + n_steps - h.rec_origin;
        if (need <= h.rec_capacity) continue;
        int64_t cap = round_up(std::max<int64_t>(need, 2 * h.rec_capacity), 256);
        const size_t es = b->elem();
        void *grown = nullptr;
        ACF_CUDA(cudaStreamSynchronize(st));
        ACF_CUDA(cudaMalloc(&grown, (size_t)h.n_rec * cap * es));
        ACF_CUDA(cudaMemset(grown, 0, (size_t)h.n_rec * cap * es));
        if (h.rec && h.rec_capacity > 0)
            ACF_CUDA(cudaMemcpy2D(grown, (size_t)cap * es, h.rec, (size_t)h.rec_capacity * es,
                                  (size_t)h.rec_capacity * es, (size_t)h.n_rec, cudaMemcpyDeviceToDevice));
        cudaFree(h.rec);
        h.rec = grown;
        h.rec_capacity = cap;
        b->graph_dirty = b->adj_graphs_dirty = true;
        b->room_table_dirty = true;
    }
    return ACF_OK;
}

// The status copied after the previous run, if it has landed: ACF_ERR_NUMERIC when a sweep saw a
// non-finite pressure, ACF_ERR_STATE when a staged sweep's wait ran out (the state is then not
// valid either way). Never waits for the device.
int pending_status(acf_batch *b) {
    if (!b->status_pending) return ACF_OK;
    const cudaError_t q = cudaEventQuery(b->status_event);
    if (q == cudaErrorNotReady) return ACF_OK;
    if (q != cudaSuccess) return fail(ACF_ERR_CUDA, "status event: %s", cudaGetErrorString(q));
    b->status_pending = false;
    const int32_t word = *b->status_host;
    if (word & kStatusNonFinite)
        return fail(ACF_ERR_NUMERIC, "a sweep produced a non-finite pressure (NaN or infinity) in "
                    "an earlier run; the state is not valid");
    if (word & kStatusWaitTimeout)
        return fail(ACF_ERR_STATE, "a staged sweep gave up waiting for its bulk copies in an "
                    "earlier run; the state is not valid");
    return ACF_OK;
}

int run_batch(acf_batch *b, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (n_steps < 0 || step_offset < 0) return fail(ACF_ERR_ARGUMENT, "negative step count or offset");
    if (n_steps == 0) return ACF_OK;
    DeviceGuard guard(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = pending_status(b);
    if (rc) return rc;
    rc = ensure_recording(b, n_steps, step_offset, st);
    if (rc) return rc;
    rc = b->precision == 8 ? run_impl<double>(b, n_steps, step_offset, st)
                           : run_impl<float>(b, n_steps, step_offset, st);
    if (rc) return rc;
    // The status word after this run, read by the next run once the copy has landed (a run
    // captured into the caller's graph leaves it to acf_device_status).
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    ACF_CUDA(cudaStreamIsCapturing(st, &capturing));
    if (capturing == cudaStreamCaptureStatusNone) {
        ACF_CUDA(cudaMemcpyAsync(b->status_host, b->error_flag(), sizeof(int32_t),
                                 cudaMemcpyDeviceToHost, st));
        ACF_CUDA(cudaEventRecord(b->status_event, st));
        b->status_pending = true;
    }
    return ACF_OK;
}

// A room cut into x slabs, one single-room two-sweep solver per part, advanced together. Each
// step launches every part's velocity sweep, then every part's pressure sweep; a pressure
// sweep updates its own planes only and stores its first and last of them into the
// neighbours' ghost planes as well (peer stores when a neighbour lives on another GPU), so no
// exchange follows the step. Parts on one GPU run in launch order on `st`. Parts on several
// GPUs run on each device's default stream, ordered by events and never by a wait inside a
// kernel: a velocity sweep waits for the neighbours' pressure sweeps of the previous step
// (they wrote its ghost planes), a pressure sweep for the neighbours' velocity sweeps of the
// same step (they read the ghost planes it overwrites).
// The fused step of every part of a slab group, for the parity the parts are at: each part
// reads its current copy and writes its next one; its p store skips the ghost planes, and its
// first and last own planes also go to the neighbours' ghost planes in the neighbours' NEXT
// copies (what they read at the following step). All parameters are formed before any part's
// copy flips; `after(q)` runs after part q's launch (an event record across GPUs).
template <typename T, typename After>
void fused_slab_step(acf_batch *const *parts, int n, const int32_t *own_lo, const int32_t *own_hi,
                     int32_t local, const std::vector<cudaStream_t> &streams, After after) {
    std::vector<FusedParams<T>> f((size_t)n);
    for (int q = 0; q < n; q++) {
        acf_batch *b = parts[q];
        FusedParams<T> &x = f[q];
        x = FusedParams<T>{};
        x.room = make_room<T>(b, 0);
        x.room.own_lo = own_lo[q];
        x.room.own_hi = own_hi[q];
        if (q > 0)
            x.room.ghost_lo = (T *)parts[q - 1]->other_ptr(0, ACF_FIELD_P) + (int64_t)own_hi[q - 1] * x.room.plane;
        if (q + 1 < n)
            x.room.ghost_hi = (T *)parts[q + 1]->other_ptr(0, ACF_FIELD_P) +
                              (int64_t)(own_lo[q + 1] - 1) * x.room.plane;
        x.np = (T *)b->other_ptr(0, ACF_FIELD_P);
        x.nvx = (T *)b->other_ptr(0, ACF_FIELD_VX);
        x.nvy = (T *)b->other_ptr(0, ACF_FIELD_VY);
        x.nvz = (T *)b->other_ptr(0, ACF_FIELD_VZ);
        x.step_base = b->step_base;
        x.local_step = local;
        x.planes = b->planes;
    }
    if constexpr (sizeof(T) == 4) {
        // Parts on one GPU with the same features and nz a multiple of 4: one launch per
        // kMaxLeanParts parts instead of one per part.
        bool combined = true;
        const RoomHost &h0 = parts[0]->rooms[0];
        for (int q = 0; q < n; q++) {
            const RoomHost &h = parts[q]->rooms[0];
            combined = combined && streams[q] == streams[0] && parts[q]->device == parts[0]->device &&
                       h.nz % kVec == 0 && h.ny == h0.ny && h.nz == h0.nz && h.has_layer == h0.has_layer &&
                       h.has_walls == h0.has_walls && h.n_relax == h0.n_relax &&
                       parts[q]->block_threads == parts[0]->block_threads;
        }
        if (combined && n > 1) {
            DeviceGuard g(parts[0]->device);
            for (int q0 = 0; q0 < n; q0 += kMaxLeanParts) {
                const int m = std::min(kMaxLeanParts, n - q0);
                LeanPartsParams lp{};
                lp.n = m;
                LaunchShape L{};
                int groups = 0;
                for (int k = 0; k < m; k++) {
                    const int q = q0 + k;
                    lp.part[k].f = f[q];
                    fill_pairs(lp.part[k].pairs, parts[q]->rooms[0]);
                    L = single_shape(parts[q]);
                    lp.first_group[k] = groups;
                    groups += (int)L.grid.z;
                }
                lp.first_group[m] = groups;
                L.grid.z = (unsigned)groups;
                dispatch_pressure<float, LeanPartsStep>(h0.has_layer, h0.has_walls, h0.n_relax, lp, L.grid,
                                                        L.block, streams[0]);
                parts[q0]->launches += 1;
            }
            for (int q = 0; q < n; q++) {
                after(q);
                parts[q]->rooms[0].cur ^= 1;
            }
            return;
        }
    }
    for (int q = 0; q < n; q++) {
        DeviceGuard g(parts[q]->device);
        const RoomHost &h = parts[q]->rooms[0];
        const LaunchShape L = single_shape(parts[q]);
        if constexpr (sizeof(T) == 4) {
            LeanParams lp{};
            lp.f = f[q];
            fill_pairs(lp.pairs, h);
            if (h.nz % kVec == 0)
                dispatch_pressure<float, LeanStep>(h.has_layer, h.has_walls, h.n_relax, lp, L.grid, L.block, streams[q]);
            else
                dispatch_pressure<float, LeanStepPadded>(h.has_layer, h.has_walls, h.n_relax, lp, L.grid,
                                                         L.block, streams[q]);
        } else {
            dispatch_pressure<T, FusedStep>(h.has_layer, h.has_walls, h.n_relax, f[q], L.grid, L.block, streams[q]);
        }
        parts[q]->launches += 1;
        after(q);
    }
    for (int q = 0; q < n; q++) parts[q]->rooms[0].cur ^= 1;
}

// Slab groups on the fused scheme: one launch per part and step. On one GPU the steps replay
// from a CUDA graph of an even number of steps (the copies come back to the same parity);
// across GPUs each part's step waits, by events, for its neighbours' previous step (which wrote
// its ghost planes and read the copy it now writes into theirs).
template <typename T>
int run_fused_slabs(acf_batch *const *parts, int n, const int32_t *own_lo, const int32_t *own_hi,
                    int64_t n_steps, int64_t step_offset, cudaStream_t st, bool one_device) {
    std::vector<cudaStream_t> streams((size_t)n, one_device ? st : (cudaStream_t)0);
    for (int q = 0; q < n; q++) {
        DeviceGuard g(parts[q]->device);
        set_step_base<<<1, 1, 0, streams[q]>>>(parts[q]->step_base, step_offset);
        parts[q]->launches += 1;
    }
    int64_t done = 0;
    if (one_device) {
        const int64_t G = 64;
        if (n_steps >= G) {
            cudaStream_t cap = nullptr;
            ACF_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            std::vector<cudaStream_t> cs((size_t)n, cap);
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            cudaError_t err = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                for (int64_t t = 0; t < G; t++) fused_slab_step<T>(parts, n, own_lo, own_hi, (int32_t)t, cs, [](int) {});
                for (int q = 0; q < n; q++) bump_step_base<<<1, 1, 0, cap>>>(parts[q]->step_base, G);
                err = cudaStreamEndCapture(cap, &graph);
            }
            if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            for (; err == cudaSuccess && done + G <= n_steps; done += G) {
                err = cudaGraphLaunch(exec, st);
                for (int q = 0; q < n; q++) parts[q]->launches += G + 1;
            }
            if (exec) cudaGraphExecDestroy(exec);
            cudaStreamDestroy(cap);
            if (err != cudaSuccess) return fail(ACF_ERR_CUDA, "slab graph: %s", cudaGetErrorString(err));
        }
        for (int64_t t = 0; done + t < n_steps; t++)
            fused_slab_step<T>(parts, n, own_lo, own_hi, (int32_t)t, streams, [](int) {});
        ACF_CUDA(cudaGetLastError());
        return ACF_OK;
    }
    std::vector<cudaEvent_t> done_ev((size_t)n, nullptr);
    auto release = [&]() {
        for (int q = 0; q < n; q++) {
            DeviceGuard g(parts[q]->device);
            if (done_ev[q]) cudaEventDestroy(done_ev[q]);
        }
    };
    for (int q = 0; q < n; q++) {
        DeviceGuard g(parts[q]->device);
        if (cudaEventCreateWithFlags(&done_ev[q], cudaEventDisableTiming) != cudaSuccess) {
            release();
            return fail(ACF_ERR_CUDA, "event creation failed");
        }
    }
    for (int64_t t = 0; t < n_steps; t++) {
        if (t > 0)
            for (int q = 0; q < n; q++) {
                DeviceGuard g(parts[q]->device);
                for (int r : {q - 1, q + 1})
                    if (r >= 0 && r < n) cudaStreamWaitEvent(streams[q], done_ev[r], 0);
            }
        fused_slab_step<T>(parts, n, own_lo, own_hi, (int32_t)t, streams,
                           [&](int q) { cudaEventRecord(done_ev[q], streams[q]); });
    }
    const cudaError_t e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return fail(ACF_ERR_CUDA, "slab step: %s", cudaGetErrorString(e));
    return ACF_OK;
}

template <typename T>
int run_slabs_impl(acf_batch *const *parts, int n, const int32_t *own_lo, const int32_t *own_hi,
                   int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    bool one_device = true;
    for (int q = 1; q < n; q++) one_device = one_device && parts[q]->device == parts[0]->device;
    std::vector<StepParams<T>> params((size_t)n);
    std::vector<LaunchShape> shapes((size_t)n);
    for (int q = 0; q < n; q++) {
        acf_batch *b = parts[q];
        StepParams<T> &p = params[q];
        p.room = make_room<T>(b, 0);
        p.room.own_lo = own_lo[q];
        p.room.own_hi = own_hi[q];
        if (q > 0)   // the left neighbour's right ghost plane: just past its own planes
            p.room.ghost_lo = (T *)parts[q - 1]->field_ptr(0, ACF_FIELD_P) + (int64_t)own_hi[q - 1] * p.room.plane;
        if (q + 1 < n)   // the right neighbour's left ghost plane: just before its own planes
            p.room.ghost_hi = (T *)parts[q + 1]->field_ptr(0, ACF_FIELD_P) + (int64_t)(own_lo[q + 1] - 1) * p.room.plane;
        p.step_base = b->step_base;
        p.planes = b->planes;
        shapes[q] = single_shape(b);
    }
    std::vector<cudaStream_t> streams((size_t)n, one_device ? st : (cudaStream_t)0);
    std::vector<cudaEvent_t> vel_done((size_t)n, nullptr), pres_done((size_t)n, nullptr);
    auto release = [&]() {
        for (int q = 0; q < n; q++) {
            DeviceGuard g(parts[q]->device);
            if (vel_done[q]) cudaEventDestroy(vel_done[q]);
            if (pres_done[q]) cudaEventDestroy(pres_done[q]);
        }
    };
    if (!one_device) {
        for (int q = 0; q < n; q++) {
            DeviceGuard g(parts[q]->device);
            for (int r : {q - 1, q + 1}) {
                if (r < 0 || r >= n || parts[r]->device == parts[q]->device) continue;
                int can = 0;
                cudaDeviceCanAccessPeer(&can, parts[q]->device, parts[r]->device);
                if (!can) {
                    release();
                    return fail(ACF_ERR_STATE, "GPU %d cannot store into GPU %d's memory",
                                parts[q]->device, parts[r]->device);
                }
                const cudaError_t e = cudaDeviceEnablePeerAccess(parts[r]->device, 0);
                if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
                else if (e != cudaSuccess) {
                    release();
                    return fail(ACF_ERR_CUDA, "peer access %d -> %d: %s", parts[q]->device,
                                parts[r]->device, cudaGetErrorString(e));
                }
            }
            if (cudaEventCreateWithFlags(&vel_done[q], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&pres_done[q], cudaEventDisableTiming) != cudaSuccess) {
                release();
                return fail(ACF_ERR_CUDA, "event creation failed");
            }
        }
    }
    auto wait_neighbours = [&](int q, const std::vector<cudaEvent_t> &done) {
        for (int r : {q - 1, q + 1})
            if (r >= 0 && r < n) cudaStreamWaitEvent(streams[q], done[r], 0);
    };
    for (int q = 0; q < n; q++) {
        DeviceGuard g(parts[q]->device);
        set_step_base<<<1, 1, 0, streams[q]>>>(parts[q]->step_base, step_offset);
        parts[q]->launches += 1;
    }
    for (int64_t t = 0; t < n_steps; t++) {
        for (int q = 0; q < n; q++) {
            DeviceGuard g(parts[q]->device);
            if (!one_device && t > 0) wait_neighbours(q, pres_done);
            StepParams<T> &p = params[q];
            p.local_step = (int32_t)t;
            const LaunchShape &L = shapes[q];
            if (parts[q]->rooms[0].has_layer) velocity_sweep<T, true><<<L.grid, L.block, 0, streams[q]>>>(p);
            else velocity_sweep<T, false><<<L.grid, L.block, 0, streams[q]>>>(p);
            if (!one_device) cudaEventRecord(vel_done[q], streams[q]);
        }
        for (int q = 0; q < n; q++) {
            DeviceGuard g(parts[q]->device);
            if (!one_device) wait_neighbours(q, vel_done);
            const RoomHost &h = parts[q]->rooms[0];
            dispatch_pressure<T, SinglePressure>(h.has_layer, h.has_walls, h.n_relax, params[q],
                                                 shapes[q].grid, shapes[q].block, streams[q]);
            if (!one_device) cudaEventRecord(pres_done[q], streams[q]);
            parts[q]->launches += 2;
        }
    }
    const cudaError_t e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return fail(ACF_ERR_CUDA, "slab step: %s", cudaGetErrorString(e));
    return ACF_OK;
}

int run_slabs(acf_solver *const *parts, int32_t n, const int32_t *own_lo, const int32_t *own_hi,
              int64_t n_steps, int64_t step_offset, acf_stream stream) {
    if (!parts || !own_lo || !own_hi || n < 1) return fail(ACF_ERR_ARGUMENT, "null or empty part list");
    if (n_steps < 0 || step_offset < 0) return fail(ACF_ERR_ARGUMENT, "negative step count or offset");
    for (int q = 0; q < n; q++) {
        const acf_batch *b = parts[q];
        if (!b) return fail(ACF_ERR_ARGUMENT, "null part %d", q);
        const RoomHost &h = b->rooms[0];
        const RoomHost &h0 = parts[0]->rooms[0];
        if (b->scheme != parts[0]->scheme ||
            (b->scheme != ACF_SCHEME_TWO_SWEEPS && b->scheme != ACF_SCHEME_FUSED))
            return fail(ACF_ERR_STATE, "part %d: slabs step with the two-sweep or the fused scheme, "
                        "the same for every part", q);
        if (b->rooms[0].cur != parts[0]->rooms[0].cur)
            return fail(ACF_ERR_STATE, "part %d: the fused copies of the parts are out of step", q);
        if (b->precision != parts[0]->precision || h.ny != h0.ny || h.nz != h0.nz)
            return fail(ACF_ERR_ARGUMENT, "part %d differs in precision, ny or nz", q);
        const bool left = q > 0, right = q + 1 < n;
        if (own_lo[q] != (left ? 1 : 0) || own_hi[q] <= own_lo[q] || own_hi[q] != h.nx - (right ? 1 : 0))
            return fail(ACF_ERR_ARGUMENT, "part %d: own planes [%d, %d) do not fit %d planes with "
                        "ghosts", q, own_lo[q], own_hi[q], h.nx);
    }
    bool one_device = true;
    for (int q = 1; q < n; q++) one_device = one_device && parts[q]->device == parts[0]->device;
    // A stream belongs to one device: parts on several GPUs run on each device's legacy default
    // stream (ordered by events between devices), so a caller's stream could order nothing.
    if (!one_device && stream != nullptr)
        return fail(ACF_ERR_ARGUMENT, "parts on several GPUs: pass a null stream (each device's "
                    "default stream is used)");
    if (n_steps == 0) return ACF_OK;
    for (int q = 0; q < n; q++) {
        DeviceGuard g(parts[q]->device);
        int rc = ensure_recording(parts[q], n_steps, step_offset, (cudaStream_t)stream);
        if (rc) return rc;
    }
    DeviceGuard guard(parts[0]->device);
    acf_batch *const *b = (acf_batch *const *)parts;
    if (parts[0]->scheme == ACF_SCHEME_FUSED)
        return parts[0]->precision == 8
                   ? run_fused_slabs<double>(b, n, own_lo, own_hi, n_steps, step_offset, (cudaStream_t)stream, one_device)
                   : run_fused_slabs<float>(b, n, own_lo, own_hi, n_steps, step_offset, (cudaStream_t)stream, one_device);
    return parts[0]->precision == 8
               ? run_slabs_impl<double>(b, n, own_lo, own_hi, n_steps, step_offset, (cudaStream_t)stream)
               : run_slabs_impl<float>(b, n, own_lo, own_hi, n_steps, step_offset, (cudaStream_t)stream);
}

int set_launch(acf_batch *b, int32_t block_threads, int32_t planes, int32_t ctas_per_sm) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (block_threads < 32 || block_threads > 256 || (block_threads & (block_threads - 1)))
        return fail(ACF_ERR_ARGUMENT, "block_threads must be a power of two in [32, 256], got %d", block_threads);
    if (planes < 1 || planes > 1024) return fail(ACF_ERR_ARGUMENT, "planes must be in [1, 1024], got %d", planes);
    if (ctas_per_sm < 0 || ctas_per_sm > 32)
        return fail(ACF_ERR_ARGUMENT, "ctas_per_sm must be in [0, 32] (0: one CTA per tile), got %d", ctas_per_sm);
    if (b->rooms.size() == 1 && (b->rooms[0].nx + planes - 1) / planes > 65535)
        return fail(ACF_ERR_ARGUMENT, "nx / planes exceeds the 65535 grid limit; use more planes per block");
    DeviceGuard guard(b->device);
    const bool changed = block_threads != b->block_threads || planes != b->planes || ctas_per_sm != b->ctas_per_sm;
    b->block_threads = block_threads;
    b->planes = planes;
    b->ctas_per_sm = ctas_per_sm;
    if (changed) {
        b->graph_dirty = b->adj_graphs_dirty = true;
        if (b->rooms.size() > 1) {
            ACF_CUDA(cudaDeviceSynchronize());
            return build_tiles(b);
        }
    }
    return ACF_OK;
}

int profile_read(acf_batch *b, double *velocity_ms, double *pressure_ms, int64_t *launches) {
    if (!b || !velocity_ms || !pressure_ms || !launches) return fail(ACF_ERR_ARGUMENT, "null argument");
    *velocity_ms = b->prof_velocity_ms;
    *pressure_ms = b->prof_pressure_ms;
    *launches = b->prof_launches;
    return ACF_OK;
}

// The status word (kStatus* bits) after every queued kernel has finished; clears it.
int device_status(acf_batch *b, int32_t *status) {
    if (!b || !status) return fail(ACF_ERR_ARGUMENT, "null argument");
    DeviceGuard guard(b->device);
    ACF_CUDA(cudaDeviceSynchronize());
    int32_t flag = 0;
    ACF_CUDA(cudaMemcpy(&flag, b->error_flag(), sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag) ACF_CUDA(cudaMemset(b->error_flag(), 0, sizeof(flag)));
    b->status_pending = false;
    *b->status_host = 0;
    *status = flag;
    return ACF_OK;
}

int profile_enable(acf_batch *b, int32_t enable) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    b->profiling = enable != 0;
    b->prof_velocity_ms = b->prof_pressure_ms = 0;
    b->prof_launches = 0;
    return ACF_OK;
}

int energy_terms(acf_batch *b, int room, double dx, double terms[7], acf_stream stream,
                 int64_t x_begin = 0, int64_t x_end = -1, int32_t far_face = 1) {
    int rc = check_room(b, room);
    if (rc) return rc;
    if (!terms) return fail(ACF_ERR_ARGUMENT, "null argument");
    if (!(dx > 0)) return fail(ACF_ERR_ARGUMENT, "dx must be positive");
    const int nx = b->rooms[room].nx;
    if (x_end < 0) x_end = nx;
    if (x_begin < 0 || x_begin > x_end || x_end > nx)
        return fail(ACF_ERR_ARGUMENT, "x planes [%lld, %lld) outside 0..%d", (long long)x_begin,
                    (long long)x_end, nx);
    const int i_faces = (int)x_end + (far_face && x_end == nx ? 1 : 0);
    DeviceGuard guard(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    return b->precision == 8
               ? energy_impl<double>(b, room, dx, terms, st, (int)x_begin, (int)x_end, i_faces)
               : energy_impl<float>(b, room, dx, terms, st, (int)x_begin, (int)x_end, i_faces);
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Schemes. The fused step keeps a second copy of p and v; the current state alternates
// between the two. Paths that work on the primary copy in place (the two sweeps, the adjoint's
// recorded runs, checkpoints) first bring the state back to it.

namespace {

int make_primary(acf_batch *b, cudaStream_t st) {
    for (size_t r = 0; r < b->rooms.size(); r++) {
        RoomHost &h = b->rooms[r];
        if (!h.cur) continue;
        const size_t bytes = (size_t)4 * h.field * b->elem();
        ACF_CUDA(cudaMemcpyAsync((char *)b->state + h.state_off, h.second, bytes, cudaMemcpyDeviceToDevice, st));
        h.cur = 0;
        b->graph_dirty = b->adj_graphs_dirty = true;
        b->room_table_dirty = true;
    }
    return ACF_OK;
}

int set_scheme(acf_batch *b, int32_t scheme) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (scheme != ACF_SCHEME_TWO_SWEEPS && scheme != ACF_SCHEME_FUSED && scheme != ACF_SCHEME_FUSED_STAGED &&
        scheme != ACF_SCHEME_PRESSURE_ONLY)
        return fail(ACF_ERR_ARGUMENT, "unknown scheme %d", scheme);
    if (scheme == ACF_SCHEME_FUSED_STAGED && b->rooms.size() != 1)
        return fail(ACF_ERR_STATE, "the staged scheme is for single rooms");
    if (scheme == ACF_SCHEME_PRESSURE_ONLY) {
        if (b->rooms.size() != 1) return fail(ACF_ERR_STATE, "the pressure-only scheme is for single rooms");
        const RoomHost &h = b->rooms[0];
        if (h.has_layer || h.n_relax > 0)
            return fail(ACF_ERR_STATE, "the pressure-only scheme has no absorbing layer or air "
                        "absorption (the second-order pressure equation keeps no velocity or "
                        "relaxation state for them)");
    }
    if (b->pressure_only() && scheme != ACF_SCHEME_PRESSURE_ONLY && b->po_started)
        return fail(ACF_ERR_STATE, "the pressure-only scheme keeps no velocities: reset the state "
                    "before switching to a scheme that steps them");
    if (scheme == ACF_SCHEME_FUSED_STAGED) {
        const RoomHost &h = b->rooms[0];
        if (staged_block_x(h, b->staged_vector) * b->staged_rows > kStagedMaxConsumers)
            return fail(ACF_ERR_ARGUMENT, "staged scheme: %d rows of %d threads exceed 256 threads per CTA",
                        b->staged_rows, staged_block_x(h, b->staged_vector));
        if (!staged_stages(b, b->staged_rows, b->staged_stages))
            return fail(ACF_ERR_ARGUMENT, "staged scheme: %d rows x %d stages do not fit in shared memory",
                        b->staged_rows, b->staged_stages);
    }
    DeviceGuard guard(b->device);
    if (scheme != ACF_SCHEME_TWO_SWEEPS) {
        for (RoomHost &h : b->rooms) {
            if (h.second) continue;
            const size_t bytes = ((size_t)4 * h.field + (size_t)h.pz) * b->elem();
            if (cudaMalloc(&h.second, bytes) != cudaSuccess)
                return fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes for the fused scheme failed", bytes);
            ACF_CUDA(cudaMemset(h.second, 0, bytes));
        }
    }
    if (scheme == ACF_SCHEME_TWO_SWEEPS) {
        int rc = make_primary(b, 0);
        if (rc) return rc;
        ACF_CUDA(cudaStreamSynchronize(0));
    }
    if (scheme != b->scheme) b->graph_dirty = b->adj_graphs_dirty = b->room_table_dirty = true;
    if (scheme == ACF_SCHEME_PRESSURE_ONLY && !b->pressure_only()) {
        b->po_first = true;      // the next step starts from the p-v state as it is now
        b->po_started = false;
    }
    b->scheme = scheme;
    return ACF_OK;
}

int set_prefetch(acf_batch *b, int32_t mode) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (mode < -1 || mode > 1) return fail(ACF_ERR_ARGUMENT, "prefetch mode must be -1, 0 or 1, got %d", mode);
    // The flag travels in the room descriptions that graphs and room tables hold.
    if (mode != b->prefetch_mode) b->graph_dirty = b->adj_graphs_dirty = b->room_table_dirty = true;
    b->prefetch_mode = mode;
    return ACF_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Adjoint orchestration (single rooms).

namespace {

template <typename T, bool L, bool W, int NR>
struct RecPressure {
    static void launch(const StepParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        pressure_sweep_rec<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanRecStep {
    static void launch(const LeanRecParams &p, dim3 g, dim3 b, cudaStream_t st) {
        lean_sweep_rec<L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct AdjPressure {
    static void launch(const AdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        adjoint_pressure_sweep<T, L, W, NR, false><<<g, b, 0, st>>>(p);
    }
};

// The air-gradient launches use two z elements per thread (launch shape single_shape_w(b, 2)).
template <typename T, bool L, bool W, int NR>
struct AdjPressureAir {
    static void launch(const AdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        if (NR > 0) adjoint_pressure_sweep<T, L, W, NR, NR != 0, 2><<<g, b, 0, st>>>(p);
        else adjoint_pressure_sweep<T, L, W, NR, false, 2><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct AdjFused {
    static void launch(const AdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        adjoint_fused_sweep<T, L, W, NR, false><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanAdjFused {
    static void launch(const LeanAdjointParams &p, dim3 g, dim3 b, cudaStream_t st) {
        lean_adjoint_sweep<L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct LeanAdjFusedAir {
    static void launch(const LeanAdjointParams &p, dim3 g, dim3 b, cudaStream_t st) {
        if constexpr (NR > 0) lean_adjoint_air_sweep<L, W, NR><<<g, b, 0, st>>>(p);
        else lean_adjoint_sweep<L, W, NR><<<g, b, 0, st>>>(p);
    }
};

// The packed coefficients of lean_adjoint_sweep, rounded to float as the room's own and
// combined in float as adjoint_pressure_column combines them.
void fill_adjoint_pairs(float2 *k, const RoomHost &h) {
    auto put = [&](int slot, float v) { k[slot] = make_float2(v, v); };
    put(kAdjNegCv, -(float)h.coef[0]);
    put(kAdjScp, (float)h.coef[3] - (float)h.coef[1]);
    for (int r = 0; r < h.n_relax; r++) {
        put(kAdjNegGain + r, -(float)h.gain[r]);
        put(kAdjOneMinusDecay + r, 1.0f - (float)h.decay[r]);
        put(kAdjMean + r, (float)h.mean[r]);
        put(kAdjNegMean + r, -(float)h.mean[r]);
        put(kAdjDecay + r, (float)h.decay[r]);
    }
}

template <typename T, bool L, bool W, int NR>
struct AdjFusedAir {
    static void launch(const AdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        if (NR > 0) adjoint_fused_sweep<T, L, W, NR, NR != 0, 2><<<g, b, 0, st>>>(p);
        else adjoint_fused_sweep<T, L, W, NR, false, 2><<<g, b, 0, st>>>(p);
    }
};

template <typename T>
History<T> make_history(const acf_batch *b) {
    History<T> h{};
    h.shell_total = b->adj.shell_total;
    for (int f = 0; f < 6; f++) h.face_off[f] = b->adj.face_off[f];
    return h;
}

// Replay `g` (a capture of `chunk` calls of launch(local) for local = 0..chunk-1 followed by
// bump(step_base, bump)) `reps` times on `st`, capturing it first if needed.
template <class F>
int replay(acf_batch *b, acf_batch::Graph &g, int64_t chunk, int64_t bump, int64_t reps,
           cudaStream_t st, F launch) {
    if (reps <= 0) return ACF_OK;
    if (b->adj_graphs_dirty) {
        b->g_record.release();
        b->g_recompute.release();
        b->g_adjoint.release();
        b->g_adjoint_odd.release();
        b->adj_graphs_dirty = false;
    }
    if (!g.exec || g.steps != chunk) {
        g.release();
        if (!b->capture_stream)
            ACF_CUDA(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
        ACF_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
        for (int64_t t = 0; t < chunk; t++) launch((int32_t)t, b->capture_stream);
        bump_step_base<<<1, 1, 0, b->capture_stream>>>(b->step_base, bump);
        cudaGraph_t graph = nullptr;
        ACF_CUDA(cudaStreamEndCapture(b->capture_stream, &graph));
        cudaError_t err = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (err != cudaSuccess) return fail(ACF_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(err));
        g.steps = chunk;
    }
    for (int64_t r = 0; r < reps; r++) ACF_CUDA(cudaGraphLaunch(g.exec, st));
    return ACF_OK;
}

constexpr int64_t kAdjointChunk = 64;

// Forward steps [s0, s0 + n) on `state` (the room's own fields, or the recompute copy), writing
// the history in `hist`. Receivers record only when `receivers` is set, so a recompute leaves
// the caller's recordings alone. With `checkpoints`, the state at every multiple of the
// checkpoint interval (counted from the recorded run's first step) is copied out first. With
// `lean` (single precision, nz a multiple of 4, the room's own fields current in its primary
// copy, no D/psi history) each step is one lean step into the other copy, flipping the current
// copy as the fused scheme does; graphs hold an even number of steps, so a replay leaves it as
// it found it.
template <typename T>
int record_steps(acf_batch *b, acf_batch::Graph &g, const void *state, const History<T> &hist,
                 int64_t s0, int64_t n, bool receivers, cudaStream_t st, bool checkpoints,
                 bool lean = false) {
    const RoomHost &h = b->rooms[0];
    StepParams<T> p{};
    p.room = make_room<T>(b, 0, state);
    if (!receivers) p.room.n_rec = 0;
    p.hist = hist;
    p.step_base = b->step_base;
    p.planes = b->planes;
    const LaunchShape L = single_shape(b);
    const int per_step = lean ? 1 : 2;
    auto launch = [&](int32_t local, cudaStream_t s) {
        if constexpr (sizeof(T) == 4) {
            if (lean) {
                RoomHost &hr = b->rooms[0];
                LeanRecParams q{};
                q.g.f.room = make_room<float>(b, 0);
                q.g.f.np = (float *)b->other_ptr(0, ACF_FIELD_P);
                q.g.f.nvx = (float *)b->other_ptr(0, ACF_FIELD_VX);
                q.g.f.nvy = (float *)b->other_ptr(0, ACF_FIELD_VY);
                q.g.f.nvz = (float *)b->other_ptr(0, ACF_FIELD_VZ);
                q.g.f.step_base = b->step_base;
                q.g.f.local_step = local;
                q.g.f.planes = b->planes;
                fill_pairs(q.g.pairs, hr);
                q.hist = hist;
                dispatch_pressure<float, LeanRecStep>(hr.has_layer, hr.has_walls, hr.n_relax, q, L.grid,
                                                      L.block, s);
                hr.cur ^= 1;
                return;
            }
        }
        StepParams<T> q = p;
        q.local_step = local;
        if (h.has_layer) velocity_sweep<T, true><<<L.grid, L.block, 0, s>>>(q);
        else velocity_sweep<T, false><<<L.grid, L.block, 0, s>>>(q);
        dispatch_pressure<T, RecPressure>(h.has_layer, h.has_walls, h.n_relax, q, L.grid, L.block, s);
    };
    const int64_t G = checkpoints ? b->adj.every : kAdjointChunk;
    int64_t done = 0;
    set_step_base<<<1, 1, 0, st>>>(b->step_base, s0);
    b->launches += 1;
    while (done < n) {
        const int64_t absolute = s0 + done;
        if (checkpoints && (absolute - b->adj.step0) % b->adj.every == 0) {
            const int64_t slot = (absolute - b->adj.step0) / b->adj.every;
            ACF_CUDA(cudaMemcpyAsync((char *)b->adj.checkpoints + slot * b->room_block_bytes(0), state,
                                     b->room_block_bytes(0), cudaMemcpyDeviceToDevice, st));
        }
        if (n - done >= G) {
            int rc = replay(b, g, G, G, 1, st, launch);
            if (rc) return rc;
            b->launches += per_step * G + 1;
            done += G;
        } else {
            // the tail: launch step by step from the counter, then advance it past them
            for (int64_t t = 0; done + t < n; t++) launch((int32_t)t, st);
            bump_step_base<<<1, 1, 0, st>>>(b->step_base, n - done);
            b->launches += per_step * (n - done) + 1;
            done = n;
        }
    }
    return ACF_OK;
}

template <typename T>
int forward_record_impl(acf_batch *b, int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    auto &A = b->adj;
    if (A.step0 != step_offset) b->adj_graphs_dirty = true;
    A.recorded = n_steps;
    A.step0 = step_offset;
    History<T> hist = make_history<T>(b);
    hist.shell = (T *)A.hist_shell;
    hist.shell_step0 = step_offset;
    hist.shell_steps = A.hist_shell ? A.capacity : 0;
    // One segment covers the whole run: the run itself keeps D and psi of every step, and the
    // adjoint recomputes nothing (and needs no checkpoint).
    const bool air = (A.flags & ACF_GRAD_AIR) && A.segment;
    A.fields_recorded = air && n_steps <= A.every;
    if (A.fields_recorded) {
        hist.fields = (T *)A.segment;
        hist.fields_step0 = step_offset;
        hist.fields_slots = A.every;
    }
    // Without air the history is the boundary shell alone, which the lean single-precision step
    // writes as it goes: one sweep per recorded step instead of two, into the second copy of p
    // and v (allocated here when the solver's scheme has none; two sweeps if that fails).
    bool lean = !air && sizeof(T) == 4 && b->rooms.size() == 1 && b->rooms[0].nz % kVec == 0 &&
                b->rooms[0].cur == 0;
    if (lean && !b->rooms[0].second) {
        RoomHost &h = b->rooms[0];
        const size_t bytes = ((size_t)4 * h.field + (size_t)h.pz) * b->elem();
        if (cudaMalloc(&h.second, bytes) != cudaSuccess) {
            cudaGetLastError();
            h.second = nullptr;
            lean = false;
        } else {
            ACF_CUDA(cudaMemsetAsync(h.second, 0, bytes, st));
        }
    }
    const int mode = A.fields_recorded ? 1 : (lean ? 2 : 0);
    if (mode != A.direct_mode) {
        b->adj_graphs_dirty = true;           // the record graph holds the history pointers
        A.direct_mode = mode;
    }
    int rc = record_steps<T>(b, b->g_record, b->field_ptr(0, ACF_FIELD_P), hist, step_offset, n_steps,
                             true, st, air && !A.fields_recorded, lean);
    if (rc) return rc;
    if (lean) {   // an odd number of steps ends in the second copy: bring the state back
        rc = make_primary(b, st);
        if (rc) return rc;
    }
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

template <typename T>
int adjoint_impl(acf_batch *b, const double *grad_rec, double *grad_src, double *grad_shell,
                 double *grad_air, cudaStream_t st) {
    auto &A = b->adj;
    const RoomHost &h = b->rooms[0];
    const int64_t n = A.recorded;
    const size_t es = b->elem();
    const bool air = (A.flags & ACF_GRAD_AIR) && h.n_relax > 0;
    const bool walls = (A.flags & ACF_GRAD_WALLS) && h.has_walls;
    if (grad_shell && !walls)
        return fail(ACF_ERR_STATE, "wall gradients need a room with wall coefficients and ACF_GRAD_WALLS");
    if (grad_air && !air)
        return fail(ACF_ERR_STATE, "air gradients need relaxation states and ACF_GRAD_AIR");

    // Device inputs and zeroed accumulators, sized for the prepared capacity so the captured
    // graphs stay valid from call to call.
    const int64_t cap = A.capacity;
    if (h.n_rec > A.grad_rows_rec || !A.grad_rec) {
        cudaFree(A.grad_rec);
        A.grad_rec = nullptr;
        A.grad_rows_rec = std::max<int64_t>(1, h.n_rec);
        ACF_CUDA(cudaMalloc(&A.grad_rec, (size_t)A.grad_rows_rec * cap * sizeof(double)));
        b->adj_graphs_dirty = true;
    }
    if (h.n_src > A.grad_rows_src || !A.grad_src) {
        cudaFree(A.grad_src);
        A.grad_src = nullptr;
        A.grad_rows_src = std::max<int64_t>(1, h.n_src);
        ACF_CUDA(cudaMalloc(&A.grad_src, (size_t)A.grad_rows_src * cap * sizeof(double)));
        b->adj_graphs_dirty = true;
    }
    if (h.n_rec > 0)
        ACF_CUDA(cudaMemcpy2DAsync(A.grad_rec, cap * sizeof(double), grad_rec, n * sizeof(double),
                                   n * sizeof(double), (size_t)h.n_rec, cudaMemcpyHostToDevice, st));
    if (h.n_src > 0)
        ACF_CUDA(cudaMemsetAsync(A.grad_src, 0, (size_t)h.n_src * cap * sizeof(double), st));
    const size_t adj_bytes = ((size_t)(5 + h.n_relax) * h.field + h.pz) * es;
    ACF_CUDA(cudaMemsetAsync(A.fields, 0, adj_bytes, st));
    if (A.grad_shell) ACF_CUDA(cudaMemsetAsync(A.grad_shell, 0, A.shell_total * sizeof(double), st));
    const LaunchShape L = single_shape(b);
    const LaunchShape LA = air ? single_shape(b, 2) : L;   // the air launches: 2 z elements each
    const int64_t blocks = (int64_t)LA.grid.x * LA.grid.y * LA.grid.z;
    const int NA = 3 * h.n_relax + 1;
    if (air) {
        if (A.air_blocks < blocks) {
            cudaFree(A.air_partials);
            A.air_partials = nullptr;
            ACF_CUDA(cudaMalloc(&A.air_partials, (size_t)blocks * NA * sizeof(double)));
            A.air_blocks = blocks;
            b->adj_graphs_dirty = true;
        }
        ACF_CUDA(cudaMemsetAsync(A.air_partials, 0, (size_t)blocks * NA * sizeof(double), st));
    }

    AdjointParams<T> a{};
    a.room = make_room<T>(b, 0);
    T *f = (T *)A.fields;
    a.lp = f;
    a.lvx = f + h.field;
    a.lvy = f + 2 * h.field;
    a.lvz = f + 3 * h.field;
    a.lpsi = f + 4 * h.field;
    a.ld = f + (4 + h.n_relax) * h.field;
    a.grad_rec = A.grad_rec;
    a.grad_src = A.grad_src;
    a.grad_stride = cap;
    a.grad_step0 = A.step0;
    a.hist = make_history<T>(b);
    a.hist.shell = (T *)A.hist_shell;
    a.hist.shell_step0 = A.step0;
    a.hist.shell_steps = A.capacity;
    a.hist.fields = (T *)A.segment;
    a.hist.fields_step0 = A.step0;
    a.hist.fields_slots = (int32_t)std::max(1, A.every);
    a.grad_shell = walls ? A.grad_shell : nullptr;
    a.air_partials = A.air_partials;
    a.step_base = b->step_base;
    a.planes = b->planes;
    a.air = air ? 1 : 0;

    // The reversed steps, last first. The last recorded step is a cell sweep alone (mu^{n+1} = 0);
    // every earlier step n is one fused launch -- the face sweep of step n + 1, then the cell sweep
    // of step n -- reading mu and lambda_D from one copy and writing them to the other; the face
    // sweep of the first step closes the run. a0 reads copy 0 (the adjoint fields) and writes
    // copy 1 (fields2); a1 the reverse.
    AdjointParams<T> a0 = a, a1 = a;
    {
        T *g2 = (T *)A.fields2;
        a0.out_vx = g2;
        a0.out_vy = g2 + h.field;
        a0.out_vz = g2 + 2 * h.field;
        a0.out_d = g2 + 3 * h.field;
        a1.lvx = a0.out_vx;
        a1.lvy = a0.out_vy;
        a1.lvz = a0.out_vz;
        a1.ld = a0.out_d;
        a1.out_vx = a.lvx;
        a1.out_vy = a.lvy;
        a1.out_vz = a.lvz;
        a1.out_d = a.ld;
    }
    int parity = 0;       // the copy holding the latest mu and lambda_D
    bool first = true;
    // Single precision with nz a multiple of 4 takes the packed step, with or without the air
    // sums (4 z elements per thread, so its grid of blocks is within the air partials' count).
    const bool lean_adjoint = sizeof(T) == 4 && h.nz % kVec == 0;
    auto fused_unit = [&](int32_t local, cudaStream_t s, int par) {
        AdjointParams<T> q = par ? a1 : a0;
        q.local_step = local;
        if constexpr (sizeof(T) == 4) {
            if (lean_adjoint) {
                LeanAdjointParams lq{};
                lq.a = q;
                fill_adjoint_pairs(lq.k, h);
                if (air)
                    dispatch_pressure<float, LeanAdjFusedAir>(h.has_layer, h.has_walls, h.n_relax, lq, L.grid,
                                                              L.block, s);
                else
                    dispatch_pressure<float, LeanAdjFused>(h.has_layer, h.has_walls, h.n_relax, lq, L.grid,
                                                           L.block, s);
                return;
            }
        }
        if (air) dispatch_pressure<T, AdjFusedAir>(h.has_layer, h.has_walls, h.n_relax, q, LA.grid, LA.block, s);
        else dispatch_pressure<T, AdjFused>(h.has_layer, h.has_walls, h.n_relax, q, L.grid, L.block, s);
    };
    // Graph chunks of at most kAdjointChunk steps (one per segment when segments are shorter),
    // one graph per starting copy. Steps [e - G, e) in reverse: graph locals are captured in
    // launch order t = 0..G-1 and reverse step base + (G - 1 - t).
    const int64_t chunk = air ? std::min<int64_t>(A.every, kAdjointChunk) : kAdjointChunk;
    auto reverse_range = [&](int64_t s0, int64_t e) -> int {
        int64_t end = e;
        if (first && end > s0) {
            set_step_base<<<1, 1, 0, st>>>(b->step_base, end - 1);
            AdjointParams<T> q = a0;
            q.local_step = 0;
            if (air) dispatch_pressure<T, AdjPressureAir>(h.has_layer, h.has_walls, h.n_relax, q, LA.grid, LA.block, st);
            else dispatch_pressure<T, AdjPressure>(h.has_layer, h.has_walls, h.n_relax, q, L.grid, L.block, st);
            b->launches += 2;
            end -= 1;
            first = false;
        }
        while (end > s0) {
            const int64_t G = std::min<int64_t>(chunk, end - s0);
            set_step_base<<<1, 1, 0, st>>>(b->step_base, end - G);
            const int p0 = parity;
            if (G == chunk) {
                int rc = replay(b, p0 ? b->g_adjoint_odd : b->g_adjoint, G, 0, 1, st,
                                [&](int32_t t, cudaStream_t s) {
                                    fused_unit((int32_t)(G - 1 - t), s, p0 ^ (int)(t & 1));
                                });
                if (rc) return rc;
                b->launches += G + 2;
            } else {
                for (int64_t t = 0; t < G; t++) fused_unit((int32_t)(G - 1 - t), st, p0 ^ (int)(t & 1));
                b->launches += G + 1;
            }
            parity ^= (int)(G & 1);
            end -= G;
        }
        return ACF_OK;
    };

    const int64_t K = air ? A.every : n;
    const int64_t n_seg = (n + K - 1) / K;
    for (int64_t seg = n_seg - 1; seg >= 0; seg--) {
        const int64_t s0 = A.step0 + seg * K;
        const int64_t s1 = std::min(s0 + K, A.step0 + n);
        if (air && !A.fields_recorded) {
            // Recompute the segment from its checkpoint, keeping D and psi of every step.
            ACF_CUDA(cudaMemcpyAsync(A.scratch, (char *)A.checkpoints + seg * b->room_block_bytes(0),
                                     b->room_block_bytes(0), cudaMemcpyDeviceToDevice, st));
            History<T> hist = make_history<T>(b);
            hist.fields = (T *)A.segment;
            hist.fields_step0 = A.step0;
            hist.fields_slots = (int32_t)K;
            int rc = record_steps<T>(b, b->g_recompute, A.scratch, hist, s0, s1 - s0, false, st, false);
            if (rc) return rc;
        }
        int rc = reverse_range(s0, s1);
        if (rc) return rc;
    }
    // The face sweep of the first recorded step, in place, then mu and lambda_D back in the
    // adjoint fields if they ended in the second copy.
    {
        AdjointParams<T> q = parity ? a1 : a0;
        q.local_step = 0;
        if (h.has_layer) adjoint_velocity_sweep<T, true><<<L.grid, L.block, 0, st>>>(q);
        else adjoint_velocity_sweep<T, false><<<L.grid, L.block, 0, st>>>(q);
        b->launches += 1;
        if (parity) {
            ACF_CUDA(cudaMemcpyAsync(a.lvx, a0.out_vx, (size_t)3 * h.field * es, cudaMemcpyDeviceToDevice, st));
            ACF_CUDA(cudaMemcpyAsync(a.ld, a0.out_d, (size_t)h.field * es, cudaMemcpyDeviceToDevice, st));
        }
    }
    a.local_step = 0;
    adjoint_finish<T><<<L.grid, L.block, 0, st>>>(a);
    b->launches += 1;
    ACF_CUDA(cudaGetLastError());

    if (grad_src && h.n_src > 0)
        ACF_CUDA(cudaMemcpy2DAsync(grad_src, n * sizeof(double), A.grad_src, cap * sizeof(double),
                                   n * sizeof(double), (size_t)h.n_src, cudaMemcpyDeviceToHost, st));
    if (grad_shell)
        ACF_CUDA(cudaMemcpyAsync(grad_shell, A.grad_shell, A.shell_total * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    std::vector<double> partials;
    if (grad_air) {
        partials.resize((size_t)blocks * NA);
        ACF_CUDA(cudaMemcpyAsync(partials.data(), A.air_partials, partials.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    }
    ACF_CUDA(cudaStreamSynchronize(st));
    if (grad_air) {
        for (int t = 0; t < NA; t++) grad_air[t] = 0.0;
        for (int64_t blk = 0; blk < blocks; blk++)
            for (int t = 0; t < NA; t++) grad_air[t] += partials[(size_t)blk * NA + t];
    }
    return ACF_OK;
}

int adjoint_prepare(acf_batch *b, int32_t flags, int64_t max_steps, int32_t every) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (b->rooms.size() != 1) return fail(ACF_ERR_STATE, "the adjoint is for single rooms");
    if (max_steps < 1) return fail(ACF_ERR_ARGUMENT, "max_steps must be >= 1");
    if ((flags & ACF_GRAD_AIR) && (every < 0 || every > max_steps))
        return fail(ACF_ERR_ARGUMENT, "checkpoint interval %d out of range", every);
    DeviceGuard guard(b->device);
    ACF_CUDA(cudaDeviceSynchronize());
    if ((flags & ACF_GRAD_AIR) && every == 0) {
        // Automatic: keep D and psi of every step when that history takes at most 60 % of the
        // free device memory (the recorded run then writes it and nothing is recomputed), else
        // checkpoints every ceil(sqrt(max_steps)) steps.
        const RoomHost &h = b->rooms[0];
        const double whole = (double)max_steps * (1 + h.n_relax) * h.field * b->elem();
        size_t free_bytes = 0, total_bytes = 0;
        ACF_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
        every = whole <= 0.6 * (double)free_bytes ? (int32_t)std::min<int64_t>(max_steps, INT32_MAX)
                                                   : (int32_t)std::ceil(std::sqrt((double)max_steps));
    }
    auto &A = b->adj;
    b->adj_graphs_dirty = true;
    void **buffers[] = {&A.hist_shell, &A.checkpoints, &A.scratch, &A.segment, &A.fields, &A.fields2};
    for (void **p : buffers) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaFree(A.grad_shell);
    A.grad_shell = nullptr;
    const RoomHost &h = b->rooms[0];
    const size_t es = b->elem();
    A.flags = flags;
    A.capacity = max_steps;
    A.every = (flags & ACF_GRAD_AIR) ? every : (int32_t)std::min<int64_t>(max_steps, INT32_MAX);
    A.recorded = 0;
    A.fields_recorded = false;
    A.direct_mode = -1;
    const int64_t sizes[6] = {(int64_t)h.ny * h.nz, (int64_t)h.ny * h.nz, (int64_t)h.nx * h.nz,
                              (int64_t)h.nx * h.nz, (int64_t)h.nx * h.ny, (int64_t)h.nx * h.ny};
    A.shell_total = 0;
    for (int q = 0; q < 6; q++) {
        A.face_off[q] = A.shell_total;
        A.shell_total += sizes[q];
    }
    const size_t adj_bytes = ((size_t)(5 + h.n_relax) * h.field + h.pz) * es;
    ACF_CUDA(cudaMalloc(&A.fields, adj_bytes));
    const size_t second = ((size_t)4 * h.field + h.pz) * es;
    ACF_CUDA(cudaMalloc(&A.fields2, second));
    ACF_CUDA(cudaMemset(A.fields2, 0, second));
    if ((flags & ACF_GRAD_WALLS) && h.has_walls) {
        const size_t bytes = (size_t)max_steps * A.shell_total * 2 * es;
        if (cudaMalloc(&A.hist_shell, bytes) != cudaSuccess)
            return fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes of wall history failed", bytes);
        ACF_CUDA(cudaMalloc(&A.grad_shell, A.shell_total * sizeof(double)));
    }
    if ((flags & ACF_GRAD_AIR) && h.n_relax > 0) {
        const int64_t n_ckpt = (max_steps + every - 1) / every;
        const size_t block = b->room_block_bytes(0);
        if (cudaMalloc(&A.checkpoints, (size_t)n_ckpt * block) != cudaSuccess)
            return fail(ACF_ERR_MEMORY, "cudaMalloc of %lld checkpoints failed", (long long)n_ckpt);
        ACF_CUDA(cudaMalloc(&A.scratch, block + (size_t)h.pz * es));
        ACF_CUDA(cudaMemset(A.scratch, 0, block + (size_t)h.pz * es));
        const size_t seg = ((size_t)every * (1 + h.n_relax) * h.field + h.pz) * es;
        if (cudaMalloc(&A.segment, seg) != cudaSuccess)
            return fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes of segment history failed", seg);
        ACF_CUDA(cudaMemset(A.segment, 0, seg));
    }
    return ACF_OK;
}

int set_coefficients(acf_batch *b, int room, const acf_config *c) {
    int rc = check_room(b, room);
    if (rc) return rc;
    if (!c) return fail(ACF_ERR_ARGUMENT, "null config");
    RoomHost &h = b->rooms[room];
    rc = validate_config(c, room);
    if (rc) return rc;
    if (c->nx != h.nx || c->ny != h.ny || c->nz != h.nz || c->precision != b->precision ||
        c->n_relax != h.n_relax)
        return fail(ACF_ERR_ARGUMENT, "new coefficients must keep the grid, precision and relaxation count");
    if ((c->cell[0] != nullptr) != h.has_layer || (c->wall_shell[0] != nullptr) != h.has_walls)
        return fail(ACF_ERR_ARGUMENT, "new coefficients must keep which of layer and walls are present");
    DeviceGuard guard(b->device);
    ACF_CUDA(cudaDeviceSynchronize());
    h.coef[0] = c->vel_coef;
    h.coef[1] = c->pres_coef;
    h.coef[2] = c->src_coef;
    h.coef[3] = c->relax_scale;
    for (int q = 0; q < ACF_MAX_RELAXATION; q++) {
        h.decay[q] = q < c->n_relax ? c->relax_decay[q] : 0.0;
        h.mean[q] = q < c->n_relax ? c->relax_mean[q] : 0.0;
        h.gain[q] = q < c->n_relax ? c->relax_gain[q] : 0.0;
    }
    const size_t es = b->elem();
    const int64_t n_axis[3] = {c->nx, c->ny, c->nz};
    if (h.has_layer) {
        std::vector<double> host;
        for (int a = 0; a < 3; a++) host.insert(host.end(), c->cell[a], c->cell[a] + n_axis[a]);
        for (int a = 0; a < 3; a++) host.insert(host.end(), c->face[a], c->face[a] + n_axis[a] + 1);
        std::vector<char> cast(host.size() * es);
        if (es == 4) cast_copy<float>(cast.data(), host.data(), host.size());
        else cast_copy<double>(cast.data(), host.data(), host.size());
        ACF_CUDA(cudaMemcpy(h.profiles, cast.data(), cast.size(), cudaMemcpyHostToDevice));
    }
    if (h.has_walls) {
        std::vector<double> host;
        for (int f = 0; f < 6; f++) {
            const int axis = f / 2;
            const int64_t nb = axis == 0 ? n_axis[1] : n_axis[0];
            const int64_t nc = axis == 2 ? n_axis[1] : n_axis[2];
            host.insert(host.end(), c->wall_shell[f], c->wall_shell[f] + 2 * nb * nc);
        }
        std::vector<char> cast(host.size() * es);
        if (es == 4) cast_copy<float>(cast.data(), host.data(), host.size());
        else cast_copy<double>(cast.data(), host.data(), host.size());
        ACF_CUDA(cudaMemcpy(h.shell, cast.data(), cast.size(), cudaMemcpyHostToDevice));
    }
    b->graph_dirty = b->adj_graphs_dirty = true;
    b->room_table_dirty = true;
    return ACF_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Adjoint of a batch of rooms: the forward records every room's boundary-shell history with
// one persistent launch per sweep; the backward runs the adjoint sweeps of all rooms together.

namespace {

template <typename T, bool L, bool W, int NR>
struct BatchRecPressure {
    static void launch(const BatchAdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        pressure_batch_rec<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct BatchAdjPressure {
    static void launch(const BatchAdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        adjoint_pressure_batch<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

template <typename T, bool L, bool W, int NR>
struct BatchAdjFused {
    static void launch(const BatchAdjointParams<T> &p, dim3 g, dim3 b, cudaStream_t st) {
        adjoint_fused_batch<T, L, W, NR><<<g, b, 0, st>>>(p);
    }
};

int batch_adjoint_prepare(acf_batch *b, int64_t max_steps) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null batch");
    if (max_steps < 1) return fail(ACF_ERR_ARGUMENT, "max_steps must be >= 1");
    if (!b->any_walls) return fail(ACF_ERR_STATE, "wall gradients need rooms with wall coefficients");
    DeviceGuard guard(b->device);
    ACF_CUDA(cudaDeviceSynchronize());
    for (auto &ra : b->badj) {
        cudaFree(ra.hist_shell);
        cudaFree(ra.fields);
        cudaFree(ra.fields2);
        cudaFree(ra.grad_shell);
        cudaFree(ra.grad_rec);
        cudaFree(ra.grad_src);
    }
    b->badj.assign(b->rooms.size(), acf_batch::RoomAdjoint());
    const size_t es = b->elem();
    for (size_t r = 0; r < b->rooms.size(); r++) {
        const RoomHost &h = b->rooms[r];
        auto &ra = b->badj[r];
        const int64_t sizes[6] = {(int64_t)h.ny * h.nz, (int64_t)h.ny * h.nz, (int64_t)h.nx * h.nz,
                                  (int64_t)h.nx * h.nz, (int64_t)h.nx * h.ny, (int64_t)h.nx * h.ny};
        for (int q = 0; q < 6; q++) {
            ra.face_off[q] = ra.shell_total;
            ra.shell_total += sizes[q];
        }
        const size_t hist = (size_t)max_steps * ra.shell_total * 2 * es;
        if (cudaMalloc(&ra.hist_shell, hist) != cudaSuccess)
            return fail(ACF_ERR_MEMORY, "room %zu: cudaMalloc of %zu bytes of wall history failed", r, hist);
        ACF_CUDA(cudaMalloc(&ra.fields, ((size_t)(5 + h.n_relax) * h.field + h.pz) * es));
        ACF_CUDA(cudaMalloc(&ra.fields2, ((size_t)4 * h.field + h.pz) * es));
        ACF_CUDA(cudaMemset(ra.fields2, 0, ((size_t)4 * h.field + h.pz) * es));
        ACF_CUDA(cudaMalloc(&ra.grad_shell, ra.shell_total * sizeof(double)));
    }
    b->badj_capacity = max_steps;
    b->badj_recorded = 0;
    return ACF_OK;
}

// Fill the device table of per-room adjoint descriptions for the current run.
template <typename T>
int upload_adjoint_table(acf_batch *b, int64_t n) {
    // Entries [0, rooms): mu and lambda_D read from the adjoint fields, written to fields2 (by
    // the fused step); entries [rooms, 2 rooms): the reverse.
    const size_t nr = b->rooms.size();
    std::vector<AdjointParams<T>> table(2 * nr);
    for (size_t r = 0; r < b->rooms.size(); r++) {
        const RoomHost &h = b->rooms[r];
        auto &ra = b->badj[r];
        AdjointParams<T> &a = table[r];
        a = AdjointParams<T>{};
        a.room = make_room<T>(b, (int)r);
        T *f = (T *)ra.fields;
        a.lp = f;
        a.lvx = f + h.field;
        a.lvy = f + 2 * h.field;
        a.lvz = f + 3 * h.field;
        a.lpsi = f + 4 * h.field;
        a.ld = f + (4 + h.n_relax) * h.field;
        a.grad_rec = ra.grad_rec;
        a.grad_src = ra.grad_src;
        a.grad_stride = b->badj_capacity;
        a.grad_step0 = b->badj_step0;
        a.hist.shell = (T *)ra.hist_shell;
        a.hist.shell_total = ra.shell_total;
        a.hist.shell_step0 = b->badj_step0;
        a.hist.shell_steps = b->badj_capacity;
        for (int q = 0; q < 6; q++) a.hist.face_off[q] = ra.face_off[q];
        a.hist.fields_slots = 1;
        a.grad_shell = h.has_walls ? ra.grad_shell : nullptr;
        a.planes = b->planes;
        T *g2 = (T *)ra.fields2;
        a.out_vx = g2;
        a.out_vy = g2 + h.field;
        a.out_vz = g2 + 2 * h.field;
        a.out_d = g2 + 3 * h.field;
        AdjointParams<T> &o = table[nr + r];
        o = a;
        o.lvx = a.out_vx;
        o.lvy = a.out_vy;
        o.lvz = a.out_vz;
        o.ld = a.out_d;
        o.out_vx = a.lvx;
        o.out_vy = a.lvy;
        o.out_vz = a.lvz;
        o.out_d = a.ld;
        (void)n;
    }
    if (!b->badj_table) ACF_CUDA(cudaMalloc(&b->badj_table, table.size() * sizeof(AdjointParams<T>)));
    ACF_CUDA(cudaMemcpy(b->badj_table, table.data(), table.size() * sizeof(AdjointParams<T>),
                        cudaMemcpyHostToDevice));
    return ACF_OK;
}

template <typename T>
int batch_forward_record_impl(acf_batch *b, int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    b->badj_step0 = step_offset;
    b->badj_recorded = n_steps;
    if (b->room_table_dirty) {
        int rc = upload_room_table<T>(b);
        if (rc) return rc;
    }
    int rc = upload_adjoint_table<T>(b, n_steps);
    if (rc) return rc;
    BatchParams<T> v{};
    v.rooms = (const Room<T> *)b->room_table;
    v.tiles = b->tiles;
    v.n_tiles = b->n_tiles;
    v.step_base = b->step_base;
    BatchAdjointParams<T> p{};
    p.rooms = (const AdjointParams<T> *)b->badj_table;
    p.tiles = b->tiles;
    p.n_tiles = b->n_tiles;
    p.step_base = b->step_base;
    const dim3 grid(b->batch_ctas), block(b->block_threads);
    set_step_base<<<1, 1, 0, st>>>(b->step_base, step_offset);
    for (int64_t t = 0; t < n_steps; t++) {
        v.local_step = p.local_step = (int32_t)t;
        if (b->any_layer) velocity_batch<T, true><<<grid, block, 0, st>>>(v);
        else velocity_batch<T, false><<<grid, block, 0, st>>>(v);
        dispatch_pressure<T, BatchRecPressure>(b->any_layer, b->any_walls, b->n_relax, p, grid, block, st);
    }
    b->launches += 2 * n_steps + 1;
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

template <typename T>
int batch_adjoint_impl(acf_batch *b, const double *grad_rec, double *grad_src, double *grad_shell,
                       cudaStream_t st) {
    const int64_t n = b->badj_recorded, cap = b->badj_capacity;
    const size_t es = b->elem();
    // Inputs and zeroed accumulators, room by room.
    int64_t rec_row = 0;
    for (size_t r = 0; r < b->rooms.size(); r++) {
        const RoomHost &h = b->rooms[r];
        auto &ra = b->badj[r];
        if (h.n_rec > ra.rows_rec || !ra.grad_rec) {
            cudaFree(ra.grad_rec);
            ra.rows_rec = std::max<int64_t>(1, h.n_rec);
            ACF_CUDA(cudaMalloc(&ra.grad_rec, (size_t)ra.rows_rec * cap * sizeof(double)));
        }
        if (h.n_src > ra.rows_src || !ra.grad_src) {
            cudaFree(ra.grad_src);
            ra.rows_src = std::max<int64_t>(1, h.n_src);
            ACF_CUDA(cudaMalloc(&ra.grad_src, (size_t)ra.rows_src * cap * sizeof(double)));
        }
        if (h.n_rec > 0)
            ACF_CUDA(cudaMemcpy2DAsync(ra.grad_rec, cap * sizeof(double), grad_rec + rec_row * n,
                                       n * sizeof(double), n * sizeof(double), (size_t)h.n_rec,
                                       cudaMemcpyHostToDevice, st));
        rec_row += h.n_rec;
        ACF_CUDA(cudaMemsetAsync(ra.grad_src, 0, (size_t)ra.rows_src * cap * sizeof(double), st));
        ACF_CUDA(cudaMemsetAsync(ra.fields, 0, ((size_t)(5 + h.n_relax) * h.field + h.pz) * es, st));
        ACF_CUDA(cudaMemsetAsync(ra.grad_shell, 0, ra.shell_total * sizeof(double), st));
    }
    int rc = upload_adjoint_table<T>(b, n);
    if (rc) return rc;
    BatchAdjointParams<T> p{};
    p.rooms = (const AdjointParams<T> *)b->badj_table;
    p.tiles = b->tiles;
    p.n_tiles = b->n_tiles;
    p.step_base = b->step_base;
    const dim3 grid(b->batch_ctas), block(b->block_threads);
    set_step_base<<<1, 1, 0, st>>>(b->step_base, b->badj_step0);
    // The last recorded step as a cell sweep alone; every earlier step as one fused launch (the
    // face sweep of step t + 1, then the cell sweep of step t), alternating between the two
    // copies of mu and lambda_D; the face sweep of step 0 closes the run.
    const AdjointParams<T> *tables[2] = {(const AdjointParams<T> *)b->badj_table,
                                         (const AdjointParams<T> *)b->badj_table + b->rooms.size()};
    int parity = 0;
    p.rooms = tables[0];
    p.local_step = (int32_t)(n - 1);
    dispatch_pressure<T, BatchAdjPressure>(b->any_layer, b->any_walls, b->n_relax, p, grid, block, st);
    for (int64_t t = n - 2; t >= 0; t--) {
        p.rooms = tables[parity];
        p.local_step = (int32_t)t;
        dispatch_pressure<T, BatchAdjFused>(b->any_layer, b->any_walls, b->n_relax, p, grid, block, st);
        parity ^= 1;
    }
    p.rooms = tables[parity];
    p.local_step = 0;
    if (b->any_layer) adjoint_velocity_batch<T, true><<<grid, block, 0, st>>>(p);
    else adjoint_velocity_batch<T, false><<<grid, block, 0, st>>>(p);
    b->launches += n + 2;
    ACF_CUDA(cudaGetLastError());
    int64_t src_row = 0, shell_at = 0;
    for (size_t r = 0; r < b->rooms.size(); r++) {
        const RoomHost &h = b->rooms[r];
        auto &ra = b->badj[r];
        if (grad_src && h.n_src > 0)
            ACF_CUDA(cudaMemcpy2DAsync(grad_src + src_row * n, n * sizeof(double), ra.grad_src,
                                       cap * sizeof(double), n * sizeof(double), (size_t)h.n_src,
                                       cudaMemcpyDeviceToHost, st));
        src_row += h.n_src;
        if (grad_shell)
            ACF_CUDA(cudaMemcpyAsync(grad_shell + shell_at, ra.grad_shell, ra.shell_total * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        shell_at += ra.shell_total;
    }
    ACF_CUDA(cudaStreamSynchronize(st));
    return ACF_OK;
}

// ------------------------------------------------------------------------------------------
// Impulse-response post-processing in FP64 (ac-fdtd src/ac_fdtd/metrics.py:57-111 and the
// spectral division of src/ac_fdtd/sources.py:80-108): the steps after the time loop, on the
// receiver signals where the recordings already are. One CTA per channel; every sum in FP64.

constexpr int kPostThreads = 1024;

// Exclusive scan of one double per thread over the CTA (kPostThreads threads, thread order);
// `shared` holds 32 doubles. Returns the sum of the values of the threads before this one;
// *total gets the CTA's sum.
__device__ double block_exclusive_scan(double v, double *shared, double *total) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double inclusive = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double up = __shfl_up_sync(0xffffffffu, inclusive, d);
        if (lane >= (unsigned)d) inclusive += up;
    }
    double within = __shfl_up_sync(0xffffffffu, inclusive, 1);
    if (lane == 0) within = 0.0;
    if (lane == 31) shared[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        double w = shared[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double up = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= (unsigned)d) w += up;
        }
        shared[lane] = w;
    }
    __syncthreads();
    const double before = warp > 0 ? shared[warp - 1] : 0.0;
    *total = shared[31];
    __syncthreads();
    return lane == 0 ? before : before + within;
}

__device__ double block_sum(double v, double *shared) {
    double total;
    block_exclusive_scan(v, shared, &total);
    return total;
}

__device__ int64_t block_min(int64_t v, int64_t *shared) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = min(v, (int64_t)__shfl_xor_sync(0xffffffffu, v, d));
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int64_t w = shared[lane];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) w = min(w, (int64_t)__shfl_xor_sync(0xffffffffu, w, d));
        if (lane == 0) shared[0] = w;
    }
    __syncthreads();
    const int64_t out = shared[0];
    __syncthreads();
    return out;
}

// Schroeder's backward integral I(k) = sum_{m >= k} h(m)^2, as 10 log10 max(I(k) / I(0),
// 1e-300) floored at `floor_db` (metrics.py:57-69). Thread t owns a contiguous run of the
// reversed signal; one CTA scan of the runs' sums gives each run's starting value.
__global__ void __launch_bounds__(kPostThreads) schroeder_decay_kernel(const double *response, int64_t n,
                                                                       double floor_db, double *decay) {
    __shared__ double shared[32];
    const double *h = response + (int64_t)blockIdx.x * n;
    double *out = decay + (int64_t)blockIdx.x * n;
    const int64_t run = (n + kPostThreads - 1) / kPostThreads;
    const int64_t q0 = min((int64_t)threadIdx.x * run, n), q1 = min(q0 + run, n);
    double mine = 0.0;
    for (int64_t q = q0; q < q1; q++) {
        const double x = h[n - 1 - q];
        mine += x * x;
    }
    double sum_all;
    const double start = block_exclusive_scan(mine, shared, &sum_all);   // the later runs in time
    // The curve is normalised by I(0) itself, as the reference divides by its first entry: the
    // thread holding sample 0 forms it with the same additions as its pass below, so the first
    // level is exactly 0 dB.
    __shared__ double first;
    if (q0 < n && q1 == n) {
        double running = start;
        for (int64_t q = q0; q < q1; q++) {
            const double x = h[n - 1 - q];
            running += x * x;
        }
        first = running;
    }
    __syncthreads();
    const double total = first;
    double running = start;
    for (int64_t q = q0; q < q1; q++) {
        const double x = h[n - 1 - q];
        running += x * x;
        const double level = 10.0 * log10(fmax(running / total, 1e-300));
        out[n - 1 - q] = fmax(level, floor_db);
    }
}

// Seconds per 60 dB from a least-squares line through the decay curve between the first sample
// at or below `upper` dB and the first at or below `lower` dB (metrics.py:72-84); NaN and
// `failed[c] = 1` when the curve does not reach `lower` after `upper`, where the reference
// raises.
__global__ void __launch_bounds__(kPostThreads) decay_fit_kernel(const double *decay, int64_t n,
                                                                 double sample_rate, double upper,
                                                                 double lower, double *seconds,
                                                                 int32_t *failed) {
    __shared__ double shared[32];
    __shared__ int64_t ishared[32];
    const double *d = decay + (int64_t)blockIdx.x * n;
    int64_t first_upper = n, first_lower = n;
    for (int64_t k = threadIdx.x; k < n; k += kPostThreads) {
        const double v = d[k];
        if (v <= upper && k < first_upper) first_upper = k;
        if (v <= lower && k < first_lower) first_lower = k;
    }
    int64_t start = block_min(first_upper, ishared), end = block_min(first_lower, ishared);
    if (start == n) start = 0;   // numpy.argmax of an all-false mask
    if (end == n) end = 0;
    if (end <= start) {
        if (threadIdx.x == 0) {
            seconds[blockIdx.x] = __longlong_as_double(0x7ff8000000000000ll);
            failed[blockIdx.x] = 1;
        }
        return;
    }
    const double m = (double)(end - start);
    double sx = 0.0, sy = 0.0;
    for (int64_t k = start + threadIdx.x; k < end; k += kPostThreads) {
        sx += (double)k / sample_rate;
        sy += d[k];
    }
    const double mean_x = block_sum(sx, shared) / m, mean_y = block_sum(sy, shared) / m;
    double sxy = 0.0, sxx = 0.0;
    for (int64_t k = start + threadIdx.x; k < end; k += kPostThreads) {
        const double x = (double)k / sample_rate - mean_x;
        sxy += x * (d[k] - mean_y);
        sxx += x * x;
    }
    const double slope = block_sum(sxy, shared) / block_sum(sxx, shared);
    if (threadIdx.x == 0) {
        seconds[blockIdx.x] = -60.0 / slope;
        failed[blockIdx.x] = 0;
    }
}

// Early-to-late energy ratio in dB with the split at sample `boundary` (metrics.py:104-110).
__global__ void __launch_bounds__(kPostThreads) clarity_kernel(const double *response, int64_t n,
                                                               int64_t boundary, double *db) {
    __shared__ double shared[32];
    const double *h = response + (int64_t)blockIdx.x * n;
    double early = 0.0, late = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += kPostThreads) {
        const double e = h[k] * h[k];
        if (k < boundary) early += e;
        else late += e;
    }
    early = block_sum(early, shared);
    late = block_sum(late, shared);
    if (threadIdx.x == 0) db[blockIdx.x] = 10.0 * log10(early / late);
}

// Largest |S(f)|^2 of the excitation's spectrum (the regularisation's scale).
__global__ void __launch_bounds__(kPostThreads) spectrum_peak_power(const double2 *source, int64_t bins,
                                                                   double *peak) {
    __shared__ double shared[32];
    double best = 0.0;
    for (int64_t k = threadIdx.x; k < bins; k += kPostThreads) {
        const double a = hypot(source[k].x, source[k].y);
        best = fmax(best, a * a);
    }
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, d));
    if (lane == 0) shared[warp] = best;
    __syncthreads();
    if (warp == 0) {
        double w = shared[lane];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, d));
        if (lane == 0) *peak = w;
    }
}

// R(f) = X(f) conj(S(f)) / (|S(f)|^2 + reg * max |S|^2), zero above max_frequency, for every
// channel's spectrum X (sources.py:103-107). Bin k is at k * bin_hz, as numpy.fft.rfftfreq.
__global__ void spectral_divide_kernel(const double2 *spectra, const double2 *source, int64_t channels,
                                       int64_t bins, double bin_hz, double max_frequency,
                                       double regularisation, const double *peak, double2 *out) {
    const int64_t at = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (at >= channels * bins) return;
    const int64_t k = at % bins;
    double2 r = make_double2(0.0, 0.0);
    if (!((double)k * bin_hz > max_frequency)) {
        const double2 x = spectra[at], src = source[k];
        const double a = hypot(src.x, src.y);
        const double denominator = a * a + regularisation * *peak;
        // x * conj(src): (x.x src.x - x.y (-src.y)) + (x.x (-src.y) + x.y src.x) i
        const double re = x.x * src.x - x.y * -src.y;
        const double im = x.x * -src.y + x.y * src.x;
        r = make_double2(re / denominator, im / denominator);
    }
    out[at] = r;
}

int check_post_args(const void *a, const void *b, int64_t channels, int64_t n) {
    if (!a || !b) return fail(ACF_ERR_ARGUMENT, "null device array");
    if (channels < 1 || channels > 65535 || n < 1) return fail(ACF_ERR_ARGUMENT, "need 1..65535 channels of at least one sample");
    return ACF_OK;
}

}  // namespace

// ==========================================================================================
// C ABI

extern "C" {

int acf_abi_version(void) { return ACF_ABI_VERSION; }

size_t acf_struct_size(void) { return sizeof(acf_config); }

const char *acf_last_error(void) { return g_last_error; }

int acf_device_count(int *count) {
    if (!count) return fail(ACF_ERR_ARGUMENT, "null count");
    ACF_CUDA(cudaGetDeviceCount(count));
    return ACF_OK;
}

int acf_set_device(int32_t device) {
    int count = 0;
    ACF_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        return fail(ACF_ERR_ARGUMENT, "device %d out of range (%d visible)", device, count);
    ACF_CUDA(cudaSetDevice(device));
    return ACF_OK;
}

// ---- one room ---------------------------------------------------------------------------

int acf_create(const acf_config *cfg, acf_solver **out) {
    if (!cfg || !out) return fail(ACF_ERR_ARGUMENT, "null config or output pointer");
    *out = nullptr;
    int rc = validate_config(cfg, 0);
    if (rc) return rc;
    acf_solver *h = new (std::nothrow) acf_solver();
    if (!h) return fail(ACF_ERR_MEMORY, "host allocation failed");
    rc = create_batch(1, cfg, h);
    if (rc) {
        free_batch(h);
        return rc;
    }
    *out = h;
    return ACF_OK;
}

int acf_destroy(acf_solver *h) {
    free_batch(h);
    return ACF_OK;
}

int acf_is_double(const acf_solver *h) { return h && h->precision == 8; }

int acf_set_sources(acf_solver *h, int64_t n, const int64_t *cell, const int64_t *length,
                    const double *signal, int64_t stride) {
    return set_sources(h, 0, n, cell, length, signal, stride);
}

int acf_set_receivers(acf_solver *h, int64_t n, const int64_t *cell, const int64_t *start_step) {
    return set_receivers(h, 0, n, cell, start_step);
}

int acf_read_recording(acf_solver *h, int64_t r, int64_t first_step, int64_t n, void *dst,
                       acf_stream stream) {
    return read_recording(h, 0, r, first_step, n, dst, stream);
}

int acf_upload(acf_solver *h, int field, const void *src, acf_stream stream) {
    int rc = check_field(h, 0, field);
    if (rc) return rc;
    if (h->pressure_only() && h->po_started && field != ACF_FIELD_P)
        return fail(ACF_ERR_STATE, "the pressure-only scheme keeps no velocities after its first step");
    if (!src) return fail(ACF_ERR_ARGUMENT, "null source");
    DeviceGuard guard(h->device);
    return copy_field(h, 0, field, const_cast<void *>(src), true, (cudaStream_t)stream);
}

int acf_download(acf_solver *h, int field, void *dst, acf_stream stream) {
    int rc = check_field(h, 0, field);
    if (rc) return rc;
    if (h->pressure_only() && h->po_started && field != ACF_FIELD_P)
        return fail(ACF_ERR_STATE, "the pressure-only scheme keeps no velocities after its first step");
    if (!dst) return fail(ACF_ERR_ARGUMENT, "null destination");
    DeviceGuard guard(h->device);
    return copy_field(h, 0, field, dst, false, (cudaStream_t)stream);
}

int acf_run(acf_solver *h, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    return run_batch(h, n_steps, step_offset, stream);
}

int acf_set_graph(acf_solver *h, int32_t steps) { return acf_batch_set_graph(h, steps); }

int acf_set_launch(acf_solver *h, int32_t block_threads, int32_t planes) {
    return set_launch(h, block_threads, planes, h ? h->ctas_per_sm : 1);
}

int acf_energy_terms(acf_solver *h, double dx, double terms[7], acf_stream stream) {
    if (h && h->pressure_only() && h->po_started)
        return fail(ACF_ERR_STATE, "the pressure-only scheme keeps no velocities: use "
                    "acf_pressure_only_energy_terms");
    return energy_terms(h, 0, dx, terms, stream);
}

int acf_pressure_only_energy_terms(acf_solver *h, double terms[2], acf_stream stream) {
    if (!h || !terms) return fail(ACF_ERR_ARGUMENT, "null argument");
    if (!h->pressure_only() || !h->po_started)
        return fail(ACF_ERR_STATE, "no pressure-only step has been taken since the scheme was selected");
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    double out[kEnergyTerms];
    if (h->precision == 8) {
        const Room<double> s = make_room<double>(h, 0);
        pressure_only_energy_partials<double><<<h->energy_blocks, 256, 0, st>>>(
            s, (const double *)h->field_ptr(0, ACF_FIELD_P), (const double *)h->other_ptr(0, ACF_FIELD_P),
            h->energy_scratch);
    } else {
        const Room<float> s = make_room<float>(h, 0);
        pressure_only_energy_partials<float><<<h->energy_blocks, 256, 0, st>>>(
            s, (const float *)h->field_ptr(0, ACF_FIELD_P), (const float *)h->other_ptr(0, ACF_FIELD_P),
            h->energy_scratch);
    }
    energy_finish<<<1, 32, 0, st>>>(h->energy_scratch, h->energy_blocks,
                                    h->energy_scratch + (size_t)h->energy_blocks * kEnergyTerms);
    h->launches += 2;
    ACF_CUDA(cudaGetLastError());
    ACF_CUDA(cudaMemcpyAsync(out, h->energy_scratch + (size_t)h->energy_blocks * kEnergyTerms,
                             kEnergyTerms * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACF_CUDA(cudaStreamSynchronize(st));
    terms[0] = out[0];
    terms[1] = out[1];
    return ACF_OK;
}

int acf_energy_terms_planes(acf_solver *h, double dx, int64_t x_begin, int64_t x_end,
                            int32_t far_face, double terms[7], acf_stream stream) {
    if (h && h->pressure_only() && h->po_started)
        return fail(ACF_ERR_STATE, "the pressure-only scheme keeps no velocities");
    return energy_terms(h, 0, dx, terms, stream, x_begin, x_end, far_face);
}

int acf_field_pointer(acf_solver *h, int field, void **ptr, int64_t strides[3]) {
    int rc = check_field(h, 0, field);
    if (rc) return rc;
    if (!ptr || !strides) return fail(ACF_ERR_ARGUMENT, "null output");
    *ptr = h->field_ptr(0, field);
    strides[0] = h->rooms[0].plane;
    strides[1] = h->rooms[0].pz;
    strides[2] = 1;
    return ACF_OK;
}

int acf_copy_plane(acf_solver *dst, int64_t dst_plane, const acf_solver *src, int64_t src_plane,
                   int field, acf_stream stream) {
    if (!dst || !src) return fail(ACF_ERR_ARGUMENT, "null solver");
    int rc = check_field(dst, 0, field);
    if (rc) return rc;
    rc = check_field(src, 0, field);
    if (rc) return rc;
    const RoomHost &hd = dst->rooms[0], &hs = src->rooms[0];
    if (dst->precision != src->precision || hd.ny != hs.ny || hd.nz != hs.nz)
        return fail(ACF_ERR_ARGUMENT, "the two rooms' planes differ in precision or shape");
    if (dst_plane < 0 || dst_plane > hd.nx || src_plane < 0 || src_plane > hs.nx)
        return fail(ACF_ERR_ARGUMENT, "plane %lld or %lld out of range", (long long)dst_plane,
                    (long long)src_plane);
    const size_t bytes = (size_t)hd.plane * dst->elem();   // one padded plane: (ny+1) x pz
    char *d = dst->field_ptr(0, field) + (size_t)dst_plane * bytes;
    const char *sp = src->field_ptr(0, field) + (size_t)src_plane * bytes;
    DeviceGuard guard(dst->device);
    if (dst->device == src->device)
        ACF_CUDA(cudaMemcpyAsync(d, sp, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    else
        ACF_CUDA(cudaMemcpyPeerAsync(d, dst->device, sp, src->device, bytes, (cudaStream_t)stream));
    return ACF_OK;
}

int acf_solver_device(const acf_solver *h) { return h ? h->device : -1; }

int acf_run_slabs(acf_solver *const *parts, int32_t n_parts, const int32_t *own_lo,
                  const int32_t *own_hi, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    return run_slabs(parts, n_parts, own_lo, own_hi, n_steps, step_offset, stream);
}

int acf_profile_enable(acf_solver *h, int32_t enable) { return profile_enable(h, enable); }

int acf_profile_read(acf_solver *h, double *velocity_ms, double *pressure_ms, int64_t *launches) {
    return profile_read(h, velocity_ms, pressure_ms, launches);
}

int64_t acf_launch_count(const acf_solver *h) { return h ? h->launches : -1; }

int acf_set_scheme(acf_solver *h, int32_t scheme) { return set_scheme(h, scheme); }

int acf_get_scheme(const acf_solver *h) { return h ? h->scheme : -1; }

int acf_set_prefetch(acf_solver *h, int32_t mode) { return set_prefetch(h, mode); }

int acf_get_prefetch(const acf_solver *h) { return h ? (prefetch_planes(h) ? 1 : 0) : -1; }

int acf_set_time_blocking(acf_solver *h, int32_t steps_per_launch) {
    return set_time_blocking(h, steps_per_launch);
}

int acf_get_time_blocking(const acf_solver *h) { return h ? h->time_block : -1; }

int acf_set_staging(acf_solver *h, int32_t rows, int32_t stages, int32_t vector) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (rows < 1 || rows > 16) return fail(ACF_ERR_ARGUMENT, "rows must be in [1, 16], got %d", rows);
    if (stages != 0 && (stages < 2 || stages > kStagedMaxStages))
        return fail(ACF_ERR_ARGUMENT, "stages must be 0 or in [2, %d], got %d", kStagedMaxStages, stages);
    if (vector != 2 && vector != 4) return fail(ACF_ERR_ARGUMENT, "vector must be 2 or 4, got %d", vector);
    const RoomHost &room = h->rooms[0];
    if (staged_block_x(room, vector) * rows > kStagedMaxConsumers)
        return fail(ACF_ERR_ARGUMENT, "%d rows of %d threads exceed 256 threads per CTA", rows,
                    staged_block_x(room, vector));
    if (!staged_stages(h, rows, stages))
        return fail(ACF_ERR_ARGUMENT, "%d rows x %d stages do not fit in shared memory", rows, stages);
    if (rows != h->staged_rows || stages != h->staged_stages || vector != h->staged_vector)
        h->graph_dirty = h->adj_graphs_dirty = true;
    h->staged_rows = rows;
    h->staged_stages = stages;
    h->staged_vector = vector;
    return ACF_OK;
}

int acf_device_status(acf_solver *h, int32_t *status) { return device_status(h, status); }

int acf_batch_device_status(acf_batch *b, int32_t *status) { return device_status(b, status); }

int acf_set_wait_test(acf_solver *h, int64_t wait_limit_ns, int32_t skip_plane) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (wait_limit_ns != 0 && (wait_limit_ns < 1000000 || wait_limit_ns > (int64_t)kWaitLimitNs))
        return fail(ACF_ERR_ARGUMENT, "wait limit must be 0 (as built) or in [1 ms, %llu ns], got %lld",
                    (unsigned long long)kWaitLimitNs, (long long)wait_limit_ns);
    if (skip_plane < -1) return fail(ACF_ERR_ARGUMENT, "skip_plane must be -1 (none) or a plane index");
    h->test_wait_limit_ns = (uint64_t)wait_limit_ns;
    h->test_skip_plane = skip_plane;
    h->graph_dirty = true;     // the staged parameters are baked into captured graphs
    return ACF_OK;
}

int acf_set_coefficients(acf_solver *h, const acf_config *config) {
    return set_coefficients(h, 0, config);
}

int acf_reset_state(acf_solver *h, acf_stream stream) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    DeviceGuard guard(h->device);
    // The primary copy becomes current. No captured graph goes stale: the run graphs are kept
    // per starting copy, and the adjoint's graphs always work on the primary copy.
    h->rooms[0].cur = 0;
    h->po_first = true;
    h->po_started = false;
    ACF_CUDA(cudaMemsetAsync(h->field_ptr(0, ACF_FIELD_P), 0, h->room_block_bytes(0), (cudaStream_t)stream));
    return ACF_OK;
}

int acf_adjoint_prepare(acf_solver *h, int32_t flags, int64_t max_steps, int32_t checkpoint_every) {
    if (h && h->pressure_only())
        return fail(ACF_ERR_STATE, "the adjoint transposes the p-v step; select another scheme");
    return adjoint_prepare(h, flags, max_steps, checkpoint_every);
}

int64_t acf_adjoint_shell_size(const acf_solver *h) { return h ? h->adj.shell_total : -1; }

int32_t acf_adjoint_checkpoint_interval(const acf_solver *h) { return h ? h->adj.every : -1; }

int acf_forward_record(acf_solver *h, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (h->pressure_only())
        return fail(ACF_ERR_STATE, "the adjoint transposes the p-v step; select another scheme");
    if (!h->adj.fields) return fail(ACF_ERR_STATE, "call acf_adjoint_prepare first");
    if (n_steps < 1 || n_steps > h->adj.capacity)
        return fail(ACF_ERR_ARGUMENT, "n_steps %lld outside 1..%lld prepared", (long long)n_steps,
                    (long long)h->adj.capacity);
    if (step_offset < 0) return fail(ACF_ERR_ARGUMENT, "negative step offset");
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    {
        int rc0 = make_primary(h, st);
        if (rc0) return rc0;
    }
    // Recording capacity as acf_run ensures it.
    int rc = ACF_OK;
    for (RoomHost &r : h->rooms) {
        if (r.n_rec == 0) continue;
        const int64_t need = step_offset + n_steps - r.rec_origin;
        if (need <= r.rec_capacity) continue;
        // Reuse acf_run's growth path with a zero-step run is not possible; grow here.
        int64_t cap = round_up(std::max<int64_t>(need, 2 * r.rec_capacity), 256);
        const size_t es = h->elem();
        void *grown = nullptr;
        ACF_CUDA(cudaStreamSynchronize(st));
        ACF_CUDA(cudaMalloc(&grown, (size_t)r.n_rec * cap * es));
        ACF_CUDA(cudaMemset(grown, 0, (size_t)r.n_rec * cap * es));
        if (r.rec && r.rec_capacity > 0)
            ACF_CUDA(cudaMemcpy2D(grown, (size_t)cap * es, r.rec, (size_t)r.rec_capacity * es,
                                  (size_t)r.rec_capacity * es, (size_t)r.n_rec, cudaMemcpyDeviceToDevice));
        cudaFree(r.rec);
        r.rec = grown;
        r.rec_capacity = cap;
        h->graph_dirty = h->adj_graphs_dirty = true;
    }
    rc = h->precision == 8 ? forward_record_impl<double>(h, n_steps, step_offset, st)
                           : forward_record_impl<float>(h, n_steps, step_offset, st);
    return rc;
}

int acf_adjoint_run(acf_solver *h, const double *grad_rec, double *grad_src, double *grad_shell,
                    double *grad_air, acf_stream stream) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (!h->adj.fields || h->adj.recorded < 1) return fail(ACF_ERR_STATE, "no recorded forward run");
    if (h->rooms[0].n_rec > 0 && !grad_rec) return fail(ACF_ERR_ARGUMENT, "null receiver gradient");
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    return h->precision == 8 ? adjoint_impl<double>(h, grad_rec, grad_src, grad_shell, grad_air, st)
                             : adjoint_impl<float>(h, grad_rec, grad_src, grad_shell, grad_air, st);
}

int acf_adjoint_download(acf_solver *h, int field, void *dst, acf_stream stream) {
    if (!h || !dst) return fail(ACF_ERR_ARGUMENT, "null argument");
    if (!h->adj.fields) return fail(ACF_ERR_STATE, "call acf_adjoint_prepare first");
    if (field < 0 || field >= h->n_fields()) return fail(ACF_ERR_ARGUMENT, "field %d out of range", field);
    DeviceGuard guard(h->device);
    const RoomHost &r = h->rooms[0];
    int64_t shape[3];
    field_shape(r, field, shape);
    const size_t es = h->elem();
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((char *)h->adj.fields + (size_t)field * r.field * es, (size_t)r.pz * es,
                                   (size_t)r.pz, (size_t)(r.ny + 1));
    p.dstPtr = make_cudaPitchedPtr(dst, (size_t)shape[2] * es, (size_t)shape[2], (size_t)shape[1]);
    p.extent = make_cudaExtent((size_t)shape[2] * es, (size_t)shape[1], (size_t)shape[0]);
    p.kind = cudaMemcpyDefault;
    ACF_CUDA(cudaMemcpy3DAsync(&p, (cudaStream_t)stream));
    ACF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return ACF_OK;
}

// ---- batches of rooms -------------------------------------------------------------------

int acf_batch_create(int32_t n_rooms, const acf_config *configs, acf_batch **out) {
    if (!configs || !out) return fail(ACF_ERR_ARGUMENT, "null configs or output pointer");
    *out = nullptr;
    if (n_rooms < 1 || n_rooms > (1 << 20))
        return fail(ACF_ERR_ARGUMENT, "room count %d out of range", n_rooms);
    acf_batch *b = new (std::nothrow) acf_batch();
    if (!b) return fail(ACF_ERR_MEMORY, "host allocation failed");
    int rc = create_batch(n_rooms, configs, b);
    if (rc) {
        free_batch(b);
        return rc;
    }
    *out = b;
    return ACF_OK;
}

int acf_batch_destroy(acf_batch *b) {
    free_batch(b);
    return ACF_OK;
}

int acf_batch_room_count(const acf_batch *b) { return b ? (int)b->rooms.size() : -1; }

int acf_batch_set_sources(acf_batch *b, int32_t room, int64_t n, const int64_t *cell,
                          const int64_t *length, const double *signal, int64_t stride) {
    return set_sources(b, room, n, cell, length, signal, stride);
}

int acf_batch_set_receivers(acf_batch *b, int32_t room, int64_t n, const int64_t *cell,
                            const int64_t *start_step) {
    return set_receivers(b, room, n, cell, start_step);
}

int acf_batch_read_recording(acf_batch *b, int32_t room, int64_t receiver, int64_t first_step,
                             int64_t n, void *dst, acf_stream stream) {
    return read_recording(b, room, receiver, first_step, n, dst, stream);
}

int acf_batch_upload(acf_batch *b, int32_t room, int field, const void *src, acf_stream stream) {
    int rc = check_field(b, room, field);
    if (rc) return rc;
    if (!src) return fail(ACF_ERR_ARGUMENT, "null source");
    DeviceGuard guard(b->device);
    return copy_field(b, room, field, const_cast<void *>(src), true, (cudaStream_t)stream);
}

int acf_batch_download(acf_batch *b, int32_t room, int field, void *dst, acf_stream stream) {
    int rc = check_field(b, room, field);
    if (rc) return rc;
    if (!dst) return fail(ACF_ERR_ARGUMENT, "null destination");
    DeviceGuard guard(b->device);
    return copy_field(b, room, field, dst, false, (cudaStream_t)stream);
}

int acf_batch_run(acf_batch *b, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    return run_batch(b, n_steps, step_offset, stream);
}

int acf_batch_set_graph(acf_batch *b, int32_t steps) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null handle");
    if (steps < 0 || steps > 4096) return fail(ACF_ERR_ARGUMENT, "steps_per_graph %d out of range", steps);
    if (steps != b->graph_steps) b->graph_dirty = b->adj_graphs_dirty = true;
    b->graph_steps = steps;
    return ACF_OK;
}

int acf_batch_set_launch(acf_batch *b, int32_t block_threads, int32_t planes, int32_t ctas_per_sm) {
    return set_launch(b, block_threads, planes, ctas_per_sm);
}

int acf_batch_energy_terms(acf_batch *b, int32_t room, double dx, double terms[7], acf_stream stream) {
    return energy_terms(b, room, dx, terms, stream);
}

int acf_batch_profile_enable(acf_batch *b, int32_t enable) { return profile_enable(b, enable); }

int acf_batch_profile_read(acf_batch *b, double *velocity_ms, double *pressure_ms, int64_t *launches) {
    return profile_read(b, velocity_ms, pressure_ms, launches);
}

int64_t acf_batch_launch_count(const acf_batch *b) { return b ? b->launches : -1; }

int acf_batch_adjoint_prepare(acf_batch *b, int64_t max_steps) { return batch_adjoint_prepare(b, max_steps); }

int64_t acf_batch_adjoint_shell_size(const acf_batch *b, int32_t room) {
    if (!b || room < 0 || room >= (int)b->badj.size()) return -1;
    return b->badj[room].shell_total;
}

int acf_batch_forward_record(acf_batch *b, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null batch");
    if (b->badj.empty()) return fail(ACF_ERR_STATE, "call acf_batch_adjoint_prepare first");
    if (b->rooms.size() < 2) return fail(ACF_ERR_STATE, "single rooms use acf_forward_record");
    if (n_steps < 1 || n_steps > b->badj_capacity)
        return fail(ACF_ERR_ARGUMENT, "n_steps %lld outside 1..%lld prepared", (long long)n_steps,
                    (long long)b->badj_capacity);
    if (step_offset < 0) return fail(ACF_ERR_ARGUMENT, "negative step offset");
    DeviceGuard guard(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    {
        int rc0 = make_primary(b, st);   // the recorded run is the two sweeps, in place
        if (rc0) return rc0;
    }
    // recording capacity, as for a run
    for (RoomHost &r : b->rooms) {
        if (r.n_rec == 0) continue;
        const int64_t need = step_offset + n_steps - r.rec_origin;
        if (need <= r.rec_capacity) continue;
        int64_t cap = round_up(std::max<int64_t>(need, 2 * r.rec_capacity), 256);
        const size_t es = b->elem();
        void *grown = nullptr;
        ACF_CUDA(cudaStreamSynchronize(st));
        ACF_CUDA(cudaMalloc(&grown, (size_t)r.n_rec * cap * es));
        ACF_CUDA(cudaMemset(grown, 0, (size_t)r.n_rec * cap * es));
        if (r.rec && r.rec_capacity > 0)
            ACF_CUDA(cudaMemcpy2D(grown, (size_t)cap * es, r.rec, (size_t)r.rec_capacity * es,
                                  (size_t)r.rec_capacity * es, (size_t)r.n_rec, cudaMemcpyDeviceToDevice));
        cudaFree(r.rec);
        r.rec = grown;
        r.rec_capacity = cap;
        b->graph_dirty = b->adj_graphs_dirty = true;
        b->room_table_dirty = true;
    }
    return b->precision == 8 ? batch_forward_record_impl<double>(b, n_steps, step_offset, st)
                             : batch_forward_record_impl<float>(b, n_steps, step_offset, st);
}

int acf_batch_adjoint_run(acf_batch *b, const double *grad_rec, double *grad_src, double *grad_shell,
                          acf_stream stream) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null batch");
    if (b->badj.empty() || b->badj_recorded < 1) return fail(ACF_ERR_STATE, "no recorded forward run");
    DeviceGuard guard(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    return b->precision == 8 ? batch_adjoint_impl<double>(b, grad_rec, grad_src, grad_shell, st)
                             : batch_adjoint_impl<float>(b, grad_rec, grad_src, grad_shell, st);
}

int acf_batch_reset_state(acf_batch *b, acf_stream stream) {
    if (!b) return fail(ACF_ERR_ARGUMENT, "null batch");
    DeviceGuard guard(b->device);
    for (RoomHost &h : b->rooms) {
        if (h.cur) b->graph_dirty = b->adj_graphs_dirty = b->room_table_dirty = true;
        h.cur = 0;
    }
    ACF_CUDA(cudaMemsetAsync(b->state, 0, b->state_bytes, (cudaStream_t)stream));
    return ACF_OK;
}

int acf_batch_set_scheme(acf_batch *b, int32_t scheme) { return set_scheme(b, scheme); }

int acf_batch_set_prefetch(acf_batch *b, int32_t mode) { return set_prefetch(b, mode); }

int acf_batch_set_coefficients(acf_batch *b, int32_t room, const acf_config *config) {
    return set_coefficients(b, room, config);
}



// ---- utilities --------------------------------------------------------------------------

int acf_energy_terms_noalloc(const void *p, const void *vx, const void *vy, const void *vz,
                             int32_t nx, int32_t ny, int32_t nz, int32_t precision, double dx,
                             double *terms_device, acf_stream stream) {
    if (!p || !vx || !vy || !vz || !terms_device) return fail(ACF_ERR_ARGUMENT, "null field or output pointer");
    if (nx < 1 || ny < 1 || nz < 1)
        return fail(ACF_ERR_ARGUMENT, "cell counts must be >= 1, got (%d, %d, %d)", nx, ny, nz);
    if (precision != 4 && precision != 8)
        return fail(ACF_ERR_ARGUMENT, "precision must be 4 or 8 bytes, got %d", precision);
    if (!(dx > 0)) return fail(ACF_ERR_ARGUMENT, "dx must be positive");
    if ((int64_t)nx + 1 > ACF_NOALLOC_MAX_PLANES)
        return fail(ACF_ERR_ARGUMENT,
                    "nx + 1 = %lld x planes exceeds the static scratch of %d planes; "
                    "use acf_energy_terms for larger grids",
                    (long long)nx + 1, ACF_NOALLOC_MAX_PLANES);
    double *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const double inv_dx = 1.0 / dx;
    if (precision == 8)
        energy_dense_planes<double><<<nx + 1, 256, 0, st>>>((const double *)p, (const double *)vx,
                                                            (const double *)vy, (const double *)vz,
                                                            nx, ny, nz, inv_dx, scratch);
    else
        energy_dense_planes<float><<<nx + 1, 256, 0, st>>>((const float *)p, (const float *)vx,
                                                           (const float *)vy, (const float *)vz,
                                                           nx, ny, nz, inv_dx, scratch);
    energy_finish<<<1, 32, 0, st>>>(scratch, nx + 1, terms_device);
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

int acf_schroeder_decay(const double *response, int64_t channels, int64_t n, double floor_db,
                        double *decay, acf_stream stream) {
    int rc = check_post_args(response, decay, channels, n);
    if (rc) return rc;
    schroeder_decay_kernel<<<(unsigned)channels, kPostThreads, 0, (cudaStream_t)stream>>>(response, n, floor_db, decay);
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

int acf_decay_fit(const double *decay, int64_t channels, int64_t n, double sample_rate, double upper_db,
                  double lower_db, double *seconds, int32_t *failed, acf_stream stream) {
    int rc = check_post_args(decay, seconds, channels, n);
    if (rc) return rc;
    if (!failed) return fail(ACF_ERR_ARGUMENT, "null device array");
    if (!(sample_rate > 0.0)) return fail(ACF_ERR_ARGUMENT, "sample rate must be positive");
    decay_fit_kernel<<<(unsigned)channels, kPostThreads, 0, (cudaStream_t)stream>>>(decay, n, sample_rate, upper_db,
                                                                                lower_db, seconds, failed);
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

int acf_clarity(const double *response, int64_t channels, int64_t n, int64_t boundary, double *db,
                acf_stream stream) {
    int rc = check_post_args(response, db, channels, n);
    if (rc) return rc;
    clarity_kernel<<<(unsigned)channels, kPostThreads, 0, (cudaStream_t)stream>>>(response, n, boundary, db);
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

int acf_spectral_divide(const void *spectra, const void *source, int64_t channels, int64_t bins,
                        double bin_hz, double max_frequency, double regularisation, double *scratch,
                        void *out, acf_stream stream) {
    int rc = check_post_args(spectra, source, channels, bins);
    if (rc) return rc;
    if (!scratch || !out) return fail(ACF_ERR_ARGUMENT, "null device array");
    cudaStream_t st = (cudaStream_t)stream;
    spectrum_peak_power<<<1, kPostThreads, 0, st>>>((const double2 *)source, bins, scratch);
    const int64_t total = channels * bins;
    spectral_divide_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        (const double2 *)spectra, (const double2 *)source, channels, bins, bin_hz, max_frequency,
        regularisation, scratch, (double2 *)out);
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

int acf_synchronize(acf_stream stream) {
    ACF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return ACF_OK;
}

int acf_host_alloc(size_t bytes, void **out) {
    if (!out) return fail(ACF_ERR_ARGUMENT, "null output");
    *out = nullptr;
    if (bytes == 0) return ACF_OK;
    if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess)
        return fail(ACF_ERR_MEMORY, "cudaHostAlloc of %zu bytes failed", bytes);
    return ACF_OK;
}

int acf_host_free(void *ptr) {
    if (ptr) ACF_CUDA(cudaFreeHost(ptr));
    return ACF_OK;
}

}  // extern "C"
