// acfdtd_b200.cu -- the staggered pressure-velocity leapfrog on sm_100a, behind a C ABI.
//
// One time step is two HBM-bound sweeps over the grid (ac-fdtd: src/ac_fdtd/scheme.py:285-296,
// src/ac_fdtd/c/acfdtd.c:110-190,342-376):
//
//   (a) velocity_sweep: v_a -= c_v (p_hi - p_lo) on interior faces, then the absorbing-layer
//       damping x, y, z in that order on every face (scheme.py:287-290,298-311).
//   (b) pressure_sweep: div v, the relaxation states, p -= c_p div, the time-centred wall
//       closed form, the layer damping, the volume sources and the receiver gather, all in the
//       registers of the thread that owns the cell (scheme.py:291-296,313-363).
//
// Arithmetic order follows the NumPy reference operation by operation and the library is
// built with -fmad=false, so no multiply-add is contracted: both precisions reproduce the
// reference's own float64/float32 arithmetic.
//
// Layout in HBM: every field uses the same padded geometry, (nx+1) planes of (ny+1) rows of
// pz elements, pz = nz+1 rounded up to a multiple of 8. Element (i,j,k) of any field is at
// (i*(ny+1) + j)*pz + k, so vx's extra plane, vy's extra row and vz's extra face all fit and a
// neighbour on any axis is a constant stride away. Rows start on 32-byte boundaries, which
// keeps every 4-element group of a thread a single aligned vector access.

#include <cuda_runtime.h>

#include <algorithm>
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
};

// ------------------------------------------------------------------------------------------
// Kernel parameters (passed by value).

template <typename T>
struct StepParams {
    int32_t nx, ny, nz, nchunks;
    int64_t pz, plane, field;      // row pitch, plane pitch, elements per field
    T *p, *vx, *vy, *vz, *psi;     // psi: n_relax fields back to back
    T cv, cp, cs, relax_scale;
    T decay[ACF_MAX_RELAXATION], mean[ACF_MAX_RELAXATION], gain[ACF_MAX_RELAXATION];
    const T *cell[3];              // layer profiles at cell centres
    const T *face[3];              // layer profiles at faces
    const T *shell[6];             // wall pairs (1/(1+a), a/(1+a)) per face cell
    int32_t n_src;
    const int64_t *src_off;        // padded offsets
    const int64_t *src_len;
    const T *src_sig;
    int64_t src_stride;
    int32_t n_rec;
    const int64_t *rec_off;        // padded offsets
    const int64_t *rec_start;      // first absolute step recorded
    T *rec;
    int64_t rec_stride, rec_origin;
    const int64_t *step_base;      // absolute step of local step 0, in device memory
    int32_t local_step;
};

// ------------------------------------------------------------------------------------------
// (a) velocity sweep. Thread (chunk c, row j) marches over planes i. Each cell owns the lower
// face of each axis; the far boundary faces (x = nx, y = ny, z = nz) are only ever damped.

template <typename T, bool LAYER>
__global__ void __launch_bounds__(256) velocity_sweep(const StepParams<T> s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= s.nchunks || j >= s.ny) return;
    const int k0 = c * kVec;
    const T cv = s.cv;

    T fk_cell[kVec], fk_face[kVec];
    T fj_cell = T(1), fj_face = T(1);
    if (LAYER) {
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = min(k0 + e, s.nz - 1);
            fk_cell[e] = s.cell[2][k];
            fk_face[e] = s.face[2][min(k0 + e, s.nz)];
        }
        fj_cell = s.cell[1][j];
        fj_face = s.face[1][j];
    }

    for (int i = blockIdx.z; i < s.nx; i += gridDim.z) {
        const int64_t base = (int64_t)i * s.plane + (int64_t)j * s.pz + k0;
        T fi_cell = T(1), fi_face = T(1);
        if (LAYER) {
            fi_cell = s.cell[0][i];
            fi_face = s.face[0][i];
        }
        T P[kVec];
        Vec4<T>::load(s.p + base, P);

        // vx, lower x face of cell (i, j, k): interior for i >= 1.
        {
            T V[kVec];
            Vec4<T>::load(s.vx + base, V);
            T Q[kVec];
            if (i > 0) Vec4<T>::load(s.p + base - s.plane, Q);
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                if (k0 + e < s.nz) {
                    T v = V[e];
                    if (i > 0) v = v - cv * (P[e] - Q[e]);
                    if (LAYER) {
                        v = v * fi_face;
                        v = v * fj_cell;
                        v = v * fk_cell[e];
                    }
                    V[e] = v;
                }
            }
            Vec4<T>::store(s.vx + base, V);
        }
        // vy, lower y face: interior for j >= 1.
        {
            T V[kVec];
            Vec4<T>::load(s.vy + base, V);
            T Q[kVec];
            if (j > 0) Vec4<T>::load(s.p + base - s.pz, Q);
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                if (k0 + e < s.nz) {
                    T v = V[e];
                    if (j > 0) v = v - cv * (P[e] - Q[e]);
                    if (LAYER) {
                        v = v * fi_cell;
                        v = v * fj_face;
                        v = v * fk_cell[e];
                    }
                    V[e] = v;
                }
            }
            Vec4<T>::store(s.vy + base, V);
        }
        // vz, lower z face: interior for k >= 1.
        {
            T V[kVec];
            Vec4<T>::load(s.vz + base, V);
            const T below = (k0 > 0) ? s.p[base - 1] : T(0);
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                const int k = k0 + e;
                if (k < s.nz) {
                    T v = V[e];
                    if (k > 0) v = v - cv * (P[e] - (e == 0 ? below : P[e - 1]));
                    if (LAYER) {
                        v = v * fi_cell;
                        v = v * fj_cell;
                        v = v * fk_face[e];
                    }
                    V[e] = v;
                }
            }
            Vec4<T>::store(s.vz + base, V);
        }
        // Far boundary faces: never updated, but the reference damps them with its slabs.
        if (LAYER) {
            if (i == s.nx - 1) {
                T V[kVec];
                Vec4<T>::load(s.vx + base + s.plane, V);
                const T f = s.face[0][s.nx];
#pragma unroll
                for (int e = 0; e < kVec; e++)
                    if (k0 + e < s.nz) {
                        T v = V[e] * f;
                        v = v * fj_cell;
                        V[e] = v * fk_cell[e];
                    }
                Vec4<T>::store(s.vx + base + s.plane, V);
            }
            if (j == s.ny - 1) {
                T V[kVec];
                Vec4<T>::load(s.vy + base + s.pz, V);
                const T f = s.face[1][s.ny];
#pragma unroll
                for (int e = 0; e < kVec; e++)
                    if (k0 + e < s.nz) {
                        T v = V[e] * fi_cell;
                        v = v * f;
                        V[e] = v * fk_cell[e];
                    }
                Vec4<T>::store(s.vy + base + s.pz, V);
            }
            if (s.nz - 1 >= k0 && s.nz - 1 < k0 + kVec) {
                T *top = s.vz + (base - k0) + s.nz;
                T v = *top * fi_cell;
                v = v * fj_cell;
                *top = v * s.face[2][s.nz];
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// (b) pressure sweep.

template <typename T>
__device__ __forceinline__ bool wall_pair(const StepParams<T> &s, int i, int j, int k, T &fu,
                                          T &fp) {
    const T *entry;
    if (i == 0) entry = s.shell[0] + 2 * ((int64_t)j * s.nz + k);
    else if (i == s.nx - 1) entry = s.shell[1] + 2 * ((int64_t)j * s.nz + k);
    else if (j == 0) entry = s.shell[2] + 2 * ((int64_t)i * s.nz + k);
    else if (j == s.ny - 1) entry = s.shell[3] + 2 * ((int64_t)i * s.nz + k);
    else if (k == 0) entry = s.shell[4] + 2 * ((int64_t)i * s.ny + j);
    else if (k == s.nz - 1) entry = s.shell[5] + 2 * ((int64_t)i * s.ny + j);
    else return false;
    fu = entry[0];
    fp = entry[1];
    return fp != T(0) || fu != T(1);
}

template <typename T, bool LAYER, bool WALLS, int NR>
__global__ void __launch_bounds__(256) pressure_sweep(const StepParams<T> s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= s.nchunks || j >= s.ny) return;
    const int k0 = c * kVec;
    const bool any_point = (s.n_src | s.n_rec) != 0;
    const int64_t step = any_point ? (*s.step_base + s.local_step) : 0;

    T fk[kVec];
    T fj = T(1);
    if (LAYER) {
#pragma unroll
        for (int e = 0; e < kVec; e++) fk[e] = s.cell[2][min(k0 + e, s.nz - 1)];
        fj = s.cell[1][j];
    }
    const T cp = s.cp;

    for (int i = blockIdx.z; i < s.nx; i += gridDim.z) {
        const int64_t base = (int64_t)i * s.plane + (int64_t)j * s.pz + k0;

        // Divergence, summed x, then y, then z as the reference does (scheme.py:317-322).
        T D[kVec];
        {
            T A[kVec], B[kVec];
            Vec4<T>::load(s.vx + base, A);
            Vec4<T>::load(s.vx + base + s.plane, B);
#pragma unroll
            for (int e = 0; e < kVec; e++) D[e] = B[e] - A[e];
            Vec4<T>::load(s.vy + base, A);
            Vec4<T>::load(s.vy + base + s.pz, B);
#pragma unroll
            for (int e = 0; e < kVec; e++) D[e] = D[e] + (B[e] - A[e]);
            Vec4<T>::load(s.vz + base, A);
            const T above = (k0 + kVec <= s.nz) ? s.vz[base + kVec] : T(0);
#pragma unroll
            for (int e = 0; e < kVec; e++) D[e] = D[e] + ((e + 1 < kVec ? A[e + 1] : above) - A[e]);
        }

        T P[kVec], Pn[kVec];
        Vec4<T>::load(s.p + base, P);
#pragma unroll
        for (int e = 0; e < kVec; e++) Pn[e] = P[e];

        // Relaxation states (scheme.py:337-358), then p -= c_p div (scheme.py:325-326).
#pragma unroll
        for (int r = 0; r < NR; r++) {
            T S[kVec];
            T *psi = s.psi + r * s.field + base;
            Vec4<T>::load(psi, S);
#pragma unroll
            for (int e = 0; e < kVec; e++) {
                if (k0 + e < s.nz) {
                    const T target = D[e] * s.gain[r];
                    const T offset = S[e] - target;
                    S[e] = offset * s.decay[r] + target;
                    Pn[e] = Pn[e] + offset * s.mean[r];
                }
            }
            Vec4<T>::store(psi, S);
        }

        const T fi = LAYER ? s.cell[0][i] : T(1);
#pragma unroll
        for (int e = 0; e < kVec; e++) {
            const int k = k0 + e;
            if (k >= s.nz) continue;
            T pe = Pn[e];
            if (NR > 0) pe = pe + D[e] * s.relax_scale;
            pe = pe - D[e] * cp;
            if (WALLS) {
                T fu, fp;
                if (wall_pair(s, i, j, k, fu, fp)) pe = pe * fu - P[e] * fp;
            }
            if (LAYER) {
                pe = pe * fi;
                pe = pe * fj;
                pe = pe * fk[e];
            }
            Pn[e] = pe;
        }

        // Sources after damping, in the order they were added (scheme.py:293,360-363).
        if (any_point) {
            for (int q = 0; q < s.n_src; q++) {
                const int64_t d = s.src_off[q] - base;
                if (d >= 0 && d < kVec && k0 + d < s.nz && step < s.src_len[q]) {
#pragma unroll
                    for (int e = 0; e < kVec; e++)
                        if (e == d) Pn[e] = Pn[e] + s.cs * s.src_sig[q * s.src_stride + step];
                }
            }
        }
        Vec4<T>::store(s.p + base, Pn);

        // Receivers read the finished p (scheme.py:294-296).
        if (any_point) {
            for (int r = 0; r < s.n_rec; r++) {
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
    }
}

__global__ void set_step_base(int64_t *base, int64_t value) { *base = value; }
__global__ void bump_step_base(int64_t *base, int64_t by) { *base += by; }

// ------------------------------------------------------------------------------------------
// Energy terms, FP64 accumulation (scheme.py:365-389). Two passes, fixed order: block partial
// sums into a scratch array, then one block sums the partials.

template <typename T>
__global__ void __launch_bounds__(256) energy_partials(const StepParams<T> s, double inv_dx,
                                                       double *partials) {
    double acc[kEnergyTerms];
#pragma unroll
    for (int t = 0; t < kEnergyTerms; t++) acc[t] = 0.0;

    const int64_t rows = (int64_t)(s.nx + 1) * (s.ny + 1);
    const int64_t total = rows * (s.nz + 1);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < total;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(n % (s.nz + 1));
        const int64_t row = n / (s.nz + 1);
        const int j = (int)(row % (s.ny + 1));
        const int i = (int)(row / (s.ny + 1));
        const int64_t o = (int64_t)i * s.plane + (int64_t)j * s.pz + k;
        const bool in_x = i < s.nx, in_y = j < s.ny, in_z = k < s.nz;
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

// ------------------------------------------------------------------------------------------
// Host side.

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

}  // namespace

struct acf_solver {
    int device = 0;
    int precision = 8;
    int32_t nx = 0, ny = 0, nz = 0, n_relax = 0;
    int64_t pz = 0, plane = 0, field = 0;
    bool has_layer = false, has_walls = false;
    double coef[4] = {0, 0, 0, 0};   // cv, cp, cs, relax_scale
    double decay[ACF_MAX_RELAXATION] = {}, mean[ACF_MAX_RELAXATION] = {},
           gain[ACF_MAX_RELAXATION] = {};

    void *state = nullptr;           // p, vx, vy, vz, psi[n_relax], contiguous fields
    void *profiles = nullptr;        // cell[3] then face[3], solver precision
    int64_t profile_off[6] = {};
    void *shell = nullptr;           // 6 faces of wall pairs, solver precision
    int64_t shell_off[6] = {};
    int64_t *step_base = nullptr;    // one int64 in device memory
    double *energy_scratch = nullptr;
    int energy_blocks = 0;

    // sources
    int64_t n_src = 0, src_stride = 0;
    int64_t *src_off = nullptr, *src_len = nullptr;
    void *src_sig = nullptr;
    // receivers
    int64_t n_rec = 0, rec_capacity = 0, rec_origin = 0;
    bool rec_origin_set = false;
    int64_t *rec_off = nullptr, *rec_start = nullptr;
    void *rec = nullptr;
    std::vector<int64_t> host_rec_cell, host_rec_start;

    // graphs
    int32_t graph_steps = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture_stream = nullptr;
    bool graph_dirty = true;

    // profiling
    bool profiling = false;
    double prof_velocity_ms = 0, prof_pressure_ms = 0;
    int64_t prof_launches = 0;
    static constexpr int64_t kRing = 64;
    cudaEvent_t ring[3 * kRing] = {};

    int64_t launches = 0;

    size_t elem() const { return (size_t)precision; }
    char *field_ptr(int f) const { return (char *)state + (size_t)f * field * elem(); }
};

namespace {

template <typename T>
StepParams<T> make_params(const acf_solver *h) {
    StepParams<T> s{};
    s.nx = h->nx;
    s.ny = h->ny;
    s.nz = h->nz;
    s.nchunks = (int32_t)((h->nz + kVec - 1) / kVec);
    s.pz = h->pz;
    s.plane = h->plane;
    s.field = h->field;
    s.p = (T *)h->field_ptr(ACF_FIELD_P);
    s.vx = (T *)h->field_ptr(ACF_FIELD_VX);
    s.vy = (T *)h->field_ptr(ACF_FIELD_VY);
    s.vz = (T *)h->field_ptr(ACF_FIELD_VZ);
    s.psi = (T *)h->field_ptr(ACF_FIELD_PSI0);
    s.cv = (T)h->coef[0];
    s.cp = (T)h->coef[1];
    s.cs = (T)h->coef[2];
    s.relax_scale = (T)h->coef[3];
    for (int r = 0; r < ACF_MAX_RELAXATION; r++) {
        s.decay[r] = (T)h->decay[r];
        s.mean[r] = (T)h->mean[r];
        s.gain[r] = (T)h->gain[r];
    }
    for (int a = 0; a < 3; a++) {
        s.cell[a] = h->has_layer ? (const T *)h->profiles + h->profile_off[a] : nullptr;
        s.face[a] = h->has_layer ? (const T *)h->profiles + h->profile_off[3 + a] : nullptr;
    }
    for (int f = 0; f < 6; f++)
        s.shell[f] = h->has_walls ? (const T *)h->shell + h->shell_off[f] : nullptr;
    s.n_src = (int32_t)h->n_src;
    s.src_off = h->src_off;
    s.src_len = h->src_len;
    s.src_sig = (const T *)h->src_sig;
    s.src_stride = h->src_stride;
    s.n_rec = (int32_t)h->n_rec;
    s.rec_off = h->rec_off;
    s.rec_start = h->rec_start;
    s.rec = (T *)h->rec;
    s.rec_stride = h->rec_capacity;
    s.rec_origin = h->rec_origin;
    s.step_base = h->step_base;
    s.local_step = 0;
    return s;
}

struct LaunchShape {
    dim3 grid, block;
};

LaunchShape sweep_shape(const acf_solver *h) {
    const int nchunks = (int)((h->nz + kVec - 1) / kVec);
    int bx = 1;
    while (bx < nchunks && bx < 32) bx <<= 1;
    int by = std::max(1, std::min<int>(h->ny, 128 / bx));
    LaunchShape L;
    L.block = dim3(bx, by, 1);
    L.grid = dim3((nchunks + bx - 1) / bx, (h->ny + by - 1) / by, std::min<int>(h->nx, 65535));
    return L;
}

template <typename T, bool LAYER>
void launch_velocity(const StepParams<T> &s, const LaunchShape &L, cudaStream_t st) {
    velocity_sweep<T, LAYER><<<L.grid, L.block, 0, st>>>(s);
}

template <typename T, bool LAYER, bool WALLS>
void launch_pressure_nr(const StepParams<T> &s, int nr, const LaunchShape &L, cudaStream_t st) {
    switch (nr) {
        case 0: pressure_sweep<T, LAYER, WALLS, 0><<<L.grid, L.block, 0, st>>>(s); break;
        case 1: pressure_sweep<T, LAYER, WALLS, 1><<<L.grid, L.block, 0, st>>>(s); break;
        case 2: pressure_sweep<T, LAYER, WALLS, 2><<<L.grid, L.block, 0, st>>>(s); break;
        case 3: pressure_sweep<T, LAYER, WALLS, 3><<<L.grid, L.block, 0, st>>>(s); break;
        default: pressure_sweep<T, LAYER, WALLS, 4><<<L.grid, L.block, 0, st>>>(s); break;
    }
}

template <typename T>
void launch_step(const acf_solver *h, StepParams<T> s, int32_t local, const LaunchShape &L,
                 cudaStream_t st, cudaEvent_t *events) {
    s.local_step = local;
    if (events) cudaEventRecord(events[0], st);
    if (h->has_layer) launch_velocity<T, true>(s, L, st);
    else launch_velocity<T, false>(s, L, st);
    if (events) cudaEventRecord(events[1], st);
    if (h->has_layer) {
        if (h->has_walls) launch_pressure_nr<T, true, true>(s, h->n_relax, L, st);
        else launch_pressure_nr<T, true, false>(s, h->n_relax, L, st);
    } else {
        if (h->has_walls) launch_pressure_nr<T, false, true>(s, h->n_relax, L, st);
        else launch_pressure_nr<T, false, false>(s, h->n_relax, L, st);
    }
    if (events) cudaEventRecord(events[2], st);
}

template <typename T>
int run_impl(acf_solver *h, int64_t n_steps, int64_t step_offset, cudaStream_t st) {
    const LaunchShape L = sweep_shape(h);
    const StepParams<T> s = make_params<T>(h);
    set_step_base<<<1, 1, 0, st>>>(h->step_base, step_offset);
    h->launches += 1;

    if (h->profiling) {
        // Event ring: the host waits on a step's events only when the ring wraps, so the
        // queue stays full while the sweeps are being timed.
        const int64_t R = acf_solver::kRing;
        auto drain = [&](int64_t slot) -> int {
            cudaEvent_t *e = h->ring + 3 * slot;
            ACF_CUDA(cudaEventSynchronize(e[2]));
            float a = 0, b = 0;
            ACF_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
            ACF_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
            h->prof_velocity_ms += a;
            h->prof_pressure_ms += b;
            h->prof_launches += 1;
            return ACF_OK;
        };
        for (int64_t t = 0; t < n_steps; t++) {
            const int64_t slot = t % R;
            if (t >= R) {
                int rc = drain(slot);
                if (rc) return rc;
            }
            launch_step<T>(h, s, (int32_t)0, L, st, h->ring + 3 * slot);
            bump_step_base<<<1, 1, 0, st>>>(h->step_base, 1);
            h->launches += 3;
        }
        for (int64_t t = std::max<int64_t>(0, n_steps - R); t < n_steps; t++) {
            int rc = drain(t % R);
            if (rc) return rc;
        }
        ACF_CUDA(cudaGetLastError());
        return ACF_OK;
    }

    int64_t done = 0;
    const int64_t G = h->graph_steps;
    if (G > 0 && n_steps >= G) {
        if (h->graph_dirty || !h->graph) {
            if (h->graph) {
                cudaGraphExecDestroy(h->graph);
                h->graph = nullptr;
            }
            if (!h->capture_stream)
                ACF_CUDA(cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking));
            ACF_CUDA(cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal));
            for (int64_t t = 0; t < G; t++) launch_step<T>(h, s, (int32_t)t, L, h->capture_stream, nullptr);
            bump_step_base<<<1, 1, 0, h->capture_stream>>>(h->step_base, G);
            cudaGraph_t graph = nullptr;
            ACF_CUDA(cudaStreamEndCapture(h->capture_stream, &graph));
            cudaError_t err = cudaGraphInstantiate(&h->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (err != cudaSuccess)
                return fail(ACF_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(err));
            h->graph_dirty = false;
        }
        for (; done + G <= n_steps; done += G) {
            ACF_CUDA(cudaGraphLaunch(h->graph, st));
            h->launches += 2 * G + 1;
        }
    }
    for (int64_t t = 0; done + t < n_steps; t++) {
        launch_step<T>(h, s, (int32_t)t, L, st, nullptr);
        h->launches += 2;
    }
    ACF_CUDA(cudaGetLastError());
    return ACF_OK;
}

template <typename T>
int energy_impl(acf_solver *h, double dx, double *terms, cudaStream_t st) {
    const StepParams<T> s = make_params<T>(h);
    energy_partials<T><<<h->energy_blocks, 256, 0, st>>>(s, 1.0 / dx, h->energy_scratch);
    energy_finish<<<1, 32, 0, st>>>(h->energy_scratch, h->energy_blocks,
                                    h->energy_scratch + (size_t)h->energy_blocks * kEnergyTerms);
    h->launches += 2;
    ACF_CUDA(cudaGetLastError());
    ACF_CUDA(cudaMemcpyAsync(terms, h->energy_scratch + (size_t)h->energy_blocks * kEnergyTerms,
                             kEnergyTerms * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACF_CUDA(cudaStreamSynchronize(st));
    return ACF_OK;
}

// Reference shape of a field: (nx + [f==VX], ny + [f==VY], nz + [f==VZ]).
void field_shape(const acf_solver *h, int f, int64_t shape[3]) {
    shape[0] = h->nx + (f == ACF_FIELD_VX);
    shape[1] = h->ny + (f == ACF_FIELD_VY);
    shape[2] = h->nz + (f == ACF_FIELD_VZ);
}

int check_field(const acf_solver *h, int f) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (f < 0 || f >= ACF_FIELD_PSI0 + h->n_relax)
        return fail(ACF_ERR_ARGUMENT, "field %d out of range (0..%d)", f, ACF_FIELD_PSI0 + h->n_relax - 1);
    return ACF_OK;
}

int copy_field(acf_solver *h, int f, void *host_or_dev, bool upload, cudaStream_t st) {
    int64_t shape[3];
    field_shape(h, f, shape);
    const size_t es = h->elem();
    cudaMemcpy3DParms p = {};
    cudaPitchedPtr dense = make_cudaPitchedPtr(host_or_dev, (size_t)shape[2] * es, (size_t)shape[2],
                                               (size_t)shape[1]);
    cudaPitchedPtr padded = make_cudaPitchedPtr(h->field_ptr(f), (size_t)h->pz * es, (size_t)h->pz,
                                                (size_t)(h->ny + 1));
    p.srcPtr = upload ? dense : padded;
    p.dstPtr = upload ? padded : dense;
    p.extent = make_cudaExtent((size_t)shape[2] * es, (size_t)shape[1], (size_t)shape[0]);
    p.kind = cudaMemcpyDefault;
    ACF_CUDA(cudaMemcpy3DAsync(&p, st));
    return ACF_OK;
}

int64_t padded_offset(const acf_solver *h, int64_t flat) {
    const int64_t k = flat % h->nz;
    const int64_t j = (flat / h->nz) % h->ny;
    const int64_t i = flat / ((int64_t)h->nz * h->ny);
    return i * h->plane + j * h->pz + k;
}

template <typename T>
void cast_copy(void *dst, const double *src, size_t n) {
    T *d = (T *)dst;
    for (size_t q = 0; q < n; q++) d[q] = (T)src[q];
}

void free_solver(acf_solver *h) {
    if (!h) return;
    DeviceGuard guard(h->device);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
    for (auto &e : h->ring)
        if (e) cudaEventDestroy(e);
    cudaFree(h->state);
    cudaFree(h->profiles);
    cudaFree(h->shell);
    cudaFree(h->step_base);
    cudaFree(h->energy_scratch);
    cudaFree(h->src_off);
    cudaFree(h->src_len);
    cudaFree(h->src_sig);
    cudaFree(h->rec_off);
    cudaFree(h->rec_start);
    cudaFree(h->rec);
    delete h;
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

int acf_create(const acf_config *cfg, acf_solver **out) {
    if (!cfg || !out) return fail(ACF_ERR_ARGUMENT, "null config or output pointer");
    *out = nullptr;
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1)
        return fail(ACF_ERR_ARGUMENT, "cell counts must be >= 1, got (%d, %d, %d)", cfg->nx, cfg->ny, cfg->nz);
    if (cfg->precision != 4 && cfg->precision != 8)
        return fail(ACF_ERR_ARGUMENT, "precision must be 4 or 8 bytes, got %d", cfg->precision);
    if (cfg->n_relax < 0 || cfg->n_relax > ACF_MAX_RELAXATION)
        return fail(ACF_ERR_ARGUMENT, "the kernel holds at most %d relaxation processes, got %d",
                    ACF_MAX_RELAXATION, cfg->n_relax);
    const bool layer = cfg->cell[0] != nullptr;
    for (int a = 0; a < 3; a++)
        if ((cfg->cell[a] != nullptr) != layer || (cfg->face[a] != nullptr) != layer)
            return fail(ACF_ERR_ARGUMENT, "layer profiles must be all given or all NULL");
    const bool walls = cfg->wall_shell[0] != nullptr;
    for (int f = 0; f < 6; f++)
        if ((cfg->wall_shell[f] != nullptr) != walls)
            return fail(ACF_ERR_ARGUMENT, "wall shells must be all given or all NULL");

    acf_solver *h = new (std::nothrow) acf_solver();
    if (!h) return fail(ACF_ERR_MEMORY, "host allocation failed");
    cudaError_t e = cudaGetDevice(&h->device);
    if (e != cudaSuccess) {
        delete h;
        return fail(ACF_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    }
    h->precision = cfg->precision;
    h->nx = cfg->nx;
    h->ny = cfg->ny;
    h->nz = cfg->nz;
    h->n_relax = cfg->n_relax;
    h->pz = round_up((int64_t)cfg->nz + 1, kRowAlign);
    h->plane = (int64_t)(cfg->ny + 1) * h->pz;
    h->field = (int64_t)(cfg->nx + 1) * h->plane;
    h->has_layer = layer;
    h->has_walls = walls;
    h->coef[0] = cfg->vel_coef;
    h->coef[1] = cfg->pres_coef;
    h->coef[2] = cfg->src_coef;
    h->coef[3] = cfg->relax_scale;
    for (int r = 0; r < ACF_MAX_RELAXATION; r++) {
        h->decay[r] = r < cfg->n_relax ? cfg->relax_decay[r] : 0.0;
        h->mean[r] = r < cfg->n_relax ? cfg->relax_mean[r] : 0.0;
        h->gain[r] = r < cfg->n_relax ? cfg->relax_gain[r] : 0.0;
    }

    auto cleanup = [&](int code) {
        free_solver(h);
        return code;
    };
    const size_t es = h->elem();
    const size_t n_fields = 4 + (size_t)h->n_relax;
    // One guard row past the last field keeps every vector access of the last row in bounds.
    const size_t state_bytes = (n_fields * (size_t)h->field + (size_t)h->pz) * es;
    if (cudaMalloc(&h->state, state_bytes) != cudaSuccess)
        return cleanup(fail(ACF_ERR_MEMORY, "cudaMalloc of %zu bytes of state failed", state_bytes));
    if (cudaMemset(h->state, 0, state_bytes) != cudaSuccess)
        return cleanup(fail(ACF_ERR_CUDA, "cudaMemset of state failed"));
    if (cudaMalloc(&h->step_base, sizeof(int64_t)) != cudaSuccess)
        return cleanup(fail(ACF_ERR_MEMORY, "cudaMalloc of step counter failed"));
    cudaMemset(h->step_base, 0, sizeof(int64_t));

    const int64_t n_axis[3] = {cfg->nx, cfg->ny, cfg->nz};
    if (layer) {
        std::vector<double> host;
        for (int a = 0; a < 3; a++) {
            h->profile_off[a] = (int64_t)host.size();
            host.insert(host.end(), cfg->cell[a], cfg->cell[a] + n_axis[a]);
        }
        for (int a = 0; a < 3; a++) {
            h->profile_off[3 + a] = (int64_t)host.size();
            host.insert(host.end(), cfg->face[a], cfg->face[a] + n_axis[a] + 1);
        }
        std::vector<char> cast(host.size() * es);
        if (es == 4) cast_copy<float>(cast.data(), host.data(), host.size());
        else cast_copy<double>(cast.data(), host.data(), host.size());
        if (cudaMalloc(&h->profiles, cast.size()) != cudaSuccess)
            return cleanup(fail(ACF_ERR_MEMORY, "cudaMalloc of layer profiles failed"));
        if (cudaMemcpy(h->profiles, cast.data(), cast.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return cleanup(fail(ACF_ERR_CUDA, "copy of layer profiles failed"));
    }
    if (walls) {
        std::vector<double> host;
        for (int f = 0; f < 6; f++) {
            const int axis = f / 2;
            const int64_t nb = axis == 0 ? n_axis[1] : n_axis[0];
            const int64_t nc = axis == 2 ? n_axis[1] : n_axis[2];
            h->shell_off[f] = (int64_t)host.size();
            host.insert(host.end(), cfg->wall_shell[f], cfg->wall_shell[f] + 2 * nb * nc);
        }
        std::vector<char> cast(host.size() * es);
        if (es == 4) cast_copy<float>(cast.data(), host.data(), host.size());
        else cast_copy<double>(cast.data(), host.data(), host.size());
        if (cudaMalloc(&h->shell, cast.size()) != cudaSuccess)
            return cleanup(fail(ACF_ERR_MEMORY, "cudaMalloc of wall shells failed"));
        if (cudaMemcpy(h->shell, cast.data(), cast.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return cleanup(fail(ACF_ERR_CUDA, "copy of wall shells failed"));
    }

    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    h->energy_blocks = 4 * sms;
    const size_t scratch = ((size_t)h->energy_blocks + 1) * kEnergyTerms * sizeof(double);
    if (cudaMalloc(&h->energy_scratch, scratch) != cudaSuccess)
        return cleanup(fail(ACF_ERR_MEMORY, "cudaMalloc of energy scratch failed"));
    for (auto &ev : h->ring)
        if (cudaEventCreate(&ev) != cudaSuccess) return cleanup(fail(ACF_ERR_CUDA, "cudaEventCreate failed"));
    *out = h;
    return ACF_OK;
}

int acf_destroy(acf_solver *h) {
    free_solver(h);
    return ACF_OK;
}

int acf_is_double(const acf_solver *h) { return h && h->precision == 8; }

int acf_set_sources(acf_solver *h, int64_t n, const int64_t *cell, const int64_t *length,
                    const double *signal, int64_t stride) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (n < 0 || n > (1 << 20)) return fail(ACF_ERR_ARGUMENT, "source count %lld out of range", (long long)n);
    if (n > 0 && (!cell || !length || (stride > 0 && !signal) || stride < 0))
        return fail(ACF_ERR_ARGUMENT, "null source arrays");
    DeviceGuard guard(h->device);
    const int64_t n_cells = (int64_t)h->nx * h->ny * h->nz;
    std::vector<int64_t> off((size_t)n), len((size_t)n);
    for (int64_t q = 0; q < n; q++) {
        if (cell[q] < 0 || cell[q] >= n_cells)
            return fail(ACF_ERR_ARGUMENT, "source %lld cell %lld outside the grid", (long long)q, (long long)cell[q]);
        if (length[q] < 0 || length[q] > stride)
            return fail(ACF_ERR_ARGUMENT, "source %lld length %lld exceeds stride %lld", (long long)q,
                        (long long)length[q], (long long)stride);
        off[q] = padded_offset(h, cell[q]);
        len[q] = length[q];
    }
    ACF_CUDA(cudaDeviceSynchronize());
    cudaFree(h->src_off);
    cudaFree(h->src_len);
    cudaFree(h->src_sig);
    h->src_off = h->src_len = nullptr;
    h->src_sig = nullptr;
    h->n_src = 0;
    h->graph_dirty = true;
    if (n == 0) return ACF_OK;
    const size_t es = h->elem();
    const size_t n_sig = (size_t)n * (size_t)std::max<int64_t>(stride, 1);
    ACF_CUDA(cudaMalloc(&h->src_off, n * sizeof(int64_t)));
    ACF_CUDA(cudaMalloc(&h->src_len, n * sizeof(int64_t)));
    ACF_CUDA(cudaMalloc(&h->src_sig, n_sig * es));
    ACF_CUDA(cudaMemcpy(h->src_off, off.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    ACF_CUDA(cudaMemcpy(h->src_len, len.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    std::vector<char> cast(n_sig * es, 0);
    if (stride > 0) {
        if (es == 4) cast_copy<float>(cast.data(), signal, (size_t)n * stride);
        else cast_copy<double>(cast.data(), signal, (size_t)n * stride);
    }
    ACF_CUDA(cudaMemcpy(h->src_sig, cast.data(), cast.size(), cudaMemcpyHostToDevice));
    h->n_src = n;
    h->src_stride = stride;
    return ACF_OK;
}

int acf_set_receivers(acf_solver *h, int64_t n, const int64_t *cell, const int64_t *start_step) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (n < 0 || n > (1 << 20)) return fail(ACF_ERR_ARGUMENT, "receiver count %lld out of range", (long long)n);
    if (n > 0 && (!cell || !start_step)) return fail(ACF_ERR_ARGUMENT, "null receiver arrays");
    DeviceGuard guard(h->device);
    const int64_t n_cells = (int64_t)h->nx * h->ny * h->nz;
    std::vector<int64_t> off((size_t)n);
    for (int64_t r = 0; r < n; r++) {
        if (cell[r] < 0 || cell[r] >= n_cells)
            return fail(ACF_ERR_ARGUMENT, "receiver %lld cell %lld outside the grid", (long long)r, (long long)cell[r]);
        if (start_step[r] < 0) return fail(ACF_ERR_ARGUMENT, "negative start step");
        off[r] = padded_offset(h, cell[r]);
    }
    ACF_CUDA(cudaDeviceSynchronize());
    if (n > 0 && !h->rec_origin_set) {
        h->rec_origin = *std::min_element(start_step, start_step + n);
        h->rec_origin_set = true;
    }
    for (int64_t r = 0; r < n; r++)
        if (start_step[r] < h->rec_origin)
            return fail(ACF_ERR_ARGUMENT, "receiver %lld starts before the recording origin", (long long)r);
    // Keep existing recordings: grow the row count, preserving rows already written.
    const size_t es = h->elem();
    if (n > 0 && h->rec_capacity > 0 && n != h->n_rec) {
        void *grown = nullptr;
        ACF_CUDA(cudaMalloc(&grown, (size_t)n * h->rec_capacity * es));
        ACF_CUDA(cudaMemset(grown, 0, (size_t)n * h->rec_capacity * es));
        const int64_t keep = std::min<int64_t>(n, h->n_rec);
        if (keep > 0 && h->rec)
            ACF_CUDA(cudaMemcpy(grown, h->rec, (size_t)keep * h->rec_capacity * es, cudaMemcpyDeviceToDevice));
        cudaFree(h->rec);
        h->rec = grown;
    }
    cudaFree(h->rec_off);
    cudaFree(h->rec_start);
    h->rec_off = h->rec_start = nullptr;
    h->n_rec = 0;
    h->graph_dirty = true;
    h->host_rec_cell.assign(cell, cell + n);
    h->host_rec_start.assign(start_step, start_step + n);
    if (n == 0) return ACF_OK;
    ACF_CUDA(cudaMalloc(&h->rec_off, n * sizeof(int64_t)));
    ACF_CUDA(cudaMalloc(&h->rec_start, n * sizeof(int64_t)));
    ACF_CUDA(cudaMemcpy(h->rec_off, off.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    ACF_CUDA(cudaMemcpy(h->rec_start, start_step, n * sizeof(int64_t), cudaMemcpyHostToDevice));
    h->n_rec = n;
    return ACF_OK;
}

int acf_read_recording(acf_solver *h, int64_t r, int64_t first_step, int64_t n, void *dst,
                       acf_stream stream) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (r < 0 || r >= h->n_rec) return fail(ACF_ERR_ARGUMENT, "receiver %lld out of range", (long long)r);
    if (n < 0 || (n > 0 && !dst)) return fail(ACF_ERR_ARGUMENT, "bad destination");
    if (n == 0) return ACF_OK;
    const int64_t col = first_step - h->rec_origin;
    if (col < 0 || col + n > h->rec_capacity || first_step < h->host_rec_start[(size_t)r])
        return fail(ACF_ERR_ARGUMENT, "steps [%lld, %lld) were not recorded by receiver %lld",
                    (long long)first_step, (long long)(first_step + n), (long long)r);
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t es = h->elem();
    ACF_CUDA(cudaMemcpyAsync(dst, (char *)h->rec + ((size_t)r * h->rec_capacity + col) * es, (size_t)n * es,
                             cudaMemcpyDeviceToHost, st));
    ACF_CUDA(cudaStreamSynchronize(st));
    return ACF_OK;
}

int acf_upload(acf_solver *h, int field, const void *src, acf_stream stream) {
    int rc = check_field(h, field);
    if (rc) return rc;
    if (!src) return fail(ACF_ERR_ARGUMENT, "null source");
    DeviceGuard guard(h->device);
    return copy_field(h, field, const_cast<void *>(src), true, (cudaStream_t)stream);
}

int acf_download(acf_solver *h, int field, void *dst, acf_stream stream) {
    int rc = check_field(h, field);
    if (rc) return rc;
    if (!dst) return fail(ACF_ERR_ARGUMENT, "null destination");
    DeviceGuard guard(h->device);
    return copy_field(h, field, dst, false, (cudaStream_t)stream);
}

int acf_run(acf_solver *h, int64_t n_steps, int64_t step_offset, acf_stream stream) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (n_steps < 0 || step_offset < 0) return fail(ACF_ERR_ARGUMENT, "negative step count or offset");
    if (n_steps == 0) return ACF_OK;
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    // Recording capacity for every step this run can write.
    if (h->n_rec > 0) {
        const int64_t need = step_offset + n_steps - h->rec_origin;
        if (need > h->rec_capacity) {
            int64_t cap = std::max<int64_t>(need, 2 * h->rec_capacity);
            cap = round_up(cap, 256);
            const size_t es = h->elem();
            void *grown = nullptr;
            ACF_CUDA(cudaStreamSynchronize(st));
            ACF_CUDA(cudaMalloc(&grown, (size_t)h->n_rec * cap * es));
            ACF_CUDA(cudaMemset(grown, 0, (size_t)h->n_rec * cap * es));
            if (h->rec && h->rec_capacity > 0)
                ACF_CUDA(cudaMemcpy2D(grown, (size_t)cap * es, h->rec, (size_t)h->rec_capacity * es,
                                      (size_t)h->rec_capacity * es, (size_t)h->n_rec, cudaMemcpyDeviceToDevice));
            cudaFree(h->rec);
            h->rec = grown;
            h->rec_capacity = cap;
            h->graph_dirty = true;
        }
    }
    return h->precision == 8 ? run_impl<double>(h, n_steps, step_offset, st)
                             : run_impl<float>(h, n_steps, step_offset, st);
}

int acf_set_graph(acf_solver *h, int32_t steps) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    if (steps < 0 || steps > 4096) return fail(ACF_ERR_ARGUMENT, "steps_per_graph %d out of range", steps);
    if (steps != h->graph_steps) h->graph_dirty = true;
    h->graph_steps = steps;
    return ACF_OK;
}

int acf_energy_terms(acf_solver *h, double dx, double terms[7], acf_stream stream) {
    if (!h || !terms) return fail(ACF_ERR_ARGUMENT, "null argument");
    if (!(dx > 0)) return fail(ACF_ERR_ARGUMENT, "dx must be positive");
    DeviceGuard guard(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    return h->precision == 8 ? energy_impl<double>(h, dx, terms, st) : energy_impl<float>(h, dx, terms, st);
}

int acf_field_pointer(acf_solver *h, int field, void **ptr, int64_t strides[3]) {
    int rc = check_field(h, field);
    if (rc) return rc;
    if (!ptr || !strides) return fail(ACF_ERR_ARGUMENT, "null output");
    *ptr = h->field_ptr(field);
    strides[0] = h->plane;
    strides[1] = h->pz;
    strides[2] = 1;
    return ACF_OK;
}

int acf_profile_enable(acf_solver *h, int32_t enable) {
    if (!h) return fail(ACF_ERR_ARGUMENT, "null solver");
    h->profiling = enable != 0;
    h->prof_velocity_ms = h->prof_pressure_ms = 0;
    h->prof_launches = 0;
    return ACF_OK;
}

int acf_profile_read(acf_solver *h, double *velocity_ms, double *pressure_ms, int64_t *launches) {
    if (!h || !velocity_ms || !pressure_ms || !launches) return fail(ACF_ERR_ARGUMENT, "null argument");
    *velocity_ms = h->prof_velocity_ms;
    *pressure_ms = h->prof_pressure_ms;
    *launches = h->prof_launches;
    return ACF_OK;
}

int64_t acf_launch_count(const acf_solver *h) { return h ? h->launches : -1; }

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
