// Shared device helpers for libsimb200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/simb200.h"

#define SIM_THREADS 256

namespace simb200 {

// ---- error plumbing --------------------------------------------------------
void set_cuda_error(cudaError_t err, const char* where);
void set_error_text(const char* msg);        // message returned by sim_last_cuda_error()
int  launch_status(const char* where);   // checks cudaGetLastError after a launch
void prepare_capture_stream();           // side stream used to capture IF-node bodies
typedef int (*BodyFn)(const void* ctx, cudaStream_t s);
int  launch_if_flag(cudaStream_t st, const int32_t* flag, BodyFn body, BodyFn eager, const void* ctx,
                    const char* what);       // IF node on *flag while capturing, else eager()
// cond(ctx, s, h) launches work that sets the IF node's value through *h
// (cudaGraphSetConditional), or the same work without it when h is null
typedef int (*CondFn)(const void* ctx, cudaStream_t s, const cudaGraphConditionalHandle* h);
int  launch_if_cond(cudaStream_t st, CondFn cond, BodyFn body, BodyFn eager, const void* ctx, const char* what);
// the engine's rebuild as an IF-node body (ungated) and eagerly (gated on flags[0]); ctx is the SimEngine
int  rebuild_body(const void* ctx, cudaStream_t s);
int  rebuild_eager(const void* ctx, cudaStream_t s);
// Persistent grid: resident blocks per SM (cached occupancy query) x SM count,
// capped by the number of atom tiles.
int persistent_grid(const void* fn, int threads, size_t smem, int64_t n);
// neighbour tiles (tiles.cu)
void launch_build_halo(const SimEngine& e, const int32_t* gate, cudaStream_t st);
bool tiled_eam_usable(const SimEngine& e, const SimEAMTables& t);
int launch_eam_density_tiled(const SimEngine& e, const SimEAMTables& t, cudaStream_t st);
int launch_eam_force_tiled(const SimEngine& e, const SimEAMTables& t, const SimIntegrator* ip, cudaStream_t st);

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// This block's share of [0, n) for the persistent per-atom passes: one
// contiguous range per block, the ranges equal to within a warp's 32 slots
// (ceil(n / blocks) rounded up to whole warps).  Against a grid-stride walk
// of blockDim-sized tiles, every SM gets the same work (a tile left over for
// some blocks held their SMs for a whole extra tile) and consecutive
// iterations of a block gather from overlapping neighbourhoods.
struct BlockRange {
    int64_t begin, end;
};
__device__ __forceinline__ BlockRange block_range(int64_t n) {
    const int64_t c = ((n + gridDim.x - 1) / gridDim.x + 31) / 32 * 32;
    const int64_t b = (int64_t)blockIdx.x * c;
    return BlockRange{b < n ? b : n, b + c < n ? b + c : n};
}

// Loads of data read once per pass (neighbour-list rows, in-cutoff masks):
// evict-first in L1 and L2, so the caches keep the gathered neighbour
// positions instead.
#ifndef SIM_STREAM_HINT
#define SIM_STREAM_HINT 1
#endif
template <class T>
__device__ __forceinline__ T ld_stream(const T* p) {
#if SIM_STREAM_HINT
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}

// The FP64 positions and velocities and the skin references are touched
// once per step by the integrator: streaming loads and stores as well.
#ifndef SIM_STATE_HINT
#define SIM_STATE_HINT 1
#endif
__device__ __forceinline__ double ld_state(const double* p) {
#if SIM_STATE_HINT
    return __ldcs(p);
#else
    return *p;
#endif
}
__device__ __forceinline__ int32_t ld_state(const int32_t* p) {
#if SIM_STATE_HINT
    return __ldcs(p);
#else
    return *p;
#endif
}
__device__ __forceinline__ void st_state(double* p, double v) {
#if SIM_STATE_HINT
    __stcs(p, v);
#else
    *p = v;
#endif
}

// Programmatic dependent launch (sm_90 and later).  A kernel launched by
// launch_pdl may be scheduled while its predecessor in the stream (or graph)
// is still finishing: pdl_wait() returns once the predecessor has completed
// and its writes are visible (at once when there is no programmatic
// dependency), so everything before it may only read data the predecessor
// does not write; pdl_trigger() lets the successor be scheduled from now on.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Mean duration in ms of reps calls of launch() on stream st, after one
// untimed call (CUDA events on st; synchronises); negative on a CUDA error.
template <class F>
inline float time_launches(F launch, int reps, cudaStream_t st) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return -1.0f;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -1.0f; }
    launch();
    cudaEventRecord(a, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(b, st);
    float ms = -1.0f;
    if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) ms /= (float)reps;
    else ms = -1.0f;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

// ---- fixed-point fractional coordinates -----------------------------------
// u = frac(s) * 2^32 stored as uint32; the difference of two codes read as
// int32 is the minimum-image fractional displacement in [-1/2, 1/2).
__device__ __forceinline__ uint32_t to_fixed(double s) {
    return (uint32_t)(unsigned long long)__double2ll_rn(s * 4294967296.0);
}
__device__ __forceinline__ float fixed_delta(int32_t a, int32_t b) {
    return __int2float_rn((int32_t)((uint32_t)a - (uint32_t)b)) * 2.3283064365386963e-10f;
}

// fractional coordinate of a Cartesian row vector x: s_k = sum_r x_r Hinv[r][k]
__device__ __forceinline__ void cart_to_frac(const SimBox& b, double x0, double x1, double x2,
                                             double* s) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
        s[k] = fma(x2, b.Hinv[6 + k], fma(x1, b.Hinv[3 + k], x0 * b.Hinv[k]));
}

// Cartesian displacement (FP32) of a fractional displacement t: r = t H
__device__ __forceinline__ void frac_to_cart_f(const SimBox& b, float t0, float t1, float t2,
                                               float& r0, float& r1, float& r2) {
    if (b.orthogonal) {
        r0 = t0 * b.Hf[0];
        r1 = t1 * b.Hf[4];
        r2 = t2 * b.Hf[8];
    } else {
        r0 = fmaf(t2, b.Hf[6], fmaf(t1, b.Hf[3], t0 * b.Hf[0]));
        r1 = fmaf(t2, b.Hf[7], fmaf(t1, b.Hf[4], t0 * b.Hf[1]));
        r2 = fmaf(t2, b.Hf[8], fmaf(t1, b.Hf[5], t0 * b.Hf[2]));
    }
}

// Minimum-image Cartesian displacement x_i - x_j (FP32) of two fixed-point positions.
__device__ __forceinline__ void pair_vector(const SimBox& b, const int4& qi, const int4& qj,
                                            float& r0, float& r1, float& r2) {
    frac_to_cart_f(b, fixed_delta(qi.x, qj.x), fixed_delta(qi.y, qj.y), fixed_delta(qi.z, qj.z), r0, r1, r2);
}

// Minimum image in FP64 following core/box.py:109-130 with torch's CPU op order
// (orthogonal: r - d*rint(r/d); triclinic: fma-chained row-vector products).
__device__ __forceinline__ void min_image_f64(const SimBox& b, double& r0, double& r1, double& r2) {
    if (b.orthogonal) {
        double d0 = b.H[0], d1 = b.H[4], d2 = b.H[8];
        r0 = __dsub_rn(r0, __dmul_rn(d0, rint(__ddiv_rn(r0, d0))));
        r1 = __dsub_rn(r1, __dmul_rn(d1, rint(__ddiv_rn(r1, d1))));
        r2 = __dsub_rn(r2, __dmul_rn(d2, rint(__ddiv_rn(r2, d2))));
    } else {
        double s[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            s[k] = __fma_rn(r2, b.Hinv[6 + k], __fma_rn(r1, b.Hinv[3 + k], __dmul_rn(r0, b.Hinv[k])));
#pragma unroll
        for (int k = 0; k < 3; ++k) s[k] = __dsub_rn(s[k], rint(s[k]));
        r0 = __fma_rn(s[2], b.H[6], __fma_rn(s[1], b.H[3], __dmul_rn(s[0], b.H[0])));
        r1 = __fma_rn(s[2], b.H[7], __fma_rn(s[1], b.H[4], __dmul_rn(s[0], b.H[1])));
        r2 = __fma_rn(s[2], b.H[8], __fma_rn(s[1], b.H[5], __dmul_rn(s[0], b.H[2])));
    }
}

__device__ __forceinline__ double norm2_f64(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// ---- reductions -------------------------------------------------------------
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce `vals[0..NV)` (FP64) and store one row of `partials` per block.
// Deterministic: fixed shuffle tree, fixed warp order.
template <int NV>
__device__ __forceinline__ void block_partials(double (&vals)[NV], double* partials, int slot0,
                                               int stride = SIM_RED_SLOTS) {
    __shared__ double red[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = warp_sum(vals[k]);
        if (lane == 0) red[k][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        partials[(size_t)blockIdx.x * stride + slot0 + threadIdx.x] = s;
    }
}

// The sums over the grid's blocks of partial slots [slot0, slot0+NV) (rows of
// `stride` doubles) into out[out0 + k], by the calling block: warp k sums
// slot k, lane l adding rows l, l+32, ... with Kahan compensation, then the
// 32 compensated sums combine in a fixed tree (TwoSum of the sums, the
// compensations added): the order depends only on the grid size.
template <int NV>
__device__ __forceinline__ void partial_sums(const double* partials, int slot0, int stride, double* out, int out0,
                                             bool accumulate = false) {
    const int lane = threadIdx.x & 31, nw = (int)(blockDim.x >> 5);
    for (int k = (int)(threadIdx.x >> 5); k < NV; k += nw) {
        double s = 0.0, c = 0.0;   // value s - c
        for (unsigned b = lane; b < gridDim.x; b += 32) {
            const double y = __ldcg(&partials[(size_t)b * stride + slot0 + k]) - c;
            const double t = s + y;
            c = (t - s) - y;
            s = t;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double s2 = __shfl_down_sync(0xffffffffu, s, o);
            const double c2 = __shfl_down_sync(0xffffffffu, c, o);
            const double t = s + s2, bp = t - s;
            const double err = (s - (t - bp)) + (s2 - bp);   // s + s2 = t + err exactly
            c = c + c2 - err;
            s = t;
        }
        if (lane == 0) out[out0 + k] = accumulate ? out[out0 + k] + (s - c) : s - c;
    }
}

// The last block to finish sums all partial rows for slots [slot0, slot0+NV)
// and resets the counter (so a captured graph can replay).  Warp k sums slot
// k: lane l adds rows l, l+32, ... with Kahan compensation, then the 32
// compensated sums combine in a fixed tree (TwoSum of the sums, the
// compensations added): the order depends only on the grid size.  Must be
// called by every thread of every block (blockDim.x a multiple of 32).  With
// `accumulate` the sums are added to what `out` holds (a further force field
// of a sum of force fields) instead of replacing it.
template <int NV>
__device__ __forceinline__ bool last_block_finalize(double* partials, uint32_t* counter,
                                                    double* out, int slot0, int stride = SIM_RED_SLOTS,
                                                    bool accumulate = false) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t done = atomicAdd(counter, 1u);
        is_last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    partial_sums<NV>(partials, slot0, stride, out, slot0, accumulate);
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// ---- Philox4x32-10 (Salmon et al., SC'11) ------------------------------------
struct U4 { uint32_t x, y, z, w; };
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Three standard normals for atom `a` at `step` (float32 Box-Muller).
__device__ __forceinline__ void langevin_normals(uint32_t a, uint64_t step, uint64_t seed,
                                                 float& z0, float& z1, float& z2) {
    U4 c{a, (uint32_t)step, (uint32_t)(step >> 32), 0u};
    U4 x = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const float sc = 2.3283064365386963e-10f;
    float u0 = __fmul_rn(__fadd_rn(__uint2float_rn(x.x), 0.5f), sc);
    float u1 = __fmul_rn(__fadd_rn(__uint2float_rn(x.y), 0.5f), sc);
    float u2 = __fmul_rn(__fadd_rn(__uint2float_rn(x.z), 0.5f), sc);
    float u3 = __fmul_rn(__fadd_rn(__uint2float_rn(x.w), 0.5f), sc);
    float r0 = sqrtf(__fmul_rn(-2.0f, logf(u0)));
    float r1 = sqrtf(__fmul_rn(-2.0f, logf(u2)));
    float s0, c0, s1, c1;
    sincospif(__fmul_rn(2.0f, u1), &s0, &c0);
    sincospif(__fmul_rn(2.0f, u3), &s1, &c1);
    z0 = __fmul_rn(r0, c0);
    z1 = __fmul_rn(r0, s0);
    z2 = __fmul_rn(r1, c1);
}

// Second half of velocity Verlet for slot i (integrator.py:102-124):
//   v = v_half * damp + xi * rff   (Langevin, noise by original index and step)
//   v = v + (0.5 * F/m) * dt
// Writes e.v and returns the new velocity in v_out.
__device__ __forceinline__ void second_half_atom(const SimEngine& e, const SimIntegrator& p, int64_t i, int type,
                                                 uint64_t step, double f0, double f1, double f2, double* v_out,
                                                 bool& bad, bool store = true, double* a_out = nullptr) {
    const int64_t P = e.n_pad;
    const double inv_m = e.inv_mass[type];
    double z[3] = {0.0, 0.0, 0.0};
    double rff = 0.0;
    if (p.langevin) {
        float z0, z1, z2;
        langevin_normals((uint32_t)e.orig[i], step, p.seed, z0, z1, z2);
        z[0] = z0; z[1] = z1; z[2] = z2;
        rff = p.rff[type];
    }
    const double f[3] = {f0, f1, f2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double vel = ld_state(&e.v[c * P + i]);
        if (p.langevin) vel = __dadd_rn(__dmul_rn(vel, p.damp), __dmul_rn(z[c], rff));
        const double a = __dmul_rn(f[c], inv_m);   // F (1/m): within 1 ulp of F/m, without a divide
        if (a_out) a_out[c] = a;
        vel = __dadd_rn(vel, __dmul_rn(__dmul_rn(0.5, a), p.dt));
        if (store) st_state(&e.v[c * P + i], vel);
        v_out[c] = vel;
        bad |= !isfinite(vel);
    }
}

// First half of velocity Verlet for atom i (integrator.py:91-99): v += F/m dt/2,
// x += v dt, refresh the fixed-point code in posq, and report whether the atom
// moved more than skin/2 from its position at the last rebuild
// (reader.py:136-163).  v_in / x_in: the velocity to kick and the position to
// drift (read from e.v / e.x when NULL); a_in: the acceleration when the
// caller already formed it (second_half_atom's a_out for the same forces).
// Both half-steps form F/m as F times the stored 1/m, which is within one
// ulp of the reference's quotient and spares an FP64 divide per component.
__device__ __forceinline__ bool place_atom(const SimEngine& e, const SimBox& b, int64_t i, int type, const double* xn,
                                           int32_t* q_out = nullptr, bool diag = false);

// H and H^-1 with off-diagonal entries exactly zero: place_atom may then skip
// the off-diagonal products (adding exact zeros changes no rounded value).
__device__ __forceinline__ bool box_is_diagonal(const SimBox& b) {
    bool z = true;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        if (k % 4 != 0) z = z && b.H[k] == 0.0 && b.Hinv[k] == 0.0;
    return z;
}

__device__ __forceinline__ bool first_half_atom(const SimEngine& e, const SimBox& b, const SimIntegrator& p, int64_t i,
                                                int type, const double* f, const double* v_in, bool& bad,
                                                const double* x_in = nullptr, int32_t* q_out = nullptr,
                                                const double* a_in = nullptr, bool diag = false) {
    const int64_t P = e.n_pad;
    const double inv_m = e.inv_mass[type];
    double xn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double a = a_in ? a_in[c] : __dmul_rn(f[c], inv_m);
        const double v0 = v_in ? v_in[c] : ld_state(&e.v[c * P + i]);
        const double vh = __dadd_rn(v0, __dmul_rn(__dmul_rn(0.5, a), p.dt));
        xn[c] = __dadd_rn(x_in ? x_in[c] : ld_state(&e.x[c * P + i]), __dmul_rn(vh, p.dt));
        st_state(&e.v[c * P + i], vh);
        bad |= !isfinite(xn[c]) || !isfinite(vh);
    }
    return place_atom(e, b, i, type, xn, q_out, diag);
}

__device__ __forceinline__ bool first_half_atom(const SimEngine& e, const SimIntegrator& p, int64_t i, int type,
                                                const double* f, const double* v_in, bool& bad) {
    return first_half_atom(e, *e.box, p, i, type, f, v_in, bad);
}

// Store position xn of slot i, refresh its fixed-point code in posq (in
// q_out instead when given: a pass that still gathers posq must not see it
// change), and report whether it is more than skin/2 from its position at the
// last rebuild (reader.py:136-163).
__device__ __forceinline__ bool place_atom(const SimEngine& e, const SimBox& b, int64_t i, int type, const double* xn,
                                           int32_t* q_out, bool diag) {
    const int64_t P = e.n_pad;
#pragma unroll
    for (int c = 0; c < 3; ++c) st_state(&e.x[c * P + i], xn[c]);
    double s[3];
    if (diag) {
#pragma unroll
        for (int k = 0; k < 3; ++k) s[k] = xn[k] * b.Hinv[4 * k];
    } else {
        cart_to_frac(b, xn[0], xn[1], xn[2], s);
    }
    int4 q;
    q.x = (int32_t)to_fixed(s[0]);
    q.y = (int32_t)to_fixed(s[1]);
    q.z = (int32_t)to_fixed(s[2]);
    q.w = type;
    reinterpret_cast<int4*>(q_out ? q_out : e.posq)[i] = q;
    // displacement since the last rebuild, minimum image in fractional space
    const double t0 = (double)(int32_t)((uint32_t)q.x - (uint32_t)ld_state(&e.xref[i])) * 2.3283064365386963e-10;
    const double t1 = (double)(int32_t)((uint32_t)q.y - (uint32_t)ld_state(&e.xref[P + i])) * 2.3283064365386963e-10;
    const double t2 = (double)(int32_t)((uint32_t)q.z - (uint32_t)ld_state(&e.xref[2 * P + i])) * 2.3283064365386963e-10;
    if (diag) {
        const double d0 = t0 * b.H[0], d1 = t1 * b.H[4], d2 = t2 * b.H[8];
        return d0 * d0 + d1 * d1 + d2 * d2 > e.skin_half2;
    }
    const double d0 = t0 * b.H[0] + t1 * b.H[3] + t2 * b.H[6];
    const double d1 = t0 * b.H[1] + t1 * b.H[4] + t2 * b.H[7];
    const double d2 = t0 * b.H[2] + t1 * b.H[5] + t2 * b.H[8];
    return d0 * d0 + d1 * d1 + d2 * d2 > e.skin_half2;
}

}  // namespace simb200
