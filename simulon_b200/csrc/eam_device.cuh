// EAM device helpers shared by the single-system and the batched kernels:
// fixed-point displacement -> Cartesian vector, table interpolation
// (eam_force_cu.py:437-459), the pass-1 density term and the pass-2 pair
// force with its energy and virial accumulation.
#pragma once
#include "common.cuh"

namespace simb200 {

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// _interp_rho for F and F' of type ti; the grid's lower end, clamp and
// inverse spacing may come from the caller (read once per thread)
__device__ __forceinline__ void embed_lookup(const SimEAMTables& t, int ti, float rho, float& F, float& Fp,
                                             const float* grid = nullptr) {
    const float lo = grid ? grid[0] : t.rho_min[ti];
    const float rc = fminf(fmaxf(rho, lo), grid ? grid[1] : t.rho_clamp_hi[ti]);
    const float idx_f = (rc - lo) * (grid ? grid[2] : t.inv_drho[ti]);
    const int i = (int)idx_f;
    const int i1 = min(i + 1, t.n_rho - 1);
    const float frac = idx_f - (float)i;
    const float* e = t.embed + (size_t)ti * t.n_rho;
    const float* d = t.embed_deriv + (size_t)ti * t.n_rho;
    F = fmaf(frac, e[i1] - e[i], e[i]);
    Fp = fmaf(frac, d[i1] - d[i], d[i]);
}

// Box terms in registers, with the 2^-32 of the fixed-point code folded in.
struct BoxF {
    float h[9];
    __device__ __forceinline__ explicit BoxF(const SimBox& b) {
#pragma unroll
        for (int k = 0; k < 9; ++k) h[k] = b.Hf[k] * 2.3283064365386963e-10f;
    }
};
template <bool ORTHO>
__device__ __forceinline__ void rvec(const BoxF& b, const int4& qi, const int4& qj, float& r0, float& r1, float& r2) {
    const float t0 = __int2float_rn((int32_t)((uint32_t)qi.x - (uint32_t)qj.x));
    const float t1 = __int2float_rn((int32_t)((uint32_t)qi.y - (uint32_t)qj.y));
    const float t2 = __int2float_rn((int32_t)((uint32_t)qi.z - (uint32_t)qj.z));
    if (ORTHO) {
        r0 = t0 * b.h[0];
        r1 = t1 * b.h[4];
        r2 = t2 * b.h[8];
    } else {
        r0 = fmaf(t2, b.h[6], fmaf(t1, b.h[3], t0 * b.h[0]));
        r1 = fmaf(t2, b.h[7], fmaf(t1, b.h[4], t0 * b.h[1]));
        r2 = fmaf(t2, b.h[8], fmaf(t1, b.h[5], t0 * b.h[2]));
    }
}

// r inside the cutoff -> table row and fraction (_interp_r)
struct Lerp {
    int k;
    float frac;
};
// Tables hold fewer rows than this (checked by every entry point that takes
// SimEAMTables), so lerp_r's truncation below is exact.
constexpr int kMaxTableRows = 1 << 22;

// trunc(idx_f) without the conversion unit: for 0 <= idx_f < 2^23 the sum
// 2^23 + idx_f rounded toward zero is 2^23 + trunc(idx_f), held in the low
// mantissa bits, and subtracting 2^23 back is exact -- the same k and fraction
// as (int)idx_f and idx_f - (float)k (tables have fewer than 2^22 rows).
__device__ __forceinline__ Lerp lerp_r(float r, const SimEAMTables& t) {
    const float idx_f = fminf(r, t.r_clamp_hi) * t.inv_dr;
    const float s = __fadd_rz(idx_f, 8388608.0f);
    return Lerp{__float_as_int(s) - 0x4B000000, idx_f - (s - 8388608.0f)};
}

// ---------------------------------------------------------------------------
// pass 1
// Shared-memory window of the r-tables: rows k in [k_lo, n_r) (r >= k_lo dr);
// the rare shorter distances read the global table.
struct Window {
    int k_lo, n_win;
};

// ONE: a single element type (type 0 throughout), so the table row needs no
// type index.
template <bool SMEM, bool ORTHO, bool ONE = false>
__device__ __forceinline__ float density_term(const BoxF& b, const int4& qi, const int4& qj, float rc2,
                                              const float2* g_i, const float2* s_i, Window w,
                                              const SimEAMTables& t, bool& inside) {
    float r0, r1, r2;
    rvec<ORTHO>(b, qi, qj, r0, r1, r2);
    const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
    inside = d2 < rc2;
    if (!inside) return 0.0f;
    const Lerp l = lerp_r(d2 * rsqrt_approx(d2), t);
    const int tj = ONE ? 0 : qj.w;
    float2 v;
    if (SMEM && l.k >= w.k_lo) v = s_i[tj * w.n_win + (l.k - w.k_lo)];
    else v = __ldg(&g_i[(size_t)tj * t.n_r + l.k]);
    return fmaf(l.frac, v.y, v.x);
}

// A row's in-cutoff slots (bit k: slot k) as two 32-bit words, since slots of
// 32 and above are rare; pop() returns the lowest one left and clears it, or
// -1 when none is left (the slots come out in increasing order).
struct SlotMask {
    uint32_t lo, hi;
    __device__ __forceinline__ explicit SlotMask(uint64_t m) : lo((uint32_t)m), hi((uint32_t)(m >> 32)) {}
    __device__ __forceinline__ int pop() {
        if (lo) {
            const int k = __ffs((int)lo) - 1;
            lo &= lo - 1;
            return k;
        }
        if (hi) {
            const int k = __ffs((int)hi) + 31;
            hi &= hi - 1;
            return k;
        }
        return -1;
    }
};

// The same slots in the same order, the leading run of set bits (slots 0 ..
// p-1, usually most of the in-cutoff set since rows are sorted by distance at
// rebuild) taken by counting instead of bit scans.
struct SlotSeq {
    SlotMask m;
    int k, p;
    __device__ __forceinline__ explicit SlotSeq(uint64_t bits) : m(bits), k(0) {
        p = m.lo == 0xFFFFFFFFu ? 32 : __ffs((int)~m.lo) - 1;
        m.lo &= m.lo + 1u;     // clears the leading run (all of lo when p = 32)
    }
    __device__ __forceinline__ int next() { return k < p ? k++ : m.pop(); }
};

// ---------------------------------------------------------------------------
// pass 2.  Per-thread accumulators: acc[0] pair energy, acc[1] scalar virial,
// acc[2..7] virial tensor (xx yy zz xy xz yz), acc[8] K, acc[9..14] K tensor;
// only the three force components are per atom.  The scalar virial sum s r is
// minus the tensor's trace (f = -s r/|r|, so f.r = -s |r|): it is not summed
// per pair but set from the thread's trace before the reduction (virial_trace).
__device__ __forceinline__ void virial_trace(float (&acc)[15]) { acc[1] = -(acc[2] + acc[3] + acc[4]); }

__device__ __forceinline__ void pair_force(float s, float phi, float r, float inv_r, float r0, float r1, float r2,
                                           float& fx, float& fy, float& fz, float (&acc)[15]) {
    const float c = -s * inv_r;            // force on i = c * r_ij
    const float ax = c * r0, ay = c * r1, az = c * r2;
    fx += ax; fy += ay; fz += az;
    acc[0] += phi;
    acc[2] = fmaf(ax, r0, acc[2]); acc[3] = fmaf(ay, r1, acc[3]); acc[4] = fmaf(az, r2, acc[4]);
    acc[5] = fmaf(ax, r1, acc[5]); acc[6] = fmaf(ax, r2, acc[6]); acc[7] = fmaf(ay, r2, acc[7]);
}

// One element type: f'_{ti,tj} = f'_{tj,ti}; tables {f', phi', df', dphi'} and
// {phi, dphi} staged in shared memory.
template <bool ORTHO>
__device__ __forceinline__ void pair_single(const BoxF& b, const int4& pi, const int4& qj, float rc2, float fpi,
                                            const float4* tab_d, const float2* tab_p, Window w,
                                            const SimEAMTables& t, float& fx, float& fy, float& fz,
                                            float (&acc)[15]) {
    float r0, r1, r2;
    rvec<ORTHO>(b, pi, qj, r0, r1, r2);
    const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
    if (!(d2 < rc2)) return;
    const float inv_r = rsqrt_approx(d2);
    const float r = d2 * inv_r;
    const Lerp l = lerp_r(r, t);
    float4 d;
    float2 p;
    if (l.k >= w.k_lo) {
        d = tab_d[l.k - w.k_lo];
        p = tab_p[l.k - w.k_lo];
    } else {
        d = __ldg(reinterpret_cast<const float4*>(t.deriv_vd) + l.k);
        p = __ldg(reinterpret_cast<const float2*>(t.pair_vd) + l.k);
    }
    const float2 dd_dp = __ffma2_rn(make_float2(l.frac, l.frac), make_float2(d.z, d.w), make_float2(d.x, d.y));
    const float phi = fmaf(l.frac, p.y, p.x);
    pair_force(fmaf(fpi + __int_as_float(qj.w), dd_dp.x, dd_dp.y), phi, r, inv_r, r0, r1, r2, fx, fy, fz, acc);
}

}  // namespace simb200
