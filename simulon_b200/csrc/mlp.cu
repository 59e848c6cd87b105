// Descriptor-MLP surrogate of the EAM force field (sm_100a).  No counterpart
// in the reference: it is the learned form of the force path, trained on
// the engine's own EAM energies and judged against EAM during a run.
//
// Per atom i, over the in-cutoff entries of the engine's list (r < 4.4 A),
// with d_j = x_j - x_i and the cosine cutoff fc(r) = (cos(pi r/rc) + 1)/2:
//   radial  G_k  = sum_j exp(-4 (r_j - R_k)^2) fc(r_j),  R_k = 2.0 + 2.4 k/7, k < 8
//   angular G_zl = 2^(1-z) sum_{a<b} (1 + l cos t_ab)^z e(r_a) e(r_b),
//            e(r) = exp(-0.01 r^2) fc(r),  z in {1,2,4,8}, l = +1, -1
// The network 16 -> 64 -> 64 -> 1 (SiLU) maps the normalised descriptors to
// the atom's energy; forces are -dE/dx through the network and descriptors.
//
// Network kernel: 128 atoms per tile, one thread per atom; the four GEMMs of
// the forward and backward passes (Z1 = G W1, Z2 = H1 W2, D1 = dZ2 W2^T,
// dG = dZ1 W1^T) run on the 5th-generation tensor cores: BF16 operands in
// shared memory in the canonical no-swizzle K-major layout (8x8 core
// matrices), FP32 accumulators in tensor memory, tcgen05.mma issued by one
// thread and completed through an mbarrier; the SiLU epilogues read the
// accumulators with tcgen05.ld.  Every wait on the mbarrier is bounded: a
// timeout sets SIM_STATUS_MLP_TIMEOUT in the status word, frees the tensor
// memory and returns.
#include <cstdio>
#include "common.cuh"
#include "eam_device.cuh"
#include <cuda_bf16.h>

namespace simb200 {

#define MLP_RC 4.4f
#define MLP_MAXN 32          // in-cutoff neighbours kept per atom (more sets SIM_STATUS_MLP_NEIGHBORS)
#define MLP_TILE 128
#define MLP_H 64
#define MLP_D 16
#define MLP_WAIT_LIMIT (1 << 24)
#define GRAD_W1 SIM_MLP_OFF_W1
#define GRAD_B1 SIM_MLP_OFF_B1
#define GRAD_W2 SIM_MLP_OFF_W2
#define GRAD_B2 SIM_MLP_OFF_B2
#define GRAD_W3 SIM_MLP_OFF_W3
#define GRAD_B3 SIM_MLP_OFF_B3

__device__ __forceinline__ float mlp_fc(float r) { return 0.5f * (__cosf(3.14159265358979f * r / MLP_RC) + 1.0f); }
__device__ __forceinline__ float mlp_dfc(float r) {
    return -0.5f * (3.14159265358979f / MLP_RC) * __sinf(3.14159265358979f * r / MLP_RC);
}
__device__ __forceinline__ float mlp_rs(int k) { return 2.0f + 2.4f * (float)k / 7.0f; }

// d = x_j - x_i (Cartesian, minimum image) from fixed-point codes
template <bool ORTHO>
__device__ __forceinline__ void mlp_dvec(const BoxF& b, const int4& qi, const int4& qj, float& d0, float& d1,
                                         float& d2) {
    rvec<ORTHO>(b, qj, qi, d0, d1, d2);
}

// Descriptor and force kernels: GRP threads per atom (4 or 8), 128 / GRP
// atoms per 128-thread block.  The group first gathers the atom's in-cutoff list
// entries into a shared-memory table (entry-major, so the eight atoms of a
// warp read eight consecutive elements), then splits the pair loops by the
// first neighbour a (a = sub, sub + 4, ...).
#define MLP_APB_MAX 32

template <int APB>
struct MlpTableU {
    float4 u[MLP_MAXN][APB];     // unit vector d/r, e(r)
};
template <int APB>
struct MlpTable {
    float4 u[MLP_MAXN][APB];     // unit vector d/r, e(r)
    float2 w[MLP_MAXN][APB];     // e'(r), e(r)/r                      (forces)
    int32_t j[MLP_MAXN][APB];    // neighbour slot                      (forces)
    float srad[MLP_MAXN][APB];   // sum_k dE/dG_k dphi_k/dr (radial)    (forces)
};

// Fills the table of local atom g (slot i) and returns the in-cutoff count
// (capped at MLP_MAXN; more sets `over`).  FORCE: radial derivative sums
// from dE/dG (gr[0..7]); otherwise the radial descriptors are added to
// rad[0..7] (this lane's share of the atom's neighbours).
template <bool ORTHO, bool FORCE, int GRP, class Table>
__device__ __forceinline__ int mlp_table(const SimEngine& e, const BoxF& b, int64_t i, bool live, int g, int sub,
                                         Table& T, const float* gr, float* rad, bool& over) {
    const int lane = threadIdx.x & 31;
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int4 qi = live ? posq[i] : make_int4(0, 0, 0, 0);
    const int nn = live ? e.nnbr[i] : 0;
    const int nn_max = __reduce_max_sync(0xffffffffu, nn);
    int cnt = 0;
    // R rounds of GRP entries at a time: their list entries, then their
    // positions, are all in flight before the first distance is needed
    constexpr int R = 4;
    for (int k0 = 0; k0 < nn_max; k0 += GRP * R) {
        int jj[R];
        int4 qq[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = k0 + r * GRP + sub;
            jj[r] = k < nn ? ld_stream(&e.nbr[(int64_t)k * e.n_pad + i]) : -1;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) qq[r] = jj[r] >= 0 ? __ldg(&posq[jj[r]]) : make_int4(0, 0, 0, 0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            bool inside = false;
            float d0 = 0.f, d1 = 0.f, d2 = 0.f, r2 = 0.f;
            const int j = jj[r];
            if (j >= 0) {
                mlp_dvec<ORTHO>(b, qi, qq[r], d0, d1, d2);
                r2 = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
                inside = r2 < MLP_RC * MLP_RC;
            }
            const unsigned grp = (__ballot_sync(0xffffffffu, inside) >> (lane & ~(GRP - 1))) & ((1u << GRP) - 1u);
            const int pos = cnt + __popc(grp & ((1u << sub) - 1u));
            if (inside) {
                if (pos < MLP_MAXN) {
                    const float r = sqrtf(r2), ir = 1.0f / r;
                    const float fc = mlp_fc(r), ex = __expf(-0.01f * r2), ev = ex * fc;
                    T.u[pos][g] = make_float4(d0 * ir, d1 * ir, d2 * ir, ev);
                    // exp(-4 (r - R_k)^2) by the recurrence over k (R_k = 2 + k h):
                    // x_{k+1} = x_k exp(8 h t0) exp(-4 h^2 (2k + 1)), t0 = r - 2
                    const float step[8] = {0.6248747f, 0.24399385f, 0.09527189f, 0.037200667f,
                                           0.014525686f, 0.005671822f, 0.0022146674f, 0.0008647577f};
                    const float t0 = r - 2.0f, q8 = __expf(2.7428572f * t0);
                    float gk = __expf(-4.0f * t0 * t0);
                    if constexpr (FORCE) {
                        const float dfc = mlp_dfc(r);
                        T.w[pos][g] = make_float2(ex * fmaf(-0.02f * r, fc, dfc), ev * ir);
                        T.j[pos][g] = j;
                        float sr = 0.0f;
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const float t = fmaf(-0.34285715f, (float)q, t0);
                            sr = fmaf(gr[q], gk * fmaf(-8.0f * t, fc, dfc), sr);
                            gk *= q8 * step[q];
                        }
                        T.srad[pos][g] = sr;
                    } else {
    #pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            rad[q] = fmaf(gk, fc, rad[q]);
                            gk *= q8 * step[q];
                        }
                    }
                } else {
                    over = true;
                }
            }
            cnt += __popc(grp);
        }
    }
    __syncwarp();
    return cnt < MLP_MAXN ? cnt : MLP_MAXN;
}

template <int GRP>
__device__ __forceinline__ float grp_sum(float v) {
#pragma unroll
    for (int o = 1; o < GRP; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The eight angular terms of one pair (raw powers of 1 +- cos; the 2^(1-z)
// after the reduction) into d[8..15].
__device__ __forceinline__ void angular_terms(const float4& ua, const float4& uc, float* d) {
    const float cs = fmaf(ua.z, uc.z, fmaf(ua.y, uc.y, ua.x * uc.x));
    const float rad = ua.w * uc.w;
    const float p1 = 1.0f + cs, m1 = 1.0f - cs;
    const float p2 = p1 * p1, m2 = m1 * m1, p4 = p2 * p2, m4 = m2 * m2;
    d[8] = fmaf(p1, rad, d[8]);
    d[9] = fmaf(m1, rad, d[9]);
    d[10] = fmaf(p2, rad, d[10]);
    d[11] = fmaf(m2, rad, d[11]);
    d[12] = fmaf(p4, rad, d[12]);
    d[13] = fmaf(m4, rad, d[13]);
    d[14] = fmaf(p4 * p4, rad, d[14]);
    d[15] = fmaf(m4 * m4, rad, d[15]);
}

template <bool ORTHO, int GRP>
__global__ void __launch_bounds__(128) k_mlp_desc(SimEngine e, float* __restrict__ G) {
    constexpr int APB = 128 / GRP;
    __shared__ MlpTableU<APB> T;
    pdl_trigger();
    pdl_wait();
    const BoxF b(*e.box);
    const int g = threadIdx.x / GRP, sub = threadIdx.x % GRP;
    bool over = false;
    for (int64_t base = blockIdx.x * (int64_t)APB; base < e.n; base += (int64_t)gridDim.x * APB) {
        const int64_t i = base + g;
        const bool live = i < e.n;
        float d[MLP_D];
#pragma unroll
        for (int q = 0; q < MLP_D; ++q) d[q] = 0.0f;
        const int cnt = mlp_table<ORTHO, false, GRP>(e, b, i, live, g, sub, T, nullptr, d, over);
        // angular: raw powers (1 +- c)^z summed over a < c; the 2^(1-z) after the
        // reduction.  Lane sub takes rows a0 = sub and a1 = 2 GRP - 1 - sub of
        // every block of 2 GRP (a long and a short row of the triangle: the
        // lanes' pair counts balance) and walks them together: c in (a0, a1]
        // pairs with a0 alone, c > a1 with both, one table load of u_c serving
        // the two pairs.
        for (int blk = 0; blk < (cnt + 2 * GRP - 1) / (2 * GRP); ++blk) {
            const int a0 = blk * 2 * GRP + sub, a1 = blk * 2 * GRP + 2 * GRP - 1 - sub;
            if (a0 >= cnt) continue;
            const float4 ua0 = T.u[a0][g];
            const int c1 = a1 < cnt ? a1 : cnt - 1;
            for (int c = a0 + 1; c <= c1; ++c) angular_terms(ua0, T.u[c][g], d);
            if (a1 >= cnt) continue;
            const float4 ua1 = T.u[a1][g];
            for (int c = a1 + 1; c < cnt; ++c) {
                const float4 uc = T.u[c][g];
                angular_terms(ua0, uc, d);
                angular_terms(ua1, uc, d);
            }
        }
#pragma unroll
        for (int q = 0; q < MLP_D; ++q) d[q] = grp_sum<GRP>(d[q]);
        d[10] *= 0.5f; d[11] *= 0.5f; d[12] *= 0.125f; d[13] *= 0.125f; d[14] *= 0.0078125f; d[15] *= 0.0078125f;
        if (live && sub < 4) {   // lane sub writes float4 number sub of the row
            float4 v = make_float4(d[0], d[1], d[2], d[3]);
#pragma unroll
            for (int q = 1; q < 4; ++q)
                if (q == sub) v = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
            reinterpret_cast<float4*>(G + i * MLP_D)[sub] = v;
        }
        __syncwarp();
    }
    if (over) atomicOr(&e.flags[1], SIM_STATUS_MLP_NEIGHBORS);
}

// Forces from dE/dG (already including the 1/sigma of the normalisation).
// With the angular part of E_i written as sum_{a<c} S(cos_ac) e_a e_c,
//   S(x) = sum_(z,l) dE/dG_zl 2^(1-z) (1 + l x)^z = sum_m s_m x^m  (degree 8),
// the derivative of E_i with respect to d_a is
//   g_a = srad_a u_a + (e_a / r_a) (A_a - B_a u_a) + e'_a C_a u_a,
//   A_a = sum_{c != a} S'(cos_ac) e_c u_c, B_a = sum_{c != a} S'(cos_ac) e_c cos_ac,
//   C_a = sum_{c != a} S(cos_ac) e_c,
// (each ordered pair evaluated by the lane owning a).  Atom j_a receives
// -g_a, atom i +sum_a g_a, by float4 atomics (the summation order, and so
// the last bits, vary from run to run).
// Sums over c of one row a of the force kernel: A_a (vector), B_a, C_a.
struct MlpRowSums {
    float Ax = 0.f, Ay = 0.f, Az = 0.f, B = 0.f, C = 0.f;
};

// Pair (a, c): S and S' of cos_ac by one Horner recurrence on FP32x2 pairs
// {S, S'} (coefficient pairs ssd, each lane rounding as the scalar fmaf),
// added to the row sums unless c is a itself.
__device__ __forceinline__ void force_pair(const float4& ua, const float4& uc, bool other, const float2 (&ssd)[8],
                                           float s0, MlpRowSums& r) {
    const float x = fmaf(ua.z, uc.z, fmaf(ua.y, uc.y, ua.x * uc.x));
    const float2 xx = make_float2(x, x);
    float2 h = ssd[0];
#pragma unroll
    for (int m = 7; m >= 1; --m) h = __ffma2_rn(h, xx, ssd[m]);
    const float S = fmaf(h.x, x, s0), Sp = h.y;
    if (other) {
        const float t1 = Sp * uc.w;
        r.Ax = fmaf(t1, uc.x, r.Ax); r.Ay = fmaf(t1, uc.y, r.Ay); r.Az = fmaf(t1, uc.z, r.Az);
        r.B = fmaf(t1, x, r.B);
        r.C = fmaf(S, uc.w, r.C);
    }
}

// Row a finished: g_a to neighbour j_a (-g_a) and to the atom's own sum.
template <class Table>
__device__ __forceinline__ void force_row(const Table& T, int a, int g, const float4& ua, const MlpRowSums& r,
                                          float4* f, float& fx, float& fy, float& fz) {
    const float2 wa = T.w[a][g];
    const float k = T.srad[a][g] - wa.y * r.B + wa.x * r.C;
    const float gx = fmaf(wa.y, r.Ax, k * ua.x), gy = fmaf(wa.y, r.Ay, k * ua.y), gz = fmaf(wa.y, r.Az, k * ua.z);
    atomicAdd(&f[T.j[a][g]], make_float4(-gx, -gy, -gz, 0.0f));
    fx += gx; fy += gy; fz += gz;
}

template <bool ORTHO, int GRP>
__global__ void __launch_bounds__(128) k_mlp_force(SimEngine e, const float* __restrict__ dEdG) {
    constexpr int APB = 128 / GRP;
    __shared__ MlpTable<APB> T;
    const BoxF b(*e.box);
    float4* f = reinterpret_cast<float4*>(e.f32);
    const int g = threadIdx.x / GRP, sub = threadIdx.x % GRP;
    bool over = false;
    for (int64_t base = blockIdx.x * (int64_t)APB; base < e.n; base += (int64_t)gridDim.x * APB) {
        const int64_t i = base + g;
        const bool live = i < e.n;
        float gr[MLP_D];
        {
            const float4* src = reinterpret_cast<const float4*>(dEdG + (live ? i : 0) * MLP_D);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = live ? __ldg(&src[q]) : make_float4(0.f, 0.f, 0.f, 0.f);
                gr[4 * q] = v.x; gr[4 * q + 1] = v.y; gr[4 * q + 2] = v.z; gr[4 * q + 3] = v.w;
            }
        }
        // monomial coefficients of S: 2^(1-z) binom(z, m) (g_z+ + (-1)^m g_z-)
        const float P1 = gr[8] + gr[9], M1 = gr[8] - gr[9], P2 = gr[10] + gr[11], M2 = gr[10] - gr[11];
        const float P4 = gr[12] + gr[13], M4 = gr[12] - gr[13], P8 = gr[14] + gr[15], M8 = gr[14] - gr[15];
        float s[9];
        s[0] = P1 + 0.5f * P2 + 0.125f * P4 + 0.0078125f * P8;
        s[1] = M1 + M2 + 0.5f * M4 + 0.0625f * M8;
        s[2] = 0.5f * P2 + 0.75f * P4 + 0.21875f * P8;
        s[3] = 0.5f * M4 + 0.4375f * M8;
        s[4] = 0.125f * P4 + 0.546875f * P8;
        s[5] = 0.4375f * M8;
        s[6] = 0.21875f * P8;
        s[7] = 0.0625f * M8;
        s[8] = 0.0078125f * P8;
        float sd[8];   // coefficients of S': (m + 1) s_(m+1)
#pragma unroll
        for (int m = 0; m < 8; ++m) sd[m] = (float)(m + 1) * s[m + 1];
        // S and S' by one Horner recurrence on FP32x2 pairs {S, S'}: coefficient
        // pairs {s_m, sd_(m-1)}; each lane rounds as the scalar fmaf
        float2 ssd[8];
#pragma unroll
        for (int m = 1; m <= 7; ++m) ssd[m] = make_float2(s[m], sd[m - 1]);
        ssd[0] = make_float2(s[8], sd[7]);
        const int cnt = mlp_table<ORTHO, true, GRP>(e, b, i, live, g, sub, T, gr, nullptr, over);
        float fx = 0.f, fy = 0.f, fz = 0.f;
        // rows a and a + GRP of the lane together: one table load of u_c
        // serves both rows' pairs
        for (int a = sub; a < cnt; a += 2 * GRP) {
            const int a2 = a + GRP;
            const bool two = a2 < cnt;
            const float4 ua = T.u[a][g];
            const float4 ub = T.u[two ? a2 : a][g];
            MlpRowSums ra, rb;
            for (int c = 0; c < cnt; ++c) {
                const float4 uc = T.u[c][g];
                force_pair(ua, uc, c != a, ssd, s[0], ra);
                if (two) force_pair(ub, uc, c != a2, ssd, s[0], rb);
            }
            force_row(T, a, g, ua, ra, f, fx, fy, fz);
            if (two) force_row(T, a2, g, ub, rb, f, fx, fy, fz);
        }
        fx = grp_sum<GRP>(fx); fy = grp_sum<GRP>(fy); fz = grp_sum<GRP>(fz);
        if (live && sub == 0) atomicAdd(&f[i], make_float4(fx, fy, fz, 0.0f));
        __syncwarp();
    }
    if (over) atomicOr(&e.flags[1], SIM_STATUS_MLP_NEIGHBORS);
}

// Per-atom EAM energy E_i = F(rho_i) + 1/2 sum_j phi(r_ij) (one element type):
// the decomposition of the EAM total that the surrogate is trained on.
__global__ void __launch_bounds__(256) k_eam_atom_energy(SimEngine e, SimEAMTables t, float* __restrict__ out) {
    const BoxF b(*e.box);
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const float2* dens = reinterpret_cast<const float2*>(t.dens_vd);
    const float2* pair = reinterpret_cast<const float2*>(t.pair_vd);
    const float rc2 = t.cutoff * t.cutoff;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int4 qi = posq[i];
        float rho = 0.0f, half = 0.0f;
        for (int k = 0; k < e.nnbr[i]; ++k) {
            const int4 qj = __ldg(&posq[ld_stream(&e.nbr[(int64_t)k * e.n_pad + i])]);
            float r0, r1, r2;
            rvec<false>(b, qi, qj, r0, r1, r2);
            const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
            if (!(d2 < rc2)) continue;
            const Lerp l = lerp_r(sqrtf(d2), t);
            const float2 dv = __ldg(&dens[l.k]);
            const float2 pv = __ldg(&pair[l.k]);
            rho += fmaf(l.frac, dv.y, dv.x);
            half = fmaf(0.5f, fmaf(l.frac, pv.y, pv.x), half);
        }
        float F, Fp;
        embed_lookup(t, 0, rho, F, Fp);
        out[i] = F + half;
    }
}

// ---------------------------------------------------------------------------
// network on the tensor cores

// Element (r, k) of a K-major operand image with K columns: 8x8 core matrices
// (8 rows of 16 bytes, 128 bytes each), row groups of 8 after one another
// every K/8 core matrices.
__device__ __forceinline__ int img_off(int r, int k, int K) { return ((r >> 3) * (K >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7); }

// Shared-memory matrix descriptor (no swizzle, K-major): start >> 4 in bits
// 0-13, leading (next 8-wide K chunk) byte offset >> 4 in 16-29, stride (next
// 8-row group) byte offset >> 4 in 32-45, descriptor version 1 in 46-47.
__device__ __forceinline__ uint64_t smem_desc(const void* p, int K) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    const uint64_t lbo = 128 >> 4, sbo = (uint64_t)((K >> 3) * 128) >> 4;
    return (uint64_t)((a >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulate (bits 4-5 = 1), BF16 A
// and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in
// bits 24-28.
__host__ __device__ constexpr uint32_t mma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"((uint32_t)__cvta_generic_to_shared(bar)) : "memory");
}

// bounded wait for the phase `parity` of an mbarrier; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (int it = 0; it < MLP_WAIT_LIMIT; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(addr));
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// logistic sigmoid as 1/2 + tanh(z/2)/2 on the hardware tanh approximation
// (tanh.approx.f32: one MUFU operation instead of an exponential and a
// reciprocal; its relative error, about 2^-11, is below the BF16 rounding of
// the activations that feed the next layer; saturates to 0 and 1)
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}

// write 8 consecutive k of row r of an operand image (16-byte store)
__device__ __forceinline__ void img_store8(__nv_bfloat16* img, int r, int k0, int K, const float* v) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16_rn(v[q]);
    *reinterpret_cast<uint4*>(img + img_off(r, k0, K)) = *reinterpret_cast<const uint4*>(h);
}

struct MlpSmem {
    __nv_bfloat16 w1t[MLP_H * MLP_D];     // B of Z1 = G W1:      rows n (64), K = 16
    __nv_bfloat16 w2t[MLP_H * MLP_H];     // B of Z2 = H1 W2:     rows n (64), K = 64
    __nv_bfloat16 w2[MLP_H * MLP_H];      // B of D1 = dZ2 W2^T:  rows k (64), K = 64
    __nv_bfloat16 w1[MLP_D * MLP_H];      // B of dG = dZ1 W1^T:  rows c (16), K = 64
    __nv_bfloat16 a0[MLP_TILE * MLP_D];   // normalised descriptors
    __nv_bfloat16 a1[MLP_TILE * MLP_H];   // H1, then dZ2
    __nv_bfloat16 a2[MLP_TILE * MLP_H];   // dZ1 (and dZ2 while training)
    __nv_bfloat16 a3[MLP_TILE * MLP_H];   // training: H1 kept for the weight gradients
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], mu[MLP_D], isg[MLP_D], b3;
    uint64_t bar;
    uint32_t tmem;
};

// Inference: E_i and dE/dG (scaled by 1/sigma) per atom.  One activation
// image serves every layer (H1, then dZ2, then dZ1: each MMA has completed
// before its operand is overwritten), so four blocks fit on an SM (tensor
// memory: 4 x 128 columns); the epilogues walk the accumulators 16 columns
// at a time, and the next tile's descriptors load while this tile's MMAs run.
struct MlpFwdSmem {
    __nv_bfloat16 w1t[MLP_H * MLP_D];
    __nv_bfloat16 w2t[MLP_H * MLP_H];
    __nv_bfloat16 w2[MLP_H * MLP_H];
    __nv_bfloat16 w1[MLP_D * MLP_H];
    __nv_bfloat16 a0[MLP_TILE * MLP_D];
    __nv_bfloat16 a1[MLP_TILE * MLP_H];
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], mu[MLP_D], isg[MLP_D], b3;
    uint64_t bar;
    uint32_t tmem;
};

__device__ __forceinline__ void mlp_load_row(const float* G, int64_t i, bool live, float* v) {
    const float4* src = reinterpret_cast<const float4*>(G + (live ? i : 0) * MLP_D);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 x = live ? __ldg(&src[q]) : make_float4(0.f, 0.f, 0.f, 0.f);
        v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
}

__global__ void __launch_bounds__(MLP_TILE) k_mlp_fwd(SimMLP m, const float* __restrict__ G, int64_t n,
                                                      float* __restrict__ e_atom, float* __restrict__ dEdG,
                                                      int32_t* status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MlpFwdSmem& S = *reinterpret_cast<MlpFwdSmem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5;
    pdl_trigger();
    {
        const uint4* src[4] = {reinterpret_cast<const uint4*>(m.w1t_img), reinterpret_cast<const uint4*>(m.w2t_img),
                               reinterpret_cast<const uint4*>(m.w2_img), reinterpret_cast<const uint4*>(m.w1_img)};
        uint4* dst[4] = {reinterpret_cast<uint4*>(S.w1t), reinterpret_cast<uint4*>(S.w2t),
                         reinterpret_cast<uint4*>(S.w2), reinterpret_cast<uint4*>(S.w1)};
        const int cnt[4] = {MLP_H * MLP_D / 8, MLP_H * MLP_H / 8, MLP_H * MLP_H / 8, MLP_D * MLP_H / 8};
#pragma unroll
        for (int w = 0; w < 4; ++w)
            for (int q = t; q < cnt[w]; q += blockDim.x) dst[w][q] = src[w][q];
        if (t < MLP_H) { S.b1[t] = m.b1[t]; S.b2[t] = m.b2[t]; S.w3[t] = m.w3[t]; }
        if (t < MLP_D) { S.mu[t] = m.mu[t]; S.isg[t] = m.inv_sigma[t]; }
        if (t == 0) S.b3 = *m.b3;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;"
                     :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"((uint32_t)__cvta_generic_to_shared(&S.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = S.tmem;
    const uint32_t lb = (uint32_t)(32 * warp) << 16;
    uint32_t phase = 0;
    bool failed = false;
    const int n_tiles = (int)((n + MLP_TILE - 1) / MLP_TILE);
    float gn[MLP_D];
    pdl_wait();   // weights and tensor memory are set up; the descriptors come from the previous kernel
    {
        const int64_t i0 = (int64_t)blockIdx.x * MLP_TILE + t;
        mlp_load_row(G, i0, i0 < n, gn);
    }
    for (int tile = blockIdx.x; tile < n_tiles && !failed; tile += gridDim.x) {
        const int64_t i = (int64_t)tile * MLP_TILE + t;
        const bool live = i < n;
#pragma unroll
        for (int c = 0; c < MLP_D; ++c) gn[c] = live ? (gn[c] - S.mu[c]) * S.isg[c] : 0.0f;
        img_store8(S.a0, t, 0, MLP_D, gn);
        img_store8(S.a0, t, 8, MLP_D, gn + 8);
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // Z1 = g W1 -> [0, 64)
            mma_bf16(tm, smem_desc(S.a0, MLP_D), smem_desc(S.w1t, MLP_D), mma_idesc(128, MLP_H), 0);
            mma_commit(&S.bar);
        }
        {   // the next tile's rows, in flight while the tensor cores work
            const int64_t inext = i + (int64_t)gridDim.x * MLP_TILE;
            mlp_load_row(G, inext, inext < n, gn);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16];
            tmem_ld16(tm + lb + 16 * q, z);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) z[c] = silu(z[c] + S.b1[16 * q + c]);
            img_store8(S.a1, t, 16 * q, MLP_H, z);
            img_store8(S.a1, t, 16 * q + 8, MLP_H, z + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // Z2 = H1 W2 -> [64, 128)
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s)
                mma_bf16(tm + 64, smem_desc(S.a1 + s * 128, MLP_H), smem_desc(S.w2t + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        float E = S.b3;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16];
            tmem_ld16(tm + lb + 64 + 16 * q, z);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int k = 16 * q + c;
                const float zz = z[c] + S.b2[k], sg = sigm(zz);
                E = fmaf(S.w3[k], zz * sg, E);
                z[c] = live ? S.w3[k] * sg * fmaf(zz, 1.0f - sg, 1.0f) : 0.0f;   // dZ2
            }
            img_store8(S.a1, t, 16 * q, MLP_H, z);
            img_store8(S.a1, t, 16 * q + 8, MLP_H, z + 8);
        }
        if (live) e_atom[i] = E;
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // D1 = dZ2 W2^T -> [64, 128)
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s)
                mma_bf16(tm + 64, smem_desc(S.a1 + s * 128, MLP_H), smem_desc(S.w2 + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], d[16];
            tmem_ld16(tm + lb + 16 * q, z);
            tmem_ld16(tm + lb + 64 + 16 * q, d);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) d[c] *= dsilu(z[c] + S.b1[16 * q + c]);   // dZ1
            img_store8(S.a1, t, 16 * q, MLP_H, d);
            img_store8(S.a1, t, 16 * q + 8, MLP_H, d + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // dG = dZ1 W1^T -> [0, 16)
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s)
                mma_bf16(tm, smem_desc(S.a1 + s * 128, MLP_H), smem_desc(S.w1 + s * 128, MLP_H),
                         mma_idesc(128, MLP_D), s > 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        float gv[MLP_D];
        tmem_ld16(tm + lb, gv);
        tmem_wait_ld();
        if (live) {
            float4* out = reinterpret_cast<float4*>(dEdG + i * MLP_D);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                out[q] = make_float4(gv[4 * q] * S.isg[4 * q], gv[4 * q + 1] * S.isg[4 * q + 1],
                                     gv[4 * q + 2] * S.isg[4 * q + 2], gv[4 * q + 3] * S.isg[4 * q + 3]);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (failed && t == 0) atomicOr(status, SIM_STATUS_MLP_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" :: "r"(tm));
}

// Energy regression: per-atom loss (E_i - target_i)^2 / n_batch, its gradient
// with respect to every weight (added to grads with atomics) and the loss sum
// (added to *loss).
__global__ void __launch_bounds__(MLP_TILE) k_mlp_train(SimMLP m, const float* __restrict__ G, int64_t n,
                                                        const float* __restrict__ target, float inv_batch,
                                                        float* __restrict__ grads, float* __restrict__ loss,
                                                        int32_t* status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5;
    // weights (pre-arranged operand images) and vectors
    {
        const uint4* src[4] = {reinterpret_cast<const uint4*>(m.w1t_img), reinterpret_cast<const uint4*>(m.w2t_img),
                               reinterpret_cast<const uint4*>(m.w2_img), reinterpret_cast<const uint4*>(m.w1_img)};
        uint4* dst[4] = {reinterpret_cast<uint4*>(S.w1t), reinterpret_cast<uint4*>(S.w2t),
                         reinterpret_cast<uint4*>(S.w2), reinterpret_cast<uint4*>(S.w1)};
        const int cnt[4] = {MLP_H * MLP_D / 8, MLP_H * MLP_H / 8, MLP_H * MLP_H / 8, MLP_D * MLP_H / 8};
#pragma unroll
        for (int w = 0; w < 4; ++w)
            for (int q = t; q < cnt[w]; q += blockDim.x) dst[w][q] = src[w][q];
        if (t < MLP_H) { S.b1[t] = m.b1[t]; S.b2[t] = m.b2[t]; S.w3[t] = m.w3[t]; }
        if (t < MLP_D) { S.mu[t] = m.mu[t]; S.isg[t] = m.inv_sigma[t]; }
        if (t == 0) S.b3 = *m.b3;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;"
                     :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"((uint32_t)__cvta_generic_to_shared(&S.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = S.tmem;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    uint32_t phase = 0;
    bool failed = false;
    const int n_tiles = (int)((n + MLP_TILE - 1) / MLP_TILE);
    // per-thread partial weight gradients are summed with atomics per tile
    for (int tile = blockIdx.x; tile < n_tiles && !failed; tile += gridDim.x) {
        const int64_t i = (int64_t)tile * MLP_TILE + t;
        const bool live = i < n;
        float gn[MLP_D];
        {
            const float4* src = reinterpret_cast<const float4*>(G + (live ? i : 0) * MLP_D);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = live ? src[q] : make_float4(0.f, 0.f, 0.f, 0.f);
                gn[4 * q] = v.x; gn[4 * q + 1] = v.y; gn[4 * q + 2] = v.z; gn[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int c = 0; c < MLP_D; ++c) gn[c] = live ? (gn[c] - S.mu[c]) * S.isg[c] : 0.0f;
            img_store8(S.a0, t, 0, MLP_D, gn);
            img_store8(S.a0, t, 8, MLP_D, gn + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // Z1 = G W1 -> tmem columns [0, 64)
        if (t == 0) {
            mma_bf16(tm, smem_desc(S.a0, MLP_D), smem_desc(S.w1t, MLP_D), mma_idesc(128, MLP_H), 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        {
            float z1[MLP_H];
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(tm + lane_base + 16 * q, z1 + 16 * q);
            tmem_wait_ld();
            float h[8];
#pragma unroll
            for (int k0 = 0; k0 < MLP_H; k0 += 8) {
#pragma unroll
                for (int q = 0; q < 8; ++q) h[q] = silu(z1[k0 + q] + S.b1[k0 + q]);
                img_store8(S.a1, t, k0, MLP_H, h);
                img_store8(S.a3, t, k0, MLP_H, h);
            }
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // Z2 = H1 W2 -> tmem columns [64, 128)
        if (t == 0) {
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s)
                mma_bf16(tm + 64, smem_desc(S.a1 + s * 2 * 64, MLP_H), smem_desc(S.w2t + s * 2 * 64, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        float z2[MLP_H];
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16(tm + lane_base + 64 + 16 * q, z2 + 16 * q);
        tmem_wait_ld();
        float E = S.b3;
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) E = fmaf(S.w3[k], silu(z2[k] + S.b2[k]), E);
        // dL/dE = 2 (E - target) / n_batch
        const float err = live ? E - target[i] : 0.0f;
        const float up = 2.0f * err * inv_batch;
        {
            const float ls = warp_sum_f(live ? err * err * inv_batch : 0.0f);
            if ((t & 31) == 0) atomicAdd(loss, ls);
        }
        {
            float d[8];
#pragma unroll
            for (int k0 = 0; k0 < MLP_H; k0 += 8) {
#pragma unroll
                for (int q = 0; q < 8; ++q) d[q] = up * S.w3[k0 + q] * dsilu(z2[k0 + q] + S.b2[k0 + q]);
                img_store8(S.a2, t, k0, MLP_H, d);
            }
            // output layer: dw3 = sum up * h2, db3 = sum up
#pragma unroll 4
            for (int k = 0; k < MLP_H; ++k) {
                const float v = warp_sum_f(up * silu(z2[k] + S.b2[k]));
                if ((t & 31) == 0) atomicAdd(&grads[GRAD_W3 + k], v);
            }
            const float v = warp_sum_f(up);
            if ((t & 31) == 0) atomicAdd(&grads[GRAD_B3], v);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // D1 = dZ2 W2^T -> tmem columns [64, 128)
        const __nv_bfloat16* dz2 = S.a2;
        if (t == 0) {
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s)
                mma_bf16(tm + 64, smem_desc(dz2 + s * 2 * 64, MLP_H), smem_desc(S.w2 + s * 2 * 64, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        float d1[MLP_H];
        {
            float z1[MLP_H];
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(tm + lane_base + 64 + 16 * q, d1 + 16 * q);
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(tm + lane_base + 16 * q, z1 + 16 * q);
            tmem_wait_ld();
#pragma unroll
            for (int k = 0; k < MLP_H; ++k) d1[k] *= dsilu(z1[k] + S.b1[k]);
        }
        // weight gradients on the CUDA cores from the tile's operands:
        // thread t owns column n = t & 63 of dW2 (rows k) and of dW1 (rows c),
        // half the rows each; sums over the tile's 128 atoms
        float dk[8];
#pragma unroll
        for (int k0 = 0; k0 < MLP_H; k0 += 8) {
#pragma unroll
            for (int q = 0; q < 8; ++q) dk[q] = d1[k0 + q];
            img_store8(S.a1, t, k0, MLP_H, dk);        // dZ1 (H1 is kept in a3)
        }
        __syncthreads();
        const int col = t & 63, half = t >> 6;
        // dW2[k][col] = sum_r H1[r][k] dZ2[r][col]; db2[col] = sum_r dZ2[r][col]
        for (int k = half * 32; k < half * 32 + 32; ++k) {
            float acc = 0.0f;
            for (int r = 0; r < MLP_TILE; ++r)
                acc = fmaf(__bfloat162float(S.a3[img_off(r, k, MLP_H)]),
                           __bfloat162float(S.a2[img_off(r, col, MLP_H)]), acc);
            atomicAdd(&grads[GRAD_W2 + k * MLP_H + col], acc);
        }
        // dW1[c][col] = sum_r G[r][c] dZ1[r][col]; db1, db2
        for (int c = half * 8; c < half * 8 + 8; ++c) {
            float acc = 0.0f;
            for (int r = 0; r < MLP_TILE; ++r)
                acc = fmaf(__bfloat162float(S.a0[img_off(r, c, MLP_D)]),
                           __bfloat162float(S.a1[img_off(r, col, MLP_H)]), acc);
            atomicAdd(&grads[GRAD_W1 + c * MLP_H + col], acc);
        }
        if (half == 0) {
            float a = 0.0f, bsum = 0.0f;
            for (int r = 0; r < MLP_TILE; ++r) {
                a += __bfloat162float(S.a1[img_off(r, col, MLP_H)]);
                bsum += __bfloat162float(S.a2[img_off(r, col, MLP_H)]);
            }
            atomicAdd(&grads[GRAD_B1 + col], a);
            atomicAdd(&grads[GRAD_B2 + col], bsum);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (failed && t == 0) atomicOr(status, SIM_STATUS_MLP_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" :: "r"(tm));
}

// Force-matching pieces.  With e = F - F_target per slot, the gradient of the
// force loss with respect to the network's parameters needs, per atom, the
// descriptor Jacobian contracted with the force errors of the atom and its
// neighbours: u_i = sum_m e_m . dG_i/dx_m = sum_j (e_j - e_i) . dG_i/dd_j.
template <bool ORTHO>
__global__ void __launch_bounds__(128) k_mlp_ucontract(SimEngine e, const float* __restrict__ ferr,
                                                        float* __restrict__ u) {
    const BoxF b(*e.box);
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const float4* __restrict__ er = reinterpret_cast<const float4*>(ferr);
    bool over = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 nb[MLP_MAXN];
        float ex[MLP_MAXN], ey[MLP_MAXN], ez[MLP_MAXN], ea[MLP_MAXN], eda[MLP_MAXN];
        const int4 qi = posq[i];
        const float4 ei = er[i];
        int cnt = 0;
        for (int k = 0; k < e.nnbr[i]; ++k) {
            const int j = ld_stream(&e.nbr[(int64_t)k * e.n_pad + i]);
            const int4 qj = __ldg(&posq[j]);
            float d0, d1, d2;
            mlp_dvec<ORTHO>(b, qi, qj, d0, d1, d2);
            const float r2 = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
            if (!(r2 < MLP_RC * MLP_RC)) continue;
            if (cnt == MLP_MAXN) { over = true; continue; }
            const float4 ej = __ldg(&er[j]);
            nb[cnt] = make_float4(d0, d1, d2, sqrtf(r2));
            ex[cnt] = ej.x - ei.x; ey[cnt] = ej.y - ei.y; ez[cnt] = ej.z - ei.z;
            ++cnt;
        }
        float g[MLP_D];
#pragma unroll
        for (int k = 0; k < MLP_D; ++k) g[k] = 0.0f;
        for (int a = 0; a < cnt; ++a) {
            const float r = nb[a].w, fc = mlp_fc(r), dfc = mlp_dfc(r);
            const float q = (ex[a] * nb[a].x + ey[a] * nb[a].y + ez[a] * nb[a].z) / r;   // (de . d)/r
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float t = r - mlp_rs(k);
                g[k] = fmaf(__expf(-4.0f * t * t) * fmaf(-8.0f * t, fc, dfc), q, g[k]);
            }
            const float xe = __expf(-0.01f * r * r);
            ea[a] = xe * fc;
            eda[a] = xe * fmaf(-0.02f * r, fc, dfc);
        }
        for (int a = 0; a < cnt; ++a) {
            const float4 da = nb[a];
            const float ira = 1.0f / da.w;
            const float qaa = ex[a] * da.x + ey[a] * da.y + ez[a] * da.z;
            for (int c = a + 1; c < cnt; ++c) {
                const float4 dc = nb[c];
                const float irc = 1.0f / dc.w;
                const float cs = (da.x * dc.x + da.y * dc.y + da.z * dc.z) * ira * irc;
                const float qac = ex[a] * dc.x + ey[a] * dc.y + ez[a] * dc.z;
                const float qca = ex[c] * da.x + ey[c] * da.y + ez[c] * da.z;
                const float qcc = ex[c] * dc.x + ey[c] * dc.y + ez[c] * dc.z;
                const float rad = ea[a] * ea[c];
                const float Xc = rad * ((qac + qca) * ira * irc - cs * (qaa * ira * ira + qcc * irc * irc));
                const float Xe = eda[a] * ea[c] * qaa * ira + ea[a] * eda[c] * qcc * irc;
                const float p1 = 1.0f + cs, m1 = 1.0f - cs;
                const float p2 = p1 * p1, m2 = m1 * m1, p4 = p2 * p2, m4 = m2 * m2;
                const float p3 = p2 * p1, m3 = m2 * m1, p7 = p4 * p3, m7 = m4 * m3, p8 = p4 * p4, m8 = m4 * m4;
                // 2^(1-z) (1 + l c)^z and its derivative in c, for (z, l) = (1,+) (1,-) (2,+) ...
                g[8] += Xc + p1 * Xe;
                g[9] += -Xc + m1 * Xe;
                g[10] += p1 * Xc + 0.5f * p2 * Xe;
                g[11] += -m1 * Xc + 0.5f * m2 * Xe;
                g[12] += 0.5f * p3 * Xc + 0.125f * p4 * Xe;
                g[13] += -0.5f * m3 * Xc + 0.125f * m4 * Xe;
                g[14] += 0.0625f * p7 * Xc + 0.0078125f * p8 * Xe;
                g[15] += -0.0625f * m7 * Xc + 0.0078125f * m8 * Xe;
            }
        }
        float4* out = reinterpret_cast<float4*>(u + i * MLP_D);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
    }
    if (over) atomicOr(&e.flags[1], SIM_STATUS_MLP_NEIGHBORS);
}

__device__ __forceinline__ float d2silu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f - s) * (2.0f + z * (1.0f - 2.0f * s));
}

struct MlpFmSmem {
    __nv_bfloat16 w1t[MLP_H * MLP_D];     // B of Z1 = g W1 and Z1' = g' W1
    __nv_bfloat16 w2t[MLP_H * MLP_H];     // B of Z2 = H1 W2 and Z2' = H1' W2
    __nv_bfloat16 w2[MLP_H * MLP_H];      // B of P1 = P2 W2^T and Q1 = Q2 W2^T
    __nv_bfloat16 g0[MLP_TILE * MLP_D];   // normalised descriptors g
    __nv_bfloat16 gd[MLP_TILE * MLP_D];   // their tangent g' = u / sigma
    __nv_bfloat16 h1[MLP_TILE * MLP_H];   // H1, later dJ/dz1
    __nv_bfloat16 hd1[MLP_TILE * MLP_H];  // H1', later dJ/dz1'
    __nv_bfloat16 p2[MLP_TILE * MLP_H];   // dJ/dz2'
    __nv_bfloat16 q2[MLP_TILE * MLP_H];   // dJ/dz2
    float b1[MLP_H], b2[MLP_H], w3[MLP_H], mu[MLP_D], isg[MLP_D], b3;
    uint64_t bar;
    uint32_t tmem;
};

// thread t owns column `col` of a 64-wide weight gradient over half the rows:
// dst[k][col] += sum_r A[r][k] B[r][col] (+ C[r][k] D[r][col]) for k in rows
__device__ __forceinline__ void outer_acc(const __nv_bfloat16* A, const __nv_bfloat16* B, const __nv_bfloat16* C,
                                          const __nv_bfloat16* D, int KA, int k0, int k1, int col, float* dst) {
    for (int k = k0; k < k1; ++k) {
        float acc = 0.0f;
        for (int r = 0; r < MLP_TILE; ++r) {
            acc = fmaf(__bfloat162float(A[img_off(r, k, KA)]), __bfloat162float(B[img_off(r, col, MLP_H)]), acc);
            acc = fmaf(__bfloat162float(C[img_off(r, k, KA)]), __bfloat162float(D[img_off(r, col, MLP_H)]), acc);
        }
        atomicAdd(&dst[k * MLP_H + col], acc);
    }
}

// Gradient of J = sum_i [a_i E_i + beta dE_i] with dE_i = u_i . dE_i/dG_i and
// a_i = alpha (E_i - target_i): the energy and force-matching terms of the
// training loss, by reverse mode through the network and its directional
// derivative.  Six tensor-core GEMMs per tile (Z1, Z1', Z2, Z2', and the two
// back-propagations through W2); weight gradients summed on the CUDA cores.
__global__ void __launch_bounds__(MLP_TILE) k_mlp_train_fm(SimMLP m, const float* __restrict__ G,
                                                           const float* __restrict__ target,
                                                           const float* __restrict__ u, int64_t n, float alpha,
                                                           float beta, float inv_n, float* __restrict__ grads,
                                                           float* __restrict__ loss, int32_t* status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MlpFmSmem& S = *reinterpret_cast<MlpFmSmem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5;
    {
        const uint4* src[3] = {reinterpret_cast<const uint4*>(m.w1t_img), reinterpret_cast<const uint4*>(m.w2t_img),
                               reinterpret_cast<const uint4*>(m.w2_img)};
        uint4* dst[3] = {reinterpret_cast<uint4*>(S.w1t), reinterpret_cast<uint4*>(S.w2t),
                         reinterpret_cast<uint4*>(S.w2)};
        const int cnt[3] = {MLP_H * MLP_D / 8, MLP_H * MLP_H / 8, MLP_H * MLP_H / 8};
#pragma unroll
        for (int w = 0; w < 3; ++w)
            for (int q = t; q < cnt[w]; q += blockDim.x) dst[w][q] = src[w][q];
        if (t < MLP_H) { S.b1[t] = m.b1[t]; S.b2[t] = m.b2[t]; S.w3[t] = m.w3[t]; }
        if (t < MLP_D) { S.mu[t] = m.mu[t]; S.isg[t] = m.inv_sigma[t]; }
        if (t == 0) S.b3 = *m.b3;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;"
                     :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"((uint32_t)__cvta_generic_to_shared(&S.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = S.tmem;
    const uint32_t lb = (uint32_t)(32 * warp) << 16;
    uint32_t phase = 0;
    bool failed = false;
    const int n_tiles = (int)((n + MLP_TILE - 1) / MLP_TILE);
    const int col = t & 63, half = t >> 6;
    for (int tile = blockIdx.x; tile < n_tiles && !failed; tile += gridDim.x) {
        const int64_t i = (int64_t)tile * MLP_TILE + t;
        const bool live = i < n;
        {
            float a[MLP_D], d[MLP_D];
            const float4* gs = reinterpret_cast<const float4*>(G + (live ? i : 0) * MLP_D);
            const float4* us = reinterpret_cast<const float4*>(u + (live ? i : 0) * MLP_D);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = gs[q], w = us[q];
                a[4 * q] = v.x; a[4 * q + 1] = v.y; a[4 * q + 2] = v.z; a[4 * q + 3] = v.w;
                d[4 * q] = w.x; d[4 * q + 1] = w.y; d[4 * q + 2] = w.z; d[4 * q + 3] = w.w;
            }
#pragma unroll
            for (int c = 0; c < MLP_D; ++c) {
                a[c] = live ? (a[c] - S.mu[c]) * S.isg[c] : 0.0f;
                d[c] = live ? d[c] * S.isg[c] : 0.0f;
            }
            img_store8(S.g0, t, 0, MLP_D, a);
            img_store8(S.g0, t, 8, MLP_D, a + 8);
            img_store8(S.gd, t, 0, MLP_D, d);
            img_store8(S.gd, t, 8, MLP_D, d + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // Z1 -> [0, 64), Z1' -> [64, 128)
            mma_bf16(tm, smem_desc(S.g0, MLP_D), smem_desc(S.w1t, MLP_D), mma_idesc(128, MLP_H), 0);
            mma_bf16(tm + 64, smem_desc(S.gd, MLP_D), smem_desc(S.w1t, MLP_D), mma_idesc(128, MLP_H), 0);
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], zd[16], h[16], hd[16];
            tmem_ld16(tm + lb + 16 * q, z);
            tmem_ld16(tm + lb + 64 + 16 * q, zd);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const float zz = z[c] + S.b1[16 * q + c];
                h[c] = silu(zz);
                hd[c] = dsilu(zz) * zd[c];
            }
            img_store8(S.h1, t, 16 * q, MLP_H, h);
            img_store8(S.h1, t, 16 * q + 8, MLP_H, h + 8);
            img_store8(S.hd1, t, 16 * q, MLP_H, hd);
            img_store8(S.hd1, t, 16 * q + 8, MLP_H, hd + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // Z2 -> [128, 192), Z2' -> [192, 256)
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s) {
                mma_bf16(tm + 128, smem_desc(S.h1 + s * 128, MLP_H), smem_desc(S.w2t + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
                mma_bf16(tm + 192, smem_desc(S.hd1 + s * 128, MLP_H), smem_desc(S.w2t + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            }
            mma_commit(&S.bar);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
        // energy first (a_i needs the full E_i)
        float E = S.b3;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16];
            tmem_ld16(tm + lb + 128 + 16 * q, z);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) E = fmaf(S.w3[16 * q + c], silu(z[c] + S.b2[16 * q + c]), E);
        }
        const float err = live ? E - target[i] : 0.0f;
        const float a_i = alpha * err;
        const float b_i = live ? beta : 0.0f;
        {
            const float l = warp_sum_f(err * err * inv_n);
            if ((t & 31) == 0) atomicAdd(loss, l);
            const float db3 = warp_sum_f(a_i);
            if ((t & 31) == 0) atomicAdd(&grads[GRAD_B3], db3);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], zd[16], pp[16], qq[16];
            tmem_ld16(tm + lb + 128 + 16 * q, z);
            tmem_ld16(tm + lb + 192 + 16 * q, zd);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int k = 16 * q + c;
                const float zz = z[c] + S.b2[k];
                const float s1 = dsilu(zz), s2 = d2silu(zz);
                pp[c] = b_i * S.w3[k] * s1;
                qq[c] = a_i * S.w3[k] * s1 + b_i * S.w3[k] * s2 * zd[c];
                const float gw3 = warp_sum_f(a_i * silu(zz) + b_i * s1 * zd[c]);
                if ((t & 31) == 0) atomicAdd(&grads[GRAD_W3 + k], gw3);
            }
            img_store8(S.p2, t, 16 * q, MLP_H, pp);
            img_store8(S.p2, t, 16 * q + 8, MLP_H, pp + 8);
            img_store8(S.q2, t, 16 * q, MLP_H, qq);
            img_store8(S.q2, t, 16 * q + 8, MLP_H, qq + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {   // P1 = P2 W2^T -> [128, 192), Q1 = Q2 W2^T -> [192, 256)
#pragma unroll
            for (int s = 0; s < MLP_H / 16; ++s) {
                mma_bf16(tm + 128, smem_desc(S.p2 + s * 128, MLP_H), smem_desc(S.w2 + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
                mma_bf16(tm + 192, smem_desc(S.q2 + s * 128, MLP_H), smem_desc(S.w2 + s * 128, MLP_H),
                         mma_idesc(128, MLP_H), s > 0);
            }
            mma_commit(&S.bar);
        }
        // while the tensor cores work: dW2 += H1'^T P2 + H1^T Q2, db2 += sum Q2
        outer_acc(S.hd1, S.p2, S.h1, S.q2, MLP_H, half * 32, half * 32 + 32, col, grads + GRAD_W2);
        if (half == 0) {
            float acc = 0.0f;
            for (int r = 0; r < MLP_TILE; ++r) acc += __bfloat162float(S.q2[img_off(r, col, MLP_H)]);
            atomicAdd(&grads[GRAD_B2 + col], acc);
        }
        failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
        phase ^= 1;
        if (failed) break;
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], zd[16], pp[16], qq[16], p1[16], q1[16];
            tmem_ld16(tm + lb + 16 * q, z);
            tmem_ld16(tm + lb + 64 + 16 * q, zd);
            tmem_ld16(tm + lb + 128 + 16 * q, pp);
            tmem_ld16(tm + lb + 192 + 16 * q, qq);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const float zz = z[c] + S.b1[16 * q + c];
                const float s1 = dsilu(zz), s2 = d2silu(zz);
                p1[c] = pp[c] * s1;
                q1[c] = pp[c] * s2 * zd[c] + qq[c] * s1;
            }
            img_store8(S.hd1, t, 16 * q, MLP_H, p1);
            img_store8(S.hd1, t, 16 * q + 8, MLP_H, p1 + 8);
            img_store8(S.h1, t, 16 * q, MLP_H, q1);
            img_store8(S.h1, t, 16 * q + 8, MLP_H, q1 + 8);
        }
        __syncthreads();
        // dW1 += g'^T P1 + g^T Q1, db1 += sum Q1
        outer_acc(S.gd, S.hd1, S.g0, S.h1, MLP_D, half * 8, half * 8 + 8, col, grads + GRAD_W1);
        if (half == 0) {
            float acc = 0.0f;
            for (int r = 0; r < MLP_TILE; ++r) acc += __bfloat162float(S.h1[img_off(r, col, MLP_H)]);
            atomicAdd(&grads[GRAD_B1 + col], acc);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (failed && t == 0) atomicOr(status, SIM_STATUS_MLP_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" :: "r"(tm));
}

// Operand images and vectors from the FP32 master parameters (flat layout
// W1 [16][64], b1, W2 [64][64], b2, w3, b3).
__global__ void k_mlp_pack(const float* __restrict__ p, __nv_bfloat16* w1t, __nv_bfloat16* w2t, __nv_bfloat16* w2,
                           __nv_bfloat16* w1) {
    const float* W1 = p + GRAD_W1;
    const float* W2 = p + GRAD_W2;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < MLP_H * MLP_H; q += gridDim.x * blockDim.x) {
        const int k = q / MLP_H, n = q % MLP_H;        // W2[k][n]
        w2t[img_off(n, k, MLP_H)] = __float2bfloat16_rn(W2[q]);
        w2[img_off(k, n, MLP_H)] = __float2bfloat16_rn(W2[q]);
        if (q < MLP_D * MLP_H) {
            const int c = q / MLP_H, kk = q % MLP_H;   // W1[c][kk]
            w1t[img_off(kk, c, MLP_D)] = __float2bfloat16_rn(W1[q]);
            w1[img_off(c, kk, MLP_H)] = __float2bfloat16_rn(W1[q]);
        }
    }
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                           float* __restrict__ m2, int n, float lr, float beta1, float beta2, float eps, float c1,
                           float c2) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float a = fmaf(beta1, m1[q], (1.0f - beta1) * gq);
        const float b = fmaf(beta2, m2[q], (1.0f - beta2) * gq * gq);
        m1[q] = a;
        m2[q] = b;
        p[q] -= lr * (a * c1) / (sqrtf(b * c2) + eps);
    }
}

}  // namespace simb200

using namespace simb200;

static bool mlp_ok(const SimMLP* m) {
    return m && m->w1t_img && m->w2t_img && m->w2_img && m->w1_img && m->b1 && m->b2 && m->w3 && m->b3 && m->mu &&
           m->inv_sigma;
}

// Dynamic shared memory of the inference kernel, padded so that at most four
// blocks fit on an SM: four x 128 columns is all of its tensor memory, so a
// fifth block would wait in tcgen05.alloc.
static size_t mlp_fwd_smem() {
    static size_t bytes = 0;
    if (bytes == 0) {
        int dev = 0, smem_sm = 228 * 1024;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        const size_t pad = (size_t)smem_sm / 4 - 1024;
        bytes = pad > sizeof(MlpFwdSmem) ? pad : sizeof(MlpFwdSmem);
    }
    return bytes;
}

static void mlp_set_attributes() {
    static bool done = false;   // the first call happens before any stream capture
    if (done) return;
    cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_fwd_smem());
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
    cudaGetLastError();
    done = true;
}

// Resident blocks per SM of a tensor-memory kernel, from its registers, its
// shared memory and the 512 tensor-memory columns of an SM (the occupancy
// query does not count tensor memory, and answers one block for these
// kernels, so the limits are worked out here).
static int mlp_resident(const void* fn, size_t smem, int tmem_cols) {
    int dev = 0, smem_sm = 228 * 1024, regs_sm = 65536;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa;
    int by_regs = 1;
    if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess && fa.numRegs > 0) {
        const int per_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
        by_regs = regs_sm / (per_warp * (MLP_TILE / 32));
        smem += fa.sharedSizeBytes;
    }
    cudaGetLastError();
    const int by_smem = (int)((size_t)smem_sm / (smem + 1024));
    int per_sm = 512 / tmem_cols;
    if (by_regs < per_sm) per_sm = by_regs;
    if (by_smem < per_sm) per_sm = by_smem;
    return per_sm < 1 ? 1 : per_sm;
}

static int mlp_grid(const void* fn, int64_t n_tiles, size_t smem, int tmem_cols) {
    static const void* fns[4];
    static int cached[4], n_cached = 0;
    int per_sm = 0;
    for (int k = 0; k < n_cached; ++k)
        if (fns[k] == fn) per_sm = cached[k];
    if (per_sm == 0) {   // the first call happens before any stream capture
        per_sm = mlp_resident(fn, smem, tmem_cols);
        if (n_cached < 4) { fns[n_cached] = fn; cached[n_cached++] = per_sm; }
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t g = (int64_t)per_sm * sms;
    return (int)(n_tiles < g ? (n_tiles < 1 ? 1 : n_tiles) : g);
}

template <int GRP>
static void launch_mlp_desc(const SimEngine& e, float* G, cudaStream_t st) {
    const int64_t groups = (e.n + 128 / GRP - 1) / (128 / GRP);
    const int g = (int)(groups < 148 * 12 ? groups : 148 * 12);
    if (e.box_orthogonal) launch_pdl(k_mlp_desc<true, GRP>, dim3(g), dim3(128), 0, st, e, G);
    else launch_pdl(k_mlp_desc<false, GRP>, dim3(g), dim3(128), 0, st, e, G);
}

template <int GRP>
static void launch_mlp_force(const SimEngine& e, const float* dEdG, cudaStream_t st) {
    const int64_t groups = (e.n + 128 / GRP - 1) / (128 / GRP);
    const int g = (int)(groups < 148 * 12 ? groups : 148 * 12);
    if (e.box_orthogonal) k_mlp_force<true, GRP><<<g, 128, 0, st>>>(e, dEdG);
    else k_mlp_force<false, GRP><<<g, 128, 0, st>>>(e, dEdG);
}

// launch[2] / launch[3]: threads per atom of the descriptor / force kernel (4 or 8; 0: 4)
static bool mlp_group_ok(int g) { return g == 0 || g == 4 || g == 8; }

extern "C" int sim_mlp_descriptors(const SimEngine* e, float* G, void* stream) {
    if (!e || !G || e->n <= 0 || !mlp_group_ok(e->launch[2])) return SIM_ERR_ARG;
    if (e->launch[2] == 8) launch_mlp_desc<8>(*e, G, (cudaStream_t)stream);
    else launch_mlp_desc<4>(*e, G, (cudaStream_t)stream);
    return launch_status("sim_mlp_descriptors");
}

extern "C" int sim_mlp_backward(const SimEngine* e, const float* dEdG, void* stream) {
    if (!e || !dEdG || e->n <= 0 || !mlp_group_ok(e->launch[3])) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(e->f32, 0, sizeof(float) * 4 * e->n_pad, st);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_mlp_backward: zero forces"); return SIM_ERR_CUDA; }
    if (e->launch[3] == 8) launch_mlp_force<8>(*e, dEdG, st);
    else launch_mlp_force<4>(*e, dEdG, st);
    return launch_status("sim_mlp_backward");
}

extern "C" int sim_autotune_mlp(const SimEngine* e, const float* dEdG, float* G, int32_t reps, float* ms,
                                int32_t* best, void* stream) {
    if (!e || !dEdG || !G || !ms || !best || reps < 1 || e->n <= 0) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const SimEngine& en = *e;
    ms[0] = time_launches([&] { launch_mlp_desc<4>(en, G, st); }, reps, st);
    ms[1] = time_launches([&] { launch_mlp_desc<8>(en, G, st); }, reps, st);
    // the force pass accumulates; zeroed once per launch like sim_mlp_backward
    ms[2] = time_launches([&] {
        cudaMemsetAsync(en.f32, 0, sizeof(float) * 4 * en.n_pad, st);
        launch_mlp_force<4>(en, dEdG, st);
    }, reps, st);
    ms[3] = time_launches([&] {
        cudaMemsetAsync(en.f32, 0, sizeof(float) * 4 * en.n_pad, st);
        launch_mlp_force<8>(en, dEdG, st);
    }, reps, st);
    if (ms[0] < 0.f || ms[1] < 0.f || ms[2] < 0.f || ms[3] < 0.f) return SIM_ERR_CUDA;
    best[0] = ms[1] < ms[0] ? 8 : 4;
    best[1] = ms[3] < ms[2] ? 8 : 4;
    return launch_status("sim_autotune_mlp");
}

extern "C" int sim_eam_atom_energy(const SimEngine* e, const SimEAMTables* t, float* e_atom, void* stream) {
    if (!e || !t || !e_atom || e->n <= 0 || t->n_types != 1 || t->n_r < 2 || t->n_r >= kMaxTableRows || !t->dens_vd ||
        !t->pair_vd)
        return SIM_ERR_ARG;
    const int g = (int)((e->n + 255) / 256 < 148 * 8 ? (e->n + 255) / 256 : 148 * 8);
    k_eam_atom_energy<<<g, 256, 0, (cudaStream_t)stream>>>(*e, *t, e_atom);
    return launch_status("sim_eam_atom_energy");
}

extern "C" int sim_mlp_forward(const SimMLP* m, const float* G, int64_t n, float* e_atom, float* dEdG,
                               int32_t* status, void* stream) {
    if (!mlp_ok(m) || !G || n <= 0 || !e_atom || !dEdG || !status) return SIM_ERR_ARG;
    mlp_set_attributes();
    const size_t smem = mlp_fwd_smem();
    const int g = mlp_grid((const void*)k_mlp_fwd, (n + MLP_TILE - 1) / MLP_TILE, smem, 128);
    launch_pdl(k_mlp_fwd, dim3(g), dim3(MLP_TILE), smem, (cudaStream_t)stream, *m, G, n, e_atom, dEdG, status);
    return launch_status("sim_mlp_forward");
}

extern "C" int sim_mlp_train_grads(const SimMLP* m, const float* G, const float* target, int64_t n, float* grads,
                                   float* loss, int32_t* status, void* stream) {
    if (!mlp_ok(m) || !G || !target || n <= 0 || !grads || !loss || !status) return SIM_ERR_ARG;
    mlp_set_attributes();
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(grads, 0, sizeof(float) * SIM_MLP_PARAMS, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(loss, 0, sizeof(float), st);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_mlp_train_grads: zero"); return SIM_ERR_CUDA; }
    const int g = mlp_grid((const void*)k_mlp_train, (n + MLP_TILE - 1) / MLP_TILE, sizeof(MlpSmem), 128);
    k_mlp_train<<<g, MLP_TILE, sizeof(MlpSmem), st>>>(*m, G, n, target, 1.0f / (float)n, grads, loss, status);
    return launch_status("sim_mlp_train_grads");
}

extern "C" int sim_mlp_pack(const float* params, uint16_t* w1t_img, uint16_t* w2t_img, uint16_t* w2_img,
                            uint16_t* w1_img, void* stream) {
    if (!params || !w1t_img || !w2t_img || !w2_img || !w1_img) return SIM_ERR_ARG;
    k_mlp_pack<<<16, 256, 0, (cudaStream_t)stream>>>(params, reinterpret_cast<__nv_bfloat16*>(w1t_img),
                                                   reinterpret_cast<__nv_bfloat16*>(w2t_img),
                                                   reinterpret_cast<__nv_bfloat16*>(w2_img),
                                                   reinterpret_cast<__nv_bfloat16*>(w1_img));
    return launch_status("sim_mlp_pack");
}

extern "C" int sim_mlp_adam(float* params, const float* grads, float* m1, float* m2, float lr, int32_t step,
                            void* stream) {
    if (!params || !grads || !m1 || !m2 || step < 1) return SIM_ERR_ARG;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    k_mlp_adam<<<8, 256, 0, (cudaStream_t)stream>>>(params, grads, m1, m2, SIM_MLP_PARAMS, lr, b1, b2, 1e-8f, c1, c2);
    return launch_status("sim_mlp_adam");
}

extern "C" int sim_mlp_force_contract(const SimEngine* e, const float* ferr, float* u, void* stream) {
    if (!e || !ferr || !u || e->n <= 0) return SIM_ERR_ARG;
    const int g = (int)((e->n + 127) / 128 < 148 * 16 ? (e->n + 127) / 128 : 148 * 16);
    if (e->box_orthogonal) k_mlp_ucontract<true><<<g, 128, 0, (cudaStream_t)stream>>>(*e, ferr, u);
    else k_mlp_ucontract<false><<<g, 128, 0, (cudaStream_t)stream>>>(*e, ferr, u);
    return launch_status("sim_mlp_force_contract");
}

extern "C" int sim_mlp_train_grads_fm(const SimMLP* m, const float* G, const float* target, const float* u,
                                      int64_t n, float w_energy, float w_force, int64_t n_force_atoms, float* grads,
                                      float* loss, int32_t* status, void* stream) {
    if (!mlp_ok(m) || !G || !target || !u || n <= 0 || n_force_atoms <= 0 || !grads || !loss || !status)
        return SIM_ERR_ARG;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_mlp_train_fm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpFmSmem));
        cudaGetLastError();
        attr = true;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(grads, 0, sizeof(float) * SIM_MLP_PARAMS, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(loss, 0, sizeof(float), st);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_mlp_train_grads_fm: zero"); return SIM_ERR_CUDA; }
    const int g = mlp_grid((const void*)k_mlp_train_fm, (n + MLP_TILE - 1) / MLP_TILE, sizeof(MlpFmSmem), 256);
    const float alpha = 2.0f * w_energy / (float)n;
    const float beta = -2.0f * w_force / (3.0f * (float)n_force_atoms);
    k_mlp_train_fm<<<g, MLP_TILE, sizeof(MlpFmSmem), st>>>(*m, G, target, u, n, alpha, beta, 1.0f / (float)n, grads,
                                                           loss, status);
    return launch_status("sim_mlp_train_grads_fm");
}

extern "C" int sim_mlp_train_step(const SimMLP* m, float* params, uint16_t* w1t_img, uint16_t* w2t_img,
                                  uint16_t* w2_img, uint16_t* w1_img, const float* G, const float* target,
                                  const float* u, int64_t n, float w_energy, float w_force, int64_t n_force_atoms,
                                  float* grads, float* adam_m, float* adam_v, float lr, int32_t step, float* loss,
                                  int32_t* status, void* stream) {
    if (!params || !adam_m || !adam_v || step < 1) return SIM_ERR_ARG;
    int rc = u ? sim_mlp_train_grads_fm(m, G, target, u, n, w_energy, w_force, n_force_atoms, grads, loss, status,
                                        stream)
               : sim_mlp_train_grads(m, G, target, n, grads, loss, status, stream);
    if (rc == SIM_OK) rc = sim_mlp_adam(params, grads, adam_m, adam_v, lr, step, stream);
    if (rc == SIM_OK) rc = sim_mlp_pack(params, w1t_img, w2t_img, w2_img, w1_img, stream);
    return rc;
}

