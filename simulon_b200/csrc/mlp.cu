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

// In-cutoff neighbours of slot i as {d, r}; returns the count (capped).
template <bool ORTHO>
__device__ __forceinline__ int mlp_neighbours(const SimEngine& e, const BoxF& b, int64_t i, float4* nb, bool& over) {
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int4 qi = posq[i];
    const int nn = e.nnbr[i];
    int cnt = 0;
    for (int k = 0; k < nn; ++k) {
        const int4 qj = __ldg(&posq[__ldg(&e.nbr[(int64_t)k * e.n_pad + i])]);
        float d0, d1, d2;
        mlp_dvec<ORTHO>(b, qi, qj, d0, d1, d2);
        const float r2 = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
        if (!(r2 < MLP_RC * MLP_RC)) continue;
        if (cnt == MLP_MAXN) { over = true; continue; }
        nb[cnt++] = make_float4(d0, d1, d2, sqrtf(r2));
    }
    return cnt;
}

template <bool ORTHO>
__global__ void __launch_bounds__(128) k_mlp_desc(SimEngine e, float* __restrict__ G) {
    const BoxF b(*e.box);
    bool over = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 nb[MLP_MAXN];
        float ea[MLP_MAXN];
        const int cnt = mlp_neighbours<ORTHO>(e, b, i, nb, over);
        float g[MLP_D];
#pragma unroll
        for (int k = 0; k < MLP_D; ++k) g[k] = 0.0f;
        for (int a = 0; a < cnt; ++a) {
            const float r = nb[a].w, fc = mlp_fc(r);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float t = r - mlp_rs(k);
                g[k] = fmaf(__expf(-4.0f * t * t), fc, g[k]);
            }
            ea[a] = __expf(-0.01f * r * r) * fc;
        }
        for (int a = 0; a < cnt; ++a) {
            const float4 da = nb[a];
            for (int c = a + 1; c < cnt; ++c) {
                const float4 dc = nb[c];
                const float cs = (da.x * dc.x + da.y * dc.y + da.z * dc.z) / (da.w * dc.w);
                const float rad = ea[a] * ea[c];
                const float p1 = 1.0f + cs, m1 = 1.0f - cs;
                const float p2 = p1 * p1, m2 = m1 * m1, p4 = p2 * p2, m4 = m2 * m2, p8 = p4 * p4, m8 = m4 * m4;
                g[8] = fmaf(p1, rad, g[8]);
                g[9] = fmaf(m1, rad, g[9]);
                g[10] = fmaf(0.5f * p2, rad, g[10]);
                g[11] = fmaf(0.5f * m2, rad, g[11]);
                g[12] = fmaf(0.125f * p4, rad, g[12]);
                g[13] = fmaf(0.125f * m4, rad, g[13]);
                g[14] = fmaf(0.0078125f * p8, rad, g[14]);
                g[15] = fmaf(0.0078125f * m8, rad, g[15]);
            }
        }
        float4* out = reinterpret_cast<float4*>(G + i * MLP_D);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
    }
    if (over) atomicOr(&e.flags[1], SIM_STATUS_MLP_NEIGHBORS);
}

// Forces from dE/dG (already including the 1/sigma of the normalisation):
// each centre i accumulates dE_i/dd_j for its in-cutoff neighbours j and adds
// -dE_i/dd_j to atom j and +sum_j dE_i/dd_j to itself (float atomics: the
// summation order, and so the last bits, vary from run to run).
template <bool ORTHO>
__global__ void __launch_bounds__(128) k_mlp_force(SimEngine e, const float* __restrict__ dEdG) {
    const BoxF b(*e.box);
    float* f = e.f32;
    bool over = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 nb[MLP_MAXN];
        float gx[MLP_MAXN], gy[MLP_MAXN], gz[MLP_MAXN], ea[MLP_MAXN], eda[MLP_MAXN];
        const int cnt = mlp_neighbours<ORTHO>(e, b, i, nb, over);
        float g[MLP_D];
        const float4* gin = reinterpret_cast<const float4*>(dEdG + i * MLP_D);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 v = gin[q];
            g[4 * q] = v.x; g[4 * q + 1] = v.y; g[4 * q + 2] = v.z; g[4 * q + 3] = v.w;
        }
        for (int a = 0; a < cnt; ++a) {
            const float r = nb[a].w, fc = mlp_fc(r), dfc = mlp_dfc(r);
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float t = r - mlp_rs(k);
                const float ex = __expf(-4.0f * t * t);
                s = fmaf(g[k], ex * fmaf(-8.0f * t, fc, dfc), s);
            }
            const float ir = 1.0f / r;
            gx[a] = s * nb[a].x * ir; gy[a] = s * nb[a].y * ir; gz[a] = s * nb[a].z * ir;
            const float ex = __expf(-0.01f * r * r);
            ea[a] = ex * fc;
            eda[a] = ex * fmaf(-0.02f * r, fc, dfc);     // d e / d r
        }
        for (int a = 0; a < cnt; ++a) {
            const float4 da = nb[a];
            const float ira = 1.0f / da.w;
            for (int c = a + 1; c < cnt; ++c) {
                const float4 dc = nb[c];
                const float irc = 1.0f / dc.w;
                const float cs = (da.x * dc.x + da.y * dc.y + da.z * dc.z) * ira * irc;
                const float p1 = 1.0f + cs, m1 = 1.0f - cs;
                const float p2 = p1 * p1, m2 = m1 * m1, p4 = p2 * p2, m4 = m2 * m2;
                const float p3 = p2 * p1, m3 = m2 * m1, p7 = p4 * p3, m7 = m4 * m3, p8 = p4 * p4, m8 = m4 * m4;
                // S_A = sum_l g_l 2^(1-z) (1 + l c)^z ; S_dA = sum_l g_l 2^(1-z) z l (1 + l c)^(z-1)
                const float SA = g[8] * p1 + g[9] * m1 + 0.5f * (g[10] * p2 + g[11] * m2) +
                                 0.125f * (g[12] * p4 + g[13] * m4) + 0.0078125f * (g[14] * p8 + g[15] * m8);
                const float SdA = (g[8] - g[9]) + (g[10] * p1 - g[11] * m1) + 0.5f * (g[12] * p3 - g[13] * m3) +
                                  0.0625f * (g[14] * p7 - g[15] * m7);
                const float rad = ea[a] * ea[c];
                // dc/dd_a = d_c/(r_a r_c) - c d_a / r_a^2 (and a <-> c)
                const float wc = SdA * rad * ira * irc;
                const float ka = SdA * rad * cs * ira * ira - SA * eda[a] * ea[c] * ira;
                const float kc = SdA * rad * cs * irc * irc - SA * ea[a] * eda[c] * irc;
                gx[a] += wc * dc.x - ka * da.x; gy[a] += wc * dc.y - ka * da.y; gz[a] += wc * dc.z - ka * da.z;
                gx[c] += wc * da.x - kc * dc.x; gy[c] += wc * da.y - kc * dc.y; gz[c] += wc * da.z - kc * dc.z;
            }
        }
        // gx[a] = dE_i / dd_a; the neighbour's slot is needed again: walk the list once more
        const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
        const int4 qi = posq[i];
        const int nn = e.nnbr[i];
        float sx = 0.f, sy = 0.f, sz = 0.f;
        int a = 0;
        for (int k = 0; k < nn && a < cnt; ++k) {
            const int j = __ldg(&e.nbr[(int64_t)k * e.n_pad + i]);
            const int4 qj = __ldg(&posq[j]);
            float d0, d1, d2;
            mlp_dvec<ORTHO>(b, qi, qj, d0, d1, d2);
            if (!(fmaf(d2, d2, fmaf(d1, d1, d0 * d0)) < MLP_RC * MLP_RC)) continue;
            atomicAdd(&f[4 * j], -gx[a]);
            atomicAdd(&f[4 * j + 1], -gy[a]);
            atomicAdd(&f[4 * j + 2], -gz[a]);
            sx += gx[a]; sy += gy[a]; sz += gz[a];
            ++a;
        }
        atomicAdd(&f[4 * i], sx);
        atomicAdd(&f[4 * i + 1], sy);
        atomicAdd(&f[4 * i + 2], sz);
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
            const int4 qj = __ldg(&posq[__ldg(&e.nbr[(int64_t)k * e.n_pad + i])]);
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

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
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

// TRAIN = false: E_i and dE/dG (scaled by 1/sigma) per atom.
// TRAIN = true : per-atom loss (E_i - target_i)^2 / n_batch, its gradient
//                with respect to every weight (added to grads with atomics)
//                and the loss sum (added to *loss).
template <bool TRAIN>
__global__ void __launch_bounds__(MLP_TILE) k_mlp_net(SimMLP m, const float* __restrict__ G, int64_t n,
                                                      float* __restrict__ e_atom, float* __restrict__ dEdG,
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
                if (TRAIN) img_store8(S.a3, t, k0, MLP_H, h);
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
        // dL/dE: 1 for forces, 2 (E - target) / n_batch while training
        float up = 1.0f;
        if (TRAIN) {
            const float err = live ? E - target[i] : 0.0f;
            up = 2.0f * err * inv_batch;
            const float l = live ? err * err * inv_batch : 0.0f;
            const float ls = warp_sum_f(l);
            if ((t & 31) == 0) atomicAdd(loss, ls);
        } else if (live) {
            e_atom[i] = E;
        }
        if (!live) up = 0.0f;
        {
            float d[8];
#pragma unroll
            for (int k0 = 0; k0 < MLP_H; k0 += 8) {
#pragma unroll
                for (int q = 0; q < 8; ++q) d[q] = up * S.w3[k0 + q] * dsilu(z2[k0 + q] + S.b2[k0 + q]);
                img_store8(TRAIN ? S.a2 : S.a1, t, k0, MLP_H, d);
            }
            if (TRAIN) {
                // output layer: dw3 = sum up * h2, db3 = sum up
#pragma unroll 4
                for (int k = 0; k < MLP_H; ++k) {
                    const float v = warp_sum_f(up * silu(z2[k] + S.b2[k]));
                    if ((t & 31) == 0) atomicAdd(&grads[GRAD_W3 + k], v);
                }
                const float v = warp_sum_f(up);
                if ((t & 31) == 0) atomicAdd(&grads[GRAD_B3], v);
            }
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // D1 = dZ2 W2^T -> tmem columns [64, 128)
        const __nv_bfloat16* dz2 = TRAIN ? S.a2 : S.a1;
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
        if (TRAIN) {
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
        } else {
            float dk[8];
#pragma unroll
            for (int k0 = 0; k0 < MLP_H; k0 += 8) {
#pragma unroll
                for (int q = 0; q < 8; ++q) dk[q] = d1[k0 + q];
                img_store8(S.a2, t, k0, MLP_H, dk);
            }
            async_proxy_fence();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            // dG = dZ1 W1^T -> tmem columns [64, 80)
            if (t == 0) {
#pragma unroll
                for (int s = 0; s < MLP_H / 16; ++s)
                    mma_bf16(tm + 64, smem_desc(S.a2 + s * 2 * 64, MLP_H), smem_desc(S.w1 + s * 2 * 64, MLP_H),
                             mma_idesc(128, MLP_D), s > 0);
                mma_commit(&S.bar);
            }
            failed = __syncthreads_or(!mbar_wait(&S.bar, phase));
            phase ^= 1;
            if (failed) break;
            tc_fence_after();
            float gv[MLP_D];
            tmem_ld16(tm + lane_base + 64, gv);
            tmem_wait_ld();
            if (live) {
                float4* out = reinterpret_cast<float4*>(dEdG + i * MLP_D);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    out[q] = make_float4(gv[4 * q] * S.isg[4 * q], gv[4 * q + 1] * S.isg[4 * q + 1],
                                         gv[4 * q + 2] * S.isg[4 * q + 2], gv[4 * q + 3] * S.isg[4 * q + 3]);
            }
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
            const int j = __ldg(&e.nbr[(int64_t)k * e.n_pad + i]);
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

static void mlp_set_attributes() {
    static bool done = false;   // the first call happens before any stream capture
    if (done) return;
    cudaFuncSetAttribute(k_mlp_net<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
    cudaFuncSetAttribute(k_mlp_net<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
    cudaGetLastError();
    done = true;
}

static int mlp_grid(const void* fn, int64_t n_tiles) {
    // every resident block holds 128 tensor-memory columns: never more than 4 per SM
    int per_sm = 0, dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, MLP_TILE, sizeof(MlpSmem)) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    const int64_t g = (int64_t)per_sm * sms;
    return (int)(n_tiles < g ? (n_tiles < 1 ? 1 : n_tiles) : g);
}

extern "C" int sim_mlp_descriptors(const SimEngine* e, float* G, void* stream) {
    if (!e || !G || e->n <= 0) return SIM_ERR_ARG;
    const int g = (int)((e->n + 127) / 128 < 148 * 16 ? (e->n + 127) / 128 : 148 * 16);
    if (e->box_orthogonal) k_mlp_desc<true><<<g, 128, 0, (cudaStream_t)stream>>>(*e, G);
    else k_mlp_desc<false><<<g, 128, 0, (cudaStream_t)stream>>>(*e, G);
    return launch_status("sim_mlp_descriptors");
}

extern "C" int sim_mlp_forces(const SimEngine* e, const float* dEdG, void* stream) {
    if (!e || !dEdG || e->n <= 0) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(e->f32, 0, sizeof(float) * 4 * e->n_pad, st);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_mlp_forces: zero forces"); return SIM_ERR_CUDA; }
    const int g = (int)((e->n + 127) / 128 < 148 * 16 ? (e->n + 127) / 128 : 148 * 16);
    if (e->box_orthogonal) k_mlp_force<true><<<g, 128, 0, st>>>(*e, dEdG);
    else k_mlp_force<false><<<g, 128, 0, st>>>(*e, dEdG);
    return launch_status("sim_mlp_forces");
}

extern "C" int sim_eam_atom_energy(const SimEngine* e, const SimEAMTables* t, float* e_atom, void* stream) {
    if (!e || !t || !e_atom || e->n <= 0 || t->n_types != 1 || !t->dens_vd || !t->pair_vd) return SIM_ERR_ARG;
    const int g = (int)((e->n + 255) / 256 < 148 * 8 ? (e->n + 255) / 256 : 148 * 8);
    k_eam_atom_energy<<<g, 256, 0, (cudaStream_t)stream>>>(*e, *t, e_atom);
    return launch_status("sim_eam_atom_energy");
}

extern "C" int sim_mlp_forward(const SimMLP* m, const float* G, int64_t n, float* e_atom, float* dEdG,
                               int32_t* status, void* stream) {
    if (!mlp_ok(m) || !G || n <= 0 || !e_atom || !dEdG || !status) return SIM_ERR_ARG;
    mlp_set_attributes();
    const int g = mlp_grid((const void*)k_mlp_net<false>, (n + MLP_TILE - 1) / MLP_TILE);
    k_mlp_net<false><<<g, MLP_TILE, sizeof(MlpSmem), (cudaStream_t)stream>>>(*m, G, n, e_atom, dEdG, nullptr, 0.0f,
                                                                            nullptr, nullptr, status);
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
    const int g = mlp_grid((const void*)k_mlp_net<true>, (n + MLP_TILE - 1) / MLP_TILE);
    k_mlp_net<true><<<g, MLP_TILE, sizeof(MlpSmem), st>>>(*m, G, n, nullptr, nullptr, target, 1.0f / (float)n, grads,
                                                         loss, status);
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
    // every resident block holds 256 tensor-memory columns: at most 2 per SM
    int per_sm = 0, dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_train_fm, MLP_TILE, sizeof(MlpFmSmem)) !=
            cudaSuccess || per_sm < 1)
        per_sm = 1;
    if (per_sm > 2) per_sm = 2;
    const int64_t tiles = (n + MLP_TILE - 1) / MLP_TILE;
    const int g = (int)(tiles < (int64_t)per_sm * sms ? tiles : (int64_t)per_sm * sms);
    const float alpha = 2.0f * w_energy / (float)n;
    const float beta = -2.0f * w_force / (3.0f * (float)n_force_atoms);
    k_mlp_train_fm<<<g, MLP_TILE, sizeof(MlpFmSmem), st>>>(*m, G, target, u, n, alpha, beta, 1.0f / (float)n, grads,
                                                           loss, status);
    return launch_status("sim_mlp_train_grads_fm");
}

