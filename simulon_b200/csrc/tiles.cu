// Neighbour tiles in shared memory (sm_100a).
//
// A tile is SIM_TILE consecutive slots.  Because slots are in cell (Morton)
// order a tile is a compact region of space, and the set of out-of-tile
// atoms its atoms interact with -- the tile's halo -- is small (about 1.5-2.5x
// the tile for BCC W at rc + skin = 4.9 A).  At every list rebuild each
// tile's halo is collected (hash set in shared memory), sorted (so that its
// slots form long consecutive runs and load coalesced) and the full list is
// rewritten with 16-bit tile-local indices: idx < SIM_TILE is own slot
// tile*SIM_TILE + idx, otherwise halo[idx - SIM_TILE].
//
// The tiled EAM passes run one 1024-thread block per SM.  A block walks its
// tiles with a grid stride; the 16-byte records of the next tile (own + halo)
// are copied into shared memory with cp.async while the current tile is
// processed (double buffering), so the neighbour loop reads only shared
// memory and the coalesced 16-bit list.
#include "common.cuh"

namespace simb200 {

#define HASH_SLOTS 8192         // hash set for halo collection (power of two)
#define HALO_SORT_MAX 4096      // the halo is sorted in shared memory; halo_cap <= this

__device__ __forceinline__ uint32_t hash_slot(int32_t j) { return ((uint32_t)j * 2654435761u) & (HASH_SLOTS - 1); }

// ---------------------------------------------------------------------------
// halo construction (after the ELL list is built)
__global__ void __launch_bounds__(SIM_TILE) k_build_halo(SimEngine e, const int32_t* gate) {
    if (gate && __ldg(gate) == 0) return;
    extern __shared__ int32_t halo_smem[];        // HASH_SLOTS + HALO_SORT_MAX ints
    int32_t* hset = halo_smem;
    int32_t* hsort = halo_smem + HASH_SLOTS;
    __shared__ int32_t s_n, s_bad;
    const int64_t P = e.n_pad;
    const int cap = e.halo_cap < HALO_SORT_MAX ? e.halo_cap : HALO_SORT_MAX;
    for (int tile = blockIdx.x; tile < e.n_tiles; tile += gridDim.x) {
        for (int s = threadIdx.x; s < HASH_SLOTS; s += blockDim.x) hset[s] = 0;
        if (threadIdx.x == 0) { s_n = 0; s_bad = 0; }
        __syncthreads();
        const int64_t t0 = (int64_t)tile * SIM_TILE;
        const int64_t t1 = t0 + SIM_TILE < e.n ? t0 + SIM_TILE : e.n;
        const int64_t i = t0 + threadIdx.x;
        const int nn = i < t1 ? e.nnbr[i] : 0;
        // 1. insert out-of-tile neighbours (linear probing, at most HASH_SLOTS probes)
        for (int k = 0; k < nn; ++k) {
            const int32_t j = e.nbr[(int64_t)k * P + i];
            if (j >= t0 && j < t1) continue;
            uint32_t h = hash_slot(j);
            int probe = 0;
            for (; probe < HASH_SLOTS; ++probe) {
                const int32_t prev = atomicCAS(&hset[h], 0, j + 1);
                if (prev == 0 || prev == j + 1) break;
                h = (h + 1) & (HASH_SLOTS - 1);
            }
            if (probe == HASH_SLOTS) s_bad = 1;
        }
        __syncthreads();
        // 2. compact the set
        for (int s = threadIdx.x; s < HASH_SLOTS; s += blockDim.x) {
            const int32_t v = hset[s];
            if (v != 0) {
                const int p = atomicAdd(&s_n, 1);
                if (p < HALO_SORT_MAX) hsort[p] = v - 1;
            }
        }
        __syncthreads();
        const int n_unique = s_n;
        const int H = n_unique < cap ? n_unique : cap;
        if (threadIdx.x == 0 && (n_unique > cap || s_bad)) {
            atomicOr(&e.flags[1], SIM_STATUS_HALO);
            atomicMax(&e.flags[4], s_bad ? HASH_SLOTS : n_unique);
        }
        // 3. bitonic sort of hsort[0, Hp)
        int Hp = 1;
        while (Hp < H) Hp <<= 1;
        for (int s = H + threadIdx.x; s < Hp; s += blockDim.x) hsort[s] = 0x7fffffff;
        __syncthreads();
        for (int size = 2; size <= Hp; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int idx = threadIdx.x; idx < (Hp >> 1); idx += blockDim.x) {
                    const int lo = 2 * stride * (idx / stride) + (idx % stride);
                    const int hi = lo + stride;
                    const bool asc = (lo & size) == 0;
                    const int32_t a = hsort[lo], b = hsort[hi];
                    if ((a > b) == asc) { hsort[lo] = b; hsort[hi] = a; }
                }
                __syncthreads();
            }
        }
        // 4. publish the halo and rewrite the row with tile-local indices
        for (int s = threadIdx.x; s < H; s += blockDim.x) e.halo[(int64_t)tile * e.halo_cap + s] = hsort[s];
        if (threadIdx.x == 0) e.halo_n[tile] = H;
        for (int k = 0; k < nn; ++k) {
            const int32_t j = e.nbr[(int64_t)k * P + i];
            int local;
            if (j >= t0 && j < t1) {
                local = (int)(j - t0);
            } else {
                int lo = 0, hi = H;                 // lower_bound(hsort, H, j)
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (hsort[mid] < j) lo = mid + 1; else hi = mid;
                }
                local = SIM_TILE + (lo < H ? lo : 0);   // a missing entry only under SIM_STATUS_HALO
            }
            e.nbr16[(int64_t)k * P + i] = (uint16_t)local;
        }
        __syncthreads();
    }
}

void launch_build_halo(const SimEngine& e, const int32_t* gate, cudaStream_t st) {
    if (!e.nbr16 || !e.halo || !e.halo_n || e.n_tiles <= 0) return;
    static bool attr = false;   // first set during the engine load, outside any capture
    const size_t smem = (HASH_SLOTS + HALO_SORT_MAX) * sizeof(int32_t);
    if (!attr) {
        cudaFuncSetAttribute(k_build_halo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int g = e.n_tiles < 148 * 2 ? e.n_tiles : 148 * 2;
    k_build_halo<<<g, SIM_TILE, smem, st>>>(e, gate);
}

// ---------------------------------------------------------------------------
// staging helpers
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Issue the copies of tile `tile`'s own and halo records (16 bytes each) into buf.
__device__ __forceinline__ void load_tile(const SimEngine& e, const int4* __restrict__ src, int tile, int4* buf) {
    const int64_t t0 = (int64_t)tile * SIM_TILE;
    const int own = (int)(e.n - t0 < SIM_TILE ? e.n - t0 : SIM_TILE);
    const int H = __ldg(&e.halo_n[tile]);
    const int32_t* halo = e.halo + (int64_t)tile * e.halo_cap;
    for (int s = threadIdx.x; s < own; s += blockDim.x) cp_async16(&buf[s], &src[t0 + s]);
    for (int s = threadIdx.x; s < H; s += blockDim.x) cp_async16(&buf[SIM_TILE + s], &src[__ldg(&halo[s])]);
}

struct TileWindow {
    int k_lo, n_win;
};

__device__ __forceinline__ float rsqrt_fast(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

struct BoxS {
    float h[9];
    __device__ __forceinline__ explicit BoxS(const SimBox& b) {
#pragma unroll
        for (int k = 0; k < 9; ++k) h[k] = b.Hf[k] * 2.3283064365386963e-10f;
    }
};
template <bool ORTHO>
__device__ __forceinline__ float pair_d2(const BoxS& b, const int4& qi, const int4& qj, float& r0, float& r1,
                                         float& r2) {
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
    return fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
}

// ---------------------------------------------------------------------------
// tiled pass 1 (one element type; the density table window is float2 {f_k, df_k})
template <bool ORTHO>
__global__ void __launch_bounds__(SIM_TILE, 1) k_eam_density_tiled(SimEngine e, SimEAMTables t, TileWindow w) {
    extern __shared__ __align__(16) unsigned char smem[];
    int4* buf0 = reinterpret_cast<int4*>(smem);
    int4* buf1 = buf0 + SIM_TILE + e.halo_cap;
    float2* tab = reinterpret_cast<float2*>(buf1 + SIM_TILE + e.halo_cap);
    {
        const float2* g = reinterpret_cast<const float2*>(t.dens_vd) + w.k_lo;
        for (int k = threadIdx.x; k < w.n_win; k += blockDim.x) tab[k] = __ldg(&g[k]);
    }
    const float2* gtab = reinterpret_cast<const float2*>(t.dens_vd);
    const BoxS b(*e.box);
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    int4* __restrict__ posfp = reinterpret_cast<int4*>(e.posfp);
    const uint16_t* __restrict__ nbr = e.nbr16;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    double acc = 0.0;
    int tile = blockIdx.x;
    if (tile < e.n_tiles) load_tile(e, posq, tile, buf0);
    cp_async_commit();
    for (int parity = 0; tile < e.n_tiles; tile += gridDim.x, parity ^= 1) {
        int4* cur = parity ? buf1 : buf0;
        const int next = tile + gridDim.x;
        if (next < e.n_tiles) load_tile(e, posq, next, parity ? buf0 : buf1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int64_t i = (int64_t)tile * SIM_TILE + threadIdx.x;
        if (i < e.n) {
            const int4 qi = cur[threadIdx.x];
            const int nn = e.nnbr[i];
            float rho = 0.0f;
            int kn = nn > 0 ? __ldg(&nbr[i]) : 0;
            for (int k = 0; k < nn; ++k) {
                const int local = kn;
                if (k + 1 < nn) kn = __ldg(&nbr[(int64_t)(k + 1) * P + i]);
                const int4 qj = cur[local];
                float r0, r1, r2;
                const float d2 = pair_d2<ORTHO>(b, qi, qj, r0, r1, r2);
                if (d2 < rc2) {
                    const float idx_f = fminf(d2 * rsqrt_fast(d2), t.r_clamp_hi) * t.inv_dr;
                    const int kr = (int)idx_f;
                    const float2 v = kr >= w.k_lo ? tab[kr - w.k_lo] : __ldg(&gtab[kr]);
                    rho += fmaf(idx_f - (float)kr, v.y, v.x);
                }
            }
            const float lo = t.rho_min[0];
            const float rcl = fminf(fmaxf(rho, lo), t.rho_clamp_hi[0]);
            const float ix = (rcl - lo) * t.inv_drho[0];
            const int m = (int)ix;
            const int m1 = min(m + 1, t.n_rho - 1);
            const float fr = ix - (float)m;
            const float F = fmaf(fr, t.embed[m1] - t.embed[m], t.embed[m]);
            const float Fp = fmaf(fr, t.embed_deriv[m1] - t.embed_deriv[m], t.embed_deriv[m]);
            posfp[i] = make_int4(qi.x, qi.y, qi.z, __float_as_int(Fp));
            acc += (double)F;
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    double vals[1] = {acc};
    block_partials<1>(vals, e.partials, SIM_RED_EPOT_EMBED);
    last_block_finalize<1>(e.partials, e.red_counter + 0, e.red_out, SIM_RED_EPOT_EMBED);
}

// ---------------------------------------------------------------------------
// tiled pass 2 (one element type).  The r-table window holds float4
// {f'_k, phi'_k, phi_k, 0} for k in [k_lo, n_r] (the last row repeated), and
// the interpolation reads rows k and k+1.
template <bool INTEG, bool ORTHO>
__global__ void __launch_bounds__(SIM_TILE, 1) k_eam_force_tiled(SimEngine e, SimEAMTables t, SimIntegrator ip,
                                                                 TileWindow w) {
    extern __shared__ __align__(16) unsigned char smem[];
    int4* buf0 = reinterpret_cast<int4*>(smem);
    int4* buf1 = buf0 + SIM_TILE + e.halo_cap;
    float4* tab = reinterpret_cast<float4*>(buf1 + SIM_TILE + e.halo_cap);
    {
        const float4* gd = reinterpret_cast<const float4*>(t.deriv_vd);
        const float2* gp = reinterpret_cast<const float2*>(t.pair_vd);
        for (int k = threadIdx.x; k <= w.n_win; k += blockDim.x) {
            const int r = min(w.k_lo + k, t.n_r - 1);
            const float4 d = __ldg(&gd[r]);
            tab[k] = make_float4(d.x, d.y, __ldg(&gp[r]).x, 0.f);
        }
    }
    const float4* gd = reinterpret_cast<const float4*>(t.deriv_vd);
    const float2* gp = reinterpret_cast<const float2*>(t.pair_vd);
    const BoxS b(*e.box);
    const int4* __restrict__ posfp = reinterpret_cast<const int4*>(e.posfp);
    const uint16_t* __restrict__ nbr = e.nbr16;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    float acc[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    const uint64_t step = INTEG && ip.step_ctr ? *ip.step_ctr : 0;
    int tile = blockIdx.x;
    if (tile < e.n_tiles) load_tile(e, posfp, tile, buf0);
    cp_async_commit();
    for (int parity = 0; tile < e.n_tiles; tile += gridDim.x, parity ^= 1) {
        int4* cur = parity ? buf1 : buf0;
        const int next = tile + gridDim.x;
        if (next < e.n_tiles) load_tile(e, posfp, next, parity ? buf0 : buf1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int64_t i = (int64_t)tile * SIM_TILE + threadIdx.x;
        if (i < e.n) {
            const int4 pi = cur[threadIdx.x];
            const float fpi = __int_as_float(pi.w);
            const int nn = e.nnbr[i];
            float fx = 0.f, fy = 0.f, fz = 0.f;
            int kn = nn > 0 ? __ldg(&nbr[i]) : 0;
            for (int k = 0; k < nn; ++k) {
                const int local = kn;
                if (k + 1 < nn) kn = __ldg(&nbr[(int64_t)(k + 1) * P + i]);
                const int4 qj = cur[local];
                float r0, r1, r2;
                const float d2 = pair_d2<ORTHO>(b, pi, qj, r0, r1, r2);
                if (!(d2 < rc2)) continue;
                const float inv_r = rsqrt_fast(d2);
                const float r = d2 * inv_r;
                const float idx_f = fminf(r, t.r_clamp_hi) * t.inv_dr;
                const int kr = (int)idx_f;
                const float frac = idx_f - (float)kr;
                float dd, dphi, phi;
                if (kr >= w.k_lo) {
                    const float4 v0 = tab[kr - w.k_lo], v1 = tab[kr - w.k_lo + 1];
                    const float2 a = __ffma2_rn(make_float2(frac, frac), make_float2(v1.x - v0.x, v1.y - v0.y),
                                                make_float2(v0.x, v0.y));
                    dd = a.x;
                    dphi = a.y;
                    phi = fmaf(frac, v1.z - v0.z, v0.z);
                } else {
                    const float4 d = __ldg(&gd[kr]);
                    const float2 p = __ldg(&gp[kr]);
                    dd = fmaf(frac, d.z, d.x);
                    dphi = fmaf(frac, d.w, d.y);
                    phi = fmaf(frac, p.y, p.x);
                }
                const float s = fmaf(fpi + __int_as_float(qj.w), dd, dphi);
                const float c = -s * inv_r;
                const float ax = c * r0, ay = c * r1, az = c * r2;
                fx += ax; fy += ay; fz += az;
                acc[0] += phi;
                acc[2] = fmaf(ax, r0, acc[2]); acc[3] = fmaf(ay, r1, acc[3]); acc[4] = fmaf(az, r2, acc[4]);
                acc[5] = fmaf(ax, r1, acc[5]); acc[6] = fmaf(ax, r2, acc[6]); acc[7] = fmaf(ay, r2, acc[7]);
            }
            reinterpret_cast<float4*>(e.f32)[i] = make_float4(fx, fy, fz, 0.0f);
            bad |= !(isfinite(fx) && isfinite(fy) && isfinite(fz));
            if (INTEG) {
                double v[3];
                second_half_atom(e, ip, i, 0, step, (double)fx, (double)fy, (double)fz, v, bad);
                const double m = e.mass[0];
                acc[8] += (float)(0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
                acc[9] += (float)(m * v[0] * v[0]); acc[10] += (float)(m * v[1] * v[1]); acc[11] += (float)(m * v[2] * v[2]);
                acc[12] += (float)(m * v[0] * v[1]); acc[13] += (float)(m * v[0] * v[2]); acc[14] += (float)(m * v[1] * v[2]);
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    acc[1] = -(acc[2] + acc[3] + acc[4]);   // scalar virial s r = minus the tensor's trace
    if (INTEG) {
        double vals[15];
#pragma unroll
        for (int k = 0; k < 15; ++k) vals[k] = k < 8 ? 0.5 * (double)acc[k] : (double)acc[k];
        block_partials<15>(vals, e.partials, SIM_RED_EPOT_PAIR);
        last_block_finalize<15>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
    } else {
        double vals[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) vals[k] = 0.5 * (double)acc[k];
        block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
        last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
    }
}

static const int kTileWindowRows = 4096;
static size_t kTileSmemLimit = 227 * 1024;

static TileWindow tile_window(const SimEAMTables& t) {
    const int n_win = t.n_r < kTileWindowRows ? t.n_r : kTileWindowRows;
    return TileWindow{t.n_r - n_win, n_win};
}
static size_t halo_bytes(const SimEngine& e) { return 2 * (size_t)(SIM_TILE + e.halo_cap) * sizeof(int4); }
static size_t tiled_smem_pass1(const SimEngine& e, const SimEAMTables& t) {
    return halo_bytes(e) + (size_t)tile_window(t).n_win * sizeof(float2);
}
static size_t tiled_smem_pass2(const SimEngine& e, const SimEAMTables& t) {
    return halo_bytes(e) + (size_t)(tile_window(t).n_win + 1) * sizeof(float4);
}

static int tiled_grid(const SimEngine& e) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return e.n_tiles < sms ? e.n_tiles : sms;
}

// Opt in to the largest dynamic shared memory the kernel can use: the device's
// per-block opt-in limit minus the kernel's static shared memory.
template <typename K>
static bool allow_smem_tiled(K kernel) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return false;
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) return false;
    if (dyn < (int)kTileSmemLimit) kTileSmemLimit = (size_t)dyn;
    return true;
}

static bool tiled_set_attributes() {
    static int state = 0;   // 0 unset, 1 ok, -1 failed; the first call precedes any stream capture
    if (state == 0) {
        bool ok = allow_smem_tiled(k_eam_density_tiled<true>) && allow_smem_tiled(k_eam_density_tiled<false>) &&
                  allow_smem_tiled(k_eam_force_tiled<true, true>) && allow_smem_tiled(k_eam_force_tiled<true, false>) &&
                  allow_smem_tiled(k_eam_force_tiled<false, true>) &&
                  allow_smem_tiled(k_eam_force_tiled<false, false>);
        state = ok ? 1 : -1;
        cudaGetLastError();   // a failed attribute call must not surface at the next launch check
    }
    return state == 1;
}

bool tiled_eam_usable(const SimEngine& e, const SimEAMTables& t) {
    return e.nbr16 && e.halo && e.halo_n && e.n_tiles > 0 && e.halo_cap > 0 && e.halo_cap <= HALO_SORT_MAX &&
           t.n_types == 1 && tiled_set_attributes() && tiled_smem_pass1(e, t) <= kTileSmemLimit &&
           tiled_smem_pass2(e, t) <= kTileSmemLimit;
}

int launch_eam_density_tiled(const SimEngine& e, const SimEAMTables& t, cudaStream_t st) {
    const int g = tiled_grid(e);
    if (g > e.n_blocks_max) return SIM_ERR_ARG;
    const size_t smem = tiled_smem_pass1(e, t);
    if (e.box_orthogonal) k_eam_density_tiled<true><<<g, SIM_TILE, smem, st>>>(e, t, tile_window(t));
    else k_eam_density_tiled<false><<<g, SIM_TILE, smem, st>>>(e, t, tile_window(t));
    return SIM_OK;
}

int launch_eam_force_tiled(const SimEngine& e, const SimEAMTables& t, const SimIntegrator* ip, cudaStream_t st) {
    const int g = tiled_grid(e);
    if (g > e.n_blocks_max) return SIM_ERR_ARG;
    const size_t smem = tiled_smem_pass2(e, t);
    SimIntegrator integ{};
    if (ip) integ = *ip;
    if (ip) {
        if (e.box_orthogonal) k_eam_force_tiled<true, true><<<g, SIM_TILE, smem, st>>>(e, t, integ, tile_window(t));
        else k_eam_force_tiled<true, false><<<g, SIM_TILE, smem, st>>>(e, t, integ, tile_window(t));
    } else {
        if (e.box_orthogonal) k_eam_force_tiled<false, true><<<g, SIM_TILE, smem, st>>>(e, t, integ, tile_window(t));
        else k_eam_force_tiled<false, false><<<g, SIM_TILE, smem, st>>>(e, t, integ, tile_window(t));
    }
    return SIM_OK;
}

}  // namespace simb200
