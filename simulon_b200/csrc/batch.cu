// Batched replicas (sm_100a): many independent EAM systems of uneven size in
// one launch per kernel.
//
// Layout: replica k owns slots [off, off + n_slots) of the shared SimEngine
// arrays, off and n_slots multiples of 32, so a warp's 32 slots always belong
// to one replica and per-replica data (box, cell grid, temperature, grip
// rate) is warp-uniform.  Positions carry the replica's own fixed-point
// fractional code, so the minimum image of every pair is the int32 difference
// as in the single-system engine; only the conversion to Cartesian uses the
// replica's box.  Neighbour rows hold batch slot indices.
//
// Rebuilds are per replica: the skin/2 trigger sets rep_flags[k], and every
// rebuild kernel skips the slots and cells of replicas that are not flagged,
// so a hot replica can rebuild every few steps without touching the others.
//
// Reductions: each warp writes the sums of its 32 slots to chunk_red; a few
// blocks per replica then add its chunks in a fixed order in FP64
// (deterministic, no atomics).
//
// Pair arithmetic, table interpolation and integration are the single-system
// engine's (eam_device.cuh, grid.cuh, common.cuh), so a replica advanced in a
// batch matches the same system advanced alone.
#include <cstdio>
#include "common.cuh"
#include "grid.cuh"
#include "eam_device.cuh"

namespace simb200 {

#define BATCH_DENSITY_THREADS 512
#define BATCH_FORCE_THREADS 1024
#define BATCH_WINDOW_ROWS 4096

__device__ __forceinline__ int slot_replica(const SimBatch& B, int64_t i, bool& real) {
    const int r = B.slot_rep[i];
    real = r >= 0;
    return r >= 0 ? r : -1 - r;
}

// ---------------------------------------------------------------------------
// rebuild of the flagged replicas.  k_bb_plan lists them with prefix sums of
// their 32-slot chunks and cells (B.work), and every later kernel walks only
// those ranges, so a rebuild costs time in proportion to the atoms rebuilt.

struct WorkList {
    const int32_t* ids;     // flagged replicas
    const int32_t* chunks;  // [nf + 1] prefix of their slot chunks
    const int32_t* cells;   // [nf + 1] prefix of their cells
    int nf;
};
__device__ __forceinline__ WorkList work_list(const SimBatch& B) {
    const int32_t* w = B.work;
    return WorkList{w + 1, w + (B.n_rep + 1), w + 2 * (B.n_rep + 1), w[0]};
}
// index f of the flagged replica whose prefix range [pre[f], pre[f+1]) holds x
__device__ __forceinline__ int work_find(const int32_t* pre, int nf, int64_t x) {
    int lo = 0, hi = nf;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}
// t-th slot of the flagged replicas (32 per chunk, padding included): false past the end
__device__ __forceinline__ bool work_slot(const SimBatch& B, const WorkList& W, int64_t t, int64_t& slot, int& k) {
    const int64_t chunk = t >> 5;
    if (W.nf == 0 || chunk >= W.chunks[W.nf]) return false;
    const int f = work_find(W.chunks, W.nf, chunk);
    k = W.ids[f];
    slot = B.rep[k].off + ((chunk - W.chunks[f]) << 5) + (t & 31);
    return true;
}

// one warp: the replicas to rebuild (all when only_flagged == 0), in order
__global__ void k_bb_plan(SimBatch B, int only_flagged) {
    const int lane = threadIdx.x & 31;
    int32_t* ids = B.work + 1;
    int32_t* chunks = B.work + (B.n_rep + 1);
    int32_t* cells = B.work + 2 * (B.n_rep + 1);
    int nf = 0, cc = 0, ce = 0;
    if (lane == 0) { chunks[0] = 0; cells[0] = 0; }
    for (int base = 0; base < B.n_rep; base += 32) {
        const int k = base + lane;
        const bool on = k < B.n_rep && (!only_flagged || B.rep_flags[k] != 0);
        const int nch = on ? (B.rep[k].n_slots >> 5) : 0;
        const int nce = on ? B.rep[k].n_cells : 0;
        const unsigned m = __ballot_sync(0xffffffffu, on);
        int ich = nch, ice = nce;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(0xffffffffu, ich, o);
            const int c = __shfl_up_sync(0xffffffffu, ice, o);
            if (lane >= o) { ich += a; ice += c; }
        }
        if (on) {
            const int pos = nf + __popc(m & ((1u << lane) - 1u));
            ids[pos] = k;
            chunks[pos + 1] = cc + ich;
            cells[pos + 1] = ce + ice;
        }
        nf += __popc(m);
        cc += __shfl_sync(0xffffffffu, ich, 31);
        ce += __shfl_sync(0xffffffffu, ice, 31);
    }
    if (lane == 0) B.work[0] = nf;
}

__global__ void k_bb_bin(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const WorkList W = work_list(B);
    int64_t i;
    int k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; work_slot(B, W, t, i, k);
         t += (int64_t)gridDim.x * blockDim.x) {
        if (i - B.rep[k].off >= B.rep[k].n) continue;   // padding
        const SimRep& R = B.rep[k];
        double s[3];
        cart_to_frac(R.box, e.x[i], e.x[e.n_pad + i], e.x[2 * e.n_pad + i], s);
        const int cx = cell_coord(s[0], R.ncell[0]);
        const int cy = cell_coord(s[1], R.ncell[1]);
        const int cz = cell_coord(s[2], R.ncell[2]);
        const int lin = cx + R.ncell[0] * (cy + R.ncell[1] * cz);
        const int c = R.cell_off + e.cell_rank[2 * R.cell_off + lin];
        e.cell_of[i] = c;
        atomicAdd(&e.cell_count[c], 1);
    }
}

// One block per replica: exclusive scan of its cell counts, based at its first
// slot; counts are zeroed for the scatter.
__global__ void __launch_bounds__(1024) k_bb_scan(SimBatch B, int only_flagged) {
    const WorkList W = work_list(B);
    if ((int)blockIdx.x >= W.nf) return;
    const SimRep& R = B.rep[W.ids[blockIdx.x]];
    int32_t* cnt = B.e.cell_count + R.cell_off;
    int32_t* start = B.e.cell_start + R.cell_off;
    const int n = R.n_cells;
    __shared__ int32_t warp_tot[32];
    __shared__ int32_t carry_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) carry_s = (int32_t)R.off;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int idx = base + tid;
        const int32_t v = idx < n ? cnt[idx] : 0;
        int32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int32_t w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
            int32_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            warp_tot[lane] = wi - w;
        }
        __syncthreads();
        const int32_t run = carry_s + warp_tot[warp] + (incl - v);
        if (idx < n) {
            start[idx] = run;
            cnt[idx] = 0;
        }
        __syncthreads();
        if (tid == blockDim.x - 1) carry_s = run + v;
        __syncthreads();
    }
    if (tid == 0) start[n] = carry_s;
}

__global__ void k_bb_scatter(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const WorkList W = work_list(B);
    int64_t i;
    int k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; work_slot(B, W, t, i, k);
         t += (int64_t)gridDim.x * blockDim.x) {
        if (i - B.rep[k].off >= B.rep[k].n) continue;   // padding
        const int c = e.cell_of[i];
        e.perm[e.cell_start[c] + atomicAdd(&e.cell_count[c], 1)] = (int32_t)i;
    }
}

// In-cell order by original index (reruns are bitwise reproducible), one
// warp per cell; counts are cleared for the next rebuild.
__global__ void k_bb_sort_cells(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const WorkList W = work_list(B);
    const int total = W.nf ? W.cells[W.nf] : 0;
    const int warps = (int)(gridDim.x * blockDim.x) >> 5;
    for (int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); t < total; t += warps) {
        const int f = work_find(W.cells, W.nf, t);
        const int c = B.rep[W.ids[f]].cell_off + (t - W.cells[f]);
        if ((threadIdx.x & 31) == 0) e.cell_count[c] = 0;
        warp_sort_cell(e.perm, e.orig, e.cell_start[c], e.cell_start[c + 1]);
    }
}

__global__ void k_bb_permute(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const int64_t P = e.n_pad;
    const WorkList W = work_list(B);
    int64_t m;
    int k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; work_slot(B, W, t, m, k);
         t += (int64_t)gridDim.x * blockDim.x) {
        if (m - B.rep[k].off >= B.rep[k].n) continue;   // padding
        const int64_t o = e.perm[m];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            e.x_alt[c * P + m] = e.x[c * P + o];
            e.v_alt[c * P + m] = e.v[c * P + o];
        }
        reinterpret_cast<float4*>(e.f32_alt)[m] = reinterpret_cast<const float4*>(e.f32)[o];
        e.orig_alt[m] = e.orig[o];
        e.cell_of[m] = e.posq[4 * o + 3];   // the type; posq is rewritten by k_bb_commit
    }
}

__global__ void k_bb_commit(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const int64_t P = e.n_pad;
    const WorkList W = work_list(B);
    int64_t m;
    int k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; work_slot(B, W, t, m, k);
         t += (int64_t)gridDim.x * blockDim.x) {
        if (m - B.rep[k].off >= B.rep[k].n) continue;   // padding
        const double x0 = e.x_alt[m], x1 = e.x_alt[P + m], x2 = e.x_alt[2 * P + m];
        e.x[m] = x0; e.x[P + m] = x1; e.x[2 * P + m] = x2;
#pragma unroll
        for (int c = 0; c < 3; ++c) e.v[c * P + m] = e.v_alt[c * P + m];
        reinterpret_cast<float4*>(e.f32)[m] = reinterpret_cast<const float4*>(e.f32_alt)[m];
        e.orig[m] = e.orig_alt[m];
        const int type = e.cell_of[m];
        double s[3];
        cart_to_frac(B.rep[k].box, x0, x1, x2, s);
        const uint32_t u0 = to_fixed(s[0]), u1 = to_fixed(s[1]), u2 = to_fixed(s[2]);
        reinterpret_cast<int4*>(e.posq)[m] = make_int4((int32_t)u0, (int32_t)u1, (int32_t)u2, type);
        e.xref[m] = (int32_t)u0; e.xref[P + m] = (int32_t)u1; e.xref[2 * P + m] = (int32_t)u2;
    }
}

// slot -> cell entry after the sort (binary search over the replica's starts)
__global__ void k_bb_slot_cells(SimBatch B, int only_flagged) {
    const SimEngine& e = B.e;
    const WorkList W = work_list(B);
    int64_t m;
    int k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; work_slot(B, W, t, m, k);
         t += (int64_t)gridDim.x * blockDim.x) {
        if (m - B.rep[k].off >= B.rep[k].n) continue;   // padding
        const SimRep& R = B.rep[k];
        int lo = R.cell_off, hi = R.cell_off + R.n_cells;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (e.cell_start[mid] <= m) lo = mid; else hi = mid;
        }
        e.cell_of[m] = lo;
    }
}

#define BATCH_ELL_WARPS 4
template <bool ORTH>
__global__ void __launch_bounds__(BATCH_ELL_WARPS * 32, ORTH ? 5 : 4) k_bb_build_ell(SimBatch B, float rc2_list,
                                                                                   int only_flagged) {
    __shared__ uint64_t keys[BATCH_ELL_WARPS][ELL_KEYS];
    const SimEngine& e = B.e;
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int warp = threadIdx.x >> 5;
    const WorkList W = work_list(B);
    const int total = W.nf ? W.cells[W.nf] : 0;
    const int64_t n_warps = (int64_t)gridDim.x * BATCH_ELL_WARPS;
    const int64_t flagged = W.nf ? (int64_t)W.chunks[W.nf] << 5 : 0;
    if (flagged <= n_warps) {
        // few atoms to rebuild (one wave of warps): one warp per row, so a
        // small replica's rows are not built one after another per cell
        // (rows equal ell_cell_warp's)
        int64_t m;
        int k;
        for (int64_t t = blockIdx.x * BATCH_ELL_WARPS + warp; work_slot(B, W, t, m, k); t += n_warps) {
            const SimRep& R = B.rep[k];
            if (m - R.off >= R.n) continue;   // padding (uniform across the warp)
            const int32_t* rank = e.cell_rank + 2 * R.cell_off;
            const CellGrid g{&R.box, R.ncell[0], R.ncell[1], R.ncell[2], rank, e.cell_start + R.cell_off};
            const int lin = rank[R.n_cells + (e.cell_of[m] - R.cell_off)];
            ell_row_warp(posq, m, lin, g, rc2_list, e.nbr, e.n_pad, e.nbr_cap, e.nnbr, e.flags, keys[warp]);
        }
        return;
    }
    for (int t = blockIdx.x * BATCH_ELL_WARPS + warp; t < total; t += gridDim.x * BATCH_ELL_WARPS) {
        const int f = work_find(W.cells, W.nf, t);
        const SimRep& R = B.rep[W.ids[f]];
        const int32_t* rank = e.cell_rank + 2 * R.cell_off;
        const CellGrid g{&R.box, R.ncell[0], R.ncell[1], R.ncell[2], rank, e.cell_start + R.cell_off};
        ell_cell_warp<ORTH>(posq, t - W.cells[f], rank + R.n_cells, g, rc2_list, e.nbr, e.n_pad, e.nbr_cap, e.nnbr,
                            e.flags, keys[warp]);
    }
}

__global__ void k_bb_finish(SimBatch B, int only_flagged) {
    bool any = false;
    for (int k = threadIdx.x; k < B.n_rep; k += blockDim.x) {
        if (!only_flagged || B.rep_flags[k] != 0) {
            B.rep_rebuilds[k] += 1;
            any = true;
        }
        B.rep_flags[k] = 0;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        if (any) B.e.flags[3] += 1;
        B.e.flags[0] = 0;
    }
}

static int grid_slots(int64_t n) {
    const int64_t g = ceil_div(n, SIM_THREADS);
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

static int batch_rebuild(const SimBatch& B, int only_flagged, cudaStream_t st) {
    const int g = grid_slots(B.e.n);
    k_bb_plan<<<1, 32, 0, st>>>(B, only_flagged);
    k_bb_bin<<<g, SIM_THREADS, 0, st>>>(B, only_flagged);
    k_bb_scan<<<B.n_rep, 1024, 0, st>>>(B, only_flagged);
    k_bb_scatter<<<g, SIM_THREADS, 0, st>>>(B, only_flagged);
    k_bb_sort_cells<<<grid_slots((int64_t)B.n_cell_entries * 32), SIM_THREADS, 0, st>>>(B, only_flagged);
    k_bb_permute<<<g, SIM_THREADS, 0, st>>>(B, only_flagged);
    k_bb_commit<<<g, SIM_THREADS, 0, st>>>(B, only_flagged);
    k_bb_slot_cells<<<g, SIM_THREADS, 0, st>>>(B, only_flagged);
    const float rc2_list = (float)(B.e.x_rc * B.e.x_rc * (1.0 + 4e-6));
    const int64_t ge = ceil_div(B.n_cell_entries, BATCH_ELL_WARPS);
    const int gb = (int)(ge > 148 * 64 ? 148 * 64 : ge);
    if (B.e.box_orthogonal)
        k_bb_build_ell<true><<<gb, BATCH_ELL_WARPS * 32, 0, st>>>(B, rc2_list, only_flagged);
    else
        k_bb_build_ell<false><<<gb, BATCH_ELL_WARPS * 32, 0, st>>>(B, rc2_list, only_flagged);
    k_bb_finish<<<1, 256, 0, st>>>(B, only_flagged);
    return launch_status("sim_batch_rebuild");
}

// ---------------------------------------------------------------------------
// load: rows in original order (replica after replica) -> slots

__global__ void k_bb_load(SimBatch B, const double* __restrict__ x_rows, const double* __restrict__ v_rows,
                          const int32_t* __restrict__ types) {
    const SimEngine& e = B.e;
    const int64_t P = e.n_pad;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < P; m += (int64_t)gridDim.x * blockDim.x) {
        bool real = false;
        int k = 0;
        if (m < e.n) k = slot_replica(B, m, real);
        e.nnbr[m] = 0;
        reinterpret_cast<float4*>(e.f32)[m] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!real) {
#pragma unroll
            for (int c = 0; c < 3; ++c) { e.x[c * P + m] = 0.0; e.v[c * P + m] = 0.0; e.xref[c * P + m] = 0; }
            reinterpret_cast<int4*>(e.posq)[m] = make_int4(0, 0, 0, 0);
            reinterpret_cast<int4*>(e.posfp)[m] = make_int4(0, 0, 0, 0);
            e.orig[m] = -1;
            continue;
        }
        const SimRep& R = B.rep[k];
        const int64_t a = R.first + (m - R.off);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            e.x[c * P + m] = x_rows[3 * a + c];
            e.v[c * P + m] = v_rows ? v_rows[3 * a + c] : 0.0;
        }
        e.orig[m] = (int32_t)a;
        reinterpret_cast<int4*>(e.posq)[m] = make_int4(0, 0, 0, types[a]);
    }
}

__global__ void k_bb_flag_all(SimBatch B) {
    for (int k = threadIdx.x; k < B.n_rep; k += blockDim.x) B.rep_flags[k] = 1;
    if (threadIdx.x == 0) B.e.flags[0] = 1;
}

// ---------------------------------------------------------------------------
// EAM pass 1: as k_eam_density (one element type), with the replica's box per warp and per-warp
// embedding-energy sums

template <bool ORTHO>
__global__ void __launch_bounds__(BATCH_DENSITY_THREADS, 3) k_bb_density(SimBatch B, SimEAMTables t, Window w) {
    extern __shared__ float2 s_dens[];
    pdl_trigger();
    const SimEngine& e = B.e;
    const float2* dens = reinterpret_cast<const float2*>(t.dens_vd);
    for (int k = threadIdx.x; k < w.n_win; k += blockDim.x) s_dens[k] = __ldg(&dens[w.k_lo + k]);
    __syncthreads();
    pdl_wait();   // the table is constant; positions, boxes and lists come from earlier kernels
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    int4* __restrict__ posfp = reinterpret_cast<int4*>(e.posfp);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    const bool use_mask = e.cut_mask != nullptr && e.nbr_cap <= 64;
    const int lane = threadIdx.x & 31;
    const BlockRange br = block_range(e.n);   // warp-aligned: a warp's 32 slots stay in one replica
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        bool real;
        const int k = slot_replica(B, i, real);
        const BoxF b(B.rep[k].box);
        float F = 0.0f;
        if (real) {
            const int4 qi = posq[i];
            const int nn = e.nnbr[i];
            float rho = 0.0f;
            uint32_t in_lo = 0, in_hi = 0;
            int kk = 0;
            for (; kk + 4 <= nn; kk += 4) {
                int j[4];
                int4 q[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) j[u] = ld_stream(&nbr[(int64_t)(kk + u) * P + i]);
#pragma unroll
                for (int u = 0; u < 4; ++u) q[u] = __ldg(&posq[j[u]]);
                uint32_t bits = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    bool in;
                    rho += density_term<true, ORTHO, true>(b, qi, q[u], rc2, dens, s_dens, w, t, in);
                    bits |= (uint32_t)in << u;
                }
                if (kk < 32) in_lo |= bits << kk;
                else in_hi |= bits << (kk - 32);
            }
            for (; kk < nn; ++kk) {
                bool in;
                rho += density_term<true, ORTHO, true>(b, qi, __ldg(&posq[ld_stream(&nbr[(int64_t)kk * P + i])]), rc2,
                                                       dens, s_dens, w, t, in);
                if (kk < 32) in_lo |= (uint32_t)in << kk;
                else in_hi |= (uint32_t)in << (kk - 32);
            }
            float Fp;
            embed_lookup(t, 0, rho, F, Fp);
            posfp[i] = make_int4(qi.x, qi.y, qi.z, __float_as_int(Fp));
            if (use_mask) e.cut_mask[i] = ((uint64_t)in_hi << 32) | in_lo;
        }
        const float sum = warp_sum_f(F);
        if (lane == 0) B.chunk_red[(i >> 5) * SIM_RED_SLOTS + SIM_RED_EPOT_EMBED] = (double)sum;
    }
}

// ---------------------------------------------------------------------------
// EAM pass 2 (+ integration): as k_eam_force<SINGLE>, with per-replica box,
// Langevin amplitude and grips, and per-warp sums of the 15 reduction slots.

// Grip atom at step `step`: its reference position moved along the grip axis
// by half the opening (lower grip -, upper grip +).
__device__ __forceinline__ void grip_position(const SimBatch& B, const SimRep& R, int code, int64_t a, uint64_t step,
                                              double* xn) {
    const double* h = R.box.H + 3 * R.grip_axis;
    const double len = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    const double d = (code == 2 ? 1.0 : -1.0) * (0.5 * R.grip_rate * (double)(step + 1)) / len;
#pragma unroll
    for (int c = 0; c < 3; ++c) xn[c] = B.gref[c * B.e.n_pad + a] + d * h[c];
}

template <int MODE, bool ORTHO>
__global__ void __launch_bounds__(BATCH_FORCE_THREADS, 1) k_bb_force(SimBatch B, SimEAMTables t, SimIntegrator ip,
                                                                     Window w) {
    extern __shared__ float4 s_tab4[];
    pdl_trigger();
    const SimEngine& e = B.e;
    float4* tab_d = s_tab4;
    float2* tab_p = reinterpret_cast<float2*>(s_tab4 + w.n_win);
    {
        const float4* gd = reinterpret_cast<const float4*>(t.deriv_vd) + w.k_lo;
        const float2* gp = reinterpret_cast<const float2*>(t.pair_vd) + w.k_lo;
        for (int k = threadIdx.x; k < w.n_win; k += blockDim.x) {
            tab_d[k] = __ldg(&gd[k]);
            tab_p[k] = __ldg(&gp[k]);
        }
        __syncthreads();
    }
    pdl_wait();   // pass 1's posfp and F' come from the previous kernel
    const int4* __restrict__ posfp = reinterpret_cast<const int4*>(e.posfp);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    const bool use_mask = e.cut_mask != nullptr && e.nbr_cap <= 64;
    const int lane = threadIdx.x & 31;
    bool bad = false;
    const uint64_t step = MODE && ip.step_ctr ? *ip.step_ctr : 0;
    const BlockRange br = block_range(e.n);   // warp-aligned: a warp's 32 slots stay in one replica
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        bool real;
        const int k = slot_replica(B, i, real);
        const SimRep& R = B.rep[k];
        const BoxF b(R.box);
        float acc[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        bool trig = false;
        if (real) {
            const int4 pi = posfp[i];
            const float fpi = __int_as_float(pi.w);
            float fx = 0.f, fy = 0.f, fz = 0.f;
            if (use_mask) {
                // in-cutoff slots only; the next two list entries are fetched
                // while the current pair is gathered and evaluated
                SlotSeq m(ld_stream(&e.cut_mask[i]));
                int ka = m.next(), kb = m.next();
                int ja = ka >= 0 ? ld_stream(&nbr[(int64_t)ka * P + i]) : 0;
                int jb = kb >= 0 ? ld_stream(&nbr[(int64_t)kb * P + i]) : 0;
                while (kb >= 0) {
                    const int j0 = ja, j1 = jb;
                    ka = m.next();
                    kb = m.next();
                    if (ka >= 0) ja = ld_stream(&nbr[(int64_t)ka * P + i]);
                    if (kb >= 0) jb = ld_stream(&nbr[(int64_t)kb * P + i]);
                    const int4 q0 = __ldg(&posfp[j0]);
                    const int4 q1 = __ldg(&posfp[j1]);
                    pair_single<ORTHO>(b, pi, q0, rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
                    pair_single<ORTHO>(b, pi, q1, rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
                }
                if (ka >= 0)
                    pair_single<ORTHO>(b, pi, __ldg(&posfp[ja]), rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
            } else {
                const int nn = e.nnbr[i];
                for (int kk = 0; kk < nn; ++kk)
                    pair_single<ORTHO>(b, pi, __ldg(&posfp[ld_stream(&nbr[(int64_t)kk * P + i])]), rc2, fpi, tab_d,
                                       tab_p, w, t, fx, fy, fz, acc);
            }
            reinterpret_cast<float4*>(e.f32)[i] = make_float4(fx, fy, fz, 0.0f);
            bad |= !(isfinite(fx) && isfinite(fy) && isfinite(fz));
            if (MODE) {
                const int64_t a = e.orig[i];
                const int code = B.grip[a];
                const double m = e.mass[0];
                double v[3] = {0.0, 0.0, 0.0}, acl[3];
                if (code == 0) {
                    SimIntegrator ipk = ip;
                    ipk.rff = B.rep_rff + k;          // one element type: rff[0] of this replica
                    second_half_atom(e, ipk, i, 0, step, (double)fx, (double)fy, (double)fz, v, bad, MODE == 1, acl);
                } else if (MODE == 1) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) e.v[c * P + i] = 0.0;
                }
                acc[8] += (float)(0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
                acc[9] += (float)(m * v[0] * v[0]); acc[10] += (float)(m * v[1] * v[1]); acc[11] += (float)(m * v[2] * v[2]);
                acc[12] += (float)(m * v[0] * v[1]); acc[13] += (float)(m * v[0] * v[2]); acc[14] += (float)(m * v[1] * v[2]);
                if (MODE == 2) {
                    if (code == 0) {
                        const double f[3] = {(double)fx, (double)fy, (double)fz};
                        trig = first_half_atom(e, R.box, ip, i, 0, f, v, bad, nullptr, nullptr, acl);
                    } else {
                        double xn[3];
                        grip_position(B, R, code, a, step + 1, xn);
#pragma unroll
                        for (int c = 0; c < 3; ++c) e.v[c * P + i] = 0.0;
                        trig = place_atom(e, R.box, i, 0, xn);
                    }
                }
            }
        }
        if (MODE == 2 && __any_sync(0xffffffffu, trig) && lane == 0) {
            B.rep_flags[k] = 1;
            e.flags[0] = 1;
        }
        virial_trace(acc);
        double* out = B.chunk_red + (i >> 5) * SIM_RED_SLOTS;
#pragma unroll
        for (int s = 0; s < 15; ++s) {
            if (!MODE && s >= 8) break;
            const float v = warp_sum_f(acc[s]);
            if (lane == 0) out[SIM_RED_EPOT_PAIR + s] = s < 8 ? 0.5 * (double)v : (double)v;
        }
    }
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

// First half-step of every replica at the start of a run (step = *ctr + 1;
// the counter itself is advanced by k_bb_advance_step afterwards).
__global__ void k_bb_first_half(SimBatch B, SimIntegrator p) {
    const SimEngine& e = B.e;
    const int64_t P = e.n_pad;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool trig = false, bad = false;
    const uint64_t step = *p.step_ctr + 1;
    int k = 0;
    if (i < e.n) {
        bool real;
        k = slot_replica(B, i, real);
        if (real) {
            const SimRep& R = B.rep[k];
            const int64_t a = e.orig[i];
            const int code = B.grip[a];
            if (code == 0) {
                const float4 f4 = reinterpret_cast<const float4*>(e.f32)[i];
                const double f[3] = {(double)f4.x, (double)f4.y, (double)f4.z};
                trig = first_half_atom(e, R.box, p, i, 0, f, nullptr, bad);
            } else {
                double xn[3];
                grip_position(B, R, code, a, step, xn);
#pragma unroll
                for (int c = 0; c < 3; ++c) e.v[c * P + i] = 0.0;
                trig = place_atom(e, R.box, i, 0, xn);
            }
        }
    }
    if (__any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) {
        B.rep_flags[k] = 1;
        e.flags[0] = 1;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

__global__ void k_bb_advance_step(uint64_t* ctr) {
    pdl_trigger();
    pdl_wait();
    *ctr += 1;
}

// Per-replica sums in two launches, both in a fixed order (deterministic, no
// atomics): SIM_BATCH_RED_SPLIT blocks per replica each add a strided share of
// its warps' partials (butterfly sums within and across warps) into the rows
// after the per-warp area of chunk_red; then one warp per replica adds those
// rows into rep_red and, with a log, into row (*step % cap).
#define BATCH_REDUCE_THREADS 512
__global__ void __launch_bounds__(BATCH_REDUCE_THREADS) k_bb_reduce(SimBatch B) {
    pdl_trigger();
    pdl_wait();
    const int k = blockIdx.x / SIM_BATCH_RED_SPLIT, sl = blockIdx.x % SIM_BATCH_RED_SPLIT;
    const SimRep& R = B.rep[k];
    const int64_t c0 = R.off >> 5, c1 = (R.off + R.n_slots) >> 5;
    __shared__ double part[SIM_RED_SLOTS][BATCH_REDUCE_THREADS / 32];
    double s[SIM_RED_SLOTS];
#pragma unroll
    for (int q = 0; q < SIM_RED_SLOTS; ++q) s[q] = 0.0;
    const int64_t stride = (int64_t)blockDim.x * SIM_BATCH_RED_SPLIT;
    for (int64_t c = c0 + sl * (int64_t)blockDim.x + threadIdx.x; c < c1; c += stride) {
        const double2* src = reinterpret_cast<const double2*>(B.chunk_red + c * SIM_RED_SLOTS);
#pragma unroll
        for (int q = 0; q < SIM_RED_SLOTS / 2; ++q) {
            const double2 v = src[q];
            s[2 * q] += v.x;
            s[2 * q + 1] += v.y;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < SIM_RED_SLOTS; ++q) {
        const double v = warp_sum(s[q]);
        if (lane == 0) part[q][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
        double* dst = B.chunk_red + ((B.e.n_pad >> 5) + blockIdx.x) * SIM_RED_SLOTS;
#pragma unroll
        for (int q = 0; q < SIM_RED_SLOTS; ++q) {
            const double v = warp_sum(lane < (int)(blockDim.x >> 5) ? part[q][lane] : 0.0);
            if (lane == 0) dst[q] = v;
        }
    }
}

__global__ void k_bb_reduce_final(SimBatch B, const uint64_t* step, double* log, int cap) {
    pdl_trigger();
    pdl_wait();
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= B.n_rep || lane >= SIM_RED_SLOTS) return;
    const double* src = B.chunk_red + ((B.e.n_pad >> 5) + (int64_t)k * SIM_BATCH_RED_SPLIT) * SIM_RED_SLOTS;
    double acc = 0.0;
    for (int sl = 0; sl < SIM_BATCH_RED_SPLIT; ++sl) acc += src[sl * SIM_RED_SLOTS + lane];
    B.rep_red[k * SIM_RED_SLOTS + lane] = acc;
    if (log) log[((*step % (uint64_t)cap) * B.n_rep + k) * SIM_RED_SLOTS + lane] = acc;
}

__global__ void k_bb_gather_f64(SimBatch B, const double* __restrict__ src, double* __restrict__ out) {
    const SimEngine& e = B.e;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < e.n; m += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = e.orig[m];
        if (B.slot_rep[m] < 0 || o < 0) continue;
        out[3 * o] = src[m];
        out[3 * o + 1] = src[e.n_pad + m];
        out[3 * o + 2] = src[2 * e.n_pad + m];
    }
}

__global__ void k_bb_gather_f32(SimBatch B, const float* __restrict__ src, double* __restrict__ out) {
    const SimEngine& e = B.e;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < e.n; m += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = e.orig[m];
        if (B.slot_rep[m] < 0 || o < 0) continue;
        const float4 f = reinterpret_cast<const float4*>(src)[m];
        out[3 * o] = f.x;
        out[3 * o + 1] = f.y;
        out[3 * o + 2] = f.z;
    }
}

}  // namespace simb200

using namespace simb200;

static bool batch_ok(const SimBatch* b) {
    return b && b->rep && b->n_rep > 0 && b->e.n > 0 && b->e.n % 32 == 0 && b->e.n_pad >= b->e.n &&
           b->e.n_pad % 128 == 0 && b->slot_rep && b->cell_rep && b->rep_flags && b->rep_rebuilds && b->grip &&
           b->gref && b->rep_rff && b->chunk_red && b->rep_red && b->e.n_types == 1 && b->e.nbr_cap > 0;
}

static Window batch_window(const SimEAMTables& t) {
    const int n_win = t.n_r < BATCH_WINDOW_ROWS ? t.n_r : BATCH_WINDOW_ROWS;
    return Window{t.n_r - n_win, n_win};
}

static bool batch_tables_ok(const SimEAMTables* t) {
    return t && t->n_types == 1 && t->n_r >= 2 && t->n_r < kMaxTableRows && t->n_rho >= 2 && t->dens_vd && t->deriv_vd && t->pair_vd &&
           t->embed && t->embed_deriv && t->rho_min && t->inv_drho && t->rho_clamp_hi;
}

static void batch_set_attributes() {
    static bool done = false;   // the first call happens before any stream capture
    if (done) return;
    const int lim = 200 * 1024;
    cudaFuncSetAttribute(k_bb_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_density<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_bb_force<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaGetLastError();
    done = true;
}

extern "C" int sim_batch_load(const SimBatch* b, const double* x_rows, const double* v_rows, const int32_t* types,
                              void* stream) {
    if (!batch_ok(b) || !x_rows || !types) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    prepare_capture_stream();
    batch_set_attributes();
    k_bb_load<<<grid_slots(b->e.n_pad), SIM_THREADS, 0, st>>>(*b, x_rows, v_rows, types);
    k_bb_flag_all<<<1, 256, 0, st>>>(*b);
    return batch_rebuild(*b, 1, st);
}

extern "C" int sim_batch_rebuild(const SimBatch* b, int32_t only_flagged, void* stream) {
    if (!batch_ok(b)) return SIM_ERR_ARG;
    return batch_rebuild(*b, only_flagged ? 1 : 0, (cudaStream_t)stream);
}

static int batch_rebuild_body(const void* ctx, cudaStream_t s) { return batch_rebuild(*(const SimBatch*)ctx, 1, s); }

extern "C" int sim_batch_rebuild_if_needed(const SimBatch* b, void* stream) {
    if (!batch_ok(b)) return SIM_ERR_ARG;
    // the replica flags gate every kernel, so the eager path is the same body
    return launch_if_flag((cudaStream_t)stream, b->e.flags, batch_rebuild_body, batch_rebuild_body, b,
                          "sim_batch_rebuild_if_needed");
}

extern "C" int sim_batch_eam_density(const SimBatch* b, const SimEAMTables* t, void* stream) {
    if (!batch_ok(b) || !batch_tables_ok(t)) return SIM_ERR_ARG;
    batch_set_attributes();
    const Window w = batch_window(*t);
    const size_t smem = (size_t)w.n_win * sizeof(float2);
    const bool ortho = b->e.box_orthogonal != 0;
    const void* fn = ortho ? (const void*)k_bb_density<true> : (const void*)k_bb_density<false>;
    const int g = persistent_grid(fn, BATCH_DENSITY_THREADS, smem, b->e.n);
    cudaStream_t st = (cudaStream_t)stream;
    if (ortho) launch_pdl(k_bb_density<true>, dim3(g), dim3(BATCH_DENSITY_THREADS), smem, st, *b, *t, w);
    else launch_pdl(k_bb_density<false>, dim3(g), dim3(BATCH_DENSITY_THREADS), smem, st, *b, *t, w);
    return launch_status("sim_batch_eam_density");
}

template <int MODE>
static void launch_bb_force(const SimBatch& b, const SimEAMTables& t, const SimIntegrator& ip, bool ortho,
                            cudaStream_t st) {
    const Window w = batch_window(t);
    const size_t smem = (size_t)w.n_win * (sizeof(float4) + sizeof(float2));
    const void* fn = ortho ? (const void*)k_bb_force<MODE, true> : (const void*)k_bb_force<MODE, false>;
    const int g = persistent_grid(fn, BATCH_FORCE_THREADS, smem, b.e.n);
    if (ortho) launch_pdl(k_bb_force<MODE, true>, dim3(g), dim3(BATCH_FORCE_THREADS), smem, st, b, t, ip, w);
    else launch_pdl(k_bb_force<MODE, false>, dim3(g), dim3(BATCH_FORCE_THREADS), smem, st, b, t, ip, w);
}

extern "C" int sim_batch_eam_force(const SimBatch* b, const SimEAMTables* t, const SimIntegrator* p, int32_t mode,
                                   void* stream) {
    if (!batch_ok(b) || !batch_tables_ok(t) || mode < 0 || mode > 2) return SIM_ERR_ARG;
    SimIntegrator ip{};
    if (mode) {
        if (!p || !p->step_ctr) return SIM_ERR_ARG;
        ip = *p;
    }
    batch_set_attributes();
    const bool ortho = b->e.box_orthogonal != 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (mode == 0) launch_bb_force<0>(*b, *t, ip, ortho, st);
    else if (mode == 1) launch_bb_force<1>(*b, *t, ip, ortho, st);
    else launch_bb_force<2>(*b, *t, ip, ortho, st);
    return launch_status("sim_batch_eam_force");
}

extern "C" int sim_batch_first_half(const SimBatch* b, const SimIntegrator* p, void* stream) {
    if (!batch_ok(b) || !p || !p->step_ctr) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_bb_first_half<<<(int)ceil_div(b->e.n, SIM_THREADS), SIM_THREADS, 0, st>>>(*b, *p);
    k_bb_advance_step<<<1, 1, 0, st>>>(p->step_ctr);
    return launch_status("sim_batch_first_half");
}

extern "C" int sim_batch_reduce(const SimBatch* b, const uint64_t* step, double* log, int32_t log_cap, void* stream) {
    if (!batch_ok(b) || (log && (log_cap <= 0 || !step))) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    launch_pdl(k_bb_reduce, dim3(b->n_rep * SIM_BATCH_RED_SPLIT), dim3(BATCH_REDUCE_THREADS), 0, st, *b);
    launch_pdl(k_bb_reduce_final, dim3((unsigned)ceil_div(b->n_rep, 8)), dim3(256), 0, st, *b, step, log, log_cap);
    return launch_status("sim_batch_reduce");
}

extern "C" int sim_batched_step(const SimBatch* b, const SimEAMTables* t, const SimIntegrator* p, int32_t last,
                                double* log, int32_t log_cap, void* stream) {
    if (!batch_ok(b) || !batch_tables_ok(t) || !p || !p->step_ctr || (log && log_cap <= 0)) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = sim_batch_eam_density(b, t, stream);
    if (rc != SIM_OK) return rc;
    rc = sim_batch_eam_force(b, t, p, last ? 1 : 2, stream);
    if (rc != SIM_OK) return rc;
    rc = sim_batch_reduce(b, p->step_ctr, log, log_cap, stream);
    if (rc != SIM_OK) return rc;
    if (last) return SIM_OK;
    launch_pdl(k_bb_advance_step, dim3(1), dim3(1), 0, st, p->step_ctr);
    rc = launch_status("sim_batched_step");
    if (rc != SIM_OK) return rc;
    return sim_batch_rebuild_if_needed(b, stream);
}

extern "C" int sim_batch_gather_f64(const SimBatch* b, const double* src_soa, double* out_rows, void* stream) {
    if (!batch_ok(b) || !src_soa || !out_rows) return SIM_ERR_ARG;
    k_bb_gather_f64<<<grid_slots(b->e.n), SIM_THREADS, 0, (cudaStream_t)stream>>>(*b, src_soa, out_rows);
    return launch_status("sim_batch_gather_f64");
}

extern "C" int sim_batch_gather_f32(const SimBatch* b, const float* src_aos4, double* out_rows, void* stream) {
    if (!batch_ok(b) || !src_aos4 || !out_rows) return SIM_ERR_ARG;
    k_bb_gather_f32<<<grid_slots(b->e.n), SIM_THREADS, 0, (cudaStream_t)stream>>>(*b, src_aos4, out_rows);
    return launch_status("sim_batch_gather_f32");
}

// ---- crack observables (w_crack.py:113-188) ---------------------------------
// Doubles as 64-bit keys whose unsigned order is the numeric order, so the
// per-bin extremes are exact atomic min / max.
__device__ __forceinline__ unsigned long long dkey(double v) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_value(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((long long)u);
}

__global__ void k_crack_init(int total_bins, int n_rep, unsigned long long* bins, double* sums) {
    const unsigned long long up0 = dkey(__longlong_as_double(0x7FF0000000000000ll));   // +inf
    const unsigned long long lo0 = dkey(__longlong_as_double((long long)0xFFF0000000000000ull));   // -inf
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * total_bins + 2 * n_rep; t += gridDim.x * blockDim.x) {
        if (t < total_bins) bins[t] = up0;
        else if (t < 2 * total_bins) bins[t] = lo0;
        else sums[t - 2 * total_bins] = 0.0;
    }
}

__global__ void k_crack_scan(SimBatch B, const SimCrack* __restrict__ crack, const int8_t* __restrict__ mouth,
                             int total_bins, unsigned long long* bins, double* sums) {
    const SimEngine& e = B.e;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        bool real;
        const int k = slot_replica(B, i, real);
        if (!real) continue;
        const SimCrack& c = crack[k];
        if (c.bins <= 0) continue;
        const double x0 = e.x[i], x1 = e.x[e.n_pad + i], x2 = e.x[2 * e.n_pad + i];
        const double vx = x0 * c.x_unit[0] + x1 * c.x_unit[1] + x2 * c.x_unit[2];
        const double vy = x0 * c.y_unit[0] + x1 * c.y_unit[1] + x2 * c.y_unit[2];
        const double span = fmax(1.0e-12, c.x_max - c.x_min);
        double bf = floor((vx - c.x_min) / span * (double)c.bins);
        bf = fmin(fmax(bf, 0.0), (double)(c.bins - 1));
        const int bin = c.bin_off + (int)bf;
        if (vy > c.y_plane) atomicMin(&bins[bin], dkey(vy));
        else if (vy < c.y_plane) atomicMax(&bins[total_bins + bin], dkey(vy));
        const int tag = mouth[e.orig[i]];
        if (tag == 1) atomicAdd(&sums[2 * k], vy);
        else if (tag == 2) atomicAdd(&sums[2 * k + 1], vy);
    }
}

__global__ void k_crack_finish(SimBatch B, const SimCrack* __restrict__ crack, int total_bins,
                               const unsigned long long* __restrict__ bins, const double* __restrict__ sums,
                               double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B.n_rep) return;
    const SimCrack& c = crack[k];
    double* o = out + (size_t)k * SIM_CRACK_OUT;
    // projected stress from the replica's sums (the last sim_batch_reduce)
    const SimBox& bx = B.rep[k].box;
    const double* H = bx.H;
    const double V = fabs(H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
                          H[2] * (H[3] * H[7] - H[4] * H[6]));
    const double* r = B.rep_red + (size_t)k * SIM_RED_SLOTS;
    const double t[6] = {r[SIM_RED_K_XX] + r[SIM_RED_W_XX], r[SIM_RED_K_YY] + r[SIM_RED_W_YY],
                         r[SIM_RED_K_ZZ] + r[SIM_RED_W_ZZ], r[SIM_RED_K_XY] + r[SIM_RED_W_XY],
                         r[SIM_RED_K_XZ] + r[SIM_RED_W_XZ], r[SIM_RED_K_YZ] + r[SIM_RED_W_YZ]};
    const double s[3][3] = {{t[0], t[3], t[4]}, {t[3], t[1], t[5]}, {t[4], t[5], t[2]}};
    const double* row = H + 3;
    const double nrm = fmax(sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]), 1e-12);
    const double ax[3] = {row[0] / nrm, row[1] / nrm, row[2] / nrm};
    double pyy = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b2 = 0; b2 < 3; ++b2) pyy += ax[a] * s[a][b2] * ax[b2];
    pyy = pyy / V * 1602176.6208;
    o[0] = -pyy;
    o[1] = pyy;
    for (int q = 2; q < SIM_CRACK_OUT; ++q) o[q] = 0.0;
    if (c.bins <= 0) return;
    if (c.n_upper > 0 && c.n_lower > 0) {
        const double sc = (sums[2 * k] / c.n_upper - sums[2 * k + 1] / c.n_lower) - c.initial_cmod;
        o[2] = fabs(sc);
        o[3] = sc;
    }
    // open bins: gap between the lowest atom above and the highest below the plane
    const double span = fmax(1.0e-12, c.x_max - c.x_min), width = span / c.bins;
    int lo_seed = -1, hi_seed = -1, n_open = 0;
    auto open_bin = [&](int q) {
        const double g = dkey_value(bins[c.bin_off + q]) - dkey_value(bins[total_bins + c.bin_off + q]);
        return isfinite(g) && g >= c.threshold;
    };
    for (int q = 0; q < c.bins; ++q) {
        if (!open_bin(q)) continue;
        ++n_open;
        const double center = c.x_min + (q + 0.5) * width;
        if (center >= c.x_center - c.half_length && center <= c.x_center + c.half_length) {
            if (lo_seed < 0) lo_seed = q;
            hi_seed = q;
        }
    }
    o[6] = (double)n_open;
    if (lo_seed < 0) return;
    while (lo_seed > 0 && open_bin(lo_seed - 1)) --lo_seed;
    while (hi_seed < c.bins - 1 && open_bin(hi_seed + 1)) ++hi_seed;
    const double length = (hi_seed - lo_seed + 1) * width;
    o[4] = length;
    o[5] = fmax(0.0, length - 2.0 * c.half_length);
}

extern "C" int sim_batch_crack_observe(const SimBatch* b, const SimCrack* crack, const int8_t* mouth,
                                       int32_t total_bins, uint64_t* bins, double* sums, double* out, void* stream) {
    if (!batch_ok(b) || !crack || !mouth || total_bins < 0 || (total_bins > 0 && !bins) || !sums || !out)
        return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* kb = reinterpret_cast<unsigned long long*>(bins);
    const int n_init = 2 * total_bins + 2 * b->n_rep;
    k_crack_init<<<(n_init + 255) / 256, 256, 0, st>>>(total_bins, b->n_rep, kb, sums);
    if (total_bins > 0)
        k_crack_scan<<<grid_slots(b->e.n), SIM_THREADS, 0, st>>>(*b, crack, mouth, total_bins, kb, sums);
    k_crack_finish<<<(b->n_rep + 63) / 64, 64, 0, st>>>(*b, crack, total_bins, kb, sums, out);
    return launch_status("sim_batch_crack_observe");
}

