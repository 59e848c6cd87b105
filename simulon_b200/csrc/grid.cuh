// Cell-grid helpers shared by the single-system and the batched neighbour
// builds: fractional cell coordinates, the periodic 27-cell stencil, and the
// construction of one full-list row in ELL layout.
#pragma once
#include "common.cuh"

namespace simb200 {

__device__ __forceinline__ int cell_coord(double s, int n) {
    s -= floor(s);
    int c = (int)(s * (double)n);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// unique stencil offsets along one axis: n>=3 -> {-1,0,1}; n==2 -> {0,1}; n==1 -> {0}
__device__ __forceinline__ int stencil_count(int n) { return n >= 3 ? 3 : n; }
__device__ __forceinline__ int stencil_cell(int c, int k, int n) {
    if (n >= 3) { int v = c + k - 1; return v < 0 ? v + n : (v >= n ? v - n : v); }
    return k;   // n <= 2: enumerate every cell once
}

#define ELL_SORT_MAX 128   // rows up to this length are sorted by distance

// One periodic box's cells: linear cell index -> rank (visiting order) ->
// first slot of the cell (start has one entry more than there are cells).
struct CellGrid {
    const SimBox* box;
    int nx, ny, nz;
    const int32_t* rank;
    const int32_t* start;
};

// Row i of the full list, built by the 32 lanes of one warp: every slot j != i
// of the 27 stencil cells around cell `lin` with d^2 < rc2_list, tested in FP32
// on fixed-point displacements (the radius carries a 2e-6 relative margin so
// that an exact FP64/FP32 filter applied later -- half-list export, force
// cutoffs -- always sees a superset).  The stencil cells' slot ranges are
// flattened into one candidate sequence (cells in kz, ky, kx order, slots
// ascending); each lane tests one candidate per round and accepted entries are
// compacted in order through a ballot into this warp's shared buffers (keys,
// js; ELL_SORT_MAX entries each).  Rows of up to ELL_SORT_MAX kept entries are
// written sorted nearest first, ties by slot -- each entry's rank is counted
// against the others -- so in a crystal every row lists the same shells in the
// same order and a warp's lanes agree on which neighbours fall inside the force
// cutoff; longer rows keep the visiting order.  A row longer than cap sets
// SIM_STATUS_OVERFLOW and the longest length in flags[2].  Every lane of the
// warp must call this.
__device__ __forceinline__ void ell_row_warp(const int4* __restrict__ posq, int64_t i, int lin, const CellGrid& g,
                                             float rc2_list, int32_t* nbr, int64_t P, int cap, int32_t* nnbr,
                                             int32_t* flags, uint32_t* keys, int* js) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const SimBox& b = *g.box;
    const int4 qi = posq[i];
    const int cx = lin % g.nx, cy = (lin / g.nx) % g.ny, cz = lin / (g.nx * g.ny);
    const int sx = stencil_count(g.nx), sy = stencil_count(g.ny), sz = stencil_count(g.nz);
    const int n_st = sx * sy * sz;
    int cs = 0, cn = 0;
    if (lane < n_st) {
        const int kx = lane % sx, ky = (lane / sx) % sy, kz = lane / (sx * sy);
        const int r = g.rank[stencil_cell(cx, kx, g.nx) + g.nx * (stencil_cell(cy, ky, g.ny) +
                                                                 g.ny * stencil_cell(cz, kz, g.nz))];
        cs = g.start[r];
        cn = g.start[r + 1] - cs;
    }
    int incl = cn;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - cn;
    const int total = __shfl_sync(FULL, incl, 31);
    const unsigned below = (1u << lane) - 1u;
    int cnt = 0;
    for (int base = 0; base < total; base += 32) {
        const int t = base + lane;
        const int tt = t < total ? t : total - 1;
        int c = 0;                                   // last stencil cell whose first candidate is <= tt
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int cc = c + step;
            const int ex = __shfl_sync(FULL, excl, cc & 31);
            if (cc < n_st && ex <= tt) c = cc;
        }
        const int j = __shfl_sync(FULL, cs, c) + (tt - __shfl_sync(FULL, excl, c));
        bool acc = false;
        float d2 = 0.0f;
        if (t < total && j != i) {
            const int4 qj = posq[j];
            float r0, r1, r2;
            frac_to_cart_f(b, fixed_delta(qi.x, qj.x), fixed_delta(qi.y, qj.y), fixed_delta(qi.z, qj.z), r0, r1, r2);
            d2 = __fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2));
            acc = d2 < rc2_list;
        }
        const unsigned m = __ballot_sync(FULL, acc);
        const int pos = cnt + __popc(m & below);
        if (acc && pos < ELL_SORT_MAX) {
            keys[pos] = __float_as_uint(d2);        // non-negative floats order like their bits
            js[pos] = j;
        }
        cnt += __popc(m);
    }
    __syncwarp();
    const int kept = cnt < cap ? cnt : cap;
    if (kept <= ELL_SORT_MAX) {
        for (int a = lane; a < kept; a += 32) {
            const uint32_t ka = keys[a];
            const int ja = js[a];
            int rank = 0;
            for (int f = 0; f < kept; ++f) {
                const uint32_t kf = keys[f];
                rank += (kf < ka || (kf == ka && js[f] < ja)) ? 1 : 0;
            }
            nbr[(int64_t)rank * P + i] = ja;
        }
    } else {
        // longer than the sort buffer: the first `kept` entries in visiting order
        int w = 0;
        for (int base = 0; base < total && w < kept; base += 32) {
            const int t = base + lane;
            const int tt = t < total ? t : total - 1;
            int c = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int cc = c + step;
                const int ex = __shfl_sync(FULL, excl, cc & 31);
                if (cc < n_st && ex <= tt) c = cc;
            }
            const int j = __shfl_sync(FULL, cs, c) + (tt - __shfl_sync(FULL, excl, c));
            bool acc = false;
            if (t < total && j != i) {
                const int4 qj = posq[j];
                float r0, r1, r2;
                frac_to_cart_f(b, fixed_delta(qi.x, qj.x), fixed_delta(qi.y, qj.y), fixed_delta(qi.z, qj.z),
                               r0, r1, r2);
                const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2));
                acc = d2 < rc2_list;
            }
            const unsigned m = __ballot_sync(FULL, acc);
            const int pos = w + __popc(m & below);
            if (acc && pos < kept) nbr[(int64_t)pos * P + i] = j;
            w += __popc(m);
        }
    }
    __syncwarp();
    if (lane == 0) {
        nnbr[i] = kept;
        if (cnt > cap) {
            atomicOr(&flags[1], SIM_STATUS_OVERFLOW);
            atomicMax(&flags[2], cnt);
        }
    }
}

}  // namespace simb200
