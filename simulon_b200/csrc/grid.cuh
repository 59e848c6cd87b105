// Cell-grid helpers shared by the single-system and the batched neighbour
// builds: fractional cell coordinates, the periodic 27-cell stencil, and the
// construction of full-list rows in ELL layout.
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

// Sort the slots perm[b0, b1) of one cell by their original index orig[perm[.]]
// (unique keys), with the 32 lanes of one warp: a cell of up to 32 atoms by
// rank -- each lane counts the smaller keys through shuffles, so no chain of
// dependent global loads -- a longer cell by lane 0's insertion sort.  Every
// lane of the warp must call this with the same b0, b1.
__device__ __forceinline__ void warp_sort_cell(int32_t* perm, const int32_t* orig, int b0, int b1) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int n = b1 - b0;
    if (n <= 1) return;
    if (n <= 32) {
        const bool on = lane < n;
        const int32_t v = on ? perm[b0 + lane] : 0;
        const int32_t key = on ? orig[v] : 0;
        int rank = 0;
        for (int s = 0; s < n; ++s) rank += __shfl_sync(FULL, key, s) < key ? 1 : 0;
        __syncwarp();
        if (on) perm[b0 + rank] = v;
        __syncwarp();
        return;
    }
    if (lane == 0) {
        for (int a = b0 + 1; a < b1; ++a) {
            const int32_t v = perm[a];
            const int32_t ko = orig[v];
            int p = a - 1;
            while (p >= b0 && orig[perm[p]] > ko) {
                perm[p + 1] = perm[p];
                --p;
            }
            perm[p + 1] = v;
        }
    }
    __syncwarp();
}

#define ELL_SORT_MAX 128    // rows up to this length are sorted by distance
#define ELL_CELL_CAND 384   // candidates of one cell's stencil kept in shared memory

// One periodic box's cells: linear cell index -> rank (visiting order) ->
// first slot of the cell (start has one entry more than there are cells).
struct CellGrid {
    const SimBox* box;
    int nx, ny, nz;
    const int32_t* rank;
    const int32_t* start;
};

// The FP32 box terms in registers (read once, not per candidate).
struct ListBox {
    float h[9];
    bool orth;
    __device__ __forceinline__ explicit ListBox(const SimBox& b) {
#pragma unroll
        for (int k = 0; k < 9; ++k) h[k] = b.Hf[k];
        orth = b.orthogonal != 0;
    }
};

// Squared minimum-image distance of two fixed-point positions, with the
// arithmetic of frac_to_cart_f and an unfused sum of squares.
__device__ __forceinline__ float list_d2(const ListBox& b, const int4& qi, const int4& qj) {
    const float t0 = fixed_delta(qi.x, qj.x), t1 = fixed_delta(qi.y, qj.y), t2 = fixed_delta(qi.z, qj.z);
    float r0, r1, r2;
    if (b.orth) {
        r0 = t0 * b.h[0];
        r1 = t1 * b.h[4];
        r2 = t2 * b.h[8];
    } else {
        r0 = fmaf(t2, b.h[6], fmaf(t1, b.h[3], t0 * b.h[0]));
        r1 = fmaf(t2, b.h[7], fmaf(t1, b.h[4], t0 * b.h[1]));
        r2 = fmaf(t2, b.h[8], fmaf(t1, b.h[5], t0 * b.h[2]));
    }
    return __fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2));
}

// Sort key of a list entry: d^2 bits (non-negative floats order like their
// bits) above the slot, so keys are unique and order by (d^2, slot).
__device__ __forceinline__ uint64_t list_key(float d2, int j) {
    return ((uint64_t)__float_as_uint(d2) << 32) | (uint32_t)j;
}

// Sorted write of a row whose first `kept` (<= ELL_SORT_MAX) accepted entries
// are in keys in visiting order: each entry's rank among them is counted and
// the entry stored at that position of the row.
__device__ __forceinline__ void ell_write_sorted(int64_t i, int kept, const uint64_t* keys, int32_t* nbr,
                                                 int64_t P) {
    for (int a = threadIdx.x & 31; a < kept; a += 32) {
        const uint64_t ka = keys[a];
        int rank = 0;
#pragma unroll 4
        for (int f = 0; f < kept; ++f) rank += keys[f] < ka ? 1 : 0;
        nbr[(int64_t)rank * P + i] = (int32_t)(uint32_t)ka;
    }
}

// The stencil of cell `lin` flattened for one warp: lane c < n_st holds stencil
// cell c's first slot (cs) and its candidates' offset in the flattened sequence
// (excl); cells are visited kz, ky, kx, slots ascending.
struct Stencil {
    int cs, excl, n_st, total;
};
__device__ __forceinline__ Stencil stencil_of(const CellGrid& g, int lin) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int cx = lin % g.nx, cy = (lin / g.nx) % g.ny, cz = lin / (g.nx * g.ny);
    const int sx = stencil_count(g.nx), sy = stencil_count(g.ny), sz = stencil_count(g.nz);
    Stencil st;
    st.n_st = sx * sy * sz;
    st.cs = 0;
    int cn = 0;
    if (lane < st.n_st) {
        const int kx = lane % sx, ky = (lane / sx) % sy, kz = lane / (sx * sy);
        const int r = g.rank[stencil_cell(cx, kx, g.nx) + g.nx * (stencil_cell(cy, ky, g.ny) +
                                                                 g.ny * stencil_cell(cz, kz, g.nz))];
        st.cs = g.start[r];
        cn = g.start[r + 1] - st.cs;
    }
    int incl = cn;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    st.excl = incl - cn;
    st.total = __shfl_sync(FULL, incl, 31);
    return st;
}
// slot of candidate t (clamped into range) of a flattened stencil
__device__ __forceinline__ int stencil_slot(const Stencil& st, int t) {
    const unsigned FULL = 0xffffffffu;
    const int tt = t < st.total ? t : st.total - 1;
    int c = 0;                                   // last stencil cell whose first candidate is <= tt
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const int cc = c + step;
        const int ex = __shfl_sync(FULL, st.excl, cc & 31);
        if (cc < st.n_st && ex <= tt) c = cc;
    }
    return __shfl_sync(FULL, st.cs, c) + (tt - __shfl_sync(FULL, st.excl, c));
}

__device__ __forceinline__ void ell_row_done(int64_t i, int cnt, int cap, int32_t* nnbr, int32_t* flags) {
    if ((threadIdx.x & 31) == 0) {
        nnbr[i] = cnt < cap ? cnt : cap;
        if (cnt > cap) {
            atomicOr(&flags[1], SIM_STATUS_OVERFLOW);
            atomicMax(&flags[2], cnt);
        }
    }
}

// Row i of the full list, built by the 32 lanes of one warp: every slot j != i
// of the 27 stencil cells around cell `lin` with d^2 < rc2_list, tested in FP32
// on fixed-point displacements (the radius carries a 2e-6 relative margin so
// that an exact FP64/FP32 filter applied later -- half-list export, force
// cutoffs -- always sees a superset).  Each lane tests one candidate of the
// flattened stencil per round and accepted entries are compacted in order
// through a ballot into this warp's shared buffer (keys; ELL_SORT_MAX
// entries).  Rows of up to ELL_SORT_MAX kept entries are written sorted
// nearest first, ties by slot, so in a crystal every row lists the same shells
// in the same order and a warp's lanes agree on which neighbours fall inside
// the force cutoff; longer rows keep the visiting order.  A row longer than cap
// sets SIM_STATUS_OVERFLOW and the longest length in flags[2].  Every lane of
// the warp must call this.
__device__ __forceinline__ void ell_row_warp(const int4* __restrict__ posq, int64_t i, int lin, const CellGrid& g,
                                             float rc2_list, int32_t* nbr, int64_t P, int cap, int32_t* nnbr,
                                             int32_t* flags, uint64_t* keys) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const ListBox b(*g.box);
    const int4 qi = posq[i];
    const Stencil st = stencil_of(g, lin);
    const unsigned below = (1u << lane) - 1u;
    int cnt = 0;
    for (int base = 0; base < st.total; base += 32) {
        const int t = base + lane;
        const int j = stencil_slot(st, t);
        bool acc = false;
        float d2 = 0.0f;
        if (t < st.total && j != i) {
            d2 = list_d2(b, qi, posq[j]);
            acc = d2 < rc2_list;
        }
        const unsigned m = __ballot_sync(FULL, acc);
        const int pos = cnt + __popc(m & below);
        if (acc && pos < ELL_SORT_MAX) keys[pos] = list_key(d2, j);
        cnt += __popc(m);
    }
    __syncwarp();
    const int kept = cnt < cap ? cnt : cap;
    if (kept <= ELL_SORT_MAX) {
        ell_write_sorted(i, kept, keys, nbr, P);
    } else {
        // longer than the sort buffer: the first `kept` entries in visiting order
        int w = 0;
        for (int base = 0; base < st.total && w < kept; base += 32) {
            const int t = base + lane;
            const int j = stencil_slot(st, t);
            const bool acc = t < st.total && j != i && list_d2(b, qi, posq[j]) < rc2_list;
            const unsigned m = __ballot_sync(FULL, acc);
            const int pos = w + __popc(m & below);
            if (acc && pos < kept) nbr[(int64_t)pos * P + i] = j;
            w += __popc(m);
        }
    }
    __syncwarp();
    ell_row_done(i, cnt, cap, nnbr, flags);
}

// All rows of the atoms in cell `r` (visiting rank), built by one warp: the
// candidates of the cell's stencil are gathered once into shared memory (cq,
// cj: ELL_CELL_CAND entries) and tested against each atom of the cell in turn,
// so a candidate's position is read from global memory once per cell instead
// of once per atom.  Rows come out equal to ell_row_warp's; cells whose
// stencil holds more than ELL_CELL_CAND atoms, and rows longer than
// ELL_SORT_MAX, are built by ell_row_warp.
__device__ __forceinline__ void ell_cell_warp(const int4* __restrict__ posq, int r, const int32_t* lin_of_rank,
                                              const CellGrid& g, float rc2_list, int32_t* nbr, int64_t P, int cap,
                                              int32_t* nnbr, int32_t* flags, uint64_t* keys, int4* cq, int* cj) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int a0 = g.start[r], a1 = g.start[r + 1];
    if (a0 == a1) return;
    const int lin = lin_of_rank[r];
    const Stencil st = stencil_of(g, lin);
    if (st.total > ELL_CELL_CAND) {
        for (int i = a0; i < a1; ++i) ell_row_warp(posq, i, lin, g, rc2_list, nbr, P, cap, nnbr, flags, keys);
        return;
    }
    for (int base = 0; base < st.total; base += 32) {
        const int t = base + lane;
        const int j = stencil_slot(st, t);
        if (t < st.total) {
            cq[t] = posq[j];
            cj[t] = j;
        }
    }
    __syncwarp();
    const ListBox b(*g.box);
    const unsigned below = (1u << lane) - 1u;
    for (int i = a0; i < a1; ++i) {
        const int4 qi = posq[i];
        int cnt = 0;
        for (int base = 0; base < st.total; base += 32) {
            const int t = base + lane;
            bool acc = false;
            float d2 = 0.0f;
            int j = 0;
            if (t < st.total) {
                j = cj[t];
                if (j != i) {
                    d2 = list_d2(b, qi, cq[t]);
                    acc = d2 < rc2_list;
                }
            }
            const unsigned m = __ballot_sync(FULL, acc);
            const int pos = cnt + __popc(m & below);
            if (acc && pos < ELL_SORT_MAX) keys[pos] = list_key(d2, j);
            cnt += __popc(m);
        }
        __syncwarp();
        const int kept = cnt < cap ? cnt : cap;
        if (kept > ELL_SORT_MAX) {
            ell_row_warp(posq, i, lin, g, rc2_list, nbr, P, cap, nnbr, flags, keys);
        } else {
            ell_write_sorted(i, kept, keys, nbr, P);
            ell_row_done(i, cnt, cap, nnbr, flags);
        }
        __syncwarp();
    }
}

}  // namespace simb200
