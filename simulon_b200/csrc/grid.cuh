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
#define ELL_REG_ROUNDS 8    // stencil candidates a warp holds in registers: 32 per round
#define ELL_KEYS (2 * ELL_SORT_MAX)   // shared key buffer of one warp (two rows)

// One periodic box's cells: linear cell index -> rank (visiting order) ->
// first slot of the cell (start has one entry more than there are cells).
struct CellGrid {
    const SimBox* box;
    int nx, ny, nz;
    const int32_t* rank;
    const int32_t* start;
};

// The FP32 box terms in registers (read once, not per candidate), each
// scaled by 2^-32: a fixed-point difference converted to float times a
// scaled term is the same float as the difference in box units
// (fixed_delta) times the term, since a power-of-two scaling is exact, so
// the distances below are those of frac_to_cart_f.
struct ListBox {
    float h[9];
    bool orth;
    __device__ __forceinline__ explicit ListBox(const SimBox& b) {
#pragma unroll
        for (int k = 0; k < 9; ++k) h[k] = b.Hf[k] * 2.3283064365386963e-10f;
        orth = b.orthogonal != 0;
    }
};

// Squared minimum-image distance of two fixed-point positions, with the
// arithmetic of frac_to_cart_f and an unfused sum of squares.
template <bool ORTH>
__device__ __forceinline__ float list_d2_t(const ListBox& b, const int4& qi, const int4& qj) {
    const float t0 = __int2float_rn((int32_t)((uint32_t)qi.x - (uint32_t)qj.x));
    const float t1 = __int2float_rn((int32_t)((uint32_t)qi.y - (uint32_t)qj.y));
    const float t2 = __int2float_rn((int32_t)((uint32_t)qi.z - (uint32_t)qj.z));
    float r0, r1, r2;
    if (ORTH) {
        r0 = __fmul_rn(t0, b.h[0]);
        r1 = __fmul_rn(t1, b.h[4]);
        r2 = __fmul_rn(t2, b.h[8]);
    } else {
        r0 = fmaf(t2, b.h[6], fmaf(t1, b.h[3], __fmul_rn(t0, b.h[0])));
        r1 = fmaf(t2, b.h[7], fmaf(t1, b.h[4], __fmul_rn(t0, b.h[1])));
        r2 = fmaf(t2, b.h[8], fmaf(t1, b.h[5], __fmul_rn(t0, b.h[2])));
    }
    return __fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2));
}
__device__ __forceinline__ float list_d2(const ListBox& b, const int4& qi, const int4& qj) {
    return b.orth ? list_d2_t<true>(b, qi, qj) : list_d2_t<false>(b, qi, qj);
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

// Sorted writes of two rows at once (i1's row empty when n1 is 0), each of up
// to 32 entries held one per lane: an entry's rank counts the row's entries
// with a smaller d^2 (shuffled from their lanes; d^2 bits are below 2^31, so
// the sign of their difference is the comparison) plus, among the entries of
// equal d^2 (__match_any_sync; a perfect lattice has many), those with a
// smaller slot -- the order of list_key.  Every lane of the warp must call
// this.
__device__ __forceinline__ void ell_write_sorted2(int64_t i0, int n0, const uint64_t* k0, int64_t i1, int n1,
                                                  const uint64_t* k1, int32_t* nbr, int64_t P) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool on0 = lane < n0, on1 = lane < n1;
    const uint64_t e0 = on0 ? k0[lane] : 0x7fffffff00000000ull, e1 = on1 ? k1[lane] : 0x7fffffff00000000ull;
    const int32_t d0 = (int32_t)(e0 >> 32), d1 = (int32_t)(e1 >> 32);   // padded lanes: 2^31 - 1, above every d^2
    const int j0 = (int32_t)(uint32_t)e0, j1 = (int32_t)(uint32_t)e1;
    const int n = n0 > n1 ? n0 : n1;
    int r0 = 0, r1 = 0;
#pragma unroll 4
    for (int f = 0; f < n; ++f) {
        r0 += (int)((uint32_t)(__shfl_sync(FULL, d0, f) - d0) >> 31);
        r1 += (int)((uint32_t)(__shfl_sync(FULL, d1, f) - d1) >> 31);
    }
    const unsigned self = 1u << lane;
    const unsigned g0 = __match_any_sync(FULL, d0), g1 = __match_any_sync(FULL, d1);
    unsigned t0 = on0 ? g0 & ~self : 0u;
    unsigned t1 = on1 ? g1 & ~self : 0u;
    while (__any_sync(FULL, (t0 | t1) != 0u)) {
        const int f0 = t0 ? __ffs(t0) - 1 : lane, f1 = t1 ? __ffs(t1) - 1 : lane;
        r0 += __shfl_sync(FULL, j0, f0) < j0 ? 1 : 0;
        r1 += __shfl_sync(FULL, j1, f1) < j1 ? 1 : 0;
        t0 &= t0 - 1u;
        t1 &= t1 - 1u;
    }
    if (on0) nbr[(int64_t)r0 * P + i0] = j0;
    if (on1) nbr[(int64_t)r1 * P + i1] = j1;
}

// Candidates of a stencil chunk in registers: lane l holds candidates
// base + l + 32 m (m < ELL_REG_ROUNDS) of the flattened stencil; slot -1 past
// its end.  Every lane of the warp must call this.
struct CellCands {
    int4 q[ELL_REG_ROUNDS];
    int j[ELL_REG_ROUNDS];
};
__device__ __forceinline__ void load_cands(const int4* __restrict__ posq, const Stencil& st, int base,
                                           CellCands& c) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int m = 0; m < ELL_REG_ROUNDS; ++m) {
        c.j[m] = -1;
        c.q[m] = make_int4(0, 0, 0, 0);
        if (base + m * 32 < st.total) {                  // uniform
            const int t = base + m * 32 + lane;
            const int j = stencil_slot(st, t);
            if (t < st.total) {
                c.j[m] = j;
                c.q[m] = posq[j];
            }
        }
    }
}

// One chunk's candidates tested against two atoms (i0, i1; i1's results
// dropped unless `two`): accepted entries are compacted in visiting order
// through ballots into the rows' key buffers (k0, k1), counts in c0, c1.
template <bool ORTH>
__device__ __forceinline__ void sweep2(const ListBox& b, const CellCands& c, int rem, int i0, int i1, int4 q0,
                                       int4 q1, bool two, float rc2_list, uint64_t* k0, uint64_t* k1, int& c0,
                                       int& c1) {
    const unsigned FULL = 0xffffffffu;
    const unsigned below = (1u << (threadIdx.x & 31)) - 1u;
#pragma unroll
    for (int m = 0; m < ELL_REG_ROUNDS; ++m) {
        if (m * 32 >= rem) break;                        // uniform
        const int j = c.j[m];
        const float d0 = list_d2_t<ORTH>(b, q0, c.q[m]);
        const float d1 = list_d2_t<ORTH>(b, q1, c.q[m]);
        const bool a0 = j >= 0 && j != i0 && d0 < rc2_list;
        const bool a1 = two && j >= 0 && j != i1 && d1 < rc2_list;
        const unsigned m0 = __ballot_sync(FULL, a0), m1 = __ballot_sync(FULL, a1);
        const int p0 = c0 + __popc(m0 & below), p1 = c1 + __popc(m1 & below);
        if (a0 && p0 < ELL_SORT_MAX) k0[p0] = list_key(d0, j);
        if (a1 && p1 < ELL_SORT_MAX) k1[p1] = list_key(d1, j);
        c0 += __popc(m0);
        c1 += __popc(m1);
    }
}

template <bool ORTH>
__device__ __forceinline__ void ell_cell_rows(const int4* __restrict__ posq, int a0, int a1, int lin,
                                              const Stencil& st, const ListBox& b, const CellGrid& g,
                                              float rc2_list, int32_t* nbr, int64_t P, int cap, int32_t* nnbr,
                                              int32_t* flags, uint64_t* keys) {
    uint64_t* k0 = keys;
    uint64_t* k1 = keys + ELL_SORT_MAX;
    const int chunk = ELL_REG_ROUNDS * 32;
    const bool one_chunk = st.total <= chunk;
    CellCands c;
    if (one_chunk) load_cands(posq, st, 0, c);
    for (int i = a0; i < a1; i += 2) {
        const bool two = i + 1 < a1;
        const int i1 = two ? i + 1 : i;
        const int4 q0 = posq[i], q1 = posq[i1];
        int c0 = 0, c1 = 0;
        for (int base = 0; base < st.total; base += chunk) {
            if (!one_chunk) load_cands(posq, st, base, c);
            sweep2<ORTH>(b, c, st.total - base, i, i1, q0, q1, two, rc2_list, k0, k1, c0, c1);
        }
        __syncwarp();
        const int kept0 = c0 < cap ? c0 : cap;
        const int kept1 = two ? (c1 < cap ? c1 : cap) : 0;
        // rows longer than the sort buffer: built again by ell_row_warp (visiting order)
        if (kept0 > ELL_SORT_MAX) ell_row_warp(posq, i, lin, g, rc2_list, nbr, P, cap, nnbr, flags, k0);
        if (kept1 > ELL_SORT_MAX) ell_row_warp(posq, i1, lin, g, rc2_list, nbr, P, cap, nnbr, flags, k1);
        const int s0 = kept0 <= ELL_SORT_MAX ? kept0 : 0;
        const int s1 = kept1 <= ELL_SORT_MAX ? kept1 : 0;
        if (s0 <= 32 && s1 <= 32) {
            ell_write_sorted2(i, s0, k0, i1, s1, k1, nbr, P);
        } else {
            ell_write_sorted(i, s0, k0, nbr, P);
            ell_write_sorted(i1, s1, k1, nbr, P);
        }
        if (kept0 <= ELL_SORT_MAX) ell_row_done(i, c0, cap, nnbr, flags);
        if (two && kept1 <= ELL_SORT_MAX) ell_row_done(i1, c1, cap, nnbr, flags);
        __syncwarp();
    }
}

// All rows of the atoms in cell `r` (visiting rank), built by one warp: the
// cell's stencil candidates are held in registers (ELL_REG_ROUNDS per lane;
// larger stencils are swept in chunks, reloaded per pair of atoms) and each
// candidate is tested against two of the cell's atoms per sweep.  Rows come
// out equal to ell_row_warp's.  keys: ELL_KEYS entries of shared memory.
// ORTH_ONLY: every box is orthogonal (the triclinic arithmetic is left out,
// which keeps the kernel's register count down).
template <bool ORTH_ONLY>
__device__ __forceinline__ void ell_cell_warp(const int4* __restrict__ posq, int r, const int32_t* lin_of_rank,
                                              const CellGrid& g, float rc2_list, int32_t* nbr, int64_t P, int cap,
                                              int32_t* nnbr, int32_t* flags, uint64_t* keys) {
    const int a0 = g.start[r], a1 = g.start[r + 1];
    if (a0 == a1) return;
    const int lin = lin_of_rank[r];
    const Stencil st = stencil_of(g, lin);
    const ListBox b(*g.box);
    if (ORTH_ONLY || b.orth)
        ell_cell_rows<true>(posq, a0, a1, lin, st, b, g, rc2_list, nbr, P, cap, nnbr, flags, keys);
    else
        ell_cell_rows<false>(posq, a0, a1, lin, st, b, g, rc2_list, nbr, P, cap, nnbr, flags, keys);
}

}  // namespace simb200
