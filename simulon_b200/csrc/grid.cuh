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

// Row i of the full list: every slot j != i of the 27 stencil cells around
// cell `lin` with d^2 < rc2_list, tested in FP32 on fixed-point displacements
// (the radius carries a 2e-6 relative margin so that an exact FP64/FP32 filter
// applied later -- half-list export, force cutoffs -- always sees a superset).
// Rows up to ELL_SORT_MAX entries are sorted nearest first, ties by slot: in a
// crystal every row then lists the same shells in the same order, so a warp's
// lanes agree on which neighbours fall inside the force cutoff.  A row longer
// than cap sets SIM_STATUS_OVERFLOW and the longest length in flags[2].
__device__ __forceinline__ void ell_row(const int4* __restrict__ posq, int64_t i, int lin, const CellGrid& g,
                                        float rc2_list, int32_t* nbr, int64_t P, int cap, int32_t* nnbr,
                                        int32_t* flags, uint32_t* key_d2, int* key_j) {
    const SimBox& b = *g.box;
    const int4 qi = posq[i];
    const int cx = lin % g.nx, cy = (lin / g.nx) % g.ny, cz = lin / (g.nx * g.ny);
    int cnt = 0;
    const int sx = stencil_count(g.nx), sy = stencil_count(g.ny), sz = stencil_count(g.nz);
    for (int kz = 0; kz < sz; ++kz) {
        const int z = stencil_cell(cz, kz, g.nz);
        for (int ky = 0; ky < sy; ++ky) {
            const int y = stencil_cell(cy, ky, g.ny);
            for (int kx = 0; kx < sx; ++kx) {
                const int xx = stencil_cell(cx, kx, g.nx);
                const int r = g.rank[xx + g.nx * (y + g.ny * z)];
                const int j0 = g.start[r], j1 = g.start[r + 1];
                for (int j = j0; j < j1; ++j) {
                    if (j == i) continue;
                    const int4 qj = posq[j];
                    float r0, r1, r2;
                    frac_to_cart_f(b, fixed_delta(qi.x, qj.x), fixed_delta(qi.y, qj.y), fixed_delta(qi.z, qj.z),
                                   r0, r1, r2);
                    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2));
                    if (d2 < rc2_list) {
                        if (cnt < cap) {
                            // non-negative floats order like their bit patterns
                            if (cnt < ELL_SORT_MAX) { key_d2[cnt] = __float_as_uint(d2); key_j[cnt] = j; }
                            nbr[(int64_t)cnt * P + i] = j;
                        }
                        ++cnt;
                    }
                }
            }
        }
    }
    const int kept = cnt < cap ? cnt : cap;
    if (kept <= ELL_SORT_MAX) {
        for (int a = 1; a < kept; ++a) {
            const uint32_t kd = key_d2[a];
            const int kj = key_j[a];
            int p = a - 1;
            while (p >= 0 && (key_d2[p] > kd || (key_d2[p] == kd && key_j[p] > kj))) {
                key_d2[p + 1] = key_d2[p];
                key_j[p + 1] = key_j[p];
                --p;
            }
            key_d2[p + 1] = kd;
            key_j[p + 1] = kj;
        }
        for (int a = 0; a < kept; ++a) nbr[(int64_t)a * P + i] = key_j[a];
    }
    nnbr[i] = kept;
    if (cnt > cap) {
        atomicOr(&flags[1], SIM_STATUS_OVERFLOW);
        atomicMax(&flags[2], cnt);
    }
}

}  // namespace simb200
