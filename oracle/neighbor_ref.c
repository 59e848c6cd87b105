/*
 * Oracle (TEST INFRASTRUCTURE ONLY): CPU restatement of the reference's
 * half Verlet-list search, with the exact floating-point operation order of
 * the torch CPU kernels it runs on, so the (i, j, image) pair set is bit-exact.
 *
 * Reference behaviour restated:
 *   core/neighbor_search/gpu_kdtree.py:90-155  find_neighbors_gpu_pbc_pytorch
 *       rij = pos_i - pos_j                      (:130)
 *       rij = box.minimum_image(rij)             (:104-106)
 *       d2  = (rij*rij).sum(-1)                  (:132)  -> ((x*x + y*y) + z*z)
 *       keep i < j and d2 < rc2                  (:135-139)
 *   core/box.py:109-130  minimum_image
 *       orthogonal: rij - d*round(rij/d)         (round = half-to-even = rint)
 *       triclinic : s = rij @ H_inv ; s -= round(s) ; s @ H
 *                   torch's CPU matmul for these shapes evaluates each output
 *                   column as fma(x2, M[2][k], fma(x1, M[1][k], x0*M[0][k]))
 *                   (checked empirically against torch 2.11 CPU).
 *   The pair set is emitted sorted by (i, j), the order torch.where produces.
 *   image = round(s) per axis (the lattice shift subtracted from x_i - x_j).
 *
 * Build: gcc -O2 -shared -fPIC -ffp-contract=off (contraction must be off so
 * that only the explicit fma() calls fuse).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { int64_t i, j; int32_t img[3]; } pair_t;

#define DEFINE_MINIMG(T, SUF, RINT, FMA)                                            \
static inline T minimg_##SUF(const T* r, const T* H, const T* Hi, const T* d,       \
                             int orth, T* out, int32_t* img) {                      \
    if (orth) {                                                                     \
        for (int k = 0; k < 3; ++k) {                                               \
            T q = r[k] / d[k];                                                      \
            T n = RINT(q);                                                          \
            T dn = d[k] * n;                                                        \
            out[k] = r[k] - dn;                                                     \
            img[k] = (int32_t)n;                                                    \
        }                                                                           \
    } else {                                                                        \
        T s[3];                                                                     \
        for (int k = 0; k < 3; ++k) {                                               \
            T p0 = r[0] * Hi[0 * 3 + k];                                            \
            s[k] = FMA(r[2], Hi[2 * 3 + k], FMA(r[1], Hi[1 * 3 + k], p0));          \
        }                                                                           \
        for (int k = 0; k < 3; ++k) {                                               \
            T n = RINT(s[k]);                                                       \
            img[k] = (int32_t)n;                                                    \
            s[k] = s[k] - n;                                                        \
        }                                                                           \
        for (int k = 0; k < 3; ++k) {                                               \
            T p0 = s[0] * H[0 * 3 + k];                                             \
            out[k] = FMA(s[2], H[2 * 3 + k], FMA(s[1], H[1 * 3 + k], p0));          \
        }                                                                           \
    }                                                                               \
    T x2 = out[0] * out[0];                                                         \
    T y2 = out[1] * out[1];                                                         \
    T z2 = out[2] * out[2];                                                         \
    T a = x2 + y2;                                                                  \
    return a + z2;                                                                  \
}

DEFINE_MINIMG(double, f64, rint, fma)
DEFINE_MINIMG(float, f32, rintf, fmaf)

static int cmp_pair(const void* a, const void* b) {
    const pair_t* p = (const pair_t*)a;
    const pair_t* q = (const pair_t*)b;
    if (p->i != q->i) return p->i < q->i ? -1 : 1;
    if (p->j != q->j) return p->j < q->j ? -1 : 1;
    return 0;
}

/* Shared driver.  cell_mode = 0: brute force over all j > i.
 * cell_mode = 1: 27-stencil over fractional cells (each cell at least rc wide
 * perpendicular to its faces, >= 3 cells per axis), candidate j > i tested by
 * the same expression.  Returns the number of pairs, or -(needed) when the
 * caller's capacity is too small (nothing written past cap). */
#define DEFINE_SEARCH(T, SUF)                                                        \
int64_t oracle_half_list_##SUF(const T* pos, int64_t n, const double* H64,           \
                                const double* Hi64, int orth, T rc2, int cell_mode,  \
                                const int32_t* ncell, int64_t* out_i, int64_t* out_j,\
                                int32_t* out_img, T* out_d2, int64_t cap) {          \
    T H[9], Hi[9], d[3];                                                             \
    for (int k = 0; k < 9; ++k) { H[k] = (T)H64[k]; Hi[k] = (T)Hi64[k]; }            \
    for (int k = 0; k < 3; ++k) d[k] = (T)H64[k * 3 + k];                            \
    int64_t cnt = 0, pcap = 1024;                                                    \
    pair_t* pairs = (pair_t*)malloc(sizeof(pair_t) * pcap);                          \
    T* d2s = (T*)malloc(sizeof(T) * pcap);                                           \
    int64_t* cell_of = NULL; int64_t* start = NULL; int64_t* members = NULL;         \
    int64_t nc = 0;                                                                  \
    if (cell_mode) {                                                                 \
        nc = (int64_t)ncell[0] * ncell[1] * ncell[2];                                \
        cell_of = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));              \
        start = (int64_t*)calloc((size_t)nc + 1, sizeof(int64_t));                   \
        members = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));               \
        for (int64_t a = 0; a < n; ++a) {                                            \
            int64_t c[3];                                                            \
            for (int k = 0; k < 3; ++k) {                                            \
                double s = (double)pos[a*3+0] * Hi64[0*3+k]                          \
                         + (double)pos[a*3+1] * Hi64[1*3+k]                          \
                         + (double)pos[a*3+2] * Hi64[2*3+k];                         \
                s -= floor(s);                                                       \
                int64_t ck = (int64_t)floor(s * ncell[k]);                           \
                if (ck < 0) ck = 0;                                                  \
                if (ck >= ncell[k]) ck = ncell[k] - 1;                               \
                c[k] = ck;                                                           \
            }                                                                        \
            cell_of[a] = c[0] + (int64_t)ncell[0] * (c[1] + (int64_t)ncell[1] * c[2]);\
            start[cell_of[a] + 1]++;                                                 \
        }                                                                            \
        for (int64_t c = 0; c < nc; ++c) start[c + 1] += start[c];                   \
        int64_t* fill = (int64_t*)calloc((size_t)nc, sizeof(int64_t));              \
        for (int64_t a = 0; a < n; ++a) members[start[cell_of[a]] + fill[cell_of[a]]++] = a; \
        free(fill);                                                                  \
    }                                                                                \
    for (int64_t i = 0; i < n; ++i) {                                                \
        int64_t nstencil = cell_mode ? 27 : 1;                                       \
        for (int64_t st = 0; st < nstencil; ++st) {                                  \
            int64_t jb = i + 1, je = n;                                              \
            const int64_t* list = NULL;                                              \
            if (cell_mode) {                                                         \
                int64_t ci = cell_of[i];                                             \
                int64_t cx = ci % ncell[0], cy = (ci / ncell[0]) % ncell[1];         \
                int64_t cz = ci / ((int64_t)ncell[0] * ncell[1]);                    \
                int64_t dx = st % 3 - 1, dy = (st / 3) % 3 - 1, dz = st / 9 - 1;     \
                int64_t nx = (cx + dx + ncell[0]) % ncell[0];                        \
                int64_t ny = (cy + dy + ncell[1]) % ncell[1];                        \
                int64_t nz = (cz + dz + ncell[2]) % ncell[2];                        \
                int64_t cj = nx + (int64_t)ncell[0] * (ny + (int64_t)ncell[1] * nz); \
                jb = start[cj]; je = start[cj + 1]; list = members;                  \
            }                                                                        \
            for (int64_t jj = jb; jj < je; ++jj) {                                   \
                int64_t j = list ? list[jj] : jj;                                    \
                if (j <= i) continue;                                                \
                T r[3], o[3]; int32_t img[3];                                        \
                for (int k = 0; k < 3; ++k) r[k] = pos[i*3+k] - pos[j*3+k];          \
                T d2 = minimg_##SUF(r, H, Hi, d, orth, o, img);                      \
                if (d2 < rc2) {                                                      \
                    if (cnt == pcap) {                                               \
                        pcap *= 2;                                                   \
                        pairs = (pair_t*)realloc(pairs, sizeof(pair_t) * pcap);      \
                        d2s = (T*)realloc(d2s, sizeof(T) * pcap);                    \
                    }                                                                \
                    pairs[cnt].i = i; pairs[cnt].j = j;                              \
                    memcpy(pairs[cnt].img, img, sizeof(img));                        \
                    d2s[cnt] = d2; cnt++;                                            \
                }                                                                    \
            }                                                                        \
        }                                                                            \
    }                                                                                \
    if (cell_mode) {                                                                 \
        /* sort by (i, j), then recompute d2 in sorted order (same bits) */         \
        qsort(pairs, (size_t)cnt, sizeof(pair_t), cmp_pair);                         \
        for (int64_t e = 0; e < cnt; ++e) {                                          \
            T r[3], o[3]; int32_t img[3];                                            \
            for (int k = 0; k < 3; ++k)                                              \
                r[k] = pos[pairs[e].i*3+k] - pos[pairs[e].j*3+k];                    \
            d2s[e] = minimg_##SUF(r, H, Hi, d, orth, o, img);                        \
        }                                                                            \
        free(cell_of); free(start); free(members);                                   \
    }                                                                                \
    if (cnt <= cap) {                                                                \
        for (int64_t e = 0; e < cnt; ++e) {                                          \
            out_i[e] = pairs[e].i; out_j[e] = pairs[e].j;                            \
            out_img[e*3+0] = pairs[e].img[0];                                        \
            out_img[e*3+1] = pairs[e].img[1];                                        \
            out_img[e*3+2] = pairs[e].img[2];                                        \
            out_d2[e] = d2s[e];                                                      \
        }                                                                            \
    }                                                                                \
    free(pairs); free(d2s);                                                          \
    return cnt <= cap ? cnt : -cnt;                                                  \
}

DEFINE_SEARCH(double, f64)
DEFINE_SEARCH(float, f32)
