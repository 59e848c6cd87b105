// Pair and EAM forces on the device (sm_100a).
//
// Engine kernels walk the full Verlet list (ELL, column-major) one atom per
// thread, so each atom's force, density and virial are gathered in registers
// and written once -- no atomics, and the result is bitwise reproducible.
// Each pair is evaluated from both sides; per-atom energies and virials carry
// a factor 1/2 so that the totals equal the reference's half-list sums.
//
// EAM follows EAMForceCUDAExt.forward (core/force/eam_force_cu.py:461-579):
//   pass 1: rho_i = sum_j f_{ti,tj}(r_ij) (r < rc), F(rho_i), F'(rho_i)
//   pass 2: s_ij = F'_i f'_{ti,tj}(r) + F'_j f'_{tj,ti}(r) + phi'_{ti,tj}(r)
//           f_i += -s_ij r_ij/r;  E_pair = 1/2 sum phi;  W = 1/2 sum s r;
//           W_ab = 1/2 sum f_a r_b
// with the reference's linear interpolation on uniform tables
// (eam_force_cu.py:437-459: clamp r to r_max(1-1e-7), idx = trunc, next = min(idx+1, n-1)).
//
// LJ follows LennardJonesForce.forward (core/force/lennard_jones_force.py:15-95)
// including the force-shift and quintic-switch modes.
#include "common.cuh"

namespace simb200 {

// ---------------------------------------------------------------------------
// table interpolation (reference _interp_r / _interp_rho)
struct Lerp {
    int i0, i1;
    float frac;
};
__device__ __forceinline__ Lerp lerp_r(float r, float r_hi, float inv_dr, int n_r) {
    float rc = fminf(fmaxf(r, 0.0f), r_hi);
    float idx_f = __fmul_rn(rc, inv_dr);
    int i = (int)idx_f;
    Lerp l;
    l.i0 = i;
    l.i1 = min(i + 1, n_r - 1);
    l.frac = __fsub_rn(idx_f, (float)i);
    return l;
}
__device__ __forceinline__ float lerp_at(const float* tab, const Lerp& l) {
    float v0 = tab[l.i0], v1 = tab[l.i1];
    return __fadd_rn(v0, __fmul_rn(l.frac, __fsub_rn(v1, v0)));
}
__device__ __forceinline__ void embed_lookup(const SimEAMTables& t, int ti, float rho, float& F, float& Fp) {
    float lo = t.rho_min[ti];
    float rc = fminf(fmaxf(rho, lo), t.rho_clamp_hi[ti]);
    float idx_f = __fmul_rn(__fsub_rn(rc, lo), t.inv_drho[ti]);
    int i = (int)idx_f;
    int i1 = min(i + 1, t.n_rho - 1);
    float frac = __fsub_rn(idx_f, (float)i);
    const float* e = t.embed + (size_t)ti * t.n_rho;
    const float* d = t.embed_deriv + (size_t)ti * t.n_rho;
    F = __fadd_rn(e[i], __fmul_rn(frac, __fsub_rn(e[i1], e[i])));
    Fp = __fadd_rn(d[i], __fmul_rn(frac, __fsub_rn(d[i1], d[i])));
}

__device__ __forceinline__ void pair_vector(const SimBox& b, const int4& qi, const int4& qj,
                                            float& r0, float& r1, float& r2) {
    frac_to_cart_f(b, fixed_delta(qi.x, qj.x), fixed_delta(qi.y, qj.y), fixed_delta(qi.z, qj.z), r0, r1, r2);
}

// ---------------------------------------------------------------------------
// EAM pass 1: density, embedding, F'(rho).
// Persistent grid (a few blocks per SM): each block stages the density table
// in shared memory once and then walks atom tiles with a grid stride.
template <bool SMEM>
__global__ void __launch_bounds__(SIM_THREADS) k_eam_density(SimEngine e, SimEAMTables t) {
    extern __shared__ float s_tab[];
    const float* dens = t.density;
    const int nt = t.n_types;
    if (SMEM) {
        const int total = nt * nt * t.n_r;
        for (int k = threadIdx.x; k < total; k += blockDim.x) s_tab[k] = __ldg(&t.density[k]);
        __syncthreads();
        dens = s_tab;
    }
    const SimBox& b = *e.box;
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc2 = __fmul_rn(t.cutoff, t.cutoff);
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int4 qi = posq[i];
        const int ti = qi.w;
        const int nn = e.nnbr[i];
        float rho = 0.0f;
        for (int k = 0; k < nn; ++k) {
            const int j = __ldg(&nbr[(int64_t)k * P + i]);
            const int4 qj = __ldg(&posq[j]);
            float r0, r1, r2;
            pair_vector(b, qi, qj, r0, r1, r2);
            const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
            if (d2 < rc2) {
                const float r = sqrtf(d2);
                if (r < t.cutoff) {
                    Lerp l = lerp_r(r, t.r_clamp_hi, t.inv_dr, t.n_r);
                    rho += lerp_at(dens + (size_t)(ti * nt + qj.w) * t.n_r, l);
                }
            }
        }
        float F, Fp;
        embed_lookup(t, ti, rho, F, Fp);
        e.fp[i] = Fp;
        acc += (double)F;
    }
    double vals[1] = {acc};
    block_partials<1>(vals, e.partials, SIM_RED_EPOT_EMBED);
    last_block_finalize<1>(e.partials, e.red_counter + 0, e.red_out, SIM_RED_EPOT_EMBED);
}

// EAM pass 2: forces, pair energy, virial.
// SINGLE (one element type): the three r-tables are interleaved in shared
// memory as float4 {f', phi, phi', 0} per grid point, so one pair costs two
// 16-byte shared loads; f'_{ti,tj} = f'_{tj,ti}.  Otherwise the tables are
// read through L1 from global memory.
#define EAM_FORCE_THREADS 1024
struct EamPairAcc {
    float fx = 0.f, fy = 0.f, fz = 0.f, ep = 0.f, vir = 0.f;
    float wxx = 0.f, wyy = 0.f, wzz = 0.f, wxy = 0.f, wxz = 0.f, wyz = 0.f;
    __device__ __forceinline__ void add(float s, float phi, float r, float r0, float r1, float r2) {
        const float c = -s / r;            // force on i: c * rij
        const float ax = c * r0, ay = c * r1, az = c * r2;
        fx += ax; fy += ay; fz += az;
        ep += phi;
        vir = fmaf(s, r, vir);
        wxx = fmaf(ax, r0, wxx); wyy = fmaf(ay, r1, wyy); wzz = fmaf(az, r2, wzz);
        wxy = fmaf(ax, r1, wxy); wxz = fmaf(ax, r2, wxz); wyz = fmaf(ay, r2, wyz);
    }
};

// INTEG: the epilogue also finishes the step for atom i -- the second half
// of velocity Verlet with the Langevin O-step (integrator.py:102-124) -- and
// accumulates K and sum m v(x)v, so forces never make a second trip through
// HBM for the half kick.
template <bool SINGLE, bool INTEG>
__global__ void __launch_bounds__(EAM_FORCE_THREADS, 1) k_eam_force(SimEngine e, SimEAMTables t, SimIntegrator ip) {
    extern __shared__ float4 s_tab4[];
    const int nt = t.n_types;
    if (SINGLE) {
        for (int k = threadIdx.x; k < t.n_r; k += blockDim.x)
            s_tab4[k] = make_float4(__ldg(&t.density_deriv[k]), __ldg(&t.pair[k]), __ldg(&t.pair_deriv[k]), 0.f);
        __syncthreads();
    }
    const SimBox& b = *e.box;
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int32_t* __restrict__ nbr = e.nbr;
    const float* __restrict__ fp = e.fp;
    const int64_t P = e.n_pad;
    const float rc2 = __fmul_rn(t.cutoff, t.cutoff);
    float acc[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    const uint64_t step = INTEG && ip.step_ctr ? *ip.step_ctr : 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int4 qi = posq[i];
        const int ti = qi.w;
        const float fpi = fp[i];
        const int nn = e.nnbr[i];
        EamPairAcc a;
        for (int k = 0; k < nn; ++k) {
            const int j = __ldg(&nbr[(int64_t)k * P + i]);
            const int4 qj = __ldg(&posq[j]);
            float r0, r1, r2;
            pair_vector(b, qi, qj, r0, r1, r2);
            const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
            if (d2 < rc2) {
                const float r = sqrtf(d2);
                if (r < t.cutoff) {
                    const float fpj = __ldg(&fp[j]);
                    Lerp l = lerp_r(r, t.r_clamp_hi, t.inv_dr, t.n_r);
                    if (SINGLE) {
                        const float4 v0 = s_tab4[l.i0], v1 = s_tab4[l.i1];
                        const float dd = __fadd_rn(v0.x, __fmul_rn(l.frac, __fsub_rn(v1.x, v0.x)));
                        const float phi = __fadd_rn(v0.y, __fmul_rn(l.frac, __fsub_rn(v1.y, v0.y)));
                        const float dphi = __fadd_rn(v0.z, __fmul_rn(l.frac, __fsub_rn(v1.z, v0.z)));
                        a.add(fmaf(fpi, dd, fmaf(fpj, dd, dphi)), phi, r, r0, r1, r2);
                    } else {
                        const int tj = qj.w;
                        const size_t oij = (size_t)(ti * nt + tj) * t.n_r;
                        const size_t oji = (size_t)(tj * nt + ti) * t.n_r;
                        const float d_col = lerp_at(t.density_deriv + oij, l);   // f'_{ti,tj}
                        const float d_row = lerp_at(t.density_deriv + oji, l);   // f'_{tj,ti}
                        const float phi = lerp_at(t.pair + oij, l);
                        const float dphi = lerp_at(t.pair_deriv + oij, l);
                        a.add(fmaf(fpi, d_col, fmaf(fpj, d_row, dphi)), phi, r, r0, r1, r2);
                    }
                }
            }
        }
        reinterpret_cast<float4*>(e.f32)[i] = make_float4(a.fx, a.fy, a.fz, 0.0f);
        acc[0] += a.ep; acc[1] += a.vir;
        acc[2] += a.wxx; acc[3] += a.wyy; acc[4] += a.wzz; acc[5] += a.wxy; acc[6] += a.wxz; acc[7] += a.wyz;
        bad |= !(isfinite(a.fx) && isfinite(a.fy) && isfinite(a.fz));
        if (INTEG) {
            double v[3];
            second_half_atom(e, ip, i, ti, step, (double)a.fx, (double)a.fy, (double)a.fz, v, bad);
            const double m = e.mass[ti];
            acc[8] += (float)(0.5 * m * v[0] * v[0] + 0.5 * m * v[1] * v[1] + 0.5 * m * v[2] * v[2]);
            acc[9] += (float)(m * v[0] * v[0]); acc[10] += (float)(m * v[1] * v[1]); acc[11] += (float)(m * v[2] * v[2]);
            acc[12] += (float)(m * v[0] * v[1]); acc[13] += (float)(m * v[0] * v[2]); acc[14] += (float)(m * v[1] * v[2]);
        }
    }
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
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

// ---------------------------------------------------------------------------
// LJ (engine).  FP32 variant on fixed-point displacements.
__global__ void __launch_bounds__(SIM_THREADS) k_lj_f32(SimEngine e, SimLJParams p) {
    const SimBox& b = *e.box;
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int64_t P = e.n_pad;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const float rc = (float)p.rc, rc2 = rc * rc, rs = (float)p.rs;
    double vals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (i < e.n) {
        const int4 qi = posq[i];
        const int ti = qi.w;
        const int nn = e.nnbr[i];
        float fx = 0.f, fy = 0.f, fz = 0.f, ep = 0.f, vir = 0.f;
        float wxx = 0.f, wyy = 0.f, wzz = 0.f, wxy = 0.f, wxz = 0.f, wyz = 0.f;
        for (int k = 0; k < nn; ++k) {
            const int j = __ldg(&e.nbr[(int64_t)k * P + i]);
            const int4 qj = posq[j];
            float r0, r1, r2;
            pair_vector(b, qi, qj, r0, r1, r2);
            const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
            if (d2 < rc2) {
                const int tt = ti * p.n_types + qj.w;
                const float sig = (float)p.sigma[tt];
                const float inv_r2 = 1.0f / d2;
                const float sr2 = sig * sig * inv_r2;
                const float sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
                float U = (float)p.c4eps[tt] * (sr12 - sr6);
                float Fr = (float)p.c24eps[tt] * (2.0f * sr12 - sr6) * inv_r2;   // |F|/r
                if (p.mode != SIM_LJ_RAW) {
                    const float r = sqrtf(d2);
                    if (p.mode == SIM_LJ_SHIFT) {
                        U = U - (float)p.u_rc[tt] + (r - rc) * (float)p.f_rc[tt];
                        Fr = Fr - (float)p.f_rc[tt] / r;
                    } else if (r > rs) {
                        const float x = (r - rs) / (rc - rs);
                        const float x2 = x * x, x3 = x2 * x;
                        const float S = 1.0f - 10.0f * x3 + 15.0f * x3 * x - 6.0f * x3 * x2;
                        const float dS = (-30.0f * x2 + 60.0f * x3 - 30.0f * x3 * x) / (rc - rs);
                        Fr = Fr * S - U * dS / r;
                        U = U * S;
                    }
                }
                const float ax = Fr * r0, ay = Fr * r1, az = Fr * r2;
                fx += ax; fy += ay; fz += az;
                ep += U;
                vir = fmaf(Fr, d2, vir);
                wxx = fmaf(ax, r0, wxx); wyy = fmaf(ay, r1, wyy); wzz = fmaf(az, r2, wzz);
                wxy = fmaf(ax, r1, wxy); wxz = fmaf(ax, r2, wxz); wyz = fmaf(ay, r2, wyz);
            }
        }
        reinterpret_cast<float4*>(e.f32)[i] = make_float4(fx, fy, fz, 0.0f);
        vals[0] = 0.5 * (double)ep; vals[1] = 0.5 * (double)vir;
        vals[2] = 0.5 * (double)wxx; vals[3] = 0.5 * (double)wyy; vals[4] = 0.5 * (double)wzz;
        vals[5] = 0.5 * (double)wxy; vals[6] = 0.5 * (double)wxz; vals[7] = 0.5 * (double)wyz;
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    }
    block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
    last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
}

// FP64 variant: positions from e.x, minimum image and pair arithmetic in the
// reference's order (lennard_jones_force.py:35-79), forces to e.f64.
__global__ void __launch_bounds__(SIM_THREADS) k_lj_f64(SimEngine e, SimLJParams p) {
    const SimBox& b = *e.box;
    const int64_t P = e.n_pad;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const double rc = p.rc, rs = p.rs;
    double vals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (i < e.n) {
        const double xi0 = e.x[i], xi1 = e.x[P + i], xi2 = e.x[2 * P + i];
        const int ti = e.posq[4 * i + 3];
        const int nn = e.nnbr[i];
        double fx = 0, fy = 0, fz = 0, ep = 0, vir = 0, wxx = 0, wyy = 0, wzz = 0, wxy = 0, wxz = 0, wyz = 0;
        for (int k = 0; k < nn; ++k) {
            const int j = __ldg(&e.nbr[(int64_t)k * P + i]);
            double r0 = __dsub_rn(xi0, e.x[j]), r1 = __dsub_rn(xi1, e.x[P + j]), r2 = __dsub_rn(xi2, e.x[2 * P + j]);
            min_image_f64(b, r0, r1, r2);
            double d2 = norm2_f64(r0, r1, r2);
            d2 = d2 < 1e-24 ? 1e-24 : d2;
            const double r = __dsqrt_rn(d2);
            if (!(r < rc)) continue;
            const int tt = ti * p.n_types + e.posq[4 * j + 3];
            const double inv_r = __drcp_rn(r);
            const double sr = __dmul_rn(p.sigma[tt], inv_r);
            const double sr6 = pow(sr, 6.0);
            const double sr12 = __dmul_rn(sr6, sr6);
            double U = __dmul_rn(p.c4eps[tt], __dsub_rn(sr12, sr6));
            double F = __dmul_rn(__dmul_rn(p.c24eps[tt], inv_r), __dsub_rn(__dmul_rn(2.0, sr12), sr6));
            if (p.mode == SIM_LJ_SHIFT) {
                U = __dadd_rn(__dsub_rn(U, p.u_rc[tt]), __dmul_rn(__dsub_rn(r, rc), p.f_rc[tt]));
                F = __dsub_rn(F, p.f_rc[tt]);
            } else if (p.mode == SIM_LJ_SWITCH) {
                double x = __ddiv_rn(__dsub_rn(r, rs), __dsub_rn(rc, rs));
                x = x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x);
                const double S_poly = __dsub_rn(__dadd_rn(__dsub_rn(1.0, __dmul_rn(10.0, pow(x, 3.0))),
                                                          __dmul_rn(15.0, pow(x, 4.0))),
                                                __dmul_rn(6.0, pow(x, 5.0)));
                const double dS_poly = __ddiv_rn(__dsub_rn(__dadd_rn(__dmul_rn(-30.0, pow(x, 2.0)), __dmul_rn(60.0, pow(x, 3.0))),
                                                           __dmul_rn(30.0, pow(x, 4.0))),
                                                 __dsub_rn(rc, rs));
                const bool mid = (r > rs) && (r < rc);
                const double S = r <= rs ? 1.0 : (mid ? S_poly : 0.0);
                const double dS = mid ? dS_poly : 0.0;
                F = __dsub_rn(__dmul_rn(F, S), __dmul_rn(U, dS));
                U = __dmul_rn(U, S);
            }
            const double ex = __dmul_rn(r0, inv_r), ey = __dmul_rn(r1, inv_r), ez = __dmul_rn(r2, inv_r);
            const double ax = __dmul_rn(F, ex), ay = __dmul_rn(F, ey), az = __dmul_rn(F, ez);
            fx += ax; fy += ay; fz += az;
            ep += U;
            vir += __dmul_rn(F, r);
            wxx += ax * r0; wyy += ay * r1; wzz += az * r2; wxy += ax * r1; wxz += ax * r2; wyz += ay * r2;
        }
        e.f64[i] = fx; e.f64[P + i] = fy; e.f64[2 * P + i] = fz;
        vals[0] = 0.5 * ep; vals[1] = 0.5 * vir;
        vals[2] = 0.5 * wxx; vals[3] = 0.5 * wyy; vals[4] = 0.5 * wzz;
        vals[5] = 0.5 * wxy; vals[6] = 0.5 * wxz; vals[7] = 0.5 * wyz;
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    }
    block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
    last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
}

// zero the embedding slot for pair-only force fields
__global__ void k_zero_slot(double* out, int slot) { out[slot] = 0.0; }

// ---------------------------------------------------------------------------
// legacy edge kernels (same semantics as cuda source/eam_cuda_ext_kernel.cu and
// lj_energy_force_kernel.cu; accumulate into caller-owned buffers)
__device__ __forceinline__ float legacy_lerp(float r, float inv_dr, int n_r, const float* __restrict__ tab) {
    float x = r * inv_dr;
    int i = (int)floorf(x);
    i = i < 0 ? 0 : (i > n_r - 2 ? n_r - 2 : i);
    float t = x - (float)i;
    float v0 = tab[i], v1 = tab[i + 1];
    return v0 + t * (v1 - v0);
}

__global__ void k_legacy_density(const float* __restrict__ dist, const int64_t* __restrict__ row,
                                 const int64_t* __restrict__ col, const int64_t* __restrict__ types,
                                 int64_t n_edges, const float* __restrict__ tab, int E, float inv_dr, int n_r,
                                 float* rho) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_edges; k += (int64_t)gridDim.x * blockDim.x) {
        float r = dist[k];
        int64_t a = row[k], b = col[k];
        int ta = (int)types[a], tb = (int)types[b];
        atomicAdd(rho + a, legacy_lerp(r, inv_dr, n_r, tab + (size_t)(ta * E + tb) * n_r));
        atomicAdd(rho + b, legacy_lerp(r, inv_dr, n_r, tab + (size_t)(tb * E + ta) * n_r));
    }
}

__global__ void k_legacy_force(const float* __restrict__ dist, const float* __restrict__ dvec,
                               const int64_t* __restrict__ row, const int64_t* __restrict__ col,
                               const int64_t* __restrict__ types, int64_t n_edges,
                               const float* __restrict__ dtab, const float* __restrict__ ptab,
                               const float* __restrict__ dF, int E, float inv_dr, int n_r, float* forces) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_edges; k += (int64_t)gridDim.x * blockDim.x) {
        float r = dist[k];
        int64_t a = row[k], b = col[k];
        int ta = (int)types[a], tb = (int)types[b];
        float d_ab = legacy_lerp(r, inv_dr, n_r, dtab + (size_t)(ta * E + tb) * n_r);
        float d_ba = legacy_lerp(r, inv_dr, n_r, dtab + (size_t)(tb * E + ta) * n_r);
        float dp = legacy_lerp(r, inv_dr, n_r, ptab + (size_t)(ta * E + tb) * n_r);
        float s = dF[a] * d_ab + dF[b] * d_ba + dp;
        float inv = 1.0f / (r + 1e-8f);
        float fx = -s * dvec[3 * k] * inv, fy = -s * dvec[3 * k + 1] * inv, fz = -s * dvec[3 * k + 2] * inv;
        atomicAdd(forces + 3 * a, fx); atomicAdd(forces + 3 * a + 1, fy); atomicAdd(forces + 3 * a + 2, fz);
        atomicAdd(forces + 3 * b, -fx); atomicAdd(forces + 3 * b + 1, -fy); atomicAdd(forces + 3 * b + 2, -fz);
    }
}

__global__ void k_legacy_lj(const float* __restrict__ pos, const int64_t* __restrict__ ei, const int64_t* __restrict__ ej,
                            int64_t n_edges, const float* __restrict__ sigma, const float* __restrict__ eps, float L,
                            int mode, float rc, float rs, float* forces, float* energy) {
    float e_loc = 0.f;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_edges; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = ei[k], j = ej[k];
        if (i == j) continue;
        float rx = pos[3 * i] - pos[3 * j], ry = pos[3 * i + 1] - pos[3 * j + 1], rz = pos[3 * i + 2] - pos[3 * j + 2];
        rx -= L * rintf(rx / L); ry -= L * rintf(ry / L); rz -= L * rintf(rz / L);
        float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 < 1e-12f) continue;
        float r = sqrtf(r2), inv_r = 1.0f / r, inv_r2 = 1.0f / r2, inv_r6 = inv_r2 * inv_r2 * inv_r2;
        float sg = sigma[k], ep = eps[k];
        float s6 = sg * sg * sg * sg * sg * sg, s12 = s6 * s6;
        float U = 4.0f * ep * (s12 * inv_r6 * inv_r6 - s6 * inv_r6);
        float Fm = 24.0f * ep * (2.0f * s12 * inv_r6 * inv_r6 - s6 * inv_r6) * inv_r;
        if (mode == SIM_LJ_SHIFT) {
            if (rc > 0.f && r >= rc) continue;
            float sr = sg / rc, sr6 = sr * sr * sr * sr * sr * sr, sr12 = sr6 * sr6;
            float Urc = 4.0f * ep * (sr12 - sr6);
            float Frc = 24.0f * ep * (2.0f * sr12 - sr6) / rc;
            U = U - Urc + (r - rc) * Frc;
            Fm = Fm - Frc;
        } else if (mode == SIM_LJ_SWITCH) {
            if (rc > 0.f && r >= rc) continue;
            if (r > rs) {
                float x = (r - rs) / (rc - rs), x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
                float S = 1.f - 10.f * x3 + 15.f * x4 - 6.f * x5;
                float dS = (-30.f * x2 + 60.f * x3 - 30.f * x4) / (rc - rs);
                Fm = Fm * S - U * dS;
                U = U * S;
            }
        }
        float sc = Fm * inv_r;
        atomicAdd(forces + 3 * i, sc * rx); atomicAdd(forces + 3 * i + 1, sc * ry); atomicAdd(forces + 3 * i + 2, sc * rz);
        atomicAdd(forces + 3 * j, -sc * rx); atomicAdd(forces + 3 * j + 1, -sc * ry); atomicAdd(forces + 3 * j + 2, -sc * rz);
        e_loc += U;
    }
    for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
    if ((threadIdx.x & 31) == 0 && e_loc != 0.f) atomicAdd(energy, e_loc);
}

static int grid_edges(int64_t n) {
    int64_t g = ceil_div(n, SIM_THREADS);
    return (int)(g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g));
}

}  // namespace simb200

using namespace simb200;

static size_t eam_smem_pass1(const SimEAMTables& t) { return (size_t)t.n_types * t.n_types * t.n_r * sizeof(float); }

static const size_t kSmemLimit = 200 * 1024;

// Persistent grid size: resident blocks per SM (occupancy query, once per
// configuration) times the SM count, never more than the atom tiles.
static int persistent_grid(const void* fn, int threads, size_t smem, int64_t n) {
    // occupancy queries are cached per (kernel, block, smem) so that calls made
    // while a stream is being captured only read the cache
    struct Entry { const void* fn; int threads; size_t smem; int per_sm; };
    static Entry cache[32];
    static int n_cache = 0;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    for (int k = 0; k < n_cache; ++k)
        if (cache[k].fn == fn && cache[k].threads == threads && cache[k].smem == smem) per_sm = cache[k].per_sm;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        if (n_cache < 32) cache[n_cache++] = Entry{fn, threads, smem, per_sm};
    }
    const int64_t tiles = ceil_div(n, threads);
    const int64_t g = (int64_t)per_sm * sms;
    return (int)(g < tiles ? g : (tiles < 1 ? 1 : tiles));
}

static void eam_set_attributes() {
    static bool done = false;   // first call happens before any stream capture
    if (!done) {
        cudaFuncSetAttribute(k_eam_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
        cudaFuncSetAttribute(k_eam_force<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
        cudaFuncSetAttribute(k_eam_force<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
        done = true;
    }
}

extern "C" int sim_eam_density(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    if (!ep || !tp || ep->n <= 0) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    const SimEAMTables& t = *tp;
    eam_set_attributes();
    const size_t s1 = eam_smem_pass1(t);
    if (s1 <= kSmemLimit) {
        const int g = persistent_grid((const void*)k_eam_density<true>, SIM_THREADS, s1, e.n);
        if (g > e.n_blocks_max) return SIM_ERR_ARG;
        k_eam_density<true><<<g, SIM_THREADS, s1, (cudaStream_t)stream>>>(e, t);
    } else {
        const int g = persistent_grid((const void*)k_eam_density<false>, SIM_THREADS, 0, e.n);
        if (g > e.n_blocks_max) return SIM_ERR_ARG;
        k_eam_density<false><<<g, SIM_THREADS, 0, (cudaStream_t)stream>>>(e, t);
    }
    return launch_status("sim_eam_density");
}

template <bool INTEG>
static int launch_eam_force(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip, void* stream) {
    if (!ep || !tp || ep->n <= 0) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    const SimEAMTables& t = *tp;
    SimIntegrator integ{};
    if (INTEG) {
        if (!ip || !ip->step_ctr || (ip->langevin && !ip->rff)) return SIM_ERR_ARG;
        integ = *ip;
    }
    eam_set_attributes();
    const size_t s2 = (size_t)t.n_r * sizeof(float4);
    if (t.n_types == 1 && s2 <= kSmemLimit) {
        const int g = persistent_grid((const void*)k_eam_force<true, INTEG>, EAM_FORCE_THREADS, s2, e.n);
        if (g > e.n_blocks_max) return SIM_ERR_ARG;
        k_eam_force<true, INTEG><<<g, EAM_FORCE_THREADS, s2, (cudaStream_t)stream>>>(e, t, integ);
    } else {
        const int g = persistent_grid((const void*)k_eam_force<false, INTEG>, EAM_FORCE_THREADS, 0, e.n);
        if (g > e.n_blocks_max) return SIM_ERR_ARG;
        k_eam_force<false, INTEG><<<g, EAM_FORCE_THREADS, 0, (cudaStream_t)stream>>>(e, t, integ);
    }
    return launch_status(INTEG ? "sim_eam_force_integrate" : "sim_eam_force");
}

extern "C" int sim_eam_force(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    return launch_eam_force<false>(ep, tp, nullptr, stream);
}

extern "C" int sim_eam_force_integrate(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip,
                                       void* stream) {
    return launch_eam_force<true>(ep, tp, ip, stream);
}

extern "C" int sim_eam_forces(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    int rc = sim_eam_density(ep, tp, stream);
    if (rc != SIM_OK) return rc;
    return sim_eam_force(ep, tp, stream);
}

extern "C" int sim_lj_forces(const SimEngine* ep, const SimLJParams* pp, int32_t precision, void* stream) {
    if (!ep || !pp || ep->n <= 0) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)ceil_div(e.n, SIM_THREADS);
    if (blocks > e.n_blocks_max) return SIM_ERR_ARG;
    k_zero_slot<<<1, 1, 0, st>>>(e.red_out, SIM_RED_EPOT_EMBED);
    if (precision == 1) {
        if (!e.f64) return SIM_ERR_ARG;
        k_lj_f64<<<blocks, SIM_THREADS, 0, st>>>(e, *pp);
    } else {
        k_lj_f32<<<blocks, SIM_THREADS, 0, st>>>(e, *pp);
    }
    return launch_status("sim_lj_forces");
}

extern "C" int sim_legacy_density_pass(const float* distances, const int64_t* row, const int64_t* col,
                                       const int64_t* atom_types, int64_t n_edges, const float* density_table,
                                       int32_t n_types, double inv_dr, int64_t n_r, float* rho_out, void* stream) {
    if (n_edges < 0 || n_r < 2 || n_types < 1) return SIM_ERR_ARG;
    if (n_edges == 0) return SIM_OK;
    if (!distances || !row || !col || !atom_types || !density_table || !rho_out) return SIM_ERR_ARG;
    k_legacy_density<<<grid_edges(n_edges), SIM_THREADS, 0, (cudaStream_t)stream>>>(
        distances, row, col, atom_types, n_edges, density_table, n_types, (float)inv_dr, (int)n_r, rho_out);
    return launch_status("sim_legacy_density_pass");
}

extern "C" int sim_legacy_force_pass(const float* distances, const float* dist_vec, const int64_t* row,
                                     const int64_t* col, const int64_t* atom_types, int64_t n_edges,
                                     const float* density_deriv_table, const float* pair_deriv_table,
                                     const float* dF_drho, int32_t n_types, double inv_dr, int64_t n_r,
                                     float* forces_out, void* stream) {
    if (n_edges < 0 || n_r < 2 || n_types < 1) return SIM_ERR_ARG;
    if (n_edges == 0) return SIM_OK;
    if (!distances || !dist_vec || !row || !col || !atom_types || !density_deriv_table || !pair_deriv_table ||
        !dF_drho || !forces_out)
        return SIM_ERR_ARG;
    k_legacy_force<<<grid_edges(n_edges), SIM_THREADS, 0, (cudaStream_t)stream>>>(
        distances, dist_vec, row, col, atom_types, n_edges, density_deriv_table, pair_deriv_table, dF_drho,
        n_types, (float)inv_dr, (int)n_r, forces_out);
    return launch_status("sim_legacy_force_pass");
}

extern "C" int sim_legacy_lj_energy_force(const float* pos, const int64_t* edge_i, const int64_t* edge_j,
                                          int64_t n_edges, const float* sigma, const float* epsilon,
                                          float box_length, int32_t mode, float rc, float rs, float* forces_out,
                                          float* energy_out, void* stream) {
    if (n_edges < 0 || mode < 0 || mode > 2) return SIM_ERR_ARG;
    if (n_edges == 0) return SIM_OK;
    if (!pos || !edge_i || !edge_j || !sigma || !epsilon || !forces_out || !energy_out) return SIM_ERR_ARG;
    k_legacy_lj<<<grid_edges(n_edges), SIM_THREADS, 0, (cudaStream_t)stream>>>(
        pos, edge_i, edge_j, n_edges, sigma, epsilon, box_length, mode, rc, rs, forces_out, energy_out);
    return launch_status("sim_legacy_lj_energy_force");
}
