// Lennard-Jones forces on the engine state (sm_100a).
//
// One thread per atom walks its full Verlet list (ELL), so forces, energy and
// virial are gathered in registers and written once -- no atomics, bitwise
// reproducible.  Each pair is seen from both sides; per-atom energy and
// virial carry 1/2.  Follows LennardJonesForce.forward
// (core/force/lennard_jones_force.py:15-95): raw, force-shift ("is_fs") and
// quintic-switch ("is_switch") modes, cutoff mask r < rc, scalar virial
// sum F r and tensor sum f (x) r.
#include "common.cuh"

namespace simb200 {

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
}  // namespace simb200

using namespace simb200;

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

