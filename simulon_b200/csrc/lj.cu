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
#include "eam_device.cuh"

namespace simb200 {

#ifndef LJ_MIN_BLOCKS
#define LJ_MIN_BLOCKS 4   // 4 x 256 threads per SM (<= 64 registers)
#endif

// Per-pair constants of one type pair, as FP32 (the FP32 path's own rounding).
struct LJConst {
    float sig, c4, c24, urc, frc;
};
__device__ __forceinline__ LJConst lj_const(const SimLJParams& p, int tt) {
    return LJConst{(float)p.sigma[tt], (float)p.c4eps[tt], (float)p.c24eps[tt], p.u_rc ? (float)p.u_rc[tt] : 0.0f,
                   p.f_rc ? (float)p.f_rc[tt] : 0.0f};
}

// One pair (r = x_i - x_j) into atom i's force and the thread's sums
// a[0] energy, a[1] scalar virial, a[2..7] virial tensor (xx yy zz xy xz yz).
__device__ __forceinline__ void lj_pair(const SimLJParams& p, const LJConst& c, float rc, float rc2, float rs,
                                        float r0, float r1, float r2, float& fx, float& fy, float& fz,
                                        float (&a)[15]) {
    const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
    if (!(d2 < rc2)) return;
    const float inv_r2 = 1.0f / d2;
    const float sr2 = c.sig * c.sig * inv_r2;
    const float sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
    float U = c.c4 * (sr12 - sr6);
    float Fr = c.c24 * (2.0f * sr12 - sr6) * inv_r2;   // |F|/r
    if (p.mode != SIM_LJ_RAW) {
        const float r = sqrtf(d2);
        if (p.mode == SIM_LJ_SHIFT) {
            U = U - c.urc + (r - rc) * c.frc;
            Fr = Fr - c.frc / r;
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
    a[0] += U;
    a[1] = fmaf(Fr, d2, a[1]);
    a[2] = fmaf(ax, r0, a[2]); a[3] = fmaf(ay, r1, a[3]); a[4] = fmaf(az, r2, a[4]);
    a[5] = fmaf(ax, r1, a[5]); a[6] = fmaf(ax, r2, a[6]); a[7] = fmaf(ay, r2, a[7]);
}

// LJ (engine), FP32 pair arithmetic on fixed-point displacements.  Persistent
// grid; the box terms, and with one element type the pair constants, sit in
// registers; list entries are gathered four at a time.  INTEG 1 / 2: the
// integrator epilogue of the EAM force pass on atom i's finished force --
// second half of the step (Langevin O-step, half kick, K and K tensor), and
// with 2 also the next step's first half (kick, drift, posq refresh, skin/2
// trigger; step_ctr[0] advanced, step_ctr[1] = this step).
// ACC (with INTEG 0): LJ as a further force field of a sum
// (SumBackboneInterface, core/md_model.py:39-46): atom i's LJ force is added
// to the force already in e.f32 and the energy and virial sums to red_out.
template <bool ORTHO, bool SINGLE, int INTEG, bool ACC = false>
__global__ void __launch_bounds__(SIM_THREADS, LJ_MIN_BLOCKS) k_lj_f32(SimEngine e, SimLJParams p, SimIntegrator ip) {
    pdl_trigger();
    pdl_wait();   // positions, box and list come from earlier kernels
    __shared__ SimBox s_box;            // the box for the integrator epilogue, read once per block
    if (INTEG == 2) {
        if (threadIdx.x == 0) s_box = *e.box;
        __syncthreads();
    }
    const bool diag = INTEG == 2 && box_is_diagonal(s_box);
    const BoxF b(*e.box);
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc = (float)p.rc, rc2 = rc * rc, rs = (float)p.rs;
    const LJConst c1 = SINGLE ? lj_const(p, 0) : LJConst{0.f, 0.f, 0.f, 0.f, 0.f};
    float acc[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};   // as k_eam_force's
    bool bad = false, trig = false;
    const uint64_t step = INTEG && ip.step_ctr ? *ip.step_ctr : 0;
    const BlockRange br = block_range(e.n);
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        const int4 qi = posq[i];
        const int ti = qi.w;
        const int nn = e.nnbr[i];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        int k = 0;
        for (; k + 4 <= nn; k += 4) {
            int j[4];
            int4 q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) j[u] = ld_stream(&nbr[(int64_t)(k + u) * P + i]);
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] = __ldg(&posq[j[u]]);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                float r0, r1, r2;
                rvec<ORTHO>(b, qi, q[u], r0, r1, r2);
                lj_pair(p, SINGLE ? c1 : lj_const(p, ti * p.n_types + q[u].w), rc, rc2, rs, r0, r1, r2, fx, fy, fz,
                        acc);
            }
        }
        for (; k < nn; ++k) {
            const int4 qj = __ldg(&posq[ld_stream(&nbr[(int64_t)k * P + i])]);
            float r0, r1, r2;
            rvec<ORTHO>(b, qi, qj, r0, r1, r2);
            lj_pair(p, SINGLE ? c1 : lj_const(p, ti * p.n_types + qj.w), rc, rc2, rs, r0, r1, r2, fx, fy, fz, acc);
        }
        if (ACC) {
            const float4 f0 = reinterpret_cast<const float4*>(e.f32)[i];
            fx = f0.x + fx; fy = f0.y + fy; fz = f0.z + fz;
        }
        reinterpret_cast<float4*>(e.f32)[i] = make_float4(fx, fy, fz, 0.0f);
        bad |= !(isfinite(fx) && isfinite(fy) && isfinite(fz));
        if (INTEG) {
            double v[3], a[3];
            second_half_atom(e, ip, i, ti, step, (double)fx, (double)fy, (double)fz, v, bad, INTEG == 1, a);
            const double m = e.mass[ti];
            acc[8] += (float)(0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
            acc[9] += (float)(m * v[0] * v[0]); acc[10] += (float)(m * v[1] * v[1]); acc[11] += (float)(m * v[2] * v[2]);
            acc[12] += (float)(m * v[0] * v[1]); acc[13] += (float)(m * v[0] * v[2]); acc[14] += (float)(m * v[1] * v[2]);
            if (INTEG == 2) {
                // the new fixed-point record goes to posfp: other threads of this
                // pass still gather posq; k_copy_records moves it after the pass
                const double f[3] = {(double)fx, (double)fy, (double)fz};
                trig |= first_half_atom(e, s_box, ip, i, ti, f, v, bad, nullptr, e.posfp, a, diag);
            }
        }
    }
    if (INTEG == 2 && __any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    if (INTEG) {
        double vals[15];
#pragma unroll
        for (int s = 0; s < 15; ++s) vals[s] = s < 8 ? 0.5 * (double)acc[s] : (double)acc[s];
        block_partials<15>(vals, e.partials, SIM_RED_EPOT_PAIR);
        const bool last = last_block_finalize<15>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
        if (INTEG == 2 && last && threadIdx.x == 0) {
            ip.step_ctr[1] = step;
            ip.step_ctr[0] = step + 1;
        }
    } else {
        double vals[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) vals[s] = 0.5 * (double)acc[s];
        block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
        last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR, SIM_RED_SLOTS, ACC);
    }
}

// FP64 variant: positions from e.x, minimum image and pair arithmetic in the
// reference's order (lennard_jones_force.py:35-79), forces to e.f64.
// Persistent grid; with one element type the pair constants sit in
// registers; the positions of two list entries are gathered together.  The
// arithmetic of each pair and the order of the sums are those of one
// pair at a time.
struct LJConst64 {
    double sig, c4, c24, urc, frc;
};
__device__ __forceinline__ LJConst64 lj_const64(const SimLJParams& p, int tt) {
    return LJConst64{p.sigma[tt], p.c4eps[tt], p.c24eps[tt], p.u_rc ? p.u_rc[tt] : 0.0, p.f_rc ? p.f_rc[tt] : 0.0};
}

// One pair: r = x_i - x_j (raw difference, then the minimum image) into atom
// i's force and per-atom sums a[0] energy, a[1] scalar virial, a[2..7]
// virial tensor (xx yy zz xy xz yz).
__device__ __forceinline__ void lj_pair_f64(const SimBox& b, const SimLJParams& p, const LJConst64& c, double rc,
                                            double rs, double r0, double r1, double r2, double& fx, double& fy,
                                            double& fz, double (&a)[8]) {
    min_image_f64(b, r0, r1, r2);
    double d2 = norm2_f64(r0, r1, r2);
    d2 = d2 < 1e-24 ? 1e-24 : d2;
    const double r = __dsqrt_rn(d2);
    if (!(r < rc)) return;
    const double inv_r = __drcp_rn(r);
    const double sr = __dmul_rn(c.sig, inv_r);
    const double sr6 = pow(sr, 6.0);
    const double sr12 = __dmul_rn(sr6, sr6);
    double U = __dmul_rn(c.c4, __dsub_rn(sr12, sr6));
    double F = __dmul_rn(__dmul_rn(c.c24, inv_r), __dsub_rn(__dmul_rn(2.0, sr12), sr6));
    if (p.mode == SIM_LJ_SHIFT) {
        U = __dadd_rn(__dsub_rn(U, c.urc), __dmul_rn(__dsub_rn(r, rc), c.frc));
        F = __dsub_rn(F, c.frc);
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
    a[0] += U;
    a[1] += __dmul_rn(F, r);
    a[2] += ax * r0; a[3] += ay * r1; a[4] += az * r2; a[5] += ax * r1; a[6] += ax * r2; a[7] += ay * r2;
}

template <bool SINGLE>
__global__ void __launch_bounds__(SIM_THREADS) k_lj_f64(SimEngine e, SimLJParams p) {
    pdl_trigger();
    pdl_wait();   // positions, box and list come from earlier kernels
    const SimBox& b = *e.box;
    const int64_t P = e.n_pad;
    const double rc = p.rc, rs = p.rs;
    const LJConst64 c1 = SINGLE ? lj_const64(p, 0) : LJConst64{0, 0, 0, 0, 0};
    double vals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const BlockRange br = block_range(e.n);
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        const double xi0 = e.x[i], xi1 = e.x[P + i], xi2 = e.x[2 * P + i];
        const int ti = e.posq[4 * i + 3];
        const int nn = e.nnbr[i];
        double fx = 0, fy = 0, fz = 0;
        double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int k = 0;
        for (; k + 2 <= nn; k += 2) {
            const int j0 = ld_stream(&e.nbr[(int64_t)k * P + i]), j1 = ld_stream(&e.nbr[(int64_t)(k + 1) * P + i]);
            const double x00 = __ldg(&e.x[j0]), x01 = __ldg(&e.x[P + j0]), x02 = __ldg(&e.x[2 * P + j0]);
            const double x10 = __ldg(&e.x[j1]), x11 = __ldg(&e.x[P + j1]), x12 = __ldg(&e.x[2 * P + j1]);
            const LJConst64 ca = SINGLE ? c1 : lj_const64(p, ti * p.n_types + e.posq[4 * j0 + 3]);
            lj_pair_f64(b, p, ca, rc, rs, __dsub_rn(xi0, x00), __dsub_rn(xi1, x01), __dsub_rn(xi2, x02), fx, fy, fz, a);
            const LJConst64 cb = SINGLE ? c1 : lj_const64(p, ti * p.n_types + e.posq[4 * j1 + 3]);
            lj_pair_f64(b, p, cb, rc, rs, __dsub_rn(xi0, x10), __dsub_rn(xi1, x11), __dsub_rn(xi2, x12), fx, fy, fz, a);
        }
        if (k < nn) {
            const int j = ld_stream(&e.nbr[(int64_t)k * P + i]);
            const LJConst64 cc = SINGLE ? c1 : lj_const64(p, ti * p.n_types + e.posq[4 * j + 3]);
            lj_pair_f64(b, p, cc, rc, rs, __dsub_rn(xi0, __ldg(&e.x[j])), __dsub_rn(xi1, __ldg(&e.x[P + j])),
                        __dsub_rn(xi2, __ldg(&e.x[2 * P + j])), fx, fy, fz, a);
        }
        e.f64[i] = fx; e.f64[P + i] = fy; e.f64[2 * P + i] = fz;
#pragma unroll
        for (int s = 0; s < 8; ++s) vals[s] += 0.5 * a[s];
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    }
    block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
    last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
}

// zero the embedding slot for pair-only force fields
__global__ void k_zero_slot(double* out, int slot) { out[slot] = 0.0; }

// posq <- posfp for the atoms (the records a mode-2 pass wrote aside)
__global__ void k_copy_records(SimEngine e) {
    pdl_trigger();
    pdl_wait();
    const int4* __restrict__ src = reinterpret_cast<const int4*>(e.posfp);
    int4* __restrict__ dst = reinterpret_cast<int4*>(e.posq);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}
}  // namespace simb200

using namespace simb200;

template <bool ORTHO, bool SINGLE, int INTEG, bool ACC>
static int launch_lj_f32(const SimEngine& e, const SimLJParams& p, const SimIntegrator& ip, cudaStream_t st) {
    const int g = persistent_grid((const void*)k_lj_f32<ORTHO, SINGLE, INTEG, ACC>, SIM_THREADS, 0, e.n);
    if (g > e.n_blocks_max) return SIM_ERR_ARG;
    const cudaError_t err =
        launch_pdl(k_lj_f32<ORTHO, SINGLE, INTEG, ACC>, dim3(g), dim3(SIM_THREADS), 0, st, e, p, ip);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_lj_forces: launch"); return SIM_ERR_CUDA; }
    return SIM_OK;
}

template <int INTEG, bool ACC = false>
static int lj_f32(const SimEngine& e, const SimLJParams& p, const SimIntegrator& ip, cudaStream_t st) {
    const bool single = p.n_types == 1;
    if (e.box_orthogonal)
        return single ? launch_lj_f32<true, true, INTEG, ACC>(e, p, ip, st)
                      : launch_lj_f32<true, false, INTEG, ACC>(e, p, ip, st);
    return single ? launch_lj_f32<false, true, INTEG, ACC>(e, p, ip, st)
                  : launch_lj_f32<false, false, INTEG, ACC>(e, p, ip, st);
}

extern "C" int sim_lj_forces(const SimEngine* ep, const SimLJParams* pp, int32_t precision, void* stream) {
    if (!ep || !pp || ep->n <= 0) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)ceil_div(e.n, SIM_THREADS);
    k_zero_slot<<<1, 1, 0, st>>>(e.red_out, SIM_RED_EPOT_EMBED);
    if (precision == 1) {
        if (!e.f64) return SIM_ERR_ARG;
        const void* fn = pp->n_types == 1 ? (const void*)k_lj_f64<true> : (const void*)k_lj_f64<false>;
        const int g = persistent_grid(fn, SIM_THREADS, 0, e.n);
        if (g > e.n_blocks_max) return SIM_ERR_ARG;
        const cudaError_t err = pp->n_types == 1 ? launch_pdl(k_lj_f64<true>, dim3(g), dim3(SIM_THREADS), 0, st, e, *pp)
                                                 : launch_pdl(k_lj_f64<false>, dim3(g), dim3(SIM_THREADS), 0, st, e, *pp);
        if (err != cudaSuccess) { set_cuda_error(err, "sim_lj_forces: launch"); return SIM_ERR_CUDA; }
    } else {
        const int rc = lj_f32<0>(e, *pp, SimIntegrator{}, st);
        if (rc != SIM_OK) return rc;
    }
    return launch_status("sim_lj_forces");
}

extern "C" int sim_lj_forces_integrate(const SimEngine* ep, const SimLJParams* pp, const SimIntegrator* ip,
                                       int32_t mode, void* stream) {
    if (!ep || !pp || !ip || ep->n <= 0 || (mode != 1 && mode != 2) || !ip->step_ctr) return SIM_ERR_ARG;
    if (ip->langevin && !ip->rff) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_zero_slot<<<1, 1, 0, st>>>(ep->red_out, SIM_RED_EPOT_EMBED);
    if (mode == 2 && !ep->posfp) return SIM_ERR_ARG;
    const int rc = mode == 1 ? lj_f32<1>(*ep, *pp, *ip, st) : lj_f32<2>(*ep, *pp, *ip, st);
    if (rc != SIM_OK) return rc;
    if (mode == 2) {
        const int64_t blocks = ceil_div(ep->n, SIM_THREADS);
        const cudaError_t err = launch_pdl(k_copy_records, dim3((unsigned)(blocks > 148 * 16 ? 148 * 16 : blocks)),
                                           dim3(SIM_THREADS), 0, st, *ep);
        if (err != cudaSuccess) { set_cuda_error(err, "sim_lj_forces_integrate: copy"); return SIM_ERR_CUDA; }
    }
    return launch_status(mode == 1 ? "sim_lj_forces_integrate" : "sim_lj_forces_integrate (drift)");
}


extern "C" int sim_lj_forces_add(const SimEngine* ep, const SimLJParams* pp, void* stream) {
    if (!ep || !pp || ep->n <= 0) return SIM_ERR_ARG;
    const int rc = lj_f32<0, true>(*ep, *pp, SimIntegrator{}, (cudaStream_t)stream);
    if (rc != SIM_OK) return rc;
    return launch_status("sim_lj_forces_add");
}
