// Two-pass EAM on the engine state (sm_100a).
//
// Follows EAMForceCUDAExt.forward (core/force/eam_force_cu.py:461-579):
//   pass 1: rho_i = sum_j f_{ti,tj}(r_ij) over r < rc; F(rho_i), F'(rho_i)
//   pass 2: s_ij = F'_i f'_{ti,tj}(r) + F'_j f'_{tj,ti}(r) + phi'_{ti,tj}(r);
//           f_i += -s_ij r_ij/r;  E_pair = 1/2 sum phi;  W = 1/2 sum s r;
//           W_ab = 1/2 sum f_a r_b        (scalar virial sign of eam_force_cu.py:569)
// with linear interpolation on the uniform tables of eam_force_cu.py:437-459
// (clamp r to r_max(1-1e-7), idx = trunc(r/dr), next = min(idx+1, n-1)).
//
// Design: one thread per atom over the full ELL list (no atomics, bitwise
// reproducible).  Persistent grids: each block stages its tables in shared
// memory once and walks one contiguous, warp-aligned share of the atoms
// (block_range), so every SM gets the same work.  Tables are stored as value
// + forward difference so each interpolation is one FMA, and pass 2 fetches
// {f', phi', df', dphi'} with one
// 16-byte load and interpolates f' and phi' with one packed FP32x2 FMA.
// Pass 1 writes a 16-byte record {fixed-point x, y, z, F'} per atom so pass 2
// gathers a neighbour's position and F'(rho) together.  Rows of the list are
// sorted by distance at rebuild, so a warp's lanes reach the in-cutoff and
// out-of-cutoff neighbours at the same k and rarely diverge.  Kernels are
// specialised for orthogonal boxes (three box terms in registers).
#include "common.cuh"
#include "eam_device.cuh"

namespace simb200 {

// Launch shapes (tuned on B200; overridable at compile time for sweeps)
#ifndef EAM_DENSITY_THREADS
#define EAM_DENSITY_THREADS 512
#endif
#ifndef EAM_DENSITY_MIN_BLOCKS
#define EAM_DENSITY_MIN_BLOCKS 2  // 2 x 512 threads per SM (<= 64 registers)
#endif
#ifndef EAM_CARVEOUT_PCT
#define EAM_CARVEOUT_PCT -1       // shared-memory carveout hint in percent (-1: driver default)
#endif
#ifndef EAM_DENSITY_UNROLL
#define EAM_DENSITY_UNROLL 8      // list entries gathered together in pass 1 (divides 32)
#endif
#ifndef EAM_FORCE_THREADS
#define EAM_FORCE_THREADS 1024
#endif
#ifndef EAM_FORCE_MIN_BLOCKS
#define EAM_FORCE_MIN_BLOCKS 1
#endif
#ifndef EAM_WINDOW_ROWS
#define EAM_WINDOW_ROWS 4096
#endif

// ONE: engine and tables hold a single element type.
template <bool SMEM, bool ORTHO, bool ONE>
__global__ void __launch_bounds__(EAM_DENSITY_THREADS, EAM_DENSITY_MIN_BLOCKS) k_eam_density(SimEngine e, SimEAMTables t, Window w) {
    extern __shared__ float2 s_dens[];
    pdl_trigger();
    const float2* dens = reinterpret_cast<const float2*>(t.dens_vd);
    const int nt = ONE ? 1 : t.n_types;
    if (SMEM) {
        for (int tt = 0; tt < nt * nt; ++tt)
            for (int k = threadIdx.x; k < w.n_win; k += blockDim.x)
                s_dens[tt * w.n_win + k] = __ldg(&dens[(size_t)tt * t.n_r + w.k_lo + k]);
        __syncthreads();
    }
    pdl_wait();   // the tables are constant; positions, box and list come from earlier kernels
    const BoxF b(*e.box);
    const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
    int4* __restrict__ posfp = reinterpret_cast<int4*>(e.posfp);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    const bool use_mask = e.cut_mask != nullptr && e.nbr_cap <= 64;
    double acc = 0.0;
    // one element type: the embedding grid's constants read once per thread
    // (the pass's own stores would make the compiler reload them per atom)
    float grid1[3] = {0.f, 0.f, 0.f};
    if (ONE) { grid1[0] = t.rho_min[0]; grid1[1] = t.rho_clamp_hi[0]; grid1[2] = t.inv_drho[0]; }
    const BlockRange br = block_range(e.n);
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        const int4 qi = posq[i];
        const int ti = ONE ? 0 : qi.w;
        const int nn = e.nnbr[i];
        const float2* g_i = dens + (size_t)ti * nt * t.n_r;
        const float2* s_i = s_dens + (size_t)ti * nt * w.n_win;
        float rho = 0.0f;
        uint32_t in_lo = 0, in_hi = 0;     // bit k: slot k inside the cutoff
        int k = 0;
        constexpr int U = EAM_DENSITY_UNROLL;
        for (; k + U <= nn; k += U) {
            int j[U];
            int4 q[U];
#pragma unroll
            for (int u = 0; u < U; ++u) j[u] = ld_stream(&nbr[(int64_t)(k + u) * P + i]);
#pragma unroll
            for (int u = 0; u < U; ++u) q[u] = __ldg(&posq[j[u]]);
            uint32_t bits = 0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                bool in;
                rho += density_term<SMEM, ORTHO, ONE>(b, qi, q[u], rc2, g_i, s_i, w, t, in);
                bits |= (uint32_t)in << u;
            }
            if (k < 32) in_lo |= bits << k;
            else in_hi |= bits << (k - 32);
        }
        for (; k < nn; ++k) {
            bool in;
            rho += density_term<SMEM, ORTHO, ONE>(b, qi, __ldg(&posq[ld_stream(&nbr[(int64_t)k * P + i])]), rc2, g_i,
                                                  s_i, w, t, in);
            if (k < 32) in_lo |= (uint32_t)in << k;
            else in_hi |= (uint32_t)in << (k - 32);
        }
        float F, Fp;
        embed_lookup(t, ti, rho, F, Fp, ONE ? grid1 : nullptr);
        posfp[i] = make_int4(qi.x, qi.y, qi.z, __float_as_int(Fp));
        if (use_mask) e.cut_mask[i] = ((uint64_t)in_hi << 32) | in_lo;
        acc += (double)F;
    }
    double vals[1] = {acc};
    block_partials<1>(vals, e.partials, SIM_RED_EPOT_EMBED);
    last_block_finalize<1>(e.partials, e.red_counter + 0, e.red_out, SIM_RED_EPOT_EMBED);
}

// INTEG 1: the epilogue also finishes the step for atom i -- the second half of
// velocity Verlet with the Langevin O-step (integrator.py:102-124) -- and
// accumulates K and sum m v(x)v, so the half kick needs no extra pass.
// INTEG 2: in addition the first half of the next step (kick with the same
// forces, drift, posq refresh, skin/2 trigger); the last block advances the
// step counter (step_ctr[0] = step + 1, step_ctr[1] = step for the step log).
// Pass 2 reads only posfp (pass 1's copy of the positions), so atoms can move
// while other threads still gather their neighbours.
// What the last block of a drift-fused pass 2 (INTEG 2) does to end the MD
// step on the device when sim_eam_step_drift launched it: append the step's
// log row (as k_log_step on step_ctr[1]) and, inside a captured graph, set
// the value of the conditional rebuild's IF node from the skin/2 trigger (as
// k_set_rebuild_condition).
struct StepEnd {
    const double* extra;
    double* log;                        // null: no log row
    int n_extra, cap;
    cudaGraphConditionalHandle h;
    int set_cond;                       // 0: no IF node (eager launch)
};

// IND (with INTEG 1 or 2): the spherical indenter of sim_indenter_add is added
// to atom i's force before the integrator epilogue (the same FP32 addition as
// k_indenter's, so the same trajectory), its 11 FP64 sums going to a second
// set of block partials (rows gridDim.x .. 2 gridDim.x - 1) that the last block
// finishes into ind.out and folds into red_out as k_indenter does.
template <bool SINGLE, int INTEG, bool ORTHO, bool IND = false>
__global__ void __launch_bounds__(EAM_FORCE_THREADS, EAM_FORCE_MIN_BLOCKS) k_eam_force(SimEngine e, SimEAMTables t, SimIntegrator ip,
                                                                    Window w, StepEnd end, SimIndenter ind) {
    extern __shared__ float4 s_tab4[];
    pdl_trigger();
    float4* tab_d = s_tab4;
    float2* tab_p = reinterpret_cast<float2*>(s_tab4 + w.n_win);
    if (SINGLE) {
        const float4* gd = reinterpret_cast<const float4*>(t.deriv_vd) + w.k_lo;
        const float2* gp = reinterpret_cast<const float2*>(t.pair_vd) + w.k_lo;
        for (int k = threadIdx.x; k < w.n_win; k += blockDim.x) {
            tab_d[k] = __ldg(&gd[k]);
            tab_p[k] = __ldg(&gp[k]);
        }
        __syncthreads();
    }
    pdl_wait();   // pass 1's posfp and F', the box and the list come from earlier kernels
    __shared__ SimBox s_box;            // the box for the integrator epilogue, read once per block
    if (INTEG == 2) {
        if (threadIdx.x == 0) s_box = *e.box;
        __syncthreads();
    }
    const bool diag = INTEG == 2 && box_is_diagonal(s_box);
    const BoxF b(*e.box);
    const int4* __restrict__ posfp = reinterpret_cast<const int4*>(e.posfp);
    const int32_t* __restrict__ nbr = e.nbr;
    const int64_t P = e.n_pad;
    const float rc2 = t.cutoff * t.cutoff;
    const bool use_mask = e.cut_mask != nullptr && e.nbr_cap <= 64;
    const bool spec2 = e.nbr_cap >= 2;
    float acc[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool bad = false, trig = false;
    const uint64_t step = INTEG && ip.step_ctr ? *ip.step_ctr : 0;
    double iv[IND ? 11 : 1] = {0};     // indenter: energy, force (3), contacts, virial xx yy zz xy xz yz
    const BlockRange br = block_range(e.n);
    for (int64_t i = br.begin + threadIdx.x; i < br.end; i += blockDim.x) {
        const int4 pi = posfp[i];
        const float fpi = __int_as_float(pi.w);
        const int nn = e.nnbr[i];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        int ti = 0;
        if (SINGLE && use_mask) {
            // only the slots pass 1 found inside the cutoff; the next two list
            // entries are fetched while the current pair is gathered and evaluated
            // slots 0 and 1 are nearly always the first two inside the cutoff:
            // their entries are loaded before the mask arrives and replaced
            // when the mask says otherwise (rows 0 and 1 exist: nbr_cap >= 2)
            int ja = ld_stream(&nbr[i]);
            int jb = spec2 ? ld_stream(&nbr[P + i]) : 0;
            SlotSeq m(ld_stream(&e.cut_mask[i]));
            int ka = m.next(), kb = m.next();
            if (ka != 0) ja = ka >= 0 ? ld_stream(&nbr[(int64_t)ka * P + i]) : 0;
            if (kb != 1 || !spec2) jb = kb >= 0 ? ld_stream(&nbr[(int64_t)kb * P + i]) : 0;
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
        } else if (SINGLE) {
            // the next two list entries are fetched while the current pair is
            // gathered and evaluated, so the list's DRAM latency overlaps work
            int jn0 = nn > 0 ? ld_stream(&nbr[i]) : 0;
            int jn1 = nn > 1 ? ld_stream(&nbr[P + i]) : 0;
            int k = 0;
            for (; k + 2 <= nn; k += 2) {
                const int j0 = jn0, j1 = jn1;
                if (k + 2 < nn) jn0 = ld_stream(&nbr[(int64_t)(k + 2) * P + i]);
                if (k + 3 < nn) jn1 = ld_stream(&nbr[(int64_t)(k + 3) * P + i]);
                const int4 q0 = __ldg(&posfp[j0]);
                const int4 q1 = __ldg(&posfp[j1]);
                pair_single<ORTHO>(b, pi, q0, rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
                pair_single<ORTHO>(b, pi, q1, rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
            }
            if (k < nn)
                pair_single<ORTHO>(b, pi, __ldg(&posfp[jn0]), rc2, fpi, tab_d, tab_p, w, t, fx, fy, fz, acc);
        } else {
            const int4* __restrict__ posq = reinterpret_cast<const int4*>(e.posq);
            const int nt = t.n_types;
            const float4* gd = reinterpret_cast<const float4*>(t.deriv_vd);
            const float2* gp = reinterpret_cast<const float2*>(t.pair_vd);
            ti = posq[i].w;
            SlotSeq m(use_mask ? ld_stream(&e.cut_mask[i]) : 0);
            for (int k = use_mask ? m.next() : 0; use_mask ? k >= 0 : k < nn; k = use_mask ? m.next() : k + 1) {
                const int j = ld_stream(&nbr[(int64_t)k * P + i]);
                const int4 qj = __ldg(&posfp[j]);
                float r0, r1, r2;
                rvec<ORTHO>(b, pi, qj, r0, r1, r2);
                const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
                if (!(d2 < rc2)) continue;
                const float inv_r = rsqrt_approx(d2);
                const float r = d2 * inv_r;
                const int tj = __ldg(&posq[j]).w;
                const Lerp l = lerp_r(r, t);
                const float4 dij = __ldg(&gd[(size_t)(ti * nt + tj) * t.n_r + l.k]);   // f'_{ti,tj}, phi'_{ti,tj}
                const float4 dji = __ldg(&gd[(size_t)(tj * nt + ti) * t.n_r + l.k]);   // f'_{tj,ti}
                const float2 p = __ldg(&gp[(size_t)(ti * nt + tj) * t.n_r + l.k]);
                const float d_col = fmaf(l.frac, dij.z, dij.x);
                const float d_row = fmaf(l.frac, dji.z, dji.x);
                const float dphi = fmaf(l.frac, dij.w, dij.y);
                const float phi = fmaf(l.frac, p.y, p.x);
                pair_force(fmaf(fpi, d_col, fmaf(__int_as_float(qj.w), d_row, dphi)), phi, r, inv_r, r0, r1, r2,
                           fx, fy, fz, acc);
            }
        }
        if (IND) {   // as k_indenter (indenter.py:40-68), on the positions of this step
            const int64_t P = e.n_pad;
            const double x0 = e.x[i], x1 = e.x[P + i], x2 = e.x[2 * P + i];
            const double d0 = x0 - ind.center[0], d1 = x1 - ind.center[1], d2 = x2 - ind.center[2];
            const double d = fmax(sqrt(d0 * d0 + d1 * d1 + d2 * d2), 1e-12);
            const double pen = ind.radius - d;
            if (pen > 0.0) {
                const double k = ind.stiffness * pen * pen;
                const double f0 = k * (d0 / d), f1 = k * (d1 / d), f2 = k * (d2 / d);
                fx += (float)f0; fy += (float)f1; fz += (float)f2;
                iv[0] += ind.stiffness / 3.0 * pen * pen * pen;
                iv[1] += f0; iv[2] += f1; iv[3] += f2;
                iv[4] += 1.0;
                iv[5] += f0 * x0; iv[6] += f1 * x1; iv[7] += f2 * x2;
                iv[8] += f0 * x1; iv[9] += f0 * x2; iv[10] += f1 * x2;
            }
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
                const double f[3] = {(double)fx, (double)fy, (double)fz};
                trig |= first_half_atom(e, s_box, ip, i, ti, f, v, bad, nullptr, nullptr, a, diag);   // the same F/m
            }
        }
    }
    virial_trace(acc);
    if (INTEG == 2 && __any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    if (INTEG) {
        double vals[15];
#pragma unroll
        for (int k = 0; k < 15; ++k) vals[k] = k < 8 ? 0.5 * (double)acc[k] : (double)acc[k];
        block_partials<15>(vals, e.partials, SIM_RED_EPOT_PAIR);
        double* ipart = e.partials + (size_t)gridDim.x * SIM_RED_SLOTS;
        if (IND) block_partials<IND ? 11 : 1>(iv, ipart, 0);
        const bool last = last_block_finalize<15>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
        if (IND && last) {            // uniform across the block
            __syncthreads();
            partial_sums<11>(ipart, 0, SIM_RED_SLOTS, ind.out, 0);
            __syncthreads();
            if (threadIdx.x == 0) {
                double* r = e.red_out;
                r[SIM_RED_EPOT_PAIR] += ind.out[0];
                r[SIM_RED_VIRIAL] += ind.out[5] + ind.out[6] + ind.out[7];
                for (int k = 0; k < 6; ++k) r[SIM_RED_W_XX + k] += ind.out[5 + k];
                for (int k = 1; k < 4; ++k) ind.out[k] = -ind.out[k];   // force on the indenter
            }
        }
        if (INTEG == 2 && last) {     // uniform across the block
            if (threadIdx.x == 0) {
                ip.step_ctr[1] = step;
                ip.step_ctr[0] = step + 1;
            }
            if (end.log || end.set_cond) {
                // every block's trigger and status writes preceded its fence
                // and counter increment; this block's red_out rows precede the barrier
                __syncthreads();
                const int k = threadIdx.x;
                if (end.log) {
                    double* row = end.log + (size_t)(step % (uint64_t)end.cap) * (SIM_RED_SLOTS + end.n_extra + 1);
                    if (k < SIM_RED_SLOTS) row[k] = __ldcg(&e.red_out[k]);
                    else if (k < SIM_RED_SLOTS + end.n_extra) row[k] = end.extra[k - SIM_RED_SLOTS];
                    else if (k == SIM_RED_SLOTS + end.n_extra) row[k] = (double)__ldcg(&e.flags[1]);
                }
                if (end.set_cond && k == 0) cudaGraphSetConditional(end.h, __ldcg(&e.flags[0]) != 0 ? 1u : 0u);
            }
        }
    } else {
        double vals[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) vals[k] = 0.5 * (double)acc[k];
        block_partials<8>(vals, e.partials, SIM_RED_EPOT_PAIR);
        last_block_finalize<8>(e.partials, e.red_counter + 1, e.red_out, SIM_RED_EPOT_PAIR);
    }
}

}  // namespace simb200

using namespace simb200;

static const size_t kSmemLimit = 200 * 1024;

// Rows of the r-tables kept in shared memory: the top kWindowRows (r from
// (n_r - kWindowRows) dr up to the cutoff; 2.2 A for an 8192-row table on
// [0, 4.4 A]).  A smaller footprint leaves L1 capacity for neighbour gathers.
static const int kWindowRows = EAM_WINDOW_ROWS;
static Window table_window(const SimEAMTables& t) {
    const int n_win = t.n_r < kWindowRows ? t.n_r : kWindowRows;
    return Window{t.n_r - n_win, n_win};
}
static size_t smem_pass1(const SimEAMTables& t) {
    return (size_t)t.n_types * t.n_types * table_window(t).n_win * sizeof(float2);
}
static size_t smem_pass2(const SimEAMTables& t) { return (size_t)table_window(t).n_win * (sizeof(float4) + sizeof(float2)); }

template <typename K>
static void allow_smem(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
    if (EAM_CARVEOUT_PCT >= 0)
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, EAM_CARVEOUT_PCT);
}

static void eam_set_attributes() {
    static bool done = false;   // the first call happens before any stream capture
    if (!done) {
        allow_smem(k_eam_density<true, true, true>);
        allow_smem(k_eam_density<true, false, true>);
        allow_smem(k_eam_density<true, true, false>);
        allow_smem(k_eam_density<true, false, false>);
        allow_smem(k_eam_force<true, 0, true>);
        allow_smem(k_eam_force<true, 1, true>);
        allow_smem(k_eam_force<true, 2, true>);
        allow_smem(k_eam_force<true, 0, false>);
        allow_smem(k_eam_force<true, 1, false>);
        allow_smem(k_eam_force<true, 2, false>);
        allow_smem(k_eam_force<true, 1, true, true>);
        allow_smem(k_eam_force<true, 2, true, true>);
        allow_smem(k_eam_force<true, 1, false, true>);
        allow_smem(k_eam_force<true, 2, false, true>);
        done = true;
    }
}

static bool valid_tables(const SimEAMTables& t) {
    return t.n_types >= 1 && t.n_r >= 2 && t.n_r < kMaxTableRows && t.n_rho >= 2 && t.embed && t.embed_deriv && t.rho_min && t.inv_drho &&
           t.rho_clamp_hi && t.dens_vd && t.deriv_vd && t.pair_vd;
}

// launch[0] / launch[1] choose the threads per block of pass 1 / pass 2
// (within each kernel's launch bound; 0: the built-in shape)
static int density_threads(const SimEngine& e) {
    const int t = e.launch[0];
    return t == 0 ? EAM_DENSITY_THREADS : (t == 128 || t == 256 || t == 512) && t <= EAM_DENSITY_THREADS ? t : -1;
}
static int force_threads(const SimEngine& e) {
    const int t = e.launch[1];
    return t == 0 ? EAM_FORCE_THREADS : (t == 256 || t == 512 || t == EAM_FORCE_THREADS) && t <= EAM_FORCE_THREADS ? t : -1;
}

template <bool SMEM, bool ORTHO, bool ONE>
static int launch_density1(const SimEngine& e, const SimEAMTables& t, size_t smem, cudaStream_t st) {
    const int threads = density_threads(e);
    if (threads < 0) return SIM_ERR_ARG;
    const int g = persistent_grid((const void*)k_eam_density<SMEM, ORTHO, ONE>, threads, smem, e.n);
    if (g > e.n_blocks_max) return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_eam_density<SMEM, ORTHO, ONE>, dim3(g), dim3(threads), smem, st, e, t,
                                       table_window(t));
    if (err != cudaSuccess) { set_cuda_error(err, "sim_eam_density: launch"); return SIM_ERR_CUDA; }
    return SIM_OK;
}
template <bool SMEM, bool ORTHO>
static int launch_density(const SimEngine& e, const SimEAMTables& t, size_t smem, cudaStream_t st) {
    return e.n_types == 1 && t.n_types == 1 ? launch_density1<SMEM, ORTHO, true>(e, t, smem, st)
                                            : launch_density1<SMEM, ORTHO, false>(e, t, smem, st);
}

extern "C" int sim_eam_density(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    if (!ep || !tp || ep->n <= 0 || !ep->posfp || !valid_tables(*tp) || tp->n_types > ep->n_types) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    const SimEAMTables& t = *tp;
    eam_set_attributes();
    const size_t s1 = smem_pass1(t);
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (tiled_eam_usable(e, t))
        rc = launch_eam_density_tiled(e, t, st);
    else if (s1 <= kSmemLimit)
        rc = e.box_orthogonal ? launch_density<true, true>(e, t, s1, st) : launch_density<true, false>(e, t, s1, st);
    else
        rc = e.box_orthogonal ? launch_density<false, true>(e, t, 0, st) : launch_density<false, false>(e, t, 0, st);
    if (rc != SIM_OK) return rc;
    return launch_status("sim_eam_density");
}

template <bool SINGLE, int INTEG, bool ORTHO, bool IND = false>
static int launch_force(const SimEngine& e, const SimEAMTables& t, const SimIntegrator& ip, const StepEnd& end,
                        cudaStream_t st, const SimIndenter& ind = SimIndenter{}) {
    const size_t smem = SINGLE ? smem_pass2(t) : 0;
    const int threads = force_threads(e);
    if (threads < 0) return SIM_ERR_ARG;
    const int g = persistent_grid((const void*)k_eam_force<SINGLE, INTEG, ORTHO, IND>, threads, smem, e.n);
    if (g * (IND ? 2 : 1) > e.n_blocks_max) return SIM_ERR_ARG;   // IND: a second set of block partials
    const cudaError_t err = launch_pdl(k_eam_force<SINGLE, INTEG, ORTHO, IND>, dim3(g), dim3(threads), smem, st, e, t,
                                       ip, table_window(t), end, ind);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_eam_force: launch"); return SIM_ERR_CUDA; }
    return SIM_OK;
}

template <int INTEG>
static int launch_eam_force(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip, void* stream,
                            const StepEnd& end = StepEnd{}) {
    if (!ep || !tp || ep->n <= 0 || !ep->posfp || !valid_tables(*tp)) return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    const SimEAMTables& t = *tp;
    SimIntegrator integ{};
    if (INTEG) {
        if (!ip || !ip->step_ctr || (ip->langevin && !ip->rff)) return SIM_ERR_ARG;
        integ = *ip;
    }
    eam_set_attributes();
    cudaStream_t st = (cudaStream_t)stream;
    const bool single = t.n_types == 1 && smem_pass2(t) <= kSmemLimit;
    int rc;
    const bool tiled = tiled_eam_usable(e, t);
    if (INTEG == 2 && tiled) {
        set_error_text("sim_eam_force_integrate_drift: not available with neighbour tiles (nbr16 set)");
        return SIM_ERR_ARG;
    }
    if (tiled)
        rc = launch_eam_force_tiled(e, t, INTEG ? &integ : nullptr, st);
    else if (single)
        rc = e.box_orthogonal ? launch_force<true, INTEG, true>(e, t, integ, end, st)
                              : launch_force<true, INTEG, false>(e, t, integ, end, st);
    else
        rc = e.box_orthogonal ? launch_force<false, INTEG, true>(e, t, integ, end, st)
                              : launch_force<false, INTEG, false>(e, t, integ, end, st);
    if (rc != SIM_OK) return rc;
    return launch_status(INTEG == 2 ? "sim_eam_force_integrate_drift"
                                    : (INTEG ? "sim_eam_force_integrate" : "sim_eam_force"));
}

extern "C" int sim_eam_force(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    return launch_eam_force<false>(ep, tp, nullptr, stream);
}

extern "C" int sim_eam_force_integrate(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip,
                                       void* stream) {
    return launch_eam_force<true>(ep, tp, ip, stream);
}

extern "C" int sim_eam_force_integrate_drift(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip,
                                             void* stream) {
    return launch_eam_force<2>(ep, tp, ip, stream);
}

namespace {
struct StepCtx {
    const SimEngine* e;
    const SimEAMTables* t;
    const SimIntegrator* ip;
    StepEnd end;
};
int step_pass2(const void* ctx, cudaStream_t st, const cudaGraphConditionalHandle* h) {
    const StepCtx& c = *static_cast<const StepCtx*>(ctx);
    StepEnd end = c.end;
    end.set_cond = h != nullptr;
    if (h) end.h = *h;
    return launch_eam_force<2>(c.e, c.t, c.ip, st, end);
}
int step_rebuild_body(const void* ctx, cudaStream_t s) { return rebuild_body(static_cast<const StepCtx*>(ctx)->e, s); }
int step_rebuild_eager(const void* ctx, cudaStream_t s) { return rebuild_eager(static_cast<const StepCtx*>(ctx)->e, s); }
}  // namespace

extern "C" int sim_eam_step_drift(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip,
                                  const double* extra, int32_t n_extra, double* log, int32_t log_capacity,
                                  void* stream) {
    if (!ep || !ep->box || !log || log_capacity <= 0 || n_extra < 0 || n_extra > 32 || (n_extra > 0 && !extra))
        return SIM_ERR_ARG;
    int rc = sim_eam_density(ep, tp, stream);
    if (rc != SIM_OK) return rc;
    StepCtx c{ep, tp, ip, StepEnd{extra, log, (int)n_extra, (int)log_capacity, 0, 0}};
    return launch_if_cond((cudaStream_t)stream, step_pass2, step_rebuild_body, step_rebuild_eager, &c,
                          "sim_eam_step_drift");
}

extern "C" int sim_eam_force_integrate_indenter(const SimEngine* ep, const SimEAMTables* tp,
                                                const SimIntegrator* ip, const SimIndenter* ind, int32_t mode,
                                                void* stream) {
    if (!ep || !tp || !ip || !ind || ep->n <= 0 || !ep->posfp || !valid_tables(*tp) || (mode != 1 && mode != 2))
        return SIM_ERR_ARG;
    if (!ind->center || !ind->out || !(ind->radius >= 0.0) || !ip->step_ctr || (ip->langevin && !ip->rff))
        return SIM_ERR_ARG;
    const SimEngine& e = *ep;
    const SimEAMTables& t = *tp;
    if (t.n_types != 1 || smem_pass2(t) > kSmemLimit || tiled_eam_usable(e, t)) {
        set_error_text("sim_eam_force_integrate_indenter: one element type, untiled kernels only");
        return SIM_ERR_ARG;
    }
    eam_set_attributes();
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (mode == 1)
        rc = e.box_orthogonal ? launch_force<true, 1, true, true>(e, t, *ip, StepEnd{}, st, *ind)
                              : launch_force<true, 1, false, true>(e, t, *ip, StepEnd{}, st, *ind);
    else
        rc = e.box_orthogonal ? launch_force<true, 2, true, true>(e, t, *ip, StepEnd{}, st, *ind)
                              : launch_force<true, 2, false, true>(e, t, *ip, StepEnd{}, st, *ind);
    if (rc != SIM_OK) return rc;
    return launch_status("sim_eam_force_integrate_indenter");
}

namespace {
struct StepIndCtx {
    const SimEngine* e;
    const SimEAMTables* t;
    const SimIntegrator* ip;
    const SimIndenter* ind;
    StepEnd end;
};
int step_ind_pass2(const void* ctx, cudaStream_t st, const cudaGraphConditionalHandle* h) {
    const StepIndCtx& c = *static_cast<const StepIndCtx*>(ctx);
    StepEnd end = c.end;
    end.set_cond = h != nullptr;
    if (h) end.h = *h;
    const SimEngine& e = *c.e;
    const int rc = e.box_orthogonal ? launch_force<true, 2, true, true>(e, *c.t, *c.ip, end, st, *c.ind)
                                    : launch_force<true, 2, false, true>(e, *c.t, *c.ip, end, st, *c.ind);
    return rc != SIM_OK ? rc : launch_status("sim_eam_step_drift_indenter");
}
int step_ind_body(const void* ctx, cudaStream_t s) { return rebuild_body(static_cast<const StepIndCtx*>(ctx)->e, s); }
int step_ind_eager(const void* ctx, cudaStream_t s) {
    return rebuild_eager(static_cast<const StepIndCtx*>(ctx)->e, s);
}
}  // namespace

extern "C" int sim_eam_step_drift_indenter(const SimEngine* ep, const SimEAMTables* tp, const SimIntegrator* ip,
                                           const SimIndenter* ind, const double* extra, int32_t n_extra, double* log,
                                           int32_t log_capacity, void* stream) {
    if (!ep || !ep->box || !tp || !ip || !ind || ep->n <= 0 || !ep->posfp || !valid_tables(*tp)) return SIM_ERR_ARG;
    if (!ind->center || !ind->out || !(ind->radius >= 0.0) || !ip->step_ctr || (ip->langevin && !ip->rff))
        return SIM_ERR_ARG;
    if (!log || log_capacity <= 0 || n_extra < 0 || n_extra > 32 || (n_extra > 0 && !extra)) return SIM_ERR_ARG;
    if (tp->n_types != 1 || smem_pass2(*tp) > kSmemLimit || tiled_eam_usable(*ep, *tp)) {
        set_error_text("sim_eam_step_drift_indenter: one element type, untiled kernels only");
        return SIM_ERR_ARG;
    }
    int rc = sim_eam_density(ep, tp, stream);
    if (rc != SIM_OK) return rc;
    eam_set_attributes();
    StepIndCtx c{ep, tp, ip, ind, StepEnd{extra, log, (int)n_extra, (int)log_capacity, 0, 0}};
    return launch_if_cond((cudaStream_t)stream, step_ind_pass2, step_ind_body, step_ind_eager, &c,
                          "sim_eam_step_drift_indenter");
}

extern "C" int sim_eam_forces(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    int rc = sim_eam_density(ep, tp, stream);
    if (rc != SIM_OK) return rc;
    return sim_eam_force(ep, tp, stream);
}

extern "C" int sim_autotune_eam(const SimEngine* ep, const SimEAMTables* tp, int32_t reps, float* ms, int32_t* best,
                                void* stream) {
    if (!ep || !tp || !ms || !best || reps < 1 || ep->n <= 0) return SIM_ERR_ARG;
    if (tiled_eam_usable(*ep, *tp)) {
        set_error_text("sim_autotune_eam: the neighbour-tile kernels have fixed shapes");
        return SIM_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    SimEngine e = *ep;
    const int d_cand[3] = {128, 256, 512}, f_cand[3] = {256, 512, EAM_FORCE_THREADS};
    for (int k = 0; k < 3; ++k) {
        e.launch[0] = d_cand[k];
        int rc = SIM_OK;
        ms[k] = time_launches([&] { if (rc == SIM_OK) rc = sim_eam_density(&e, tp, stream); }, reps, st);
        if (rc != SIM_OK) return rc;
    }
    e.launch[0] = ep->launch[0];
    for (int k = 0; k < 3; ++k) {
        e.launch[1] = f_cand[k];
        int rc = SIM_OK;
        ms[3 + k] = time_launches([&] { if (rc == SIM_OK) rc = sim_eam_force(&e, tp, stream); }, reps, st);
        if (rc != SIM_OK) return rc;
    }
    for (int k = 0; k < 6; ++k)
        if (ms[k] < 0.0f) return SIM_ERR_CUDA;
    int bd = 0, bf = 0;
    for (int k = 1; k < 3; ++k) {
        if (ms[k] < ms[bd]) bd = k;
        if (ms[3 + k] < ms[3 + bf]) bf = k;
    }
    best[0] = d_cand[bd];
    best[1] = f_cand[bf];
    return SIM_OK;
}

