// Velocity Verlet / Langevin / Berendsen on the device, FP64 state (sm_100a).
//
// first_half  (core/integrator/integrator.py:91-99):
//     a = F/m;  v_half = v + (0.5 a) dt;  x = x + v_half dt
//   fused with the skin/2 rebuild trigger of AtomFileReader.update_coordinates
//   (io_utils/reader.py:136-163): |min_image(x - x_last)| > skin/2 for any
//   atom sets flags[0]; the fixed-point positions used by the pair kernels
//   are refreshed in the same pass.
// second_half (integrator.py:102-124):
//     v = v_half damp + xi rff (Langevin);  v = v + (0.5 a') dt;
//     K = sum 0.5 m v^2,  K_ab = sum m v_a v_b (md_model.py:83-86)
//   Langevin noise xi comes from Philox4x32-10 keyed by (seed, original atom
//   index, step), so it does not depend on the cell order.
// Berendsen (core/barostat.py:36-68): P, mu and the box update are computed on
// the device in FP64; no host round trip.
// The arithmetic order matches the reference (explicit _rn intrinsics keep
// nvcc from contracting into FMAs).
#include <cstdio>
#include <cstring>
#include "common.cuh"

namespace simb200 {

static char g_err[512] = "";

void set_cuda_error(cudaError_t err, const char* where) {
    snprintf(g_err, sizeof(g_err), "%s: %s (%s)", where, cudaGetErrorString(err), cudaGetErrorName(err));
}

void set_error_text(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

int persistent_grid(const void* fn, int threads, size_t smem, int64_t n) {
    // cached per (kernel, block, smem) so calls made while a stream is being
    // captured only read the cache
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

int launch_status(const char* where) {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_cuda_error(err, where);
        return SIM_ERR_CUDA;
    }
    return SIM_OK;
}

__device__ __forceinline__ double load_force(const SimEngine& e, int prec, int64_t i, int c) {
    if (prec == 1) return e.f64[c * e.n_pad + i];
    return (double)e.f32[4 * i + c];
}

__global__ void __launch_bounds__(SIM_THREADS) k_first_half(SimEngine e, SimIntegrator p, int prec) {
    pdl_trigger();
    pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool trigger = false, bad = false;
    if (i == 0 && p.step_ctr) *p.step_ctr += 1;   // the step index sim_integrate_second reads
    if (i < e.n) {
        const double f[3] = {load_force(e, prec, i, 0), load_force(e, prec, i, 1), load_force(e, prec, i, 2)};
        trigger = first_half_atom(e, p, i, e.posq[4 * i + 3], f, nullptr, bad);
    }
    if (__any_sync(0xffffffffu, trigger) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

__device__ __forceinline__ void ke_terms(double m, const double* v, double* vals) {
    const double hm = 0.5 * m;
    vals[0] += hm * v[0] * v[0] + hm * v[1] * v[1] + hm * v[2] * v[2];
    vals[1] += m * v[0] * v[0];
    vals[2] += m * v[1] * v[1];
    vals[3] += m * v[2] * v[2];
    vals[4] += m * v[0] * v[1];
    vals[5] += m * v[0] * v[2];
    vals[6] += m * v[1] * v[2];
}

// Second half of the step (grid-stride over the atoms): kick, Langevin O-step,
// kinetic energy and tensor.
__global__ void __launch_bounds__(SIM_THREADS) k_second_half(SimEngine e, SimIntegrator p, int prec) {
    pdl_trigger();
    pdl_wait();
    double vals[7] = {0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    const uint64_t step = *p.step_ctr;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int type = e.posq[4 * i + 3];
        double v[3];
        second_half_atom(e, p, i, type, step, load_force(e, prec, i, 0), load_force(e, prec, i, 1),
                         load_force(e, prec, i, 2), v, bad);
        ke_terms(e.mass[type], v, vals);
    }
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    block_partials<7>(vals, e.partials, SIM_RED_KE);
    last_block_finalize<7>(e.partials, e.red_counter + 2, e.red_out, SIM_RED_KE);
}

// Second half of step s and first half of step s+1 with the same forces (for
// force fields whose kernel cannot finish the step itself, e.g. one that
// scatters forces with atomics): kinetic terms of step s, then kick, drift,
// posq refresh and the skin/2 trigger; the last block advances the step
// counter (step_ctr[0] = s + 1, step_ctr[1] = s for the step log).
__global__ void __launch_bounds__(SIM_THREADS) k_second_first(SimEngine e, SimIntegrator p, int prec) {
    pdl_trigger();
    pdl_wait();
    double vals[7] = {0, 0, 0, 0, 0, 0, 0};
    bool bad = false, trig = false;
    const uint64_t step = *p.step_ctr;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int type = e.posq[4 * i + 3];
        const double f[3] = {load_force(e, prec, i, 0), load_force(e, prec, i, 1), load_force(e, prec, i, 2)};
        double v[3], a[3];
        second_half_atom(e, p, i, type, step, f[0], f[1], f[2], v, bad, false, a);
        ke_terms(e.mass[type], v, vals);
        trig |= first_half_atom(e, *e.box, p, i, type, f, v, bad, nullptr, nullptr, a);
    }
    if (__any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (bad) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
    block_partials<7>(vals, e.partials, SIM_RED_KE);
    if (last_block_finalize<7>(e.partials, e.red_counter + 2, e.red_out, SIM_RED_KE) && threadIdx.x == 0) {
        p.step_ctr[1] = step;
        p.step_ctr[0] = step + 1;
    }
}

// ---- spherical indenter (indenter.py:40-68) ----------------------------------
__global__ void __launch_bounds__(SIM_THREADS) k_indenter(SimEngine e, SimIndenter p, int prec) {
    pdl_trigger();
    pdl_wait();
    const int64_t P = e.n_pad;
    const double c0 = p.center[0], c1 = p.center[1], c2 = p.center[2];
    double vals[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < e.n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x0 = e.x[i], x1 = e.x[P + i], x2 = e.x[2 * P + i];
        const double d0 = x0 - c0, d1 = x1 - c1, d2 = x2 - c2;
        const double d = fmax(sqrt(d0 * d0 + d1 * d1 + d2 * d2), 1e-12);
        const double pen = p.radius - d;
        if (!(pen > 0.0)) continue;
        const double k = p.stiffness * pen * pen;
        const double f0 = k * (d0 / d), f1 = k * (d1 / d), f2 = k * (d2 / d);
        if (prec == 1) {
            e.f64[i] += f0;
            e.f64[P + i] += f1;
            e.f64[2 * P + i] += f2;
        } else {
            float4* f = reinterpret_cast<float4*>(e.f32) + i;
            float4 v = *f;
            v.x += (float)f0; v.y += (float)f1; v.z += (float)f2;
            *f = v;
        }
        vals[0] += p.stiffness / 3.0 * pen * pen * pen;
        vals[1] += f0; vals[2] += f1; vals[3] += f2;
        vals[4] += 1.0;
        vals[5] += f0 * x0; vals[6] += f1 * x1; vals[7] += f2 * x2;
        vals[8] += f0 * x1; vals[9] += f0 * x2; vals[10] += f1 * x2;
    }
    block_partials<11>(vals, e.partials, 0);
    if (last_block_finalize<11>(e.partials, e.red_counter + 3, p.out, 0)) {
        __syncthreads();
        if (threadIdx.x == 0) {
            double* r = e.red_out;
            r[SIM_RED_EPOT_PAIR] += p.out[0];
            r[SIM_RED_VIRIAL] += p.out[5] + p.out[6] + p.out[7];
            for (int k = 0; k < 6; ++k) r[SIM_RED_W_XX + k] += p.out[5 + k];
            for (int k = 1; k < 4; ++k) p.out[k] = -p.out[k];   // force on the indenter
        }
    }
}

// ---- anisotropic pressure control and box scaling ---------------------------
// (barostat.py:137-208, loading.py:41-80)  The new box is prepared by one
// thread into work (from double 16), the atoms are mapped through fractional
// coordinates of the old box into the new one and wrapped, then the box is
// committed.

__device__ double det3(const double* H);

__device__ __forceinline__ SimBox& work_box(double* work) { return *reinterpret_cast<SimBox*>(work + 16); }

// new box = diag(scale) H; H^-1 columns divided by the same factors
__device__ void prepare_scaled_box(const SimBox& b, const double* scale, SimBox& nb) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            nb.H[3 * r + c] = scale[r] * b.H[3 * r + c];
            nb.Hinv[3 * r + c] = b.Hinv[3 * r + c] / scale[c];
            nb.Hf[3 * r + c] = (float)nb.H[3 * r + c];
        }
    nb.orthogonal = b.orthogonal;
    nb.pad[0] = nb.pad[1] = nb.pad[2] = 0;
}

__device__ void aniso_control(const SimEngine& e, SimAniso p, double* work) {
    const SimBox& b = *e.box;
    const double* H = b.H;
    const double* r = e.red_out;
    const double V = fabs(det3(H));
    const double kt[6] = {r[SIM_RED_K_XX] + r[SIM_RED_W_XX], r[SIM_RED_K_YY] + r[SIM_RED_W_YY],
                          r[SIM_RED_K_ZZ] + r[SIM_RED_W_ZZ], r[SIM_RED_K_XY] + r[SIM_RED_W_XY],
                          r[SIM_RED_K_XZ] + r[SIM_RED_W_XZ], r[SIM_RED_K_YZ] + r[SIM_RED_W_YZ]};
    const double pm[3][3] = {{kt[0] / V, kt[3] / V, kt[4] / V}, {kt[3] / V, kt[1] / V, kt[5] / V},
                             {kt[4] / V, kt[5] / V, kt[2] / V}};
    double p_bar[3], delta[3];
    bool within[3], any_within = false;
    for (int a = 0; a < 3; ++a) {
        const double* row = H + 3 * a;
        const double nrm = fmax(sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]), 1e-12);
        const double ax[3] = {row[0] / nrm, row[1] / nrm, row[2] / nrm};
        double pa = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) pa += ax[i] * pm[i][j] * ax[j];
        p_bar[a] = pa * 1602176.6208;
        delta[a] = p_bar[a] - p.target_bar[a];
        within[a] = fabs(delta[a]) <= p.tol_bar;
        any_within |= within[a];
    }
    float z[3] = {0.f, 0.f, 0.f};
    if (p.stochastic) langevin_normals(0xA5150u, *p.counter, p.seed, z[0], z[1], z[2]);
    const double noise_sd = p.kappa_bar_inv * 8.617333262e-5 * fmax(p.temperature, 1.0) / fmax(p.tau_p, 1e-12);
    double scale[3], vscale[3];
    for (int a = 0; a < 3; ++a) {
        const double eta = p.eta_dot[a];
        double accel = p.kappa_bar_inv * (within[a] ? 0.0 : delta[a]) / fmax(p.tau_p * p.tau_p, 1e-12);
        if (p.gamma_p > 0.0) accel -= p.gamma_p * eta;
        if (p.stochastic) accel += (double)z[a] * noise_sd;
        if (any_within && within[a]) accel = -fmax(p.gamma_p, 5.0) * eta;
        double en = eta + p.dt * accel;
        en = fmin(fmax(en, -p.max_eta_dot), p.max_eta_dot);
        if (!p.control[a]) en = 0.0;
        if (within[a] && fabs(en) < 1e-7) en = 0.0;
        p.eta_dot[a] = en;
        scale[a] = p.control[a] ? exp(p.dt * en) : 1.0;
        vscale[a] = p.control[a] ? exp(-p.dt * en) : 1.0;
        work[a] = p_bar[a];
        work[3 + a] = scale[a];
        work[6 + a] = vscale[a];
    }
    if (p.stochastic) *p.counter += 1;
    prepare_scaled_box(b, scale, work_box(work));
}

__global__ void k_aniso_control(SimEngine e, SimAniso p, double* work) {
    pdl_wait();
    aniso_control(e, p, work);
}

__global__ void k_box_prepare(SimEngine e, SimBoxScale p, double* work) {
    pdl_wait();
    for (int a = 0; a < 3; ++a) {
        work[a] = 0.0;
        work[3 + a] = p.scale[a];
        work[6 + a] = p.vel_scale[a];
    }
    prepare_scaled_box(*e.box, p.scale, work_box(work));
}

// Positions through fractional coordinates of the old box into the new one,
// wrapped into [0, 1) of it (box.py:132-142), velocities scaled per Cartesian
// component (the reference applies the axis factors to columns), posq, the
// skin test and (reset) the reference reset.
__global__ void __launch_bounds__(SIM_THREADS) k_scale_atoms(SimEngine e, const double* work, int reset) {
    pdl_trigger();
    pdl_wait();
    const int64_t P = e.n_pad;
    const SimBox& ob = *e.box;
    const SimBox& nb = *reinterpret_cast<const SimBox*>(work + 16);
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool trig = false, bad = false;
    if (i < e.n) {
        double s[3], xn[3];
        cart_to_frac(ob, e.x[i], e.x[P + i], e.x[2 * P + i], s);
#pragma unroll
        for (int c = 0; c < 3; ++c) xn[c] = fma(s[2], nb.H[6 + c], fma(s[1], nb.H[3 + c], s[0] * nb.H[c]));
        if (nb.orthogonal) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double d = nb.H[4 * c];
                xn[c] = xn[c] - floor(xn[c] / d) * d;
            }
        } else {
            double t[3];
            cart_to_frac(nb, xn[0], xn[1], xn[2], t);
#pragma unroll
            for (int c = 0; c < 3; ++c) t[c] -= floor(t[c]);
#pragma unroll
            for (int c = 0; c < 3; ++c) xn[c] = fma(t[2], nb.H[6 + c], fma(t[1], nb.H[3 + c], t[0] * nb.H[c]));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double vc = e.v[c * P + i] * work[6 + c];
            e.v[c * P + i] = vc;
            bad |= !isfinite(xn[c]) || !isfinite(vc);
        }
        trig = place_atom(e, nb, i, e.posq[4 * i + 3], xn);
        if (reset) {
            e.xref[i] = e.posq[4 * i];
            e.xref[P + i] = e.posq[4 * i + 1];
            e.xref[2 * P + i] = e.posq[4 * i + 2];
        }
    }
    if (__any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

// UniaxialTensileLoader.step's bookkeeping (loading.py:41-80) on the device,
// after the box update: row lengths and the loading axis' engineering strain;
// a list rebuild requested through flags[0] (taken at the next conditional
// rebuild) when the box has deformed by more than rebuild_strain since the
// list the rule last forced (the skin test compares fractional positions, so
// it does not see an affine change); and a regrid request when a cell would
// come within regrid_margin of the list cutoff across any axis of >= 3 cells
// (the host regrids between graph replays, before the cells are too small).
// state: SIM_LOADER_STATE doubles, see simb200.h.
__device__ void loader_check(const SimEngine& e, const SimLoaderCheck& p, double* state) {
    const double* H = e.box->H;
    double len[3];
    for (int a = 0; a < 3; ++a) {
        const double* r = H + 3 * a;
        len[a] = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        state[13 + a] = len[a];
    }
    state[12] = len[p.axis] / state[9 + p.axis] - 1.0;
    // M = H inv(H_list); deviation from the identity
    const double* L = state;
    const double det = det3(L);
    double inv[9];
    inv[0] = (L[4] * L[8] - L[5] * L[7]) / det; inv[1] = (L[2] * L[7] - L[1] * L[8]) / det;
    inv[2] = (L[1] * L[5] - L[2] * L[4]) / det; inv[3] = (L[5] * L[6] - L[3] * L[8]) / det;
    inv[4] = (L[0] * L[8] - L[2] * L[6]) / det; inv[5] = (L[2] * L[3] - L[0] * L[5]) / det;
    inv[6] = (L[3] * L[7] - L[4] * L[6]) / det; inv[7] = (L[1] * L[6] - L[0] * L[7]) / det;
    inv[8] = (L[0] * L[4] - L[1] * L[3]) / det;
    double dev = 0.0;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const double m = H[3 * r] * inv[c] + H[3 * r + 1] * inv[3 + c] + H[3 * r + 2] * inv[6 + c];
            dev = fmax(dev, fabs(m - (r == c ? 1.0 : 0.0)));
        }
    if (dev > p.rebuild_strain) {
        e.flags[0] = 1;
        for (int k = 0; k < 9; ++k) state[k] = H[k];
        state[16] += 1.0;
    }
    const double V = fabs(det3(H));
    for (int a = 0; a < 3; ++a) {
        if (e.ncell[a] < 3) continue;
        const double* u = H + 3 * ((a + 1) % 3);
        const double* w = H + 3 * ((a + 2) % 3);
        const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        if (V / sqrt(cx * cx + cy * cy + cz * cz) < e.x_rc * (1.0 + p.regrid_margin) * (double)e.ncell[a])
            state[17] = 1.0;
    }
}

__global__ void k_loader_check(SimEngine e, SimLoaderCheck p, double* state) {
    pdl_wait();
    loader_check(e, p, state);
}

__global__ void k_box_commit(SimEngine e, const double* work) {
    pdl_wait();
    *e.box = *reinterpret_cast<const SimBox*>(work + 16);
}

// A loader's box update prepared on the box that an earlier update in the
// same step (the barostat's, work_prev) is about to commit: as k_box_prepare
// with work_prev's new box in place of *e.box.
__device__ void box_prepare_after(const SimBoxScale& p, const double* work_prev, double* work) {
    for (int a = 0; a < 3; ++a) {
        work[a] = 0.0;
        work[3 + a] = p.scale[a];
        work[6 + a] = p.vel_scale[a];
    }
    prepare_scaled_box(*reinterpret_cast<const SimBox*>(work_prev + 16), p.scale, work_box(work));
}
__global__ void k_box_prepare_after(SimBoxScale p, const double* work_prev, double* work) {
    pdl_wait();
    box_prepare_after(p, work_prev, work);
}

// One box update of an atom held in registers, with k_scale_atoms' arithmetic:
// position through fractional coordinates of box ob into nb and wrapped,
// velocity scaled, the skin test against the reference code xr, and (reset)
// the reference moved to the new code.
__device__ __forceinline__ bool scale_atom_regs(const SimEngine& e, const SimBox& ob, const SimBox& nb,
                                                const double* vs, double* x, double* v, uint32_t* xr, int reset,
                                                bool& bad) {
    double s[3], xn[3];
    cart_to_frac(ob, x[0], x[1], x[2], s);
#pragma unroll
    for (int c = 0; c < 3; ++c) xn[c] = fma(s[2], nb.H[6 + c], fma(s[1], nb.H[3 + c], s[0] * nb.H[c]));
    if (nb.orthogonal) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double d = nb.H[4 * c];
            xn[c] = xn[c] - floor(xn[c] / d) * d;
        }
    } else {
        double t[3];
        cart_to_frac(nb, xn[0], xn[1], xn[2], t);
#pragma unroll
        for (int c = 0; c < 3; ++c) t[c] -= floor(t[c]);
#pragma unroll
        for (int c = 0; c < 3; ++c) xn[c] = fma(t[2], nb.H[6 + c], fma(t[1], nb.H[3 + c], t[0] * nb.H[c]));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        x[c] = xn[c];
        v[c] = v[c] * vs[c];
        bad |= !isfinite(xn[c]) || !isfinite(v[c]);
    }
    // place_atom's code and skin test, in registers
    double f[3];
    cart_to_frac(nb, xn[0], xn[1], xn[2], f);
    const uint32_t q[3] = {to_fixed(f[0]), to_fixed(f[1]), to_fixed(f[2])};
    const double t0 = (double)(int32_t)(q[0] - xr[0]) * 2.3283064365386963e-10;
    const double t1 = (double)(int32_t)(q[1] - xr[1]) * 2.3283064365386963e-10;
    const double t2 = (double)(int32_t)(q[2] - xr[2]) * 2.3283064365386963e-10;
    const double d0 = t0 * nb.H[0] + t1 * nb.H[3] + t2 * nb.H[6];
    const double d1 = t0 * nb.H[1] + t1 * nb.H[4] + t2 * nb.H[7];
    const double d2 = t0 * nb.H[2] + t1 * nb.H[5] + t2 * nb.H[8];
    if (reset) {
        xr[0] = q[0]; xr[1] = q[1]; xr[2] = q[2];
    }
    return d0 * d0 + d1 * d1 + d2 * d2 > e.skin_half2;
}

// Two box updates in sequence -- the barostat's of step s (w1) then a
// loader's of step s+1 (w2, prepared by k_box_prepare_after) -- followed by
// the first half of step s+1 (as k_first_half, in box w2), in one pass over
// the atoms: the operations and their order are those of k_scale_atoms twice
// and k_first_half, so the results are the same bits.  The box is committed
// by k_box_commit(w2) afterwards.
__global__ void __launch_bounds__(SIM_THREADS) k_two_scales_first(SimEngine e, const double* w1, const double* w2,
                                                                  int reset1, int reset2, SimIntegrator p, int prec) {
    pdl_trigger();
    pdl_wait();
    const int64_t P = e.n_pad;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool trig = false, bad = false;
    if (i == 0 && p.step_ctr) *p.step_ctr += 1;   // as k_first_half
    if (i < e.n) {
        const SimBox& ob = *e.box;
        const SimBox& nb1 = *reinterpret_cast<const SimBox*>(w1 + 16);
        const SimBox& nb2 = *reinterpret_cast<const SimBox*>(w2 + 16);
        double x[3], v[3];
        uint32_t xr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = e.x[c * P + i];
            v[c] = e.v[c * P + i];
            xr[c] = (uint32_t)e.xref[c * P + i];
        }
        trig |= scale_atom_regs(e, ob, nb1, w1 + 6, x, v, xr, reset1, bad);
        trig |= scale_atom_regs(e, nb1, nb2, w2 + 6, x, v, xr, reset2, bad);
#pragma unroll
        for (int c = 0; c < 3; ++c) e.xref[c * P + i] = (int32_t)xr[c];
        const double f[3] = {load_force(e, prec, i, 0), load_force(e, prec, i, 1), load_force(e, prec, i, 2)};
        trig |= first_half_atom(e, nb2, p, i, e.posq[4 * i + 3], f, v, bad, x);
    }
    if (__any_sync(0xffffffffu, trig) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

// The end of tensile step s and the start of step s+1 with an anisotropic
// barostat (sim_tensile_link): k_link_control does on one thread what
// k_aniso_control, k_log_step and k_box_prepare_after do, in that order;
// k_two_scales_first follows; then k_link_commit does what k_box_commit,
// k_loader_check and (while capturing) k_set_rebuild_condition do.  The same
// operations in the same order as the seven launches, so the same bits.
__global__ void k_link_control(SimEngine e, SimAniso a, double* wb, const uint64_t* ctr, const double* extra,
                               int n_extra, double* log, int cap, SimBoxScale q, double* wl) {
    pdl_trigger();
    pdl_wait();
    aniso_control(e, a, wb);
    const int w = SIM_RED_SLOTS + n_extra + 1;
    double* row = log + (size_t)((ctr ? *ctr : 0) % (uint64_t)cap) * w;
    for (int k = 0; k < SIM_RED_SLOTS; ++k) row[k] = e.red_out[k];
    for (int k = 0; k < n_extra; ++k) row[SIM_RED_SLOTS + k] = extra[k];
    row[SIM_RED_SLOTS + n_extra] = (double)e.flags[1];
    box_prepare_after(q, wb, wl);
}

__global__ void k_link_commit(SimEngine e, const double* wl, SimLoaderCheck c, double* state,
                              cudaGraphConditionalHandle h, int set_cond) {
    pdl_wait();
    *e.box = *reinterpret_cast<const SimBox*>(wl + 16);
    loader_check(e, c, state);
    if (set_cond) cudaGraphSetConditional(h, e.flags[0] != 0 ? 1u : 0u);
}

static int launch_box_scale(const SimEngine& e, double* work, int reset, cudaStream_t st, const char* what) {
    cudaError_t err = launch_pdl(k_scale_atoms, dim3((unsigned)ceil_div(e.n, SIM_THREADS)), dim3(SIM_THREADS), 0, st,
                                 e, (const double*)work, reset);
    if (err == cudaSuccess) err = launch_pdl(k_box_commit, dim3(1), dim3(1), 0, st, e, (const double*)work);
    if (err != cudaSuccess) { set_cuda_error(err, what); return SIM_ERR_CUDA; }
    return launch_status(what);
}

// ---- Berendsen -------------------------------------------------------------
__device__ double det3(const double* H) {
    return H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
           H[2] * (H[3] * H[7] - H[4] * H[6]);
}

__global__ void k_berendsen_mu(SimEngine e, SimBerendsen p, double* out) {
    SimBox& b = *e.box;
    const double V = fabs(det3(b.H));
    const double* r = e.red_out;
    // stress = (K + W)/V; P = trace/3 (eV/A^3) -> bar
    const double sxx = (r[SIM_RED_K_XX] + r[SIM_RED_W_XX]) / V;
    const double syy = (r[SIM_RED_K_YY] + r[SIM_RED_W_YY]) / V;
    const double szz = (r[SIM_RED_K_ZZ] + r[SIM_RED_W_ZZ]) / V;
    const double P = ((sxx + syy) + szz) / 3.0 * 1602176.6208;
    double mu3 = 1.0 + p.kappa * (p.dt / p.tau) * (P - p.target_bar);
    const double lo = (1.0 - p.mu_max) * (1.0 - p.mu_max) * (1.0 - p.mu_max);
    const double hi = (1.0 + p.mu_max) * (1.0 + p.mu_max) * (1.0 + p.mu_max);
    mu3 = fmax(mu3, lo);
    mu3 = fmin(mu3, hi);
    const double mu = pow(mu3, 1.0 / 3.0);
    for (int k = 0; k < 9; ++k) {
        b.H[k] *= mu;
        b.Hinv[k] /= mu;
        b.Hf[k] = (float)b.H[k];
    }
    out[0] = P;
    out[1] = mu;
}

__global__ void __launch_bounds__(SIM_THREADS) k_berendsen_scale(SimEngine e, SimBerendsen p, const double* mu_p) {
    const int64_t P = e.n_pad;
    const SimBox& b = *e.box;
    const double mu = mu_p[1];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= e.n) return;
    double x[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double xc = e.x[c * P + i];
        for (int k = 0; k < p.coordinate_scale_power; ++k) xc = __dmul_rn(xc, mu);
        e.x[c * P + i] = xc;
        x[c] = xc;
        e.v[c * P + i] = __dmul_rn(e.v[c * P + i], mu);
    }
    double s[3];
    cart_to_frac(b, x[0], x[1], x[2], s);
    int4* posq = reinterpret_cast<int4*>(e.posq);
    int4 q = posq[i];
    q.x = (int32_t)to_fixed(s[0]);
    q.y = (int32_t)to_fixed(s[1]);
    q.z = (int32_t)to_fixed(s[2]);
    posq[i] = q;
    if (p.reset_reference) {
        e.xref[i] = q.x;
        e.xref[P + i] = q.y;
        e.xref[2 * P + i] = q.z;
    }
}

// The atoms' part of the previous step's Berendsen update (as k_berendsen_scale,
// with the mu that k_berendsen_mu left in mu_p[1] after scaling the box)
// followed by this step's first half (as k_first_half), in one pass: the same
// operations in the same order as the two launches, so the same bits.  The
// fixed-point code of the scaled position is needed only as the new skin
// reference; posq gets the drifted position's.
__global__ void __launch_bounds__(SIM_THREADS) k_berendsen_scale_first(SimEngine e, SimBerendsen bp,
                                                                       const double* mu_p, SimIntegrator p, int prec) {
    pdl_trigger();
    pdl_wait();
    const int64_t P = e.n_pad;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool trigger = false, bad = false;
    if (i == 0 && p.step_ctr) *p.step_ctr += 1;
    if (i < e.n) {
        const SimBox& b = *e.box;
        const double mu = mu_p[1];
        double xs[3], vs[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double xc = ld_state(&e.x[c * P + i]);
            for (int k = 0; k < bp.coordinate_scale_power; ++k) xc = __dmul_rn(xc, mu);
            xs[c] = xc;
            vs[c] = __dmul_rn(ld_state(&e.v[c * P + i]), mu);
        }
        if (bp.reset_reference) {
            double s[3];
            cart_to_frac(b, xs[0], xs[1], xs[2], s);
            e.xref[i] = (int32_t)to_fixed(s[0]);
            e.xref[P + i] = (int32_t)to_fixed(s[1]);
            e.xref[2 * P + i] = (int32_t)to_fixed(s[2]);
        }
        const double f[3] = {load_force(e, prec, i, 0), load_force(e, prec, i, 1), load_force(e, prec, i, 2)};
        trigger = first_half_atom(e, b, p, i, e.posq[4 * i + 3], f, vs, bad, xs);
    }
    if (__any_sync(0xffffffffu, trigger) && (threadIdx.x & 31) == 0) e.flags[0] = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&e.flags[1], SIM_STATUS_NONFINITE);
}

// ---- load / gather ------------------------------------------------------------
__global__ void k_load(SimEngine e, const double* __restrict__ xr, const double* __restrict__ vr,
                       const int32_t* __restrict__ types) {
    const int64_t P = e.n_pad;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        const bool live = i < e.n;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            e.x[c * P + i] = live ? xr[3 * i + c] : 0.0;
            e.v[c * P + i] = live && vr ? vr[3 * i + c] : 0.0;
            if (e.f64) e.f64[c * P + i] = 0.0;
        }
        reinterpret_cast<float4*>(e.f32)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        e.orig[i] = live ? (int32_t)i : -1;
        reinterpret_cast<int4*>(e.posq)[i] = make_int4(0, 0, 0, live ? types[i] : 0);
        e.nnbr[i] = 0;
    }
}

__global__ void k_zero_i32(int32_t* p, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = 0;
}

__global__ void k_gather_f64(SimEngine e, const double* __restrict__ src, double* __restrict__ out) {
    const int64_t P = e.n_pad;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < e.n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = e.orig[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) out[3 * o + c] = src[c * P + k];
    }
}

__global__ void k_scatter_f64(SimEngine e, const double* __restrict__ rows, double* __restrict__ dst) {
    const int64_t P = e.n_pad;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < e.n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = e.orig[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c * P + k] = rows[3 * o + c];
    }
}

__global__ void k_log_step(SimEngine e, const uint64_t* ctr, const double* extra, int n_extra, double* log, int cap) {
    pdl_trigger();
    pdl_wait();
    const int w = SIM_RED_SLOTS + n_extra + 1;
    const uint64_t s = ctr ? *ctr : 0;
    double* row = log + (size_t)(s % (uint64_t)cap) * w;
    const int t = threadIdx.x;
    if (t < SIM_RED_SLOTS) row[t] = e.red_out[t];
    else if (t < SIM_RED_SLOTS + n_extra) row[t] = extra[t - SIM_RED_SLOTS];
    else if (t == SIM_RED_SLOTS + n_extra) row[t] = (double)e.flags[1];
}

__global__ void k_gather_f32(SimEngine e, const float* __restrict__ src, double* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < e.n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = e.orig[k];
        const float4 f = reinterpret_cast<const float4*>(src)[k];
        out[3 * o] = f.x;
        out[3 * o + 1] = f.y;
        out[3 * o + 2] = f.z;
    }
}

static int grid_atoms(int64_t n) {
    int64_t g = ceil_div(n, SIM_THREADS);
    return (int)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace simb200

using namespace simb200;

extern "C" int sim_integrate_first(const SimEngine* ep, const SimIntegrator* p, int32_t force_precision, void* stream) {
    if (!ep || !p || ep->n <= 0 || (force_precision == 1 && !ep->f64)) return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_first_half, dim3((unsigned)ceil_div(ep->n, SIM_THREADS)), dim3(SIM_THREADS), 0,
                                       (cudaStream_t)stream, *ep, *p, force_precision);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_integrate_first: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_integrate_first");
}

extern "C" int sim_integrate_second(const SimEngine* ep, const SimIntegrator* p, int32_t force_precision, void* stream) {
    if (!ep || !p || ep->n <= 0 || (force_precision == 1 && !ep->f64)) return SIM_ERR_ARG;
    if (p->langevin && !p->rff) return SIM_ERR_ARG;
    int blocks = persistent_grid((const void*)k_second_half, SIM_THREADS, 0, ep->n);
    if (blocks > ep->n_blocks_max) blocks = (int)ep->n_blocks_max;
    const cudaError_t err = launch_pdl(k_second_half, dim3(blocks), dim3(SIM_THREADS), 0, (cudaStream_t)stream, *ep,
                                       *p, force_precision);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_integrate_second: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_integrate_second");
}

extern "C" int sim_integrate_second_first(const SimEngine* ep, const SimIntegrator* p, int32_t force_precision,
                                          void* stream) {
    if (!ep || !p || ep->n <= 0 || !p->step_ctr || (force_precision == 1 && !ep->f64)) return SIM_ERR_ARG;
    if (p->langevin && !p->rff) return SIM_ERR_ARG;
    int blocks = persistent_grid((const void*)k_second_first, SIM_THREADS, 0, ep->n);
    if (blocks > ep->n_blocks_max) blocks = (int)ep->n_blocks_max;
    const cudaError_t err = launch_pdl(k_second_first, dim3(blocks), dim3(SIM_THREADS), 0, (cudaStream_t)stream, *ep,
                                       *p, force_precision);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_integrate_second_first: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_integrate_second_first");
}

extern "C" int sim_berendsen(const SimEngine* ep, const SimBerendsen* p, double* pressure_out, void* stream) {
    if (!ep || !p || !pressure_out || p->tau <= 0.0) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_berendsen_mu<<<1, 1, 0, st>>>(*ep, *p, pressure_out);
    k_berendsen_scale<<<(int)ceil_div(ep->n, SIM_THREADS), SIM_THREADS, 0, st>>>(*ep, *p, pressure_out);
    return launch_status("sim_berendsen");
}

extern "C" int sim_berendsen_mu(const SimEngine* ep, const SimBerendsen* p, double* pressure_out, void* stream) {
    if (!ep || !p || !pressure_out || p->tau <= 0.0) return SIM_ERR_ARG;
    k_berendsen_mu<<<1, 1, 0, (cudaStream_t)stream>>>(*ep, *p, pressure_out);
    return launch_status("sim_berendsen_mu");
}

extern "C" int sim_berendsen_scale_first(const SimEngine* ep, const SimBerendsen* bp, const double* mu_in,
                                         const SimIntegrator* p, int32_t force_precision, void* stream) {
    if (!ep || !bp || !mu_in || !p || ep->n <= 0 || (force_precision == 1 && !ep->f64)) return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_berendsen_scale_first, dim3((unsigned)ceil_div(ep->n, SIM_THREADS)),
                                       dim3(SIM_THREADS), 0, (cudaStream_t)stream, *ep, *bp, mu_in, *p,
                                       force_precision);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_berendsen_scale_first: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_berendsen_scale_first");
}

extern "C" int sim_engine_load(const SimEngine* ep, const double* x_rows, const double* v_rows, const int32_t* types,
                               void* stream) {
    if (!ep || !x_rows || !types || ep->n <= 0 || ep->n_pad < ep->n || (ep->n_pad % 128) != 0) return SIM_ERR_ARG;
    if (ep->nbr_cap <= 0 || ep->n_cells <= 0) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const SimEngine& e = *ep;
    prepare_capture_stream();   // outside any capture: create the IF-body capture stream once
    k_load<<<grid_atoms(e.n_pad), SIM_THREADS, 0, st>>>(e, x_rows, v_rows, types);
    k_zero_i32<<<grid_atoms(e.n_cells + 1), SIM_THREADS, 0, st>>>(e.cell_count, e.n_cells + 1);
    k_zero_i32<<<1, 32, 0, st>>>(e.flags, 8);
    k_zero_i32<<<1, 32, 0, st>>>((int32_t*)e.red_counter, 4);
    int rc = launch_status("sim_engine_load");
    if (rc != SIM_OK) return rc;
    return sim_rebuild(ep, 0, stream);
}

extern "C" int sim_gather_original_f64(const SimEngine* ep, const double* src_soa, double* out_rows, void* stream) {
    if (!ep || !src_soa || !out_rows) return SIM_ERR_ARG;
    k_gather_f64<<<grid_atoms(ep->n), SIM_THREADS, 0, (cudaStream_t)stream>>>(*ep, src_soa, out_rows);
    return launch_status("sim_gather_original_f64");
}

extern "C" int sim_scatter_original_f64(const SimEngine* ep, const double* rows, double* dst_soa, void* stream) {
    if (!ep || !rows || !dst_soa) return SIM_ERR_ARG;
    k_scatter_f64<<<grid_atoms(ep->n), SIM_THREADS, 0, (cudaStream_t)stream>>>(*ep, rows, dst_soa);
    return launch_status("sim_scatter_original_f64");
}

extern "C" int sim_log_step(const SimEngine* ep, const uint64_t* step_ctr, const double* extra, int32_t n_extra,
                            double* log, int32_t capacity, void* stream) {
    if (!ep || !log || capacity <= 0 || n_extra < 0 || n_extra > 32 || (n_extra > 0 && !extra)) return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_log_step, dim3(1), dim3(64), 0, (cudaStream_t)stream, *ep, step_ctr, extra,
                                       n_extra, log, capacity);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_log_step: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_log_step");
}

extern "C" int sim_gather_original_f32(const SimEngine* ep, const float* src_soa, double* out_rows, void* stream) {
    if (!ep || !src_soa || !out_rows) return SIM_ERR_ARG;
    k_gather_f32<<<grid_atoms(ep->n), SIM_THREADS, 0, (cudaStream_t)stream>>>(*ep, src_soa, out_rows);
    return launch_status("sim_gather_original_f32");
}

extern "C" const char* sim_last_cuda_error(void) { return g_err; }
extern "C" int sim_version(void) { return 1; }

extern "C" int sim_struct_sizes(int64_t* out, int32_t n) {
    const int64_t sizes[14] = {(int64_t)sizeof(SimBox), (int64_t)sizeof(SimEngine), (int64_t)sizeof(SimEAMTables),
                               (int64_t)sizeof(SimLJParams), (int64_t)sizeof(SimIntegrator),
                               (int64_t)sizeof(SimBerendsen), (int64_t)sizeof(SimRep), (int64_t)sizeof(SimBatch),
                               (int64_t)sizeof(SimMLP), (int64_t)sizeof(SimAniso), (int64_t)sizeof(SimBoxScale),
                               (int64_t)sizeof(SimIndenter), (int64_t)sizeof(SimCrack),
                               (int64_t)sizeof(SimLoaderCheck)};
    if (!out || n < 13) return SIM_ERR_ARG;
    for (int k = 0; k < 14 && k < n; ++k) out[k] = sizes[k];
    return SIM_OK;
}

extern "C" int sim_aniso_npt(const SimEngine* ep, const SimAniso* p, double* work, void* stream) {
    if (!ep || !p || !work || ep->n <= 0 || !p->eta_dot || (p->stochastic && !p->counter)) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const cudaError_t err = launch_pdl(k_aniso_control, dim3(1), dim3(1), 0, st, *ep, *p, work);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_aniso_npt: control"); return SIM_ERR_CUDA; }
    return launch_box_scale(*ep, work, p->reset_reference, st, "sim_aniso_npt");
}

extern "C" int sim_box_scale(const SimEngine* ep, const SimBoxScale* p, double* work, void* stream) {
    if (!ep || !p || !work || ep->n <= 0) return SIM_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (!(p->scale[a] > 0.0) || !(p->vel_scale[a] > 0.0)) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const cudaError_t err = launch_pdl(k_box_prepare, dim3(1), dim3(1), 0, st, *ep, *p, work);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_box_scale: prepare"); return SIM_ERR_CUDA; }
    return launch_box_scale(*ep, work, p->reset_reference, st, "sim_box_scale");
}

extern "C" int sim_indenter_add(const SimEngine* ep, const SimIndenter* p, int32_t force_precision, void* stream) {
    if (!ep || !p || !p->center || !p->out || ep->n <= 0 || (force_precision == 1 && !ep->f64) ||
        !(p->radius >= 0.0))
        return SIM_ERR_ARG;
    int blocks = persistent_grid((const void*)k_indenter, SIM_THREADS, 0, ep->n);
    if (blocks > ep->n_blocks_max) blocks = (int)ep->n_blocks_max;
    const cudaError_t err = launch_pdl(k_indenter, dim3(blocks), dim3(SIM_THREADS), 0, (cudaStream_t)stream, *ep, *p,
                                       force_precision);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_indenter_add: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_indenter_add");
}


namespace {
struct LinkCtx {
    const SimEngine* e;
    const SimAniso* a;
    double* wb;
    const uint64_t* ctr;
    const double* extra;
    int n_extra;
    double* log;
    int cap;
    const SimBoxScale* q;
    double* wl;
    const SimIntegrator* ip;
    int prec;
    const SimLoaderCheck* c;
    double* state;
};

int link_cond(const void* ctx, cudaStream_t st, const cudaGraphConditionalHandle* h) {
    const LinkCtx& c = *static_cast<const LinkCtx*>(ctx);
    const SimEngine& e = *c.e;
    cudaError_t err = launch_pdl(k_link_control, dim3(1), dim3(1), 0, st, e, *c.a, c.wb, c.ctr, c.extra, c.n_extra,
                                 c.log, c.cap, *c.q, c.wl);
    if (err == cudaSuccess)
        err = launch_pdl(k_two_scales_first, dim3((unsigned)ceil_div(e.n, SIM_THREADS)), dim3(SIM_THREADS), 0, st, e,
                         (const double*)c.wb, (const double*)c.wl, (int)c.a->reset_reference,
                         (int)c.q->reset_reference, *c.ip, c.prec);
    if (err == cudaSuccess)
        err = launch_pdl(k_link_commit, dim3(1), dim3(1), 0, st, e, (const double*)c.wl, *c.c, c.state,
                         h ? *h : (cudaGraphConditionalHandle)0, h ? 1 : 0);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_tensile_link: launch"); return SIM_ERR_CUDA; }
    return SIM_OK;
}
int link_body(const void* ctx, cudaStream_t s) { return sim_rebuild(static_cast<const LinkCtx*>(ctx)->e, 0, s); }
int link_eager(const void* ctx, cudaStream_t s) { return sim_rebuild(static_cast<const LinkCtx*>(ctx)->e, 1, s); }
}  // namespace

extern "C" int sim_tensile_link(const SimEngine* ep, const SimAniso* baro, double* work_baro, const uint64_t* step_ctr,
                                const double* extra, int32_t n_extra, double* log, int32_t capacity,
                                const SimBoxScale* load, double* work_load, const SimIntegrator* integ,
                                int32_t force_precision, const SimLoaderCheck* check, double* state, void* stream) {
    if (!ep || !ep->box || ep->n <= 0 || !baro || !work_baro || !baro->eta_dot || (baro->stochastic && !baro->counter))
        return SIM_ERR_ARG;
    if (!log || capacity <= 0 || n_extra < 0 || n_extra > 32 || (n_extra > 0 && !extra)) return SIM_ERR_ARG;
    if (!load || !work_load || !integ || (force_precision == 1 && !ep->f64)) return SIM_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (!(load->scale[a] > 0.0) || !(load->vel_scale[a] > 0.0)) return SIM_ERR_ARG;
    if (!check || !state || check->axis < 0 || check->axis > 2 || !(check->rebuild_strain >= 0.0) ||
        !(check->regrid_margin >= 0.0))
        return SIM_ERR_ARG;
    const LinkCtx c{ep, baro, work_baro, step_ctr, extra, (int)n_extra, log, (int)capacity, load, work_load, integ,
                    (int)force_precision, check, state};
    return launch_if_cond((cudaStream_t)stream, link_cond, link_body, link_eager, &c, "sim_tensile_link");
}

extern "C" int sim_loader_check(const SimEngine* ep, const SimLoaderCheck* p, double* state, void* stream) {
    if (!ep || !p || !state || p->axis < 0 || p->axis > 2 || !(p->rebuild_strain >= 0.0) ||
        !(p->regrid_margin >= 0.0))
        return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_loader_check, dim3(1), dim3(1), 0, (cudaStream_t)stream, *ep, *p, state);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_loader_check: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_loader_check");
}

extern "C" int sim_aniso_control(const SimEngine* ep, const SimAniso* p, double* work, void* stream) {
    if (!ep || !p || !work || ep->n <= 0 || !p->eta_dot || (p->stochastic && !p->counter)) return SIM_ERR_ARG;
    const cudaError_t err = launch_pdl(k_aniso_control, dim3(1), dim3(1), 0, (cudaStream_t)stream, *ep, *p, work);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_aniso_control: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_aniso_control");
}

extern "C" int sim_box_scale_after_first(const SimEngine* ep, const double* work_prev, int32_t reset_prev,
                                         const SimBoxScale* p, double* work, const SimIntegrator* integ,
                                         int32_t force_precision, void* stream) {
    if (!ep || !work_prev || !p || !work || !integ || ep->n <= 0 || (force_precision == 1 && !ep->f64))
        return SIM_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (!(p->scale[a] > 0.0) || !(p->vel_scale[a] > 0.0)) return SIM_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = launch_pdl(k_box_prepare_after, dim3(1), dim3(1), 0, st, *p, work_prev, work);
    if (err == cudaSuccess)
        err = launch_pdl(k_two_scales_first, dim3((unsigned)ceil_div(ep->n, SIM_THREADS)), dim3(SIM_THREADS), 0, st,
                         *ep, work_prev, (const double*)work, (int)reset_prev, (int)p->reset_reference, *integ,
                         (int)force_precision);
    if (err == cudaSuccess) err = launch_pdl(k_box_commit, dim3(1), dim3(1), 0, st, *ep, (const double*)work);
    if (err != cudaSuccess) { set_cuda_error(err, "sim_box_scale_after_first: launch"); return SIM_ERR_CUDA; }
    return launch_status("sim_box_scale_after_first");
}
