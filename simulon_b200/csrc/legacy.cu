// Drop-ins for the reference's edge-based native kernels (sm_100a):
// density_pass / force_pass (cuda source/eam_cuda_ext_kernel.cu) and
// lj_energy_force_cuda (cuda source/lj_energy_force_kernel.cu), same argument
// meaning, accumulating into caller-owned buffers with atomics as the
// originals do (the half-list edge interface requires scattering to both ends).
#include "common.cuh"

namespace simb200 {

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
