/*
 * simb200.h -- C ABI of the B200-native Simulon force path (libsimb200.so).
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), launches asynchronously on that stream and returns an
 * int status (SIM_OK = 0).  Nothing is allocated inside the library and no
 * device state is kept between calls: the caller (PyTorch on the Python side)
 * owns every buffer (one exception: the fixed scratch array used by
 * sim_eam_forces_static).  Errors found on the device (neighbour-list overflow,
 * non-finite values, box too small) are reported through a caller-owned
 * device status word that the host reads when it chooses to synchronise.
 *
 * Three groups of entry points (the third, batched replicas, is described
 * at its declarations below):
 *
 *  1. Drop-ins for the reference's native module `simulon_cuda`
 *     (cuda source/ops.cpp:47-53), same argument meaning:
 *       sim_legacy_density_pass   <- density_pass   (cuda source/eam_cuda_ext.cpp:30-42)
 *       sim_legacy_force_pass     <- force_pass     (cuda source/eam_cuda_ext.cpp:44-60)
 *       sim_legacy_lj_energy_force<- lj_energy_force_cuda (cuda source/lj_energy_force.cpp:10-20)
 *                                    + configure_lj_smoothing (ops.cpp:43-45) folded into
 *                                    the mode/rc/rs arguments (no device globals)
 *       sim_half_list_*           <- neighbor_search_cuda (cuda source/neighbor_search_kernel.cu:73-138)
 *                                    and find_neighbors_gpu_pbc (core/neighbor_search/gpu_kdtree.py:56-87):
 *                                    half list i<j in the caller's dtype, bit-exact
 *                                    with the reference's torch arithmetic, any box.
 *
 *  2. The device-resident engine (atoms kept in cell order, full Verlet list in
 *     ELL layout, FP64 integration state), which replaces the per-step work of
 *     BaseModel.forward (core/md_model.py:88-166):
 *       sim_rebuild               <- AtomFileReader.update_neighbor_list (io_utils/reader.py:212-242)
 *       sim_eam_forces            <- EAMForceCUDAExt.forward (core/force/eam_force_cu.py:461-579)
 *       sim_lj_forces             <- LennardJonesForce.forward (core/force/lennard_jones_force.py:15-95)
 *       sim_integrate_first       <- VerletIntegrator.first_half + update_coordinates' skin/2
 *                                    trigger (core/integrator/integrator.py:91-99, io_utils/reader.py:136-163)
 *       sim_integrate_second      <- VerletIntegrator.second_half (integrator.py:102-124)
 *       sim_berendsen             <- BerendsenBarostat.step (core/barostat.py:36-68)
 *       sim_gather_original       -- un-permute per-atom arrays to the caller's atom order
 */
#ifndef SIMB200_H
#define SIMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (return values and device status-word bits) ---------- */
#define SIM_OK               0
#define SIM_ERR_ARG          1   /* bad argument (null pointer, size, unsupported combination) */
#define SIM_ERR_CUDA         2   /* a CUDA launch failed; see sim_last_cuda_error()            */
#define SIM_ERR_BOX          4   /* box too small for the cutoff (needs L > 2 (rc+skin))       */
#define SIM_STATUS_OVERFLOW  8   /* device: a neighbour row exceeded the ELL capacity          */
#define SIM_STATUS_NONFINITE 16  /* device: NaN/Inf in forces, positions or velocities         */
#define SIM_STATUS_CELLCAP   32  /* device: half-list export row capacity exceeded             */
#define SIM_STATUS_HALO      64  /* device: a tile's halo exceeded halo_cap (flags[4] = size)  */
#define SIM_STATUS_CELLS     512 /* device: the box shrank below the cell grid's rc + skin width
                                    (a rebuild may miss pairs: rebuild the grid, MDEngine.regrid) */

#define SIM_TILE 1024            /* atoms per neighbour tile (= threads of a tiled block)      */

/* ---- simulation box (rows are lattice vectors, row-vector convention) -- */
typedef struct SimBox {
    double H[9];        /* H[3*r + c]                                          */
    double Hinv[9];
    float  Hf[9];       /* H rounded to float (used by the FP32 pair kernels)  */
    int32_t orthogonal; /* off-diagonals all within 1e-8 of zero (core/box.py:54-57) */
    int32_t pad[3];
} SimBox;

/* ---- engine description: caller-allocated device buffers ---------------- *
 * n atoms live in "slots" 0..n-1 in cell order; per-atom arrays have stride
 * n_pad (a multiple of 128).  SoA FP64 vectors are [3][n_pad].              */
typedef struct SimEngine {
    int64_t n, n_pad;
    int32_t n_types, nbr_cap;        /* ELL capacity (neighbours per atom)      */
    int32_t ncell[3], n_cells;       /* cell grid, fixed for the engine's life  */
    double  x_rc;                    /* list cutoff rc + skin                   */
    double  skin_half2;              /* (skin/2)^2 for the rebuild trigger      */
    SimBox* box;                     /* device, updated in place by Berendsen  */
    /* integration state, cell order */
    double* x;        /* [3][n_pad] positions (unwrapped, as the reference)   */
    double* v;        /* [3][n_pad] velocities                               */
    float*  f32;      /* [n_pad][4] forces (FP32 pair path, float4; .w unused) */
    double* f64;      /* [3][n_pad] forces (FP64 pair path) or NULL            */
    int32_t* posq;    /* [n_pad][4] int4: fixed-point fractional coordinates
                         u = frac(x H^-1) * 2^32 (uint32) in .xyz, type in .w;
                         the int32 difference of two codes is the minimum-image
                         fractional displacement (16-byte gathers)            */
    int32_t* xref;    /* [3][n_pad] fixed-point positions at the last rebuild */
    int32_t* orig;    /* [n_pad] original atom index of each slot             */
    int32_t* posfp;   /* [n_pad][4] int4 {posq.x, posq.y, posq.z, F'(rho) bits}
                         written by EAM pass 1, gathered by pass 2            */
    int32_t* nbr;     /* [nbr_cap][n_pad] neighbour slots (ELL, column-major) */
    int32_t* nnbr;    /* [n_pad] neighbour counts                             */
    /* rebuild scratch */
    int32_t* cell_of;     /* [n_pad] */
    int32_t* cell_count;  /* [n_cells + 1] */
    int32_t* cell_start;  /* [n_cells + 1] */
    int32_t* cell_rank;   /* [2*n_cells]: linear cell -> Morton rank, then rank -> linear */
    int32_t* perm;        /* [n_pad] new slot -> old slot */
    double*  x_alt;       /* [3][n_pad] */
    double*  v_alt;       /* [3][n_pad] */
    float*   f32_alt;     /* [n_pad][4] */
    double*  f64_alt;     /* [3][n_pad] or NULL */
    int32_t* orig_alt;    /* [n_pad] */
    /* per-type constants */
    double*  inv_mass;    /* [n_types] 1/m in ps^2 A^-2 eV^-1 ... see integrator */
    double*  mass;        /* [n_types] m in eV ps^2 / A^2                        */
    /* control and reductions */
    int32_t* flags;       /* [8]: [0] rebuild requested, [1] status bits, [2] longest
                             neighbour row seen on overflow, [3] rebuilds performed */
    double*  partials;    /* [n_blocks_max * SIM_RED_SLOTS] */
    uint32_t* red_counter;/* [4] last-block counters (self-resetting) */
    double*  red_out;     /* [SIM_RED_SLOTS] final FP64 sums */
    int32_t  n_blocks_max;
    int32_t  box_orthogonal;  /* 1 if the box is (and stays) orthogonal: selects the
                                 kernels specialised for a diagonal H */
    /* neighbour tiles: SIM_TILE consecutive slots per tile; the tile's halo is the
     * sorted set of out-of-tile neighbour slots; nbr16 holds the list as tile-local
     * indices (< SIM_TILE: own slot tile*SIM_TILE + idx; else halo[idx - SIM_TILE]).
     * NULL nbr16 disables the tiled kernels.                                     */
    int32_t  n_tiles, halo_cap;
    int32_t* halo;        /* [n_tiles][halo_cap] */
    int32_t* halo_n;      /* [n_tiles] */
    uint16_t* nbr16;      /* [nbr_cap][n_pad] */
    /* EAM pass 1 records which list slots lie inside the cutoff (bit k of
     * cut_mask[i] for slot k of atom i) and pass 2 visits only those; needs
     * nbr_cap <= 64.  NULL: pass 2 tests every slot itself.                      */
    uint64_t* cut_mask;   /* [n_pad] or NULL */
    /* launch shapes (0: built-in default), as picked by sim_autotune_*:
     * [0] EAM pass-1 threads per block (128, 256, 512), [1] EAM pass-2 threads
     * per block (256, 512, 1024), [2] / [3] threads per atom of the MLP
     * descriptor / force kernels (4, 8).                                        */
    int32_t launch[4];
} SimEngine;

/* reduction slot layout (FP64 Kahan-compensated sums over all atoms) */
#define SIM_RED_EPOT_EMBED 0
#define SIM_RED_EPOT_PAIR  1
#define SIM_RED_VIRIAL     2   /* scalar virial, force-field sign convention  */
#define SIM_RED_W_XX 3
#define SIM_RED_W_YY 4
#define SIM_RED_W_ZZ 5
#define SIM_RED_W_XY 6
#define SIM_RED_W_XZ 7
#define SIM_RED_W_YZ 8
#define SIM_RED_KE   9
#define SIM_RED_K_XX 10
#define SIM_RED_K_YY 11
#define SIM_RED_K_ZZ 12
#define SIM_RED_K_XY 13
#define SIM_RED_K_XZ 14
#define SIM_RED_K_YZ 15
#define SIM_RED_SLOTS 16

/* ---- EAM tables (FP32, uniform grids; eam_force_cu.py:334-396) ---------- */
typedef struct SimEAMTables {
    const float* density;        /* [E][E][n_r]  host type, neighbour type  */
    const float* density_deriv;  /* [E][E][n_r]                              */
    const float* pair;           /* [E][E][n_r]                              */
    const float* pair_deriv;     /* [E][E][n_r]                              */
    const float* embed;          /* [E][n_rho]                               */
    const float* embed_deriv;    /* [E][n_rho]                               */
    const float* rho_min;        /* [E]  (device)                            */
    const float* inv_drho;       /* [E]                                      */
    const float* rho_clamp_hi;   /* [E]  rho_min + drho (n_rho-1)(1-1e-7)    */
    /* the same r-tables as value + forward difference, so v(k + frac) =
     * fma(frac, d_k, v_k) with d_k = v_{min(k+1,n-1)} - v_k (float32):       */
    const float* dens_vd;        /* [E][E][n_r] float2 {f_k, df_k}                 */
    const float* deriv_vd;       /* [E][E][n_r] float4 {f'_k, phi'_k, df'_k, dphi'_k} */
    const float* pair_vd;        /* [E][E][n_r] float2 {phi_k, dphi_k}             */
    int32_t n_types, n_r, n_rho, pad;   /* 2 <= n_r < 2^22 (larger tables: SIM_ERR_ARG) */
    float cutoff, inv_dr, r_clamp_hi, pad2;   /* r_clamp_hi = r_max (1-1e-7) */
} SimEAMTables;

/* ---- LJ parameters (per type pair; lennard_jones_force.py:41-79) ------- */
#define SIM_LJ_RAW    0
#define SIM_LJ_SHIFT  1   /* force shift ("is_fs")                        */
#define SIM_LJ_SWITCH 2   /* quintic switch on [rs, rc] ("is_switch")     */
typedef struct SimLJParams {
    const double* c4eps;    /* [E*E] 4*eps formed as the reference does (float32) */
    const double* c24eps;   /* [E*E] 24*eps (float32 product)                      */
    const double* sigma;    /* [E*E]                                               */
    const double* u_rc;     /* [E*E] shift-mode energy at rc                       */
    const double* f_rc;     /* [E*E] shift-mode force magnitude at rc              */
    int32_t n_types, mode;
    double rc, rs;
} SimLJParams;

/* ---- integrator parameters (integrator.py:45-124) ---------------------- */
typedef struct SimIntegrator {
    double dt;
    double damp;            /* exp(-gamma dt); 1 when not Langevin          */
    const double* rff;      /* [n_types] sqrt(kB T/m (1-exp(-2 gamma dt))) or NULL */
    uint64_t seed;          /* Philox key                                   */
    uint64_t* step_ctr;     /* device step counter: incremented by
                               sim_integrate_first, read by sim_integrate_second
                               (so a captured graph draws fresh noise each replay) */
    int32_t langevin;
    int32_t pad;
} SimIntegrator;

/* ---- anisotropic pressure control (barostat.py:78-208) and box scaling --- */
typedef struct SimAniso {
    double target_bar[3];      /* per lattice axis                                  */
    double tau_p, gamma_p, max_eta_dot, kappa_bar_inv, tol_bar, dt, temperature;
    double* eta_dot;           /* [3] device state: log strain rate per axis (1/ps) */
    uint64_t* counter;         /* [1] device: calls so far (Philox counter of the noise) */
    int32_t control[3];        /* 1 = the axis is controlled                        */
    int32_t stochastic;        /* 1 = add the reference's thermal noise (Philox)    */
    int32_t reset_reference;   /* 1 = last_positions reset after the step (reference) */
    uint32_t seed;
} SimAniso;
/* work buffer of sim_aniso_npt / sim_box_scale: SIM_BOXSCALE_WORK doubles;
 * [0..2] axis pressures (bar), [3..5] box scale, [6..8] velocity scale, then
 * the new box (SimBox layout, from double 16). */
#define SIM_BOXSCALE_WORK 64
typedef struct SimBoxScale {
    double scale[3];           /* H <- diag(scale) H                                 */
    double vel_scale[3];       /* v_c <- v_c * vel_scale[c]                           */
    int32_t reset_reference;   /* 1 = last_positions reset (loading.py:78)            */
    int32_t pad;
} SimBoxScale;

/* UniaxialTensileLoader bookkeeping on the device (sim_loader_check) */
typedef struct SimLoaderCheck {
    int32_t axis;              /* loading axis 0..2                                  */
    int32_t pad;
    double rebuild_strain;     /* max |H inv(H_list) - I| that forces a list rebuild */
    double regrid_margin;      /* request a regrid when a cell is narrower than
                                  x_rc (1 + margin)                                  */
} SimLoaderCheck;
/* state of sim_loader_check: SIM_LOADER_STATE doubles, host-initialised:
 * [0..8] H at the list the rule last forced (set to the box at start),
 * [9..11] initial row lengths; written by the device: [12] engineering strain
 * of the loading axis, [13..15] current row lengths, [16] forced rebuilds,
 * [17] 1 = regrid requested (the host clears it after MDEngine-style regrid). */
#define SIM_LOADER_STATE 32

/* ---- spherical indenter (core/mechanics/indenter.py:7-68) --------------- */
typedef struct SimIndenter {
    const double* center;      /* [3] device (settable between graph replays)      */
    double radius, stiffness;  /* R (A), K (eV/A^3)                                  */
    double* out;               /* [11] device: energy, force on the indenter (3),
                                  contact atoms, virial xx yy zz xy xz yz            */
} SimIndenter;

/* ---- Berendsen (barostat.py:21-68) -------------------------------------- */
typedef struct SimBerendsen {
    double target_bar, tau, kappa, mu_max, dt;
    int32_t coordinate_scale_power;   /* 2 = the reference's behaviour (coordinates
                                         and graph_data.pos alias, both scaled)     */
    int32_t reset_reference;          /* 1 = last_positions reset after scaling    */
} SimBerendsen;

/* ==== group 1: drop-ins for the reference's native module ================ */

/* density_pass (eam_cuda_ext.cpp:30-42): rho_out[row] += f_{t_row,t_col}(r),
 * rho_out[col] += f_{t_col,t_row}(r) per half-list edge; accumulates in place. */
int sim_legacy_density_pass(const float* distances, const int64_t* row, const int64_t* col,
                            const int64_t* atom_types, int64_t n_edges,
                            const float* density_table, int32_t n_types,
                            double inv_dr, int64_t n_r, float* rho_out, void* stream);

/* force_pass (eam_cuda_ext.cpp:44-60): forces_out[row] += -s rij/r, forces_out[col] -= ... */
int sim_legacy_force_pass(const float* distances, const float* dist_vec, const int64_t* row,
                          const int64_t* col, const int64_t* atom_types, int64_t n_edges,
                          const float* density_deriv_table, const float* pair_deriv_table,
                          const float* dF_drho, int32_t n_types, double inv_dr, int64_t n_r,
                          float* forces_out, void* stream);

/* lj_energy_force_cuda (lj_energy_force.cpp:10-20) with the smoothing mode of
 * configure_lj_smoothing (ops.cpp:43-45) passed explicitly.  forces_out [N,3]
 * and energy_out [1] must be zeroed by the caller (the reference allocates zeros). */
int sim_legacy_lj_energy_force(const float* pos, const int64_t* edge_i, const int64_t* edge_j,
                               int64_t n_edges, const float* sigma, const float* epsilon,
                               float box_length, int32_t mode, float rc, float rs,
                               float* forces_out, float* energy_out, void* stream);

/* Half Verlet list in the caller's atom order and dtype (find_neighbors_gpu_pbc,
 * gpu_kdtree.py:56-155 + reader.py:477-484).  Two phases:
 *   sim_half_list_count: bins atoms, counts pairs j>i with d^2 < rc2 per atom,
 *     writes row_ptr[n+1] (exclusive scan, int64) -- total = row_ptr[n];
 *   sim_half_list_fill : writes edge_i/edge_j (int64, sorted by (i,j)),
 *     image (int32 [E,3], optional) and dist (|min image|, optional).
 * dtype_code: 0 = float32 positions, 1 = float64.  Scratch: see the Python
 * wrapper (cell arrays of size n_cells+1 and n, one int64 per atom).       */
int sim_half_list_count(const void* pos, int32_t dtype_code, int64_t n, const SimBox* box_host,
                        double rc2, const int32_t* ncell, int32_t* cell_of, int32_t* cell_count,
                        int32_t* cell_start, int32_t* sorted_idx, int64_t* row_ptr,
                        void* stream);
int sim_half_list_fill(const void* pos, int32_t dtype_code, int64_t n, const SimBox* box_host,
                       double rc2, const int32_t* ncell, const int32_t* cell_start,
                       const int32_t* sorted_idx, const int32_t* cell_of, const int64_t* row_ptr,
                       int64_t* edge_i, int64_t* edge_j, int32_t* image, void* dist,
                       void* stream);

/* ==== group 2: the device-resident engine ================================ */

/* Load atoms (original order, host-layout [N,3] FP64 device arrays) into slot
 * order 0..n-1 and run the first full rebuild.  types: int32 [N]. */
int sim_engine_load(const SimEngine* e, const double* x_rows, const double* v_rows,
                    const int32_t* types, void* stream);

/* Rebuild (cell binning, counting sort, deterministic in-cell order by original
 * index, permutation of the state, ELL list).  With only_if_flagged = 1 the
 * kernels read flags[0] and do nothing unless a rebuild was requested. */
int sim_rebuild(const SimEngine* e, int32_t only_if_flagged, void* stream);

/* Rebuild only if flags[0] is set.  While `stream` is being captured into a
 * CUDA graph this adds a one-thread kernel and an IF conditional node whose
 * body is the rebuild (so a step without a rebuild launches one tiny kernel);
 * otherwise it is sim_rebuild(e, 1, stream). */
int sim_rebuild_if_needed(const SimEngine* e, void* stream);

/* EAM forces on the engine state.  Writes f32 (or f64), fp, and the
 * reduction slots EPOT_*, VIRIAL, W_* (red_out).  Scalar virial follows the
 * reference's EAM convention: sum over pairs of s*r (eam_force_cu.py:569). */
int sim_eam_forces(const SimEngine* e, const SimEAMTables* t, void* stream);
/* The two passes of sim_eam_forces as separate launches (pass 1 writes fp
 * and EPOT_EMBED; pass 2 needs pass 1's fp of the same positions). */
int sim_eam_density(const SimEngine* e, const SimEAMTables* t, void* stream);
int sim_eam_force(const SimEngine* e, const SimEAMTables* t, void* stream);
/* Pass 2 with the second half of the velocity-Verlet step (Langevin O-step,
 * half kick, K and K tensor) fused into its epilogue; equivalent to
 * sim_eam_force followed by sim_integrate_second with FP32 forces. */
int sim_eam_force_integrate(const SimEngine* e, const SimEAMTables* t, const SimIntegrator* p, void* stream);
/* sim_eam_force_integrate plus the first half of the NEXT step in the same
 * pass (kick with the new forces, drift, posq refresh, skin/2 trigger into
 * flags[0]): bit for bit sim_eam_force_integrate followed by
 * sim_integrate_first(force_precision 0).  p->step_ctr must point to two
 * words: [0] is advanced to the next step, [1] receives this step's index
 * (pass &step_ctr[1] to sim_log_step for this step).  The state between such
 * calls holds half-step velocities; end a run with sim_eam_force_integrate.
 * Not available with neighbour tiles (nbr16 set): SIM_ERR_ARG. */
int sim_eam_force_integrate_drift(const SimEngine* e, const SimEAMTables* t, const SimIntegrator* p,
                                  void* stream);
/* EAM pass 2 as sim_eam_force_integrate (mode 1) or
 * sim_eam_force_integrate_drift (mode 2) with the spherical indenter of
 * sim_indenter_add added to each atom's force before the integrator epilogue
 * (indenter.py:40-68, the force field and the indenter summed as
 * SumBackboneInterface sums them, md_model.py:33-52): bit for bit the
 * positions and velocities of sim_eam_force + sim_indenter_add +
 * sim_integrate_second (+ sim_integrate_first), with ind->out written as
 * sim_indenter_add writes it and its energy and virial added to red_out.
 * One element type, untiled kernels (else SIM_ERR_ARG); needs 2 x the
 * persistent grid in n_blocks_max (a second set of block partials). */
int sim_eam_force_integrate_indenter(const SimEngine* e, const SimEAMTables* t, const SimIntegrator* p,
                                     const SimIndenter* ind, int32_t mode, void* stream);
/* sim_eam_force_integrate_indenter in mode 2, sim_log_step on step_ctr[1] and
 * sim_rebuild_if_needed, with the log row and (while the stream is captured)
 * the rebuild's IF-node value written by the force pass's last block, as
 * sim_eam_step_drift does for EAM alone: the same bits, two kernels fewer
 * per step.  One element type, untiled kernels. */
int sim_eam_step_drift_indenter(const SimEngine* e, const SimEAMTables* t, const SimIntegrator* integ,
                                const SimIndenter* ind, const double* extra, int32_t n_extra, double* log,
                                int32_t log_capacity, void* stream);
/* One whole MD step of the drift-fused form ended on the device: EAM pass 1,
 * then pass 2 as sim_eam_force_integrate_drift, whose last block also appends
 * the step's log row (as sim_log_step on &step_ctr[1]) and decides the
 * conditional rebuild (as sim_rebuild_if_needed): while `stream` is being
 * captured, an IF node holding the rebuild follows pass 2, which sets the
 * node's value itself (no separate log or condition kernel in the graph);
 * otherwise the flag-gated rebuild is launched after it.  Same results, bit
 * for bit, as sim_eam_density + sim_eam_force_integrate_drift + sim_log_step +
 * sim_rebuild_if_needed.  Replaces one pass of BaseModel.forward's step
 * (md_model.py:107-139: first_half with its list update, sum_bone,
 * second_half) plus the step's energy record.  n_extra <= 32. */
int sim_eam_step_drift(const SimEngine* e, const SimEAMTables* t, const SimIntegrator* p, const double* extra,
                       int32_t n_extra, double* log, int32_t log_capacity, void* stream);

/* sim_eam_forces without caller-allocated scratch.  No counterpart in the
 * reference (which allocates through PyTorch on every call); it exists for
 * callers that cannot allocate device memory for the call -- a host code
 * whose device memory is all handed out up front by its own pool, or one that
 * binds this library over a plain C FFI with no device allocator.
 *   Scratch: the per-atom {x, y, z, F'} records passed from the density pass
 *   to the force pass, the reduction partials and the last-block counters come
 *   from one fixed 4,456,704-byte array inside the library; e->posfp,
 *   e->partials, e->red_counter and e->n_blocks_max are ignored (may be NULL /
 *   0).  e->cut_mask is ignored as well (neither read nor written; the force
 *   pass tests every list entry against the cutoff instead, same results).
 *   Every other SimEngine buffer and the outputs (f32 or f64, red_out, flags)
 *   are the caller's, as for sim_eam_forces.
 *   Limit: e->n_pad <= SIM_STATIC_MAX_ATOMS; a larger system returns
 *   SIM_ERR_ARG before any CUDA call, with the reason in sim_last_cuda_error().
 *   Set-up: every call looks up the array's device address on the current
 *   device (cudaGetSymbolAddress); the first call on a device also loads the
 *   array there, so make it before any stream capture.  Each call zeroes the counters itself (cudaMemsetAsync on
 *   `stream`); nothing else has to start at zero.
 *   Concurrency: one array per device, shared by all calls -- calls that can
 *   overlap (other streams or host threads on the same device) race on it;
 *   serialise them.
 *   Allocates nothing: no cudaMalloc / cudaFree, no allocating library call. */
#define SIM_STATIC_MAX_ATOMS 262144
int sim_eam_forces_static(const SimEngine* e, const SimEAMTables* t, void* stream);

/* LJ forces; precision 0 = FP32 pair arithmetic, 1 = FP64 (positions read
 * from e->x, forces to e->f64).  Scalar virial = sum F*r (lennard_jones_force.py:93). */
int sim_lj_forces(const SimEngine* e, const SimLJParams* p, int32_t precision, void* stream);
/* FP32-pair LJ forces (as sim_lj_forces, precision 0) with the integrator
 * fused into the same pass over the atoms, like the EAM force pass: mode 1
 * adds the second half of the step (as sim_integrate_second,
 * integrator.py:102-124); mode 2 adds the next step's first half as well
 * (as sim_integrate_first, integrator.py:91-99: kick with the new forces,
 * drift, posq refresh, skin/2 trigger), advancing p->step_ctr[0] and setting
 * step_ctr[1] to this step like sim_eam_force_integrate_drift.  Mode 2 writes
 * the new fixed-point records to e->posfp (required; the pass still gathers
 * posq) and copies them to posq after the pass. */
int sim_lj_forces_integrate(const SimEngine* e, const SimLJParams* p, const SimIntegrator* integ, int32_t mode,
                            void* stream);
/* FP32-pair LJ as a further force field of a sum (SumBackboneInterface.forward,
 * core/md_model.py:39-46, which adds each backbone's forces, energy, virial
 * and virial tensor into shared buffers): atom i's LJ force is added to
 * e->f32, the pair energy, scalar virial (sum F r) and virial tensor to
 * red_out.  Run after the first force field's pass (e.g. sim_eam_forces). */
int sim_lj_forces_add(const SimEngine* e, const SimLJParams* p, void* stream);

/* first_half: v += 0.5 a dt; x += v dt; refresh posq; skin/2 trigger -> flags[0].
 * force_precision: 0 reads f32, 1 reads f64. */
int sim_integrate_first(const SimEngine* e, const SimIntegrator* p, int32_t force_precision,
                        void* stream);

/* second_half: Langevin O-step (Philox noise by original index), half kick,
 * kinetic energy and kinetic tensor sum m v(x)v into red_out. */
int sim_integrate_second(const SimEngine* e, const SimIntegrator* p, int32_t force_precision,
                         void* stream);

/* second_half of step s and first_half of step s+1 with the same forces, in
 * one pass (for force fields that cannot finish the step inside their own
 * kernel); advances step_ctr like sim_eam_force_integrate_drift. */
int sim_integrate_second_first(const SimEngine* e, const SimIntegrator* p, int32_t force_precision,
                               void* stream);

/* Berendsen: reads red_out (K tensor, W tensor) and the device box, computes
 * P (bar) and mu on the device in FP64, scales box, coordinates (mu^power),
 * velocities; writes pressure_out[0] = P (bar), pressure_out[1] = mu. */
int sim_berendsen(const SimEngine* e, const SimBerendsen* p, double* pressure_out, void* stream);
/* sim_berendsen in two parts, so that a run of NPT steps passes over the atoms
 * once less per step.  sim_berendsen_mu: the controller alone (P, mu, the box
 * scaled by mu; pressure_out as sim_berendsen) -- BerendsenBarostat.step's
 * pressure, mu and box scale (barostat.py:44-61).  sim_berendsen_scale_first: the atoms'
 * part of that update (coordinates x mu^power, velocities x mu, the skin
 * reference reset; barostat.py:63-68; mu = mu_in[1] from sim_berendsen_mu)
 * fused with the NEXT step's first half (as sim_integrate_first,
 * integrator.py:91-99), bit for bit sim_berendsen followed by
 * sim_integrate_first. */
int sim_berendsen_mu(const SimEngine* e, const SimBerendsen* p, double* pressure_out, void* stream);
int sim_berendsen_scale_first(const SimEngine* e, const SimBerendsen* p, const double* mu_in,
                              const SimIntegrator* integ, int32_t force_precision, void* stream);

/* AnisotropicNPTBarostat.step (barostat.py:137-208) on the device in FP64:
 * axis pressures from the kinetic and virial tensors in red_out projected on
 * the normalised lattice rows, the deadband, the damped strain-rate update
 * (clamped, masked), H <- diag(exp(dt eta_dot)) H, positions through
 * fractional coordinates into the new box and wrapped (box.py:132-142),
 * velocities * exp(-dt eta_dot), posq refreshed, the skin test against the
 * last rebuild and (reset_reference) the reference reset.  work: see
 * SIM_BOXSCALE_WORK. */
int sim_aniso_npt(const SimEngine* e, const SimAniso* p, double* work, void* stream);
/* UniaxialTensileLoader.step's box update (loading.py:41-80): H <- diag(scale) H
 * and the same position, velocity (vel_scale), posq and reference handling. */
int sim_box_scale(const SimEngine* e, const SimBoxScale* p, double* work, void* stream);
/* The controller half of sim_aniso_npt (AnisotropicNPTBarostat.step,
 * barostat.py:137-208): axis pressures, the strain-rate update and the new box
 * prepared in `work`, without moving the atoms (sim_box_scale_after_first
 * moves them together with the next step's loader update and first half). */
int sim_aniso_control(const SimEngine* e, const SimAniso* p, double* work, void* stream);
/* The end of a tensile step and the start of the next in one pass over the
 * atoms (run_scripts/w_tensile.py's loop: barostat.step after model(), then
 * loader.step and the next model()'s first_half, integrator.py:91-99): the box
 * update prepared in work_prev (sim_aniso_control), then the loader's box
 * update p prepared on that box into `work`, then the first half of the next
 * step in the new box; the same operations in the same order as
 * sim_box_scale (or sim_aniso_npt's scaling), sim_box_scale and
 * sim_integrate_first launched one after another, so the same bits.  The box
 * is committed; sim_loader_check follows as after sim_box_scale.  work:
 * SIM_BOXSCALE_WORK doubles. */
int sim_box_scale_after_first(const SimEngine* e, const double* work_prev, int32_t reset_prev, const SimBoxScale* p,
                              double* work, const SimIntegrator* integ, int32_t force_precision, void* stream);
/* The rest of UniaxialTensileLoader.step (loading.py:41-80) on the device, to
 * run after sim_box_scale so that the loop needs no host read per step: the
 * box row lengths and the loading axis' engineering strain (state[12]); a
 * list rebuild requested through flags[0] (taken by the next conditional
 * rebuild) once the box has deformed by more than p->rebuild_strain since the
 * list this rule last forced; state[17] = 1 when the cell grid comes within
 * p->regrid_margin of the list cutoff (the host regrids between launches or
 * graph replays).  One thread; graph-capturable. */
int sim_loader_check(const SimEngine* e, const SimLoaderCheck* p, double* state, void* stream);
/* One tensile MD step's end and the next one's start with an anisotropic
 * barostat (run_scripts/w_tensile.py's loop, barostat.py:137-208,
 * loading.py:41-80): what sim_aniso_control(baro, work_baro),
 * sim_log_step(step_ctr, extra, n_extra, log, capacity),
 * sim_box_scale_after_first(work_baro, baro->reset_reference, load,
 * work_load, integ, force_precision), sim_loader_check(check, state) and
 * sim_rebuild_if_needed do one after another, in three kernels (the
 * controller, the log row and the loader's box prepared on one thread; the
 * pass over the atoms; the box committed, the loader's bookkeeping and, while
 * the stream is captured, the value of the rebuild's IF node on one thread)
 * and the rebuild's IF node instead of seven kernels: the same operations in
 * the same order, so the same bits.  Arguments as in those calls. */
int sim_tensile_link(const SimEngine* e, const SimAniso* baro, double* work_baro, const uint64_t* step_ctr,
                     const double* extra, int32_t n_extra, double* log, int32_t capacity, const SimBoxScale* load,
                     double* work_load, const SimIntegrator* integ, int32_t force_precision,
                     const SimLoaderCheck* check, double* state, void* stream);

/* SphericalIndenterForce.forward (indenter.py:40-68) added to the engine's
 * forces (force_precision 0: f32, 1: f64) after a force field's pass: for
 * atoms with d = |x - c| < R, F = K (R - d)^2 (x - c)/d, U = K/3 (R - d)^3,
 * virial F (x) x; the energy, the trace and the tensor's upper triangle are
 * added to red_out (EPOT_PAIR, VIRIAL, W), and out[] gets the indenter's own
 * sums.  Positions are the FP64 unwrapped ones, without periodic images. */
int sim_indenter_add(const SimEngine* e, const SimIndenter* p, int32_t force_precision, void* stream);

/* Scatter caller rows into slots: dst_soa[c*n_pad + k] = rows[orig[k]*3 + c]. */
int sim_scatter_original_f64(const SimEngine* e, const double* rows, double* dst_soa, void* stream);

/* Append red_out (SIM_RED_SLOTS doubles), extra[0..n_extra) and the status
 * word to log[(step_ctr % capacity) * row_width ...]; row_width = SIM_RED_SLOTS + n_extra + 1. */
int sim_log_step(const SimEngine* e, const uint64_t* step_ctr, const double* extra, int32_t n_extra,
                 double* log, int32_t capacity, void* stream);

/* Host helper of the simulator's trajectory file (no device work): rows
 * "<symbols[type[i]]> <x> <y> <z>\n" for i < n with the coordinates in fixed
 * notation, six decimals, digits as Python's format(v, ".6f") (correctly
 * rounded, ties to even; NaN as "nan") -- the rows that
 * MDSimulator._dump_step_outputs writes (core/md_simulation.py:125-168).
 * type may be NULL (all symbols[0]).  Writes into out[0, cap) and returns the
 * byte count, or -1 for a bad argument or a buffer that may be too small
 * (cap below n * (longest symbol + 196) always suffices). */
int64_t sim_format_xyz_rows(const double* xyz, const int32_t* type, int64_t n, const char* const* symbols,
                            int32_t n_symbols, char* out, int64_t cap);

/* Un-permute: out_rows[orig[k]*3 + c] = src[c*n_pad + k] (FP64 or FP32 source). */
int sim_gather_original_f64(const SimEngine* e, const double* src_soa, double* out_rows, void* stream);
int sim_gather_original_f32(const SimEngine* e, const float* src_soa, double* out_rows, void* stream);

/* Export the engine's list as the reference's half list (pairs i<j by
 * original index, sorted by (i,j)) -- count then fill, like sim_half_list_*. */
int sim_engine_half_count(const SimEngine* e, double rc2, int64_t* row_ptr, void* stream);
int sim_engine_half_fill(const SimEngine* e, double rc2, const int64_t* row_ptr,
                         int64_t* edge_i, int64_t* edge_j, double* dist, void* stream);

/* Exclusive scan of int64 counts: out[0]=0, out[k+1]=sum in[0..k] (n+1 entries;
 * in may be NULL when n = 0). */
int sim_scan_i64(const int64_t* in, int64_t n, int64_t* out, void* stream);

/* ==== group 3: batched replicas ========================================== *
 * Many independent systems (replicas) of uneven size -- a temperature scan or
 * a sweep of crack slabs, each run by the reference as its own BaseModel loop
 * (run_scripts/w_crack.py:433-440) -- advance together: one launch of each
 * kernel covers every replica.  Replica k owns the slots [off, off + n_slots)
 * of the SimEngine arrays, with off and n_slots multiples of 32 so that every
 * warp's 32 slots belong to one replica; its n atoms fill the first n slots,
 * the remaining slots are padding that no kernel reads or writes.  Each
 * replica has its own periodic box, cell grid, rebuild flag (only replicas
 * whose atoms moved more than skin/2 are rebuilt) and Langevin temperature,
 * and may hold atoms in grips that open at a fixed rate per step
 * (w_crack.py:384-392: grip atoms keep their reference positions shifted by
 * half the opening, with zero velocity).  One element type (n_types == 1). */
typedef struct SimRep {
    SimBox  box;
    int64_t off;            /* first slot                                          */
    int64_t first;          /* original index of the replica's first atom          */
    int32_t n, n_slots;     /* atoms; slots reserved (n rounded up to 32)           */
    int32_t ncell[3], n_cells;
    int32_t cell_off;       /* first entry of this replica in the batch cell arrays:
                               cell_count / cell_start hold n_cells + 1 entries from
                               cell_off, cell_rank 2 * n_cells entries from 2 * cell_off
                               (linear cell -> visiting rank, then rank -> linear)   */
    int32_t grip_axis;      /* box row along which the grips open; -1: no grips     */
    double  grip_rate;      /* opening per step (A): at step s the lower grip sits
                               0.5 * rate * (s + 1) below its reference position,
                               the upper grip as far above it                       */
} SimRep;

#define SIM_BATCH_RED_SPLIT 8   /* blocks that share one replica's reduction */
typedef struct SimBatch {
    SimEngine e;            /* slot arrays; e.n = slots in use (sum of n_slots),
                               e.n_pad >= e.n, a multiple of 128.  e.box, e.ncell,
                               e.n_cells are not used (per replica); e.cell_count,
                               e.cell_start index batch cell entries; e.flags[0] is
                               set when some replica asks for a rebuild, [1] status
                               bits, [2] longest row on overflow, [3] rebuild events */
    SimRep*  rep;           /* [n_rep] device                                        */
    int32_t  n_rep;
    int32_t  n_cell_entries;/* sum over replicas of n_cells + 1                       */
    int32_t* slot_rep;      /* [e.n_pad] replica k of each slot; -1 - k for padding    */
    int32_t* cell_rep;      /* [n_cell_entries] replica of each cell entry             */
    int32_t* rep_flags;     /* [n_rep] 1: rebuild this replica                         */
    int32_t* rep_rebuilds;  /* [n_rep] rebuilds performed                              */
    int32_t* work;          /* [3 * (n_rep + 1)] rebuild work list, written by the rebuild:
                               replicas to rebuild and their slot-chunk and cell prefixes */
    int8_t*  grip;          /* [atoms, original order] 0 free, 1 lower grip, 2 upper   */
    double*  gref;          /* [3][e.n_pad] grip reference positions, by original index */
    double*  rep_rff;       /* [n_rep] Langevin noise amplitude sqrt(kB T (1-damp^2)/m) */
    double*  chunk_red;     /* [e.n_pad / 32 + SIM_BATCH_RED_SPLIT * n_rep][SIM_RED_SLOTS]:
                               per-warp partial sums, then per-block sums of the reduction */
    double*  rep_red;       /* [n_rep][SIM_RED_SLOTS] per-replica FP64 sums            */
} SimBatch;

/* Load atoms x_rows/v_rows [atoms][3] FP64 and types [atoms] (original order,
 * replica after replica) into their slots and build every replica's list. */
int sim_batch_load(const SimBatch* b, const double* x_rows, const double* v_rows, const int32_t* types,
                   void* stream);
/* Rebuild the replicas whose rep_flags are set (all with only_flagged = 0). */
int sim_batch_rebuild(const SimBatch* b, int32_t only_flagged, void* stream);
/* As sim_rebuild_if_needed: an IF node on flags[0] while capturing. */
int sim_batch_rebuild_if_needed(const SimBatch* b, void* stream);
/* EAM pass 1 over all replicas (writes posfp, cut_mask, EPOT_EMBED partials). */
int sim_batch_eam_density(const SimBatch* b, const SimEAMTables* t, void* stream);
/* EAM pass 2 over all replicas.  mode 0: forces and pair reductions; 1: plus
 * the second half-step (Langevin with rep_rff, grips held); 2: plus the first
 * half of the next step (as sim_eam_force_integrate_drift).  p->rff is not
 * used (rep_rff is); p->step_ctr[0] is this step's index. */
int sim_batch_eam_force(const SimBatch* b, const SimEAMTables* t, const SimIntegrator* p, int32_t mode,
                        void* stream);
/* First half-step of every replica (advances step_ctr[0]; grips placed). */
int sim_batch_first_half(const SimBatch* b, const SimIntegrator* p, void* stream);
/* Per-replica FP64 sums of the partials into rep_red; when log != NULL also
 * into log row (*step % log_cap), laid out [log_cap][n_rep][SIM_RED_SLOTS]. */
int sim_batch_reduce(const SimBatch* b, const uint64_t* step, double* log, int32_t log_cap, void* stream);
/* One whole step of every replica: pass 1, pass 2 (mode 2, or mode 1 when
 * last != 0), the per-replica sums and log row, and (unless last) the advance
 * of step_ctr[0] and the conditional rebuild.  A run of k steps is
 * sim_batch_first_half followed by k calls, the last one with last = 1. */
int sim_batched_step(const SimBatch* b, const SimEAMTables* t, const SimIntegrator* p, int32_t last,
                     double* log, int32_t log_cap, void* stream);
/* Slot arrays -> rows in original order (padding skipped). */
int sim_batch_gather_f64(const SimBatch* b, const double* src_soa, double* out_rows, void* stream);
int sim_batch_gather_f32(const SimBatch* b, const float* src_aos4, double* out_rows, void* stream);

/* ==== group 4: descriptor-MLP surrogate (no counterpart in the reference) == *
 * A learned stand-in for the EAM force field: per atom, 8 radial and 8
 * angular symmetry-function descriptors of the in-cutoff neighbourhood
 * (r < 4.4 A), a 16 -> 64 -> 64 -> 1 SiLU network giving the atom's energy,
 * forces = -dE/dx.  The network's GEMMs run on the tensor cores in BF16 with
 * FP32 accumulation; it is trained on the engine's own per-atom EAM energies
 * with these kernels.  Parameters live in one FP32 array (offsets below); the
 * kernels read BF16 operand images made from it by sim_mlp_pack. */
#define SIM_MLP_OFF_W1 0        /* W1 [16][64]  */
#define SIM_MLP_OFF_B1 1024     /* b1 [64]      */
#define SIM_MLP_OFF_W2 1088     /* W2 [64][64]  */
#define SIM_MLP_OFF_B2 5184     /* b2 [64]      */
#define SIM_MLP_OFF_W3 5248     /* w3 [64]      */
#define SIM_MLP_OFF_B3 5312     /* b3           */
#define SIM_MLP_PARAMS 5313
#define SIM_STATUS_MLP_NEIGHBORS 128  /* device: > 32 in-cutoff neighbours (extra ones ignored) */
#define SIM_STATUS_MLP_TIMEOUT   256  /* device: a tensor-core completion wait timed out        */
typedef struct SimMLP {
    const uint16_t* w1t_img;  /* BF16 operand images from sim_mlp_pack (2, 8, 8, 2 KB) */
    const uint16_t* w2t_img;
    const uint16_t* w2_img;
    const uint16_t* w1_img;
    const float* b1;          /* [64] (inside the FP32 parameter array)         */
    const float* b2;          /* [64]                                           */
    const float* w3;          /* [64]                                           */
    const float* b3;          /* [1]                                            */
    const float* mu;          /* [16] descriptor means                          */
    const float* inv_sigma;   /* [16] 1 / descriptor standard deviations        */
} SimMLP;

/* Descriptors of every slot: G [n_pad][16] FP32. */
int sim_mlp_descriptors(const SimEngine* e, float* G, void* stream);
/* Per-atom energies e_atom [n] and dE/dG [n][16] (with respect to the raw
 * descriptors) for n rows of G; status gets SIM_STATUS_MLP_TIMEOUT on a
 * tensor-core wait that did not complete. */
int sim_mlp_forward(const SimMLP* m, const float* G, int64_t n, float* e_atom, float* dEdG, int32_t* status,
                    void* stream);
/* Forces -dE/dx into e->f32 (overwritten) from dE/dG of every slot. */
int sim_mlp_backward(const SimEngine* e, const float* dEdG, void* stream);
/* Training: gradient of mean_i (E_i - target_i)^2 over n rows with respect to
 * every parameter into grads [SIM_MLP_PARAMS] (overwritten), loss into *loss. */
int sim_mlp_train_grads(const SimMLP* m, const float* G, const float* target, int64_t n, float* grads,
                        float* loss, int32_t* status, void* stream);
/* Force matching, step 1: with ferr [n_pad][4] = F - F_target per slot
 * (float4, .w unused), u [n][16] = sum_m ferr_m . dG_i/dx_m per atom. */
int sim_mlp_force_contract(const SimEngine* e, const float* ferr, float* u, void* stream);
/* Force matching, step 2: gradient of
 *   w_energy mean_i (E_i - target_i)^2 + w_force sum_m |F_m - F_target,m|^2 / (3 n_force_atoms)
 * with respect to every parameter into grads (overwritten), through the
 * network and its directional derivative along u (held fixed); the energy
 * term's mean square into *loss. */
int sim_mlp_train_grads_fm(const SimMLP* m, const float* G, const float* target, const float* u, int64_t n,
                           float w_energy, float w_force, int64_t n_force_atoms, float* grads, float* loss,
                           int32_t* status, void* stream);
/* BF16 operand images of W1, W2 from the FP32 parameter array. */
int sim_mlp_pack(const float* params, uint16_t* w1t_img, uint16_t* w2t_img, uint16_t* w2_img, uint16_t* w1_img,
                 void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the parameter array; step >= 1. */
int sim_mlp_adam(float* params, const float* grads, float* m1, float* m2, float lr, int32_t step, void* stream);
/* One training step on the parameter array params [SIM_MLP_PARAMS] (the
 * array m's vectors point into; the four images are m's, rewritten): the
 * gradient (u NULL: sim_mlp_train_grads, energy term only, w_energy and
 * w_force unused; else sim_mlp_train_grads_fm), one Adam step with moments
 * adam_m, adam_v, and sim_mlp_pack. */
int sim_mlp_train_step(const SimMLP* m, float* params, uint16_t* w1t_img, uint16_t* w2t_img, uint16_t* w2_img,
                       uint16_t* w1_img, const float* G, const float* target, const float* u, int64_t n,
                       float w_energy, float w_force, int64_t n_force_atoms, float* grads, float* adam_m,
                       float* adam_v, float lr, int32_t step, float* loss, int32_t* status, void* stream);
/* Per-atom EAM energies F(rho_i) + 1/2 sum_j phi(r_ij) of every slot (one
 * element type): the surrogate's training targets. */
int sim_eam_atom_energy(const SimEngine* e, const SimEAMTables* t, float* e_atom, void* stream);

/* ---- group 5: launch-shape autotuning (SimEngine.launch) ------------------
 * Each call times every candidate shape of its kernels on the engine's
 * current state with CUDA events (reps launches after one untimed launch;
 * synchronises the stream, so never while a stream is being captured) and
 * returns the mean milliseconds and the fastest shapes; the caller stores
 * them in SimEngine.launch.  No counterpart in the reference (whose kernels
 * have fixed launch shapes).
 * sim_autotune_eam: ms[0..2] pass 1 at 128/256/512 threads, ms[3..5] pass 2
 *   (forces, energy, virial; no integrator epilogue) at 256/512/1024;
 *   best[0] = pass-1 threads, best[1] = pass-2 threads.  Rewrites the
 *   engine's posfp, cut_mask, f32 and red_out (as sim_eam_forces does).
 * sim_autotune_mlp: ms[0..1] descriptors at 4/8 threads per atom, ms[2..3]
 *   forces from dEdG at 4/8; best[0] / best[1] = descriptor / force threads
 *   per atom.  Rewrites G [n_pad][16] and the engine's f32.               */
int sim_autotune_eam(const SimEngine* e, const SimEAMTables* t, int32_t reps, float* ms, int32_t* best,
                     void* stream);
int sim_autotune_mlp(const SimEngine* e, const float* dEdG, float* G, int32_t reps, float* ms, int32_t* best,
                     void* stream);

/* ---- group 6: crack observables of the batched form (w_crack.py:113-188) --
 * Per replica, from the current positions: the crack-mouth opening (mean
 * height of the upper mouth atoms minus that of the lower ones, minus its
 * initial value), the crack length (positions binned along the crack axis;
 * a bin is open where the lowest atom above the crack plane and the highest
 * below it are at least `threshold` apart; the open run through the bins
 * inside the initial crack, grown to both sides), and the projected stress
 * ((K + W)/V in bar on the normalised box rows; the reference reports the
 * negated y component as the opening stress).  No counterpart in the
 * reference's kernels (its script computes these on the host each step). */
typedef struct SimCrack {
    double x_unit[3], y_unit[3];    /* normalised box rows 0 and 1                    */
    double y_plane, x_min, x_max, x_center, half_length, threshold, initial_cmod;
    int32_t bins, bin_off;          /* bins (0: not a crack replica), first bin        */
    int32_t n_upper, n_lower;       /* mouth atoms (tags 1 and 2)                      */
} SimCrack;
#define SIM_CRACK_OUT 8   /* per replica: stress_bar, native_stress_yy_bar, cmod, signed_cmod,
                             crack_length, crack_extension, open bins, 0 */
/* crack [n_rep] device; mouth [atoms, original order] 0 / 1 upper / 2 lower;
 * bins [2 * total bins] and sums [2 * n_rep] scratch; out [n_rep][SIM_CRACK_OUT].
 * Reads the per-replica sums of the last sim_batch_reduce for the stress.
 * The mouth heights are summed with FP64 atomics: the last bits of the
 * opening vary from run to run. */
int sim_batch_crack_observe(const SimBatch* b, const SimCrack* crack, const int8_t* mouth, int32_t total_bins,
                            uint64_t* bins, double* sums, double* out, void* stream);

/* Message for the last CUDA error seen by this library (host string). */
const char* sim_last_cuda_error(void);
int sim_version(void);
/* sizeof of SimBox, SimEngine, SimEAMTables, SimLJParams, SimIntegrator,
 * SimBerendsen, SimRep, SimBatch, SimMLP, SimAniso, SimBoxScale, SimIndenter,
 * SimCrack, SimLoaderCheck (host-only; lets bindings verify their struct
 * layouts; n >= 13, the first min(n, 14) are written). */
int sim_struct_sizes(int64_t* out, int32_t n);

#ifdef __cplusplus
}
#endif
#endif /* SIMB200_H */
