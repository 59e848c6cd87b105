"""ctypes binding of libsimb200.so (the C ABI declared in include/simb200.h).

The library is built in-tree (``simulon_b200/lib/libsimb200.so``) by
``simulon_b200.build``.  There is no CPU fallback: importing the engine on a
machine without the built library, or calling it with CPU tensors, raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsimb200.so")

SIM_OK = 0
SIM_ERR_ARG = 1
SIM_ERR_CUDA = 2
SIM_ERR_BOX = 4
SIM_STATUS_OVERFLOW = 8
SIM_STATUS_NONFINITE = 16
SIM_STATUS_HALO = 64
SIM_STATUS_MLP_NEIGHBORS = 128
SIM_STATUS_MLP_TIMEOUT = 256
SIM_STATUS_CELLS = 512
BOXSCALE_WORK = 64          # doubles of the sim_aniso_npt / sim_box_scale work buffer
SIM_STATIC_MAX_ATOMS = 262144   # atom-slot limit of sim_eam_forces_static
SIM_BATCH_RED_SPLIT = 8         # blocks that share one replica's reduction

RED_EPOT_EMBED, RED_EPOT_PAIR, RED_VIRIAL = 0, 1, 2
RED_W = slice(3, 9)          # xx yy zz xy xz yz
RED_KE = 9
RED_K = slice(10, 16)
RED_SLOTS = 16

c_p = ctypes.c_void_p


class SimBox(ctypes.Structure):
    _fields_ = [("H", ctypes.c_double * 9), ("Hinv", ctypes.c_double * 9), ("Hf", ctypes.c_float * 9),
                ("orthogonal", ctypes.c_int32), ("pad", ctypes.c_int32 * 3)]


class SimEngine(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("n_pad", ctypes.c_int64),
                ("n_types", ctypes.c_int32), ("nbr_cap", ctypes.c_int32),
                ("ncell", ctypes.c_int32 * 3), ("n_cells", ctypes.c_int32),
                ("x_rc", ctypes.c_double), ("skin_half2", ctypes.c_double),
                ("box", c_p),
                ("x", c_p), ("v", c_p), ("f32", c_p), ("f64", c_p), ("posq", c_p), ("xref", c_p),
                ("orig", c_p), ("posfp", c_p), ("nbr", c_p), ("nnbr", c_p),
                ("cell_of", c_p), ("cell_count", c_p), ("cell_start", c_p), ("cell_rank", c_p),
                ("perm", c_p), ("x_alt", c_p), ("v_alt", c_p), ("f32_alt", c_p), ("f64_alt", c_p),
                ("orig_alt", c_p),
                ("inv_mass", c_p), ("mass", c_p),
                ("flags", c_p), ("partials", c_p), ("red_counter", c_p), ("red_out", c_p),
                ("n_blocks_max", ctypes.c_int32), ("box_orthogonal", ctypes.c_int32),
                ("n_tiles", ctypes.c_int32), ("halo_cap", ctypes.c_int32),
                ("halo", c_p), ("halo_n", c_p), ("nbr16", c_p), ("cut_mask", c_p),
                ("launch", ctypes.c_int32 * 4)]


class SimEAMTables(ctypes.Structure):
    _fields_ = [("density", c_p), ("density_deriv", c_p), ("pair", c_p), ("pair_deriv", c_p),
                ("embed", c_p), ("embed_deriv", c_p), ("rho_min", c_p), ("inv_drho", c_p),
                ("rho_clamp_hi", c_p), ("dens_vd", c_p), ("deriv_vd", c_p), ("pair_vd", c_p),
                ("n_types", ctypes.c_int32), ("n_r", ctypes.c_int32), ("n_rho", ctypes.c_int32),
                ("pad", ctypes.c_int32),
                ("cutoff", ctypes.c_float), ("inv_dr", ctypes.c_float), ("r_clamp_hi", ctypes.c_float),
                ("pad2", ctypes.c_float)]


class SimLJParams(ctypes.Structure):
    _fields_ = [("c4eps", c_p), ("c24eps", c_p), ("sigma", c_p), ("u_rc", c_p), ("f_rc", c_p),
                ("n_types", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("rc", ctypes.c_double), ("rs", ctypes.c_double)]


class SimIntegrator(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("damp", ctypes.c_double), ("rff", c_p),
                ("seed", ctypes.c_uint64), ("step_ctr", c_p),
                ("langevin", ctypes.c_int32), ("pad", ctypes.c_int32)]


class SimBerendsen(ctypes.Structure):
    _fields_ = [("target_bar", ctypes.c_double), ("tau", ctypes.c_double), ("kappa", ctypes.c_double),
                ("mu_max", ctypes.c_double), ("dt", ctypes.c_double),
                ("coordinate_scale_power", ctypes.c_int32), ("reset_reference", ctypes.c_int32)]


class SimAniso(ctypes.Structure):
    _fields_ = [("target_bar", ctypes.c_double * 3), ("tau_p", ctypes.c_double), ("gamma_p", ctypes.c_double),
                ("max_eta_dot", ctypes.c_double), ("kappa_bar_inv", ctypes.c_double), ("tol_bar", ctypes.c_double),
                ("dt", ctypes.c_double), ("temperature", ctypes.c_double), ("eta_dot", ctypes.c_void_p),
                ("counter", ctypes.c_void_p), ("control", ctypes.c_int32 * 3), ("stochastic", ctypes.c_int32),
                ("reset_reference", ctypes.c_int32), ("seed", ctypes.c_uint32)]


class SimBoxScale(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_double * 3), ("vel_scale", ctypes.c_double * 3),
                ("reset_reference", ctypes.c_int32), ("pad", ctypes.c_int32)]


class SimLoaderCheck(ctypes.Structure):
    _fields_ = [("axis", ctypes.c_int32), ("pad", ctypes.c_int32), ("rebuild_strain", ctypes.c_double),
                ("regrid_margin", ctypes.c_double)]


LOADER_STATE = 32


class SimIndenter(ctypes.Structure):
    _fields_ = [("center", ctypes.c_void_p), ("radius", ctypes.c_double), ("stiffness", ctypes.c_double),
                ("out", ctypes.c_void_p)]


class SimCrack(ctypes.Structure):
    _fields_ = [("x_unit", ctypes.c_double * 3), ("y_unit", ctypes.c_double * 3), ("y_plane", ctypes.c_double),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double), ("x_center", ctypes.c_double),
                ("half_length", ctypes.c_double), ("threshold", ctypes.c_double), ("initial_cmod", ctypes.c_double),
                ("bins", ctypes.c_int32), ("bin_off", ctypes.c_int32), ("n_upper", ctypes.c_int32),
                ("n_lower", ctypes.c_int32)]


SIM_CRACK_OUT = 8


class SimRep(ctypes.Structure):
    _fields_ = [("box", SimBox), ("off", ctypes.c_int64), ("first", ctypes.c_int64),
                ("n", ctypes.c_int32), ("n_slots", ctypes.c_int32), ("ncell", ctypes.c_int32 * 3),
                ("n_cells", ctypes.c_int32), ("cell_off", ctypes.c_int32), ("grip_axis", ctypes.c_int32),
                ("grip_rate", ctypes.c_double)]


class SimBatch(ctypes.Structure):
    _fields_ = [("e", SimEngine), ("rep", c_p), ("n_rep", ctypes.c_int32), ("n_cell_entries", ctypes.c_int32),
                ("slot_rep", c_p), ("cell_rep", c_p), ("rep_flags", c_p), ("rep_rebuilds", c_p), ("work", c_p), ("grip", c_p),
                ("gref", c_p), ("rep_rff", c_p), ("chunk_red", c_p), ("rep_red", c_p)]


class SimMLP(ctypes.Structure):
    _fields_ = [("w1t_img", c_p), ("w2t_img", c_p), ("w2_img", c_p), ("w1_img", c_p), ("b1", c_p), ("b2", c_p),
                ("w3", c_p), ("b3", c_p), ("mu", c_p), ("inv_sigma", c_p)]


_P = ctypes.POINTER
# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "sim_legacy_density_pass": [c_p, c_p, c_p, c_p, ctypes.c_int64, c_p, ctypes.c_int32, ctypes.c_double,
                                ctypes.c_int64, c_p, c_p],
    "sim_legacy_force_pass": [c_p, c_p, c_p, c_p, c_p, ctypes.c_int64, c_p, c_p, c_p, ctypes.c_int32,
                              ctypes.c_double, ctypes.c_int64, c_p, c_p],
    "sim_legacy_lj_energy_force": [c_p, c_p, c_p, ctypes.c_int64, c_p, c_p, ctypes.c_float, ctypes.c_int32,
                                   ctypes.c_float, ctypes.c_float, c_p, c_p, c_p],
    "sim_half_list_count": [c_p, ctypes.c_int32, ctypes.c_int64, _P(SimBox), ctypes.c_double, c_p, c_p, c_p,
                            c_p, c_p, c_p, c_p],
    "sim_half_list_fill": [c_p, ctypes.c_int32, ctypes.c_int64, _P(SimBox), ctypes.c_double, c_p, c_p, c_p,
                           c_p, c_p, c_p, c_p, c_p, c_p, c_p],
    "sim_engine_load": [_P(SimEngine), c_p, c_p, c_p, c_p],
    "sim_rebuild": [_P(SimEngine), ctypes.c_int32, c_p],
    "sim_rebuild_if_needed": [_P(SimEngine), c_p],
    "sim_eam_forces": [_P(SimEngine), _P(SimEAMTables), c_p],
    "sim_eam_forces_static": [_P(SimEngine), _P(SimEAMTables), c_p],
    "sim_eam_density": [_P(SimEngine), _P(SimEAMTables), c_p],
    "sim_eam_force": [_P(SimEngine), _P(SimEAMTables), c_p],
    "sim_eam_force_integrate": [_P(SimEngine), _P(SimEAMTables), _P(SimIntegrator), c_p],
    "sim_eam_force_integrate_drift": [_P(SimEngine), _P(SimEAMTables), _P(SimIntegrator), c_p],
    "sim_eam_force_integrate_indenter": [_P(SimEngine), _P(SimEAMTables), _P(SimIntegrator), _P(SimIndenter),
                                         ctypes.c_int32, c_p],
    "sim_eam_step_drift_indenter": [_P(SimEngine), _P(SimEAMTables), _P(SimIntegrator), _P(SimIndenter), c_p,
                                    ctypes.c_int32, c_p, ctypes.c_int32, c_p],
    "sim_eam_step_drift": [_P(SimEngine), _P(SimEAMTables), _P(SimIntegrator), c_p, ctypes.c_int32, c_p,
                           ctypes.c_int32, c_p],
    "sim_lj_forces": [_P(SimEngine), _P(SimLJParams), ctypes.c_int32, c_p],
    "sim_lj_forces_integrate": [_P(SimEngine), _P(SimLJParams), _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_lj_forces_add": [_P(SimEngine), _P(SimLJParams), c_p],
    "sim_integrate_first": [_P(SimEngine), _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_integrate_second": [_P(SimEngine), _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_integrate_second_first": [_P(SimEngine), _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_berendsen": [_P(SimEngine), _P(SimBerendsen), c_p, c_p],
    "sim_berendsen_mu": [_P(SimEngine), _P(SimBerendsen), c_p, c_p],
    "sim_berendsen_scale_first": [_P(SimEngine), _P(SimBerendsen), c_p, _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_aniso_npt": [_P(SimEngine), _P(SimAniso), c_p, c_p],
    "sim_box_scale": [_P(SimEngine), _P(SimBoxScale), c_p, c_p],
    "sim_loader_check": [_P(SimEngine), _P(SimLoaderCheck), c_p, c_p],
    "sim_aniso_control": [_P(SimEngine), _P(SimAniso), c_p, c_p],
    "sim_box_scale_after_first": [_P(SimEngine), c_p, ctypes.c_int32, _P(SimBoxScale), c_p, _P(SimIntegrator),
                                  ctypes.c_int32, c_p],
    "sim_tensile_link": [_P(SimEngine), _P(SimAniso), c_p, c_p, c_p, ctypes.c_int32, c_p, ctypes.c_int32,
                         _P(SimBoxScale), c_p, _P(SimIntegrator), ctypes.c_int32, _P(SimLoaderCheck), c_p, c_p],
    "sim_indenter_add": [_P(SimEngine), _P(SimIndenter), ctypes.c_int32, c_p],
    "sim_batch_crack_observe": [c_p, c_p, c_p, ctypes.c_int32, c_p, c_p, c_p, c_p],
    "sim_gather_original_f64": [_P(SimEngine), c_p, c_p, c_p],
    "sim_gather_original_f32": [_P(SimEngine), c_p, c_p, c_p],
    "sim_scatter_original_f64": [_P(SimEngine), c_p, c_p, c_p],
    "sim_log_step": [_P(SimEngine), c_p, c_p, ctypes.c_int32, c_p, ctypes.c_int32, c_p],
    "sim_format_xyz_rows": [c_p, c_p, ctypes.c_int64, c_p, ctypes.c_int32, c_p, ctypes.c_int64],
    "sim_engine_half_count": [_P(SimEngine), ctypes.c_double, c_p, c_p],
    "sim_engine_half_fill": [_P(SimEngine), ctypes.c_double, c_p, c_p, c_p, c_p, c_p],
    "sim_scan_i64": [c_p, ctypes.c_int64, c_p, c_p],
    "sim_batch_load": [_P(SimBatch), c_p, c_p, c_p, c_p],
    "sim_batch_rebuild": [_P(SimBatch), ctypes.c_int32, c_p],
    "sim_batch_rebuild_if_needed": [_P(SimBatch), c_p],
    "sim_batch_eam_density": [_P(SimBatch), _P(SimEAMTables), c_p],
    "sim_batch_eam_force": [_P(SimBatch), _P(SimEAMTables), _P(SimIntegrator), ctypes.c_int32, c_p],
    "sim_batch_first_half": [_P(SimBatch), _P(SimIntegrator), c_p],
    "sim_batch_reduce": [_P(SimBatch), c_p, c_p, ctypes.c_int32, c_p],
    "sim_batched_step": [_P(SimBatch), _P(SimEAMTables), _P(SimIntegrator), ctypes.c_int32, c_p, ctypes.c_int32,
                         c_p],
    "sim_batch_gather_f64": [_P(SimBatch), c_p, c_p, c_p],
    "sim_batch_gather_f32": [_P(SimBatch), c_p, c_p, c_p],
    "sim_mlp_descriptors": [_P(SimEngine), c_p, c_p],
    "sim_mlp_forward": [_P(SimMLP), c_p, ctypes.c_int64, c_p, c_p, c_p, c_p],
    "sim_mlp_backward": [_P(SimEngine), c_p, c_p],
    "sim_mlp_train_grads": [_P(SimMLP), c_p, c_p, ctypes.c_int64, c_p, c_p, c_p, c_p],
    "sim_mlp_force_contract": [_P(SimEngine), c_p, c_p, c_p],
    "sim_mlp_train_grads_fm": [_P(SimMLP), c_p, c_p, c_p, ctypes.c_int64, ctypes.c_float, ctypes.c_float,
                               ctypes.c_int64, c_p, c_p, c_p, c_p],
    "sim_mlp_train_step": [_P(SimMLP), c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, ctypes.c_int64, ctypes.c_float,
                           ctypes.c_float, ctypes.c_int64, c_p, c_p, c_p, ctypes.c_float, ctypes.c_int32, c_p, c_p,
                           c_p],
    "sim_mlp_pack": [c_p, c_p, c_p, c_p, c_p, c_p],
    "sim_autotune_eam": [_P(SimEngine), _P(SimEAMTables), ctypes.c_int32, c_p, c_p, c_p],
    "sim_autotune_mlp": [_P(SimEngine), c_p, c_p, ctypes.c_int32, c_p, c_p, c_p],
    "sim_mlp_adam": [c_p, c_p, c_p, c_p, ctypes.c_float, ctypes.c_int32, c_p],
    "sim_eam_atom_energy": [_P(SimEngine), _P(SimEAMTables), c_p, c_p],
    "sim_last_cuda_error": [],
    "sim_version": [],
    "sim_struct_sizes": [c_p, ctypes.c_int32],
}
STRUCTS = (SimBox, SimEngine, SimEAMTables, SimLJParams, SimIntegrator, SimBerendsen, SimRep, SimBatch, SimMLP,
           SimAniso, SimBoxScale, SimIndenter, SimCrack, SimLoaderCheck)
_RESTYPES = {"sim_last_cuda_error": ctypes.c_char_p, "sim_format_xyz_rows": ctypes.c_int64}

_lib = None


class SimError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Load the shared library and declare every exported entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libsimb200.so not built ({path}); run `python -m simulon_b200.build`")
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(rc: int, what: str):
    if rc == SIM_OK:
        return
    msg = {SIM_ERR_ARG: "invalid argument", SIM_ERR_CUDA: "CUDA error", SIM_ERR_BOX: "box too small"}.get(rc, str(rc))
    detail = ""
    if rc == SIM_ERR_CUDA:
        detail = ": " + load().sim_last_cuda_error().decode()
    raise SimError(f"{what} failed ({msg}){detail}")


def call(name: str, *args):
    """Call an entry point and raise SimError on a non-zero status."""
    check(getattr(load(), name)(*args), name)


def ptr(t) -> int:
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_of(device=None) -> int:
    import torch
    return torch.cuda.current_stream(device).cuda_stream
