"""sim_eam_forces_static (EAM forces with the library's fixed scratch array)
against sim_eam_forces (caller-allocated scratch) on the same engine state.

Tolerance: forces within 1e-6 eV/A absolute, energies and virial within
1e-12 relative (the two calls run the same kernels, so they normally agree
bit for bit).  The file name keeps it last in collection order, so it runs
both alone and after every other GPU test in the same process.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import inputs as oin


@pytest.fixture(scope="module")
def sb():
    import simulon_b200
    from simulon_b200 import build
    build.build()
    simulon_b200._lib.load()
    return simulon_b200


@pytest.fixture(scope="module")
def fsw_path(tmp_path_factory):
    return oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))


def test_static_scratch_rejects_oversize_system(sb):
    """Too many atom slots: SIM_ERR_ARG with the limit in the message, before any CUDA call."""
    lib, L = sb._lib.load(), sb._lib
    e = L.SimEngine()
    e.n = L.SIM_STATIC_MAX_ATOMS + 1
    e.n_pad = L.SIM_STATIC_MAX_ATOMS + 128
    t = L.SimEAMTables()
    assert lib.sim_eam_forces_static(ctypes.byref(e), ctypes.byref(t), None) == L.SIM_ERR_ARG
    assert str(L.SIM_STATIC_MAX_ATOMS).encode() in lib.sim_last_cuda_error()
    assert lib.sim_eam_forces_static(None, ctypes.byref(t), None) == L.SIM_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("tri", [False, True])
def test_static_scratch_matches_sim_eam_forces(sb, fsw_path, tri):
    dev = torch.device("cuda")
    if tri:
        x, H = oin.bcc_triclinic(12)
    else:
        x, Lb = oin.bcc_lattice(16)
        H = np.diag([Lb] * 3)
    x = oin.jitter(x, 0.07, 61)
    parser = sb.EAMParser(fsw_path)
    tables = sb.EAMDeviceTables(parser, dev)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], H, parser.cutoff, 0.5, device=dev)
    assert eng.n_pad <= sb._lib.SIM_STATIC_MAX_ATOMS
    eng.eam_forces(tables)
    f_ref = eng.gather("f").cpu()
    red_ref = eng.red_out.cpu().numpy().copy()
    # the engine's own scratch is filled with garbage and must stay untouched
    eng.posfp.fill_(0x7F7F7F7F)
    posfp_before = eng.posfp.clone()
    for _ in range(2):
        eng.f32.zero_()
        eng.red_out.zero_()
        sb._lib.call("sim_eam_forces_static", eng.st_ref, tables.ref, eng.stream)
        torch.cuda.synchronize()
        f = eng.gather("f").cpu()
        red = eng.red_out.cpu().numpy()
        torch.testing.assert_close(f, f_ref, rtol=0.0, atol=1e-6)
        np.testing.assert_allclose(red[:9], red_ref[:9], rtol=1e-12, atol=1e-12)
        assert eng.status() == 0
    assert torch.equal(eng.posfp, posfp_before)
