"""Launch-shape autotuning on the GPU: every candidate shape gives the same
results (EAM forces bit-identical, energies to FP64 summation order; MLP
descriptors to FP32 summation order, forces from the same dE/dG to
float-atomic order), and the
tuner stores shapes from its candidate lists."""
import numpy as np
import pytest
import torch

from oracle import inputs as oin

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def sb():
    import simulon_b200
    simulon_b200._lib.load()
    return simulon_b200


@pytest.fixture(scope="module")
def tables(sb, tmp_path_factory):
    path = oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))
    return sb.EAMDeviceTables(sb.EAMParser(path), DEV)


def _engine(sb, n=12, seed=31):
    x, L = oin.bcc_lattice(n)
    x = oin.jitter(x, 0.06, seed)
    return sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)


def test_eam_shapes_agree_and_tuner_picks_a_candidate(sb, tables, tmp_path):
    from simulon_b200 import autotune
    eng = _engine(sb)
    eng.eam_forces(tables)
    f0, e0 = eng.f32.clone(), eng.red_out.clone()
    for d in autotune.EAM_DENSITY_THREADS:
        for f in autotune.EAM_FORCE_THREADS:
            eng.set_launch(eam_density_threads=d, eam_force_threads=f)
            eng.eam_forces(tables)
            assert torch.equal(eng.f32, f0), (d, f)
            torch.testing.assert_close(eng.red_out, e0, rtol=1e-12, atol=1e-9)
    hit = autotune.tune_eam(eng, tables, reps=3, path=str(tmp_path / "c.json"))
    assert hit["density_threads"] in autotune.EAM_DENSITY_THREADS
    assert hit["force_threads"] in autotune.EAM_FORCE_THREADS
    assert eng.launch[:2] == [hit["density_threads"], hit["force_threads"]]
    assert all(v > 0 for v in hit["ms"].values())
    eng.eam_forces(tables)
    assert torch.equal(eng.f32, f0) and eng.status() == 0


def test_mlp_groups_agree_and_tuner_picks_a_candidate(sb, tmp_path):
    from simulon_b200 import autotune, mlp
    eng = _engine(sb, n=10, seed=32)
    net = mlp.MLPNet.load(mlp.default_weights_path(), DEV)
    out = {}
    d = None   # one dE/dG for both force kernels (the network rounds its inputs to BF16)
    for g in autotune.MLP_GROUPS:
        eng.set_launch(mlp_desc_group=g, mlp_force_group=g)
        G = mlp.descriptors(eng)
        if d is None:
            _, d = net.forward(G, eng.n)
        mlp.mlp_forces(eng, d)
        out[g] = (G[:eng.n].clone(), eng.f32[:eng.n, :3].clone())
    torch.testing.assert_close(out[4][0], out[8][0], rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(out[4][1], out[8][1], rtol=1e-4, atol=1e-5)
    hit = autotune.tune_mlp(eng, reps=3, path=str(tmp_path / "c.json"), dEdG=d)
    assert hit["desc_group"] in autotune.MLP_GROUPS and hit["force_group"] in autotune.MLP_GROUPS
    assert eng.launch[2:] == [hit["desc_group"], hit["force_group"]]
    assert eng.status() == 0
