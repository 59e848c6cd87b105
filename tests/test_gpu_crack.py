"""Crack observables on the device (sim_batch_crack_observe) against the
reference's own functions (tests/golden/crack_obs_w3000.npz): two replicas
of one batch, the precracked slab and the opened one, measured from the
precracked reference positions; crack length and extension exact, CMOD to
1e-10 A; the projected stress against the formula on the replica sums."""
import numpy as np
import pytest
import torch

from oracle import inputs as oin

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def test_crack_observables_match_reference(tmp_path):
    import os
    import simulon_b200 as sb
    from simulon_b200 import _lib
    from simulon_b200.batch import BatchedEngine, CrackObserver, Replica, crack_slab
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with np.load(os.path.join(here, "crack_obs_w3000.npz")) as z:
        g = {k: z[k] for k in z.files}
    base = crack_slab(3000, seed=5)
    np.testing.assert_array_equal(base.positions, g["x0"])
    reps = [Replica(positions=g[k], H=g["H"], velocities=np.zeros_like(g[k]), temperature=300.0, grip=base.grip,
                    grip_axis=1, grip_rate=0.0, meta=dict(base.meta)) for k in ("x0", "x1")]
    batch = BatchedEngine(reps, oin.W_MASS, 4.4, 0.75, device=DEV)
    ref = np.concatenate([g["x0"], g["x0"]])
    obs = CrackObserver(batch, threshold=float(g["threshold"]), bins=int(g["bins"]), reference_positions=ref)
    pot = oin.write_fs_w_setfl(str(tmp_path / "W.eam.fs"))
    tables = sb.EAMDeviceTables(sb.EAMParser(pot), DEV)
    batch.eam_forces(tables)
    out = obs.observe().cpu().numpy()
    for k, tag in enumerate(("0", "1")):
        assert out[k, 4] == float(g["length" + tag]), (k, out[k, 4], float(g["length" + tag]))
        assert abs(out[k, 5] - float(g["extension" + tag])) < 1e-12
        assert abs(out[k, 3] - float(g["cmod" + tag])) < 1e-10
        assert abs(out[k, 2] - abs(float(g["cmod" + tag]))) < 1e-10
    # stress: (K + W) / V projected on the normalised box row 1, in bar
    red = batch.rep_red.cpu().numpy()
    for k in range(2):
        r = red[k]
        t = np.array([[r[10] + r[3], r[13] + r[6], r[14] + r[7]], [r[13] + r[6], r[11] + r[4], r[15] + r[8]],
                      [r[14] + r[7], r[15] + r[8], r[12] + r[5]]])
        H = g["H"]
        yu = H[1] / np.linalg.norm(H[1])
        pyy = yu @ t @ yu / abs(np.linalg.det(H)) * 1602176.6208
        assert abs(out[k, 1] - pyy) <= 1e-9 * max(1.0, abs(pyy)) and out[k, 0] == -out[k, 1]
    assert batch.status() == 0
    # the observation can be captured with the batched steps
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gr, stream=s):
        obs.observe()
    torch.cuda.current_stream().wait_stream(s)
    obs.out.zero_()
    gr.replay()
    torch.cuda.synchronize()
    np.testing.assert_allclose(obs.out.cpu().numpy(), out, rtol=1e-12, atol=1e-12)   # FP64 atomic sums
    assert _lib.SIM_CRACK_OUT == 8
