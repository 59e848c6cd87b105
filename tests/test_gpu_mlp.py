"""Descriptor-MLP surrogate on the GPU (C ABI group 4).

* descriptors against the FP64 restatement in oracle/mlp.py: 1e-4 relative
  (FP32 exponentials and cosines);
* forces from given dE/dG against autograd through the FP64 descriptors:
  2e-4 of the largest force component;
* the tensor-core network against a torch FP32 reference that rounds the
  same operands to BF16 (normalised descriptors, weights, hidden
  activations, backward deltas) -- remaining differences are FP32 summation
  order and exponentials: 5e-3 absolute on energies and dE/dG;
* training gradients against torch autograd of that reference: 3% of each
  parameter block's gradient norm (the kernel forms weight gradients from
  BF16-rounded activations and deltas);
* a short training run on EAM data cuts the energy loss tenfold and the
  force error of the untrained network at least in half.
"""
import numpy as np
import pytest
import torch

from oracle import inputs as oin
from oracle import mlp as omlp
from oracle import neighbor as onb
from oracle.box import OracleBox

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


def _system(sb, n=4, seed=3, tri=False):
    if tri:
        x, H = oin.bcc_triclinic(n)
    else:
        x, L = oin.bcc_lattice(n)
        H = np.diag([L] * 3)
    x = oin.jitter(x, 0.08, seed)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], H, 4.4, 0.5, device=DEV)
    hl = onb.half_list(x, OracleBox(H), 4.9 ** 2)
    pi = np.concatenate([hl["i"], hl["j"]])
    pj = np.concatenate([hl["j"], hl["i"]])
    return x, H, eng, pi, pj


def _slots_to_orig(eng, a):
    out = torch.empty_like(a[:eng.n])
    out[eng.orig[:eng.n].long()] = a[:eng.n]
    return out


@pytest.mark.parametrize("tri", [False, True])
def test_descriptors_match_oracle(sb, tri):
    from simulon_b200 import mlp
    x, H, eng, pi, pj = _system(sb, tri=tri)
    G = _slots_to_orig(eng, mlp.descriptors(eng)).cpu().double()
    Go = omlp.descriptors(torch.tensor(x), OracleBox(H), pi, pj)
    np.testing.assert_allclose(G.numpy(), Go.numpy(), rtol=1e-4, atol=1e-5)
    assert eng.status() == 0


def test_forces_from_descriptor_gradients_match_autograd(sb):
    from simulon_b200 import mlp
    x, H, eng, pi, pj = _system(sb, n=5, seed=4)
    net = omlp.random_net(1)
    G_slots = mlp.descriptors(eng)[:eng.n].double().cpu()
    net["mu"], net["sigma"] = G_slots.mean(0).numpy(), G_slots.std(0).numpy()
    Gr = G_slots.clone().requires_grad_(True)
    e = omlp.atom_energies(Gr, {k: torch.as_tensor(v) for k, v in net.items()})
    (dEdG,) = torch.autograd.grad(e.sum(), Gr)
    mlp.mlp_forces(eng, dEdG.float().to(DEV).contiguous())
    f = eng.gather("f").cpu().numpy()
    _, fo, _ = omlp.energy_forces(x, OracleBox(H), pi, pj, net)
    fo = fo.numpy()
    assert np.abs(f - fo).max() <= 2e-4 * np.abs(fo).max(), np.abs(f - fo).max()


def _bf(t):
    return t.to(torch.bfloat16).float()


def _torch_reference(G, net, target=None):
    """FP32 network with the kernel's BF16 roundings; returns (E, dEdG) or the loss."""
    p = {k: torch.as_tensor(v, dtype=torch.float32, device=G.device) for k, v in net.items()}
    g = _bf((G - p["mu"]) / p["sigma"])
    W1, W2 = _bf(p["W1"]), _bf(p["W2"])
    z1 = g @ W1 + p["b1"]
    h1 = _bf(torch.nn.functional.silu(z1))
    z2 = h1 @ W2 + p["b2"]
    E = torch.nn.functional.silu(z2) @ p["w3"] + p["b3"]
    if target is not None:
        return E
    s2 = torch.sigmoid(z2)
    d2 = _bf(p["w3"] * s2 * (1 + z2 * (1 - s2)))
    s1 = torch.sigmoid(z1)
    d1 = _bf((d2 @ W2.T) * s1 * (1 + z1 * (1 - s1)))
    return E, (d1 @ W1.T) / p["sigma"]


def _random_rows(n, seed=0):
    rng = np.random.default_rng(seed)
    G = np.abs(rng.normal(1.0, 0.6, (n, 16))) * np.linspace(0.5, 4.0, 16)
    return torch.tensor(G, dtype=torch.float32, device=DEV)


def test_tensor_core_network_matches_torch(sb):
    from simulon_b200 import mlp
    G = _random_rows(1000, 1)
    p = omlp.random_net(2, mu=G.mean(0).cpu().numpy(), sigma=G.std(0).cpu().numpy())
    net = mlp.MLPNet(DEV, p)
    E_ref, d_ref = _torch_reference(G, p)
    for _ in range(2):
        E, d = net.forward(G, G.shape[0])
        torch.cuda.synchronize()
        assert int(net.status.item()) == 0
        assert (E - E_ref).abs().max() < 5e-3, float((E - E_ref).abs().max())
        assert (d - d_ref).abs().max() < 5e-3 * max(1.0, float(d_ref.abs().max())), float((d - d_ref).abs().max())


def test_training_gradients_match_autograd(sb):
    from simulon_b200 import mlp
    G = _random_rows(640, 5)
    rng = np.random.default_rng(6)
    target = torch.tensor(rng.normal(-8.0, 0.3, 640), dtype=torch.float32, device=DEV)
    p = omlp.random_net(7, mu=G.mean(0).cpu().numpy(), sigma=G.std(0).cpu().numpy())
    net = mlp.MLPNet(DEV, p)
    grads = torch.zeros(mlp.N_PARAMS, device=DEV)
    loss = torch.zeros(1, device=DEV)
    net.train_grads(G, target, grads, loss)
    torch.cuda.synchronize()
    leaves = {k: torch.tensor(np.asarray(p[k], np.float32), device=DEV, requires_grad=True)
              for k in ("W1", "b1", "W2", "b2", "w3", "b3")}
    ref = dict(p)
    ref.update(leaves)
    E = _torch_reference(G, ref, target=target)
    L = ((E - target) ** 2).mean()
    L.backward()
    assert abs(float(loss) - float(L.detach())) <= 1e-3 * float(L.detach())
    for k, (o, shp) in mlp.OFF.items():
        n = int(np.prod(shp)) if shp else 1
        got = grads[o:o + n].cpu()
        want = leaves[k].grad.reshape(-1).cpu()
        assert float((got - want).norm()) <= 0.03 * float(want.norm()) + 1e-7, k


def test_training_reduces_energy_and_force_errors(sb, tables):
    from simulon_b200 import mlp
    G, E = mlp.generate_dataset(tables, n_cells=4, temperatures=(300.0, 1500.0), strains=(-0.03, 0.03),
                                frames_per_run=10, stride=10, equilibrate=50, seed=1, device=DEV)
    _, _, frames = mlp.generate_dataset(tables, n_cells=4, temperatures=(900.0,), strains=(0.0,), frames_per_run=3,
                                        stride=15, equilibrate=40, seed=2, device=DEV, with_forces=True)
    untrained = mlp.MLPNet(DEV, seed=3)
    untrained.set_normalisation(G)
    untrained.pack()
    rmse0 = mlp.force_rmse(untrained, tables, frames, DEV)
    net = mlp.MLPNet(DEV, seed=3)
    losses = mlp.train(net, G, E, steps=600, batch=2048, lr=3e-3, lr_final=3e-4, seed=4).cpu().numpy()
    first, last = losses[:20].mean(), losses[-20:].mean()
    assert last < 0.1 * first, (first, last)
    rmse = mlp.force_rmse(net, tables, frames, DEV)
    assert rmse < 0.5 * rmse0, (rmse0, rmse)


def test_surrogate_run_judges_and_falls_back(sb, tables):
    """The committed weights keep a 300 K run on the surrogate (force RMSE
    against EAM below 0.05 eV/A at each judgement); an untrained network is
    caught at the first judgement and the run continues on EAM."""
    from simulon_b200 import mlp
    from simulon_b200.engine import integrator_params
    x, L = oin.bcc_lattice(8)
    v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 300.0, 8)
    for weights, expect_mlp in ((mlp.default_weights_path(), True), (None, False)):
        eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, velocities=v,
                          device=DEV)
        net = mlp.MLPNet.load(weights, DEV) if weights else mlp.MLPNet(DEV, seed=0)
        ip = integrator_params(eng, 0.002, langevin=True, temperature=300.0, gamma=10.0, seed=1)
        run = mlp.SurrogateRun(eng, net, tables, ip, judge_every=100, tolerance=0.05).run(300)
        torch.cuda.synchronize()
        assert eng.status() == 0 and int(net.status.item()) == 0
        assert run.use_mlp == expect_mlp, run.rmse_history
        assert len(run.rmse_history) == (3 if expect_mlp else 1)
        assert np.isfinite(eng.gather("x").cpu().numpy()).all()


def test_force_contraction_matches_directional_derivative(sb):
    """u_i = sum_m e_m . dG_i/dx_m against a central difference of the FP64
    descriptors along e: 3e-4 of the largest component (FP32 exponentials)."""
    from simulon_b200 import mlp
    x, H, eng, pi, pj = _system(sb, n=4, seed=9, tri=False)
    rng = np.random.default_rng(10)
    e = rng.normal(0.0, 1.0, x.shape)
    ferr = torch.zeros(eng.n_pad, 4, device=DEV)
    slots = eng.orig[:eng.n].long().cpu()
    ferr[:eng.n, :3] = torch.tensor(e[slots.numpy()], dtype=torch.float32, device=DEV)
    u = _slots_to_orig(eng, mlp.force_contract(eng, ferr)).cpu().double().numpy()
    h = 1e-5
    box = OracleBox(H)
    Gp = omlp.descriptors(torch.tensor(x + h * e), box, pi, pj).numpy()
    Gm = omlp.descriptors(torch.tensor(x - h * e), box, pi, pj).numpy()
    want = (Gp - Gm) / (2 * h)
    assert np.abs(u - want).max() <= 3e-4 * np.abs(want).max(), np.abs(u - want).max()
    assert eng.status() == 0


def test_force_matching_gradients_match_double_backward(sb):
    """Kernel gradient of J = w_E mean (E - t)^2 + beta sum_i dE_i/dG_i . u_i
    (u fixed) against torch double-backward in FP32: 5% of each parameter
    block's gradient norm (BF16 operands of six GEMMs and the outer products);
    b3's gradient within 2 w_E x the 5e-3 energy tolerance."""
    from simulon_b200 import mlp
    n = 700
    G = _random_rows(n, 11)
    rng = np.random.default_rng(12)
    u = torch.tensor(rng.normal(0.0, 1.0, (n, 16)), dtype=torch.float32, device=DEV) * G.std(0)
    target = torch.tensor(rng.normal(-8.0, 0.3, n), dtype=torch.float32, device=DEV)
    p = omlp.random_net(13, mu=G.mean(0).cpu().numpy(), sigma=G.std(0).cpu().numpy())
    net = mlp.MLPNet(DEV, p)
    grads = torch.zeros(mlp.N_PARAMS, device=DEV)
    loss = torch.zeros(1, device=DEV)
    w_e, w_f, n_f = 0.7, 1.3, 500
    net.train_grads_fm(G, target, u, n, w_e, w_f, n_f, grads, loss)
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    leaves = {k: torch.tensor(np.asarray(p[k], np.float32), device=DEV, requires_grad=True)
              for k in ("W1", "b1", "W2", "b2", "w3", "b3")}
    ref = {k: torch.as_tensor(np.asarray(v, np.float32), device=DEV) for k, v in p.items()}
    ref.update(leaves)
    Gr = G.clone().requires_grad_(True)
    E = omlp.atom_energies(Gr, ref)
    (dEdG,) = torch.autograd.grad(E.sum(), Gr, create_graph=True)
    beta = -2.0 * w_f / (3.0 * n_f)
    J = w_e * ((E - target) ** 2).mean() + beta * (dEdG * u).sum()
    J.backward()
    mse = float(((E - target) ** 2).mean().detach())
    assert abs(float(loss) - mse) <= 2e-3 * mse
    for k, (o, shp) in mlp.OFF.items():
        cnt = int(np.prod(shp)) if shp else 1
        got = grads[o:o + cnt].cpu()
        want = leaves[k].grad.reshape(-1).cpu()
        if k == "b3":   # 2 w_E mean(E - t): a cancelling sum, bounded by the 5e-3 energy error
            assert abs(float(got - want)) <= 2 * w_e * 5e-3, (float(got), float(want))
            continue
        assert float((got - want).norm()) <= 0.05 * float(want.norm()) + 1e-7, (k, float((got - want).norm()),
                                                                                float(want.norm()))


def test_force_loss_gradient_matches_oracle(sb):
    """Whole force-matching chain (network, forces, contraction, gradient)
    against autograd of sum |F - F_t|^2 / (3n) through the FP64 oracle
    descriptors and network: 5% of each block's gradient norm."""
    from simulon_b200 import mlp
    x, H, eng, pi, pj = _system(sb, n=4, seed=14)
    G = mlp.descriptors(eng)
    Gn = G[:eng.n].double().cpu()
    p = omlp.random_net(15, mu=Gn.mean(0).numpy(), sigma=Gn.std(0).numpy())
    net = mlp.MLPNet(DEV, p)
    rng = np.random.default_rng(16)
    f_t = rng.normal(0.0, 0.5, x.shape)
    F_slots = torch.zeros(eng.n_pad, 4, device=DEV)
    slots = eng.orig[:eng.n].long().cpu().numpy()
    F_slots[:eng.n, :3] = torch.tensor(f_t[slots], dtype=torch.float32, device=DEV)
    e, d = net.forward(G, eng.n)
    mlp.mlp_forces(eng, d)
    ferr = eng.f32 - F_slots
    u = mlp.force_contract(eng, ferr)
    grads = torch.zeros(mlp.N_PARAMS, device=DEV)
    loss = torch.zeros(1, device=DEV)
    net.train_grads_fm(G, torch.zeros(eng.n, device=DEV), u, eng.n, 0.0, 1.0, eng.n, grads, loss)
    torch.cuda.synchronize()
    leaves = {k: torch.tensor(np.asarray(p[k]), dtype=torch.float64, requires_grad=True)
              for k in ("W1", "b1", "W2", "b2", "w3", "b3")}
    ref = {k: torch.as_tensor(np.asarray(v), dtype=torch.float64) for k, v in p.items()}
    ref.update(leaves)
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    Eo = omlp.atom_energies(omlp.descriptors(xt, OracleBox(H), pi, pj), ref)
    (gx,) = torch.autograd.grad(Eo.sum(), xt, create_graph=True)
    L = ((-gx - torch.tensor(f_t)) ** 2).sum() / (3 * len(x))
    L.backward()
    for k, (o, shp) in mlp.OFF.items():
        cnt = int(np.prod(shp)) if shp else 1
        got = grads[o:o + cnt].cpu().double()
        g = leaves[k].grad   # None for b3: a constant shift moves no force
        want = torch.zeros(cnt, dtype=torch.float64) if g is None else g.reshape(-1)
        assert float((got - want).norm()) <= 0.05 * float(want.norm()) + 1e-9, (k, float((got - want).norm()),
                                                                                float(want.norm()))


def test_autograd_function_matches_fp64_and_finite_differences(sb):
    """mlp_energy (torch.autograd.Function): its gradient against autograd of
    the FP64 restatement with the same weights (3% of the gradient norm: BF16
    network operands), whose own gradient matches central finite differences
    along random directions (1e-6 relative)."""
    from simulon_b200 import mlp
    x, H, eng, pi, pj = _system(sb, n=4, seed=22)
    net = mlp.MLPNet.load(mlp.default_weights_path(), DEV)
    p64 = {k: torch.as_tensor(v, dtype=torch.float64) for k, v in net.to_dict().items()}
    xt = torch.tensor(x, device=DEV, requires_grad=True)
    E = mlp.mlp_energy(xt, eng, net)
    (g,) = torch.autograd.grad(E, xt)
    g = g.cpu()
    box = OracleBox(H)

    def e64(xx):
        return omlp.atom_energies(omlp.descriptors(xx, box, pi, pj), p64).sum()
    xo = torch.tensor(x, requires_grad=True)
    Eo = e64(xo)
    (go,) = torch.autograd.grad(Eo, xo)
    assert abs(float(E.detach()) - float(Eo.detach())) <= 2e-3 * len(x)
    assert float((g - go).norm()) <= 0.03 * float(go.norm()), (float((g - go).norm()), float(go.norm()))
    rng = np.random.default_rng(23)
    h = 1e-4
    with torch.no_grad():
        for _ in range(3):
            v = torch.tensor(rng.normal(size=x.shape))
            v /= v.norm()
            fd = (e64(torch.tensor(x) + h * v) - e64(torch.tensor(x) - h * v)) / (2 * h)
            assert abs(float(fd) - float((go * v).sum())) <= 1e-6 * float(go.norm()) + 1e-9
    assert eng.status() == 0
