"""Differentiation and Newton polish: autograd gradients against the binary128 oracle's
analytic derivatives and against exact-phase central differences; batched Newton steps."""
import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu

K, TOL = 1.5e-10, 1e-10


@pytest.fixture(scope="module")
def setup(gpu):
    import torch
    from mertens_bound_b200.autograd import K2Torch
    data = synth.make_table(100_000, seed=1)
    t = k2.ZeroTable.from_data(data)
    ev = K2Torch(t, tol=TOL)
    yield torch, data, t, ev
    ev.close()
    t.close()


def _cand_tensors(torch, cd):
    dev = torch.device("cuda", 0)
    vi = torch.from_numpy(cd.v_int.view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(cd.v_frac.view(np.int64).copy()).to(dev)
    d = torch.from_numpy(cd.delta.copy()).to(dev)
    return vi, vf, d


def test_autograd_matches_oracle_derivatives(setup, oracle):
    torch, data, t, ev = setup
    cd = synth.make_candidates(16, seed=71)
    cd.delta[:] = np.linspace(-5e-5, 5e-5, 16)
    vi, vf, d = _cand_tensors(torch, cd)
    d.requires_grad_(True)
    k = torch.tensor(K, dtype=torch.float64, device=d.device, requires_grad=True)
    val = ev(vi, vf, d, k)
    w = torch.linspace(1.0, 2.0, 16, dtype=torch.float64, device=d.device)
    (w * val).sum().backward()
    hi, lo = oracle.k2(cd, data, K, data.n)
    wn = np.linspace(1.0, 2.0, 16)
    assert np.max(np.abs(val.detach().cpu().numpy() - hi[:, 0])) <= TOL
    gd = d.grad.cpu().numpy() / wn
    assert np.max(np.abs(gd - hi[:, 1])) <= 1e-6 * np.max(np.abs(hi[:, 1]))
    gk = float(k.grad.item())
    assert abs(gk - float(np.sum(wn * hi[:, 2]))) <= 1e-6 * float(np.sum(np.abs(wn * hi[:, 2])))


def test_gradient_vs_central_differences(setup, oracle):
    """dK2/ddelta against exact-phase central differences of K2: with step 1e-8 (where the
    difference quotient approximates the derivative to ~1e-7) and with step 1e-4 (compared
    with the oracle's own difference quotient at that step)."""
    torch, data, t, ev = setup
    cd = synth.make_candidates(8, seed=72)
    vi, vf, d = _cand_tensors(torch, cd)
    val, dd, dk = ev.evaluate(vi, vf, d, K)
    for h, rel in ((1e-8, 2e-6), (1e-4, None)):
        vp, _, _ = ev.evaluate(vi, vf, d + h, K)
        vm, _, _ = ev.evaluate(vi, vf, d - h, K)
        fd = ((vp - vm) / (2 * h)).cpu().numpy()
        if rel is not None:
            assert np.max(np.abs(fd - dd.cpu().numpy())) <= rel * np.max(np.abs(dd.cpu().numpy()))
        else:
            cp = cd.subset(np.arange(8)); cp.delta[:] = h
            cm = cd.subset(np.arange(8)); cm.delta[:] = -h
            op, _ = oracle.k2(cp, data, K, data.n)
            om, _ = oracle.k2(cm, data, K, data.n)
            ofd = (op[:, 0] - om[:, 0]) / (2 * h)
            assert np.max(np.abs(fd - ofd)) <= 2 * TOL / (2 * h) + 1e-9


def test_newton_polish_increases_abs_k2(setup, oracle):
    torch, data, t, ev = setup
    cd = synth.make_candidates(64, seed=73)
    vi, vf, d = _cand_tensors(torch, cd)
    d0 = d.clone()
    h0, val, dd, dk = ev.newton(vi, vf, d, K, iters=8, max_step=1e-4)
    h0, val, dd = h0.cpu().numpy(), val.cpu().numpy(), dd.cpu().numpy()
    delta = d.cpu().numpy()
    assert np.all(np.abs(val) >= np.abs(h0))
    moved = delta != d0.cpu().numpy()
    assert moved.sum() >= 32
    # at a moved point the slope is (nearly) zero and the value matches the oracle there
    assert np.median(np.abs(dd[moved])) < 1e-3 * np.median(np.abs(dk[moved].cpu().numpy()) * 1e-4)
    sub = cd.subset(np.arange(8))
    sub.delta[:] = delta[:8]
    hi, _ = oracle.k2(sub, data, K, data.n)
    assert np.max(np.abs(val[:8] - hi[:, 0])) <= TOL
