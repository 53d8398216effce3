"""Adjoint gradient of the loss as a torch.autograd.Function, against central
finite differences of the library's own loss (h = 1e-6, relative 1e-6) and
against the oracle's gradient (the reference's formula, 1e-9 relative)."""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from gprat_b200 import capi, autograd
    assert capi.device_count() >= 1
    n, T, d = 1024, 128, 8
    x, y, _ = O.synthetic(n, 16, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    return torch, autograd, gp, (x, y, n, T, d)


@pytest.mark.parametrize("hyper", [(1.0, 1.0, 0.1), (0.7, 1.5, 0.02)])
def test_backward_matches_central_differences(setup, hyper):
    torch, autograd, gp, _ = setup
    h = torch.tensor(hyper, dtype=torch.float64, requires_grad=True)
    loss = autograd.nlml(gp, h)
    loss.backward()
    g = h.grad.numpy()
    step = 1e-6
    fd = np.zeros(3)
    for p in range(3):
        hp, hm = list(hyper), list(hyper)
        hp[p] += step
        hm[p] -= step
        fd[p] = (gp.compute_loss(hp) - gp.compute_loss(hm)) / (2 * step)
    assert np.allclose(g, fd, rtol=1e-6, atol=1e-9), (g, fd)
    assert abs(loss.item() - gp.compute_loss(hyper)) <= 1e-14 * abs(loss.item())


def test_backward_matches_oracle_gradient(setup):
    torch, autograd, gp, (x, y, n, T, d) = setup
    hyper = (1.2, 0.9, 0.05)
    h = torch.tensor(hyper, dtype=torch.float64, requires_grad=True)
    autograd.nlml(gp, h).backward()
    o = O.OracleGP(x, y, n // T, T, d, hyper)
    loss_o, g_u = o.gradient()
    scale = np.array([O.sigmoid(O.to_unconstrained(hyper[0], False)), O.sigmoid(O.to_unconstrained(hyper[1], False)),
                      O.sigmoid(O.to_unconstrained(hyper[2], True))])
    g_o = g_u / scale
    assert np.allclose(h.grad.numpy(), g_o, rtol=1e-9, atol=1e-12)


def test_chain_rule_through_torch_ops(setup):
    """The loss composes with other torch ops (log-parameterised hyper-parameters)."""
    torch, autograd, gp, _ = setup
    logh = torch.log(torch.tensor([1.0, 1.0, 0.1], dtype=torch.float64)).requires_grad_(True)
    loss = autograd.nlml(gp, torch.exp(logh)) * 2.0
    loss.backward()
    h = torch.tensor([1.0, 1.0, 0.1], dtype=torch.float64, requires_grad=True)
    autograd.nlml(gp, h).backward()
    assert torch.allclose(logh.grad, 2.0 * h.grad * torch.tensor([1.0, 1.0, 0.1], dtype=torch.float64), rtol=1e-12)
    # a few gradient-descent steps on the loss lower it
    p = torch.tensor([1.0, 1.0, 0.1], dtype=torch.float64).log().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.05)
    first = None
    for _ in range(10):
        opt.zero_grad()
        lo = autograd.nlml(gp, p.exp())
        lo.backward()
        opt.step()
        first = lo.item() if first is None else first
    assert autograd.nlml(gp, p.exp().detach()).item() < first
