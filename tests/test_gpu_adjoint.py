"""The P2M adjoint in the form the benchmark times (mixed precision) at the
adjoint workload's size, and the autograd wrapper of the test harness.

Workload (128^3 periodic mesh, 4,194,304 particles uniform in the cube, lda 1,
w ~ N(0,1), target T ~ N(0,1) per unique node): loss L = 0.5 |P2M(x,w) - T|^2.
dL/dw is the oracle's M2P of the residual r = P2M(x,w) - T (after a ghost
get, the reference's M2P semantics); dL/dx is checked against FP64 central
differences of the oracle's loss (step 1e-6 h) on 200 particles.
"""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import max_rel, periodic_fill, random_particles, topo_for, unique_view
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_next_id = [1400]


def registered(nc):
    _next_id[0] += 1
    t = topo_for(3, nc, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def _spread(rng, xp, nc, k, sep=6):
    """k particle indices whose stencil origins are >= sep cells apart
    (periodic Chebyshev distance): their 6-node windows never overlap."""
    cells = np.floor(xp * nc).astype(np.int64)
    chosen = []
    for p in rng.permutation(xp.shape[1]):
        c = cells[:, p]
        ok = True
        for q in chosen:
            d = np.abs(c - cells[:, q])
            d = np.minimum(d, nc - d)
            if d.max() < sep:
                ok = False
                break
        if ok:
            chosen.append(p)
            if len(chosen) == k:
                break
    return np.array(chosen)


def fd_gradients(t, xp, w, r_unique, idx, nc, kernel=2):
    """FP64 central differences of L = 0.5 |P2M(x, w) - T|^2 with respect to
    the positions of particles idx (their stencils pairwise disjoint), from the
    oracle's P2M of the moved particles alone:
    L(x+e) - L(x-e) = sum_n r_n (d+_n - d-_n) + (d+_n^2 - d-_n^2) / 2, with
    d+- the change of particle p's deposit and r the residual at x."""
    h = 1.0 / nc
    e = 1e-6 * h
    g = [2, 2, 2]
    xs = np.asfortranarray(xp[:, idx])
    ws = np.asfortranarray(w[:, idx])
    f0, lb, _ = O.p2m(t, xs, ws, kernel, g)
    base = unique_view(f0, lb, [nc] * 3, 3)[0]
    cells = np.floor(xs * nc).astype(np.int64)
    # nodes i0-2 .. i0+3 of each particle (its support, also after a move across a face)
    win = [(cells[a][:, None] + np.arange(-2, 4)[None, :]) % nc for a in range(3)]
    out = np.zeros((3, len(idx)))
    for a in range(3):
        dp, dm = [], []
        for sgn, acc in ((1.0, dp), (-1.0, dm)):
            xm = xs.copy(order="F")
            xm[a] += sgn * e
            fm, lbm, _ = O.p2m(t, xm, ws, kernel, g)
            acc.append(unique_view(fm, lbm, [nc] * 3, 3)[0] - base)
        dp, dm = dp[0], dm[0]
        for j in range(len(idx)):
            sl = np.ix_(win[0][j], win[1][j], win[2][j])
            rp, pp, mm = r_unique[sl], dp[sl], dm[sl]
            dl = (rp * (pp - mm)).sum() + 0.5 * ((pp * pp).sum() - (mm * mm).sum())
            out[a, j] = dl / (2 * e)
    return out


@pytest.mark.slow
@pytest.mark.parametrize("mode", [1, 0])
def test_adjoint_at_workload_size(mode):
    """Mixed (the benchmarked form) and FP64: dw against the oracle's M2P of
    the residual (<= 1e-6 mixed, <= 1e-13 FP64), dx against FP64 central
    differences (<= 1e-4), the forward field against the oracle."""
    rng = np.random.default_rng(4)
    nc = 128
    n = 4_194_304
    t = registered(nc)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, n)
    w = np.asfortranarray(rng.standard_normal((1, n)))
    T = rng.standard_normal((1, nc, nc, nc))
    ppmg.set_precision(mode)
    try:
        ext = nc + 1 + 4
        f = np.zeros((1, ext, ext, ext, 1), order="F")
        assert ppmg.ppm_interp_p2m(xp, n, w, 1, t.topo_id, t.mesh_id, 2, g, f) == 0, \
            ppmg.last_error()
        fref, lbo, _ = O.p2m(t, xp, w, 2, g)
        fu = unique_view(f, [-1, -1, -1], [nc] * 3, 3)
        fru = unique_view(fref, lbo, [nc] * 3, 3)
        tol = 1e-6 if mode == 1 else 1e-13
        assert max_rel(fu, fru) < tol
        R = np.asfortranarray((fu - T)[..., None])
        dw = np.zeros((1, n), order="F")
        dx = np.zeros((3, n), order="F")
        assert ppmg.ppm_interp_p2m_adjoint(xp, n, w, 1, t.topo_id, t.mesh_id, 2, R, dw, dx,
                                           field_lb=[1, 1, 1]) == 0, ppmg.last_error()
        # dL/dw = M2P of the residual, by the oracle (periodic ghost fill = ghost get)
        lb, ub = [1 - 2] * 3, [nc + 1 + 2] * 3
        Rg = periodic_fill(R[..., 0], lb, ub, 3)
        dwo = O.m2p(t, xp, Rg, lb, ub, 1, 2, g)
        assert max_rel(dw, dwo) < (1e-6 if mode == 1 else 1e-13)
        # dL/dx against FP64 central differences of the oracle's loss
        ru = (fru - T)[0]
        idx = _spread(rng, xp, nc, 200)
        fd = fd_gradients(t, xp, w, ru, idx, nc)
        got = dx[:, idx]
        err = np.abs(got - fd) / np.maximum(1.0, np.abs(fd))
        assert err.max() <= 1e-4, err.max()
        assert max_rel(got, fd) <= 1e-4
    finally:
        ppmg.set_precision(0)


@pytest.mark.parametrize("kernel,lda", [(2, 1), (2, 2), (1, 1)])
def test_autograd_gradcheck(kernel, lda):
    """torch.autograd.gradcheck of the wrapper (forward P2M, backward adjoint)
    in FP64 on an 8^3 mesh: dL/dx and dL/dw against numerical derivatives."""
    torch = pytest.importorskip("torch")
    from _autograd import P2M
    nc = 8
    t = registered(nc)
    rng = np.random.default_rng(11 + kernel + lda)
    n = 6
    x0 = random_particles(rng, 3, n, 0.1, 0.9)
    xp = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.tensor(rng.standard_normal((lda, n)), dtype=torch.float64, device="cuda",
                     requires_grad=True)
    ppmg.set_precision(0)

    def fn(x, u):
        return P2M.apply(x, u, t.topo_id, t.mesh_id, nc, kernel)

    assert torch.autograd.gradcheck(fn, (xp, w), eps=1e-6, atol=1e-6, rtol=1e-4)


def test_autograd_loss_gradient_matches_oracle():
    """Backward of L = 0.5 |P2M(x, w) - T|^2 through the wrapper equals the
    oracle's adjoint of the same residual (FP64, 16^3)."""
    torch = pytest.importorskip("torch")
    from _autograd import P2M
    nc = 16
    t = registered(nc)
    rng = np.random.default_rng(12)
    n = 3000
    x0 = random_particles(rng, 3, n)
    w0 = rng.standard_normal((1, n))
    T = torch.tensor(rng.standard_normal((1, nc, nc, nc)), device="cuda")
    xp = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.tensor(w0, dtype=torch.float64, device="cuda", requires_grad=True)
    ppmg.set_precision(0)
    f = P2M.apply(xp, w, t.topo_id, t.mesh_id, nc, 2)
    loss = 0.5 * ((f - T) ** 2).sum()
    loss.backward()
    r = np.asfortranarray((f - T).detach().cpu().numpy()[..., None])
    dwo, dxo = O.p2m_adjoint(t, np.asfortranarray(x0), np.asfortranarray(w0), r, [1, 1, 1],
                             [nc] * 3, 2)
    assert max_rel(w.grad.cpu().numpy(), dwo) < 1e-13
    assert max_rel(xp.grad.cpu().numpy(), dxo) < 1e-12
