"""GPU parity of remeshing, ghost get/put, cell ranking and the P2M adjoint."""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import (box_bounds, golden_cases, max_rel, periodic_fill, random_particles, topo_for,
                   unique_view)
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_next_id = [500]


def registered(dim, nc, lo=None, hi=None):
    _next_id[0] += 1
    t = topo_for(dim, nc, lo, hi, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


@pytest.mark.parametrize("dim,kernel,nc,box", [
    (3, 2, 16, None), (3, 1, 12, None), (2, 2, 24, None),
    (3, 2, 10, ([0.0, 0.0, 0.0], [1.3, 1.0, 0.7])),
])
def test_comp_weights_and_remesh_match_oracle(dim, kernel, nc, box):
    rng = np.random.default_rng(40 + nc)
    lo, hi = box if box else (None, None)
    t = registered(dim, nc, lo, hi)
    g = [2] * dim
    xp = random_particles(rng, dim, 2 * nc ** dim, t.min_phys[:dim], t.max_phys[:dim])
    up = np.asfortranarray(rng.standard_normal((3, xp.shape[1])))
    np_ = xp.shape[1]
    ks = 2 if kernel == 2 else 1
    wx = [np.zeros((2 * ks, 1, np_ + 2 * ks), order="F") for _ in range(3)]
    info = ppmg.ppm_rmsh_comp_weights(xp, np_, t.topo_id, t.mesh_id, kernel, wx[0], wx[1],
                                      wx[2] if dim == 3 else None)
    assert info == 0, ppmg.last_error()
    wo, lst, si = O.comp_weights(t, xp, kernel)
    for a in range(dim):
        # the oracle's list is ascending particle id, as is the user layout here
        assert np.array_equal(wx[a], wo[a])
    lb, ub = box_bounds(t, g)
    f = np.full((3,) + tuple(ub[a] - lb[a] + 1 for a in range(dim)) + (1,), 5.0, order="F")
    info = ppmg.ppm_rmsh_remesh(xp, np_, up, 3, t.topo_id, t.mesh_id, kernel, g, f)
    assert info == 0, ppmg.last_error()
    fo, lbo, ubo = O.remesh(t, xp, up, kernel, g, wo, lst, si)
    real = (slice(None),) + tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(dim)) + (0,)
    assert max_rel(f[real], fo[real]) < 1e-13


def test_remesh_without_weights_is_refused():
    t = registered(3, 8)
    xp = random_particles(np.random.default_rng(0), 3, 10)
    f = np.zeros((1, 13, 13, 13, 1), order="F")
    info = ppmg.ppm_rmsh_remesh(xp, 10, np.ones((1, 10), order="F"), 1, t.topo_id, t.mesh_id, 2,
                                [2, 2, 2], f)
    assert info == -2 and "weights" in ppmg.last_error()[2]


@pytest.mark.parametrize("dim,lda,weights", [(3, 3, False), (3, 1, False), (2, 2, True)])
def test_create_part_matches_oracle(dim, lda, weights):
    rng = np.random.default_rng(50 + lda)
    nc = 12
    t = registered(dim, nc)
    g = [1] * dim
    lb, ub = box_bounds(t, g)
    U = rng.standard_normal((lda,) + (nc,) * dim)
    U[np.abs(U) < 0.8] = 0.0
    F = periodic_fill(U, lb, ub, dim)
    cw = [0.5, 2.0][:lda] if weights else None
    cut = [0.3, 2.5]
    info, n, up, xp, _ = ppmg.ppm_rmsh_create_part(F, t.topo_id, t.mesh_id, cut, lda=lda,
                                                   resetpos=True, cutoff_weights=cw, ghostsize=g)
    assert info == 0, ppmg.last_error()
    no, upo, xpo, _ = O.create_part(t, F, lb, ub, cut, cutoff_weights=cw)
    assert n == no and n > 0
    assert np.array_equal(up.reshape(lda, -1), upo)
    assert np.array_equal(xp, xpo)


@pytest.mark.parametrize("dim,lda", [(3, 3), (2, 1)])
def test_ghost_get_put_match_oracle(dim, lda):
    rng = np.random.default_rng(60 + dim)
    nc = 10
    t = registered(dim, nc)
    g = [2] * dim
    lb, ub = box_bounds(t, g)
    # put: start from an arbitrary box (stale ghosts, as after a deposit)
    F = np.asfortranarray(rng.standard_normal((lda,) + tuple(ub[a] - lb[a] + 1 for a in range(dim)) + (1,)))
    Fo = F.copy(order="F")
    O.ghost_put(t, Fo, lb, ub, g)
    Fg = F.copy(order="F")
    assert ppmg.ppm_map_field_ghost(Fg, lda, t.topo_id, t.mesh_id, g,
                                    ppmg.params.ppm_param_map_ghost_put) == 0
    assert max_rel(Fg, Fo) < 1e-15
    # get on a consistent field reproduces the periodic images exactly
    U = rng.standard_normal((lda,) + (nc,) * dim)
    G = periodic_fill(U, lb, ub, dim)
    G2 = np.zeros_like(G, order="F")
    real = (slice(None),) + tuple(slice(1 - lb[a], 1 - lb[a] + nc) for a in range(dim)) + (0,)
    G2[real] = U  # only the real unique nodes are set; ghosts and node Nm are stale
    assert ppmg.ppm_map_field_ghost(G2, lda, t.topo_id, t.mesh_id, g,
                                    ppmg.params.ppm_param_map_ghost_get) == 0
    assert np.array_equal(G2, G)


@pytest.mark.parametrize("case", golden_cases("rank"), ids=lambda c: c["name"])
def test_util_rank_bit_exact(case):
    xp = np.asfortranarray(np.array(case["xp"]).T,
                           dtype=np.float32 if case.get("prec") == "s" else np.float64)
    info, lpdx, lhbx = ppmg.ppm_util_rank(xp, xp.shape[1], case["xmin"], case["xmax"],
                                          case["Nm"], case["Ngl"])
    assert info == 0, ppmg.last_error()
    assert lpdx.tolist() == case["lpdx"]
    assert lhbx.tolist() == case["lhbx"]


def test_neighlist_clist_large_bit_exact():
    rng = np.random.default_rng(70)
    t = topo_for(3, 64)
    xp = random_particles(rng, 3, 300000)
    xp[:, :1000] = 0.5  # a crowded cell (block-cooperative sort path)
    info, lpdx, lhbx, Nm = ppmg.ppm_neighlist_clist(xp, xp.shape[1], 1.0 / 40, False, t)
    assert info == 0
    ref_l, ref_h, ic = O.rank(xp, t.min_sub[0], t.max_sub[0], [40, 40, 40], [1] * 6)
    assert np.array_equal(lpdx, ref_l) and np.array_equal(lhbx, ref_h)


@pytest.mark.parametrize("kernel", [2, 1])
def test_adjoint_matches_oracle_and_finite_differences(kernel):
    rng = np.random.default_rng(80 + kernel)
    nc = 16
    t = registered(3, nc)
    lb = [1, 1, 1]
    np_ = 3000
    xp = random_particles(rng, 3, np_, 0.05, 0.95)
    up = np.asfortranarray(rng.standard_normal((2, np_)))
    R = np.asfortranarray(rng.standard_normal((2, nc, nc, nc, 1)))
    dw = np.zeros((2, np_), order="F")
    dx = np.zeros((3, np_), order="F")
    info = ppmg.ppm_interp_p2m_adjoint(xp, np_, up, 2, t.topo_id, t.mesh_id, kernel, R, dw, dx,
                                       field_lb=lb)
    assert info == 0, ppmg.last_error()
    dwo, dxo = O.p2m_adjoint(t, xp, up, R, lb, [nc] * 3, kernel)
    assert max_rel(dw, dwo) < 1e-13
    assert max_rel(dx, dxo) < 1e-12
    # central finite differences of L = <P2M(x, w), R> in FP64 (step 1e-6 h)
    h = 1.0 / nc
    g = [2, 2, 2]
    Ru = R[..., 0]

    def loss(xq):
        f, lbq, _ = O.p2m(t, xq, up[:, :5], kernel, g)
        return float((unique_view(f, lbq, [nc] * 3, 3) * Ru).sum())

    for p in range(5):
        for a in range(3):
            e = 1e-6 * h
            xa = xp[:, :5].copy(order="F")
            xb = xp[:, :5].copy(order="F")
            xa[a, p] += e
            xb[a, p] -= e
            fd = (loss(xa) - loss(xb)) / (2 * e)
            assert abs(fd - dx[a, p]) <= 1e-4 * max(1.0, abs(fd))


def test_adjoint_reuses_p2m_order_only_for_identical_positions():
    """The adjoint after a P2M of the same positions reuses its cell order; the
    result equals the adjoint on a fresh sort (and the oracle) bit for bit."""
    rng = np.random.default_rng(85)
    nc = 16
    t = registered(3, nc)
    np_ = 4000
    xp = random_particles(rng, 3, np_)
    up = np.asfortranarray(rng.standard_normal((3, np_)))
    R = np.asfortranarray(rng.standard_normal((3, nc, nc, nc, 1)))
    g = [2, 2, 2]
    lb, ub = box_bounds(t, g)
    f = np.zeros((3,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,), order="F")
    for mode in (0, 1):
        ppmg.set_precision(mode)
        res = []
        for warm in (False, True):
            if warm:
                assert ppmg.ppm_interp_p2m(xp, np_, up, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
            else:  # a different position set first: no order to reuse
                xq = random_particles(rng, 3, np_)
                assert ppmg.ppm_interp_p2m(xq, np_, up, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
            dw = np.zeros((3, np_), order="F")
            dx = np.zeros((3, np_), order="F")
            assert ppmg.ppm_interp_p2m_adjoint(xp, np_, up, 3, t.topo_id, t.mesh_id, 2, R, dw,
                                               dx, field_lb=[1, 1, 1]) == 0
            res.append((dw, dx))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
        if mode == 0:
            dwo, dxo = O.p2m_adjoint(t, xp, up, R, [1, 1, 1], [nc] * 3, 2)
            assert max_rel(res[1][0], dwo) < 1e-13 and max_rel(res[1][1], dxo) < 1e-12
    ppmg.set_precision(0)


@pytest.mark.parametrize("dim,kernel", [(3, 2), (3, 1), (2, 2)])
def test_remeshing_device_twins_match_host_entry_points(dim, kernel):
    """comp_weights, remesh and create_part on device arrays (the `_dev`
    twins, on the torch stream) equal the host-pointer entry points bit for bit."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(90 + dim + kernel)
    nc = 12
    t = registered(dim, nc)
    g = [2] * dim
    np_ = 3 * nc ** dim
    xp = random_particles(rng, dim, np_)
    up = np.asfortranarray(rng.standard_normal((3, np_)))
    ks = 2 if kernel == 2 else 1
    lb, ub = box_bounds(t, g)
    shape = (3,) + tuple(ub[a] - lb[a] + 1 for a in range(dim)) + (1,)

    def cm(a):
        d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
        return d.permute(*reversed(range(d.dim())))

    def host(a):
        return a.permute(*reversed(range(a.dim()))).contiguous().cpu().numpy().T

    wh = [np.zeros((2 * ks, 1, np_ + 2 * ks), order="F") for _ in range(dim)]
    assert ppmg.ppm_rmsh_comp_weights(xp, np_, t.topo_id, t.mesh_id, kernel, *wh) == 0
    fh = np.zeros(shape, order="F")
    assert ppmg.ppm_rmsh_remesh(xp, np_, up, 3, t.topo_id, t.mesh_id, kernel, g, fh) == 0
    cut = [0.05, 1e300]
    ih, nh, uh, xh, _ = ppmg.ppm_rmsh_create_part(fh, t.topo_id, t.mesh_id, cut, lda=3,
                                                  resetpos=True, ghostsize=g)
    assert ih == 0 and nh > 0
    dxp, dup = cm(xp), cm(up)
    wd = [cm(np.zeros((2 * ks, 1, np_ + 2 * ks))) for _ in range(dim)]
    assert ppmg.ppm_rmsh_comp_weights(dxp, np_, t.topo_id, t.mesh_id, kernel, *wd) == 0
    fd = cm(np.full(shape, 3.0))
    assert ppmg.ppm_rmsh_remesh(dxp, np_, dup, 3, t.topo_id, t.mesh_id, kernel, g, fd) == 0
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
    for a in range(dim):
        assert np.array_equal(host(wd[a]), wh[a])
    assert np.array_equal(host(fd), fh)
    idv, nd, ud, xd, _ = ppmg.ppm_rmsh_create_part(fd, t.topo_id, t.mesh_id, cut, lda=3,
                                                   resetpos=True, ghostsize=g)
    assert idv == 0 and nd == nh
    torch.cuda.synchronize()
    assert np.array_equal(host(ud), uh) and np.array_equal(host(xd), xh)


@pytest.mark.parametrize("dim,kernel", [(3, 2), (3, 1), (2, 2)])
def test_single_precision_remeshing_matches_oracle(dim, kernel):
    """comp_weights_s, remesh_sv and create_part_s against the oracle's single
    routines: weights bit for bit, the field to FP32 summation order (1e-5
    normwise), and create_part's particles from a field both sides share."""
    rng = np.random.default_rng(110 + dim + kernel)
    nc = 12
    t = registered(dim, nc)
    g = [2] * dim
    np_ = 2 * nc ** dim
    xp = random_particles(rng, dim, np_).astype(np.float32, order="F")
    up = rng.standard_normal((3, np_)).astype(np.float32, order="F")
    ks = 2 if kernel == 2 else 1
    wx = [np.zeros((2 * ks, 1, np_ + 2 * ks), dtype=np.float32, order="F") for _ in range(dim)]
    assert ppmg.ppm_rmsh_comp_weights(xp, np_, t.topo_id, t.mesh_id, kernel, *wx) == 0
    wo, lst, si = O.comp_weights(t, xp, kernel)
    for a in range(dim):
        assert np.array_equal(wx[a], wo[a])
    lb, ub = box_bounds(t, g)
    f = np.full((3,) + tuple(ub[a] - lb[a] + 1 for a in range(dim)) + (1,), 5.0,
                dtype=np.float32, order="F")
    assert ppmg.ppm_rmsh_remesh(xp, np_, up, 3, t.topo_id, t.mesh_id, kernel, g, f) == 0, \
        ppmg.last_error()
    fo, _, _ = O.remesh(t, xp, up, kernel, g, wo, lst, si)
    real = (slice(None),) + tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(dim)) + (0,)
    assert max_rel(f[real].astype(np.float64), fo[real].astype(np.float64)) < 1e-5
    # create_part on the GPU's field: same count, order, strengths and positions
    cut = [0.2, 1e30]
    info, n, upn, xpn, _ = ppmg.ppm_rmsh_create_part(f, t.topo_id, t.mesh_id, cut, lda=3,
                                                     resetpos=True, ghostsize=g)
    assert info == 0, ppmg.last_error()
    no, upo, xpo, _ = O.create_part(t, f, lb, ub, cut)
    assert n == no and n > 0 and upn.dtype == np.float32
    assert np.array_equal(upn, upo) and np.array_equal(xpn, xpo)
    # single weights do not feed a double remesh
    fd = np.zeros(f.shape, order="F")
    info = ppmg.ppm_rmsh_remesh(xp.astype(np.float64), np_, up.astype(np.float64), 3, t.topo_id,
                                t.mesh_id, kernel, g, fd)
    assert info == -2 and "weights" in ppmg.last_error()[2]


def test_single_precision_remeshing_device_twins():
    """float32 torch arrays take the single `_dev` twins and equal the host calls."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(120)
    nc = 10
    t = registered(3, nc)
    g = [2, 2, 2]
    np_ = 3 * nc ** 3
    xp = random_particles(rng, 3, np_).astype(np.float32, order="F")
    up = rng.standard_normal((2, np_)).astype(np.float32, order="F")
    lb, ub = box_bounds(t, g)
    shape = (2,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)

    def cm(a):
        d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
        return d.permute(*reversed(range(d.dim())))

    def host(a):
        return a.permute(*reversed(range(a.dim()))).contiguous().cpu().numpy().T

    assert ppmg.ppm_rmsh_comp_weights(xp, np_, t.topo_id, t.mesh_id, 2) == 0
    fh = np.zeros(shape, dtype=np.float32, order="F")
    assert ppmg.ppm_rmsh_remesh(xp, np_, up, 2, t.topo_id, t.mesh_id, 2, g, fh) == 0
    ih, nh, uh, xh, _ = ppmg.ppm_rmsh_create_part(fh, t.topo_id, t.mesh_id, [0.1, 1e30], lda=2,
                                                  resetpos=True, ghostsize=g)
    assert ih == 0 and nh > 0
    dxp, dup = cm(xp), cm(up)
    assert ppmg.ppm_rmsh_comp_weights(dxp, np_, t.topo_id, t.mesh_id, 2) == 0
    fd = cm(np.full(shape, 3.0, dtype=np.float32))
    assert ppmg.ppm_rmsh_remesh(dxp, np_, dup, 2, t.topo_id, t.mesh_id, 2, g, fd) == 0
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
    assert fd.dtype == torch.float32 and np.array_equal(host(fd), fh)
    idv, nd, ud, xd, _ = ppmg.ppm_rmsh_create_part(fd, t.topo_id, t.mesh_id, [0.1, 1e30], lda=2,
                                                   resetpos=True, ghostsize=g)
    assert idv == 0 and nd == nh
    torch.cuda.synchronize()
    assert ud.dtype == torch.float32
    assert np.array_equal(host(ud), uh) and np.array_equal(host(xd), xh)


@pytest.mark.parametrize("dim", [3, 2])
def test_util_rank_single_large_bit_exact(dim):
    """ppm_util_rank{2,3}d_s on 200k FP32 positions over a box whose FP32 cell
    spacing rounds (crowded cell included) equals the oracle's single routine."""
    rng = np.random.default_rng(75 + dim)
    xmin = np.array([0.1, -0.3, 0.25][:dim], dtype=np.float32)
    xmax = np.array([0.7, 0.9, 1.0][:dim], dtype=np.float32)
    Nm = [37, 41, 29][:dim]
    Ngl = [1] * (2 * dim)
    xp = (xmin[:, None] + rng.random((dim, 200000)) * (xmax - xmin)[:, None]).astype(np.float32)
    xp[:, :2000] = ((xmin + xmax) / 2)[:, None]
    xp = np.asfortranarray(xp)
    info, lpdx, lhbx = ppmg.ppm_util_rank(xp, xp.shape[1], xmin, xmax, Nm, Ngl)
    assert info == 0, ppmg.last_error()
    ref_l, ref_h, _ = O.rank(xp, xmin, xmax, Nm, Ngl)
    assert np.array_equal(lpdx, ref_l) and np.array_equal(lhbx, ref_h)


@pytest.mark.parametrize("maptype", ["put", "get"])
def test_ghost_single_device_twin_matches_host(maptype):
    """ppmg_map_field_ghost_s_dev on a float32 torch field equals the host
    ppmg_map_field_ghost_s bit for bit (and the oracle within FP32 rounding)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(130)
    nc = 9
    t = registered(3, nc)
    g = [2, 1, 3]
    lb, ub = box_bounds(t, g)
    F = rng.standard_normal((2,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,))
    F = np.asfortranarray(F.astype(np.float32))
    mt = getattr(ppmg.params, f"ppm_param_map_ghost_{maptype}")
    Fh = F.copy(order="F")
    assert ppmg.ppm_map_field_ghost(Fh, 2, t.topo_id, t.mesh_id, g, mt) == 0, ppmg.last_error()
    d = torch.from_numpy(np.ascontiguousarray(F.T)).cuda()
    Fd = d.permute(*reversed(range(d.dim())))
    assert ppmg.ppm_map_field_ghost(Fd, 2, t.topo_id, t.mesh_id, g, mt) == 0, ppmg.last_error()
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
    got = Fd.permute(*reversed(range(Fd.dim()))).contiguous().cpu().numpy().T
    assert got.dtype == np.float32 and np.array_equal(got, Fh)
    if maptype == "put":
        Fo = F.astype(np.float64, order="F")
        O.ghost_put(t, Fo, lb, ub, g)
        assert max_rel(Fh.astype(np.float64), Fo) < 1e-6


@pytest.mark.parametrize("dim,dtype", [(3, np.float64), (2, np.float64), (3, np.float32),
                                       (2, np.float32)])
def test_util_rank_device_twins_match_host(dim, dtype):
    """ppm_util_rank on torch CUDA positions (the `_dev` twins, lists left on
    the device) equals the host entry points bit for bit."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(140 + dim)
    xmin = np.array([0.1, -0.3, 0.25][:dim])
    xmax = np.array([0.7, 0.9, 1.0][:dim])
    Nm = [23, 17, 11][:dim]
    Ngl = [1] * (2 * dim)
    xp = (xmin[:, None] - 0.05 + rng.random((dim, 50000)) * (xmax - xmin + 0.1)[:, None])
    xp = np.asfortranarray(xp.astype(dtype))
    ih, lh, hh = ppmg.ppm_util_rank(xp, xp.shape[1], xmin, xmax, Nm, Ngl)
    xd = torch.from_numpy(np.ascontiguousarray(xp.T)).cuda().t()
    idv, ld, hd = ppmg.ppm_util_rank(xd, xp.shape[1], xmin, xmax, Nm, Ngl)
    assert ih == 0 and idv == 0, ppmg.last_error()
    assert ld.is_cuda and hd.is_cuda
    assert np.array_equal(ld.cpu().numpy(), lh) and np.array_equal(hd.cpu().numpy(), hh)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_fdsolver_poisson_matches_oracle(dtype, tol):
    """ppm_fdsolver_poisson on a non-cubic periodic mesh against the oracle's
    spectral restatement: phi at the real nodes and every periodic image of
    the ghost layers; the device twin equals the host entry point."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(150)
    nc = (24, 16, 20)
    lo, hi = [0.0, -1.0, 0.5], [1.5, 0.0, 2.5]
    t = registered(3, list(nc), lo, hi)
    g = [2, 1, 2]
    lb, ub = box_bounds(t, g)
    U = rng.standard_normal((3,) + nc)
    F = periodic_fill(U, lb, ub, 3).astype(dtype)
    Fh = F.copy(order="F")
    assert ppmg.ppm_fdsolver_poisson(Fh, 3, t.topo_id, t.mesh_id, g) == 0, ppmg.last_error()
    phi = O.poisson(U.astype(dtype).astype(np.float64),
                    [hi[a] - lo[a] for a in range(3)])
    ref = periodic_fill(phi, lb, ub, 3)
    assert max_rel(Fh.astype(np.float64), ref) < tol
    d = torch.from_numpy(np.ascontiguousarray(F.T)).cuda()
    Fd = d.permute(*reversed(range(d.dim())))
    assert ppmg.ppm_fdsolver_poisson(Fd, 3, t.topo_id, t.mesh_id, g) == 0, ppmg.last_error()
    torch.cuda.synchronize()
    got = Fd.permute(*reversed(range(Fd.dim()))).contiguous().cpu().numpy().T
    assert np.array_equal(got, Fh)


def test_fdsolver_poisson_refuses_a_slab():
    import copy
    t = topo_for(3, 12, decomp=(1, 1, 2), topo_id=7950)
    assert ppmg.register(copy.deepcopy(t), isub=0) == 0
    F = np.zeros((1, 13, 13, 7, 1), order="F")
    assert ppmg.ppm_fdsolver_poisson(F, 1, 7950, 1, [0, 0, 0]) == -2
    ppmg.unregister(t)
