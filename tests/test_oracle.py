"""The CPU restatement (oracle) pinned against the exact-rational golden vectors
and the analytic identities of the kernels (no GPU)."""
import numpy as np
import pytest

from _util import (box_bounds, golden_cases, max_rel, periodic_fill, random_particles, topo_for,
                   unique_view)
from oracle import oracle as O


@pytest.mark.parametrize("case", golden_cases("p2m"), ids=lambda c: c["name"])
def test_oracle_p2m_matches_golden(case):
    dim, nc = case["dim"], case["nc"]
    t = topo_for(dim, nc, case["lo"], case["hi"])
    xp = np.asfortranarray(np.array(case["xp"]).T)
    up = np.asfortranarray(np.array(case["up"]).T)
    g = [2] * dim
    f, lb, ub = O.p2m(t, xp, up, case["kernel"], g)
    got = unique_view(f, lb, nc, dim)
    ref = np.array(case["field"]).reshape((case["lda"],) + tuple(nc), order="F")
    assert max_rel(got, ref) < 1e-14


@pytest.mark.parametrize("case", golden_cases("m2p"), ids=lambda c: c["name"])
def test_oracle_m2p_matches_golden(case):
    dim, nc, lda = case["dim"], case["nc"], case["lda"]
    t = topo_for(dim, nc, case["lo"], case["hi"])
    xp = np.asfortranarray(np.array(case["xp"]).T)
    U = np.array(case["F"]).reshape((lda,) + tuple(nc), order="F")
    g = [2] * dim
    lb, ub = box_bounds(t, g)
    F = periodic_fill(U, lb, ub, dim)
    up = O.m2p(t, xp, F, lb, ub, lda, case["kernel"], g)
    ref = np.array(case["up"]).T
    assert max_rel(up, ref) < 1e-14


@pytest.mark.parametrize("case", golden_cases("rank"), ids=lambda c: c["name"])
def test_oracle_rank_matches_golden(case):
    """Cases with prec "s" hold FP32 positions: the single routine runs."""
    xp = np.asfortranarray(np.array(case["xp"]).T,
                           dtype=np.float32 if case.get("prec") == "s" else np.float64)
    lpdx, lhbx, ic = O.rank(xp, case["xmin"], case["xmax"], case["Nm"], case["Ngl"])
    assert ic == len(case["lpdx"])
    assert lpdx.tolist() == case["lpdx"]
    assert lhbx.tolist() == case["lhbx"]


def test_partition_of_unity_and_moments():
    """sum_n W = 1 and M2P of a mesh-sampled polynomial of degree <= 2 is exact
    for M'4 (degree <= 1 for bsp2) on a periodic mesh away from the wrap."""
    rng = np.random.default_rng(3)
    nc = 16
    t = topo_for(3, nc)
    g = [2, 2, 2]
    lb, ub = box_bounds(t, g)
    xp = random_particles(rng, 3, 200, 0.3, 0.7)
    h = 1.0 / nc
    for kernel, deg in ((2, 2), (1, 1)):
        X = [np.arange(nc) * h for _ in range(3)]
        Xg = np.meshgrid(*X, indexing="ij")
        polys = [np.ones_like(Xg[0]), Xg[0], Xg[1] ** deg, Xg[0] * Xg[2]]
        U = np.stack(polys[:3] if deg == 1 else polys)
        F = periodic_fill(U, lb, ub, 3)
        up = O.m2p(t, xp, F, lb, ub, U.shape[0], kernel, g)
        exact = [np.ones(xp.shape[1]), xp[0], xp[1] ** deg, xp[0] * xp[2]][: U.shape[0]]
        for c in range(U.shape[0]):
            np.testing.assert_allclose(up[c], exact[c], rtol=0, atol=1e-13)


def test_transpose_identity():
    """<P2M(w), F> = <w, M2P(F)> on a periodic mesh (power-of-two spacing)."""
    rng = np.random.default_rng(4)
    for dim, kernel in ((3, 2), (3, 1), (2, 2)):
        nc = 12
        t = topo_for(dim, nc)
        g = [2] * dim
        xp = random_particles(rng, dim, 300)
        up = rng.standard_normal((2, 300))
        f, lb, ub = O.p2m(t, xp, up, kernel, g)
        U = rng.standard_normal((2,) + (nc,) * dim)
        F = periodic_fill(U, lb, ub, dim)
        u2 = O.m2p(t, xp, F, lb, ub, 2, kernel, g)
        lhs = (unique_view(f, lb, [nc] * dim, dim) * U).sum()
        rhs = (up * u2).sum()
        assert abs(lhs - rhs) < 1e-12 * max(1.0, abs(lhs))


def test_ghost_semantics_single_sub():
    """After the put: node Nm equals node 1 on real nodes; the get fills every
    ghost with the periodic image and leaves a consistent field unchanged."""
    rng = np.random.default_rng(5)
    nc = 8
    t = topo_for(3, nc)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, 100)
    up = rng.standard_normal((1, 100))
    f, lb, ub = O.p2m(t, xp, up, 2, g)
    i1, iN = 1 - lb[0], nc + 1 - lb[0]
    real = (slice(1 - lb[1], nc + 2 - lb[1]), slice(1 - lb[2], nc + 2 - lb[2]))
    # equal up to the order in which the images are added (block order)
    np.testing.assert_allclose(f[(0, i1) + real], f[(0, iN) + real], rtol=0, atol=1e-15)
    f2 = f.copy(order="F")
    O.ghost_get(t, f2, lb, ub, g)
    U = unique_view(f, lb, [nc] * 3, 3)
    np.testing.assert_allclose(f2, periodic_fill(U, lb, ub, 3), rtol=0, atol=1e-15)


def test_multisub_equals_single_sub():
    """A 2x2x1 cartesian split (ghost put across subs) gives the single-sub field."""
    rng = np.random.default_rng(6)
    t1 = topo_for(3, 8)
    t2 = topo_for(3, 8, decomp=(2, 2, 1))
    xp = random_particles(rng, 3, 400)
    up = rng.standard_normal((3, 400))
    f1, lb, _ = O.p2m(t1, xp, up, 2, [2, 2, 2])
    f2, lb2, _ = O.p2m(t2, xp, up, 2, [2, 2, 2])
    for s in range(t2.nsubs):
        i0 = t2.istart[s] - 1
        nn = t2.nnodes[s]
        a = f2[:, 1 - lb2[0]:1 - lb2[0] + nn[0], 1 - lb2[1]:1 - lb2[1] + nn[1],
               1 - lb2[2]:1 - lb2[2] + nn[2], s]
        b = f1[:, 1 - lb[0] + i0[0]:1 - lb[0] + i0[0] + nn[0],
               1 - lb[1] + i0[1]:1 - lb[1] + i0[1] + nn[1],
               1 - lb[2] + i0[2]:1 - lb[2] + i0[2] + nn[2], 0]
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)


def test_roundtrip_owned_matches_serial():
    """The CPU baseline (one thread per sub) equals the serial reference loops."""
    rng = np.random.default_rng(7)
    t1 = topo_for(3, 8)
    t2 = topo_for(3, 8, decomp=(2, 1, 2))
    xp = random_particles(rng, 3, 300)
    up = np.asfortranarray(rng.standard_normal((3, 300)))
    lst, si = O.assign(t2, xp)
    owner = np.repeat(np.arange(t2.nsubs), si)
    own = np.empty(300, dtype=np.int32)
    own[lst] = owner
    f, lb, ub, out = O.roundtrip_owned(t2, xp, own, up, 2, [2, 2, 2], nthreads=2)
    f1, lb1, ub1 = O.p2m(t1, xp, up, 2, [2, 2, 2])
    O.ghost_get(t1, f1, lb1, ub1, [2, 2, 2])
    ref = O.m2p(t1, xp, f1, lb1, ub1, 3, 2, [2, 2, 2])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)


def test_unassigned_particle_is_fatal():
    t = topo_for(3, 8)
    xp = np.asfortranarray([[0.5, 1.0], [0.5, 0.5], [0.5, 0.5]])  # x = max_phys: unassigned
    with pytest.raises(O.OracleError) as ei:
        O.p2m(t, xp, np.ones((1, 2)), 2, [2, 2, 2])
    assert ei.value.info == -1 and ei.value.errno == 405


def test_remesh_equals_p2m_on_power_of_two_mesh():
    """comp_weights + remesh deposits the same field as P2M (exact spacing)."""
    rng = np.random.default_rng(8)
    for dim in (2, 3):
        t = topo_for(dim, 8)
        g = [2] * dim
        xp = random_particles(rng, dim, 150)
        up = rng.standard_normal((2, 150))
        wx, lst, si = O.comp_weights(t, xp, 2)
        fr, lb, ub = O.remesh(t, xp, up, 2, g, wx, lst, si)
        fp, _, _ = O.p2m(t, xp, up, 2, g)
        np.testing.assert_allclose(unique_view(fr, lb, [8] * dim, dim),
                                   unique_view(fp, lb, [8] * dim, dim), rtol=0, atol=1e-14)


def test_create_part_order_and_band():
    t = topo_for(3, 4)
    g = [1, 1, 1]
    lb, ub = box_bounds(t, g)
    U = np.zeros((2, 4, 4, 4))
    U[0, 1, 2, 3] = 3.0
    U[1, 3, 0, 0] = 0.5
    U[0, 0, 0, 0] = 1e-9
    F = periodic_fill(U, lb, ub, 3)
    n, up, xp, _ = O.create_part(t, F, lb, ub, [1e-8, 10.0])
    assert n == 2
    # (k, j, i) order with i fastest: (3,0,0) comes before (1,2,3)
    np.testing.assert_array_equal(up.T, [[0.0, 0.5], [3.0, 0.0]])
    np.testing.assert_allclose(xp.T, [[0.75, 0.0, 0.0], [0.25, 0.5, 0.75]])


def test_single_precision_remeshing_tracks_double():
    """The single variants (comp_weights_s, remesh_sv, create_part_s) compute in
    FP32 and agree with the double routines to FP32 rounding on the same inputs."""
    rng = np.random.default_rng(9)
    for dim, kernel in ((3, 2), (2, 1)):
        t = topo_for(dim, 10)
        g = [2] * dim
        x32 = random_particles(rng, dim, 400).astype(np.float32, order="F")
        u32 = rng.standard_normal((2, 400)).astype(np.float32, order="F")
        w32, lst, si = O.comp_weights(t, x32, kernel)
        w64, lst64, _ = O.comp_weights(t, x32.astype(np.float64), kernel)
        assert w32[0].dtype == np.float32 and np.array_equal(lst, lst64)
        for a in range(dim):
            assert np.abs(w32[a] - w64[a]).max() < 2e-6
        f32, lb, _ = O.remesh(t, x32, u32, kernel, g, w32, lst, si)
        f64, _, _ = O.remesh(t, x32.astype(np.float64), u32.astype(np.float64), kernel, g, w64,
                             lst, si)
        assert f32.dtype == np.float32
        assert max_rel(f32.astype(np.float64), f64) < 1e-5
        n32, up32, xp32, _ = O.create_part(t, f32, lb, [lb[a] + f32.shape[1 + a] - 1
                                                       for a in range(dim)], [0.5, 1e30])
        n64, up64, xp64, _ = O.create_part(t, f32.astype(np.float64), lb,
                                           [lb[a] + f32.shape[1 + a] - 1 for a in range(dim)],
                                           [0.5, 1e30])
        assert n32 == n64 and up32.dtype == np.float32
        assert np.array_equal(up32.astype(np.float64), up64)
        assert np.abs(xp32 - xp64).max() < 1e-6


def test_oracle_poisson_recovers_an_analytic_solution():
    """The Poisson restatement inverts the periodic Laplacian: for
    phi = sin(2 pi x / Lx) cos(4 pi y / Ly) sin(2 pi z / Lz) on a non-cubic
    box, omega = lap(phi) = -(2pi)^2 (1/Lx^2 + 4/Ly^2 + 1/Lz^2) phi gives phi
    back (a band-limited field: exact up to rounding)."""
    L = (1.5, 1.0, 2.0)
    n = (24, 16, 20)
    x, y, z = np.meshgrid(*[np.arange(n[a]) * L[a] / n[a] for a in range(3)], indexing="ij")
    phi = np.sin(2 * np.pi * x / L[0]) * np.cos(4 * np.pi * y / L[1]) * np.sin(2 * np.pi * z / L[2])
    lam = -(2 * np.pi) ** 2 * (1 / L[0] ** 2 + 4 / L[1] ** 2 + 1 / L[2] ** 2)
    got = O.poisson((lam * phi)[None], L)[0]
    assert np.abs(got - phi).max() < 1e-12
    # the mean of omega (the zero mode) does not enter phi
    got2 = O.poisson((lam * phi + 3.0)[None], L)[0]
    assert np.abs(got2 - phi).max() < 1e-12


def test_p2m_conserves_moments_0_1_2():
    """The oracle's P2M conserves total strength for every particle and, for
    particles whose support does not wrap, moments 1 and 2 per axis (M'4
    reproduces polynomials of degree <= 2); bsp2 conserves moments 0 and 1."""
    from _util import interior_mask, moment_errors, unique_view
    rng = np.random.default_rng(31)
    nc = 24
    h = 1.0 / nc
    t = topo_for(3, nc)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, 4000)
    up = rng.standard_normal((3, 4000))
    inner = interior_mask(xp, nc)
    assert 0 < inner.sum() < xp.shape[1]
    for kernel, deg in ((2, 2), (1, 1)):
        f, lb, _ = O.p2m(t, xp, up, kernel, g)
        e0 = moment_errors(unique_view(f, lb, [nc] * 3, 3), h, xp, up)[0]
        assert e0 < 1e-14
        ui = np.where(inner[None, :], up, 0.0)
        f, lb, _ = O.p2m(t, xp, ui, kernel, g)
        errs = moment_errors(unique_view(f, lb, [nc] * 3, 3), h, xp, ui)
        assert max(errs[: deg + 1]) < 1e-13, errs
        if deg < 2:  # CIC does not reproduce x^2 (it adds f(1-f) h^2 per particle)
            assert errs[2] > 1e-6
