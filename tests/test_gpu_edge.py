"""Edge cases of the GPU path against the oracle: dense cells (P2M layers cut
into several staging units), non-cubic meshes, ghost widths 0, uneven and
wider than the mesh, particle counts around the sort's sub-tile size, and
positions on cell faces and next to the upper box face."""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import box_bounds, max_rel, periodic_fill, random_particles, topo_for, unique_view
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_next_id = [3000]
TOL = {0: 1e-13, 1: 1e-6}


def registered(dim, nc, lo=None, hi=None):
    _next_id[0] += 1
    t = topo_for(dim, nc, lo, hi, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def p2m_both(t, xp, up, kernel, g):
    """(GPU field, oracle field, lb, oracle lb) of one P2M.  The oracle, like
    the reference, deposits into the ghost box and needs ghost layers at
    least as wide as the stencil's reach (2 for M'4, 1 for bsp2); it runs with
    max(g, reach) and only its real nodes are compared."""
    lb, ub = box_bounds(t, g)
    lda = up.shape[0]
    f = np.full((lda,) + tuple(ub[a] - lb[a] + 1 for a in range(t.dim)) + (1,), 7.0, order="F")
    info = ppmg.ppm_interp_p2m(np.asfortranarray(xp), xp.shape[1], np.asfortranarray(up), lda,
                               t.topo_id, t.mesh_id, kernel, g, f)
    assert info == 0, ppmg.last_error()
    reach = 2 if kernel == 2 else 1
    fo, lbo, _ = O.p2m(t, np.asfortranarray(xp), np.asfortranarray(up), kernel,
                       [max(int(x), reach) for x in g])
    return f, fo, lb, lbo


def real_nodes(f, lb, t):
    return f[(slice(None),) + tuple(slice(1 - lb[a], int(t.Nm[a]) + 1 - lb[a])
                                    for a in range(t.dim)) + (0,)]


def check_p2m(t, xp, up, kernel, g, mode):
    f, fo, lb, lbo = p2m_both(t, xp, up, kernel, g)
    nc = [int(t.Nm[a]) - 1 for a in range(t.dim)]
    assert max_rel(real_nodes(f, lb, t), real_nodes(fo, lbo, t)) < TOL[mode]
    # every ghost node holds the periodic image of its real node
    U = unique_view(f, lb, nc, t.dim)
    ub = [int(t.Nm[a]) + g[a] for a in range(t.dim)]
    assert np.array_equal(f, periodic_fill(U, lb, ub, t.dim))


@pytest.fixture(params=[0, 1], ids=["fp64", "mixed"])
def mode(request):
    ppmg.set_precision(request.param)
    yield request.param
    ppmg.set_precision(0)


def test_dense_cells_cut_into_units(mode):
    """Half of the particles in three cells (hundreds per cell): the layers
    holding them exceed the staging capacity and are processed in units."""
    rng = np.random.default_rng(301)
    nc = 16
    t = registered(3, nc)
    n = 24000
    xp = random_particles(rng, 3, n)
    h = 1.0 / nc
    for c, cell in enumerate([(3, 4, 5), (3, 5, 5), (10, 2, 14)]):
        sel = slice(c * n // 6, (c + 1) * n // 6)
        xp[:, sel] = (np.array(cell)[:, None] + rng.random((3, n // 6))) * h
    up = rng.standard_normal((3, n))
    check_p2m(t, xp, up, 2, [2, 2, 2], mode)
    # M2P of the same positions reuses this cell order
    f, _, lb, _ = p2m_both(t, xp, up, 2, [2, 2, 2])
    out = np.zeros((3, n), order="F")
    assert ppmg.ppm_interp_m2p(xp, n, out, 3, t.topo_id, t.mesh_id, 2, [2, 2, 2], f) == 0
    ref = O.m2p(t, xp, f, lb, [int(t.Nm[a]) + 2 for a in range(3)], 3, 2, [2, 2, 2])
    assert max_rel(out, ref) <= (0.0 if mode == 0 else 1e-6)


@pytest.mark.parametrize("nc,kernel", [((24, 16, 40), 2), ((9, 31, 6), 1)])
def test_non_cubic_mesh(mode, nc, kernel):
    rng = np.random.default_rng(sum(nc))
    t = registered(3, list(nc), [0.0, -1.0, 0.5], [1.5, 1.0, 2.0])
    n = 2 * int(np.prod(nc))
    xp = random_particles(rng, 3, n, t.min_phys[:3], t.max_phys[:3])
    up = rng.standard_normal((2, n))
    check_p2m(t, xp, up, kernel, [2, 2, 2], mode)


@pytest.mark.parametrize("nc,g", [(12, [0, 0, 0]), (12, [0, 1, 3]), (3, [4, 3, 7]), (2, [1, 5, 2])])
def test_ghost_widths(nc, g):
    """Ghost widths 0, uneven, and wider than the mesh (several periodic
    images of a node in the written box)."""
    rng = np.random.default_rng(400 + nc + sum(g))
    t = registered(3, nc)
    n = 3 * nc ** 3 + 5
    xp = random_particles(rng, 3, n)
    up = rng.standard_normal((1, n))
    check_p2m(t, xp, up, 2, g, 0)


@pytest.mark.parametrize("n,nc", [(1, 8), (2, 8), (4095, 8), (4096, 8), (4097, 8), (8191, 8),
                                  (8192, 8), (8193, 8), (16385, 8), (8191, 40), (8193, 40),
                                  (24577, 40)])
def test_ragged_particle_counts(n, nc):
    """Particle counts around the radix sort's 4096-item sub-tile, with one
    sort pass (8^3 cells) and two (40^3 cells)."""
    rng = np.random.default_rng(n + nc)
    t = registered(3, nc)
    xp = random_particles(rng, 3, n)
    up = rng.standard_normal((3, n))
    check_p2m(t, xp, up, 2, [2, 2, 2], 0)
    f, _, lb, _ = p2m_both(t, xp, up, 2, [2, 2, 2])
    out = np.zeros((3, n), order="F")
    assert ppmg.ppm_interp_m2p(xp, n, out, 3, t.topo_id, t.mesh_id, 2, [2, 2, 2], f) == 0
    ref = O.m2p(t, xp, f, lb, [int(t.Nm[a]) + 2 for a in range(3)], 3, 2, [2, 2, 2])
    assert np.array_equal(out, ref)


def test_positions_on_faces_and_near_the_upper_face():
    """Particles exactly on cell faces, at the lower box face and one ulp
    below the upper face (xi may round to Nc: the periodic image of node 1)."""
    t = registered(3, 10)
    below = np.nextafter(1.0, 0.0)
    pts = [[0.0, 0.0, 0.0], [0.1, 0.2, 0.3], [0.5, 0.5, 0.5], [below, below, below],
           [below, 0.0, 0.7], [0.9, below, 0.1], [0.3, 0.6, below]]
    xp = np.asfortranarray(np.array(pts).T)
    up = np.asfortranarray(np.random.default_rng(5).standard_normal((2, xp.shape[1])))
    check_p2m(t, xp, up, 2, [2, 2, 2], 0)
    check_p2m(t, xp, up, 1, [1, 1, 1], 0)


@pytest.mark.parametrize("mode", [0, 1])
def test_m2p_non_finite_positions(mode):
    """M2P with non-finite positions among ~9000 valid ones (more than two
    sort sub-tiles): the sort drops them into its invalid bucket, their rows
    of up are zero, info = -2 / errno 503, and every valid particle still
    gets the oracle's value (FP64 bit for bit, mixed to <= 1e-6)."""
    rng = np.random.default_rng(77 + mode)
    t = registered(3, 12)
    g = [2, 2, 2]
    n = 9001
    xp = random_particles(rng, 3, n)
    bad = np.array([0, 3, 4095, 4096, 8191, 9000])
    xp[0, bad[:2]] = np.nan
    xp[1, bad[2]] = np.inf
    xp[2, bad[3]] = -np.inf
    xp[:, bad[4]] = np.nan
    xp[2, bad[5]] = np.nan
    ok = np.ones(n, dtype=bool)
    ok[bad] = False
    src = random_particles(rng, 3, 3000)
    # the GPU's field: every periodic image holds its node's value, the
    # field the oracle's M2P reads as given and the GPU's reads with wrap
    f, _, lb, _ = p2m_both(t, src, rng.standard_normal((3, 3000)), 2, g)
    ub = [int(t.Nm[a]) + 2 for a in range(3)]
    out = np.full((3, n), 7.0, order="F")
    ppmg.set_precision(mode)
    try:
        info = ppmg.ppm_interp_m2p(np.asfortranarray(xp), n, out, 3, t.topo_id, t.mesh_id, 2, g, f)
        err = ppmg.last_error()  # before the next library call replaces it
    finally:
        ppmg.set_precision(0)
    assert info == -2
    assert err[1] == 503
    assert np.all(out[:, ~ok] == 0.0)
    ref = O.m2p(t, np.asfortranarray(xp[:, ok]), f, lb, ub, 3, 2, g)
    if mode == 0:
        assert np.array_equal(out[:, ok], ref)
    else:
        assert max_rel(out[:, ok], ref) < 1e-6
