"""Particles that arrive in cell order (as ppm_rmsh_create_part emits them)
take the sort's fast path: the first pass finds the keys in order and the
radix passes are skipped.  Results must equal the oracle as for any order;
one pair out of order, or an invalid particle before valid ones, must take
the full sort and still be right."""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import box_bounds, jittered_particles, max_rel, topo_for, unique_view
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_next_id = [9500]


def registered(nc):
    _next_id[0] += 1
    t = topo_for(3, nc, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def round_trip(t, xp, up, g):
    lb, ub = box_bounds(t, g)
    lda = up.shape[0]
    f = np.zeros((lda,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,), order="F")
    i1 = ppmg.ppm_interp_p2m(xp, xp.shape[1], up, lda, t.topo_id, t.mesh_id, 2, g, f)
    out = np.zeros((lda, xp.shape[1]), order="F")
    i2 = ppmg.ppm_interp_m2p(xp, xp.shape[1], out, lda, t.topo_id, t.mesh_id, 2, g, f)
    return i1, i2, f, out, lb


@pytest.mark.parametrize("case", ["sorted", "swapped", "dense_sorted"])
@pytest.mark.parametrize("mode", [0, 1])
def test_cell_ordered_input_matches_oracle(case, mode):
    rng = np.random.default_rng(61)
    nc = 32
    t = registered(nc)
    g = [2, 2, 2]
    xp = jittered_particles(rng, 3, nc)  # cell order, x fastest
    if case == "dense_sorted":  # several particles per cell, still in cell order
        xp = np.asfortranarray(np.repeat(xp, 3, axis=1) +
                               rng.uniform(-0.1, 0.1, (3, 3 * xp.shape[1])) / nc)
        cells = np.floor(xp * nc).astype(int)
        key = cells[0] + nc * (cells[1] + nc * cells[2])
        xp = np.asfortranarray(xp[:, np.argsort(key, kind="stable")] % 1.0)
    if case == "swapped":  # one pair out of order: the full sort
        xp[:, [100, 2000]] = xp[:, [2000, 100]]
    n = xp.shape[1]
    up = np.asfortranarray(rng.standard_normal((3, n)))
    ppmg.set_precision(mode)
    try:
        i1, i2, f, out, lb = round_trip(t, xp, up, g)
        assert i1 == 0 and i2 == 0, ppmg.last_error()
        ref, lbo, ubo = O.p2m(t, xp, up, 2, g)
        tol = 1e-13 if mode == 0 else 1e-6
        assert max_rel(unique_view(f, lb, [nc] * 3, 3), unique_view(ref, lbo, [nc] * 3, 3)) < tol
        O.ghost_get(t, ref, lbo, ubo, g)
        assert max_rel(out, O.m2p(t, xp, ref, lbo, ubo, 3, 2, g)) < tol
        # deterministic: a second call gives the same bits
        _, _, f2, out2, _ = round_trip(t, xp, up, g)
        assert np.array_equal(f, f2) and np.array_equal(out, out2)
    finally:
        ppmg.set_precision(0)


def test_invalid_particles_at_the_end_and_in_the_middle():
    """Particles outside the subdomain (P2M: info -1, errno 405): the valid
    ones are still deposited, whether the invalid ones come last (keys still
    in order) or among the valid ones (full sort)."""
    rng = np.random.default_rng(62)
    nc = 16
    t = registered(nc)
    g = [2, 2, 2]
    xp = jittered_particles(rng, 3, nc)
    n = xp.shape[1]
    up = np.asfortranarray(rng.standard_normal((1, n)))
    ref, lbo, _ = O.p2m(t, xp, up, 2, g)
    for where in (n, n // 2):
        bad = np.array([[1.5, 1.7], [0.5, 0.5], [0.5, 0.5]])
        xb = np.concatenate([xp[:, :where], bad, xp[:, where:]], axis=1)
        ub = np.concatenate([up[:, :where], [[3.0, 4.0]], up[:, where:]], axis=1)
        lb, ubd = box_bounds(t, g)
        f = np.zeros((1,) + tuple(ubd[a] - lb[a] + 1 for a in range(3)) + (1,), order="F")
        info = ppmg.ppm_interp_p2m(np.asfortranarray(xb), n + 2, np.asfortranarray(ub), 1,
                                   t.topo_id, t.mesh_id, 2, g, f)
        assert info == -1 and ppmg.last_error()[1] == 405
        assert max_rel(unique_view(f, lb, [nc] * 3, 3), unique_view(ref, lbo, [nc] * 3, 3)) < 1e-13
