"""GPU parity of P2M / M2P (through the C-ABI) against the oracle.

Tolerances (normwise max relative error, max|a-ref| / max|ref|):
  FP64 form: P2M 1e-13 (different summation order), M2P bit-identical to the
  reference arithmetic (same weights, same term order, no contraction);
  mixed form (FP64 offsets, FP32 weights, compensated FP32 sums): 1e-6;
  single-precision API: 2e-5 against the FP64 oracle.
"""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import (box_bounds, jittered_particles, max_rel, periodic_fill, random_particles,
                   topo_for, unique_view, golden_cases)
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_next_id = [100]


def registered(dim, nc, lo=None, hi=None):
    _next_id[0] += 1
    t = topo_for(dim, nc, lo, hi, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def gpu_p2m(t, xp, up, kernel, g, dtype=np.float64, scalar=False, field_lb=None, pad=0):
    dim = t.dim
    lb, ub = box_bounds(t, g)
    if field_lb is not None:
        lb = list(field_lb)
    shape = tuple(ub[a] - lb[a] + 1 + pad for a in range(dim))
    lda = 1 if scalar else up.shape[0]
    if scalar:
        f = np.full(shape + (1,), 7.0, dtype=dtype, order="F")
        info = ppmg.ppm_interp_p2m(np.asfortranarray(xp, dtype=dtype), xp.shape[1],
                                   np.ascontiguousarray(up.reshape(-1), dtype=dtype), t.topo_id,
                                   t.mesh_id, kernel, g, f, field_lb=lb)
    else:
        f = np.full((lda,) + shape + (1,), 7.0, dtype=dtype, order="F")
        info = ppmg.ppm_interp_p2m(np.asfortranarray(xp, dtype=dtype), xp.shape[1],
                                   np.asfortranarray(up, dtype=dtype), lda, t.topo_id, t.mesh_id,
                                   kernel, g, f, field_lb=lb)
    assert info == 0, ppmg.last_error()
    return f, lb


def gpu_m2p(t, xp, F, lda, kernel, g, dtype=np.float64, lb=None):
    up = np.zeros((lda, xp.shape[1]), dtype=dtype, order="F")
    info = ppmg.ppm_interp_m2p(np.asfortranarray(xp, dtype=dtype), xp.shape[1], up, lda,
                               t.topo_id, t.mesh_id, kernel, g, np.asfortranarray(F, dtype=dtype),
                               field_lb=lb)
    assert info == 0, ppmg.last_error()
    return up


@pytest.fixture(params=["fp64", "mixed"])
def precision(request):
    mode = 0 if request.param == "fp64" else 1
    assert ppmg.set_precision(mode) == 0
    yield request.param
    ppmg.set_precision(0)


TOL_P2M = {"fp64": 1e-13, "mixed": 1e-6}


@pytest.mark.parametrize("dim,kernel,nc,lda", [
    (3, 2, 16, 3), (3, 2, 24, 1), (3, 1, 16, 3), (3, 2, 20, 5), (3, 2, 33, 2), (3, 2, 5, 1),
    (2, 2, 64, 1), (2, 2, 40, 3),
])
def test_p2m_matches_oracle(precision, dim, kernel, nc, lda):
    rng = np.random.default_rng(nc * 10 + lda)
    t = registered(dim, nc)
    g = [2] * dim
    xp = random_particles(rng, dim, 3 * nc ** dim // 2)
    up = rng.standard_normal((lda, xp.shape[1]))
    f, lb = gpu_p2m(t, xp, up, kernel, g)
    fo, lbo, ubo = O.p2m(t, xp, up, kernel, g)
    # real nodes (incl. the duplicate node Nm) against the reference after put
    real = (slice(None),) + tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(dim)) + (0,)
    assert max_rel(f[real], fo[real]) < TOL_P2M[precision]
    # ghost layers: the periodic images of the real nodes
    U = unique_view(f, lb, [nc] * dim, dim)
    assert max_rel(f, periodic_fill(U, lb, [t.Nm[a] + g[a] for a in range(dim)], dim)) == 0.0


@pytest.mark.parametrize("case", golden_cases("p2m"), ids=lambda c: c["name"])
def test_p2m_matches_golden(precision, case):
    dim, nc = case["dim"], case["nc"]
    t = registered(dim, nc, case["lo"], case["hi"])
    xp = np.asfortranarray(np.array(case["xp"]).T)
    up = np.asfortranarray(np.array(case["up"]).T)
    f, lb = gpu_p2m(t, xp, up, case["kernel"], [2] * dim)
    ref = np.array(case["field"]).reshape((case["lda"],) + tuple(nc), order="F")
    assert max_rel(unique_view(f, lb, nc, dim), ref) < TOL_P2M[precision]


def test_p2m_is_deterministic_and_order_independent():
    """Bitwise identical across runs and under a permutation of the particles
    (the per-cell order is the ascending particle id)."""
    rng = np.random.default_rng(11)
    t = registered(3, 24)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, 40000)
    up = rng.standard_normal((3, 40000))
    for mode in (0, 1):
        ppmg.set_precision(mode)
        f1, _ = gpu_p2m(t, xp, up, 2, g)
        f2, _ = gpu_p2m(t, xp, up, 2, g)
        assert np.array_equal(f1, f2)
    ppmg.set_precision(0)


def test_p2m_scalar_and_single_variants():
    rng = np.random.default_rng(12)
    t = registered(3, 16)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, 5000)
    up = rng.standard_normal((1, 5000))
    fo, lbo, _ = O.p2m(t, xp, up, 2, g)
    fs, lb = gpu_p2m(t, xp, up, 2, g, scalar=True)
    real3 = tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(3)) + (0,)
    assert max_rel(fs[real3], fo[0][real3]) < 1e-13
    f32, lb = gpu_p2m(t, xp, up, 2, g, dtype=np.float32)
    real = (slice(None),) + tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(3)) + (0,)
    assert max_rel(f32[real].astype(np.float64), fo[real]) < 2e-5


def test_p2m_larger_allocation_keeps_outside_values():
    """A field allocated beyond 1-g:Nm+g keeps what lies outside the box."""
    rng = np.random.default_rng(13)
    t = registered(3, 12)
    g = [1, 1, 1]
    xp = random_particles(rng, 3, 2000)
    up = rng.standard_normal((2, 2000))
    lb = [-2, -2, -2]
    f, _ = gpu_p2m(t, xp, up, 2, g, field_lb=lb, pad=2)
    fo, lbo, _ = O.p2m(t, xp, up, 2, g)
    # outside the written box the 7.0 fill survives
    assert np.all(f[:, 0, :, :, 0] == 7.0) and np.all(f[:, -1, :, :, 0] == 7.0)
    off = [lbo[a] - lb[a] for a in range(3)]
    sub = f[:, off[0]:off[0] + fo.shape[1], off[1]:off[1] + fo.shape[2], off[2]:off[2] + fo.shape[3]]
    real = (slice(None),) + tuple(slice(1 - lbo[a], t.Nm[a] + 1 - lbo[a]) for a in range(3)) + (0,)
    assert max_rel(sub[real], fo[real]) < 1e-13


def test_p2m_particles_outside_are_fatal():
    t = registered(3, 8)
    xp = np.asfortranarray([[0.5, 1.0, 0.2], [0.5, 0.5, 0.3], [0.5, 0.5, 0.4]])
    up = np.ones((1, 3), order="F")
    f = np.zeros((1, 13, 13, 13, 1), order="F")
    info = ppmg.ppm_interp_p2m(xp, 3, up, 1, t.topo_id, t.mesh_id, 2, [2, 2, 2], f)
    assert info == -1
    assert ppmg.last_error()[1] == 405


def test_p2m_zero_particles_zeroes_the_box():
    t = registered(3, 8)
    f = np.full((2, 13, 13, 13, 1), 3.0, order="F")
    info = ppmg.ppm_interp_p2m(np.zeros((3, 1), order="F"), 0, np.zeros((2, 1), order="F"), 2,
                               t.topo_id, t.mesh_id, 2, [2, 2, 2], f)
    assert info == 0 and np.all(f == 0.0)


@pytest.mark.parametrize("dim,kernel,nc,lda,box", [
    (3, 2, 16, 3, None), (3, 1, 16, 2, None), (3, 2, 11, 1, ([0.0, -0.5, 0.25], [1.3, 0.5, 1.0])),
    (2, 2, 32, 2, None), (2, 1, 20, 1, ([0.0, 0.0], [2.0, 1.5])),
])
def test_m2p_fp64_bit_identical_to_reference(dim, kernel, nc, lda, box):
    rng = np.random.default_rng(21 + nc)
    lo, hi = box if box else (None, None)
    t = registered(dim, nc, lo, hi)
    g = [2] * dim
    lb, ub = box_bounds(t, g)
    lo_ = t.min_phys[:dim]
    hi_ = t.max_phys[:dim]
    xp = random_particles(rng, dim, 4000, lo_, hi_)
    U = rng.standard_normal((lda,) + (nc,) * dim)
    F = periodic_fill(U, lb, ub, dim)
    ref = O.m2p(t, xp, F, lb, ub, lda, kernel, g)
    got = gpu_m2p(t, xp, F, lda, kernel, g)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("case", golden_cases("m2p"), ids=lambda c: c["name"])
def test_m2p_matches_golden(precision, case):
    dim, nc, lda = case["dim"], case["nc"], case["lda"]
    t = registered(dim, nc, case["lo"], case["hi"])
    xp = np.asfortranarray(np.array(case["xp"]).T)
    U = np.array(case["F"]).reshape((lda,) + tuple(nc), order="F")
    g = [2] * dim
    lb, ub = box_bounds(t, g)
    got = gpu_m2p(t, xp, periodic_fill(U, lb, ub, dim), lda, case["kernel"], g)
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert max_rel(got, np.array(case["up"]).T) < tol


def test_m2p_mixed_and_single_tolerance():
    rng = np.random.default_rng(31)
    t = registered(3, 32)
    g = [2, 2, 2]
    lb, ub = box_bounds(t, g)
    xp = random_particles(rng, 3, 50000)
    U = rng.standard_normal((3, 32, 32, 32))
    F = periodic_fill(U, lb, ub, 3)
    ref = O.m2p(t, xp, F, lb, ub, 3, 2, g)
    ppmg.set_precision(1)
    try:
        got = gpu_m2p(t, xp, F, 3, 2, g)
    finally:
        ppmg.set_precision(0)
    assert max_rel(got, ref) < 1e-6
    got32 = gpu_m2p(t, xp, F, 3, 2, g, dtype=np.float32)
    assert max_rel(got32.astype(np.float64), ref) < 2e-5


def test_roundtrip_config1_2d():
    """Config 1 shape: 2D M'4, 64^2 periodic, 1 particle per cell jittered, lda 1."""
    rng = np.random.default_rng(1)
    t = registered(2, 64)
    g = [2, 2]
    xp = jittered_particles(rng, 2, 64)
    up = rng.standard_normal((1, xp.shape[1]))
    f, lb = gpu_p2m(t, xp, up, 2, g)
    fo, lbo, ubo = O.p2m(t, xp, up, 2, g)
    real = (slice(None),) + tuple(slice(1 - lb[a], t.Nm[a] + 1 - lb[a]) for a in range(2)) + (0,)
    assert max_rel(f[real], fo[real]) < 1e-13
    O.ghost_get(t, fo, lbo, ubo, g)
    ref = O.m2p(t, xp, fo, lbo, ubo, 1, 2, g)
    got = gpu_m2p(t, xp, f, 1, 2, g)
    assert max_rel(got, ref) < 1e-13
