"""Device-pointer entry points (`_dev`) driven with torch CUDA tensors, and
size-independent properties at the benchmark's configuration sizes."""
import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import box_bounds, jittered_particles, max_rel, random_particles, topo_for
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [900]


def registered(dim, nc):
    _next_id[0] += 1
    t = topo_for(dim, nc, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def colmajor(a, dev="cuda"):
    """numpy (F-order) -> column-major torch tensor of the same shape."""
    a = np.asarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(dev)
    return t.permute(*reversed(range(t.dim())))


def test_dev_roundtrip_matches_host_path():
    rng = np.random.default_rng(90)
    t = registered(3, 32)
    g = [2, 2, 2]
    xp = random_particles(rng, 3, 60000)
    up = rng.standard_normal((3, 60000))
    lb, ub = box_bounds(t, g)
    shape = (3,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)
    f_host = np.zeros(shape, order="F")
    assert ppmg.ppm_interp_p2m(np.asfortranarray(xp), 60000, np.asfortranarray(up), 3, t.topo_id,
                               t.mesh_id, 2, g, f_host) == 0
    dxp, dup = colmajor(xp), colmajor(up)
    dfield = colmajor(np.zeros(shape))
    assert ppmg.ppm_interp_p2m(dxp, 60000, dup, 3, t.topo_id, t.mesh_id, 2, g, dfield) == 0
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
    f_dev = dfield.permute(*reversed(range(5))).contiguous().cpu().numpy().T
    assert np.array_equal(f_dev, f_host)
    dout = colmajor(np.zeros((3, 60000)))
    assert ppmg.ppm_interp_m2p(dxp, 60000, dout, 3, t.topo_id, t.mesh_id, 2, g, dfield) == 0
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
    out_host = np.zeros((3, 60000), order="F")
    assert ppmg.ppm_interp_m2p(np.asfortranarray(xp), 60000, out_host, 3, t.topo_id, t.mesh_id,
                               2, g, f_host) == 0
    assert np.array_equal(dout.t().contiguous().cpu().numpy().T, out_host)


def test_dev_out_of_box_particles_latched():
    t = registered(3, 8)
    xp = colmajor(np.array([[0.5, 1.5], [0.5, 0.5], [0.5, 0.5]]))
    up = colmajor(np.ones((1, 2)))
    f = colmajor(np.zeros((1, 13, 13, 13, 1)))
    assert ppmg.ppm_interp_p2m(xp, 2, up, 1, t.topo_id, t.mesh_id, 2, [2, 2, 2], f) == 0
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == -1
    assert ppmg.last_error()[1] == 405
    assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0  # cleared


@pytest.mark.slow
def test_config2_round_trip_properties():
    """128^3, 1 particle per cell jittered, lda 3: conservation of total strength,
    linearity and bitwise determinism, FP64 vs mixed agreement (<= 1e-6)."""
    rng = np.random.default_rng(2)
    nc = 128
    t = registered(3, nc)
    g = [2, 2, 2]
    xp = jittered_particles(rng, 3, nc)
    n = xp.shape[1]
    up = rng.standard_normal((3, n))
    lb, ub = box_bounds(t, g)
    shape = (3,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)
    dxp, dup = colmajor(xp), colmajor(up)
    res = {}
    for mode in (0, 1):
        ppmg.set_precision(mode)
        f = colmajor(np.zeros(shape))
        assert ppmg.ppm_interp_p2m(dxp, n, dup, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
        f2 = colmajor(np.zeros(shape))
        assert ppmg.ppm_interp_p2m(dxp, n, dup, 3, t.topo_id, t.mesh_id, 2, g, f2) == 0
        assert torch.equal(f, f2)
        out = colmajor(np.zeros((3, n)))
        assert ppmg.ppm_interp_m2p(dxp, n, out, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
        assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
        fu = f[:, 2:2 + nc, 2:2 + nc, 2:2 + nc, 0]
        tot = fu.sum(dim=(1, 2, 3)).cpu().numpy()
        np.testing.assert_allclose(tot, up.sum(axis=1), rtol=0,
                                   atol=1e-10 * np.abs(up).sum(axis=1).max())
        res[mode] = (fu.cpu().numpy(), out.cpu().numpy())
    ppmg.set_precision(0)
    assert max_rel(res[1][0], res[0][0]) < 1e-6
    assert max_rel(res[1][1], res[0][1]) < 1e-6
    # linearity: P2M(2u) == 2 P2M(u) exactly (power-of-two scaling)
    f3 = colmajor(np.zeros(shape))
    assert ppmg.ppm_interp_p2m(dxp, n, dup * 2, 3, t.topo_id, t.mesh_id, 2, g, f3) == 0
    assert torch.equal(f3[:, 2:2 + nc, 2:2 + nc, 2:2 + nc, 0].cpu(),
                       torch.from_numpy(res[0][0] * 2))


def _sorts_since_last_read():
    """Cell sorts the library ran since the previous read (device timing on)."""
    import ctypes as C
    ms, n = C.c_double(0.0), C.c_int64(0)
    assert ppmg.lib().ppmg_kernel_timing_read(2, C.byref(ms), C.byref(n)) == 0
    return int(n.value)


@pytest.mark.parametrize("n", [20000, 20001])
def test_m2p_reuses_p2m_order_only_for_identical_positions(n):
    """M2P after P2M of the same positions reuses P2M's cell order (fingerprint
    match: no second sort); after the positions change (even one particle, one
    ulp) it sorts again.  Both must equal the oracle.  An odd count covers the
    last particle of the paired fingerprint reads."""
    rng = np.random.default_rng(95)
    t = registered(3, 16)
    g = [2, 2, 2]
    lb, ub = box_bounds(t, g)
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((3, n)))
    shape = (3,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)
    ppmg.lib().ppmg_kernel_timing(1)
    try:
        for mode in (0, 1):
            ppmg.set_precision(mode)
            f = np.zeros(shape, order="F")
            _sorts_since_last_read()
            assert ppmg.ppm_interp_p2m(xp, n, up, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
            assert _sorts_since_last_read() == 1
            for moved in (False, True):
                xq = xp.copy(order="F")
                if moved:
                    xq[0, 7] = np.nextafter(xq[0, 7], 2.0)
                    xq[:, 100:200] = xq[:, 100:200][:, ::-1]
                out = np.zeros((3, n), order="F")
                assert ppmg.ppm_interp_m2p(xq, n, out, 3, t.topo_id, t.mesh_id, 2, g, f) == 0
                assert _sorts_since_last_read() == (1 if moved else 0), (mode, moved)
                ref = O.m2p(t, xq, f, lb, ub, 3, 2, g)
                tol = 0.0 if mode == 0 else 1e-6
                assert max_rel(out, ref) <= tol, (mode, moved)
    finally:
        ppmg.lib().ppmg_kernel_timing(0)
        ppmg.set_precision(0)


@pytest.mark.parametrize("lda", [5, 8])
def test_mixed_many_components_against_oracle(lda):
    """Mixed precision with lda > 4: the sort's record rows carry two strength
    chunks (three 16-byte units per particle) and P2M runs one launch per
    chunk.  P2M and M2P agree with the FP64 oracle to <= 1e-6.  The cluster
    puts thousands of particles into single cells; there the partial sums of
    a staging unit, plain FP32 before the compensated fold, bound the
    conservation of total strength to ~3e-9 of sum |u| (1e-10 holds at the
    benchmark densities, test_config2_round_trip_properties)."""
    rng = np.random.default_rng(500 + lda)
    nc = 24
    t = registered(3, nc)
    g = [2, 2, 2]
    n = 30000
    # a dense cluster (several staging units per layer) over a uniform background
    xp = np.concatenate([random_particles(rng, 3, n // 2),
                         np.clip(0.4 + 0.03 * rng.standard_normal((3, n - n // 2)), 0.0, 0.999)],
                        axis=1)
    up = rng.standard_normal((lda, n))
    ref, lb, ub = O.p2m(t, xp, up, 2, g)
    shape = ref.shape
    dxp, dup = colmajor(xp), colmajor(up)
    ppmg.set_precision(1)
    try:
        f = colmajor(np.zeros(shape))
        assert ppmg.ppm_interp_p2m(dxp, n, dup, lda, t.topo_id, t.mesh_id, 2, g, f) == 0
        assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
        fh = f.cpu().numpy()
        s = tuple(slice(g[a], g[a] + nc + 1) for a in range(3))
        assert max_rel(fh[(slice(None),) + s], ref[(slice(None),) + s]) < 1e-6
        tot = fh[(slice(None),) + tuple(slice(g[a], g[a] + nc) for a in range(3))].sum(
            axis=(1, 2, 3, 4))
        np.testing.assert_allclose(tot, up.sum(axis=1), rtol=0,
                                   atol=1e-8 * np.abs(up).sum(axis=1).max())
        out = colmajor(np.zeros((lda, n)))
        assert ppmg.ppm_interp_m2p(dxp, n, out, lda, t.topo_id, t.mesh_id, 2, g, f) == 0
        assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
        oref = O.m2p(t, xp, fh, lb, ub, lda, 2, g)
        assert max_rel(out.cpu().numpy(), oref) < 1e-6
    finally:
        ppmg.set_precision(0)
