"""The P2M entry point that allocates nothing (ppmg_interp_p2m_dv_3d_noalloc),
called through the C-ABI and checked against ppmg_interp_p2m_dv_3d_dev on the
same inputs.  Two calls in a row share the library's fixed scratch array, so
the second one also shows that nothing of the first call's contents leaks."""
import ctypes as C

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from _util import box_bounds, max_rel, random_particles, topo_for
from ppm_legacy_b200._lib import int_array, last_error, lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [7000]


def registered(nc):
    _next_id[0] += 1
    t = topo_for(3, nc, topo_id=_next_id[0], mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    return t


def colmajor(a):
    """numpy (F-order) -> column-major CUDA tensor of the same shape."""
    d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
    return d.permute(*reversed(range(d.dim())))


def p2m_call(name, t, xp, np_, up, lda, kernel, g, field):
    """One P2M through the C-ABI on the current torch stream; returns info."""
    lb, ub = box_bounds(t, g)
    info = C.c_int(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    getattr(lib(), name)(xp.data_ptr(), xp.shape[0], np_, up.data_ptr(), up.shape[0], lda,
                         t.topo_id, t.mesh_id, kernel, int_array(g), field.data_ptr(),
                         field.shape[0], int_array(lb, C.c_int64), int_array(ub, C.c_int64),
                         C.byref(info), stream)
    return info.value


def case(seed, nc, np_, lda, kernel):
    rng = np.random.default_rng(seed)
    t = registered(nc)
    g = [2, 2, 2]
    xp = colmajor(random_particles(rng, 3, np_))
    up = colmajor(rng.standard_normal((lda, np_)))
    lb, ub = box_bounds(t, g)
    shape = (lda,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)
    return t, g, xp, up, shape


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_p2m_matches_dev_entry_point_twice(mode):
    ppmg.set_precision(mode)
    try:
        calls = [case(11, 48, 100000, 3, 2), case(12, 32, 30000, 4, 1)]
        lda_k = [(3, 2), (4, 1)]
        fresh = []
        # two no-alloc calls in a row on one stream (the second reuses the array)
        for (t, g, xp, up, shape), (lda, kernel) in zip(calls, lda_k):
            f = colmajor(np.full(shape, 7.0))
            info = p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, xp.shape[1], up, lda,
                            kernel, g, f)
            assert info == 0, last_error()
            fresh.append(f)
        for (t, g, xp, up, shape), (lda, kernel), f in zip(calls, lda_k, fresh):
            ref = colmajor(np.full(shape, 7.0))
            info = p2m_call("ppmg_interp_p2m_dv_3d_dev", t, xp, xp.shape[1], up, lda, kernel,
                            g, ref)
            assert info == 0, last_error()
            assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0
            a, b = f.cpu().numpy(), ref.cpu().numpy()
            assert np.isfinite(a).all()
            assert max_rel(a, b) <= 1e-13
    finally:
        ppmg.set_precision(0)


def test_noalloc_p2m_rejects_sizes_beyond_its_scratch():
    t, g, xp, up, shape = case(13, 8, 131073, 1, 2)
    f = colmajor(np.zeros(shape))
    assert p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, 131073, up, 1, 2, g, f) == -2
    info, errnum, msg = last_error()
    assert errnum == 503 and "131072" in msg
    t, g, xp, up, shape = case(14, 8, 100, 5, 2)
    f = colmajor(np.zeros(shape))
    assert p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, 100, up, 5, 2, g, f) == -2
    t, g, xp, up, shape = case(15, 65, 100, 1, 2)  # 65^3 cells > 262144
    f = colmajor(np.zeros(shape))
    assert p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, 100, up, 1, 2, g, f) == -2
    torch.cuda.synchronize()


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_p2m_at_its_documented_maxima(mode):
    """Np = 131072 particles on 64^3 = 262144 cells with lda 4 (the largest
    call the header promises; in FP64 its views take ~12.5 of the 16 MiB):
    the same field as the _dev entry point, twice in a row."""
    ppmg.set_precision(mode)
    try:
        t, g, xp, up, shape = case(21, 64, 131072, 4, 2)
        ref = colmajor(np.full(shape, 3.0))
        assert p2m_call("ppmg_interp_p2m_dv_3d_dev", t, xp, 131072, up, 4, 2, g, ref) == 0
        assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0, last_error()
        for _ in range(2):
            f = colmajor(np.full(shape, 3.0))
            info = p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, 131072, up, 4, 2, g, f)
            assert info == 0, last_error()
            assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0, last_error()
            assert max_rel(f.cpu().numpy(), ref.cpu().numpy()) <= 1e-13
    finally:
        ppmg.set_precision(0)


def test_noalloc_p2m_leaves_device_memory_unchanged():
    """After one warm-up call (which may load the kernels' code), a call on a
    freshly registered handle changes the free device memory by nothing."""
    t, g, xp, up, shape = case(31, 48, 100000, 3, 2)
    f = colmajor(np.zeros(shape))
    assert p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t, xp, 100000, up, 3, 2, g, f) == 0
    torch.cuda.synchronize()
    t2, g2, xp2, up2, shape2 = case(32, 48, 100000, 3, 2)
    f2 = colmajor(np.zeros(shape2))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert p2m_call("ppmg_interp_p2m_dv_3d_noalloc", t2, xp2, 100000, up2, 3, 2, g2, f2) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert ppmg.sync_status(t2.topo_id, t2.mesh_id) == 0, last_error()


@pytest.mark.parametrize("bad", ["outside", "nan"])
def test_noalloc_p2m_reports_invalid_particles_like_dev(bad):
    """A few particles outside [min_sub, max_sub) or with a NaN coordinate:
    the same info and errnum from ppmg_sync_status as the _dev entry point,
    and the same field from the valid particles."""
    rng = np.random.default_rng(41)
    t = registered(32)
    g = [2, 2, 2]
    n = 20000
    x = random_particles(rng, 3, n)
    if bad == "outside":
        x[0, 5], x[1, 77], x[2, 901] = 1.25, -0.5, 1.0
    else:
        x[1, 5], x[2, 77] = np.nan, np.nan
    xp = colmajor(x)
    up = colmajor(rng.standard_normal((3, n)))
    lb, ub = box_bounds(t, g)
    shape = (3,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,)
    res = {}
    for name in ("ppmg_interp_p2m_dv_3d_dev", "ppmg_interp_p2m_dv_3d_noalloc"):
        f = colmajor(np.zeros(shape))
        assert p2m_call(name, t, xp, n, up, 3, 2, g, f) == 0, last_error()
        info = ppmg.sync_status(t.topo_id, t.mesh_id)
        res[name] = (info, last_error()[1], f.cpu().numpy())
        assert ppmg.sync_status(t.topo_id, t.mesh_id) == 0  # cleared
    a, b = res.values()
    assert a[0] == b[0] and a[0] < 0
    assert a[1] == b[1] and a[1] > 0
    assert max_rel(b[2], a[2]) <= 1e-13
