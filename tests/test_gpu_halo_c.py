"""The ghost exchange between z-slab subdomains through the C-ABI: a transport
registered on each slab handle (ppmg_halo_set_transport, here halo.CTransport
over halo.ThreadMover), with every slab's call on a host thread of its own,
as one process per GPU calls it on its own slab.  The library's results must
equal the Python exchange (halo.put / halo.get over LocalComm) bit for bit:
P2M ending with the put, the standalone ghost get followed by M2P, remesh
ending with the put, through the device and the host entry points."""
import copy
import threading

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import halo
from _util import random_particles, topo_for
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [9100]


def slab_handles(t, mover=None):
    out = []
    for s in range(t.nsubs):
        _next_id[0] += 1
        ts = copy.deepcopy(t)
        ts.topo_id = _next_id[0]
        assert ppmg.register(ts, isub=s) == 0, ppmg.last_error()
        if mover is not None:
            halo.CTransport(ts.topo_id, ts.mesh_id, s, mover)
        out.append(ts)
    return out


def dev_f(a):
    d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
    return d.permute(*reversed(range(d.dim())))


def host(a):
    if isinstance(a, np.ndarray):
        return a
    return a.permute(*reversed(range(a.dim()))).contiguous().cpu().numpy().T


def in_threads(fn, n):
    """fn(s) for every slab s, each on a thread of its own; returns the infos."""
    res, errs = [None] * n, []

    def run(s):
        try:
            res[s] = fn(s)
        except Exception as e:  # noqa: BLE001
            errs.append(repr(e))
    th = [threading.Thread(target=run, args=(s,)) for s in range(n)]
    for x in th:
        x.start()
    for x in th:
        x.join(timeout=120)
    assert not errs, errs
    return res


def setup(nc, nslab, lda, seed):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    n = 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    return t, xp, up, ids


def shape_of(t, s, nc, g, lda):
    nz = int(t.nnodes[s, 2]) - 1
    return (lda, nc + 1 + 2 * g, nc + 1 + 2 * g, nz + 1 + 2 * g, 1)


@pytest.mark.parametrize("nslab,kernel,g,lda,mode,entry", [
    (2, 2, 2, 3, 0, "dev"), (3, 2, 2, 1, 1, "dev"), (3, 1, 1, 2, 0, "host"),
    (2, 2, 3, 3, 1, "host")])
def test_c_exchange_equals_python_exchange(nslab, kernel, g, lda, mode, entry):
    nc = 12
    t, xp, up, ids = setup(nc, nslab, lda, seed=40 + nslab + g)
    gg = [g] * 3
    lb = [1 - g] * 3
    wrap = dev_f if entry == "dev" else (lambda a: np.asfortranarray(a))
    ppmg.set_precision(mode)
    try:
        # Python exchange (the reference for this test)
        hp = slab_handles(t)
        fp = {}
        for s, ts in enumerate(hp):
            f = dev_f(np.full(shape_of(t, s, nc, g, lda), 9.0))
            assert ppmg.ppm_interp_p2m(dev_f(xp[:, ids[s]]), len(ids[s]), dev_f(up[:, ids[s]]),
                                       lda, ts.topo_id, 1, kernel, gg, f, exchange=False) == 0
            fp[s] = f
        halo.put(fp, t, gg, lb, halo.LocalComm())
        # the library's exchange: P2M on every slab ends with the put
        mover = halo.ThreadMover(timeout=60)
        hc = slab_handles(t, mover)
        fc = {s: wrap(np.full(shape_of(t, s, nc, g, lda), 9.0)) for s in range(nslab)}
        xs = {s: wrap(xp[:, ids[s]]) for s in range(nslab)}
        us = {s: wrap(up[:, ids[s]]) for s in range(nslab)}

        def p2m(s):
            info = ppmg.ppm_interp_p2m(xs[s], len(ids[s]), us[s], lda, hc[s].topo_id, 1, kernel,
                                       gg, fc[s])
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        assert in_threads(p2m, nslab) == [0] * nslab, ppmg.last_error()
        for s in range(nslab):
            assert np.array_equal(host(fc[s]), host(fp[s])), s
        # ghost get (standalone) then M2P on every slab
        halo.get(fp, t, gg, lb, halo.LocalComm())

        def get(s):
            info = ppmg.ppm_map_field_ghost(fc[s], lda, hc[s].topo_id, 1, gg,
                                            ppmg.params.ppm_param_map_ghost_get)
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        assert in_threads(get, nslab) == [0] * nslab, ppmg.last_error()
        for s in range(nslab):
            assert np.array_equal(host(fc[s]), host(fp[s])), s
            out_c = wrap(np.zeros((lda, len(ids[s]))))
            out_p = dev_f(np.zeros((lda, len(ids[s]))))
            assert ppmg.ppm_interp_m2p(xs[s], len(ids[s]), out_c, lda, hc[s].topo_id, 1, kernel,
                                       gg, fc[s]) == 0
            assert ppmg.ppm_interp_m2p(dev_f(xp[:, ids[s]]), len(ids[s]), out_p, lda,
                                       hp[s].topo_id, 1, kernel, gg, fp[s]) == 0
            assert ppmg.sync_status(hc[s].topo_id, 1) == 0
            assert ppmg.sync_status(hp[s].topo_id, 1) == 0
            assert np.array_equal(host(out_c), host(out_p))
    finally:
        ppmg.set_precision(0)


def test_c_remesh_ends_with_the_put():
    nc, nslab, g, lda = 12, 3, 2, 3
    t, xp, up, ids = setup(nc, nslab, lda, seed=77)
    gg = [g] * 3
    hp = slab_handles(t)
    hc = slab_handles(t, halo.ThreadMover(timeout=60))
    fp, fc = {}, {}
    for s in range(nslab):
        xs = np.asfortranarray(xp[:, ids[s]])
        us = np.asfortranarray(up[:, ids[s]])
        for hs, fd in ((hp, fp), (hc, fc)):
            assert ppmg.ppm_rmsh_comp_weights(xs, len(ids[s]), hs[s].topo_id, 1, 2) == 0
        fp[s] = np.zeros(shape_of(t, s, nc, g, lda), order="F")
        assert ppmg.ppm_rmsh_remesh(xs, len(ids[s]), us, lda, hp[s].topo_id, 1, 2, gg, fp[s],
                                    exchange=False) == 0
        fc[s] = np.zeros(shape_of(t, s, nc, g, lda), order="F")
    halo.put({s: torch.from_numpy(fp[s]) for s in fp}, t, gg, [1 - g] * 3, halo.LocalComm())

    def remesh(s):
        return ppmg.ppm_rmsh_remesh(np.asfortranarray(xp[:, ids[s]]), len(ids[s]),
                                    np.asfortranarray(up[:, ids[s]]), lda, hc[s].topo_id, 1, 2,
                                    gg, fc[s])
    assert in_threads(remesh, nslab) == [0] * nslab, ppmg.last_error()
    for s in range(nslab):
        assert np.array_equal(fc[s], fp[s])


class _Failing:
    def exchange(self, me, sends, recvs, on_device, stream):
        raise RuntimeError("link down")


def test_failing_transport_is_reported():
    nc, g = 12, 2
    t, xp, up, ids = setup(nc, 2, 1, seed=5)
    hc = slab_handles(t, _Failing())
    f = dev_f(np.zeros(shape_of(t, 0, nc, g, 1)))
    info = ppmg.ppm_interp_p2m(dev_f(xp[:, ids[0]]), len(ids[0]), dev_f(up[:, ids[0]]), 1,
                               hc[0].topo_id, 1, 2, [g] * 3, f)
    assert info == -1 and ppmg.last_error()[1] == 2
    info = ppmg.ppm_map_field_ghost(f, 1, hc[0].topo_id, 1, [g] * 3,
                                    ppmg.params.ppm_param_map_ghost_put)
    assert info == -1 and ppmg.last_error()[1] == 2
    halo.c_transport(hc[0].topo_id, 1).close()
    assert not halo.has_c_transport(hc[0].topo_id, 1)
    # without a transport the library refuses the slab (the caller exchanges)
    import ctypes as C
    from ppm_legacy_b200._lib import int_array
    fh = np.zeros(shape_of(t, 0, nc, g, 1), order="F")
    lb = [1 - g] * 3
    ub = [lb[a] + fh.shape[1 + a] - 1 for a in range(3)]
    i = C.c_int(0)
    ppmg.lib().ppmg_map_field_ghost_d(fh.ctypes.data, 1, 1, int_array(lb, C.c_int64),
                                      int_array(ub, C.c_int64), hc[0].topo_id, 1,
                                      int_array([g] * 3), 6, C.byref(i))
    assert i.value == -2 and ppmg.last_error()[1] == 503
