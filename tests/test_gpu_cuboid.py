"""3D P2M, M2P, the P2M adjoint and remeshing on subdomains of cartesian
decompositions cut along several axes (2 x 2 x 2, 2 x 2 x 1, 3 x 1 x 2 ...),
against the oracle's multi-subdomain routines (ppm_interp_p2m.f,
ppm_interp_m2p.f and ppm_rmsh_remesh.f on every subdomain of the topology,
ppm_map_field_ghost between them).

Every subdomain is a handle of its own in this process.  The library's
exchange (a transport registered with ppmg_halo_set_transport, here
halo.CTransport over halo.ThreadMover, each subdomain's call on a host thread
of its own) must equal the Python exchange (halo.put / halo.get over
LocalComm, the same boxes) bit for bit, and both the oracle."""
import copy
import threading

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import halo
from _util import max_rel, random_particles, topo_for
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [11000]


def sub_handles(t, mover=None):
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


def release(hs):
    for ts in hs:
        tr = halo.c_transport(ts.topo_id, ts.mesh_id)
        if tr is not None:
            tr.close()
        ppmg.unregister(ts)


def dev_f(a):
    d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
    return d.permute(*reversed(range(d.dim())))


def host(a):
    if isinstance(a, np.ndarray):
        return a
    return a.permute(*reversed(range(a.dim()))).contiguous().cpu().numpy().T


def in_threads(fn, n):
    """fn(s) for every subdomain s, each on a thread of its own."""
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
        x.join(timeout=180)
    assert not errs, errs
    return res


def nodes(t, s):
    return [int(t.nnodes[s, a]) for a in range(3)]


def shape_of(t, s, g, lda):
    n = nodes(t, s)
    return (lda,) + tuple(n[a] + 2 * g[a] for a in range(3)) + (1,)


def real_of(t, s, g):
    n = nodes(t, s)
    return (slice(None),) + tuple(slice(g[a], g[a] + n[a]) for a in range(3)) + (0,)


def oracle_real(fo, lbo, t, s):
    n = nodes(t, s)
    return fo[(slice(None),) + tuple(slice(1 - lbo[a], 1 - lbo[a] + n[a]) for a in range(3))
              + (s,)]


def setup(nc, decomp, lda, seed, n=None):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=decomp)
    n = n or 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    return t, xp, up, ids


@pytest.mark.parametrize("nc,decomp,kernel,g,lda,mode,entry", [
    (12, (2, 2, 2), 2, (2, 2, 2), 3, 0, "dev"),
    (12, (2, 2, 1), 2, (1, 2, 2), 1, 0, "host"),
    (13, (3, 1, 2), 1, (1, 1, 1), 2, 0, "dev"),
    (16, (2, 2, 2), 2, (2, 2, 2), 2, 1, "dev"),
    (16, (1, 2, 2), 2, (2, 3, 2), 5, 0, "host"),
    (40, (2, 1, 1), 2, (2, 2, 2), 1, 0, "dev")])
def test_cuboid_p2m_put_get_m2p(nc, decomp, kernel, g, lda, mode, entry):
    t, xp, up, ids = setup(nc, decomp, lda, seed=nc + sum(decomp) + lda)
    ns = t.nsubs
    wrap = dev_f if entry == "dev" else (lambda a: np.asfortranarray(a))
    lb = [1 - g[a] for a in range(3)]
    ppmg.set_precision(mode)
    hp = sub_handles(t)
    hc = sub_handles(t, halo.ThreadMover(timeout=120))
    try:
        # the Python exchange over the library's local deposits
        fp = {}
        for s, ts in enumerate(hp):
            f = dev_f(np.full(shape_of(t, s, g, lda), 9.0))
            assert ppmg.ppm_interp_p2m(dev_f(xp[:, ids[s]]), len(ids[s]), dev_f(up[:, ids[s]]),
                                       lda, ts.topo_id, 1, kernel, list(g), f,
                                       exchange=False) == 0, ppmg.last_error()
            fp[s] = f
        halo.put(fp, t, list(g), lb, halo.LocalComm())
        # the library's exchange: P2M on every subdomain ends with the put
        fc = {s: wrap(np.full(shape_of(t, s, g, lda), 9.0)) for s in range(ns)}
        xs = {s: wrap(xp[:, ids[s]]) for s in range(ns)}
        us = {s: wrap(up[:, ids[s]]) for s in range(ns)}

        def p2m(s):
            info = ppmg.ppm_interp_p2m(xs[s], len(ids[s]), us[s], lda, hc[s].topo_id, 1, kernel,
                                       list(g), fc[s])
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        assert in_threads(p2m, ns) == [0] * ns, ppmg.last_error()
        fo, lbo, ubo = O.p2m(t, xp, up, kernel, list(g))
        tol = 1e-13 if mode == 0 else 1e-6
        for s in range(ns):
            assert np.array_equal(host(fc[s]), host(fp[s])), s
            got = host(fc[s])[real_of(t, s, g)]
            ref = oracle_real(fo, lbo, t, s)
            assert max_rel(got, ref) < tol, (s, max_rel(got, ref))
        # ghost get (standalone), then M2P on every subdomain
        halo.get(fp, t, list(g), lb, halo.LocalComm())

        def get(s):
            info = ppmg.ppm_map_field_ghost(fc[s], lda, hc[s].topo_id, 1, list(g),
                                            ppmg.params.ppm_param_map_ghost_get)
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        assert in_threads(get, ns) == [0] * ns, ppmg.last_error()
        O.ghost_get(t, fo, lbo, ubo, list(g))
        ref = O.m2p(t, xp, fo, lbo, ubo, lda, kernel, list(g))
        mt = 1e-13 if mode == 0 else 1e-6
        for s in range(ns):
            assert np.array_equal(host(fc[s]), host(fp[s])), s
            out = wrap(np.zeros((lda, len(ids[s]))))
            assert ppmg.ppm_interp_m2p(xs[s], len(ids[s]), out, lda, hc[s].topo_id, 1, kernel,
                                       list(g), fc[s]) == 0, ppmg.last_error()
            assert ppmg.sync_status(hc[s].topo_id, 1) == 0, ppmg.last_error()
            assert max_rel(host(out), ref[:, ids[s]]) <= mt, (s, max_rel(host(out),
                                                                       ref[:, ids[s]]))
    finally:
        ppmg.set_precision(0)
        release(hp + hc)


def test_cuboid_particles_on_the_faces():
    """Particles on the faces between subdomains and one ulp below them, on
    every cut axis (the stencil origin may round up to the subdomain's upper
    face)."""
    rng = np.random.default_rng(12)
    nc, decomp, g, lda = 12, (2, 2, 2), (2, 2, 2), 2
    t = topo_for(3, nc, decomp=decomp)
    n = 6000
    xp = random_particles(rng, 3, n)
    for a in range(3):
        faces = np.unique(np.concatenate([t.min_sub[:, a], t.max_sub[:, a]]))
        faces = faces[faces < 1.0]
        pick = np.concatenate([faces, np.nextafter(faces[1:], 0.0)])
        sel = rng.random(n) < 0.3
        xp[a, sel] = rng.choice(pick, sel.sum())
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    hc = sub_handles(t, halo.ThreadMover(timeout=120))
    try:
        fc = {s: dev_f(np.zeros(shape_of(t, s, g, lda))) for s in range(t.nsubs)}

        def p2m(s):
            info = ppmg.ppm_interp_p2m(dev_f(xp[:, ids[s]]), len(ids[s]), dev_f(up[:, ids[s]]),
                                       lda, hc[s].topo_id, 1, 2, list(g), fc[s])
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        assert in_threads(p2m, t.nsubs) == [0] * t.nsubs, ppmg.last_error()
        fo, lbo, _ = O.p2m(t, xp, up, 2, list(g))
        for s in range(t.nsubs):
            got = host(fc[s])[real_of(t, s, g)]
            assert max_rel(got, oracle_real(fo, lbo, t, s)) < 1e-13, s
    finally:
        release(hc)


@pytest.mark.parametrize("decomp,kernel", [((2, 2, 2), 2), ((2, 1, 3), 1)])
def test_cuboid_adjoint_matches_global_oracle(decomp, kernel):
    """The P2M adjoint on every subdomain (r's ghost layers by the library's
    ghost get, which the Python wrapper runs first) equals the oracle's
    adjoint over the whole domain."""
    rng = np.random.default_rng(900 + sum(decomp))
    nc, lda, g = 12, 2, (2, 2, 2)
    t = topo_for(3, nc, decomp=decomp)
    t1 = topo_for(3, nc)
    n = 4000
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    R = rng.standard_normal((lda, nc, nc, nc))
    dwo, dxo = O.p2m_adjoint(t1, xp, up, np.asfortranarray(R[..., None]), [1, 1, 1], [nc] * 3,
                             kernel)
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    hc = sub_handles(t, halo.ThreadMover(timeout=120))
    try:
        rs = {}
        for s in range(t.nsubs):
            n_ = nodes(t, s)
            idx, ghost = [], []
            for a in range(3):
                i0 = int(t.istart[s, a]) - 1
                idx.append((i0 + np.arange(1 - g[a], n_[a] + g[a] + 1) - 1) % nc)
            loc = np.array(R[np.ix_(range(lda), *idx)])
            for a in range(3):  # ghost layers of the cut axes: junk, the get fills them
                if n_[a] != nc + 1:
                    sl = [slice(None)] * 4
                    sl[1 + a] = slice(0, g[a])
                    loc[tuple(sl)] = 1e6
                    sl[1 + a] = slice(n_[a] + g[a], None)
                    loc[tuple(sl)] = 1e6
            rs[s] = dev_f(loc[..., None])
        res = {}

        def adj(s):
            m = len(ids[s])
            dw = dev_f(np.zeros((lda, m)))
            dx = dev_f(np.zeros((3, m)))
            info = ppmg.ppm_interp_p2m_adjoint(dev_f(xp[:, ids[s]]), m, dev_f(up[:, ids[s]]),
                                               lda, hc[s].topo_id, 1, kernel, rs[s], dw, dx,
                                               ghostsize=list(g))
            info = info if info else ppmg.sync_status(hc[s].topo_id, 1)
            res[s] = (dw, dx)
            return info
        assert in_threads(adj, t.nsubs) == [0] * t.nsubs, ppmg.last_error()
        for s in range(t.nsubs):
            dw, dx = res[s]
            assert max_rel(host(dw), dwo[:, ids[s]]) < 1e-12, s
            assert max_rel(host(dx), dxo[:, ids[s]]) < 1e-11, s
    finally:
        release(hc)


@pytest.mark.parametrize("decomp,kernel", [((2, 2, 2), 2), ((3, 2, 1), 1)])
def test_cuboid_remesh_and_create_part(decomp, kernel):
    """comp_weights, remesh (ending with the library's put) and create_part
    on every subdomain: the field's real nodes equal the oracle's, and the
    particles created by all subdomains together equal the oracle's, each
    shared upper node of a cut axis creating none."""
    rng = np.random.default_rng(300 + sum(decomp) + kernel)
    nc, lda = 12, 2
    t = topo_for(3, nc, decomp=decomp)
    n = 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    g = (2, 2, 2) if kernel == 2 else (1, 1, 1)
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    wo, lsto, sio = O.comp_weights(t, xp, kernel)
    fo, lbo, ubo = O.remesh(t, xp, up, kernel, list(g), wo, lsto, sio)
    cut = [0.2, 1e300]
    no, upo, xpo, _ = O.create_part(t, fo, lbo, ubo, cut)
    hp = sub_handles(t)
    hc = sub_handles(t, halo.ThreadMover(timeout=120))
    try:
        fp, fc = {}, {}
        for s in range(t.nsubs):
            xs = np.asfortranarray(xp[:, ids[s]])
            for hs in (hp, hc):
                assert ppmg.ppm_rmsh_comp_weights(xs, len(ids[s]), hs[s].topo_id, 1,
                                                  kernel) == 0, ppmg.last_error()
            fp[s] = np.zeros(shape_of(t, s, g, lda), order="F")
            assert ppmg.ppm_rmsh_remesh(xs, len(ids[s]), np.asfortranarray(up[:, ids[s]]), lda,
                                        hp[s].topo_id, 1, kernel, list(g), fp[s],
                                        exchange=False) == 0, ppmg.last_error()
            fc[s] = dev_f(np.zeros(shape_of(t, s, g, lda)))
        halo.put({s: torch.from_numpy(fp[s]) for s in fp}, t, list(g), [1 - v for v in g],
                 halo.LocalComm())

        def remesh(s):
            info = ppmg.ppm_rmsh_remesh(dev_f(xp[:, ids[s]]), len(ids[s]), dev_f(up[:, ids[s]]),
                                        lda, hc[s].topo_id, 1, kernel, list(g), fc[s])
            return info if info else ppmg.sync_status(hc[s].topo_id, 1)
        # device remesh needs device weights: recompute them on device positions
        for s in range(t.nsubs):
            assert ppmg.ppm_rmsh_comp_weights(dev_f(xp[:, ids[s]]), len(ids[s]), hc[s].topo_id,
                                              1, kernel) == 0, ppmg.last_error()
        assert in_threads(remesh, t.nsubs) == [0] * t.nsubs, ppmg.last_error()
        ups, xps = [], []
        for s, ts in enumerate(hc):
            assert np.array_equal(host(fc[s]), fp[s]), s
            got = host(fc[s])[real_of(t, s, g)]
            assert max_rel(got, oracle_real(fo, lbo, t, s)) < 1e-13, s
            info, m, upn, xpn, _ = ppmg.ppm_rmsh_create_part(fc[s], ts.topo_id, 1, cut, lda=lda,
                                                             resetpos=True, ghostsize=list(g))
            assert info == 0, ppmg.last_error()
            ups.append(host(upn).reshape(lda, -1))
            xps.append(host(xpn))
        upg, xpg = np.concatenate(ups, axis=1), np.concatenate(xps, axis=1)
        assert upg.shape[1] == no
        # the oracle lists the subdomains' particles in the same order
        assert max_rel(upg, upo) < 1e-13 and np.array_equal(xpg, xpo)
    finally:
        release(hp + hc)


def test_cuboid_global_routing():
    """ppm_map_part_global's routing on a 2 x 2 x 2 cut: every particle goes
    to the subdomain whose box contains it."""
    from test_halo_boxes import sub_of
    rng = np.random.default_rng(4)
    t = topo_for(3, 12, decomp=(2, 2, 2))
    hs = sub_handles(t)
    try:
        x = random_particles(rng, 3, 20000)
        x[:, :50] = 1.5  # outside the domain: in no subdomain
        own = np.full(x.shape[1], t.nsubs)
        own[50:] = sub_of(t, x[:, 50:])
        from ppm_legacy_b200 import mapping
        info, perm, counts = mapping.device_route_global(hs[0].topo_id, 1, dev_f(x), t.nsubs)
        assert info == 0, ppmg.last_error()
        perm = perm.cpu().numpy()
        start = 0
        for c in range(t.nsubs + 1):
            got = perm[start:start + counts[c]]
            assert np.array_equal(got, np.flatnonzero(own == c)), c
            start += counts[c]
    finally:
        release(hs)


@pytest.mark.parametrize("decomp,dtype,tol,entry", [
    ((2, 2, 2), np.float64, 1e-12, "dev"), ((2, 1, 3), np.float64, 1e-12, "host"),
    ((1, 2, 2), np.float32, 1e-5, "dev"), ((3, 2, 1), np.float64, 1e-12, "dev")])
def test_cuboid_poisson_matches_oracle(decomp, dtype, tol, entry):
    """The FFT Poisson solver on a cut along several axes (omega to virtual
    z-slabs, the slab form there, phi back to every subdomain's whole box):
    every subdomain ends with the oracle's solution on the whole domain at
    its real nodes, ghost nodes and periodic images."""
    rng = np.random.default_rng(170 + sum(decomp))
    nc = (24, 16, 20)
    lo, hi = [0.0, -1.0, 0.5], [1.5, 0.0, 2.5]
    t = topo_for(3, list(nc), lo, hi, decomp=decomp)
    g = (2, 1, 2)
    lda = 2
    U = rng.standard_normal((lda,) + nc)
    phi = O.poisson(U.astype(dtype).astype(np.float64), [hi[a] - lo[a] for a in range(3)])
    hs = sub_handles(t, halo.ThreadMover(timeout=120))
    try:
        fields, idx = {}, {}
        for s in range(t.nsubs):
            n = nodes(t, s)
            cut = [n[a] != nc[a] + 1 for a in range(3)]
            # global 0-based unique index of every local node 1-g .. n+g
            idx[s] = [((int(t.istart[s, a]) - 1 if cut[a] else 0)
                       + np.arange(1 - g[a], n[a] + g[a] + 1) - 1) % nc[a] for a in range(3)]
            F = np.full(shape_of(t, s, g, lda), 7.0, order="F")
            # omega at the real nodes 1..n (the solver reads the unique ones), junk elsewhere
            re = tuple(slice(g[a], g[a] + n[a]) for a in range(3))
            F[(slice(None),) + re + (0,)] = U[np.ix_(range(lda), *[idx[s][a][g[a]:g[a] + n[a]]
                                                                 for a in range(3)])]
            F = F.astype(dtype)
            fields[s] = dev_f(F) if entry == "dev" else np.asfortranarray(F)

        def solve(s):
            info = ppmg.ppm_fdsolver_poisson(fields[s], lda, hs[s].topo_id, 1, list(g))
            return info if info or entry != "dev" else ppmg.sync_status(hs[s].topo_id, 1)
        assert in_threads(solve, t.nsubs) == [0] * t.nsubs, ppmg.last_error()
        for s in range(t.nsubs):
            want = phi[np.ix_(range(lda), *idx[s])]
            got = host(fields[s])[..., 0].astype(np.float64)
            assert max_rel(got, want) < tol, (s, max_rel(got, want))
    finally:
        release(hs)


def test_cuboid_refusals():
    """A cut with more subdomains than y or z cells refuses the FFT solver
    (errno 503), as does a non-cartesian decomposition at registration."""
    t = topo_for(3, 12, decomp=(4, 4, 1))
    hs = sub_handles(t, halo.ThreadMover(timeout=30))
    try:
        f = np.zeros(shape_of(t, 0, (1, 1, 1), 1), order="F")
        info = ppmg.ppm_fdsolver_poisson(f, 1, hs[0].topo_id, 1, [1, 1, 1])
        assert info == -2 and ppmg.last_error()[1] == 503
    finally:
        release(hs)
    bad = topo_for(3, 12, decomp=(2, 2, 1))
    bad.istart = bad.istart.copy()
    bad.istart[1, 0] += 1  # one interval shifted: no longer cartesian
    bad.nnodes = bad.nnodes.copy()
    bad.nnodes[1, 0] -= 1
    _next_id[0] += 1
    bad.topo_id = _next_id[0]
    assert ppmg.register(bad, isub=0) != 0
    assert "cartesian" in ppmg.last_error()[2] or "cover" in ppmg.last_error()[2]
    ppmg.unregister(bad)


@pytest.mark.parametrize("decomp,far", [((2, 2, 2), 0), ((4, 2, 1), 9)])
def test_cuboid_partial_mapping(decomp, far):
    """ppm_map_part_partial on a cut along several axes: the device routing
    over the neighbour list equals the rule restated on CPU, every subdomain
    ends with exactly its particles (kept ones, then the arrivals by
    ascending source), and particles beyond the neighbours give 405."""
    from ppm_legacy_b200 import mapping
    from test_map_cuboid import check, make_before, partial_rule
    t = topo_for(3, 12, decomp=decomp)
    hs = sub_handles(t)
    try:
        before = make_before(t, 3000, far)
        for s, ts in enumerate(hs):
            info, perm, cnt = mapping.device_route_partial(ts.topo_id, 1, dev_f(before[s][0]),
                                                           t.nsubs)
            errno = ppmg.last_error()[1]  # before the next library call clears it
            cls = partial_rule(t, s, before[s][0])
            want = np.concatenate([np.flatnonzero(cls == c) for c in range(t.nsubs + 1)])
            assert np.array_equal(perm.cpu().numpy()[:len(want)], want), s
            assert cnt == [int((cls == c).sum()) for c in range(t.nsubs + 1)]
            assert info == (-2 if (cls == t.nsubs).any() else 0)
            if info:
                assert errno == 405
        parts = {s: (ts.topo_id, 1, dev_f(before[s][0]),
                     [dev_f(before[s][1]), dev_f(before[s][2])]) for s, ts in enumerate(hs)}
        info, res = mapping.map_subs(parts, t, halo.LocalComm())
        after = {s: (host(x), host(p[0]), host(p[1])) for s, (x, p) in res.items()}
        check(t, before, after)
        assert info == (-2 if far else 0)
    finally:
        release(hs)
