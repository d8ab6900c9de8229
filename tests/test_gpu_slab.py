"""3D P2M and M2P on z-slab subdomains (ppmg_mesh_set_local_sub) against the
oracle's multi-subdomain routines, on one GPU: every slab is a handle of its
own in this process and the ghost exchange between them runs in-process
(halo.LocalComm, the same block arithmetic that DistComm sends between
ranks)."""
import copy

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import halo
from _util import max_rel, random_particles, topo_for
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [7000]


def slab_handles(t):
    """One handle per slab (topo ids of their own), local sub = the slab."""
    out = []
    for s in range(t.nsubs):
        _next_id[0] += 1
        ts = copy.deepcopy(t)
        ts.topo_id = _next_id[0]
        assert ppmg.register(ts, isub=s) == 0, ppmg.last_error()
        out.append(ts)
    return out


def dev_f(a):
    d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
    return d.permute(*reversed(range(d.dim())))


def host(a):
    return a.permute(*reversed(range(a.dim()))).contiguous().cpu().numpy().T


def run(nc, nslab, kernel, g, lda, mode, seed, n=None):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    n = n or 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    gg = [g] * 3
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    hs = slab_handles(t)
    ppmg.set_precision(mode)
    lb = [1 - g] * 3
    fields = {}
    for s, ts in enumerate(hs):
        nz = int(t.nnodes[s, 2]) - 1
        shape = (lda, nc + 1 + 2 * g, nc + 1 + 2 * g, nz + 1 + 2 * g, 1)
        f = dev_f(np.full(shape, 9.0))
        xs = dev_f(xp[:, ids[s]])
        us = dev_f(up[:, ids[s]])
        assert ppmg.ppm_interp_p2m(xs, len(ids[s]), us, lda, ts.topo_id, 1, kernel, gg, f,
                                   exchange=False) == 0, ppmg.last_error()
        fields[s] = f
    halo.put(fields, t, gg, lb, halo.LocalComm())
    fo, lbo, ubo = O.p2m(t, xp, up, kernel, gg)
    tol = 1e-13 if mode == 0 else 1e-6
    for s in range(nslab):
        nz = int(t.nnodes[s, 2]) - 1
        got = host(fields[s])
        real = (slice(None),) + tuple(slice(g, g + nc + 1) for _ in range(2)) + (slice(g, g + nz + 1), 0)
        ref = fo[(slice(None),) + tuple(slice(1 - lbo[a], 1 - lbo[a] + nc + 1) for a in range(2))
                 + (slice(1 - lbo[2], 1 - lbo[2] + nz + 1), s)]
        assert max_rel(got[real], ref) < tol, (s, max_rel(got[real], ref))
    # M2P: ghost get between the slabs, then every slab gathers its particles
    halo.get(fields, t, gg, lb, halo.LocalComm())
    O.ghost_get(t, fo, lbo, ubo, gg)
    ref = O.m2p(t, xp, fo, lbo, ubo, lda, kernel, gg)
    for s, ts in enumerate(hs):
        out = dev_f(np.zeros((lda, len(ids[s]))))
        assert ppmg.ppm_interp_m2p(dev_f(xp[:, ids[s]]), len(ids[s]), out, lda, ts.topo_id, 1,
                                   kernel, gg, fields[s]) == 0, ppmg.last_error()
        assert ppmg.sync_status(ts.topo_id, 1) == 0, ppmg.last_error()
        got = host(out)
        mt = 1e-14 if mode == 0 else 1e-6
        assert max_rel(got, ref[:, ids[s]]) <= mt, (s, max_rel(got, ref[:, ids[s]]))
    ppmg.set_precision(0)
    for ts in hs:
        ppmg.unregister(ts)


@pytest.mark.parametrize("nc,nslab,kernel,g,lda", [
    (16, 2, 2, 2, 3), (12, 3, 2, 2, 1), (16, 4, 1, 1, 2), (12, 2, 2, 3, 5), (13, 3, 2, 2, 3)])
def test_slab_p2m_put_get_m2p_match_oracle(nc, nslab, kernel, g, lda):
    run(nc, nslab, kernel, g, lda, 0, seed=nc * nslab + kernel)


def test_slab_mixed_precision_within_tolerance():
    run(24, 3, 2, 2, 3, 1, seed=5)


def test_slab_particles_on_the_slab_faces():
    """Particles on the planes between slabs and one ulp below them (the
    stencil origin may round up to the slab's top face)."""
    rng = np.random.default_rng(11)
    nc, nslab = 12, 3
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    faces = np.unique(np.concatenate([t.min_sub[:, 2], t.max_sub[:, 2]]))
    faces = faces[faces < 1.0]
    below = np.nextafter(faces[1:], 0.0)
    z = np.concatenate([faces, below])
    n = z.size * 20
    xp = random_particles(rng, 3, n)
    xp[2] = np.repeat(z, 20)
    up = np.asfortranarray(rng.standard_normal((2, n)))
    gg = [2, 2, 2]
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    hs = slab_handles(t)
    fields = {}
    for s, ts in enumerate(hs):
        nz = int(t.nnodes[s, 2]) - 1
        f = dev_f(np.zeros((2, nc + 5, nc + 5, nz + 5, 1)))
        assert ppmg.ppm_interp_p2m(dev_f(xp[:, ids[s]]), len(ids[s]), dev_f(up[:, ids[s]]), 2,
                                   ts.topo_id, 1, 2, gg, f, exchange=False) == 0
        fields[s] = f
    halo.put(fields, t, gg, [-1, -1, -1], halo.LocalComm())
    fo, lbo, _ = O.p2m(t, xp, up, 2, gg)
    for s in range(nslab):
        nz = int(t.nnodes[s, 2]) - 1
        got = host(fields[s])[:, 2:nc + 3, 2:nc + 3, 2:nz + 3, 0]
        ref = fo[:, 1 - lbo[0]:2 - lbo[0] + nc, 1 - lbo[1]:2 - lbo[1] + nc,
                 1 - lbo[2]:2 - lbo[2] + nz, s]
        assert max_rel(got, ref) < 1e-13
    for ts in hs:
        ppmg.unregister(ts)


def test_slab_particle_outside_its_slab_is_unassigned():
    t = topo_for(3, 12, decomp=(1, 1, 2))
    hs = slab_handles(t)
    xp = dev_f(np.array([[0.5], [0.5], [0.75]]))  # in slab 1, given to slab 0
    f = dev_f(np.zeros((1, 17, 17, 11, 1)))
    ppmg.ppm_interp_p2m(xp, 1, dev_f(np.ones((1, 1))), 1, hs[0].topo_id, 1, 2, [2, 2, 2], f,
                        exchange=False)
    info = ppmg.sync_status(hs[0].topo_id, 1)
    assert info == -1 and ppmg.last_error()[1] == 405
    for ts in hs:
        ppmg.unregister(ts)


def test_slab_handle_refuses_other_routines():
    """Without a transport the C-ABI ghost mapping leaves the exchange between
    slabs to the host; cartesian decompositions are accepted, others not."""
    import ctypes as C
    from ppm_legacy_b200._lib import int_array
    t = topo_for(3, 12, decomp=(1, 1, 2))
    hs = slab_handles(t)
    F = np.zeros((1, 17, 17, 11, 1), order="F")
    info = C.c_int(0)
    ppmg.lib().ppmg_map_field_ghost_d(F.ctypes.data, 1, 1, int_array([-1] * 3, C.c_int64),
                                      int_array([15, 15, 9], C.c_int64), hs[0].topo_id, 1,
                                      int_array([2, 2, 2]), 5, C.byref(info))
    assert info.value == -2 and "subdomain of several" in ppmg.last_error()[2]
    t2 = topo_for(3, 12, decomp=(2, 1, 1), topo_id=7900)
    ppmg.register(t2)
    import ctypes as C
    info = C.c_int(0)
    ppmg.lib().ppmg_mesh_set_local_sub(7900, 1, 0, C.byref(info))
    assert info.value == 0, ppmg.last_error()
    ppmg.unregister(t2)
    t3 = topo_for(3, 12, decomp=(2, 1, 1), topo_id=7901)
    t3.nnodes = t3.nnodes.copy()
    t3.istart = t3.istart.copy()
    t3.nnodes[0, 0] -= 1  # the intervals no longer meet: not a cartesian cut
    ppmg.register(t3)
    ppmg.lib().ppmg_mesh_set_local_sub(7901, 1, 0, C.byref(info))
    assert info.value == -2 and "cartesian" in ppmg.last_error()[2]
    ppmg.unregister(t3)
    for ts in hs:
        ppmg.unregister(ts)


@pytest.mark.parametrize("nslab,kernel,lda,nc", [(2, 2, 3, 12), (3, 1, 1, 12), (3, 2, 2, 13)])
def test_slab_remeshing_chain_matches_oracle(nslab, kernel, lda, nc):
    """comp_weights, remesh (+ ghost put between the slabs) and create_part on
    every slab against the oracle's multi-subdomain remeshing: weights bit for
    bit, the field to summation order, the new particles slab by slab in the
    reference's order (the shared upper plane of a slab creates none)."""
    rng = np.random.default_rng(200 + nslab + nc)
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    n = 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    g = [2, 2, 2] if kernel == 2 else [1, 1, 1]
    ks = 2 if kernel == 2 else 1
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    wo, lsto, sio = O.comp_weights(t, xp, kernel)
    fo, lbo, ubo = O.remesh(t, xp, up, kernel, g, wo, lsto, sio)
    cut = [0.2, 1e300]
    no, upo, xpo, _ = O.create_part(t, fo, lbo, ubo, cut)
    hs = slab_handles(t)
    fields, wxs = {}, {}
    lb = [1 - g[0]] * 3
    for s, ts in enumerate(hs):
        ns = len(ids[s])
        xs = np.asfortranarray(xp[:, ids[s]])
        wx = [np.zeros((2 * ks, 1, ns + 2 * ks), order="F") for _ in range(3)]
        assert ppmg.ppm_rmsh_comp_weights(xs, ns, ts.topo_id, 1, kernel, *wx) == 0, \
            ppmg.last_error()
        for a in range(3):
            assert np.array_equal(wx[a][:, 0, :], wo[a][:, s, :ns + 2 * ks])
        nz = int(t.nnodes[s, 2]) - 1
        f = dev_f(np.full((lda, nc + 1 + 2 * g[0], nc + 1 + 2 * g[0], nz + 1 + 2 * g[0], 1), 5.0))
        assert ppmg.ppm_rmsh_remesh(dev_f(xs), ns, dev_f(up[:, ids[s]]), lda, ts.topo_id, 1,
                                    kernel, g, f, exchange=False) == 0, ppmg.last_error()
        fields[s] = f
    halo.put(fields, t, g, lb, halo.LocalComm())
    ups, xps = [], []
    for s, ts in enumerate(hs):
        nz = int(t.nnodes[s, 2]) - 1
        got = host(fields[s])[(slice(None),) + (slice(g[0], g[0] + nc + 1),) * 2 +
                              (slice(g[0], g[0] + nz + 1), 0)]
        ref = fo[(slice(None),) + tuple(slice(1 - lbo[a], 2 - lbo[a] + nc) for a in range(2)) +
                 (slice(1 - lbo[2], 2 - lbo[2] + nz), s)]
        assert max_rel(got, ref) < 1e-13
        info, ns, upn, xpn, _ = ppmg.ppm_rmsh_create_part(fields[s], ts.topo_id, 1, cut, lda=lda,
                                                          resetpos=True, ghostsize=g)
        assert info == 0, ppmg.last_error()
        ups.append(host(upn).reshape(lda, -1))
        xps.append(host(xpn))
    upg, xpg = np.concatenate(ups, axis=1), np.concatenate(xps, axis=1)
    assert upg.shape[1] == no
    assert max_rel(upg, upo) < 1e-13 and np.array_equal(xpg, xpo)
    for ts in hs:
        ppmg.unregister(ts)


@pytest.mark.parametrize("nslab,far", [(3, 0), (2, 0), (4, 5)])
def test_particle_redistribution_on_gpu(nslab, far):
    """ppm_map_part_partial's routing and packing kernels on every slab, the
    blocks exchanged in-process: each slab ends with exactly the particles it
    contains (kept ones first, then arrivals from below, then from above),
    their properties intact; particles two slabs away are reported (405) and
    dropped."""
    from ppm_legacy_b200 import mapping
    from test_slab_exchange import check_mapping, moved_particles, route_rule
    t = topo_for(3, 12, decomp=(1, 1, nslab))
    hs = slab_handles(t)
    before, parts = {}, {}
    for s, ts in enumerate(hs):
        rng = np.random.default_rng(600 + s)
        x = moved_particles(t, s, 5000, rng, far=far)
        ids = np.arange(s * 100000, s * 100000 + 5000, dtype=np.int64)[None, :]
        u = np.asfortranarray(rng.standard_normal((3, 5000)))
        before[s] = (x, ids, u)
        parts[s] = (ts.topo_id, 1, dev_f(x), [dev_f(ids), dev_f(u)])
    info, res = mapping.map_subs(parts, t, halo.LocalComm())
    after = {s: (host(x2), host(p2[0]), host(p2[1])) for s, (x2, p2) in res.items()}
    if far:
        assert info == -2
        for s in before:  # the far particles are dropped before the check
            keep = route_rule(t, s, before[s][0]) < 3
            before[s] = tuple(np.asfortranarray(a[:, keep]) for a in before[s])
    else:
        assert info == 0, ppmg.last_error()
    check_mapping(t, before, after)
    assert sum(a[0].shape[1] for a in after.values()) == sum(b[0].shape[1]
                                                             for b in before.values())
    for ts in hs:
        ppmg.unregister(ts)


@pytest.mark.parametrize("nslab,kernel", [(3, 2), (2, 1)])
def test_slab_adjoint_matches_global_oracle(nslab, kernel):
    """The P2M adjoint on every slab (r's z ghost planes by the ghost get
    between the slabs) equals the oracle's adjoint over the whole domain."""
    rng = np.random.default_rng(700 + nslab)
    nc, lda = 12, 2
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    t1 = topo_for(3, nc)
    n = 3000
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    R = rng.standard_normal((lda, nc, nc, nc))
    dwo, dxo = O.p2m_adjoint(t1, xp, up, np.asfortranarray(R[..., None]), [1, 1, 1], [nc] * 3,
                             kernel)
    lst, si = O.assign(t, xp)
    ids = np.split(lst, np.cumsum(si)[:-1])
    hs = slab_handles(t)
    g = 2
    rs = {}
    for s in range(nslab):
        z0 = int(t.istart[s, 2]) - 1
        nz = int(t.nnodes[s, 2]) - 1
        zi = (z0 + np.arange(1 - g, nz + 2 + g) - 1) % nc
        loc = np.array(R[:, :, :, zi])
        loc[:, :, :, :g] = 0.0          # ghost planes: from the neighbours
        loc[:, :, :, nz + 1 + g:] = 0.0
        rs[s] = dev_f(loc[..., None])
    halo.get(rs, t, [0, 0, g], [1, 1, 1 - g], halo.LocalComm())
    for s, ts in enumerate(hs):
        m = len(ids[s])
        dw = dev_f(np.zeros((lda, m)))
        dx = dev_f(np.zeros((3, m)))
        assert ppmg.ppm_interp_p2m_adjoint(dev_f(xp[:, ids[s]]), m, dev_f(up[:, ids[s]]), lda,
                                           ts.topo_id, 1, kernel, rs[s], dw, dx,
                                           field_lb=[1, 1, 1 - g], exchange=False) == 0
        assert ppmg.sync_status(ts.topo_id, 1) == 0, ppmg.last_error()
        assert max_rel(host(dw), dwo[:, ids[s]]) < 1e-12
        assert max_rel(host(dx), dxo[:, ids[s]]) < 1e-11
    for ts in hs:
        ppmg.unregister(ts)
