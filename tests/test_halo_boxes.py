"""The exchange of a cartesian decomposition (cuts along x, y and z) as the
library plans it (ppmg_halo_plan_boxes, the blocks of
ppm_map_field_ghost_init.f:234-447 for every neighbour and periodic shift),
applied here in numpy on CPU.

Each subdomain's field is built as the library's P2M on that subdomain leaves
it: the deposit of the subdomain's own particles (the oracle's periodic
deposit of those particles alone) over its ghost-extended box, whose nodes
are distinct modulo the mesh on every cut axis (so that the periodic view
equals the open deposit).  After the put every subdomain's real nodes must
hold the deposit of all particles; after the get its whole box must."""
import numpy as np
import pytest

from _util import random_particles, topo_for, unique_view
from oracle import oracle as O
from ppm_legacy_b200 import halo


def sub_of(t, xp):
    """0-based subdomain of every particle (closed-lower / open-upper boxes)."""
    own = np.full(xp.shape[1], -1)
    for s in range(t.nsubs):
        inside = np.ones(xp.shape[1], bool)
        for a in range(3):
            inside &= (xp[a] >= t.min_sub[s, a]) & (xp[a] < t.max_sub[s, a])
        own[inside & (own < 0)] = s
    assert (own >= 0).all()
    return own


def local_box(t, s, g):
    """Global 1-based node indices of the local nodes 1-g .. (last)+g per axis."""
    out = []
    for a in range(3):
        cut = int(t.nnodes[s, a]) != int(t.Nm[a])
        n = int(t.nnodes[s, a]) if cut else int(t.Nm[a])
        off = int(t.istart[s, a]) - 1 if cut else 0
        out.append(off + np.arange(1 - g[a], n + g[a] + 1))
    return out


def view(U, t, s, g):
    """The periodic values U(lda, Nc, Nc, Nc) at the local box of subdomain s."""
    idx = [(b - 1) % U.shape[1 + a] for a, b in enumerate(local_box(t, s, g))]
    return np.ascontiguousarray(U[np.ix_(range(U.shape[0]), *idx)])


def case(nc, decomp, kernel, g, lda, seed):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=decomp)
    t1 = topo_for(3, nc)
    n = 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    own = sub_of(t, xp)
    fa, lba, _ = O.p2m(t1, xp, up, kernel, [1, 1, 1])
    Ua = unique_view(fa, lba, [nc] * 3, 3)
    local, want = {}, {}
    for s in range(t.nsubs):
        sel = own == s
        fs, lbs, _ = O.p2m(t1, np.asfortranarray(xp[:, sel]), np.asfortranarray(up[:, sel]),
                           kernel, [1, 1, 1])
        local[s] = view(unique_view(fs, lbs, [nc] * 3, 3), t, s, g)
        want[s] = view(Ua, t, s, g)
    return t, local, want


def sl(lo, hi, g):
    """numpy slices of local nodes lo..hi (1-based) in an array whose first
    node is 1-g."""
    return (slice(None),) + tuple(slice(lo[a] - (1 - g[a]), hi[a] - (1 - g[a]) + 1)
                                  for a in range(3))


def apply(t, fields, g, put):
    """Every subdomain packs its sends, then applies its receives in order."""
    plans = {s: halo.plan_boxes(t, s, g, put) for s in fields}
    wire = {}
    for s, p in plans.items():
        for peer, tag, lo, hi in p["send"]:
            key = (s, peer, tag)
            assert key not in wire, key  # a tag names one block per pair
            wire[key] = fields[s][sl(lo, hi, g)].copy()
    for s, p in plans.items():
        for peer, tag, lo, hi in p["recv"]:
            blk = wire.pop((peer, s, tag))
            dst = fields[s][sl(lo, hi, g)]
            assert dst.shape == blk.shape, (s, peer, tag)
            if put:
                fields[s][sl(lo, hi, g)] = dst + blk
            else:
                fields[s][sl(lo, hi, g)] = blk
    assert not wire, sorted(wire)  # every send has its receive


def real(t, s, g):
    cut = [int(t.nnodes[s, a]) != int(t.Nm[a]) for a in range(3)]
    lo = [1 if cut[a] else 1 - g[a] for a in range(3)]
    hi = [int(t.nnodes[s, a]) if cut[a] else int(t.Nm[a]) + g[a] for a in range(3)]
    return sl(lo, hi, g)


@pytest.mark.parametrize("nc,decomp,kernel,g,lda", [
    (12, (2, 2, 2), 2, (2, 2, 2), 2),
    (12, (2, 2, 1), 2, (1, 2, 3), 1),
    (12, (1, 2, 2), 1, (1, 1, 1), 3),
    (12, (3, 2, 2), 2, (2, 1, 2), 1),
    (12, (2, 1, 3), 2, (1, 3, 2), 1),
    (12, (1, 1, 3), 2, (2, 2, 2), 1),
    (12, (4, 1, 1), 2, (2, 1, 1), 1)])
def test_put_then_get(nc, decomp, kernel, g, lda):
    t, local, want = case(nc, decomp, kernel, g, lda, seed=sum(decomp) + nc)
    scale = max(np.abs(w).max() for w in want.values())
    apply(t, local, g, put=True)
    for s in local:
        r = real(t, s, g)
        assert np.abs(local[s][r] - want[s][r]).max() <= 1e-13 * scale, s
    apply(t, local, g, put=False)
    for s in local:
        assert np.abs(local[s] - want[s]).max() <= 1e-13 * scale, s


def test_get_never_writes_real_nodes():
    t = topo_for(3, 12, decomp=(2, 2, 2))
    g = (2, 2, 2)
    for s in range(t.nsubs):
        for _, _, lo, hi in halo.plan_boxes(t, s, g, put=False)["recv"]:
            inside = all(lo[a] >= 1 and hi[a] <= int(t.nnodes[s, a]) for a in range(3))
            assert not inside
            # a box lies outside the real box along at least one axis
            assert any(hi[a] < 1 or lo[a] > int(t.nnodes[s, a]) for a in range(3))


def test_plan_is_refused_for_bad_geometry():
    t = topo_for(3, 12, decomp=(2, 2, 2))
    with pytest.raises(ValueError):
        halo.plan_boxes(t, 0, (7, 1, 1), put=True)  # wider than a subdomain
    bad = topo_for(3, 12, decomp=(2, 2, 2))
    bad.nnodes = bad.nnodes.copy()
    bad.nnodes[0, 0] = int(bad.Nm[0])  # spans x while the others are cut
    with pytest.raises(ValueError):
        halo.plan_boxes(bad, 1, (1, 1, 1), put=True)
