"""The device routing of ppm_map_part_global (ppmg_map_part_global_route_*)
against its restatement on CPU, and the whole global mapping on slabs held
in one process (device routing and packing, the exchange in-process)."""
import copy

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import halo, mapping
from _util import topo_for
from test_map_global import check, global_rule, make_before

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [9300]


def slab_handles(t):
    out = []
    for s in range(t.nsubs):
        _next_id[0] += 1
        ts = copy.deepcopy(t)
        ts.topo_id = _next_id[0]
        assert ppmg.register(ts, isub=s) == 0, ppmg.last_error()
        out.append(ts)
    return out


def dev_f(a, dtype=torch.float64):
    d = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).to("cuda", dtype)
    return d.permute(*reversed(range(d.dim())))


@pytest.mark.parametrize("nslab,n,dtype", [(4, 20000, torch.float64), (3, 9001, torch.float32),
                                           (2, 70000, torch.float64)])
def test_device_route_equals_the_rule(nslab, n, dtype):
    t = topo_for(3, 16, decomp=(1, 1, nslab))
    hs = slab_handles(t)
    rng = np.random.default_rng(nslab + n)
    x = rng.random((3, n)) * 1.2 - 0.1  # some outside the domain
    xd = dev_f(x, dtype)
    xr = xd.cpu().double().numpy()  # the positions in their own precision
    cls = global_rule(t, xr)
    info, perm, cnt = mapping.device_route_global(hs[1].topo_id, 1, xd, nslab)
    assert ppmg.sync_status(hs[1].topo_id, 1) == 0
    assert info == 0
    assert cnt == [int((cls == c).sum()) for c in range(nslab + 1)]
    want = np.concatenate([np.nonzero(cls == c)[0] for c in range(nslab + 1)])
    assert np.array_equal(perm.cpu().numpy()[:n], want)


def test_global_mapping_on_slabs_in_one_process():
    t = topo_for(3, 12, decomp=(1, 1, 4))
    hs = slab_handles(t)
    before = make_before(t, 4, n=5000)
    parts = {s: (hs[s].topo_id, 1, dev_f(x), [dev_f(i), dev_f(u)])
             for s, (x, i, u) in before.items()}
    info, res = mapping.map_global(parts, t, halo.LocalComm())
    assert info == 0
    got = {s: (x.cpu().numpy(), i.cpu().numpy().astype(np.int64), u.cpu().numpy())
           for s, (x, (i, u)) in res.items()}
    check(t, before, got)
