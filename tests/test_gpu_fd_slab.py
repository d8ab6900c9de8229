"""The FFT Poisson solver on z-slab subdomains (the slab form of
ppm_fdsolver_solve, ppm_fdsolver_solve_3d.f:18-21: xy transforms on every
slab, an all-to-all to z pencils, the z transforms and the spectral step,
and back), through the halo transport registered on each slab handle.
Every slab's call runs on a host thread of its own (halo.ThreadMover); each
slab must end with the oracle's solution on the whole domain at its real
nodes and at every image of its ghost box."""
import copy
import threading

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import halo
from _util import max_rel, periodic_fill, topo_for
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_next_id = [9700]


def slab_handles(t, mover):
    out = []
    for s in range(t.nsubs):
        _next_id[0] += 1
        ts = copy.deepcopy(t)
        ts.topo_id = _next_id[0]
        assert ppmg.register(ts, isub=s) == 0, ppmg.last_error()
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


@pytest.mark.parametrize("nslab,dtype,tol,entry", [
    (2, np.float64, 1e-12, "dev"), (3, np.float64, 1e-12, "host"), (3, np.float32, 1e-5, "dev"),
    (4, np.float64, 1e-12, "dev")])
def test_slab_poisson_matches_oracle(nslab, dtype, tol, entry):
    rng = np.random.default_rng(160 + nslab)
    nc = (24, 16, 20)
    lo, hi = [0.0, -1.0, 0.5], [1.5, 0.0, 2.5]
    t = topo_for(3, list(nc), lo, hi, decomp=(1, 1, nslab))
    g = [2, 1, 2]
    lda = 2
    U = rng.standard_normal((lda,) + nc)
    phi = O.poisson(U.astype(dtype).astype(np.float64), [hi[a] - lo[a] for a in range(3)])
    hs = slab_handles(t, halo.ThreadMover(timeout=60))
    fields = {}
    for s in range(nslab):
        z0 = int(t.istart[s, 2]) - 1
        nz = int(t.nnodes[s, 2]) - 1
        lb = [1 - g[0], 1 - g[1], 1 - g[2]]
        ub = [nc[0] + 1 + g[0], nc[1] + 1 + g[1], nz + 1 + g[2]]
        # omega on the slab's real planes 1..nz (the solver reads those), junk elsewhere
        F = np.full((lda,) + tuple(ub[a] - lb[a] + 1 for a in range(3)) + (1,), 7.0, order="F")
        xi = (np.arange(lb[0], ub[0] + 1) - 1) % nc[0]
        yi = (np.arange(lb[1], ub[1] + 1) - 1) % nc[1]
        zi = z0 + np.arange(nz)
        F[:, :, :, 1 - lb[2]:1 - lb[2] + nz, 0] = U[np.ix_(range(lda), xi, yi, zi)]
        F = F.astype(dtype)
        fields[s] = dev_f(F) if entry == "dev" else np.asfortranarray(F)
    res = [None] * nslab

    def solve(s):
        res[s] = ppmg.ppm_fdsolver_poisson(fields[s], lda, hs[s].topo_id, 1, g)
        if res[s] == 0 and entry == "dev":
            res[s] = ppmg.sync_status(hs[s].topo_id, 1)
    th = [threading.Thread(target=solve, args=(s,)) for s in range(nslab)]
    for x in th:
        x.start()
    for x in th:
        x.join(timeout=120)
    assert res == [0] * nslab, ppmg.last_error()
    for s in range(nslab):
        z0 = int(t.istart[s, 2]) - 1
        nz = int(t.nnodes[s, 2]) - 1
        lb = [1 - g[0], 1 - g[1], 1 - g[2]]
        ub = [nc[0] + 1 + g[0], nc[1] + 1 + g[1], nz + 1 + g[2]]
        # phi at every position of the slab's box: x, y images, z ghost planes
        xi = (np.arange(lb[0], ub[0] + 1) - 1) % nc[0]
        yi = (np.arange(lb[1], ub[1] + 1) - 1) % nc[1]
        zi = (z0 + np.arange(lb[2], ub[2] + 1) - 1) % nc[2]
        want = phi[np.ix_(range(lda), xi, yi, zi)]
        got = host(fields[s])[..., 0].astype(np.float64)
        assert max_rel(got, want) < tol, (s, max_rel(got, want))
