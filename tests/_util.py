"""Shared helpers of the test-suite (geometry, periodic layouts, metrics)."""
from __future__ import annotations

import json
import os

import numpy as np

from ppm_legacy_b200 import topo as T

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")


def golden_cases(kind=None):
    with open(GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    return [c for c in cases if kind is None or c["kind"] == kind]


def topo_for(dim, nc, lo=None, hi=None, decomp=None, topo_id=1, mesh_id=1):
    return T.cartesian(dim, nc, decomp=decomp, min_phys=lo, max_phys=hi, topo_id=topo_id,
                       mesh_id=mesh_id)


def box_bounds(topo, ghost):
    lb = [1 - int(ghost[a]) for a in range(topo.dim)]
    ub = [int(topo.Nm[a]) + int(ghost[a]) for a in range(topo.dim)]
    return lb, ub


def unique_view(field, lb, nc, dim, sub=0):
    """Real unique nodes 1..Nc of field(lda, lb:..., nsub) as (lda, nc...)."""
    sl = (slice(None),) + tuple(slice(1 - lb[a], 1 - lb[a] + nc[a]) for a in range(dim)) + (sub,)
    return field[sl]


def periodic_fill(U, lb, ub, dim):
    """Expand unique-node values U(lda, Nc...) to a consistent periodic box."""
    lda = U.shape[0]
    nc = U.shape[1:]
    idx = [(np.arange(lb[a], ub[a] + 1) - 1) % nc[a] for a in range(dim)]
    F = U[np.ix_(range(lda), *idx)]
    return np.asfortranarray(F[..., None])


def random_particles(rng, dim, n, lo=0.0, hi=1.0):
    lo = np.resize(np.asarray(lo, dtype=np.float64), dim)
    hi = np.resize(np.asarray(hi, dtype=np.float64), dim)
    xp = lo[:, None] + rng.random((dim, n)) * (hi - lo)[:, None]
    xp = np.minimum(xp, np.nextafter(hi, lo)[:, None])
    return np.asfortranarray(xp)


def jittered_particles(rng, dim, nc, jitter=0.25):
    """One particle per cell at the centre + U[-jitter h, jitter h] (cell order)."""
    grids = np.meshgrid(*[np.arange(nc) for _ in range(dim)], indexing="ij")
    cells = np.stack([g.reshape(-1, order="F") for g in grids])  # x fastest
    h = 1.0 / nc
    xp = (cells + 0.5) * h + rng.uniform(-jitter * h, jitter * h, cells.shape)
    return np.asfortranarray(xp % 1.0)


def max_rel(a, ref):
    """max |a - ref| / max |ref| (normwise max relative error)."""
    den = np.abs(ref).max()
    return float(np.abs(a - ref).max() / (den if den > 0 else 1.0))


def rms_rel(a, ref):
    den = np.sqrt((ref ** 2).sum())
    return float(np.sqrt(((a - ref) ** 2).sum()) / (den if den > 0 else 1.0))
