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


def interior_mask(xp, nc, lo=0.0, hi=1.0):
    """Particles whose M'4 support stays inside one periodic image of the box:
    stencil origin xi = (x - lo) / h in [1, nc - 2) on every axis, so the
    nodes i0-1 .. i0+2 never wrap.  Moments 1 and 2 of the deposited field
    equal the particles' only for these (the node coordinate of a wrapped
    node is a period away from the particle)."""
    h = (hi - lo) / nc
    xi = (np.asarray(xp)[:3] - lo) / h
    return np.all((xi >= 1.0) & (xi < nc - 2.0), axis=0)


def mesh_moments(U, h, lo=0.0):
    """sum_n x_n^k f_n over the unique nodes U(lda, nx, ny, nz) for k = 0, 1, 2
    and every axis: array [k, axis, component] (k = 0 repeated per axis)."""
    U = np.asarray(U, dtype=np.float64)
    lda = U.shape[0]
    out = np.zeros((3, 3, lda))
    for d in range(3):
        other = tuple(a + 1 for a in range(3) if a != d)
        s = U.sum(axis=other)  # (lda, n_d)
        x = lo + np.arange(U.shape[1 + d]) * h
        for k in range(3):
            out[k, d] = s @ (x ** k)
    return out


def particle_moments(xp, up):
    """sum_p x_p^k u_p and sum_p |x_p^k u_p|: arrays [k, axis, component]."""
    xp = np.asarray(xp, dtype=np.float64)[:3]
    up = np.asarray(up, dtype=np.float64)
    up = up if up.ndim == 2 else up[None]
    lda = up.shape[0]
    val = np.zeros((3, 3, lda))
    mag = np.zeros((3, 3, lda))
    for d in range(3):
        for k in range(3):
            xk = xp[d] ** k
            val[k, d] = up @ xk
            mag[k, d] = np.abs(up) @ np.abs(xk)
    return val, mag


def moment_errors(U, h, xp, up, lo=0.0):
    """Relative conservation error of moments 0, 1, 2 (max over axes and
    components): |sum_n x^k f - sum_p x^k u| / sum_p |x^k u|."""
    m = mesh_moments(U, h, lo)
    v, a = particle_moments(xp, up)
    rel = np.abs(m - v) / np.where(a > 0, a, 1.0)
    return [float(rel[k].max()) for k in range(3)]


class PairOrderComm:
    """Every subdomain in this process, subdomain s on rank s, matched the way
    NCCL matches point-to-point messages: the k-th send one rank posts to
    another meets the k-th receive that rank posts from it, tags not
    compared.  Each subdomain posts in the order DistComm.posting_order
    gives, so a plan whose sides list their messages in different orders
    fails here (shape mismatch or wrong values) as it would over NCCL."""

    def __init__(self):
        from ppm_legacy_b200 import halo
        self.order = halo.DistComm()

    def exchange(self, sends, recvs):
        import collections
        by_src = collections.defaultdict(list)
        for i, m in enumerate(sends):
            by_src[m[0]].append(i)
        queues = collections.defaultdict(collections.deque)
        for src, idx in by_src.items():
            mine = [sends[i] for i in idx]
            so, _ = self.order.posting_order(mine, [])
            for k in so:
                queues[(src, mine[k][1])].append(mine[k][3])
        by_dst = collections.defaultdict(list)
        for i, r in enumerate(recvs):
            by_dst[r[0]].append(i)
        out = [None] * len(recvs)
        for dst, idx in by_dst.items():
            mine = [recvs[i] for i in idx]
            _, ro = self.order.posting_order([], mine)
            for k in ro:
                src, like = mine[k][1], mine[k][3]
                blk = queues[(src, dst)].popleft()
                if blk.shape != like.shape:
                    raise ValueError("messages paired out of order (block shapes differ)")
                out[idx[k]] = blk.clone()
        return out
