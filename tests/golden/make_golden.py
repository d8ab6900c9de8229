"""Generate the golden vectors in tests/golden/golden.json.

The reference (PPM) ships no tests or fixtures and cannot be compiled here
(no Fortran compiler), so these vectors come from the kernel definitions
evaluated in exact rational arithmetic (``fractions.Fraction``), applied to the
stencil coordinate xi exactly as the reference rounds it in floating point:

  * M'4:  W(s) = 1 - 5/2 s^2 + 3/2 |s|^3 (|s| < 1), 1/2 (2-|s|)^2 (1-|s|)
          (1 <= |s| < 2), 0 otherwise  (ppm_interp_p2m.f:839-853)
  * bsp2: W(s) = 1 - |s| (|s| < 1)      (ppm_interp_p2m.f:3057-3110)
  * xi = fl((x - min) * dxi) with dxi = fl(1 / fl(len / Nc)) in FP64 for P2M
    and the FP32 mesh spacing for M2P (ppm_interp_m2p.f:221-222, 486-489)
  * periodic mesh: node n and node n + Nc are the same point.

Cell ranking vectors restate ppm_util_rank3d.f:353-533 in plain Python.
Run: python tests/golden/make_golden.py  (deterministic, seed 1234)
"""
from __future__ import annotations

import json
import math
import os
from fractions import Fraction as Fr

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def w_mp4(s: Fr) -> Fr:
    a = abs(s)
    if a < 1:
        return 1 - Fr(5, 2) * a * a + Fr(3, 2) * a ** 3
    if a < 2:
        return Fr(1, 2) * (2 - a) ** 2 * (1 - a)
    return Fr(0)


def w_bsp2(s: Fr) -> Fr:
    a = abs(s)
    return 1 - a if a < 1 else Fr(0)


def dxi_fp64(lo, hi, nc):
    return 1.0 / ((hi - lo) / float(nc))


def dxi_fp32_quirk(lo, hi, nc):
    ln = np.float32(hi - lo)
    dx = np.float32(np.float64(ln) / np.float64(nc))
    return float(np.float32(1.0 / np.float64(dx)))


def stencil(xi: float, kernel: int):
    """(nodes, weights) exactly; nodes are 0-based unwrapped node indices."""
    x = Fr(xi)
    i0 = math.floor(xi)
    if kernel == 2:
        nodes = [i0 - 1, i0, i0 + 1, i0 + 2]
        return nodes, [w_mp4(x - n) for n in nodes]
    nodes = [i0, i0 + 1]
    return nodes, [w_bsp2(x - n) for n in nodes]


def p2m_exact(xp, up, lo, hi, nc, kernel):
    dim, npart = xp.shape
    lda = up.shape[0]
    dxi = [dxi_fp64(lo[a], hi[a], nc[a]) for a in range(dim)]
    field = {}
    for p in range(npart):
        st = []
        for a in range(dim):
            xi = (xp[a, p] - lo[a]) * dxi[a]
            st.append(stencil(xi, kernel))
        for idx in np.ndindex(*([len(st[0][0])] * dim)):
            node = tuple(st[a][0][idx[a]] % nc[a] for a in range(dim))
            w = Fr(1)
            for a in range(dim):
                w *= st[a][1][idx[a]]
            for c in range(lda):
                field[(c,) + node] = field.get((c,) + node, Fr(0)) + w * Fr(up[c, p])
    out = np.zeros((lda,) + tuple(nc[:dim]))
    for k, v in field.items():
        out[k] = float(v)
    return out


def m2p_exact(xp, F, lo, hi, nc, kernel, quirk=True):
    dim, npart = xp.shape
    lda = F.shape[0]
    dxi = [dxi_fp32_quirk(lo[a], hi[a], nc[a]) if quirk else dxi_fp64(lo[a], hi[a], nc[a])
           for a in range(dim)]
    out = np.zeros((lda, npart))
    for p in range(npart):
        st = []
        for a in range(dim):
            xi = (xp[a, p] - lo[a]) * dxi[a]
            st.append(stencil(xi, kernel))
        for c in range(lda):
            acc = Fr(0)
            for idx in np.ndindex(*([len(st[0][0])] * dim)):
                node = tuple(st[a][0][idx[a]] % nc[a] for a in range(dim))
                w = Fr(1)
                for a in range(dim):
                    w *= st[a][1][idx[a]]
                acc += w * Fr(F[(c,) + node])
            out[c, p] = float(acc)
    return out


def rank_py(xp, xmin, xmax, Nm, Ngl, single=False):
    """Plain restatement of ppm_util_rank{2,3}d (1-based lpdx, lhbx); single:
    the _s variant, every operation rounded to FP32 (numpy float32 scalars)."""
    dim, npart = xp.shape
    Nt = [Nm[a] + Ngl[a] + Ngl[dim + a] for a in range(dim)]
    nbox = int(np.prod(Nt))
    if single:
        f = np.float32
        xp = xp.astype(np.float32)
        xmin = [f(v) for v in xmin]
        xmax = [f(v) for v in xmax]
        rd = [f(Nm[a]) / (xmax[a] - xmin[a]) for a in range(dim)]
    else:
        rd = [Nm[a] / (xmax[a] - xmin[a]) for a in range(dim)]
    pbox = []
    for p in range(npart):
        c = []
        for a in range(dim):
            i = math.floor((xp[a, p] - xmin[a]) * rd[a]) + Ngl[a]
            if xp[a, p] >= xmax[a] and i < Nm[a] + Ngl[a]:
                i = Nm[a] + Ngl[a]
            c.append(i)
        for a in range(dim):
            if xp[a, p] < xmax[a] and c[a] >= Nm[a] + Ngl[a]:
                c[a] = Nm[a] + Ngl[a] - 1
        if all(0 <= c[a] < Nt[a] for a in range(dim)):
            b = c[0] + 1 + c[1] * Nt[0] + (c[2] * Nt[0] * Nt[1] if dim == 3 else 0)
        else:
            b = -1
        pbox.append(b)
    cnt = [0] * nbox
    for b in pbox:
        if b > 0:
            cnt[b - 1] += 1
    lhbx = [1]
    for b in range(nbox):
        lhbx.append(lhbx[-1] + cnt[b])
    cur = lhbx[:-1].copy()
    lpdx = [0] * sum(cnt)
    for p, b in enumerate(pbox):
        if b > 0:
            lpdx[cur[b - 1] - 1] = p + 1
            cur[b - 1] += 1
    return lpdx, lhbx


def main():
    rng = np.random.default_rng(1234)
    cases = []

    def add_p2m(name, dim, nc, lo, hi, npart, lda, kernel):
        xp = np.empty((dim, npart))
        for a in range(dim):
            xp[a] = lo[a] + rng.random(npart) * (hi[a] - lo[a])
            xp[a] = np.minimum(xp[a], np.nextafter(hi[a], lo[a]))
        up = rng.standard_normal((lda, npart))
        f = p2m_exact(xp, up, lo, hi, nc, kernel)
        cases.append(dict(kind="p2m", name=name, dim=dim, nc=list(nc[:dim]), lo=list(lo[:dim]),
                          hi=list(hi[:dim]), kernel=kernel, lda=lda, xp=xp.T.tolist(),
                          up=up.T.tolist(), field=f.reshape(lda, -1, order="F").tolist()))

    def add_m2p(name, dim, nc, lo, hi, npart, lda, kernel):
        xp = np.empty((dim, npart))
        for a in range(dim):
            xp[a] = lo[a] + rng.random(npart) * (hi[a] - lo[a])
            xp[a] = np.minimum(xp[a], np.nextafter(hi[a], lo[a]))
        F = rng.standard_normal((lda,) + tuple(nc[:dim]))
        up = m2p_exact(xp, F, lo, hi, nc, kernel)
        cases.append(dict(kind="m2p", name=name, dim=dim, nc=list(nc[:dim]), lo=list(lo[:dim]),
                          hi=list(hi[:dim]), kernel=kernel, lda=lda, xp=xp.T.tolist(),
                          F=F.reshape(lda, -1, order="F").tolist(), up=up.T.tolist()))

    add_p2m("p2m_3d_mp4_n8", 3, [8, 8, 8], [0.0] * 3, [1.0] * 3, 40, 3, 2)
    add_p2m("p2m_3d_mp4_n6_box1p3", 3, [6, 7, 5], [0.0, -0.5, 0.25], [1.3, 0.5, 1.0], 30, 2, 2)
    add_p2m("p2m_3d_bsp2_n8", 3, [8, 8, 8], [0.0] * 3, [1.0] * 3, 40, 1, 1)
    add_p2m("p2m_2d_mp4_n16", 2, [16, 16], [0.0] * 2, [1.0] * 2, 60, 1, 2)
    add_p2m("p2m_2d_mp4_n10_box", 2, [10, 12], [0.0, 0.0], [2.0, 1.5], 50, 2, 2)
    add_m2p("m2p_3d_mp4_n8", 3, [8, 8, 8], [0.0] * 3, [1.0] * 3, 40, 3, 2)
    add_m2p("m2p_3d_mp4_n6_box1p3", 3, [6, 7, 5], [0.0, -0.5, 0.25], [1.3, 0.5, 1.0], 30, 2, 2)
    add_m2p("m2p_3d_bsp2_n8", 3, [8, 8, 8], [0.0] * 3, [1.0] * 3, 40, 1, 1)
    add_m2p("m2p_2d_mp4_n16", 2, [16, 16], [0.0] * 2, [1.0] * 2, 60, 1, 2)
    add_m2p("m2p_2d_bsp2_n10", 2, [10, 12], [0.0, 0.0], [2.0, 1.5], 50, 2, 1)

    # a particle exactly on a node deposits a delta there (M'4 interpolates)
    xp = np.array([[3.0 / 8.0], [5.0 / 8.0], [1.0 / 8.0]])
    up = np.array([[2.5]])
    f = p2m_exact(xp, up, [0.0] * 3, [1.0] * 3, [8, 8, 8], 2)
    cases.append(dict(kind="p2m", name="p2m_on_node_delta", dim=3, nc=[8, 8, 8], lo=[0.0] * 3,
                      hi=[1.0] * 3, kernel=2, lda=1, xp=xp.T.tolist(), up=up.T.tolist(),
                      field=f.reshape(1, -1, order="F").tolist()))

    # cell ranking (with particles on and beyond the upper boundary)
    for dim in (2, 3):
        npart = 200
        xmin = [0.0] * dim
        xmax = [1.0] * dim
        xp = rng.random((dim, npart))
        xp[:, :5] = 1.0                        # exactly on xmax: corrected into a ghost cell
        xp[:, 5:10] = np.nextafter(1.0, 0.0)   # just below xmax
        xp[0, 10:15] = 1.2                     # outside the extended mesh
        xp[:, 15:20] = -0.05                   # lower ghost layer
        Nm = [5] * dim
        Ngl = [1] * (2 * dim)
        lpdx, lhbx = rank_py(xp, xmin, xmax, Nm, Ngl)
        cases.append(dict(kind="rank", name=f"rank{dim}d", dim=dim, xmin=xmin, xmax=xmax, Nm=Nm,
                          Ngl=Ngl, xp=xp.T.tolist(), lpdx=lpdx, lhbx=lhbx))

    # single-precision ranking (ppm_util_rank{2,3}d_s) on a box whose FP32
    # cell spacing rounds: particles on the FP32 cell faces, one ulp either
    # side of them, on and beyond the upper face, in the lower ghost layer
    for dim in (2, 3):
        npart = 240
        xmin = [0.1, -0.3, 0.25][:dim]
        xmax = [0.7, 0.9, 1.0][:dim]
        Nm = [7, 9, 6][:dim]
        Ngl = [1] * (2 * dim)
        f32 = np.float32
        xp = (np.array(xmin)[:, None] + rng.random((dim, npart)) *
              (np.array(xmax) - np.array(xmin))[:, None]).astype(np.float32)
        for a in range(dim):
            h = (f32(xmax[a]) - f32(xmin[a])) / f32(Nm[a])
            faces = np.array([f32(xmin[a]) + f32(k) * h for k in range(Nm[a] + 1)], np.float32)
            sel = faces[rng.integers(0, Nm[a] + 1, 60)]
            xp[a, :60] = sel
            xp[a, 60:90] = np.nextafter(sel[:30], np.float32(np.inf))
            xp[a, 90:120] = np.nextafter(sel[30:], np.float32(-np.inf))
        xp[:, 120:125] = np.array(xmax, np.float32)[:, None]
        xp[0, 125:130] = np.float32(xmax[0] + 0.5)
        xp[:, 130:135] = (np.array(xmin) - 0.01).astype(np.float32)[:, None]
        lpdx, lhbx = rank_py(xp, xmin, xmax, Nm, Ngl, single=True)
        cases.append(dict(kind="rank", name=f"rank{dim}d_s", prec="s", dim=dim, xmin=xmin,
                          xmax=xmax, Nm=Nm, Ngl=Ngl, xp=xp.astype(np.float64).T.tolist(),
                          lpdx=lpdx, lhbx=lhbx))

    with open(OUT, "w") as fh:
        json.dump(dict(generator="tests/golden/make_golden.py", seed=1234, cases=cases), fh,
                  separators=(",", ":"))
    print(OUT, len(cases), "cases")


if __name__ == "__main__":
    main()
