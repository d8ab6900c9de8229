"""Benchmark: particles/s of the 3D M'4 P2M + M2P round trip on B200.

One step = ppm_interp_p2m then ppm_interp_m2p over the whole particle set
(lda = 3, periodic unit cube, ghostsize 2), through the library's
device-pointer C-ABI entry points with inputs resident in HBM (`value`), and
through the host-pointer entry points with host<->device copies inside the
timed region (`e2e`).  Default workload: 512^3 mesh, 134,217,728 particles
(50% uniform + 4 Gaussian blobs, sigma 0.05, lda 3 ~ N(0,1)), mixed
precision (FP64 offsets, FP32 weights, compensated FP32 sums); the plain FP64
form is measured on the same data and reported beside it.

`--impl reference` times the reference algorithm's CPU path (the C++
restatement of the Fortran loops, one thread per subdomain as `mpirun -np P`
would run it) on a bounded sample of the same workload.

Multi-GPU (torchrun): weak scaling by domain decomposition.  N ranks own the
N z-slabs of a 512 x 512 x 512N periodic mesh (one 512^3 slab and its own
134M particles per GPU); a step is the local P2M with the ghost put between
neighbouring slabs (NCCL point-to-point, ppm_legacy_b200.halo), the ghost
get, and the local M2P; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

CONFIGS = {
    # name: (mesh cells per axis, particles, distribution)
    "512": (512, 134_217_728, "clustered"),
    "256": (256, 16_777_216, "clustered"),
    "128": (128, 2_097_152, "jittered"),
}


L2_BYTES = 126 * 2**20  # B200 L2


class L2Flush:
    """Writes a buffer twice the L2 size between timed steps (outside their
    events) when a workload's inputs are smaller than the L2."""

    def __init__(self, torch, device):
        self.buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)

    def __call__(self):
        self.buf.fill_(1.0)


def hbm_peak():
    try:
        with open(PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def alg_bytes(np_, nc, lda=3, dim=3, b=8):
    """Compulsory bytes of one P2M + M2P round trip at the API precision:
    xp read twice, up read (P2M) and written (M2P), the unique field nodes
    written once and read once."""
    return np_ * (2 * dim * 8 + 2 * lda * b) + (nc ** dim) * lda * 2 * b


def max_over_ranks(x, dist=None, device=None):
    """Max of a per-rank scalar over all ranks of the default process group
    (every rank receives it); the value itself without a group."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(x)
    import torch
    if dist.get_backend() != "nccl":
        device = "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def kernel_bytes(np_, nc, lda, g, mixed):
    """Algorithmic bytes of one launch of each timed part (FP64 field and
    strengths at the API, records in the compute precision):
    p2m_gather: sorted records + strength chunks read, the written node box
      (Nm + 2g)^3 x lda x 8 (real nodes and every periodic image);
    m2p_gather: the unique nodes read once, records and particle ids read,
      up(lda, Np) written;
    cell_sort: xp and up read, key, id, record and strengths written, the
      cell offsets (Nc^3 + 1) written."""
    v = 16 if mixed else 32
    chunks = (lda + 3) // 4
    box = (nc + 1 + 2 * g) ** 3
    return {
        "p2m_gather": np_ * v * (1 + chunks) + box * lda * 8,
        "m2p_gather": nc ** 3 * lda * 8 + np_ * (v + 4 + lda * 8),
        "cell_sort": np_ * (3 * 8 + lda * 8) + np_ * (8 + v * (1 + chunks)) + (nc ** 3 + 1) * 4,
    }


def measured_traffic(kernel, np_):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary (profiles/dram_traffic.json), scaled to np_ particles; None when
    that kernel has no capture."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as fh:
            d = json.load(fh)[kernel]
        return d["bytes_per_launch"] * np_ / d["particles"]
    except Exception:
        return None


def _mesh_moments(torch, U, h):
    """sum_n x_n^k f_n over the unique nodes U(lda, nx, ny, nz) (FP64), for
    k = 0, 1, 2 and every axis: tensor [k, axis, component]."""
    lda = U.shape[0]
    out = torch.zeros((3, 3, lda), dtype=torch.float64, device=U.device)
    for d in range(3):
        s = U.sum(dim=[a + 1 for a in range(3) if a != d])  # (lda, n_d)
        x = torch.arange(U.shape[1 + d], dtype=torch.float64, device=U.device) * h
        for k in range(3):
            out[k, d] = s @ x ** k
    return out


def _particle_moments(torch, xp, up):
    """sum_p x_p^k u_p and sum_p |x_p^k u_p|: tensors [k, axis, component]."""
    lda = up.shape[0]
    val = torch.zeros((3, 3, lda), dtype=torch.float64, device=up.device)
    mag = torch.zeros_like(val)
    au = up.abs()
    for d in range(3):
        xd = xp[d]
        for k in range(3):
            xk = xd ** k
            val[k, d] = up @ xk
            mag[k, d] = au @ xk.abs()
    return val, mag


def moment_errors(torch, U, h, xp, up):
    """Relative conservation error of moments 0, 1, 2 (max over axes and
    components): |sum_n x^k f - sum_p x^k u| / sum_p |x^k u|."""
    m = _mesh_moments(torch, U, h)
    v, a = _particle_moments(torch, xp, up)
    rel = (m - v).abs() / torch.where(a > 0, a, torch.ones_like(a))
    return [float(rel[k].max()) for k in range(3)]


def rel_errors(torch, a, ref):
    """Normwise max and RMS relative error of a against ref."""
    d = a - ref
    den_max = float(ref.abs().max())
    den_rms = float(torch.linalg.vector_norm(ref))
    return (float(d.abs().max()) / (den_max or 1.0),
            float(torch.linalg.vector_norm(d)) / (den_rms or 1.0))


def slab_topology(ppmg, nc, world, topo_id=1, mesh_id=1):
    """The weak-scaling domain: world z-slabs of nc^3 cells, cubic cells of
    size 1/nc, periodic; slab r covers z in [r, r+1)."""
    return ppmg.cartesian(3, [nc, nc, nc * world], decomp=(1, 1, world),
                          min_phys=[0.0, 0.0, 0.0], max_phys=[1.0, 1.0, float(world)],
                          topo_id=topo_id, mesh_id=mesh_id)


def shift_to_slab(torch, xp, rank):
    """Move positions from [0,1)^3 into slab `rank` (z in [rank, rank+1)); a
    z that rounds up to the slab's top face goes to its bottom face."""
    if rank == 0:
        return xp
    z = xp[2] + float(rank)
    xp[2] = torch.where(z >= float(rank + 1), torch.full_like(z, float(rank)), z)
    return xp


def gen_particles(torch, cfg, device, seed):
    nc, n, dist = CONFIGS[cfg]
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if dist == "jittered":
        idx = torch.arange(n, device=device, dtype=torch.int64)
        cells = torch.stack([idx % nc, (idx // nc) % nc, idx // (nc * nc)]).to(torch.float64)
        h = 1.0 / nc
        jit = (torch.rand((3, n), generator=g, device=device, dtype=torch.float64) - 0.5) * 0.5 * h
        xp = torch.remainder((cells + 0.5) * h + jit, 1.0)
    else:
        nu = n // 2
        nb = (n - nu) // 4
        parts = [torch.rand((3, nu), generator=g, device=device, dtype=torch.float64)]
        centres = 0.2 + 0.6 * torch.rand((4, 3), generator=g, device=device, dtype=torch.float64)
        for b in range(4):
            m = nb if b < 3 else n - nu - 3 * nb
            z = torch.randn((3, m), generator=g, device=device, dtype=torch.float64)
            parts.append(torch.remainder(centres[b][:, None] + 0.05 * z, 1.0))
        xp = torch.cat(parts, dim=1)
    # positions in [0, 1): remainder can round up to exactly 1.0
    xp = torch.where(xp >= 1.0, torch.zeros_like(xp), xp)
    up = torch.randn((3, n), generator=g, device=device, dtype=torch.float64)
    # column-major (Fortran) layout: shape (3, n), strides (1, 3)
    return xp.t().contiguous().t(), up.t().contiguous().t(), nc, n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_baseline(args, seconds_hint=False):
    """The reference algorithm on the host cores: P threads, one subdomain each
    (cartesian split), on a bounded sample of the workload (config at 1/8 of the
    volume: same density and distribution), round trip per step."""
    from oracle import oracle as O
    from ppm_legacy_b200 import topo as T

    cores = os.cpu_count() or 1
    sample = {"512": "256", "256": "128", "128": "128"}[args.config]
    nc, n, dist = CONFIGS[sample]
    rng = np.random.default_rng(7)
    if dist == "jittered":
        idx = np.arange(n)
        cells = np.stack([idx % nc, (idx // nc) % nc, idx // (nc * nc)])
        h = 1.0 / nc
        xp = ((cells + 0.5) * h + rng.uniform(-0.25 * h, 0.25 * h, (3, n))) % 1.0
    else:
        nu = n // 2
        nb = (n - nu) // 4
        parts = [rng.random((3, nu))]
        centres = 0.2 + 0.6 * rng.random((4, 3))
        for b in range(4):
            m = nb if b < 3 else n - nu - 3 * nb
            parts.append((centres[b][:, None] + 0.05 * rng.standard_normal((3, m))) % 1.0)
        xp = np.concatenate(parts, axis=1)
    xp = np.asfortranarray(np.where(xp >= 1.0, 0.0, xp))
    up = np.asfortranarray(rng.standard_normal((3, n)))
    # factor the core count into a cartesian split of the box
    p = cores
    dec = [1, 1, 1]
    while p > 1:
        for f in (2, 3, 5, 7, 11, 13):
            if p % f == 0:
                break
        else:
            f = p
        a = dec.index(min(dec))
        dec[a] *= f
        p //= f
    t = T.cartesian(3, nc, decomp=tuple(dec))
    lst, si = O.assign(t, xp)
    own = np.empty(n, dtype=np.int32)
    own[lst] = np.repeat(np.arange(t.nsubs, dtype=np.int32), si)
    times = []
    steps = args.cpu_steps
    for i in range(args.cpu_warmup + steps):
        t0 = time.perf_counter()
        O.roundtrip_owned(t, xp, own, up, 2, [2, 2, 2], nthreads=cores)
        t1 = time.perf_counter()
        if i >= args.cpu_warmup:
            times.append(t1 - t0)
    best = min(times)
    return {"value": n / best, "unit": "particles/s", "cores": cores, "kind": "port",
            "sample": f"{sample}^3 mesh, {n} particles ({dist}, 1/8 of the benchmark volume at "
                      f"the same density), round trip P2M+ghost put/get+M2P, "
                      f"{t.nsubs} subdomains {tuple(dec)}, best of {steps}",
            "seconds_per_step": best}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    args.cpu_warmup = args.warmup
    args.cpu_steps = args.steps
    cb = cpu_baseline(args)
    nc, n, _ = CONFIGS[args.config]
    line = {
        "impl": "reference", "metric": "particles/s for 3D M'4 P2M+M2P round trip",
        "value": cb["value"], "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": cb["seconds_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"3D M'4 P2M+M2P, {nc}^3 periodic, {n} particles, lda 3",
                   "sample": cb["sample"]},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _cfg3_particles(nc, seed=3):
    """256^3 remesh workload: particles at cell centres displaced by 8 smooth
    Fourier modes (max displacement 0.5 h), vortex-tube strengths (lda 3)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / nc
    i = np.arange(nc, dtype=np.float64)
    X, Y, Z = np.meshgrid((i + 0.5) * h, (i + 0.5) * h, (i + 0.5) * h, indexing="ij")
    x = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")])
    del X, Y, Z
    d = np.zeros_like(x)
    amps = rng.random(8)
    amps *= 0.5 * h / amps.sum()
    for m in range(8):
        k = rng.integers(-4, 5, size=3)
        while np.abs(k).max() < 1:
            k = rng.integers(-4, 5, size=3)
        e = rng.standard_normal(3)
        e /= np.linalg.norm(e)
        ph = rng.uniform(0, 2 * np.pi)
        d += amps[m] * e[:, None] * np.sin(2 * np.pi * (k @ x) + ph)[None, :]
    xp = np.asfortranarray((x + d) % 1.0)
    xp[xp >= 1.0] = 0.0
    tp = 2 * np.pi
    up = np.asfortranarray(np.stack([
        np.sin(tp * xp[0]) * np.cos(tp * xp[1]) * np.cos(tp * xp[2]),
        np.cos(tp * xp[0]) * np.sin(tp * xp[1]) * np.cos(tp * xp[2]),
        -2 * np.cos(tp * xp[0]) * np.cos(tp * xp[1]) * np.sin(tp * xp[2])]))
    return xp, up


def cfg3_particles_dev(torch, nc, device, seed=3):
    """The 256^3 remesh workload generated on the device (the construction of
    _cfg3_particles with torch's seeded generator): cell centres displaced by
    8 Fourier modes (integer wavevectors, |k|_inf in [1, 4], random unit
    directions and phases, amplitudes summing to 0.5 h), vortex-tube
    strengths.  Returns column-major xp(3, n), up(3, n)."""
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    h = 1.0 / nc
    i = (torch.arange(nc, dtype=torch.float64, device=device) + 0.5) * h
    X = i[:, None, None].expand(nc, nc, nc)   # x slowest here; flattened in F order below
    Y = i[None, :, None].expand(nc, nc, nc)
    Z = i[None, None, :].expand(nc, nc, nc)
    # Fortran order of the node (x fastest): transpose to (z, y, x) then flatten
    x = torch.stack([X.permute(2, 1, 0).reshape(-1), Y.permute(2, 1, 0).reshape(-1),
                     Z.permute(2, 1, 0).reshape(-1)])
    d = torch.zeros_like(x)
    amps = torch.rand(8, generator=g, dtype=torch.float64)
    amps *= 0.5 * h / amps.sum()
    for m in range(8):
        k = torch.randint(-4, 5, (3,), generator=g)
        while int(k.abs().max()) < 1:
            k = torch.randint(-4, 5, (3,), generator=g)
        e = torch.randn(3, generator=g, dtype=torch.float64)
        e /= e.norm()
        ph = float(torch.rand(1, generator=g, dtype=torch.float64)) * 2 * np.pi
        kx = (k.to(torch.float64).to(device)[:, None] * x).sum(0)
        d += float(amps[m]) * e.to(device)[:, None] * torch.sin(2 * np.pi * kx + ph)[None, :]
    xp = torch.remainder(x + d, 1.0)
    xp = torch.where(xp >= 1.0, torch.zeros_like(xp), xp)
    tp = 2 * np.pi
    s, c = torch.sin(tp * xp), torch.cos(tp * xp)
    up = torch.stack([s[0] * c[1] * c[2], c[0] * s[1] * c[2], -2 * c[0] * c[1] * s[2]])
    return xp.t().contiguous().t(), up.t().contiguous().t()


def remesh_extra(torch, ppmg, dev, warmup, steps, peak):
    """One remeshing step on the 256^3 workload (comp_weights, remesh with
    M'4, lda 3, ghostsize 2, create_part with cutoff (1e-8, huge) on |u|_2 and
    resetpos) through the device entry points, timed with CUDA events; bytes
    per step: P2M's Np (24 + 24) + N^3 24, the create_part read N^3 24, the
    new particles' writes np_new (24 + 24)."""
    nc = 256
    xp, up = cfg3_particles_dev(torch, nc, dev)
    n = xp.shape[1]
    t = ppmg.cartesian(3, nc, topo_id=3, mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    g = [2, 2, 2]
    ext = nc + 1 + 2 * g[0]
    f = torch.zeros((1, ext, ext, ext, 3), device=dev, dtype=torch.float64).permute(4, 3, 2, 1, 0)
    cut = [1e-8, 1e300]
    stream = torch.cuda.current_stream()

    def step():
        assert ppmg.ppm_rmsh_comp_weights(xp, n, 3, 1, 2) == 0, ppmg.last_error()
        assert ppmg.ppm_rmsh_remesh(xp, n, up, 3, 3, 1, 2, g, f) == 0, ppmg.last_error()
        info, npn, _, _, _ = ppmg.ppm_rmsh_create_part(f, 3, 1, cut, lda=3, resetpos=True,
                                                       ghostsize=g)
        assert info == 0, ppmg.last_error()
        return npn

    for _ in range(max(warmup, 3)):
        npn = step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        npn = step()
    e1.record(stream)
    torch.cuda.synchronize()
    assert ppmg.sync_status(3, 1) == 0, ppmg.last_error()
    ppmg.unregister(t)
    ms = e0.elapsed_time(e1) / steps
    B = n * (24 + 24) + nc ** 3 * 24 + nc ** 3 * 24 + npn * (24 + 24)
    return {"workload": f"remesh: {nc}^3 periodic, {n} particles (cell centres + 8 smooth "
                        "modes, vortex-tube strengths), comp_weights + remesh + create_part",
            "ms_per_step": ms, "particles_per_s": n / (ms / 1e3), "new_particles": npn,
            "alg_bytes": B, "achieved_gbs": B / (ms / 1e3) / 1e9,
            "frac_of_hbm_roofline": B / (ms / 1e3) / 1e9 / peak, "steps": steps,
            "l2": "inputs larger than L2 (xp/up/field each > 126 MB)"}


def run_remesh(args):
    """One remeshing step on the 256^3 workload: ppm_rmsh_comp_weights +
    ppm_rmsh_remesh (M'4, lda 3, ghostsize 2) + ppm_rmsh_create_part (cutoff
    (1e-8, huge), |u|_2, resetpos).  `value`: device arrays through the `_dev`
    twins, CUDA-event time (the create_part count call synchronises once per
    step); `e2e`: the host-pointer entry points with copies, wall clock."""
    import torch
    import ppm_legacy_b200 as ppmg
    nc = 256
    dev = torch.device("cuda", 0)
    dx, du = cfg3_particles_dev(torch, nc, dev)
    xp = np.asfortranarray(dx.cpu().numpy())
    up = np.asfortranarray(du.cpu().numpy())
    n = xp.shape[1]
    t = ppmg.cartesian(3, nc, topo_id=3, mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    ppmg.set_precision(1 if args.precision != "fp64" else 0)
    g = [2, 2, 2]
    ext = nc + 1 + 2 * g[0]
    cut = [1e-8, 1e300]

    def step(x, u, f):
        assert ppmg.ppm_rmsh_comp_weights(x, n, 3, 1, 2) == 0, ppmg.last_error()
        assert ppmg.ppm_rmsh_remesh(x, n, u, 3, 3, 1, 2, g, f) == 0, ppmg.last_error()
        info, npn, _, _, _ = ppmg.ppm_rmsh_create_part(f, 3, 1, cut, lda=3, resetpos=True,
                                                       ghostsize=g)
        assert info == 0, ppmg.last_error()
        return npn

    df = torch.zeros((1, ext, ext, ext, 3), device=dev, dtype=torch.float64).permute(4, 3, 2, 1, 0)
    stream = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 1)):
        npn = step(dx, du, df)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        npn = step(dx, du, df)
    e1.record(stream)
    torch.cuda.synchronize()
    assert ppmg.sync_status(3, 1) == 0, ppmg.last_error()
    ms = e0.elapsed_time(e1) / args.steps
    field = np.zeros((3, ext, ext, ext, 1), order="F")
    step(xp, up, field)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step(xp, up, field)
        times.append(time.perf_counter() - t0)
    best = min(times)
    print(json.dumps({
        "workload": "remesh", "metric": "particles/s for one remeshing step",
        "value": n / (ms / 1e3), "unit": "particles/s", "ms_per_step": ms,
        "steps": args.steps, "warmup": max(args.warmup, 1), "higher_is_better": True,
        "dtype": "mixed" if args.precision != "fp64" else "f64",
        "config": {"mesh": f"{nc}^3 periodic", "particles": n, "lda": 3, "kernel": "M'4",
                   "ghostsize": 2, "new_particles": npn,
                   "data": "cell centres + 8 smooth modes (max 0.5 h), vortex-tube strengths",
                   "l2": "inputs larger than L2 (xp/up/field each > 126 MB)"},
        "path": "device arrays through the _dev twins (comp_weights, remesh, create_part)",
        "e2e": {"value": n / best, "unit": "particles/s", "ms_per_step": best * 1e3,
                "path": "host-pointer entry points, host<->device copies inside, wall clock"}}))


def run_adjoint(args):
    """128^3 adjoint workload: 4,194,304 uniform particles, lda 1, loss
    0.5 |P2M(x, w) - T|^2 with T ~ N(0, 1); one step = forward P2M, the
    residual on the device, the adjoint pass (dw, dx); device pointers."""
    import torch
    import ppm_legacy_b200 as ppmg
    dev = torch.device("cuda", 0)
    nc, n = 128, 4_194_304
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    xp = torch.rand((n, 3), generator=g, device=dev, dtype=torch.float64).t()
    w = torch.randn((n, 1), generator=g, device=dev, dtype=torch.float64).t()
    T = torch.randn((nc, nc, nc), generator=g, device=dev, dtype=torch.float64)
    t = ppmg.cartesian(3, nc, topo_id=4, mesh_id=1)
    assert ppmg.register(t) == 0, ppmg.last_error()
    ppmg.set_precision(1 if args.precision != "fp64" else 0)
    gh = [2, 2, 2]
    ext = nc + 1 + 4
    # column-major (Fortran) arrays: allocate the reversed shape, view it transposed
    field = torch.zeros((1, ext, ext, ext, 1), device=dev, dtype=torch.float64).permute(
        4, 3, 2, 1, 0)
    R = torch.empty((1, nc, nc, nc, 1), device=dev, dtype=torch.float64).permute(4, 3, 2, 1, 0)
    dw = torch.empty((n, 1), device=dev, dtype=torch.float64).t()
    dx = torch.empty((n, 3), device=dev, dtype=torch.float64).t()
    stream = torch.cuda.current_stream()

    def step():
        assert ppmg.ppm_interp_p2m(xp, n, w, 1, 4, 1, 2, gh, field) == 0
        R[0, :, :, :, 0] = field[0, 2:2 + nc, 2:2 + nc, 2:2 + nc, 0] - T
        assert ppmg.ppm_interp_p2m_adjoint(xp, n, w, 1, 4, 1, 2, R, dw, dx,
                                           field_lb=[1, 1, 1]) == 0

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    # the inputs (100 MB of positions, a 2 MB field) fit in the L2: flush it
    # between steps, outside each step's events
    flush = L2Flush(torch, dev)
    ms = 0.0
    for _ in range(args.steps):
        flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    assert ppmg.sync_status(4, 1) == 0, ppmg.last_error()
    ms /= args.steps
    print(json.dumps({
        "workload": "adjoint", "metric": "particles/s for forward P2M + adjoint (dL/dw, dL/dx)",
        "value": n / (ms / 1e3), "unit": "particles/s", "ms_per_step": ms,
        "steps": args.steps, "warmup": max(args.warmup, 3), "higher_is_better": True,
        "dtype": "mixed" if args.precision != "fp64" else "f64",
        "config": {"mesh": f"{nc}^3 periodic", "particles": n, "lda": 1,
                   "data": "uniform positions, w ~ N(0,1), target T ~ N(0,1) per node",
                   "l2": "L2 flushed between timed steps (outside the steps' events)"}}))


def launch_ranks(n):
    """Re-run this command as n ranks on this node (torch.distributed.run on
    127.0.0.1, a free port); returns the launcher's exit status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def launch_check(args):
    """Every rank joins the process group; rank 0 prints how many did."""
    import datetime

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    seen = 1
    if world > 1:
        if args.dist_backend == "nccl":
            local = int(os.environ.get("LOCAL_RANK", "0"))
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
            dev = torch.device("cuda", local)
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
            dev = "cpu"
        t = torch.ones(1, device=dev)
        dist.all_reduce(t)
        seen = int(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"launch_check": True, "n_gpus": world, "ranks_joined": seen,
                          "backend": args.dist_backend if world > 1 else None}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="512", choices=sorted(CONFIGS))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-warmup", type=int, default=0)
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the sorted-input round trip and the 256^3 remesh workload")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="N > 1: the process-group backend (gloo stages the slab exchange "
                         "through host memory)")
    ap.add_argument("--workload", default="roundtrip", choices=["roundtrip", "remesh", "adjoint"],
                    help="roundtrip: the metric (default); remesh / adjoint: the 256^3 remesh "
                         "and 128^3 adjoint workloads, one JSON line each")
    ap.add_argument("--launch-check", action="store_true",
                    help="start the ranks and the process group only (no GPU work) and print "
                         "one line with the number of ranks that joined")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: start the N ranks here through torch.distributed.run
        return launch_ranks(args.gpus)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but {world} ranks were started "
                         f"(WORLD_SIZE); launch with --nproc-per-node {args.gpus}")
    if args.launch_check:
        return launch_check(args)
    if args.workload == "remesh":
        return run_remesh(args)
    if args.workload == "adjoint":
        return run_adjoint(args)

    import torch
    import torch.distributed as dist

    import ppm_legacy_b200 as ppmg

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0")) % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        if args.dist_backend == "nccl":
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=dev)
        else:  # host-staged transport (validation of the multi-rank flow)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    xp, up, nc, n = gen_particles(torch, args.config, dev, seed=1000 + rank)
    if world > 1:
        # one z-slab per rank; P2M ends with the ghost put between the slabs
        t = slab_topology(ppmg, nc, world)
        xp = shift_to_slab(torch, xp, rank)
        assert ppmg.register(t, isub=rank) == 0, ppmg.last_error()
    else:
        t = ppmg.cartesian(3, nc, topo_id=1, mesh_id=1)
        assert ppmg.register(t) == 0, ppmg.last_error()
    g = [2, 2, 2]
    ext = nc + 1 + 2 * g[0]
    field = torch.empty((ext, ext, ext, 3), device=dev, dtype=torch.float64).permute(3, 2, 1, 0)
    field = field.unsqueeze(-1)
    out = torch.empty((n, 3), device=dev, dtype=torch.float64).t()
    stream = torch.cuda.current_stream()

    def kernel_time(part):
        """(total ms, launches) the library timed for a part since the last read."""
        import ctypes as C
        tot = C.c_double(0.0)
        cnt = C.c_int64(0)
        ppmg.lib().ppmg_kernel_timing_read(part, C.byref(tot), C.byref(cnt))
        return float(tot.value), int(cnt.value)

    get = ppmg.params.ppm_param_map_ghost_get

    def ghost_get(f):
        # the slabs' z ghost planes from the neighbours (M2P reads them)
        if world > 1 and ppmg.ppm_map_field_ghost(f, 3, 1, 1, g, get):
            raise RuntimeError(f"library error {ppmg.last_error()}")

    def step():
        i1 = ppmg.ppm_interp_p2m(xp, n, up, 3, 1, 1, 2, g, field)
        ghost_get(field)
        i2 = ppmg.ppm_interp_m2p(xp, n, out, 3, 1, 1, 2, g, field)
        if i1 or i2:
            raise RuntimeError(f"library error {ppmg.last_error()}")

    # inputs (positions, strengths, field) below the L2 size: flush between steps
    in_bytes = min(xp.numel() * 8, up.numel() * 8, field.numel() * 8)
    flush = L2Flush(torch, dev) if in_bytes < L2_BYTES else None
    l2_note = ("inputs larger than L2 (xp/up/field each > 126 MB)" if flush is None else
               "L2 flushed between timed steps (a 252 MB buffer written outside the steps' "
               "events); ms_per_step sums the steps' own events")

    def timed(prec):
        ppmg.set_precision(prec)
        for _ in range(args.warmup):
            step()
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for part in range(3):  # drop anything recorded before the timed region
            kernel_time(part)
        ppmg.lib().ppmg_kernel_timing(1)
        l0 = ppmg.lib().ppmg_launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        evp = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev0.record(stream)
        p2m_ms = []
        for k in range(args.steps):
            if flush is not None:
                flush()
            evp[0].record(stream)
            ppmg.ppm_interp_p2m(xp, n, up, 3, 1, 1, 2, g, field)
            evp[1].record(stream)
            ghost_get(field)
            ppmg.ppm_interp_m2p(xp, n, out, 3, 1, 1, 2, g, field)
            evp[2].record(stream)
            evp[2].synchronize()
            p2m_ms.append((evp[0].elapsed_time(evp[1]), evp[1].elapsed_time(evp[2])))
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = ppmg.lib().ppmg_launch_count() - l0
        ppmg.lib().ppmg_kernel_timing(0)
        kparts = [kernel_time(part) for part in range(3)]
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        if flush is None:
            ms = ev0.elapsed_time(ev1) / args.steps
        else:  # the steps' own events: the flushes between them are not timed
            ms = float(sum(a + b for a, b in p2m_ms)) / args.steps
        if world > 1:
            ms = max_over_ranks(ms, dist, dev)
            dist.barrier()
        p2m = float(np.median([a for a, _ in p2m_ms]))
        m2p = float(np.median([b for _, b in p2m_ms]))
        return ms, p2m, m2p, launches, kparts

    sampler = ClockSampler(local)
    sampler.start()
    res = {}
    snap = {}
    precs = {"both": [1, 0], "mixed": [1], "fp64": [0]}[args.precision]
    for prec in precs:
        res[prec] = timed(prec)
        if world == 1 and len(precs) == 2:
            # the last timed step's results of this form (accuracy block below)
            snap[prec] = (field[:, g[0]:g[0] + nc, g[1]:g[1] + nc, g[2]:g[2] + nc, 0].clone(),
                          out.clone())
    clocks = sampler.stop()

    accuracy = None
    if snap:
        # Mixed form against the plain FP64 form on the benchmark's own data
        # (the FP64 form matches the oracle to <= 1e-13 in the parity tests),
        # and conservation of moments 0, 1, 2 by both forms.  Moment 0 is taken
        # from the timed steps' fields over all particles; moments 1 and 2 per
        # axis from one more P2M per form of the particles whose support does
        # not wrap (stencil origin in [1, Nc-2) on every axis), since a wrapped
        # node sits a period away from its particle.
        h = 1.0 / nc
        pm, rm = rel_errors(torch, snap[1][0], snap[0][0])
        po, ro = rel_errors(torch, snap[1][1], snap[0][1])
        xi = xp * nc
        inner = torch.all((xi >= 1.0) & (xi < nc - 2.0), dim=0)
        up_in = (up.t() * inner[:, None]).t()  # column-major like up
        cons = {}
        for prec in (1, 0):
            e0 = moment_errors(torch, snap[prec][0], h, xp, up)[0]
            ppmg.set_precision(prec)
            if ppmg.ppm_interp_p2m(xp, n, up_in, 3, 1, 1, 2, g, field):
                raise RuntimeError(f"library error {ppmg.last_error()}")
            U = field[:, g[0]:g[0] + nc, g[1]:g[1] + nc, g[2]:g[2] + nc, 0]
            e = moment_errors(torch, U, h, xp, up_in)
            cons["mixed" if prec == 1 else "fp64"] = {"moment0": e0, "moment1": e[1],
                                                      "moment2": e[2]}
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        accuracy = {
            "data": f"the benchmark's {nc}^3 data ({n} {CONFIGS[args.config][2]} particles, "
                    f"lda 3), results of the last timed step of each form",
            "mixed_vs_fp64": {"p2m_max_rel": pm, "p2m_rms_rel": rm,
                              "m2p_max_rel": po, "m2p_rms_rel": ro},
            "conservation": cons,
            "moment_rule": ("|sum_n x_n^k f_n - sum_p x_p^k u_p| / sum_p |x_p^k u_p|, max over "
                            "axes and components; k = 0 over all particles, k = 1, 2 over the "
                            f"{int(inner.sum())} particles whose support does not wrap"),
            "targets": {"max_rel": 1e-6, "moments": 1e-10},
        }
        del snap, up_in, inner, xi

    peak, peak_src = hbm_peak()
    head = precs[0]
    ms, p2m_ms, m2p_ms, launches, kparts = res[head]
    total = n * world
    value = total / (ms / 1e3)
    B = alg_bytes(n, nc)
    # per-part algorithmic bytes per launch (see kernel_bytes) over the mean
    # CUDA-event duration of that part's launches in the timed region
    kb = kernel_bytes(n, nc, 3, 2, head == 1)
    names = ["p2m_gather", "m2p_gather", "cell_sort"]
    kinfo = {}
    for i, nm in enumerate(names):
        tms, cnt = kparts[i]
        if cnt == 0:
            continue
        avg = tms / cnt
        ach = kb[nm] / (avg / 1e3) / 1e9
        kinfo[nm] = {"launches": cnt, "ms_per_launch": avg, "alg_bytes": kb[nm],
                     "achieved_gbs": ach, "frac": ach / peak,
                     "share_of_step": tms / (ms * args.steps)}
    dom = max(kinfo, key=lambda k: kinfo[k]["ms_per_launch"] * kinfo[k]["launches"])
    traffic = measured_traffic(dom, n)
    roof = {"bound": "hbm", "achieved": kinfo[dom]["achieved_gbs"], "peak": peak,
            "unit": "GB/s", "frac": kinfo[dom]["frac"], "traffic": traffic,
            "kernel": dom, "alg_bytes_per_launch": kb[dom],
            "ms_per_launch": kinfo[dom]["ms_per_launch"],
            "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs, of measured)",
            "parts": kinfo,
            "step": {"alg_bytes": B, "achieved_gbs": B / (ms / 1e3) / 1e9,
                     "frac": B / (ms / 1e3) / 1e9 / peak}}
    parts = {}
    for prec in precs:
        m, a, b, _, _ = res[prec]
        nm = "mixed" if prec == 1 else "fp64"
        bp = n * 48 + nc ** 3 * 24
        bm = n * 48 + nc ** 3 * 24
        parts[nm] = {"ms_per_step": m, "particles_per_s": total / (m / 1e3),
                     "frac_of_hbm_roofline": (B / (m / 1e3) / 1e9) / peak,
                     "p2m_ms": a, "m2p_ms": b,
                     "p2m_frac": (bp / (a / 1e3) / 1e9) / peak,
                     "m2p_frac": (bm / (b / 1e3) / 1e9) / peak}

    adj = None
    # the adjoint keeps one periodic subdomain per GPU: single-GPU runs only
    if not args.no_adjoint and world == 1:
        # the adjoint pass of P2M at the same workload: dw = M2P(r), dx from the
        # kernel derivative, r ~ N(0, 1) on the unique nodes (device pointers)
        ppmg.set_precision(head)
        gr = torch.Generator(device=dev)
        gr.manual_seed(77)
        R = torch.randn((1, nc, nc, nc, 3), generator=gr, device=dev,
                        dtype=torch.float64).permute(4, 3, 2, 1, 0)
        dw = torch.empty((n, 3), device=dev, dtype=torch.float64).t()
        dx = torch.empty((n, 3), device=dev, dtype=torch.float64).t()

        # one step = the forward P2M and its adjoint (the adjoint reuses the
        # forward pass's cell order, as a training step would)
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

        def adj_step(timed=False):
            if timed:
                evs[0].record(stream)
            if ppmg.ppm_interp_p2m(xp, n, up, 3, 1, 1, 2, g, field):
                raise RuntimeError(f"library error {ppmg.last_error()}")
            if timed:
                evs[1].record(stream)
            if ppmg.ppm_interp_p2m_adjoint(xp, n, up, 3, 1, 1, 2, R, dw, dx, field_lb=[1, 1, 1]):
                raise RuntimeError(f"library error {ppmg.last_error()}")
            if timed:
                evs[2].record(stream)
                evs[2].synchronize()
                return evs[0].elapsed_time(evs[1]), evs[1].elapsed_time(evs[2])
            return None

        ksteps = min(args.steps, 5)
        for _ in range(3):
            adj_step()
        torch.cuda.synchronize()
        fw, bw = [], []
        for _ in range(ksteps):
            a, b = adj_step(True)
            fw.append(a)
            bw.append(b)
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        red = dist if world > 1 else None
        fms = max_over_ranks(float(np.median(fw)), red, dev)
        bms = max_over_ranks(float(np.median(bw)), red, dev)
        ab = n * (3 * 8 + 3 * 8 + 3 * 8 + 3 * 8) + nc ** 3 * 3 * 8
        adj = {"forward_p2m_ms": fms, "adjoint_ms": bms, "steps": ksteps,
               "particles_per_s": total / ((fms + bms) / 1e3),
               "adjoint_alg_bytes": ab, "adjoint_frac_of_hbm_roofline": ab / (bms / 1e3) / 1e9 / peak,
               "form": "mixed" if head == 1 else "fp64",
               "what": "forward ppmg_interp_p2m_dv_3d_dev, then ppmg_interp_p2m_adjoint_dv_3d_dev "
                       "(reuses the forward cell order; dw, dx gather with recomputed weights; "
                       "xp, up, r read, dw, dx written); medians of CUDA-event times"}
        del R, dw, dx

    e2e = None
    if not args.no_e2e:
        # host API with pinned host buffers: copies are inside the timed region
        ppmg.set_precision(head)
        hxp = xp.cpu().pin_memory()
        hup = up.cpu().pin_memory()
        hf = torch.empty(field.permute(4, 3, 2, 1, 0).shape, dtype=torch.float64).pin_memory()
        hf = hf.permute(4, 3, 2, 1, 0)
        hout = torch.empty((n, 3), dtype=torch.float64).pin_memory().t()
        nx, nu, nf, no = (x.numpy() for x in (hxp, hup, hf, hout))

        def e2e_step():
            i1 = ppmg.ppm_interp_p2m(nx, n, nu, 3, 1, 1, 2, g, nf)
            ghost_get(nf)
            i2 = ppmg.ppm_interp_m2p(nx, n, no, 3, 1, 1, 2, g, nf)
            if i1 or i2:
                raise RuntimeError(f"library error {ppmg.last_error()}")

        e2e_step()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        t1 = time.perf_counter()
        el = t1 - t0
        if world > 1:
            el = max_over_ranks(el, dist, dev)
        t1 = t0 + el
        fbytes = nf.nbytes
        h2d = nx.nbytes * 2 + nu.nbytes + fbytes
        d2h = fbytes + no.nbytes
        e2e = {"value": n * world / ((t1 - t0) / args.e2e_steps), "unit": "particles/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps,
               "path": "host-pointer C-ABI (ppmg_interp_p2m_dv_3d, ppmg_interp_m2p_dv_3d), "
                       "pinned host buffers"}

    extra = None
    if world == 1 and not args.no_extra:
        # (1) the same particles in cell order, as ppm_rmsh_create_part emits
        # them (or a caller that keeps its particles sorted): the sort's
        # gather reads and M2P's result rows become nearly sequential
        ppmg.set_precision(head)
        cells = torch.floor(xp * nc).to(torch.int64).clamp_(0, nc - 1)
        order = torch.argsort(cells[0] + nc * (cells[1] + nc * cells[2]), stable=True)
        del cells
        xs = xp[:, order].t().contiguous().t()
        us = up[:, order].t().contiguous().t()
        del order
        for _ in range(max(args.warmup, 3)):
            ppmg.ppm_interp_p2m(xs, n, us, 3, 1, 1, 2, g, field)
            ppmg.ppm_interp_m2p(xs, n, out, 3, 1, 1, 2, g, field)
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        torch.cuda.synchronize()
        for part in range(3):
            kernel_time(part)
        ppmg.lib().ppmg_kernel_timing(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ppmg.ppm_interp_p2m(xs, n, us, 3, 1, 1, 2, g, field)
            ppmg.ppm_interp_m2p(xs, n, out, 3, 1, 1, 2, g, field)
        e1.record(stream)
        torch.cuda.synchronize()
        ppmg.lib().ppmg_kernel_timing(0)
        sp = [kernel_time(part) for part in range(3)]
        assert ppmg.sync_status(1, 1) == 0, ppmg.last_error()
        sms = e0.elapsed_time(e1) / args.steps
        del xs, us
        sorted_in = {
            "workload": "the round trip above with the particles given in cell order",
            "ms_per_step": sms, "particles_per_s": n / (sms / 1e3),
            "frac_of_hbm_roofline": B / (sms / 1e3) / 1e9 / peak,
            "parts_ms_per_launch": {nm: (sp[i][0] / sp[i][1] if sp[i][1] else None)
                                    for i, nm in enumerate(names)},
            "form": "mixed" if head == 1 else "fp64", "steps": args.steps}
        # (2) the remeshing workload (comp_weights + remesh + create_part, 256^3)
        extra = {"sorted_input": sorted_in,
                 "remesh": remesh_extra(torch, ppmg, dev, args.warmup, args.steps, peak)}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(args)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": "particles/s for 3D M'4 P2M+M2P round trip",
            "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (mixed: FP64 offsets, FP32 weights, compensated FP32 sums)"
            if head == 1 else "f64",
            "data": "synthetic (seeded, generated on device)",
            "config": {"workload": (f"3D M'4 P2M+M2P round trip, {nc}^3 periodic mesh"
                                    if world == 1 else
                                    f"3D M'4 P2M+M2P round trip, one {nc}^3 slab per GPU of a "
                                    f"{nc}x{nc}x{nc * world} periodic mesh") +
                                   f", {n} particles per GPU ({CONFIGS[args.config][2]}), lda 3, "
                                   f"ghostsize 2",
                       "l2": l2_note,
                       "parallelism": "1 periodic subdomain" if world == 1 else
                       f"{world} z-slab subdomains of a {nc}x{nc}x{nc * world} periodic mesh, "
                       f"ghost put/get between neighbouring slabs over "
                       f"{args.dist_backend.upper()}"},
            "roofline": roof, "forms": parts, "clocks": clocks, "gpu_launches": launches,
            "e2e": e2e, "cpu_baseline": cb, "adjoint": adj, "accuracy": accuracy,
            "extra": extra,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
