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

Multi-GPU (torchrun): weak scaling, every rank runs its own subdomain-sized
problem (independent replicas, no data-path collective); time = max over ranks.
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
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    import ppm_legacy_b200 as ppmg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    xp, up, nc, n = gen_particles(torch, args.config, dev, seed=1000 + rank)
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

    def step():
        i1 = ppmg.ppm_interp_p2m(xp, n, up, 3, 1, 1, 2, g, field)
        i2 = ppmg.ppm_interp_m2p(xp, n, out, 3, 1, 1, 2, g, field)
        if i1 or i2:
            raise RuntimeError(f"library error {ppmg.last_error()}")

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
            evp[0].record(stream)
            ppmg.ppm_interp_p2m(xp, n, up, 3, 1, 1, 2, g, field)
            evp[1].record(stream)
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
        ms = ev0.elapsed_time(ev1) / args.steps
        if world > 1:
            tt = torch.tensor([ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
            if world > 1:
                dist.barrier()
        p2m = float(np.median([a for a, _ in p2m_ms]))
        m2p = float(np.median([b for _, b in p2m_ms]))
        return ms, p2m, m2p, launches, kparts

    sampler = ClockSampler(local)
    sampler.start()
    res = {}
    precs = {"both": [1, 0], "mixed": [1], "fp64": [0]}[args.precision]
    for prec in precs:
        res[prec] = timed(prec)
    clocks = sampler.stop()

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
            tt = torch.tensor([el], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        t1 = t0 + el
        fbytes = nf.nbytes
        h2d = nx.nbytes * 2 + nu.nbytes + fbytes
        d2h = fbytes + no.nbytes
        e2e = {"value": n * world / ((t1 - t0) / args.e2e_steps), "unit": "particles/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps,
               "path": "host-pointer C-ABI (ppmg_interp_p2m_dv_3d, ppmg_interp_m2p_dv_3d), "
                       "pinned host buffers"}

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
            "config": {"workload": f"3D M'4 P2M+M2P round trip, {nc}^3 periodic mesh, {n} "
                                   f"particles per GPU ({CONFIGS[args.config][2]}), lda 3, "
                                   f"ghostsize 2",
                       "l2": "inputs larger than L2 (xp/up/field each > 126 MB)",
                       "parallelism": f"{world} independent subdomain replicas"},
            "roofline": roof, "forms": parts, "clocks": clocks, "gpu_launches": launches,
            "e2e": e2e, "cpu_baseline": cb,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
