"""Host logic of the multi-GPU benchmark path on CPU: world_size-2 `gloo`
process groups (the GPU path runs the same code over NCCL, one process per
GPU, as independent subdomain replicas with no data-path collective)."""
import json
import os
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _rank_main(rank, world, port, values, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(values[rank], dist)
        dist.barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_gloo_world2():
    """Every rank gets the slowest rank's time (the timing rule for N > 1)."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    values = [12.5, 17.25]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 17.25, 1: 17.25}


def test_max_over_ranks_without_group_is_identity():
    assert bench.max_over_ranks(3.0) == 3.0


def test_reference_arm_other_ranks_print_nothing():
    """Under torchrun only rank 0 of the reference arm runs and prints."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_weak_scaling_units_and_bytes():
    """Algorithmic bytes per round trip at lda 3 with FP64 I/O: 96 B per
    particle (xp read twice, up read and written) + 48 B per node (field
    written and read once): 144 B per particle at one particle per cell."""
    np_, nc = 2_097_152, 128
    assert bench.alg_bytes(np_, nc) == np_ * 96 + nc ** 3 * 48
    assert bench.alg_bytes(nc ** 3, nc) == nc ** 3 * 144
    kb = bench.kernel_bytes(np_, nc, 3, 2, True)
    assert kb["p2m_gather"] == np_ * 32 + (nc + 5) ** 3 * 24
    assert kb["m2p_gather"] == nc ** 3 * 24 + np_ * 44


def test_weak_scaling_slab_topology_and_particle_shift():
    """The N-GPU benchmark domain: slab r is z in [r, r+1) with cubic cells of
    1/nc, and every particle shifted into slab r stays inside it (a z that
    would round up to the slab's top face moves to its bottom face)."""
    import numpy as np

    import ppm_legacy_b200 as ppmg
    from ppm_legacy_b200 import halo
    world, nc = 3, 8
    t = bench.slab_topology(ppmg, nc, world)
    assert t.nsubs == world and list(t.Nm) == [nc + 1, nc + 1, nc * world + 1]
    assert np.allclose(t.h, 1.0 / nc)
    for r in range(world):
        assert t.min_sub[r, 2] == r and t.max_sub[r, 2] == r + 1
        assert halo.neighbours(t, r) == ((r - 1) % world, (r + 1) % world)
        xp = torch.rand((3, 1000), dtype=torch.float64)
        xp[2, :3] = torch.tensor([0.0, np.nextafter(1.0, 0.0), 0.5])
        xp = bench.shift_to_slab(torch, xp.t().contiguous().t(), r)
        z = xp[2].numpy()
        assert (z >= t.min_sub[r, 2]).all() and (z < t.max_sub[r, 2]).all()
