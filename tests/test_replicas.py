"""The multi-GPU path of bench.py is replicas only (independent products, no
data-path collective); these CPU tests run its rank plumbing as two gloo
processes: the max-over-ranks timing, and the reference arm under torchrun
(rank 0 alone works and prints; the other ranks exit 0)."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(10.0 * (rank + 1), dist, world, "cpu")
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert dict(out) == {0: 20.0, 1: 20.0}


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--ring", "1024"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    # the reference's own kernels under its CPU emulation when that binary was built, else the C restatement
    from tests import reference_emulation as emu

    want_kind = "reference" if emu.available() else "port"
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == want_kind
    assert line["e2e"]["h2d_bytes_per_step"] == 0
