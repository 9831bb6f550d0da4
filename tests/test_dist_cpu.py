"""The replicas-only multi-GPU path, exercised with two gloo ranks on CPU:
sharding covers every line exactly once, the per-rank results assembled
from the shards equal the single-rank result (each rank transforms its lines
with the oracle standing in for its GPU), and the timed region's max over
ranks is the max."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from metalfft_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    r, w, _ = D.rank_world()
    x = O.uniform_c64((37, 256), seed=123)  # the same full batch on every rank
    start, count = D.shard(len(x), r, w)
    y = O.ref_fft(x[start:start + count])
    t = D.max_over_ranks(float(r + 1) * 1.5)
    dist.barrier()
    out_q.put((r, start, count, y, t))
    dist.destroy_process_group()


def test_shard_covers_once():
    for total in [0, 1, 7, 16384]:
        for world in [1, 2, 3, 8]:
            seen = []
            for r in range(world):
                s, c = D.shard(total, r, world)
                seen.extend(range(s, s + c))
            assert seen == list(range(total))


def test_two_gloo_ranks():
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    x = O.uniform_c64((37, 256), seed=123)
    full = O.ref_fft(x)
    got = np.concatenate([r[3] for r in res])
    assert np.array_equal(got, full)
    assert all(r[4] == 3.0 for r in res)  # max over ranks of 1.5 and 3.0


def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched as the driver launches every arm
    for N > 1: rank 0 alone times the host path and prints one JSON line, on
    every core the process may use although torchrun sets OMP_NUM_THREADS=1;
    the other rank exits 0 without work."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--batch", "64"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    assert d["cpu_baseline"]["cores"] == cores
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
