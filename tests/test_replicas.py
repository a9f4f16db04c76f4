"""The multi-rank path on CPU: two gloo ranks (processes) share a list of
models, each evaluates its contiguous shard (here with the C oracle, the
engine's stand-in on a machine without GPUs), and the gathered chi**2 and
light curves equal a single process evaluating every model; the job time is
the slower rank's."""
import os
import socket

import numpy as np
import pytest

from lcurve_re_b200.replicas import gather_rows, max_over_ranks, shard


def test_shard_covers_every_unit_once():
    for n in (0, 1, 7, 256, 1001):
        for world in (1, 2, 3, 8):
            got = [shard(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [hi - lo for lo, hi in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _models():
    from lcurve_re_b200 import workloads as W
    return [W.model(nlat1f=10, nlat2f=16, q=0.2 + 0.01 * k) for k in range(5)]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from oracle_lib import Oracle
        from lcurve_re_b200 import workloads as W
        ms, d = _models(), W.data(60)
        o = Oracle()
        lo, hi = shard(len(ms), rank, world)
        rows = []
        for m in ms[lo:hi]:
            st, err, calc, sf, sc = o.light_curve(m, d)
            rows.append(np.r_[sc[1], calc])
        full = gather_rows(np.array(rows).reshape(hi - lo, -1), len(ms), dist)
        t = max_over_ranks(1.0 + rank, dist)
        q.put((rank, full, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle_lib import Oracle
    from lcurve_re_b200 import workloads as W
    d = W.data(60)
    serial = []
    for m in _models():
        st, err, calc, sf, sc = Oracle().light_curve(m, d)
        serial.append(np.r_[sc[1], calc])
    serial = np.array(serial)
    for rank, full, t in res:
        assert np.array_equal(full, serial), rank
        assert t == 2.0


def test_bench_gpus_flag_launches_one_process_per_rank():
    """bench.py --gpus 2 without a launcher starts two ranks itself (RANK,
    LOCAL_RANK, WORLD_SIZE, MASTER_* set as torch.distributed.run sets them);
    rank 0 alone prints one line, which reports n_gpus 2. The reference arm
    needs no GPU, so it runs here."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--workload", "wd_dm_small", "--steps", "1", "--warmup",
                        "0"], capture_output=True, text=True, timeout=600, env=env, cwd=root)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
