"""bench.py's multi-process plumbing on CPU: two ranks over gloo (127.0.0.1), as the driver
launches the N > 1 bench with one process per GPU.  The path shards with no exchange (every rank
runs an independent replica), so the only collectives are the barrier around the timed region
and the max over ranks of the measured time; both are checked here without a GPU."""
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

_RANK_CODE = """
import sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_init()
bench.barrier(ws)
m = bench.max_over_ranks(ws, 10.0 * (rank + 1))
bench.barrier(ws)
import torch.distributed as dist
dist.destroy_process_group()
print("RESULT", ws, rank, local, m, flush=True)
"""


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    env = {k: os.environ.get(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        for k in env:
            os.environ.pop(k, None)
        ws, rank, local = bench.dist_init()
        assert (ws, rank, local) == (1, 0, 0)
        bench.barrier(ws)
        assert bench.max_over_ranks(ws, 3.5) == 3.5
    finally:
        for k, v in env.items():
            if v is not None:
                os.environ[k] = v


def test_two_ranks_barrier_and_max_over_ranks_gloo():
    port = _free_port()
    code = _RANK_CODE.format(root=str(ROOT))
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), V3DM_BENCH_BACKEND="gloo")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    results = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=240)
            assert p.returncode == 0, err[-2000:]
            line = [x for x in out.splitlines() if x.startswith("RESULT")][-1].split()
            results.append((int(line[1]), int(line[2]), int(line[3]), float(line[4])))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert sorted(r[1] for r in results) == [0, 1]
    for ws, rank, local, m in results:
        assert ws == 2 and local == rank
        assert m == 20.0  # the slower rank's time, on every rank
