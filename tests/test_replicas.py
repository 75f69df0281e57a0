"""The replicas path of bench.py on the CPU: two gloo ranks (world size 2)
run the same rank plumbing the GPU bench uses (barrier, max over ranks of the
timed region, whole-job rate), and a rank that raises makes the launcher fail
instead of hanging the others (short process-group timeout)."""
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def run_ranks(body, world=2, timeout=120):
    code = textwrap.dedent(f"""
        import os, sys, json
        sys.path.insert(0, {ROOT!r})
        import bench
        r = bench.Ranks("gloo", timeout_s=20)
    """) + textwrap.dedent(body)
    port = free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        outs.append((p.returncode, o, e))
    return outs


def test_max_over_ranks_and_whole_job_rate():
    outs = run_ranks("""
        r.barrier()
        slow = r.max(1.0 + r.rank)              # rank 1 is the slowest: 2.0 s
        rate = bench.whole_job_rate(100, r.world, slow)
        r.barrier()
        print(json.dumps({"rank": r.rank, "world": r.world, "slow": slow, "rate": rate}))
        r.close()
    """)
    import json
    res = [json.loads(o.strip().splitlines()[-1]) for rc, o, e in outs if rc == 0]
    assert len(res) == 2, outs
    for d in res:
        assert d["world"] == 2 and d["slow"] == 2.0 and d["rate"] == 100.0   # 200 units / 2.0 s


def test_failing_rank_does_not_hang_the_other():
    outs = run_ranks("""
        if r.rank == 1:
            raise SystemExit(3)                 # leaves before the collective
        try:
            r.max(1.0)
            print("unexpected: collective completed")
        except Exception as e:
            print("collective failed:", type(e).__name__)
            sys.exit(5)
    """, timeout=90)
    (rc0, o0, e0), (rc1, o1, e1) = outs
    assert rc1 == 3
    assert rc0 != 0 and "unexpected" not in o0


def test_single_rank_needs_no_process_group():
    import bench
    os.environ.pop("WORLD_SIZE", None)
    r = bench.Ranks("gloo")
    assert r.world == 1 and r.max(3.5) == 3.5
    r.barrier()
    r.close()
    assert bench.whole_job_rate(10, 1, 2.0) == 5.0
