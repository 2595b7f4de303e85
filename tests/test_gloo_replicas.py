"""Multi-process (gloo, world size 2) coverage of bench.py's replica plumbing:
barrier, max-over-ranks timing and the split of forward solves over ranks."""
import os
import socket
import subprocess
import sys
import textwrap

from conftest import ROOT


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_bench_replica_plumbing_gloo(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(textwrap.dedent("""
        import os, sys, json
        sys.path.insert(0, %r)
        import bench
        world, rank, local = bench.dist_init(2)
        bench.barrier(world)
        t = bench.max_over_ranks(world, 1.0 + rank)
        units = bench.shard_units(5, world, rank)
        print(json.dumps({"rank": rank, "max": t, "units": units}))
        import torch.distributed as dist
        dist.destroy_process_group()
    """ % ROOT))
    env = dict(os.environ, TDEM_BENCH_BACKEND="gloo", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(free_port()),
               WORLD_SIZE="2")
    procs = []
    for r in range(2):
        e = dict(env, RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=e, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    import json
    res = sorted((json.loads(o[0].strip().splitlines()[-1]) for o in outs), key=lambda d: d["rank"])
    assert all(p.returncode == 0 for p in procs), [o[1] for o in outs]
    assert res[0]["max"] == 2.0 and res[1]["max"] == 2.0
    assert res[0]["units"] + res[1]["units"] == [0, 1, 2, 3, 4]
