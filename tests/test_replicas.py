"""bench.py on N GPUs: independent replicas, a gloo group for the barriers and the max over ranks.

Run here as two CPU processes (world size 2, gloo on 127.0.0.1): every rank gets the max of the
ranks' timings, rank 0 builds first and the other rank after the barrier, and the reference arm
runs on rank 0 alone (the other rank exits 0 without output).
"""
import os
import socket
import subprocess
import sys
import textwrap

from conftest import REPO


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CHILD = textwrap.dedent("""
    import importlib.util, json, os, sys
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(sys.argv[1], "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    reps = bench.Replicas(timeout_s=60)
    order = os.path.join(sys.argv[2], "order.txt")

    def make():
        with open(order, "a") as f:
            f.write(str(reps.rank))
        return reps.rank

    built = reps.rank0_first(make)
    synced = []
    reps.barrier(lambda: synced.append(1))
    m = reps.max(1.5 + reps.rank)
    reps.close()
    print(json.dumps({"rank": reps.rank, "world": reps.world, "max": m, "built": built, "synced": len(synced)}))
""")


def test_two_replicas_share_barriers_and_the_max(tmp_path):
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, REPO, str(tmp_path)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    import json
    res = []
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
        res.append(json.loads(o.strip().splitlines()[-1]))
    assert [r["rank"] for r in res] == [0, 1] and all(r["world"] == 2 for r in res)
    assert all(r["max"] == 2.5 for r in res)
    assert [r["built"] for r in res] == [0, 1] and all(r["synced"] == 1 for r in res)
    assert (tmp_path / "order.txt").read_text() == "01"


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_arm_runs_the_workload_sizes():
    """The reference arm runs one thread-rank per subdomain of the main workload: by default 100^3,
    64 subdomains and overlap 1 (the reference's, so both arms run the same matrix, partition and
    preconditioner and name it in the same words); on a small case its line names the sizes it ran."""
    import importlib.util
    import json
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(REPO, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    a = bench.parse([])
    wl = bench.main_workload(a)
    assert (wl.nx, wl.nsub, wl.opts.overlap, a.overlap) == (100, 64, 1, 1)
    assert "overlap 1" in bench.workload_desc(wl, a.overlap)
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "s2l_ref")):
        return
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--nx", "12",
                        "--nsub", "4", "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][-1])
    assert "12^3" in line["config"]["workload"] and "4 subdomains" in line["config"]["workload"]
    small = bench.parse(["--nx", "12", "--nsub", "4"])
    assert line["config"]["workload"] == bench.workload_desc(bench.main_workload(small), 1)
    assert line["cpu_baseline"]["sample"].startswith("1 full solves, 4 thread-ranks")
    assert line["config"]["true_rel_residual"] <= 1.1e-8
