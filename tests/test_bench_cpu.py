"""bench.py's reference arm on the CPU: `--impl reference` times the reference's own host solve
(oracle/_ref, else the oracle port) and prints one JSON line with the keys the measurement contract
names. A small box keeps it to seconds."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--n", "20",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, cwd=REPO, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] == 1 and cb["value"] == d["value"]
    assert cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["cells"] == 20 ** 3
    # the workload is worded by the one function both arms use
    assert d["config"]["workload"] == _bench().workload_name(20)
    init, final, iters = d["config"]["solver_perf"]
    assert init == 1.0 and 0 < final < 0.05 and iters >= 1
    # both arms word the workload from one function, so the driver sees the same configuration
    sys.path.insert(0, REPO)
    import bench
    assert d["config"]["workload"] == bench.workload_name(20)
    assert d["cpu_baseline"]["cpu_model"]


def _bench():
    sys.path.insert(0, REPO)
    import bench
    return bench


def test_cases_for_rank_shards_every_case_once():
    # the batched workload's sharding by case: every case on exactly one rank, the largest cases
    # spread first, so no rank carries much more than its share
    bench = _bench()
    cells = [4096 * (1 + (7 * i) % 23) for i in range(57)]
    for world in (1, 2, 3, 8):
        shards = [bench.cases_for_rank(cells, r, world) for r in range(world)]
        seen = sorted(i for s in shards for i in s)
        assert seen == list(range(len(cells)))
        loads = [sum(cells[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(cells)
        assert all(s == sorted(s) for s in shards)


def test_traffic_per_launch_reads_the_committed_summary():
    bench = _bench()
    with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
        d = json.load(f)
    for workload, kernels in d.items():
        for kernel, v in kernels.items():
            if isinstance(v, (int, float)):
                assert bench.traffic_per_launch(kernel, workload) == float(v)
    assert bench.traffic_per_launch("no such kernel", "no such workload") is None
