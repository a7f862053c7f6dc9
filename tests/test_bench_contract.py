"""The bench's JSON contract pieces that need no GPU: both arms report the
same workload config, and the dominant kernel's per-launch figures parse from
the committed ncu summary."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_workload_config_shared_by_both_arms():
    b = _bench()
    c1, c4 = b.workload_config(1), b.workload_config(4)
    assert c1["workload"] == c4["workload"] and "6048x4024" in c1["workload"]
    assert c1["global_batch"] == 1 and c4["global_batch"] == 4
    assert c4["parallelism"] == "replicas x4"


def test_ncu_figures_parse():
    b = _bench()
    traffic = b.ncu_figure("traffic_bytes_per_launch")
    inst = b.ncu_figure("warp_instructions_per_launch")
    assert isinstance(traffic, int) and traffic > 0
    assert isinstance(inst, int) and inst > 0
    assert b.ncu_figure("no_such_figure") is None


def _run_bench(*argv):
    import json
    import subprocess
    import sys
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *argv], capture_output=True, text=True,
                       timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    return json.loads(lines[0])


def test_gpus_flag_launches_ranks_itself():
    """`python bench.py --gpus 2` without torchrun starts two ranks (torchrun
    on 127.0.0.1); --dry-run keeps them on gloo with no GPU work.  Both ranks
    take part in the max-over-ranks reduction and rank 0 reports n_gpus 2."""
    for impl in ("imops_b200", "reference"):
        line = _run_bench("--gpus", "2", "--dry-run", "--steps", "2", "--warmup", "1", "--impl", impl)
        assert line["dry_run"] is True and line["impl"] == impl
        assert line["n_gpus"] == 2 and line["ranks_reporting"] == 2
        assert line["config"]["parallelism"] == "replicas x2"


def test_single_rank_dry_run():
    line = _run_bench("--dry-run", "--steps", "1", "--warmup", "1")
    assert line["n_gpus"] == 1 and line["ranks_reporting"] == 1
