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
