"""bench.py's host-side helpers (CPU): the L2 note, the lookups in the
committed ncu summaries, and the config object both arms print."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from mls_mpm_b200 import scenes  # noqa: E402


def test_l2_note_sizes_the_working_set():
    big = bench.l2_note(1 << 20, 128 ** 3, 262144)
    assert big.startswith("working set > 126 MB L2") and "particles 72 MB" in big and "grids 64 MB" in big
    small = bench.l2_note(65536, 64 ** 3, 0)
    assert small.startswith("working set <= 126 MB L2")


def test_profile_lookups_follow_the_workload():
    # the committed captures of the 1M and 8M dam breaks carry traffic and
    # issue use of the dominant kernel (below its algorithmic bytes: 113.2 MB
    # and 771.8 MB per launch); a workload without a capture has none
    t = bench._profile_traffic("p2g_mom", "dam_break_1m")
    assert isinstance(t, int) and 50_000_000 < t < 113_246_208
    issue = bench._profile_value("issue_active_per_launch", "p2g_mom", "dam_break_1m")
    assert 0.0 < issue <= 1.0
    t8 = bench._profile_traffic("p2g_mom", "dam_break_sphere_8m")
    assert isinstance(t8, int) and 400_000_000 < t8 < 771_751_936
    assert bench._profile_traffic("p2g_mom", "dam_break_64") is None
    assert bench._profile_traffic("no_such_phase", "dam_break_1m") is None


def test_both_arms_share_one_config():
    sc = scenes.WORKLOADS["dam_break_64"](seed=0)
    c1 = bench.run_config("dam_break_64", sc, 1)
    c4 = bench.run_config("dam_break_64", sc, 4)
    assert c1["particles"] == sc.n and c1["grid"] == list(sc.grid) and c1["parallelism"] == "single scene"
    assert c4["parallelism"] == "scene-sharded x4"
    assert set(c1) == {"workload", "grid", "particles", "diffuse_pool", "substeps_per_step", "parallelism", "l2"}
