"""bench.py's host-side contract (no GPU): the committed ncu summaries it quotes
carry the figures it reads, both arms of the headline share one config builder, and
the option parser keeps its defaults."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_committed_summaries_carry_the_quoted_figures():
    for kernel in ("lambda", "delta"):
        for key in ("dram_bytes_per_launch", "issue_active_pct", "l2_hit_pct"):
            v = bench.committed_value(kernel, bench.MIX, key)
            assert v is not None and v > 0, (kernel, key)
    for kernel in ("lambda", "delta", "xsph_normals", "aniso"):
        v = bench.committed_value(kernel, "medium_bodies_264k", "dram_bytes_per_launch")
        assert v is not None and v > 0, kernel
    assert bench.committed_value("no_such_kernel", bench.MIX, "dram_bytes_per_launch") is None


def test_profiles_hold_text_summaries_only():
    names = os.listdir(os.path.join(ROOT, "profiles"))
    assert names and all(n.endswith((".txt", ".md")) for n in names), names


def test_default_options(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse_args()
    assert (a.gpus, a.steps, a.warmup, a.impl, a.workload) == (1, 20, 5, "ours", bench.MIX)
    assert a.lanes == 2 and a.io_groups == 0 and a.warmup >= 3


def test_both_arms_build_the_headline_config_alike():
    import inspect
    assert "mix_config(mix, world)" in inspect.getsource(bench.run_reference)
    assert "mix_config(mix, world)" in inspect.getsource(bench.run_mix)
