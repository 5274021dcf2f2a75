"""Host-side pieces of the bench line that need no GPU: the digest that
guards the committed DRAM-traffic figure, and the config object both arms
print."""
import importlib.util
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_kernel_digest_ignores_comments_and_whitespace_only():
    bench = load_bench()
    code = {"recon_kernel.cu": "int a = 1; // one\n/* block\ncomment */ int b = 2;\n",
            "lifting.cuh": "x  =  y;\n", "engine.h": "struct S { int v; };\n"}
    base = bench.kernel_source_digest(lambda name: code[name])
    commented = dict(code, **{"recon_kernel.cu": "int a = 1;   // another note\n\n int b = 2; /* x */\n"})
    assert bench.kernel_source_digest(lambda name: commented[name]) == base
    changed = dict(code, **{"recon_kernel.cu": "int a = 1; int b = 3;\n"})
    assert bench.kernel_source_digest(lambda name: changed[name]) != base


def test_traffic_figure_is_withheld_when_the_kernel_changed(tmp_path, monkeypatch):
    bench = load_bench()
    monkeypatch.setattr(bench, "kernel_source_digest", lambda read=None: "0" * 64)
    got = bench.captured_traffic("c2")
    assert got["traffic"] is None and "predates" in got["traffic_note"]


def test_config_carries_the_keys_both_arms_print():
    bench = load_bench()
    for workload in ("c2", "c3", "c4"):
        cfg = bench.config_of(workload, 1)
        assert {"workload", "global_batch", "parallelism", "l2"} <= set(cfg)
        assert cfg == bench.config_of(workload, 1)
