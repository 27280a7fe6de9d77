"""The reference arm of bench.py (the CPU oracle of run_matching) keeps its
JSON-line contract: one line on rank 0 with the metric, the workload, a
cpu_baseline describing the run and an end-to-end entry with no copies;
nothing from other ranks."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "dtype", "data", "config", "cpu_baseline",
                "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "channel-samples/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert "C=384" in d["config"]["workload"] and "K=600" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_print_nothing():
    assert _run({"RANK": "1", "WORLD_SIZE": "2"}) == []


def test_workload_options_parse():
    """Every workload and the extra-workload switch are accepted by the
    command line (the device runs need a GPU; the parser does not)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    argv = sys.argv
    try:
        for w in ("np1", "uneven", "adjoint", "stream", "detect", "extract", "filter"):
            sys.argv = ["bench.py", "--workload", w, "--no-extra", "--steps", "2", "--warmup", "3"]
            a = bench.parse()
            assert a.workload == w and a.no_extra and a.steps == 2 and a.warmup == 3
        sys.argv = ["bench.py"]
        a = bench.parse()
        assert a.workload == "np1" and not a.no_extra and a.gpus == 1
    finally:
        sys.argv = argv
