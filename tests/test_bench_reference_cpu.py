"""The reference arm of bench.py runs on the host alone: the oracle (the CPU
restatement of the reference search) on a bounded sample of the workload,
printed as one JSON line with the keys the benchmark contract names, the
engine arm's exact workload definition, and without loading the engine."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# runs bench.py's reference arm, then reports whether any engine module or
# engine library was loaded into the process
PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
mods = [m for m in sys.modules if m.startswith("td16_b200")]
maps = open("/proc/self/maps").read()
print("LOADED", json.dumps({"modules": mods, "libtd16b200": "libtd16b200.so" in maps}))
""".replace("import runpy, sys", "import json, runpy, sys")


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["nproc"] >= 1 and cb["cpu_model"] and cb["nodes_per_s"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.bench_config(1)
    loaded = json.loads([l for l in out.stdout.splitlines() if l.startswith("LOADED")][0].split(" ", 1)[1])
    assert loaded == {"modules": [], "libtd16b200": False}
