"""The JSON line of bench.py's reference arm (the oracle's PCG on the host
cores), run at a small size on the CPU: one JSON line with the benchmark
keys, the same metric and units as the product arm, and the e2e and
cpu_baseline objects it has to carry, and a process that mapped none of
the product's libraries."""

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--n", "12",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    # one host V-cycle, against the same algorithmic bytes as the GPU cycle
    assert d["cpu_baseline"]["vcycle_ms"] > 0 and d["cpu_baseline"]["vcycle_GBps"] > 0
    assert d["config"]["workload"].startswith("3D 7-point heterogeneous diffusion 12^3")
    assert d["relres_fp64_verified"] < 1e-8
    # the timed process ran the oracle only: the product library is not mapped
    libs = d["loaded_repo_libraries"]
    assert "oracle/liboracle.so" in libs and not any("libdraugr_b200" in x for x in libs), libs
