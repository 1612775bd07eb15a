"""bench.py's reference arm on the CPU: one JSON line with the keys of the
benchmark contract (the reference's own solve path, oracle/_ref, timed on the
host cores; 32^3 configuration)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libbdg_ref.so")),
                    reason="oracle build missing")
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "32",
                        "--steps", "1", "--warmup", "1", "--no-anchor"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT, env={**os.environ, "RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["steps"] == 1 and d["warmup"] == 1 and len(d["step_seconds"]) == 1
    assert abs(d["ms_per_step"] - 1e3 * d["step_seconds"][0]) < 1e-6 * d["ms_per_step"]
    assert d["value"] >= d["setup_seconds"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_projection_and_cache_key():
    """The reference arm's time to tolerance: live set-up plus the cached
    solve's loop time scaled by the live/cached ratio of the sampled
    iterations; the cached solve is used only for the psi0 whose mu it was
    made from."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench

    cached = {"timeline": np.array([0.0, 10.0, 12.0, 14.0, 16.0, 18.0]), "iterations": 4}
    tl = np.array([100.0, 105.0, 106.0, 107.0, 108.0])  # set-up 5 s, iterations of 1 s
    value, live, n = bench.project_to_tolerance(tl, 1, 2, cached)
    assert n == 4 and list(live) == [1.0, 1.0]
    assert abs(value - (5.0 + 8.0 * 0.5)) < 1e-12  # cached loop 8 s at half the cached speed
    value, live, n = bench.project_to_tolerance(tl, 1, 2, None)
    assert value is None and n is None
    c = bench.cached_solve(128)
    assert c is not None and int(c["iterations"]) > 0
    assert bench.cached_solve(128, float(c["mu"])) is not None
    assert bench.cached_solve(128, float(c["mu"]) * (1 + 1e-6)) is None
