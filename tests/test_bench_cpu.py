"""Host side of bench.py without a GPU: the reference arm's JSON line (the oracle
port timed on the host cores) and the seeded workload generators."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "updates/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] >= 3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"].startswith("large plain WBP")


def test_c4_jobs_are_seeded_and_in_range():
    a, b = bench.c4_jobs(), bench.c4_jobs()
    assert len(a) == 64
    for x, y in zip(a, b):
        assert x["w"] == y["w"] and x["thick"] == y["thick"] and x["sirt"] == y["sirt"]
        np.testing.assert_array_equal(x["ang"], y["ang"])
    assert {j["w"] for j in a} <= {256, 384, 512, 768, 1024}
    assert all(41 <= len(j["ang"]) <= 121 and 100 <= j["thick"] <= 500 for j in a)
    assert sum(j["sirt"] > 0 for j in a) == 16  # WBP:SIRT(10) = 3:1
    for j in a:  # angles increase over about +-U(50, 70) deg
        assert np.all(np.diff(j["ang"]) > 0) and 49.0 < -j["ang"][0] < 71.0
    j = a[0]
    assert bench.job_updates(j) == float(j["w"]) ** 2 * j["thick"] * len(j["ang"]) * (1 + 2 * j["sirt"])


def test_hbm_peak_is_read_from_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6463.0}))
    v, how = bench.hbm_peak()
    assert v == 6463.0 and "measured" in how


def test_roofline_traffic_comes_from_the_capture_of_the_timed_tile_shape():
    # the committed summaries list one capture per tile shape the tuner picks; each
    # `variant:` line is followed by that capture's per-launch DRAM bytes
    for storage in ("fp16", "fp32"):
        seen = {}
        cur = None
        for line in open(os.path.join(ROOT, "profiles", f"bp_fast_c2strip_{storage}.md")):
            key, _, val = line.partition(":")
            if key == "variant":
                cur = val.strip()
            elif key == "traffic_bytes_per_launch":
                seen.setdefault(cur, float(val))
        assert set(seen) >= {"S8K4TX64NT256V4N3", "S8K4TX32NT256V8N2"}
        for name, want in seen.items():
            assert bench.read_traffic(name, storage) == want
            # staged windows once + the 13.42 GB volume once (about 15.1 GB FP16, 17.2 GB FP32)
            assert 13.4e9 < want < 18e9
    assert bench.read_traffic("S16K2TX32NT256V4N3", "fp16") is None  # no capture: no claim
