"""Host-side helpers of bench.py that shape its JSON line: the clock record taken during the
timed region, the roofline peak (measured file or fallback) and the DRAM traffic read from
the committed ncu summary."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_clock_record_median_and_throttle_reasons():
    c = bench.Clocks(0)
    rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1940, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
            "garbage"]
    c.f.write("\n".join(rows) + "\n")
    s = c.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                 "samples": 3}


def test_clock_record_without_samples():
    s = bench.Clocks(0).summary()
    assert s["samples"] == 0 and s["reasons"] == ["unavailable"] and s["sm_mhz"] is None


def test_roofline_peak_measured_or_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6450.3}))
    assert bench.peaks() == (6450.3, "measured")


def test_traffic_from_committed_profile():
    t = bench.profiled_traffic("k_staged_n100k.md")
    text = open(os.path.join(ROOT, "profiles", "k_staged_n100k.md")).read()
    assert t is not None and f"traffic_bytes_per_launch: {int(t)}" in text
    assert 1.0 < t / (28 * 800_000 + 8 * 100_000) < 2.0  # DRAM bytes vs algorithmic bytes
    assert bench.profiled_traffic("no_such_summary.md") is None


def test_reference_arm_runs_the_reference_alone_on_the_bench_config():
    """`bench.py --impl reference` times the unmodified reference integrator on the bench
    formula and initial state, built without this repository's library, for exactly the
    steps it reports, and prints this arm's config."""
    import subprocess

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "2", "--warmup", "3", "--procs", "2"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["config"] == bench.bench_config(1)
    assert line["steps_done_per_process"] == [2, 2]
    assert line["repo_libraries_loaded"] == ["oracle/_ref/libdynex_ref.so"]
    assert line["cpu_baseline"]["cores"] == 2 and line["e2e"]["value"] == line["value"]
