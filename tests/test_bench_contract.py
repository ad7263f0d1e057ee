"""CPU checks of bench.py's reporting logic (no GPU): the roofline object carries the keys the
benchmark line promises, its fraction is achieved / peak, the HBM peak names its source (the
measured figure when MEASURED_PEAKS.json is there, the fallback otherwise), and the clock
sampler reads samples taken inside the timed region (against an nvidia-smi stand-in)."""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

PEAKS = {"mul_lo_per_s": 18.4e12, "mul_hi_per_s": 9.2e12, "modmul_per_s": 3.37e12, "p24_perms_per_s": 3.25e9}


def test_hbm_peak_source(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    value, source = bench.read_hbm_peak()
    assert value == 6650.0 and source.startswith("fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6542.7}))
    value, source = bench.read_hbm_peak()
    assert value == 6542.7 and "measured" in source
    (tmp_path / "MEASURED_PEAKS.json").write_text("{}")  # a file without the key falls back
    assert bench.read_hbm_peak()[1].startswith("fallback")


def test_roofline_object():
    profile = {"merkle_tree": (16.5 * 5, 25), "lde": (4.0 * 5, 55)}
    breakdown = {"merkle_tree": (16.5, 5), "lde": (4.0, 11), "other": (9.0, 261)}
    r = bench.roofline(profile, breakdown, 20, PEAKS, 6650.0, 5, "fallback: test")
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in r, key
    assert r["kernel"] == "merkle_tree" and r["bound"] == "int"
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert abs(r["share_of_kernel_time"] - 16.5 / 29.5) < 1e-12
    assert r["hbm"]["peak"] == 6650.0 and r["hbm"]["peak_source"] == "fallback: test"
    # a Montgomery product takes two low-word and two high-word multiplies
    assert abs(r["peak"] * 1e12 - 1.0 / (2 / PEAKS["mul_lo_per_s"] + 2 / PEAKS["mul_hi_per_s"])) < 1.0


def _fake_smi(tmp_path, reasons):
    """An nvidia-smi stand-in that prints one sample line every 10 ms until it is stopped."""
    script = tmp_path / "nvidia-smi"
    line = "0, 1965 MHz, 1965 MHz, 350.00 W, 0x0, " + ", ".join(reasons)
    script.write_text("#!" + sys.executable + "\n"
                      "import sys, time\n"
                      "while True:\n"
                      f"    print({line!r}, flush=True)\n"
                      "    time.sleep(0.01)\n")
    script.chmod(0o755)
    return str(tmp_path)


def test_clock_sampler_reads_the_timed_region(tmp_path, monkeypatch):
    idle = ["Not Active"] * 4
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, idle) + os.pathsep + os.environ["PATH"])
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.25)
    c = s.stop()
    assert c["samples_in_region"] and c["samples"] >= 5
    assert c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0 and c["reasons"] == []
    # a region shorter than the interval keeps the sample just before it
    s = bench.ClockSampler(0)
    s.start()
    c = s.stop()
    assert c["samples"] >= 1 and c["sm_mhz"] == 1965.0


def test_clock_sampler_reports_throttle_reasons(tmp_path, monkeypatch):
    capped = ["Not Active", "Not Active", "Not Active", "Active"]
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, capped) + os.pathsep + os.environ["PATH"])
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.1)
    assert s.stop()["reasons"] == ["sw_power_cap"]
