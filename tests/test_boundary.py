"""CPU checks of the product boundary: the C-ABI library loads and exports every entry
point include/whirlaway_b200.h declares, host-only entry points work without a GPU, and the
device field arithmetic (compiled for the host) matches plain modular arithmetic."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "whirlaway_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(?:wl_status|void|int32_t|uint64_t|const char\*|void\*)\s+\*?(wl_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(wl):
    lib = wl.load_library()
    names = declared_functions()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", wl.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (wl_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_host_entry_points_without_gpu(wl, oracle):
    c, i = wl.generate_workload(5, -1)
    c2, i2 = oracle.workload(5, -1)
    assert np.array_equal(c, c2) and np.array_equal(i, i2)
    assert wl.air_columns() == 165 and wl.constants_len() == 148 + 148 + 215
    s = wl.AirSettings()
    assert wl.proof_len_bound(s, 12) > 40000
    with pytest.raises(wl.ProverError):
        wl.proof_len_bound(wl.AirSettings(univariate_skips=4), 4)  # skips must be < log_n
    assert wl.proof_footprint_bytes(20) > 3 << 30
    # rate 1/8 quadruples the first commitment; invalid settings give 0
    assert wl.proof_footprint_bytes(20, wl.AirSettings(log_inv_rate=3)) > 2 * wl.proof_footprint_bytes(20)
    assert wl.proof_footprint_bytes(3, wl.AirSettings(univariate_skips=4)) == 0


def test_device_field_arithmetic_on_host(tmp_path):
    exe = tmp_path / "field_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "whirlaway_b200", "csrc"),
                    os.path.join(ROOT, "tests", "field_host_check.cpp"),
                    os.path.join(ROOT, "whirlaway_b200", "csrc", "host_perm.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_tuner_interface_without_device(wl):
    """The autotuner's process-wide controls work without a GPU: families by name, plans in
    range, an empty report before any proof."""
    rep = wl.tune_report()
    assert set(rep) == {"lde", "leaf", "merkle", "inner"}
    wl.tune_force("lde", 5)
    wl.tune_force("lde", -1)
    for fam, plan in (("lde", 6), ("leaf", 3), ("inner", 2), ("nope", 0)):
        with pytest.raises(wl.ProverError):
            wl.tune_force(fam, plan)
