"""The deterministic accumulation's arithmetic (CPU test).

fx_add in csrc/pfk_device.cuh turns each J/K contribution v into two 64-bit
integer words without a float-to-integer conversion, by rounding through
1.5 2^52 with fused multiply-adds.  tests/fx_split_check.c restates those
steps in host C (the same operations, IEEE double with the C library's fma)
and checks them against exact integer arithmetic: hi 2^36 + lo equals
rint(v 2^60) for 2.1 M seeded values across every binade the device uses
and for the edge cases (ties, the range limits), |lo| <= 2^35, the words of
a sum do not depend on the order of the adds, and the value rule returns
the exact sum rounded once.  The GPU determinism tests check the device
itself (tests/test_determinism_gpu.py)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_fixed_point_split_is_exact(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "fx_split_check"
    r = subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", os.path.join(HERE, "fx_split_check.c"),
                        "-lm", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
    assert int(r.stdout.split()[1]) > 2_000_000
