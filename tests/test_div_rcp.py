"""The FP64 kernels divide by run constants (cell widths, molar masses, reduced
masses) and by cell values used several times through fhd::div_rcp /
div_rcp_any (Markstein's correction step with a known reciprocal).  Bitwise
parity with the oracle needs those quotients to equal the IEEE division exactly:
this runs the same header on the host against a / b over ~1e8 dividend/divisor
pairs, including signed zeros over divisors of both signs, subnormals, inf/NaN,
window edges and quotients next to rounding midpoints (and the zero-dividend
short cut div_zero_short), and checks that the check itself catches an
uncorrected quotient."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fhdex_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "cpp", "div_rcp_check.cpp")


def build(tmp_path, include_dir):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "div_rcp_check")
    cmd = [cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-Wextra", "-Werror",
           "-I", include_dir, SRC, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_div_rcp_equals_ieee_division(tmp_path):
    exe = build(tmp_path, CSRC)
    r = subprocess.run([exe, "20000000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("mismatches 0"), r.stdout


def test_check_detects_an_uncorrected_quotient(tmp_path):
    """The same check against a planted mistake (the quotient a*y without the
    remainder correction) must report mismatches."""
    src = open(os.path.join(CSRC, "fhd_div.h")).read()
    good = "return fma(fma(-q, b, a), y, q);"
    assert src.count(good) == 3, "the planted mistake targets every correction step"
    planted = tmp_path / "planted"
    planted.mkdir()
    (planted / "fhd_div.h").write_text(src.replace(good, "return q;"))
    exe = build(tmp_path, str(planted))
    r = subprocess.run([exe, "200000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 1
    n_bad = int(r.stdout.strip().split()[-1])
    assert n_bad > 1000, r.stdout
