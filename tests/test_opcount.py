"""Source-level operation counts behind the throughput roofline.

bench.py counts 224 FP64 operations per RK4 oculomotor orbit-step: four
right-hand sides of 35 operations (the reference's examples/oculomotor.cl,
branch-independent for y5 != 0) plus 14 per equation of RK4 stage arithmetic.
The counts come from compiling the system file with a counting scalar type
(oracle/opcount.cpp)."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# verbatim copies of the reference's files, staged by oracle/build.py
REFERENCE_ROOT = os.path.join(REPO, "baseline", "_ref")
OCM = ["120", "1.5", "0.0045", "0.05", "600", "9"]


def count(system_file, neq, npar, args, jacobian, tmp_path):
    exe = str(tmp_path / "opcount")
    cmd = ["g++", "-std=c++17", "-O0", "-DSYSTEM_FILE=\"%s\"" % system_file, "-DNUMEQ=%d" % neq,
           "-DNUMPAR=%d" % npar, os.path.join(REPO, "oracle", "opcount.cpp"), "-o", exe]
    if jacobian:
        cmd.insert(3, "-DHAS_JACOBIAN")
    subprocess.run(cmd, check=True)
    out = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, check=True).stdout
    return {line.split()[0]: int(line.split()[1]) for line in out.splitlines()}


def test_oculomotor_counts(tmp_path):
    path = os.path.join(REPO, "sodecl_b200", "systems", "oculomotor.cl")
    for y5 in ("2", "-2"):
        c = count(path, 6, 6, ["0"] * 5 + [y5] + OCM, True, tmp_path)
        # y3 - y4 is computed once here; the reference's text repeats it
        assert c["rhs"] == 33
        assert c["jacobian"] == 33


def test_kuramoto_counts(tmp_path):
    path = os.path.join(REPO, "sodecl_b200", "systems", "kuramoto.cl")
    for n in (4, 8):
        c = count(path, n, n + 1, list(range(n)) + [1] * (n + 1), False, tmp_path)
        assert c["rhs"] == 3 * n * n + 3 * n


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE_ROOT, "examples")), reason="the reference's files are not staged (oracle/build.py stages them where the reference checkout is present)")
def test_reference_oculomotor_rhs_count(tmp_path):
    c = count(os.path.join(REFERENCE_ROOT, "examples", "oculomotor.cl"), 6, 6, ["0"] * 5 + ["2"] + OCM, True, tmp_path)
    assert c["rhs"] == 35
    rk4_per_orbit_step = 4 * c["rhs"] + 6 * 14
    assert rk4_per_orbit_step == 224
    # Newton passes of the implicit solvers on this file (bench.py's implicit
    # midpoint roofline): a converged pass stops after the residual test, a
    # full pass adds the Jacobian, its scaling, the banded solve and the update
    assert c["jacobian"] == 33
    assert (c["ie_pass_converged"], c["ie_pass_full"]) == (59, 217)
    assert (c["im_pass_converged"], c["im_pass_full"]) == (78, 236)
