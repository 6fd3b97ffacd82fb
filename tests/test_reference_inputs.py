"""The reference's own inputs and callers, unchanged, through this library.

A user of the reference brings three things to the drop-in: their system
file (the reference ships examples/oculomotor.cl and examples/kuramoto.cl),
their Python code written against interfaces/python/sodecl.py, and their
expectations, which the reference pins in tests/sodecl_python_tests.py.
oracle/build.py stages verbatim copies of these files under baseline/_ref
(git-ignored; the GPU machines have no reference checkout), and here:

* the reference's known-answer test file runs unmodified, in a copy of its
  directory, with the reference's sodecl.py first on the import path and this
  library's sodecl_interface module under it;
* the reference's system files, as shipped, run through the C ABI for every
  solver they support, and their records are compared with the reference's
  own kernels compiled as C (oracle/_ref) on the same inputs, within the
  floor-based tolerance of tests/parity.py (the floor: the same file through
  the CPU restatement built with FMA contraction).
"""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from sodecl_b200 import _native as N
from sodecl_b200 import Integrator
from parity import assert_parity

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STAGED = os.path.join(REPO, "baseline", "_ref")
PACKAGE_DIR = os.path.join(REPO, "sodecl_b200")
REF_LIB_DIR = os.path.join(REPO, "oracle", "_ref")
NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])

needs_staged = pytest.mark.skipif(
    not os.path.isfile(os.path.join(STAGED, "tests", "sodecl_python_tests.py")),
    reason="the reference's files are not staged (oracle/build.py stages them where the reference checkout is present)")


def staged(rel):
    return os.path.join(STAGED, rel)


def reference_python_env():
    """Environment in which `import sodecl` finds the reference's sodecl.py
    and `import sodecl_interface` finds this library's module."""
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([staged("interfaces/python"), PACKAGE_DIR] +
                                        ([env["PYTHONPATH"]] if env.get("PYTHONPATH") else []))
    return env


@needs_staged
def test_reference_python_layer_binds_to_this_library():
    """No GPU needed: the reference's unmodified sodecl.py imports and its
    sodecl_interface is this library's pybind11 module."""
    code = "import sodecl, os; print(os.path.realpath(sodecl.__file__)); " \
           "print(os.path.realpath(sodecl.sodecl_interface.__file__))"
    out = subprocess.run([sys.executable, "-c", code], env=reference_python_env(), capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    sodecl_file, module_file = out.stdout.split()[-2:]
    assert sodecl_file == os.path.realpath(staged("interfaces/python/sodecl.py"))
    assert os.path.dirname(module_file) == os.path.realpath(PACKAGE_DIR)


@needs_staged
@pytest.mark.gpu
def test_reference_known_answer_tests_run_unmodified(tmp_path):
    """tests/sodecl_python_tests.py of the reference (Euler, RK4, implicit
    Euler and implicit midpoint on its oculomotor.cl, compared with its
    golden pickles by numpy.isclose), run as the reference runs it: from its
    own directory, through its own sodecl.py."""
    if N.device_count() < 1:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    work = tmp_path / "tests"
    shutil.copytree(staged("tests"), work)
    out = subprocess.run([sys.executable, "-m", "unittest", "-v", "sodecl_python_tests"], cwd=work,
                         env=reference_python_env(), capture_output=True, text=True, timeout=600)
    print(out.stdout[-4000:], out.stderr[-4000:])
    assert out.returncode == 0
    assert "Ran 4 tests" in out.stderr and "OK" in out.stderr.splitlines()[-1]
    # the manager's side effects in the working directory, as the reference
    # leaves them: the last call's log and its normal-exit line
    log = (work / "sodecllog.txt").read_text()
    assert "Selected device name: " in log and "Compute results runtime: " in log
    assert (work / "sodeclexitstatus.txt").read_text() == "1 Normal."
    assert (work / "Generated_kernel.cl").is_file()


def oculomotor_case(solver, n, seed):
    rng = np.random.default_rng(seed)
    nnoi = 2 if solver == 0 else 0
    p = NOMINAL * rng.uniform(0.5, 1.5, (n, 6))
    if nnoi:
        p = np.concatenate([p, rng.uniform(0.0, 0.01, (n, nnoi))], axis=1)
    dt = {0: 1e-5, 1: 1e-6, 2: 1e-5, 3: 1e-3, 4: 1e-3}[solver]
    cnt = np.arange(n) * 1000.0 if nnoi else None
    return np.zeros(n), np.tile(Y0, (n, 1)), p, cnt, dict(dt=dt, tspan=300 * dt, ksteps=30, neq=6, npar=6 + nnoi,
                                                          nnoi=nnoi)


def kuramoto_case(solver, n, seed, N_osc=8):
    rng = np.random.default_rng(seed)
    nnoi = N_osc if solver == 0 else 0
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1))] +
                       ([rng.uniform(0, 0.5, (n, N_osc))] if nnoi else []), axis=1)
    th0 = rng.uniform(0, 2 * np.pi, (n, N_osc))
    cnt = rng.integers(0, 2 ** 40, n).astype(float) if nnoi else None
    return np.zeros(n), th0, p, cnt, dict(dt=0.01, tspan=2.0, ksteps=20, neq=N_osc, npar=p.shape[1], nnoi=nnoi)


@needs_staged
@pytest.mark.gpu
@pytest.mark.parametrize("fmad", [0, 1])
@pytest.mark.parametrize("system,solver", [("oculomotor", s) for s in (0, 1, 2, 3, 4)] +
                         [("kuramoto", s) for s in (0, 1, 2)])
def test_reference_system_file_against_reference_kernels(system, solver, fmad):
    """examples/<system>.cl exactly as the reference ships it, through the C
    ABI, against the reference's kernels and the same file compiled as C."""
    from oracle.oracle import Oracle, ReferenceBuild

    if N.device_count() < 1:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    n = 1000  # not a multiple of the block size
    case = oculomotor_case if system == "oculomotor" else kuramoto_case
    t0, y0, p, cnt, kw = case(solver, n, 100 + solver)
    with Integrator(staged("examples/%s.cl" % system), solver, orbits=n, fmad=bool(fmad), **kw) as sim:
        sim.upload(t0, y0, p, cnt)
        rec = sim.run()
        t, y, c = sim.state()
    want = ReferenceBuild(system, solver).run(t0, y0, p, counters=cnt, **kw)
    alt = Oracle("refsys_" + system, "fp64fma", lib_dir=REF_LIB_DIR).run(solver, t0, y0, p, counters=cnt, **kw)
    assert_parity("examples/%s.cl solver %d fmad=%d" % (system, solver, fmad), rec, want.records, alt.records)
    np.testing.assert_array_equal(t, want.t)
    if cnt is not None:
        np.testing.assert_array_equal(c, want.counters)
