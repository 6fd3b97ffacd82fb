"""The C ABI library on a machine without a GPU: it loads, exports every entry
point include/sodecl_cuda.h declares, validates configurations, and builds
programs with NVRTC (which needs no device).  Failure paths return the
documented status codes."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from sodecl_b200 import _native as N
from sodecl_b200 import Integrator, system_path

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "sodecl_cuda.h")
# verbatim copies of the reference's files, staged by oracle/build.py
REFERENCE_ROOT = os.path.join(REPO, "baseline", "_ref")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sodecl_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the ctypes binding declares each of them
    assert sorted(N.SIGNATURES) == names


def test_abi_version_and_strerror():
    assert N.lib.sodecl_cuda_abi_version() == N.ABI_VERSION == 4
    assert N.lib.sodecl_cuda_strerror(N.ERR_NO_JACOBIAN).decode().startswith("implicit solver")


def _cfg(**kw):
    cfg = N.Cfg()
    N.lib.sodecl_cfg_init(C.byref(cfg))
    base = dict(solver=2, dt=1e-3, int_time=1.0, kernel_steps=10, num_equat=6, num_params=6, list_size=8)
    base.update(kw)
    for k, v in base.items():
        setattr(cfg, k, v)
    return cfg


def _create(**kw):
    ctx = C.c_void_p()
    rc = N.lib.sodecl_cuda_create(C.byref(_cfg(**kw)), C.byref(ctx))
    return rc, ctx


def test_cfg_defaults():
    cfg = N.Cfg()
    N.lib.sodecl_cfg_init(C.byref(cfg))
    assert cfg.solver == N.EULER and cfg.fmad == 1 and cfg.precision == N.FP64
    assert cfg.newton_tol == 1e-7 and cfg.newton_max_iter == 1000
    assert cfg.rtol == 1e-6 and cfg.atol == 1e-9 and cfg.max_steps == 100000


@pytest.mark.parametrize("bad", [dict(solver=6), dict(solver=-1), dict(num_equat=0), dict(list_size=0),
                                 dict(solver=5, rtol=0.0), dict(solver=5, atol=-1.0), dict(solver=5, max_steps=0),
                                 dict(solver=5, rtol=float("inf")), dict(solver=5, lanes_per_orbit=4),
                                 dict(dt=0.0), dict(dt=float("nan")), dict(kernel_steps=0),
                                 dict(solver=0, num_noi=0), dict(precision=2), dict(int_time=-1.0),
                                 dict(local_group_size=2048), dict(dt=1e-12, int_time=1.0, kernel_steps=1)])
def test_create_rejects_invalid_configuration(bad):
    rc, ctx = _create(**bad)
    assert rc == N.ERR_INVALID_ARG
    assert not ctx.value


def test_record_count():
    rc, ctx = _create(dt=1e-6, int_time=0.1, kernel_steps=400)
    assert rc == N.OK
    assert N.lib.sodecl_cuda_num_records(ctx) == 252
    N.lib.sodecl_cuda_destroy(ctx)


def _compile(ctx, src):
    b = src.encode() if isinstance(src, str) else src
    return N.lib.sodecl_cuda_compile(ctx, b, len(b))


@pytest.mark.parametrize("solver", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("precision", [0, 1])
def test_compile_every_solver_without_gpu(solver, precision):
    nnoi = 2 if solver == 0 else 0
    rc, ctx = _create(solver=solver, num_noi=nnoi, num_params=6 + nnoi, precision=precision)
    assert rc == N.OK
    src = open(system_path("oculomotor")).read()
    assert _compile(ctx, src) == N.OK, N.last_error(ctx)
    text = N.program_source(ctx)
    # the reference's program defines, same names and printed values
    for line in ("#define _numnoi_ %d" % nnoi, "#define _numsteps_ 10", "#define _numeq_ 6",
                 "#define _numpar_ %d" % (6 + nnoi)):
        assert line in text
    assert ("#define _m_dt_ 0.001f" if precision else "#define _m_dt_ 0.001\n") in text
    assert "ptxas" in N.build_log(ctx)  # resource usage is reported
    N.lib.sodecl_cuda_destroy(ctx)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("tol", [1e-7, 1e-10, 3e-5, 1e-3, 0.5, 7.25e-13])
def test_midpoint_stop_bound_is_exact(precision, tol):
    """The implicit midpoint stops when sqrt(norm) < tol (src/kernels/im.cl);
    the program tests norm < t instead, with t from the host: the least value
    whose correctly rounded square root reaches tol.  Both tests agree for every
    norm exactly when sqrt(t) >= tol > sqrt(t's predecessor)."""
    rc, ctx = _create(solver=N.IMPLICIT_MIDPOINT, precision=precision, newton_tol=tol)
    assert rc == N.OK
    assert _compile(ctx, open(system_path("oculomotor")).read()) == N.OK, N.last_error(ctx)
    text = N.program_source(ctx)
    N.lib.sodecl_cuda_destroy(ctx)
    m = re.search(r"#define SODECL_L2_BOUND (\S+)", text)
    assert m, "no bound in the program"
    ft = np.float32 if precision else np.float64
    t = ft(float.fromhex(m.group(1).rstrip("f")))
    # tol as the program's _epsilon1_ literal reads it (float literals parse straight to float)
    eps_text = re.search(r"#define _epsilon1_ (\S+)", text).group(1).rstrip("f").encode()
    libc = C.CDLL(None)
    libc.strtof.restype, libc.strtod.restype = C.c_float, C.c_double
    libc.strtof.argtypes = libc.strtod.argtypes = [C.c_char_p, C.c_void_p]
    eps = ft(libc.strtof(eps_text, None) if precision else libc.strtod(eps_text, None))
    assert np.sqrt(t) >= eps and np.sqrt(np.nextafter(t, ft(0))) < eps
    v = t
    for _ in range(64):  # and on either side of it
        v = np.nextafter(v, ft(0))
    for _ in range(128):
        assert (np.sqrt(v) < eps) == (v < t)
        v = np.nextafter(v, ft(np.inf))


@pytest.mark.parametrize("division,scalar", [(N.DIV_IEEE, "float"), (N.DIV_RECIPROCAL, "sodecl_num")])
def test_fp32_program_rewrites_literals(division, scalar):
    rc, ctx = _create(precision=1, division=division)
    assert _compile(ctx, open(system_path("oculomotor")).read()) == N.OK
    text = N.program_source(ctx)
    assert "#define double %s" % scalar in text
    assert "#define OCM_T1 0.15f" in text and "(1.00f / p[2])" in text
    assert "/* burst-neuron firing-rate non-linearity:" in text  # comments untouched
    N.lib.sodecl_cuda_destroy(ctx)


def test_zero_size_parameter_bounds_are_relaxed():
    # the system file declares `double noise[_numnoi_]`; _numnoi_ is 0 for ODE runs
    rc, ctx = _create(solver=2)
    assert _compile(ctx, open(system_path("oculomotor")).read()) == N.OK
    text = N.program_source(ctx)
    assert re.search(r"double noise\[\s*\]", text)
    assert re.search(r"double jac\[\s*\]\[_numeq_\]", text)
    N.lib.sodecl_cuda_destroy(ctx)


def test_missing_jacobian_and_stochastic_term():
    kura = open(system_path("kuramoto")).read()
    no_jac = re.sub(r"void calc_jacobian.*?\n}\n", "", kura, flags=re.S)
    assert "void calc_jacobian" not in no_jac
    rc, ctx = _create(solver=3, num_equat=4, num_params=5)
    assert _compile(ctx, no_jac) == N.ERR_NO_JACOBIAN
    assert "calc_jacobian" in N.last_error(ctx)
    N.lib.sodecl_cuda_destroy(ctx)
    no_stoch = re.sub(r"void sode_system_stoch.*?\n}\n", "", kura, flags=re.S)
    rc, ctx = _create(solver=0, num_equat=4, num_params=9, num_noi=4)
    assert _compile(ctx, no_stoch) == N.ERR_NO_STOCH
    N.lib.sodecl_cuda_destroy(ctx)


def test_compile_error_reports_nvrtc_log():
    rc, ctx = _create()
    bad = "void sode_system(double t, double y[_numeq_], double yout[_numeq_], double p[_numpar_]) { yout[0] = y[0] +; }"
    assert _compile(ctx, bad) == N.ERR_COMPILE
    assert "error" in N.last_error(ctx)
    assert _compile(ctx, "int nothing_here;") == N.ERR_COMPILE  # no sode_system
    N.lib.sodecl_cuda_destroy(ctx)


def test_out_of_order_calls():
    rc, ctx = _create()
    out = np.zeros(10)
    assert N.lib.sodecl_cuda_run(ctx, out.ctypes.data, out.size) == N.ERR_STATE
    assert N.lib.sodecl_cuda_download_state(ctx, None, None, None) == N.ERR_STATE
    z = np.zeros(48)
    # upload before compile
    assert N.lib.sodecl_cuda_upload(ctx, z.ctypes.data, z.ctypes.data, z.ctypes.data, None) == N.ERR_STATE
    assert N.lib.sodecl_cuda_upload(None, None, None, None, None) == N.ERR_INVALID_ARG
    N.lib.sodecl_cuda_destroy(ctx)
    N.lib.sodecl_cuda_destroy(None)


@pytest.mark.skipif(N.device_count() > 0, reason="checks the no-device path")
def test_no_device_is_reported():
    sim = Integrator(system_path("oculomotor"), "rk4", dt=1e-3, tspan=0.01, ksteps=10, neq=6, npar=6, orbits=4)
    with pytest.raises(N.SodeclError) as e:
        sim.upload(np.zeros(4), np.zeros(24), np.ones(24))
    assert e.value.status == N.ERR_NO_DEVICE
    assert N.lib.sodecl_cuda_noise_stream(0, np.zeros(1, np.int64).ctypes.data, np.zeros(1).ctypes.data, 1, 2, 0.1, 1,
                                          np.zeros(2).ctypes.data, None, None) == N.ERR_NO_DEVICE


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE_ROOT, "examples")), reason="the reference's files are not staged (oracle/build.py stages them where the reference checkout is present)")
@pytest.mark.parametrize("path,solvers", [("examples/oculomotor.cl", [0, 1, 2, 3, 4]), ("tests/oculomotor.cl", [2, 4]),
                                          ("examples/kuramoto.cl", [0, 1, 2]), ("tests/kuramoto.cl", [0, 1])])
def test_reference_system_files_compile_unchanged(path, solvers):
    """Drop-in: the reference's own system files build as they are."""
    src = open(os.path.join(REFERENCE_ROOT, path)).read()
    neq = 6 if "oculomotor" in path else 5
    for solver in solvers:
        nnoi = (2 if neq == 6 else neq) if solver == 0 else 0
        npar = (6 if neq == 6 else neq + 1) + nnoi
        rc, ctx = _create(solver=solver, num_equat=neq, num_params=npar, num_noi=nnoi)
        assert rc == N.OK
        assert _compile(ctx, src) == N.OK, N.last_error(ctx)
        N.lib.sodecl_cuda_destroy(ctx)


def test_python_module_fails_cleanly_without_device(tmp_path, monkeypatch):
    """Without a device the call returns an empty list.  The manager still
    leaves the reference's side effects in the working directory: the
    assembled program (built without a GPU), sodecllog.txt (started empty; no
    run, so nothing appended) and sodeclexitstatus.txt with the normal-exit
    line its destructor writes."""
    from sodecl_b200 import sodecl_interface

    if N.device_count() > 0:
        pytest.skip("checks the no-device path")
    monkeypatch.chdir(tmp_path)
    (tmp_path / "sodecllog.txt").write_text("left over from an earlier call")
    out = sodecl_interface.sodeclcall([0.0], [0, 0, 0, 0, 0, 2.0], [120, 1.5, 0.0045, 0.05, 600, 9.0], 0, 0,
                                      system_path("oculomotor"), 2, 1, 6, 6, 0, 1e-3, 0.01, 10, 0)
    assert out == []
    assert (tmp_path / "Generated_kernel.cl").read_text().startswith("// SODECL program generated")
    assert (tmp_path / "sodecllog.txt").read_text() == ""
    assert (tmp_path / "sodeclexitstatus.txt").read_text() == "1 Normal."
    out = sodecl_interface.sodeclcall([0.0], [0.0] * 6, [1.0] * 6, 0, 0, system_path("oculomotor"), 9, 1, 6, 6, 0,
                                      1e-3, 0.01, 10, 0)
    assert out == []


def test_division_modes_and_fallback():
    """The default: the reciprocal quotient in FP64, IEEE division in FP32 and
    for the adaptive solver;
    either precision builds the reciprocal form when asked.  A system file
    that needs the plain scalar (an implicit conversion) falls back to IEEE
    division."""
    kw = dict(dt=1e-3, tspan=0.1, ksteps=10, neq=6, npar=6, orbits=4)
    assert Integrator(system_path("oculomotor"), "rk4", division="reciprocal", **kw).division == "reciprocal"
    assert Integrator(system_path("oculomotor"), "rk4", **kw).division == "reciprocal"  # the default
    assert Integrator(system_path("oculomotor"), "rk4", division="ieee", **kw).division == "ieee"
    assert Integrator(system_path("oculomotor"), "rk4", precision="fp32", **kw).division == "ieee"  # the default
    assert Integrator(system_path("oculomotor"), "dp45", **kw).division == "ieee"  # the default
    assert Integrator(system_path("oculomotor"), "dp45", division="reciprocal", **kw).division == "reciprocal"
    assert Integrator(system_path("oculomotor"), "rk4", division="reciprocal", precision="fp32",
                      **kw).division == "reciprocal"
    assert Integrator(system_path("oculomotor"), "rk4", division="ieee", precision="fp32", **kw).division == "ieee"
    src = open(system_path("oculomotor")).read().replace("double drive = y[3] - y[4];", "float drive = y[3] - y[4];")
    for prec in ("fp64", "fp32"):
        sim = Integrator(None, "rk4", system_src=src, division="reciprocal", precision=prec, **kw)
        assert sim.division == "ieee"
        assert "#define SODECL_FAST_DIV 0" in sim.program_source
    text = Integrator(system_path("oculomotor"), "rk4", division="reciprocal", **kw).program_source
    assert "#define SODECL_FAST_DIV 1" in text and "#define double sodecl_num" in text
    with pytest.raises(ValueError):
        Integrator(system_path("oculomotor"), "rk4", division="fast", **kw)


def test_get_cfg_returns_the_configuration():
    cfg = N.Cfg()
    N.lib.sodecl_cfg_init(C.byref(cfg))
    cfg.solver, cfg.dt, cfg.int_time, cfg.kernel_steps = N.RUNGE_KUTTA, 1e-5, 1e-4, 10
    cfg.num_equat, cfg.num_params, cfg.list_size, cfg.local_group_size = 6, 6, 16, 96
    ctx = C.c_void_p()
    assert N.lib.sodecl_cuda_create(C.byref(cfg), C.byref(ctx)) == N.OK
    back = N.Cfg()
    assert N.lib.sodecl_cuda_get_cfg(ctx, C.byref(back)) == N.OK
    assert bytes(back) == bytes(cfg)
    assert N.lib.sodecl_cuda_get_cfg(None, C.byref(back)) == N.ERR_INVALID_ARG
    N.lib.sodecl_cuda_destroy(ctx)
