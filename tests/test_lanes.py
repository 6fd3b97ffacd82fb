"""Lanes per orbit (wide systems): several lanes of a warp share one orbit,
each evaluating some of its equations through the system file's
sode_system_row / sode_system_stoch_row.

Checked: the same records, states and draw counters as one thread per orbit,
bit for bit without FMA contraction (each row's arithmetic is the same
sequence of IEEE operations), and parity with the CPU oracle with contraction
on; odd sizes (rows and noise pairs not a multiple of the lanes, orbits not a
multiple of the orbits per block), FP32, and noise counters on the slow path
of the counter arithmetic (non-integers, values near 2^53).  The configuration
errors are checked without a GPU."""
import ctypes as C

import numpy as np
import pytest

from sodecl_b200 import _native as N
from sodecl_b200 import Integrator, system_path
from oracle.oracle import Oracle


def kuramoto_inputs(n, N_osc, nnoi, seed, counters="integer"):
    rng = np.random.default_rng(seed)
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1))] +
                       ([rng.uniform(0, 0.5, (n, N_osc))] if nnoi else []), axis=1)
    th0 = rng.uniform(0, 2 * np.pi, (n, N_osc))
    cnt = None
    if nnoi:
        if counters == "integer":
            cnt = rng.integers(0, 2 ** 40, n).astype(float)
        else:  # slow path: halves, and integers just below 2^53
            cnt = np.where(np.arange(n) % 2 == 0, rng.integers(0, 2 ** 20, n) + 0.5,
                           2.0 ** 53 - rng.integers(1, 40, n).astype(float))
    return np.zeros(n), th0, p, cnt


def run(solver, lanes, t0, y0, p, cnt, **kw):
    n = len(t0)
    with Integrator(system_path("kuramoto"), solver, orbits=n, lanes=lanes, **kw) as sim:
        sim.upload(t0, y0, p, cnt)
        rec = sim.run()
        t, y, c = sim.state()
        _, flags = sim.status()
    return rec, t, y, c, flags


# (oscillators, solver, noise processes, lanes)
CASES = [(32, "se", 32, 32), (32, "se", 32, 8), (5, "se", 5, 4), (33, "rk4", 0, 32), (16, "rk4", 0, 16),
         (8, "euler", 0, 4), (64, "rk4", 0, 32), (64, "se", 64, 16), (64, "ie", 0, 32), (16, "im", 0, 8),
         (5, "ie", 0, 4), (33, "im", 0, 32), (2, "ie", 0, 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("N_osc,solver,nnoi,lanes", CASES)
def test_lanes_match_one_thread_per_orbit_bit_for_bit(N_osc, solver, nnoi, lanes):
    n = 301
    t0, y0, p, cnt = kuramoto_inputs(n, N_osc, nnoi, N_osc + lanes)
    kw = dict(dt=0.01, tspan=1.0, ksteps=10, neq=N_osc, npar=p.shape[1], nnoi=nnoi, fmad=False)
    one = run(solver, 1, t0, y0, p, cnt, **kw)
    many = run(solver, lanes, t0, y0, p, cnt, **kw)
    for a, b in zip(one, many):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("N_osc,solver,nnoi,lanes", [(32, "se", 32, 32), (16, "rk4", 0, 8), (8, "euler", 0, 4),
                                                     (16, "ie", 0, 8), (8, "im", 0, 4)])
def test_lanes_parity_with_oracle(N_osc, solver, nnoi, lanes):
    from test_gpu_parity import assert_parity

    n = 300
    t0, y0, p, cnt = kuramoto_inputs(n, N_osc, nnoi, 11)
    kw = dict(dt=0.01, tspan=2.0, ksteps=20, neq=N_osc, npar=p.shape[1], nnoi=nnoi)
    rec, t, y, c, _ = run(solver, lanes, t0, y0, p, cnt, **kw)
    sid = {"se": 0, "euler": 1, "rk4": 2, "ie": 3, "im": 4}[solver]
    ref = Oracle("kuramoto").run(sid, t0, y0, p, counters=cnt, **kw)
    alt = Oracle("kuramoto", "fp64fma").run(sid, t0, y0, p, counters=cnt, **kw)
    assert_parity("lanes %d kuramoto N=%d %s" % (lanes, N_osc, solver), rec, ref.records, alt.records)
    if nnoi:
        np.testing.assert_array_equal(c, ref.counters)


@pytest.mark.gpu
def test_lanes_fp32_and_slow_counter_path():
    n = 200
    t0, y0, p, cnt = kuramoto_inputs(n, 12, 12, 5, counters="slow")
    kw = dict(dt=0.01, tspan=0.5, ksteps=10, neq=12, npar=p.shape[1], nnoi=12, fmad=False)
    for precision in ("fp64", "fp32"):
        one = run("se", 1, t0, y0, p, cnt, precision=precision, **kw)
        many = run("se", 8, t0, y0, p, cnt, precision=precision, **kw)
        for a, b in zip(one, many):
            np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_autotune_considers_lanes_and_keeps_results():
    n = 4096
    t0, y0, p, cnt = kuramoto_inputs(n, 32, 32, 3)
    kw = dict(dt=0.01, tspan=0.5, ksteps=10, neq=32, npar=p.shape[1], nnoi=32)
    with Integrator(system_path("kuramoto"), "se", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p, cnt)
        want = sim.run()
        sim.upload(t0, y0, p, cnt)
        choice = sim.autotune(sample_orbits=n, sample_steps=20)
        print("tuned:", choice)
        assert choice["lanes"] in (1, 4, 8, 16, 32)
        got = sim.run()
    from test_gpu_parity import rel_error

    err, nan_mismatch = rel_error(got, want)
    assert err < 1e-12 and nan_mismatch == 0


# ---------------------------------------------------------------- no GPU needed


@pytest.mark.gpu
@pytest.mark.parametrize("N_osc,solver,lanes,precision", [(64, "ie", 32, "fp64"), (16, "im", 8, "fp64"),
                                                          (33, "ie", 32, "fp32"), (20, "im", 16, "fp64")])
def test_row_band_hook_gives_the_same_records(N_osc, solver, lanes, precision):
    """With sode_system_row_band in the system file, a Newton pass takes a row's
    right-hand side and band from one evaluation (sin and cos from one
    sincos); without it, from sode_system_row and calc_jacobian_band.  The
    records, pass counts and flags are the same, with FMA contraction on."""
    n = 257
    t0, y0, p, _ = kuramoto_inputs(n, N_osc, 0, 7 * N_osc + lanes)
    src = open(system_path("kuramoto")).read()
    assert "sode_system_row_band(" in src
    outs = []
    for text in (src, src.replace("sode_system_row_band(", "unused_row_band(")):
        with Integrator(None, solver, orbits=n, lanes=lanes, dt=0.01, tspan=1.0, ksteps=10, neq=N_osc,
                        npar=p.shape[1], precision=precision, newton_tol=1e-7 if precision == "fp64" else 1e-4,
                        system_src=text) as sim:
            assert ("#define SODECL_HAS_ROW_BAND 1" in sim.program_source) == (text is src)
            sim.upload(t0, y0, p)
            rec = sim.run()
            passes, flags = sim.status()
        outs.append((rec, passes, flags))
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def _create(solver, lanes, system="kuramoto", neq=8, npar=9, nnoi=0, drop=None):
    cfg = N.Cfg()
    N.lib.sodecl_cfg_init(C.byref(cfg))
    cfg.solver, cfg.dt, cfg.int_time, cfg.kernel_steps = solver, 0.01, 1.0, 10
    cfg.num_equat, cfg.num_params, cfg.num_noi, cfg.list_size = neq, npar, nnoi, 64
    cfg.lanes_per_orbit = lanes
    ctx = C.c_void_p()
    rc = N.lib.sodecl_cuda_create(C.byref(cfg), C.byref(ctx))
    if rc != N.OK:
        return rc, None
    with open(system_path(system), "rb") as f:
        src = f.read()
    if drop:  # rename a function so the file no longer defines it
        src = src.replace(drop.encode() + b"(", b"unused_" + drop.encode() + b"(")
    rc = N.lib.sodecl_cuda_compile(ctx, src, len(src))
    return rc, ctx


@pytest.mark.parametrize("lanes", [3, 64, -1])
def test_lanes_must_be_a_power_of_two_up_to_32(lanes):
    rc, _ = _create(N.RUNGE_KUTTA, lanes)
    assert rc == N.ERR_INVALID_ARG


@pytest.mark.parametrize("solver,drop,nnoi", [(N.RUNGE_KUTTA, "sode_system_row", 0),
                                              (N.IMPLICIT_EULER, "calc_jacobian_band", 0),
                                              (N.IMPLICIT_MIDPOINT, "calc_jacobian_band", 0),
                                              (N.STOCHASTIC_EULER, "sode_system_stoch_row", 8)])
def test_lanes_need_the_row_functions(solver, drop, nnoi):
    rc, ctx = _create(solver, 4, nnoi=nnoi, npar=9 + nnoi)
    assert rc == N.OK
    N.lib.sodecl_cuda_destroy(ctx)
    rc, ctx = _create(solver, 4, nnoi=nnoi, npar=9 + nnoi, drop=drop)
    assert rc == N.ERR_UNSUPPORTED and drop in N.last_error(ctx)
    N.lib.sodecl_cuda_destroy(ctx)
    rc, ctx = _create(N.RUNGE_KUTTA, 4, system="oculomotor", neq=6, npar=6)
    assert rc == N.ERR_UNSUPPORTED and "sode_system_row" in N.last_error(ctx)
    N.lib.sodecl_cuda_destroy(ctx)


def test_lanes_program_compiles_without_gpu():
    rc, ctx = _create(N.STOCHASTIC_EULER, 16, neq=32, npar=65, nnoi=32)
    assert rc == N.OK
    src = N.program_source(ctx)
    assert "#define SODECL_LANES 16" in src and "#define SODECL_HAS_STOCH_ROW 1" in src
    N.lib.sodecl_cuda_destroy(ctx)
    rc, ctx = _create(N.IMPLICIT_EULER, 32, neq=64, npar=65)
    assert rc == N.OK
    assert "#define SODECL_HAS_ROW_BAND 1" in N.program_source(ctx)
    N.lib.sodecl_cuda_destroy(ctx)
    rc, ctx = _create(N.IMPLICIT_EULER, 32, neq=64, npar=65, drop="sode_system_row_band")
    assert rc == N.OK  # an accelerator only: the lanes still run without it
    assert "#define SODECL_HAS_ROW_BAND 0" in N.program_source(ctx)
    N.lib.sodecl_cuda_destroy(ctx)
