"""The adaptive solver (SODECL_DORMAND_PRINCE, solver 5): Dormand-Prince 5(4)
with per-orbit step sizes, records on the fixed-step solvers' grid.  The
reference has no variable-step solver (its README lists one as future work),
so nothing of the reference pins it; it is checked instead

  * on the CPU: the oracle's restatement against a fine fixed-step RK4 run of
    the reference's own algorithm (accuracy), and split runs against one run
    (the step size rides in the counters array);
  * on the GPU: against the oracle's restatement (same algorithm and order of
    operations; CUDA's exp and glibc's differ in the last bit, and step
    decisions can flip on that, so the bound is set by the tolerance, not by
    rounding), against fine RK4, across run splits bit for bit, and on the
    step limit."""
import re

import numpy as np
import pytest

from oracle.oracle import Oracle
from sodecl_b200 import _native as N
from sodecl_b200 import Integrator, system_path

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])
TOL = dict(rtol=1e-8, atol=1e-10)


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    return np.zeros(n), np.tile(Y0, (n, 1)), NOMINAL * rng.uniform(0.5, 1.5, (n, 6))


def rel(a, b, floor=1e-3):
    return float(np.max(np.abs(a - b) / (np.abs(b) + floor)))


def test_oracle_matches_fine_rk4():
    """rtol 1e-8: the records agree with RK4 at dt 1e-6 (itself accurate to
    about 1e-12 here) to 1e-6 of their scale, over stiff and mild orbits."""
    t0, y0, p = inputs(8, 1)
    o = Oracle("oculomotor")
    kw = dict(neq=6, npar=6, nchunks=4)
    dp = o.run(5, t0, y0, p, dt=1e-3, ksteps=50, counters=np.zeros(8), **kw, **TOL)
    ref = o.run(2, t0, y0, p, dt=1e-6, ksteps=50000, **kw)
    assert rel(dp.records, ref.records) < 1e-6
    assert (dp.flags == 0).all() and (dp.newton_passes > 0).all()
    np.testing.assert_allclose(dp.t, ref.t, rtol=1e-12)


def test_oracle_runs_split_equal_one_run():
    t0, y0, p = inputs(6, 2)
    o = Oracle("oculomotor")
    kw = dict(neq=6, npar=6, dt=1e-3, ksteps=20, **TOL)
    whole = o.run(5, t0, y0, p, nchunks=6, counters=np.zeros(6), **kw)
    a = o.run(5, t0, y0, p, nchunks=2, counters=np.zeros(6), **kw)
    b = o.run(5, a.t, a.y, p, nchunks=4, counters=a.counters, **kw)
    np.testing.assert_array_equal(np.concatenate([a.records, b.records[1:]]), whole.records)
    np.testing.assert_array_equal(b.counters, whole.counters)


def test_oracle_step_limit_gives_nan_and_flag():
    t0, y0, p = inputs(3, 3)
    r = Oracle("oculomotor").run(5, t0, y0, p, neq=6, npar=6, dt=1e-3, ksteps=50, nchunks=2, counters=np.zeros(3),
                                 rtol=1e-8, atol=1e-10, max_steps=3)
    assert (r.flags & 1).all()
    assert np.isnan(r.records[1:]).all() and np.isfinite(r.records[0]).all()


def test_oracle_kuramoto_and_fp32():
    """A second system (Kuramoto N=8, non-stiff) against fine RK4, and the FP32
    build against the FP64 one."""
    rng = np.random.default_rng(9)
    n, N = 6, 8
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N), (n, 1))], axis=1)
    th0 = rng.uniform(0, 2 * np.pi, (n, N))
    kw = dict(neq=N, npar=N + 1, nchunks=5)
    o = Oracle("kuramoto")
    dp = o.run(5, np.zeros(n), th0, p, dt=0.01, ksteps=20, counters=np.zeros(n), **kw, **TOL)
    ref = o.run(2, np.zeros(n), th0, p, dt=1e-4, ksteps=2000, **kw)
    assert rel(dp.records, ref.records, floor=1.0) < 1e-7
    assert (dp.newton_passes < 5 * 20).all()  # far fewer steps than the fixed-step grid
    t0, y0, pp = inputs(4, 10)
    f64 = Oracle("oculomotor").run(5, t0, y0, pp, neq=6, npar=6, dt=1e-3, ksteps=50, nchunks=2,
                                   counters=np.zeros(4), rtol=1e-5, atol=1e-7)
    f32 = Oracle("oculomotor", "fp32").run(5, t0, y0, pp, neq=6, npar=6, dt=1e-3, ksteps=50, nchunks=2,
                                           counters=np.zeros(4), rtol=1e-5, atol=1e-7)
    assert (f32.flags == 0).all() and rel(f32.records, f64.records, floor=0.1) < 1e-2


def test_program_carries_tolerances():
    sim = Integrator(system_path("oculomotor"), "dp45", dt=1e-3, tspan=0.1, ksteps=10, neq=6, npar=6, orbits=4,
                     rtol=2.5e-7, atol=1e-11, max_steps=777)
    src = sim.program_source
    assert "#define SODECL_SOLVER 5" in src and "#define SODECL_MAX_STEPS 777" in src
    # the tolerances as exact hexadecimal literals
    assert float.fromhex(re.search(r"#define SODECL_RTOL (\S+)", src).group(1)) == 2.5e-7
    assert float.fromhex(re.search(r"#define SODECL_ATOL (\S+)", src).group(1)) == 1e-11
    sim.close()
    with pytest.raises(N.SodeclError):
        Integrator(system_path("kuramoto"), "dp45", dt=0.01, tspan=0.1, ksteps=10, neq=16, npar=17, orbits=4, lanes=8)


# ---------------------------------------------------------------------------
# GPU


def run_gpu(t0, y0, p, solver="dp45", h0=None, **kw):
    with Integrator(system_path("oculomotor"), solver, orbits=len(t0), **kw) as sim:
        sim.upload(t0, y0, p, h0)
        rec = sim.run()
        t, y, h = sim.state()
        passes, flags = sim.status()
    return rec, t, y, h, passes, flags


@pytest.mark.gpu
@pytest.mark.parametrize("fmad", [False, True])
def test_gpu_matches_oracle_and_fine_rk4(fmad):
    n = 3000
    t0, y0, p = inputs(n, 4)
    kw = dict(dt=1e-3, tspan=0.2, ksteps=50, neq=6, npar=6)
    rec, t, y, h, passes, flags = run_gpu(t0, y0, p, fmad=fmad, **kw, **TOL)
    assert (flags == 0).all()
    idx = np.random.default_rng(5).choice(n, 64, replace=False)
    o = Oracle("oculomotor")
    want = o.run(5, t0[idx], y0[idx], p[idx], neq=6, npar=6, dt=1e-3, ksteps=50, nchunks=4,
                 counters=np.zeros(idx.size), **TOL)
    g = rec[:, :, idx]
    # same algorithm; step decisions may flip on last-bit differences of exp,
    # so the two agree to the tolerance's scale, not to rounding (the scale
    # floor 0.1: some components pass through values near 1e-4, where both
    # carry the same absolute error of about 1e-8)
    assert rel(g, want.records, floor=0.1) < 1e-6
    np.testing.assert_array_equal(t[idx], want.t)  # every interval lands on its end exactly
    # accepted steps: equal for most orbits
    assert np.mean(passes[idx] == want.newton_passes) > 0.8
    # accuracy against RK4 at dt 1e-6 on the GPU: the same error distribution
    # as the oracle's against the same reference
    fine, *_ = run_gpu(t0[idx], y0[idx], p[idx], solver="rk4", fmad=fmad, dt=1e-6, tspan=0.2, ksteps=50000, neq=6,
                       npar=6)
    # 0.2 / (1e-6 * 50000) rounds just above 4, so the reference's count adds an interval
    fine = fine[:rec.shape[0]]
    assert rel(g, fine, floor=0.1) < 1e-6
    per_orbit = lambda a: np.max(np.abs(a - fine) / (np.abs(fine) + 1e-3), axis=(0, 1))  # noqa: E731
    assert np.median(per_orbit(g)) < 2 * np.median(per_orbit(want.records)) + 1e-9


@pytest.mark.gpu
def test_gpu_split_runs_equal_one_run():
    """The step sizes ride in the counters array, and the first stage is
    re-evaluated at every interval's start: a run split in two (the state and
    step sizes carried on the device) gives the records of one run, bit for
    bit, whatever the grouping of intervals into launches."""
    n = 2000
    t0, y0, p = inputs(n, 6)
    kw = dict(dt=1e-3, ksteps=25, neq=6, npar=6, **TOL)
    whole, *_ = run_gpu(t0, y0, p, tspan=0.2, **kw)
    with Integrator(system_path("oculomotor"), "dp45", orbits=n, tspan=0.1, **kw) as sim:
        sim.upload(t0, y0, p)
        a = sim.run()
        b = sim.run()
    np.testing.assert_array_equal(np.concatenate([a, b[1:]]), whole)


@pytest.mark.gpu
def test_gpu_launch_shapes_agree():
    """The adaptive kernel's warps hand out ranges of orbits to their lanes,
    and the host launches only the blocks that give each lane the fewest
    orbits that fit the resident threads.  Block sizes that are not a multiple
    of 32, more orbits than resident threads (several orbits a lane) and a
    register cap all give each orbit the records, step sizes, accepted-step
    counts and flags of integrating it alone, bit for bit."""
    n = 150000
    t0, y0, p = inputs(n, 8)
    kw = dict(dt=1e-3, tspan=0.06, ksteps=20, neq=6, npar=6, rtol=1e-6, atol=1e-9)
    outs = []
    for block, minb in ((128, 0), (100, 0), (33, 0), (512, 0), (128, 2)):
        rec, t, y, h, passes, flags = run_gpu(t0, y0, p, block=block, min_blocks=minb, **kw)
        outs.append((rec, h, passes, flags))
    for got in outs[1:]:
        for x, want in zip(got, outs[0]):
            np.testing.assert_array_equal(x, want)
    # a few orbits alone
    idx = [0, 1, 77, 4097, n - 1]
    rec1, _, _, h1, passes1, flags1 = run_gpu(t0[idx], y0[idx], p[idx], **kw)
    np.testing.assert_array_equal(rec1, outs[0][0][:, :, idx])
    np.testing.assert_array_equal(h1, outs[0][1][idx])
    np.testing.assert_array_equal(passes1, outs[0][2][idx])
    np.testing.assert_array_equal(flags1, outs[0][3][idx])


@pytest.mark.gpu
def test_gpu_step_limit_and_fp32():
    n = 500
    t0, y0, p = inputs(n, 7)
    rec, _, _, _, _, flags = run_gpu(t0, y0, p, dt=1e-3, tspan=0.1, ksteps=50, neq=6, npar=6, rtol=1e-8, atol=1e-10,
                                     max_steps=3)
    assert (flags & N.FLAG_NEWTON_CAP).all() and np.isnan(rec[1:]).all()
    r64, *_ = run_gpu(t0, y0, p, dt=1e-3, tspan=0.1, ksteps=50, neq=6, npar=6, rtol=1e-5, atol=1e-7)
    r32, _, _, _, _, f32 = run_gpu(t0, y0, p, dt=1e-3, tspan=0.1, ksteps=50, neq=6, npar=6, rtol=1e-5, atol=1e-7,
                                   precision="fp32")
    assert (f32 == 0).all()
    # FP32 at rtol 1e-5 on this stiff model: float rounding accumulates over
    # thousands of adaptive steps; measured 1.3e-3 of the state's scale
    assert rel(r32, r64, floor=0.1) < 1e-2
