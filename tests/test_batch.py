"""Heterogeneous batches: one persistent kernel over orbits of several system x
solver classes with per-orbit step counts (sodecl_batch_* C ABI).

Every orbit of a batch runs the same device code as the single-system kernel
(sodecl_advance), so its final state must equal, bit for bit, what the
single-system kernel gives for that orbit alone; that kernel is itself checked
against the oracle in test_gpu_parity.py."""
import re

import numpy as np
import pytest

from sodecl_b200 import _native as N
from sodecl_b200 import Integrator, system_path
from sodecl_b200.batch import Batch

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])

# (system, solver, neq, npar, nnoi, dt)
CLASSES = [("kuramoto", "euler", 4, 5, 0, 0.01), ("kuramoto", "rk4", 16, 17, 0, 0.01),
           ("kuramoto", "ie", 8, 9, 0, 0.01), ("oculomotor", "rk4", 6, 6, 0, 1e-5),
           ("oculomotor", "ie", 6, 6, 0, 1e-3), ("kuramoto", "se", 5, 11, 5, 0.01),
           ("oculomotor", "im", 6, 6, 0, 1e-3)]


def make_batch(fmad=True, classes=CLASSES):
    b = Batch(fmad=fmad)
    for system, solver, neq, npar, nnoi, dt in classes:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt)
    return b.compile()


def make_items(n, seed, classes=CLASSES, steps=(0, 1, 7, 50, 123, 400)):
    rng = np.random.default_rng(seed)
    cls = rng.integers(0, len(classes), n).astype(np.int32)
    nsteps = rng.choice(steps, n).astype(np.int64)
    t0 = rng.uniform(0, 1, n)
    y0, p = [], []
    for c in cls:
        system, solver, neq, npar, nnoi, dt = classes[c]
        if system == "oculomotor":
            y0.append(Y0.copy())
            p.append(NOMINAL * rng.uniform(0.5, 1.5, 6))
        else:
            y0.append(rng.uniform(0, 2 * np.pi, neq))
            q = np.concatenate([[rng.uniform(0, 5)], rng.normal(size=neq)])
            if nnoi:
                q = np.concatenate([q, rng.uniform(0, 0.5, nnoi)])
            p.append(q)
    counters = rng.integers(0, 2 ** 40, n).astype(float)
    return cls, nsteps, t0, y0, p, counters


def test_batch_program_builds_without_gpu():
    b = make_batch()
    text = b.program_source
    assert len(re.findall(r"namespace sodecl_cls_\d+ \{", text)) == len(CLASSES)
    assert "sodecl_batch(const sodecl_batch_args a)" in text
    assert len(re.findall(r"case \d+: sodecl_cls_\d+::sodecl_class_run", text)) == len(CLASSES)


def test_batch_validation():
    b = Batch()
    kura = open(system_path("kuramoto")).read()
    no_jac = re.sub(r"void calc_jacobian.*?\n}\n", "", kura, flags=re.S)
    with pytest.raises(N.SodeclError) as e:
        b.add_class(None, "ie", neq=4, npar=5, dt=0.01, system_src=no_jac)
    assert e.value.status == N.ERR_NO_JACOBIAN
    with pytest.raises(N.SodeclError):
        b.add_class(system_path("kuramoto"), "rk4", neq=0, npar=1, dt=0.01)
    with pytest.raises(N.SodeclError):
        b.add_class(system_path("kuramoto"), "se", neq=4, npar=5, dt=0.01)  # noise without processes
    for _ in range(32):
        b.add_class(system_path("kuramoto"), "euler", neq=2, npar=3, dt=0.01)
    with pytest.raises(N.SodeclError):
        b.add_class(system_path("kuramoto"), "euler", neq=2, npar=3, dt=0.01)
    with pytest.raises(N.SodeclError) as e:
        Batch().set_items([0], [1], [0.0], [0.0], [0.0])
    assert e.value.status == N.ERR_STATE


def single_kernel_final_state(system, solver, neq, npar, nnoi, dt, nsteps, t0, y0, p, counters, gid, fmad):
    """The same orbit through the single-system kernel, as the tail of a list
    so its noise stream is keyed by the same global orbit index."""
    if nsteps == 0:
        return t0, y0, counters
    n = gid + 1
    with Integrator(system_path(system), solver, dt=dt, tspan=nsteps * dt, ksteps=nsteps, neq=neq, npar=npar,
                    nnoi=nnoi, orbits=n, fmad=fmad) as sim:
        assert sim.num_chunks == 1
        sim.upload(np.full(n, t0), np.tile(y0, (n, 1)), np.tile(p, (n, 1)),
                   np.full(n, counters) if nnoi else None)
        sim.run(discard=True)
        t, y, c = sim.state()
    return t[gid], y[gid], c[gid]


@pytest.mark.gpu
@pytest.mark.parametrize("fmad", [False, True])
def test_batch_matches_single_system_kernel_bit_for_bit(fmad):
    """Without FMA contraction both kernels evaluate every operation as
    written, so the states agree bit for bit.  With contraction (fmad=1) the
    compiler chooses which products to fuse separately in the two programs, so
    last-bit differences may appear and grow over the steps: there the states
    agree to 1e-9 relative (the parity tolerance of these step counts), the
    times and draw counters exactly."""
    n = 3000
    cls, nsteps, t0, y0, p, counters = make_items(n, 1)
    b = make_batch(fmad)
    b.set_items(cls, nsteps, t0, y0, p, counters)
    b.run(graph=False)
    t, y, cnt, passes, flags = b.results()
    rng = np.random.default_rng(2)
    for i in rng.choice(n, 60, replace=False):
        system, solver, neq, npar, nnoi, dt = CLASSES[cls[i]]
        tt, yy, cc = single_kernel_final_state(system, solver, neq, npar, nnoi, dt, nsteps[i], t0[i], y0[i], p[i],
                                               counters[i], i, fmad)
        if fmad:
            np.testing.assert_allclose(y[i], yy, rtol=1e-9, atol=1e-12 * np.abs(yy).max())
        else:
            np.testing.assert_array_equal(y[i], yy)
        assert t[i] == tt
        if nnoi:
            assert cnt[i] == cc
    # orbits with no steps come back untouched
    zero = nsteps == 0
    assert np.array_equal(t[zero], t0[zero])


@pytest.mark.gpu
def test_batch_graph_replay_continues_from_state():
    n = 2000
    cls, nsteps, t0, y0, p, counters = make_items(n, 3)
    b = make_batch()
    b.set_items(cls, nsteps, t0, y0, p, counters)
    b.run(graph=True)
    b.run(graph=True)  # replay: a second pass from the stored states
    t2, y2, c2, _, _ = b.results()
    b2 = make_batch()
    b2.set_items(cls, 2 * nsteps, t0, y0, p, counters)
    b2.run(graph=False)
    t, y, c, _, _ = b2.results()
    np.testing.assert_array_equal(np.concatenate(y2), np.concatenate(y))
    np.testing.assert_array_equal(t2, t)
    np.testing.assert_array_equal(c2, c)


@pytest.mark.gpu
def test_batch_tuner_and_launch_shapes_agree():
    n = 4000
    cls, nsteps, t0, y0, p, counters = make_items(n, 4)
    outs = []
    for shape in ((64, 0), (256, 1)):
        b = make_batch()
        b.set_items(cls, nsteps, t0, y0, p, counters)
        b.set_launch(*shape)
        b.run()
        outs.append(np.concatenate(b.results()[1]))
    np.testing.assert_array_equal(outs[0], outs[1])
    b = make_batch()
    b.set_items(cls, nsteps, t0, y0, p, counters)
    block, bps, ms = b.tune()
    assert block in (64, 128, 256) and ms > 0


@pytest.mark.gpu
def test_batch_tuner_picks_lanes_and_keeps_results():
    """The tuner times lanes per orbit for automatic classes (program rebuilt
    per candidate); whatever it picks, the states equal the untuned run's bit
    for bit without FMA contraction."""
    classes = [c[:6] for c in LANES_CLASSES]
    n = 600
    cls, nsteps, t0, y0, p, counters = make_items(n, 8, classes=classes, steps=(0, 1, 7, 50))

    def build():
        b = Batch(fmad=False)
        for system, solver, neq, npar, nnoi, dt, lanes in LANES_CLASSES:
            b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt, lanes=lanes)
        return b.compile()

    want = build()
    want.set_items(cls, nsteps, t0, y0, p, counters)
    want.run()
    tuned = build()
    tuned.set_items(cls, nsteps, t0, y0, p, counters)
    tuned.tune()
    lanes = tuned.lanes
    print("tuned lanes per class:", lanes)
    assert lanes[0] == 32 and lanes[2] == 4  # explicit choices are kept
    tuned.set_items(cls, nsteps, t0, y0, p, counters)
    tuned.run()
    for a, b in zip(want.results(), tuned.results()):
        if isinstance(a, list):
            np.testing.assert_array_equal(np.concatenate(a), np.concatenate(b))
        else:
            np.testing.assert_array_equal(a, b)


# (system, solver, neq, npar, nnoi, dt, lanes): wide classes with lanes per orbit
# (0: automatic), next to one-lane classes in the same program
LANES_CLASSES = [("kuramoto", "ie", 64, 65, 0, 0.01, 32), ("kuramoto", "se", 32, 65, 32, 0.01, 0),
                 ("kuramoto", "rk4", 16, 17, 0, 0.01, 4), ("kuramoto", "euler", 12, 13, 0, 0.01, 0),
                 ("kuramoto", "im", 20, 21, 0, 0.01, 8), ("kuramoto", "rk4", 4, 5, 0, 0.01, 0),
                 ("oculomotor", "ie", 6, 6, 0, 1e-3, 0)]


def test_batch_lanes_program_builds_without_gpu():
    b = Batch(fmad=False)
    for system, solver, neq, npar, nnoi, dt, lanes in LANES_CLASSES:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt, lanes=lanes)
    text = b.compile().program_source
    lanes = [int(x) for x in re.findall(r"#define SODECL_NEWTON_MAX \d+\n#define SODECL_LANES (\d+)", text)]
    assert lanes == [32, 16, 4, 8, 8, 1, 1]
    assert re.search(r"#define SODECL_BATCH_WARP_WORDS [1-9]\d*", text)
    with pytest.raises(N.SodeclError) as e:
        Batch().add_class(system_path("oculomotor"), "rk4", neq=6, npar=6, dt=1e-5, lanes=4)
    assert e.value.status == N.ERR_UNSUPPORTED


@pytest.mark.gpu
def test_batch_lanes_classes_match_single_system_kernel_bit_for_bit():
    classes = [c[:6] for c in LANES_CLASSES]
    b = Batch(fmad=False)
    for system, solver, neq, npar, nnoi, dt, lanes in LANES_CLASSES:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt, lanes=lanes)
    b.compile()
    n = 700
    cls, nsteps, t0, y0, p, counters = make_items(n, 5, classes=classes, steps=(0, 1, 7, 50, 123))
    b.set_items(cls, nsteps, t0, y0, p, counters)
    b.run(graph=True)
    t, y, cnt, passes, flags = b.results()
    rng = np.random.default_rng(6)
    for i in rng.choice(n, 50, replace=False):
        system, solver, neq, npar, nnoi, dt = classes[cls[i]]
        tt, yy, cc = single_kernel_final_state(system, solver, neq, npar, nnoi, dt, nsteps[i], t0[i], y0[i], p[i],
                                               counters[i], i, False)
        np.testing.assert_array_equal(y[i], yy)
        assert t[i] == tt
        if nnoi:
            assert cnt[i] == cc


def assert_batch_final_states_match_oracle(classes, cls, nsteps, t0, y0, p, counters, t, y, cnt, per_class, seed):
    """Samples up to `per_class` orbits (with steps) of every class and checks
    their final states against the oracle run at each orbit's own step count
    (noise keyed by the orbit's index, as the batch keys it), within the
    floor-based tolerance of tests/parity.py."""
    from oracle.oracle import Oracle
    from parity import assert_parity

    rng = np.random.default_rng(seed)
    for k, (system, solver, neq, npar, nnoi, dt) in enumerate(classes):
        members = np.nonzero((cls == k) & (nsteps > 0))[0]
        assert members.size > 0, "class %d has no orbit with steps" % k
        pick = np.sort(rng.choice(members, min(per_class, members.size), replace=False))
        solver_id = {"se": 0, "euler": 1, "rk4": 2, "ie": 3, "im": 4}[solver]
        want, alt = np.empty((1, neq, pick.size)), np.empty((1, neq, pick.size))
        for j, i in enumerate(pick):
            kw = dict(neq=neq, npar=npar, nnoi=nnoi, dt=dt, ksteps=int(nsteps[i]), nchunks=1, records=False,
                      counters=[counters[i]] if nnoi else None, orbit_offset=int(i))
            r = Oracle(system).run(solver_id, [t0[i]], [y0[i]], [p[i]], **kw)
            a = Oracle(system, "fp64fma").run(solver_id, [t0[i]], [y0[i]], [p[i]], **kw)
            want[0, :, j], alt[0, :, j] = r.y[0], a.y[0]
            assert t[i] == r.t[0]
            if nnoi:
                assert cnt[i] == r.counters[0]
        got = np.stack([y[i] for i in pick], axis=1)[None]
        assert_parity("batch class %d (%s %s N=%d) vs oracle" % (k, system, solver, neq), got, want, alt)


@pytest.mark.gpu
def test_batch_classes_match_oracle():
    """Every class of a batch (one lane per orbit: Kuramoto Euler / RK4 /
    implicit Euler / Euler-Maruyama, oculomotor RK4 / implicit Euler /
    implicit midpoint) against the CPU oracle, not only against the
    single-system kernel.  Kuramoto implicit Euler uses this library's
    Kuramoto file, which adds the calc_jacobian the reference's lacks."""
    n = 3000
    cls, nsteps, t0, y0, p, counters = make_items(n, 21)
    b = make_batch()
    b.set_items(cls, nsteps, t0, y0, p, counters)
    b.run(graph=True)
    t, y, cnt, _, _ = b.results()
    assert_batch_final_states_match_oracle(CLASSES, cls, nsteps, t0, y0, p, counters, t, y, cnt, 12, 22)


@pytest.mark.gpu
def test_batch_lanes_classes_match_oracle():
    """The wide classes that run several lanes per orbit (N up to 64,
    implicit Euler and midpoint among them) against the CPU oracle."""
    classes = [c[:6] for c in LANES_CLASSES]
    b = Batch()
    for system, solver, neq, npar, nnoi, dt, lanes in LANES_CLASSES:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt, lanes=lanes)
    b.compile()
    n = 700
    cls, nsteps, t0, y0, p, counters = make_items(n, 23, classes=classes, steps=(1, 7, 50, 123))
    b.set_items(cls, nsteps, t0, y0, p, counters)
    b.run(graph=True)
    t, y, cnt, _, _ = b.results()
    assert_batch_final_states_match_oracle(classes, cls, nsteps, t0, y0, p, counters, t, y, cnt, 6, 24)
