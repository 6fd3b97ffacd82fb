"""sodecl_batch_run_noalloc: the allocation-free launch of a batch.

Some callers cannot let a library allocate device memory: a custom operator
inside a framework whose allocator owns all device memory, or a service that
allocates its working set once at start-up.  For them the batch kernel's
scratch (its work-queue heads) lives in a device array inside the library and
they pass every input and output as their own device buffers.

Checked here: through the C ABI, two calls in a row (the second on a scratch
array still holding the first call's values) give exactly what the regular
entry point (sodecl_batch_set_items + sodecl_batch_run) gives -- bit for bit,
the tolerance the other batch tests use -- and sampled orbits of every class
match the CPU oracle within the floor-based tolerance of tests/parity.py.
This file is collected last so a run that stops at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from sodecl_b200 import _native as N
from sodecl_b200 import system_path
from sodecl_b200.batch import Batch

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])
# (system, solver, neq, npar, nnoi, dt); the two wide Kuramoto classes run
# several lanes per orbit, whose state lives in the kernel's dynamic shared
# memory, which the allocation-free launch sizes as the regular one does
CLASSES = [("kuramoto", "rk4", 8, 9, 0, 0.01), ("oculomotor", "rk4", 6, 6, 0, 1e-5),
           ("oculomotor", "ie", 6, 6, 0, 1e-3), ("kuramoto", "se", 4, 9, 4, 0.01),
           ("kuramoto", "rk4", 16, 17, 0, 0.01), ("kuramoto", "ie", 20, 21, 0, 0.01)]


def build_batch():
    b = Batch()
    for system, solver, neq, npar, nnoi, dt in CLASSES:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt)
    return b.compile()


def class_grouped_items(per_class, seed):
    """Orbits grouped by class (class 0 first), uneven step counts."""
    rng = np.random.default_rng(seed)
    cls, steps, t0, y0, p = [], [], [], [], []
    for c, (system, solver, neq, npar, nnoi, dt) in enumerate(CLASSES):
        for _ in range(per_class[c]):
            cls.append(c)
            steps.append(int(rng.integers(0, 300)))
            t0.append(rng.uniform(0, 1))
            if system == "oculomotor":
                y0.append(Y0.copy())
                p.append(NOMINAL * rng.uniform(0.5, 1.5, 6))
            else:
                y0.append(rng.uniform(0, 2 * np.pi, neq))
                q = np.concatenate([[rng.uniform(0, 5)], rng.normal(size=neq)])
                p.append(np.concatenate([q, rng.uniform(0, 0.5, nnoi)]) if nnoi else q)
    counters = rng.integers(0, 2 ** 40, len(cls)).astype(float)
    return (np.array(cls, np.int32), np.array(steps, np.int64), np.array(t0), y0, p, counters)


@pytest.mark.gpu
def test_noalloc_batch_run_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    if N.device_count() < 1:
        pytest.fail("no CUDA device")
    per_class = [700, 900, 300, 500, 400, 200]
    cls, steps, t0, y0, p, counters = class_grouped_items(per_class, 11)

    # the regular entry point: the library allocates and uploads
    ref = build_batch()
    ref.set_items(cls, steps, t0, y0, p, counters)
    ref.run(graph=False)
    t_ref, y_ref, c_ref, passes_ref, flags_ref = ref.results()
    y_ref = np.concatenate(y_ref)

    # the allocation-free entry point: the caller owns every buffer
    b = build_batch()
    assert max(b.lanes) > 1  # some classes run lanes per orbit
    dev = torch.device("cuda", 0)
    y_flat, p_flat = np.concatenate(y0), np.concatenate(p)
    counts = np.array(per_class, dtype=np.int64)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        t_d = torch.tensor(t0, device=dev)
        y_d = torch.tensor(y_flat, device=dev)
        p_d = torch.tensor(p_flat, device=dev)
        c_d = torch.tensor(counters, device=dev)
        s_d = torch.tensor(steps, device=dev)
        passes_d = torch.zeros(len(cls), dtype=torch.int64, device=dev)
        flags_d = torch.zeros(len(cls), dtype=torch.int32, device=dev)
        io = N.BatchIO()
        io.t, io.y, io.params, io.counters = t_d.data_ptr(), y_d.data_ptr(), p_d.data_ptr(), c_d.data_ptr()
        io.nsteps, io.newton_passes, io.flags = s_d.data_ptr(), passes_d.data_ptr(), flags_d.data_ptr()
        io.class_count = counts.ctypes.data
        rc = N.lib.sodecl_batch_run_noalloc(b._b, C.byref(io), C.c_void_p(stream.cuda_stream))
        assert rc == N.OK, "call %d failed" % call
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t_d.cpu().numpy(), t_ref)
        np.testing.assert_array_equal(y_d.cpu().numpy(), y_ref)
        np.testing.assert_array_equal(c_d.cpu().numpy(), c_ref)
        np.testing.assert_array_equal(passes_d.cpu().numpy(), passes_ref)
        np.testing.assert_array_equal(flags_d.cpu().numpy(), flags_ref)

    # and against the CPU oracle, not only against the library's other entry
    # point: sampled orbits of every class at their own step counts
    from test_batch import assert_batch_final_states_match_oracle

    widths = np.array([CLASSES[c][2] for c in cls])
    y_orbits = np.split(y_d.cpu().numpy(), np.cumsum(widths)[:-1])
    assert_batch_final_states_match_oracle(CLASSES, cls, steps, t0, y0, p, counters, t_d.cpu().numpy(), y_orbits,
                                           c_d.cpu().numpy(), 8, 12)


@pytest.mark.gpu
def test_noalloc_step_count_below_zero_takes_no_step():
    """The allocation-free launch reads step counts from the caller's device
    memory, which the host never inspects: a count below zero must take no
    step, like zero, and the launch must return.  Every orbit with such a
    count keeps its state; the others equal the regular entry point's run
    with those counts at zero."""
    torch = pytest.importorskip("torch")
    if N.device_count() < 1:
        pytest.fail("no CUDA device")
    per_class = [64, 64, 32, 32, 32, 32]
    cls, steps, t0, y0, p, counters = class_grouped_items(per_class, 5)
    negative = np.zeros(len(cls), bool)
    negative[::7] = True
    steps_zeroed = np.where(negative, 0, steps)

    ref = build_batch()
    ref.set_items(cls, steps_zeroed, t0, y0, p, counters)
    ref.run(graph=False)
    t_ref, y_ref, c_ref, passes_ref, _ = ref.results()

    b = build_batch()
    dev = torch.device("cuda", 0)
    t_d = torch.tensor(t0, device=dev)
    y_d = torch.tensor(np.concatenate(y0), device=dev)
    p_d = torch.tensor(np.concatenate(p), device=dev)
    c_d = torch.tensor(counters, device=dev)
    s_d = torch.tensor(np.where(negative, -1, steps).astype(np.int64), device=dev)
    passes_d = torch.zeros(len(cls), dtype=torch.int64, device=dev)
    io = N.BatchIO()
    io.t, io.y, io.params, io.counters = t_d.data_ptr(), y_d.data_ptr(), p_d.data_ptr(), c_d.data_ptr()
    io.nsteps, io.newton_passes, io.flags = s_d.data_ptr(), passes_d.data_ptr(), None
    counts = np.array(per_class, dtype=np.int64)
    io.class_count = counts.ctypes.data
    stream = torch.cuda.current_stream(dev)
    assert N.lib.sodecl_batch_run_noalloc(b._b, C.byref(io), C.c_void_p(stream.cuda_stream)) == N.OK
    torch.cuda.synchronize()
    t_got = t_d.cpu().numpy()
    np.testing.assert_array_equal(t_got, t_ref)
    np.testing.assert_array_equal(t_got[negative], t0[negative])
    np.testing.assert_array_equal(y_d.cpu().numpy(), np.concatenate(y_ref))
    np.testing.assert_array_equal(c_d.cpu().numpy(), c_ref)
    np.testing.assert_array_equal(passes_d.cpu().numpy(), passes_ref)
    assert (passes_d.cpu().numpy()[negative] == 0).all()


@pytest.mark.gpu
def test_noalloc_refuses_host_buffers():
    """A pageable host array in place of a device buffer is refused on the
    host, before the scratch is touched or anything is launched; the next call
    with device buffers runs and matches the regular entry point."""
    torch = pytest.importorskip("torch")
    if N.device_count() < 1:
        pytest.fail("no CUDA device")
    per_class = [32, 32, 16, 16, 16, 16]
    cls, steps, t0, y0, p, counters = class_grouped_items(per_class, 7)
    ref = build_batch()
    ref.set_items(cls, steps, t0, y0, p, counters)
    ref.run(graph=False)
    _, y_ref, _, _, _ = ref.results()

    b = build_batch()
    dev = torch.device("cuda", 0)
    t_d = torch.tensor(t0, device=dev)
    y_d = torch.tensor(np.concatenate(y0), device=dev)
    p_d = torch.tensor(np.concatenate(p), device=dev)
    c_d = torch.tensor(counters, device=dev)
    s_d = torch.tensor(steps, device=dev)
    counts = np.array(per_class, dtype=np.int64)
    host_steps = np.ascontiguousarray(steps)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    io = N.BatchIO()
    io.t, io.y, io.params, io.counters = t_d.data_ptr(), y_d.data_ptr(), p_d.data_ptr(), c_d.data_ptr()
    io.nsteps, io.class_count = host_steps.ctypes.data, counts.ctypes.data
    assert N.lib.sodecl_batch_run_noalloc(b._b, C.byref(io), stream) == N.ERR_INVALID_ARG
    io.nsteps = s_d.data_ptr()
    assert N.lib.sodecl_batch_run_noalloc(b._b, C.byref(io), stream) == N.OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(y_d.cpu().numpy(), np.concatenate(y_ref))
