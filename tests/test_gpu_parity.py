"""Parity of the CUDA path with the CPU oracle and the reference's known answers.

Every result goes through libsodecl_cuda.so (C ABI) on cuda:0 and is compared
with the oracle (oracle/oracle_solvers.h, itself pinned to the reference in
test_oracle.py) on the same inputs.

Error measure: per element, |gpu - oracle| / (|oracle| + 1e-3 * S_e), S_e the
largest |value| of equation e in the run (values crossing zero are measured
against their equation's scale); NaN/Inf positions must agree.

Tolerance (FP64): max(1e-12, 10 x the oracle's own noise floor), the floor
being the same error measure between the oracle built with and without FMA
contraction on the same inputs.  Last-bit differences (CUDA's exp/log/sin/cos
against glibc's, FMA contraction) are all the GPU adds; how far they travel is
a property of the dynamics: ~1e-14 for Euler, ~1e-11 for 1000 RK4 steps of the
stiff oculomotor model, ~1e-6 for implicit midpoint, whose Newton stop test at
1e-7 flips on last-bit differences in the oracle itself.
FP32: error against the FP64 oracle within max(1e-5, 10 x that of the FP32
oracle).  Threefry words, u01 doubles and draw counters: bit-exact.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import sodecl_b200
from sodecl_b200 import _native as N
from sodecl_b200 import Integrator, system_path
from oracle.oracle import Oracle, printed_dt, to_reference_layout
from parity import RTOL, assert_parity, rel_error  # noqa: F401

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if N.device_count() < 1:
        pytest.fail("no CUDA device: the gpu tests need a B200")


def run_gpu(system, solver, t0, y0, p, counters=None, **kw):
    n = len(t0)
    with Integrator(system_path(system), solver, orbits=n, **kw) as sim:
        sim.upload(t0, y0, p, counters)
        rec = sim.run()
        t, y, cnt = sim.state()
        passes, flags = sim.status()
    return rec, t, y, cnt, passes, flags


# --------------------------------------------------------------------------
# the reference's own known-answer tests, through the drop-in Python API


@pytest.mark.parametrize("name,solver,dt,ksteps", [("euler", 1, 1e-8, 40000), ("rk", 2, 1e-6, 400),
                                                    ("ie", 3, 1e-6, 400), ("im", 4, 1e-6, 400)])
def test_reference_known_answers_through_sodecl_py(name, solver, dt, ksteps):
    from sodecl_b200.sodecl import sodecl

    orbits, nequat = 2, 6
    initx = np.tile(Y0, (orbits, 1))
    params = np.tile(NOMINAL, (orbits, 1))
    t, results = sodecl(0, 0, system_path("oculomotor"), initx, params, solver, orbits, nequat, 0, dt, 0.1, ksteps, 0)
    golden = np.load(os.path.join(GOLDEN, "oculomotor_%s.npy" % name))
    assert results.shape == golden.shape
    assert np.isclose(results, golden).all()  # the reference test's rule
    kw = dict(neq=6, npar=6, dt=dt, tspan=0.1, ksteps=ksteps)
    want = Oracle("oculomotor").run(solver, np.zeros(2), initx, params, **kw).records
    alt = Oracle("oculomotor", "fp64fma").run(solver, np.zeros(2), initx, params, **kw).records
    got = results.T.reshape(want.shape)
    assert_parity("golden %s" % name, got, want, alt)


def test_sodecl_py_time_axis():
    """The reference's time axis (kept by default) can disagree with the record
    count; exact_time gives one time per record."""
    from sodecl_b200.sodecl import sodecl

    orbits = 2
    initx = np.tile(Y0, (orbits, 1))
    params = np.tile(NOMINAL, (orbits, 1))
    # tspan 0.2 with dt*ksteps 0.1: the reference loop makes 2 intervals (3 records)
    t_ref, res = sodecl(0, 0, system_path("oculomotor"), initx, params, 2, orbits, 6, 0, 1e-3, 0.2, 100, 0)
    t_exact, res2 = sodecl(0, 0, system_path("oculomotor"), initx, params, 2, orbits, 6, 0, 1e-3, 0.2, 100, 0,
                           exact_time=True)
    assert res.shape == (orbits * 6, 3)
    assert t_ref.size == 4  # as the reference returns it
    np.testing.assert_allclose(t_exact, [0.0, 0.1, 0.2])
    np.testing.assert_array_equal(res, res2)


def test_reference_python_module_list_interface():
    from sodecl_b200 import sodecl_interface

    out = sodecl_interface.sodeclcall([0.0, 0.0], list(np.tile(Y0, 2)), list(np.tile(NOMINAL, 2)), 0, 0,
                                      system_path("oculomotor"), 2, 2, 6, 6, 0, 1e-6, 0.1, 400, 0)
    golden = np.load(os.path.join(GOLDEN, "oculomotor_rk.npy"))
    res = np.array(out).reshape(12, -1, order="F")
    assert np.isclose(res, golden).all()


# --------------------------------------------------------------------------
# fixtures produced by the reference's kernels compiled as C


@pytest.mark.parametrize("fmad", [0, 1])
@pytest.mark.parametrize("name,system", [("kuramoto_euler", "kuramoto"), ("kuramoto_se", "kuramoto"),
                                         ("kuramoto32_se", "kuramoto"), ("oculomotor_se", "oculomotor"),
                                         ("oculomotor_im", "oculomotor"), ("oculomotor_ie", "oculomotor"),
                                         ("oculomotor_rk4", "oculomotor")])
def test_reference_build_fixtures(name, system, fmad):
    f = dict(np.load(os.path.join(GOLDEN, "ref_%s.npz" % name)))
    n = len(f["t0"])
    solver = int(f["solver"])
    kw = dict(dt=float(f["dt"]), tspan=float(f["tspan"]), ksteps=int(f["ksteps"]), neq=int(f["neq"]),
              npar=int(f["npar"]), nnoi=int(f["nnoi"]), fmad=bool(fmad))
    if int(f["orbit_offset"]):
        # the noise stream is keyed by the global orbit index: run the fixture's
        # orbits as the tail of a larger list
        off = int(f["orbit_offset"])
        pad = lambda a: np.concatenate([np.repeat(a[:1], off, axis=0), a])  # noqa: E731
        rec, t, y, cnt, _, _ = run_gpu(system, solver, pad(f["t0"]), pad(f["y0"]), pad(f["params"]),
                                       pad(f["counters"]) if "counters" in f else None, **kw)
        rec, t, y, cnt = rec[:, :, off:], t[off:], y[off:], cnt[off:]
    else:
        rec, t, y, cnt, _, _ = run_gpu(system, solver, f["t0"], f["y0"], f["params"], f.get("counters"), **kw)
    assert rec.shape == f["records"].shape
    alt = Oracle(system, "fp64fma").run(solver, f["t0"], f["y0"], f["params"], neq=kw["neq"], npar=kw["npar"],
                                        nnoi=kw["nnoi"], dt=kw["dt"], ksteps=kw["ksteps"], nchunks=int(f["nchunks"]),
                                        counters=f.get("counters"), orbit_offset=int(f["orbit_offset"])).records
    assert_parity("%s fmad=%d" % (name, fmad), rec, f["records"], alt)
    np.testing.assert_array_equal(t, f["t_final"])
    if "counters" in f:
        np.testing.assert_array_equal(cnt, f["counters_final"])


# --------------------------------------------------------------------------
# oracle parity on random inputs, every solver, both precisions


def oculomotor_inputs(n, seed, nnoi=0):
    rng = np.random.default_rng(seed)
    p = NOMINAL * rng.uniform(0.5, 1.5, (n, 6))
    if nnoi:
        p = np.concatenate([p, rng.uniform(0.0, 0.01, (n, nnoi))], axis=1)
    return np.zeros(n), np.tile(Y0, (n, 1)), p


@pytest.mark.parametrize("fmad", [0, 1])
@pytest.mark.parametrize("solver,dt", [(1, 1e-6), (2, 1e-5), (3, 1e-3), (4, 1e-3), (0, 1e-5)])
def test_oculomotor_parity_fp64(solver, dt, fmad):
    n = 1000  # not a multiple of the block size
    nnoi = 2 if solver == 0 else 0
    t0, y0, p = oculomotor_inputs(n, solver, nnoi)
    cnt = np.arange(n) * 1000.0 if nnoi else None
    kw = dict(dt=dt, tspan=300 * dt, ksteps=30, neq=6, npar=6 + nnoi, nnoi=nnoi)
    rec, t, y, c, passes, flags = run_gpu("oculomotor", solver, t0, y0, p, cnt, fmad=bool(fmad), **kw)
    ref = Oracle("oculomotor").run(solver, t0, y0, p, counters=cnt, **kw)
    alt = Oracle("oculomotor", "fp64fma").run(solver, t0, y0, p, counters=cnt, **kw)
    assert_parity("oculomotor solver %d fmad=%d" % (solver, fmad), rec, ref.records, alt.records)
    np.testing.assert_array_equal(t, ref.t)
    if solver in (3, 4):
        # same iterates -> same pass counts, but for orbits whose Newton stop
        # test flipped on a last-bit difference (as between the two oracles)
        assert np.mean(passes == ref.newton_passes) >= min(0.95, np.mean(alt.newton_passes == ref.newton_passes))
        assert abs(passes.sum() / ref.newton_passes.sum() - 1) < 1e-3
        # the quasi-Newton stalls above the tolerance for some draws, in the oracle too
        np.testing.assert_array_equal(flags & N.FLAG_NEWTON_CAP, ref.flags & N.FLAG_NEWTON_CAP)
    if nnoi:
        np.testing.assert_array_equal(c, ref.counters)


@pytest.mark.parametrize("solver,dt", [(1, 1e-6), (2, 1e-5), (3, 1e-4), (4, 1e-4)])
def test_oculomotor_parity_fp32(solver, dt):
    n = 512
    t0, y0, p = oculomotor_inputs(n, 10 + solver)
    kw = dict(dt=dt, tspan=100 * dt, ksteps=10, neq=6, npar=6)
    rec, *_ = run_gpu("oculomotor", solver, t0, y0, p, precision="fp32", **kw)
    ref32 = Oracle("oculomotor", "fp32").run(solver, t0, y0, p, **kw).records
    ref64 = Oracle("oculomotor", "fp64").run(solver, t0, y0, p, **kw).records
    # error against the FP64 oracle, no worse than (10x) the CPU's own FP32 run
    assert_parity("fp32 solver %d vs fp64 oracle" % solver, rec, ref64, ref32, rtol=1e-5)


@pytest.mark.parametrize("N_osc,solver,nnoi", [(8, 1, 0), (8, 2, 0), (16, 3, 0), (4, 4, 0), (32, 0, 32), (5, 0, 5)])
def test_kuramoto_parity(N_osc, solver, nnoi):
    n = 300
    rng = np.random.default_rng(N_osc)
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1))] +
                       ([rng.uniform(0, 0.5, (n, N_osc))] if nnoi else []), axis=1)
    th0 = rng.uniform(0, 2 * np.pi, (n, N_osc))
    cnt = rng.integers(0, 2 ** 40, n).astype(float) if nnoi else None
    kw = dict(dt=0.01, tspan=2.0, ksteps=20, neq=N_osc, npar=p.shape[1], nnoi=nnoi)
    rec, t, y, c, *_ = run_gpu("kuramoto", solver, np.zeros(n), th0, p, cnt, **kw)
    ref = Oracle("kuramoto").run(solver, np.zeros(n), th0, p, counters=cnt, **kw)
    alt = Oracle("kuramoto", "fp64fma").run(solver, np.zeros(n), th0, p, counters=cnt, **kw)
    assert_parity("kuramoto N=%d solver %d" % (N_osc, solver), rec, ref.records, alt.records)
    if nnoi:
        np.testing.assert_array_equal(c, ref.counters)


# --------------------------------------------------------------------------
# the noise stream, bit for bit


def test_noise_stream_bit_exact():
    o = Oracle("kuramoto")
    rng = np.random.default_rng(5)
    gids = np.concatenate([np.arange(8), rng.integers(0, 2 ** 31, 56)])
    counters = np.concatenate([np.zeros(8), rng.integers(0, 2 ** 52, 48).astype(float), -rng.uniform(0, 1e11, 8)])
    nnoi, nsteps, dt = 5, 7, 0.01
    normals, words, u01 = sodecl_b200.noise_stream(gids, counters, nnoi, printed_dt(dt), nsteps, words=True, u01=True)
    ncalls = (nnoi + 1) // 2
    for i in range(len(gids)):
        c = counters[i]
        for s in range(nsteps):
            for k in range(ncalls):
                w = o.threefry2x64_20([int(gids[i]), o.counter_word(c)], [0, 0xF00DCAFE])
                np.testing.assert_array_equal(words[i, s, k], w)
                assert u01[i, s, k, 0] == o.u01_open_open(int(w[0]))
                assert u01[i, s, k, 1] == o.u01_open_open(int(w[1]))
                c += 1
        want = o.noise_stream(int(gids[i]), counters[i], nnoi, dt, nsteps)
        # Box-Muller through CUDA's and glibc's log/sin/cos: a few ulp
        ulp = np.spacing(np.abs(want))
        assert np.max(np.abs(normals[i] - want) / ulp) <= 8


# --------------------------------------------------------------------------
# status words, continuation, output modes, scale


def test_newton_cap_and_nonfinite_flags():
    n = 64
    t0, y0, p = oculomotor_inputs(n, 1)
    rec, t, y, c, passes, flags = run_gpu("oculomotor", 4, t0, y0, p, dt=1e-3, tspan=0.01, ksteps=10, neq=6, npar=6,
                                          newton_tol=1e-14, newton_max_iter=3)
    assert (flags & N.FLAG_NEWTON_CAP).all()
    assert (passes == 30).all()
    # RK4 at dt=1e-3 diverges for this model
    rec, t, y, c, passes, flags = run_gpu("oculomotor", 2, t0, y0, p, dt=1e-3, tspan=2.0, ksteps=100, neq=6, npar=6)
    bad = ~np.isfinite(rec[-1]).all(axis=0)
    assert bad.any()
    np.testing.assert_array_equal((flags & N.FLAG_NONFINITE) != 0, ~np.isfinite(rec).all(axis=(0, 1)))


def test_second_run_continues_from_device_state():
    n = 200
    t0, y0, p = oculomotor_inputs(n, 2)
    kw = dict(dt=1e-5, ksteps=20, neq=6, npar=6)
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, tspan=2e-3, **kw) as sim:
        sim.upload(t0, y0, p)
        a = sim.run()
        b = sim.run()
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, tspan=4e-3, **kw) as sim:
        sim.upload(t0, y0, p)
        whole = sim.run()
    np.testing.assert_array_equal(b[0], a[-1])
    np.testing.assert_array_equal(np.concatenate([a, b[1:]]), whole)


@pytest.mark.parametrize("nchunks", [0, 1, 2, 3, 10, 33])
def test_output_modes_agree(nchunks):
    """Pageable host memory (records staged through pinned slots by copy
    threads, launch groups of equal then halving size), pinned host memory
    (halving groups, copy engine), device memory (one launch) and no output
    give the same records and final state, for record-interval counts that
    exercise every grouping."""
    torch = pytest.importorskip("torch")
    n = 4096
    t0, y0, p = oculomotor_inputs(n, 3)
    kw = dict(dt=1e-5, tspan=nchunks * 10 * 1e-5 - 1e-9 if nchunks else 0.0, ksteps=10, neq=6, npar=6)
    outs = []
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        assert sim.num_chunks == nchunks
        shape = (sim.num_records, 6, n)
        sim.upload(t0, y0, p)
        outs.append(sim.run())                                     # pageable host
        sim.upload(t0, y0, p)
        pinned = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        sim.run_into(pinned.data_ptr(), pinned.numel())            # pinned host
        outs.append(pinned.numpy().copy())
        sim.upload(t0, y0, p)
        dev = torch.empty(shape, dtype=torch.float64, device="cuda")
        sim.run_into(dev.data_ptr(), dev.numel())                  # device
        torch.cuda.synchronize()
        outs.append(dev.cpu().numpy())
        sim.upload(t0, y0, p)
        assert sim.run(discard=True) is None                       # output_Type::None
        t_none, y_none, _ = sim.state()
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    np.testing.assert_array_equal(y_none, outs[0][-1].T)


def test_device_launch_api_in_chunks():
    torch = pytest.importorskip("torch")
    n = 3000
    t0, y0, p = oculomotor_inputs(n, 4)
    kw = dict(dt=1e-5, tspan=2e-3, ksteps=20, neq=6, npar=6)
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p)
        want = sim.run()
        nchunks = sim.num_chunks
        dt_ = torch.tensor(t0, device="cuda")
        dy = torch.tensor(y0, device="cuda")
        dp = torch.tensor(p, device="cuda")
        rec = torch.full((nchunks + 1, 6, n), float("nan"), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        # two orbit halves x three interval ranges
        for lo, hi in ((0, 1000), (1000, n)):
            for c0, c1 in ((0, 3), (3, 7), (7, nchunks)):
                sim.launch(t=dt_[lo:].data_ptr(), y=dy[lo:].data_ptr(), params=dp[lo:].data_ptr(),
                           records=rec.data_ptr(), n=hi - lo, orbit_offset=lo, rec_stride=n, rec_col0=lo,
                           chunk_begin=c0, chunk_end=c1, write_final=(c1 == nchunks), stream=stream)
        torch.cuda.synchronize()
    np.testing.assert_array_equal(rec.cpu().numpy(), want)


def test_many_orbits_indexing():
    n = 1 << 18
    t0, y0, p = oculomotor_inputs(n, 6)
    kw = dict(dt=1e-5, tspan=2e-4, ksteps=5, neq=6, npar=6)
    rec, *_ = run_gpu("oculomotor", 2, t0, y0, p, **kw)
    idx = np.r_[0:256, n // 2 - 128:n // 2 + 128, n - 256:n]
    ref = Oracle("oculomotor").run(2, t0[idx], y0[idx], p[idx], **kw).records
    alt = Oracle("oculomotor", "fp64fma").run(2, t0[idx], y0[idx], p[idx], **kw).records
    assert_parity("2^18 orbits subsample", rec[:, :, idx], ref, alt)
    assert np.isfinite(rec).all()


def test_cpp_sodeclmgr_drop_in(tmp_path):
    """The C++ manager with the reference's call sequence (interfaces/python/sodecl.cpp:56-94)."""
    src = os.path.join(REPO, "tests", "cpp", "sodeclmgr_golden.cpp")
    exe = str(tmp_path / "sodeclmgr_golden")
    lib_dir = os.path.join(REPO, "sodecl_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), src, "-o", exe, "-L", lib_dir,
                    "-lsodecl_cuda", "-Wl,-rpath," + lib_dir], check=True)
    out_file = str(tmp_path / "out.bin")
    proc = subprocess.run([exe, system_path("oculomotor"), out_file], capture_output=True, text=True, cwd=tmp_path)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "Compute results runtime" in proc.stdout
    res = np.fromfile(out_file).reshape(12, -1, order="F")
    golden = np.load(os.path.join(GOLDEN, "oculomotor_rk.npy"))
    assert np.isclose(res, golden).all()
    filemode = np.fromfile(str(tmp_path / "sodecloutput.bin"))
    np.testing.assert_array_equal(filemode, np.fromfile(out_file))
    # the assembled program in the working directory, as the reference leaves
    # its OpenCL source there (src/sodeclmgr.cpp:497-500)
    dumped = (tmp_path / "Generated_kernel.cl").read_text()
    assert "#define _m_dt_" in dumped and "sode_system" in dumped and "sodecl_orbits" in dumped


@pytest.mark.parametrize("solver", ["ie", "im"])
def test_implicit_kernel_launch_shapes_agree(solver):
    """The implicit kernel's warps hand out ranges of orbits to their lanes, and
    the host launches only as many blocks as give each lane the fewest orbits
    that fit the resident threads.  Block sizes that are not a multiple of 32
    (partial warps), more orbits than resident threads (several orbits a
    lane), the register cap lifted, and sodecl_cuda_launch on a slice of the
    orbits in two interval ranges all give the same records, pass counts and
    flags, bit for bit."""
    import torch

    n = 150000  # above the resident threads of a B200 at 128 registers
    t0, y0, p = oculomotor_inputs(n, 31)
    kw = dict(dt=1e-3, tspan=60e-3, ksteps=20, neq=6, npar=6)
    outs = []
    for block, minb in ((128, 0), (100, 0), (33, 0), (512, 0), (128, 1)):
        with Integrator(system_path("oculomotor"), solver, orbits=n, block=block, min_blocks=minb, **kw) as sim:
            sim.upload(t0, y0, p)
            rec = sim.run()
            passes, flags = sim.status()
        outs.append((rec, passes, flags))
    for rec, passes, flags in outs[1:]:
        np.testing.assert_array_equal(rec, outs[0][0])
        np.testing.assert_array_equal(passes, outs[0][1])
        np.testing.assert_array_equal(flags, outs[0][2])
    # a slice of the orbits through the device launch
    lo, hi = 4321, 104321
    dev = torch.device("cuda", 0)
    with Integrator(system_path("oculomotor"), solver, orbits=n, **kw) as sim:
        T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
        td, yd, pd = T(t0[lo:hi]), T(y0[lo:hi]), T(p[lo:hi])
        nchunks = sim.num_chunks
        rec = torch.full((nchunks + 1, 6, n), float("nan"), dtype=torch.float64, device=dev)
        for c0, c1 in ((0, 1), (1, nchunks)):  # the second launch continues from the first's state
            sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=rec.data_ptr(), n=hi - lo,
                       orbit_offset=lo, rec_stride=n, rec_col0=lo, chunk_begin=c0, chunk_end=c1,
                       write_final=(c1 == nchunks), stream=torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rec[:, :, lo:hi].cpu().numpy(), outs[0][0][:, :, lo:hi])


def test_pair_stores_write_the_same_records():
    """Paired record stores (neighbouring orbits swap values and each writes
    one equation of both as a vector store) give the records of direct
    stores bit for bit: even and odd orbit counts (a last orbit without a
    partner), a block size that is odd (direct stores throughout), an odd
    equation count (the last equation stored alone), FP32 compute and, through
    sodecl_cuda_launch, an odd first column, an odd row stride, a record base
    off the 16-byte grid and float records."""
    import torch

    dev = torch.device("cuda", 0)
    kw = dict(dt=1e-3, tspan=30e-3, ksteps=10, neq=6, npar=6)
    for n in (1, 2, 33, 1000, 4097):
        t0, y0, p = oculomotor_inputs(n, 40 + n)
        for solver, block, prec in (("rk4", 128, "fp64"), ("rk4", 33, "fp64"), ("euler", 64, "fp64"),
                                    ("rk4", 128, "fp32")):
            outs = []
            for store in ("direct", "pairs"):
                with Integrator(system_path("oculomotor"), solver, orbits=n, block=block, precision=prec,
                                record_store=store, **kw) as sim:
                    sim.upload(t0, y0, p)
                    outs.append(sim.run())
            np.testing.assert_array_equal(outs[1], outs[0])
    # the implicit and adaptive kernels hand orbits to lanes out of order and
    # store per lane: they keep the direct stores whatever is asked
    n = 1000
    t0, y0, p = oculomotor_inputs(n, 43)
    for solver in ("ie", "im", "dp45"):
        outs = []
        for store in ("direct", "pairs"):
            with Integrator(system_path("oculomotor"), solver, orbits=n, record_store=store, **kw) as sim:
                assert "#define SODECL_PAIR_STORES 1" not in sim.program_source
                sim.upload(t0, y0, p)
                outs.append(sim.run())
        np.testing.assert_array_equal(outs[1], outs[0])
    # an odd equation count: Kuramoto with 5 phases
    rng = np.random.default_rng(41)
    n, N_osc = 1001, 5
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1)),
                        rng.uniform(0, 0.5, (n, N_osc))], axis=1)
    y0 = rng.uniform(0, 2 * np.pi, (n, N_osc))
    outs = []
    for store in ("direct", "pairs"):
        with Integrator(system_path("kuramoto"), "euler", orbits=n, dt=0.01, tspan=0.3, ksteps=10, neq=N_osc,
                        npar=2 * N_osc + 1, record_store=store) as sim:
            sim.upload(np.zeros(n), y0, p)
            outs.append(sim.run())
    np.testing.assert_array_equal(outs[1], outs[0])
    # the device launch: column offsets, strides, bases and record types; every
    # record of the orbit range is written (the fill is exact in float too)
    FILL = -1234.5
    n = 5000
    t0, y0, p = oculomotor_inputs(n, 42)
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    for lo, stride_pad, base_off, f32 in ((1, 0, 0, False), (2, 1, 0, False), (0, 0, 1, False), (3, 0, 0, True),
                                          (0, 0, 0, True)):
        m = n - 7
        stride = lo + m + stride_pad
        outs = []
        for store in ("direct", "pairs"):
            with Integrator(system_path("oculomotor"), "rk4", orbits=n, record_store=store, record_f32=f32,
                            **kw) as sim:
                td, yd, pd = T(t0[:m]), T(y0[:m]), T(p[:m])
                nchunks = sim.num_chunks
                rec = torch.full(((nchunks + 1) * 6 * stride + base_off,), FILL,
                                 dtype=torch.float32 if f32 else torch.float64, device=dev)
                sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(),
                           records=rec.data_ptr() + base_off * rec.element_size(), n=m, rec_stride=stride,
                           rec_col0=lo, chunk_begin=0, chunk_end=nchunks, write_final=True,
                           stream=torch.cuda.current_stream(dev).cuda_stream)
                torch.cuda.synchronize()
                outs.append(rec.cpu().numpy())
        np.testing.assert_array_equal(outs[1], outs[0])
        assert not (outs[0][base_off:].reshape(nchunks + 1, 6, stride)[:, :, lo:lo + m] == FILL).any()


def test_record_buffer_passes_to_the_next_context():
    """A destroyed context leaves its device record buffer to the next one on
    the device (the reference's callers make a manager per call); the next
    run allocates nothing new and gives the same records, and
    sodecl_cuda_release_cached frees the buffer."""
    import torch

    n = 1 << 18
    t0, y0, p = oculomotor_inputs(n, 44)
    kw = dict(dt=1e-3, tspan=0.1, ksteps=10, neq=6, npar=6)
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p)
        first = sim.run()
        held = first.nbytes
    torch.cuda.synchronize()
    f1 = torch.cuda.mem_get_info()[0]
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p)
        again = sim.run()
        f2 = torch.cuda.mem_get_info()[0]
    np.testing.assert_array_equal(again, first)
    assert f1 - f2 < held // 2  # the state buffers only: the records came from the first context
    f3 = torch.cuda.mem_get_info()[0]
    N.check(N.lib.sodecl_cuda_release_cached(0))
    f4 = torch.cuda.mem_get_info()[0]
    assert f4 - f3 >= 0.9 * held
    N.check(N.lib.sodecl_cuda_release_cached(0))  # nothing left: a no-op


# --------------------------------------------------------------------------
# the reciprocal quotient


def test_reciprocal_quotient_equals_ieee_division():
    bad, a, b = C.c_int64(), C.c_double(), C.c_double()
    N.check(N.lib.sodecl_cuda_division_check(0, 1 << 33, 20240601, C.byref(bad), C.byref(a), C.byref(b)))
    assert bad.value == 0, "first differing pair %r / %r" % (a.value, b.value)


def test_reciprocal_quotient_f32_equals_ieee_division():
    bad, a, b = C.c_int64(), C.c_float(), C.c_float()
    N.check(N.lib.sodecl_cuda_division_check_f32(0, 1 << 33, 20240602, C.byref(bad), C.byref(a), C.byref(b)))
    assert bad.value == 0, "first differing pair %r / %r" % (a.value, b.value)


@pytest.mark.parametrize("system,solver,dt", [("oculomotor", "rk4", 1e-3), ("oculomotor", "rk4", 1e-5),
                                              ("oculomotor", "im", 1e-3), ("kuramoto", "se", 0.01)])
def test_fp32_division_modes_give_identical_records(system, solver, dt):
    """FP32 programs: the reciprocal quotient and IEEE division (the default)
    give the same records, diverging orbits (dt 1e-3) included."""
    n = 2048
    if system == "oculomotor":
        t0, y0, p = oculomotor_inputs(n, 17)
        kw = dict(neq=6, npar=6)
        cnt = None
    else:
        rng = np.random.default_rng(18)
        N_osc = 16
        p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1)),
                            rng.uniform(0, 0.5, (n, N_osc))], axis=1)
        t0, y0, cnt = np.zeros(n), rng.uniform(0, 2 * np.pi, (n, N_osc)), np.arange(n) * 4096.0
        kw = dict(neq=N_osc, npar=2 * N_osc + 1, nnoi=N_osc)
    kw.update(dt=dt, tspan=400 * dt, ksteps=40, precision="fp32", newton_tol=1e-4)
    out = {}
    for mode in ("default", "ieee", "reciprocal"):
        with Integrator(system_path(system), solver, orbits=n, division=mode, **kw) as sim:
            assert sim.division == ("ieee" if mode == "default" else mode)
            sim.upload(t0, y0, p, cnt)
            out[mode] = sim.run()
    np.testing.assert_array_equal(out["reciprocal"], out["ieee"])
    np.testing.assert_array_equal(out["default"], out["ieee"])


@pytest.mark.parametrize("fmad", [0, 1])
@pytest.mark.parametrize("system,solver,dt", [("oculomotor", "rk4", 1e-5), ("oculomotor", "ie", 1e-3),
                                              ("oculomotor", "im", 1e-3), ("oculomotor", "euler", 1e-6),
                                              ("kuramoto", "se", 0.01)])
def test_division_modes_give_identical_records(system, solver, dt, fmad):
    n = 2048
    if system == "oculomotor":
        t0, y0, p = oculomotor_inputs(n, 7)
        kw = dict(neq=6, npar=6)
        cnt = None
    else:
        rng = np.random.default_rng(8)
        N_osc = 16
        p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N_osc), (n, 1)),
                            rng.uniform(0, 0.5, (n, N_osc))], axis=1)
        t0, y0, cnt = np.zeros(n), rng.uniform(0, 2 * np.pi, (n, N_osc)), np.arange(n) * 4096.0
        kw = dict(neq=N_osc, npar=2 * N_osc + 1, nnoi=N_osc)
    kw.update(dt=dt, tspan=400 * dt, ksteps=40, fmad=bool(fmad))
    out = {}
    for mode in ("ieee", "reciprocal"):
        with Integrator(system_path(system), solver, orbits=n, division=mode, **kw) as sim:
            assert sim.division == mode
            sim.upload(t0, y0, p, cnt)
            out[mode] = sim.run()
    np.testing.assert_array_equal(out["reciprocal"], out["ieee"])


def test_autotune_keeps_results():
    n = 20000
    t0, y0, p = oculomotor_inputs(n, 9)
    kw = dict(dt=1e-5, tspan=5e-4, ksteps=10, neq=6, npar=6)
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p)
        want = sim.run()
        sim.upload(t0, y0, p)
        choice = sim.autotune(sample_orbits=8192, sample_steps=50)
        assert choice["block"] in (64, 128, 256) and choice["division"] in ("ieee", "reciprocal")
        assert sim.division == choice["division"]
        t, y, _ = sim.state()
        np.testing.assert_array_equal(y, y0)  # tuning ran on copies
        got = sim.run()
    np.testing.assert_array_equal(got, want)


def test_device_entry_points_refuse_host_buffers():
    """sodecl_cuda_launch and sodecl_cuda_adjoint take device pointers.  A
    pageable host array handed to them by mistake is refused on the host,
    before any launch (a kernel would fault on it), and the context stays
    usable: the next launch with device buffers gives the records the
    host-output run gives."""
    torch = pytest.importorskip("torch")
    from sodecl_b200.fit import Adjoint

    n = 64
    t0, y0, p = oculomotor_inputs(n, 9)
    kw = dict(dt=1e-5, tspan=5e-4, ksteps=10, neq=6, npar=6)
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw) as sim:
        sim.upload(t0, y0, p)
        want = sim.run()
        dev = torch.device("cuda")
        td, yd, pd = (torch.tensor(x, device=dev) for x in (t0, y0, p))
        rec = torch.empty((sim.num_records, 6, n), dtype=torch.float64, device=dev)
        host_y = np.ascontiguousarray(y0)
        with pytest.raises(N.SodeclError, match="not memory this device can access"):
            sim.launch(t=td.data_ptr(), y=host_y.ctypes.data, params=pd.data_ptr(), records=rec.data_ptr())
        host_rec = np.empty((sim.num_records, 6, n))
        with pytest.raises(N.SodeclError, match="not memory this device can access"):
            sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=host_rec.ctypes.data)
        targets = torch.tensor(want, device=dev)
        with pytest.raises(N.SodeclError, match="not memory this device can access"):
            Adjoint(sim)(td, torch.tensor(y0), pd, targets)   # y0 left in host memory
        sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=rec.data_ptr(),
                   stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rec.cpu().numpy(), want)
