"""CPU oracle for the SODECL integrators -- TEST INFRASTRUCTURE ONLY.

Python access (ctypes) to the libraries oracle/build.py makes:

* ``Oracle(system, precision)`` -- the plain-C restatement of the reference's
  solvers (oracle_solvers.h) compiled with a system file from
  sodecl_b200/systems;
* ``ReferenceBuild(system, solver)`` -- the reference's own kernel sources
  compiled as C (oracle/_ref), present only where they were built.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker of the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")

STOCHASTIC_EULER, EULER, RUNGE_KUTTA, IMPLICIT_EULER, IMPLICIT_MIDPOINT = range(5)
REF_SOLVER_NAMES = {0: "se", 1: "euler", 2: "rk4", 3: "ie", 4: "im"}
NEWTON_TOL_DEFAULT = 1e-7     # src/sodeclmgr.cpp:425
NEWTON_MAX_DEFAULT = 1000     # src/kernels/ie.cl:69, im.cl:65


def printed_dt(dt: float) -> float:
    """The step the reference's program is built with: ``dt`` printed by a
    default ``std::ostream`` (6 significant digits, %g) into the
    ``#define _m_dt_`` line (src/sodeclmgr.cpp:356-367, :405-410)."""
    return float("%g" % dt)


def num_chunks(tspan: float, dt: float, ksteps: int) -> int:
    """Launches of the reference's run loop: ``for (int j = 0; j <
    (m_int_time/(m_dt*m_kernel_steps)); j++)`` (src/sodeclmgr.cpp:951), in
    double arithmetic with the unprinted dt.  Records = launches + 1."""
    x = tspan / (dt * ksteps)
    if not x > 0:
        return 0
    return int(math.ceil(x))


class _Job(C.Structure):
    _fields_ = [("solver", C.c_int), ("neq", C.c_int), ("npar", C.c_int), ("nnoi", C.c_int),
                ("ksteps", C.c_int), ("dt", C.c_double), ("nchunks", C.c_long), ("n", C.c_long),
                ("orbit_offset", C.c_long), ("t", C.c_void_p), ("y", C.c_void_p), ("p", C.c_void_p),
                ("counters", C.c_void_p), ("records", C.c_void_p), ("newton_tol", C.c_double),
                ("newton_max_iter", C.c_int), ("newton_passes", C.c_void_p), ("flags", C.c_void_p),
                ("nthreads", C.c_int), ("rtol", C.c_double), ("atol", C.c_double), ("max_steps", C.c_int)]


class _RefJob(C.Structure):
    _fields_ = [("neq", C.c_int), ("npar", C.c_int), ("nnoi", C.c_int), ("ksteps", C.c_int),
                ("dt", C.c_double), ("nchunks", C.c_long), ("n", C.c_long), ("orbit_offset", C.c_long),
                ("t", C.c_void_p), ("y", C.c_void_p), ("p", C.c_void_p), ("counters", C.c_void_p),
                ("records", C.c_void_p), ("eps", C.c_double), ("nthreads", C.c_int)]


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None:
        a = a.reshape(shape)
    return a.copy()


def _ptr(a):
    return None if a is None else a.ctypes.data


class Result:
    """Records ``[record][equation][orbit]`` plus the final state."""

    def __init__(self, records, t, y, counters, newton_passes=None, flags=None):
        self.records = records
        self.t = t
        self.y = y
        self.counters = counters
        self.newton_passes = newton_passes
        self.flags = flags


class Oracle:
    def __init__(self, system: str, precision: str = "fp64", lib_dir: str = BUILD_DIR):
        path = os.path.join(lib_dir, "liboracle_%s_%s.so" % (system, precision))
        if not os.path.exists(path):
            raise FileNotFoundError("%s not built (run oracle/build.py)" % path)
        self.lib = C.CDLL(path)
        self.lib.oracle_run.argtypes = [C.POINTER(_Job)]
        self.lib.oracle_run.restype = C.c_int
        self.lib.oracle_threefry2x64_20.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.oracle_u01_open_open_64_53.argtypes = [C.c_uint64]
        self.lib.oracle_u01_open_open_64_53.restype = C.c_double
        self.lib.oracle_counter_word.argtypes = [C.c_double]
        self.lib.oracle_counter_word.restype = C.c_uint64
        self.lib.oracle_noise_stream.argtypes = [C.c_long, C.c_double, C.c_int, C.c_double, C.c_long, C.c_void_p]
        self.system, self.precision = system, precision

    def run(self, solver, t0, y0, params, *, neq, npar, nnoi=0, dt, tspan=None, ksteps,
            nchunks=None, counters=None, orbit_offset=0, newton_tol=NEWTON_TOL_DEFAULT,
            newton_max_iter=NEWTON_MAX_DEFAULT, records=True, nthreads=0, rtol=1e-6, atol=1e-9,
            max_steps=100000) -> Result:
        """Integrate like the reference's run loop.  ``dt`` is the user's step;
        the solver steps with ``printed_dt(dt)``.  Solver 5 (Dormand-Prince,
        adaptive; no reference counterpart) takes ``printed_dt(dt)`` as its
        first step and ``counters`` as the orbits' step sizes (in/out)."""
        if nchunks is None:
            nchunks = num_chunks(tspan, dt, ksteps)
        t = _f64(t0)
        n = t.size
        y = _f64(y0, (n, neq))
        p = _f64(params, (n, npar))
        cnt = None if counters is None else _f64(counters, (n,))
        rec = np.empty((nchunks + 1, neq, n), dtype=np.float64) if records else None
        passes = np.zeros(n, dtype=np.int64)
        flags = np.zeros(n, dtype=np.int32)
        job = _Job(solver, neq, npar, nnoi, ksteps, printed_dt(dt), nchunks, n, orbit_offset,
                   _ptr(t), _ptr(y), _ptr(p), _ptr(cnt), _ptr(rec), newton_tol, newton_max_iter,
                   _ptr(passes), _ptr(flags), nthreads, rtol, atol, max_steps)
        rc = self.lib.oracle_run(C.byref(job))
        if rc != 0:
            raise RuntimeError("oracle_run failed with %d" % rc)
        return Result(rec, t, y, cnt, passes, flags)

    def threefry2x64_20(self, ctr, key):
        c = np.asarray(ctr, dtype=np.uint64).copy()
        k = np.asarray(key, dtype=np.uint64).copy()
        out = np.zeros(2, dtype=np.uint64)
        self.lib.oracle_threefry2x64_20(c.ctypes.data, k.ctypes.data, out.ctypes.data)
        return out

    def u01_open_open(self, w: int) -> float:
        return self.lib.oracle_u01_open_open_64_53(w)

    def counter_word(self, c: float) -> int:
        return self.lib.oracle_counter_word(c)

    def noise_stream(self, gid: int, counter: float, nnoi: int, dt: float, nsteps: int):
        out = np.empty((nsteps, nnoi), dtype=np.float64)
        self.lib.oracle_noise_stream(gid, counter, nnoi, printed_dt(dt), nsteps, out.ctypes.data)
        return out


class ReferenceBuild:
    """The reference's own kernels compiled as C (oracle/_ref)."""

    def __init__(self, system: str, solver: int, lib_dir: str = REF_DIR):
        path = os.path.join(lib_dir, "libref_%s_%s.so" % (system, REF_SOLVER_NAMES[solver]))
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.lib.ref_run.argtypes = [C.POINTER(_RefJob)]
        self.lib.ref_run.restype = C.c_int
        self.solver = solver

    @staticmethod
    def available(system: str, solver: int, lib_dir: str = REF_DIR) -> bool:
        return os.path.exists(os.path.join(lib_dir, "libref_%s_%s.so" % (system, REF_SOLVER_NAMES[solver])))

    def run(self, t0, y0, params, *, neq, npar, nnoi=0, dt, tspan=None, ksteps, nchunks=None,
            counters=None, orbit_offset=0, records=True, nthreads=0) -> Result:
        if nchunks is None:
            nchunks = num_chunks(tspan, dt, ksteps)
        t = _f64(t0)
        n = t.size
        y = _f64(y0, (n, neq))
        p = _f64(params, (n, npar))
        cnt = None if counters is None else _f64(counters, (n,))
        if self.solver == STOCHASTIC_EULER and cnt is None:
            raise ValueError("the stochastic build needs counters")
        rec = np.empty((nchunks + 1, neq, n), dtype=np.float64) if records else None
        job = _RefJob(neq, npar, nnoi, ksteps, printed_dt(dt), nchunks, n, orbit_offset, _ptr(t), _ptr(y),
                      _ptr(p), _ptr(cnt), _ptr(rec), printed_dt(NEWTON_TOL_DEFAULT), nthreads)
        rc = self.lib.ref_run(C.byref(job))
        if rc != 0:
            raise RuntimeError("ref_run failed with %d" % rc)
        return Result(rec, t, y, cnt)


def to_reference_layout(records: np.ndarray) -> np.ndarray:
    """``[record][equation][orbit]`` -> the ``(orbits*nequat, nrec)`` array the
    reference's Python wrapper returns (interfaces/python/sodecl.py:80)."""
    nrec = records.shape[0]
    return records.reshape(nrec, -1).T.copy()


def reference_gradient(system_file, solver, neq, npar, dt, ksteps, nchunks, t0, y0, params, targets,
                       newton_tol=1e-7, newton_max_iter=1000):
    """(loss[n], grad_params[n,npar], grad_y0[n,neq]) of the per-orbit MSE by
    forward-mode dual numbers through the system file (oracle/gradient.cpp),
    stepping with printed_dt(dt); the implicit solvers (3, 4) stop their
    Newton passes at printed_dt(newton_tol) or newton_max_iter passes."""
    import hashlib
    import subprocess
    import tempfile

    src = open(system_file, "rb").read()
    tag = hashlib.sha256(src + open(os.path.join(HERE, "gradient.cpp"), "rb").read()
                         + ("%d %d" % (neq, npar)).encode()).hexdigest()[:16]
    exe = os.path.join(BUILD_DIR, "gradient_%s" % tag)
    if not os.path.exists(exe):
        os.makedirs(BUILD_DIR, exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", '-DSYSTEM_FILE="%s"' % os.path.abspath(system_file),
                        "-DNUMEQ=%d" % neq, "-DNUMPAR=%d" % npar, os.path.join(HERE, "gradient.cpp"), "-o", exe],
                       check=True)
    t0 = np.ascontiguousarray(t0, dtype=np.float64)
    n = t0.size
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([n, nchunks, ksteps], dtype=np.int64).tobytes())
            f.write(np.array([printed_dt(dt)], dtype=np.float64).tobytes())
            for a in (t0, y0, params, targets):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        subprocess.run([exe, str(solver), fin, fout, repr(printed_dt(newton_tol)), str(int(newton_max_iter))],
                       check=True)
        out = np.fromfile(fout)
    return out[:n], out[n:n + n * npar].reshape(n, npar), out[n + n * npar:].reshape(n, neq)
