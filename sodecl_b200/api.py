"""numpy-level API over the C ABI (include/sodecl_cuda.h).

    from sodecl_b200 import Integrator
    sim = Integrator("sodecl_b200/systems/oculomotor.cl", solver=2, dt=1e-6, tspan=0.1,
                     ksteps=400, neq=6, npar=6, orbits=1024)
    sim.upload(t0, y0, params)
    records = sim.run()          # (num_records, neq, orbits), [record][equation][orbit]

Every call goes to libsodecl_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N

SOLVERS = {"se": N.STOCHASTIC_EULER, "stochastic_euler": N.STOCHASTIC_EULER, "euler": N.EULER, "e": N.EULER,
           "rk4": N.RUNGE_KUTTA, "r": N.RUNGE_KUTTA, "runge_kutta": N.RUNGE_KUTTA, "ie": N.IMPLICIT_EULER,
           "implicit_euler": N.IMPLICIT_EULER, "im": N.IMPLICIT_MIDPOINT, "implicit_midpoint": N.IMPLICIT_MIDPOINT,
           "dp45": N.DORMAND_PRINCE, "dopri5": N.DORMAND_PRINCE, "dormand_prince": N.DORMAND_PRINCE}
SYSTEMS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "systems")


def system_path(name: str) -> str:
    """Path of a system file shipped in sodecl_b200/systems (e.g. 'oculomotor')."""
    p = os.path.join(SYSTEMS_DIR, name if name.endswith(".cl") else name + ".cl")
    if not os.path.exists(p):
        raise FileNotFoundError(p)
    return p


def _solver_id(solver) -> int:
    if isinstance(solver, str):
        return SOLVERS[solver.lower()]
    return int(solver)


def _f64(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64)).reshape(-1)
    if a.size != n:
        raise ValueError("expected %d values, got %d" % (n, a.size))
    return a


class Integrator:
    """One configured run: a compiled program plus the orbits' state on a GPU."""

    def __init__(self, system, solver, *, dt, tspan, ksteps, neq, npar, orbits, nnoi=0, device=0,
                 precision="fp64", fmad=True, newton_tol=1e-7, newton_max_iter=1000, block=0,
                 record_f32=False, min_blocks=0, division="default", lanes=1, system_src=None, rtol=1e-6,
                 atol=1e-9, max_steps=100000, record_store="direct"):
        cfg = N.Cfg()
        N.lib.sodecl_cfg_init(C.byref(cfg))
        cfg.solver = _solver_id(solver)
        cfg.dt = float(dt)
        cfg.int_time = float(tspan)
        cfg.kernel_steps = int(ksteps)
        cfg.num_equat = int(neq)
        cfg.num_params = int(npar)
        cfg.num_noi = int(nnoi)
        cfg.list_size = int(orbits)
        cfg.device = int(device)
        cfg.local_group_size = int(block)
        cfg.precision = N.FP32 if str(precision).lower() in ("fp32", "float32", "1") else N.FP64
        cfg.fmad = 1 if fmad else 0
        cfg.newton_tol = float(newton_tol)
        cfg.newton_max_iter = int(newton_max_iter)
        cfg.record_f32 = 1 if record_f32 else 0
        cfg.min_blocks_per_sm = int(min_blocks)
        modes = {"default": N.DIV_DEFAULT, "reciprocal": N.DIV_RECIPROCAL, "ieee": N.DIV_IEEE}
        if str(division).lower() not in modes:
            raise ValueError("division must be 'default', 'reciprocal' or 'ieee', not %r" % (division,))
        cfg.division = modes[str(division).lower()]
        cfg.lanes_per_orbit = int(lanes)
        cfg.rtol = float(rtol)
        cfg.atol = float(atol)
        cfg.max_steps = int(max_steps)
        stores = {"direct": N.STORE_DIRECT, "pairs": N.STORE_PAIRS}
        if str(record_store).lower() not in stores:
            raise ValueError("record_store must be 'direct' or 'pairs', not %r" % (record_store,))
        cfg.record_store = stores[str(record_store).lower()]
        self.cfg = cfg
        self._ctx = C.c_void_p()
        rc = N.lib.sodecl_cuda_create(C.byref(cfg), C.byref(self._ctx))
        if rc != N.OK:
            raise N.SodeclError(rc, "invalid configuration")
        if system_src is None:
            with open(system, "rb") as f:
                system_src = f.read()
        elif isinstance(system_src, str):
            system_src = system_src.encode()
        self.system_src = system_src
        N.check(N.lib.sodecl_cuda_compile(self._ctx, system_src, len(system_src)), self._ctx)

    # ------------------------------------------------------------------ info
    @property
    def ctx(self):
        return self._ctx

    @property
    def orbits(self) -> int:
        return self.cfg.list_size

    @property
    def neq(self) -> int:
        return self.cfg.num_equat

    @property
    def num_records(self) -> int:
        return int(N.lib.sodecl_cuda_num_records(self._ctx))

    @property
    def num_chunks(self) -> int:
        return self.num_records - 1

    @property
    def program_source(self) -> str:
        return N.program_source(self._ctx)

    @property
    def build_log(self) -> str:
        return N.build_log(self._ctx)

    @property
    def division(self) -> str:
        """Division mode the program was built with ('reciprocal' or 'ieee')."""
        return "ieee" if N.lib.sodecl_cuda_program_division(self._ctx) == N.DIV_IEEE else "reciprocal"

    def autotune(self, sample_orbits=1 << 17, sample_steps=200):
        """Picks threads per block, the resident-block hint, the division mode,
        (for system files with sode_system_row) lanes per orbit and the record
        store form by timing them on copies of uploaded orbits; returns the
        choice."""
        b, m, d, ln, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        N.check(N.lib.sodecl_cuda_autotune(self._ctx, int(sample_orbits), int(sample_steps), C.byref(b), C.byref(m),
                                           C.byref(d), C.byref(ln), C.byref(ms)), self._ctx)
        N.check(N.lib.sodecl_cuda_get_cfg(self._ctx, C.byref(self.cfg)), self._ctx)
        return {"block": b.value, "min_blocks": m.value,
                "division": "reciprocal" if d.value == N.DIV_RECIPROCAL else "ieee", "lanes": ln.value,
                "record_store": "pairs" if self.cfg.record_store == N.STORE_PAIRS else "direct",
                "sample_ms": ms.value}

    def kernel_info(self):
        regs, local, mt = C.c_int(), C.c_int(), C.c_int()
        N.check(N.lib.sodecl_cuda_kernel_info(self._ctx, C.byref(regs), C.byref(local), C.byref(mt)), self._ctx)
        return {"registers": regs.value, "local_bytes": local.value, "max_threads": mt.value}

    def last_run_ms(self):
        k, t = C.c_double(), C.c_double()
        N.lib.sodecl_cuda_last_run_ms(self._ctx, C.byref(k), C.byref(t))
        return k.value, t.value

    # ----------------------------------------------------------------- state
    def upload(self, t0, y0, params, counters=None):
        n, neq, npar = self.cfg.list_size, self.cfg.num_equat, self.cfg.num_params
        self._t0 = _f64(t0, n)
        self._y0 = _f64(y0, n * neq)
        self._p = _f64(params, n * npar) if npar else np.zeros(1)
        self._cnt = None if counters is None else _f64(counters, n)
        N.check(N.lib.sodecl_cuda_upload(self._ctx, self._t0.ctypes.data, self._y0.ctypes.data, self._p.ctypes.data,
                                         None if self._cnt is None else self._cnt.ctypes.data), self._ctx)
        return self

    def run(self, out=None, discard=False):
        """Integrates over tspan from the current state; returns the records
        as an array (num_records, neq, orbits).  `out` may be a preallocated
        float64 array (e.g. pinned) of that size; discard=True keeps nothing."""
        if discard:
            N.check(N.lib.sodecl_cuda_run(self._ctx, None, 0), self._ctx)
            return None
        shape = (self.num_records, self.cfg.num_equat, self.cfg.list_size)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != int(np.prod(shape)):
            raise ValueError("out must be a C-contiguous float64 array of %s values" % (shape,))
        N.check(N.lib.sodecl_cuda_run(self._ctx, out.ctypes.data, out.size), self._ctx)
        return out.reshape(shape)

    def run_into(self, ptr: int, length: int):
        """run() into caller memory given as a raw address (host or device)."""
        N.check(N.lib.sodecl_cuda_run(self._ctx, C.c_void_p(ptr), int(length)), self._ctx)

    def state(self):
        n, neq = self.cfg.list_size, self.cfg.num_equat
        t = np.empty(n)
        y = np.empty((n, neq))
        cnt = np.empty(n)
        N.check(N.lib.sodecl_cuda_download_state(self._ctx, t.ctypes.data, y.ctypes.data, cnt.ctypes.data), self._ctx)
        return t, y, cnt

    def status(self):
        n = self.cfg.list_size
        passes = np.empty(n, dtype=np.int64)
        flags = np.empty(n, dtype=np.int32)
        N.check(N.lib.sodecl_cuda_status(self._ctx, passes.ctypes.data, flags.ctypes.data), self._ctx)
        return passes, flags

    # ------------------------------------------------------- device buffers
    def launch(self, *, t, y, params, counters=None, records=None, n=None, orbit_offset=0, rec_stride=None,
               rec_col0=0, chunk_begin=0, chunk_end=None, rec_first=0, write_final=True, newton_passes=None,
               flags=None, stream=None):
        """One launch over device buffers given as raw device addresses."""
        n = self.cfg.list_size if n is None else int(n)
        la = N.Launch()
        la.t, la.y, la.params, la.counters, la.records = t, y, params, counters, records
        la.n = n
        la.orbit_offset = orbit_offset
        la.rec_stride = n if rec_stride is None else rec_stride
        la.rec_col0 = rec_col0
        la.chunk_begin = chunk_begin
        la.chunk_end = self.num_chunks if chunk_end is None else chunk_end
        la.rec_first = rec_first
        la.write_final = 1 if write_final else 0
        la.newton_passes = newton_passes
        la.flags = flags
        N.check(N.lib.sodecl_cuda_launch(self._ctx, C.byref(la), stream), self._ctx)

    def release_scratch(self):
        """Frees the device buffers kept between calls (records of host-output
        runs, the adjoint's trajectory or checkpoints); later calls allocate
        them again."""
        N.check(N.lib.sodecl_cuda_release_scratch(self._ctx), self._ctx)

    def close(self):
        if self._ctx:
            N.lib.sodecl_cuda_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def noise_stream(gids, counters, nnoi, dt_program, nsteps, device=0, words=False, u01=False):
    """The Euler-Maruyama noise computed on the GPU (helper kernel sharing the
    solver's generator code): normals (n, nsteps, nnoi) and optionally the raw
    Threefry words / (0,1) doubles (n, nsteps, ncalls, 2)."""
    g = np.ascontiguousarray(np.asarray(gids, dtype=np.int64))
    c = np.ascontiguousarray(np.asarray(counters, dtype=np.float64))
    n = g.size
    ncalls = (nnoi + 1) // 2
    normals = np.empty((n, nsteps, nnoi))
    w = np.empty((n, nsteps, ncalls, 2), dtype=np.uint64) if words else None
    u = np.empty((n, nsteps, ncalls, 2)) if u01 else None
    N.check(N.lib.sodecl_cuda_noise_stream(device, g.ctypes.data, c.ctypes.data, n, nnoi, float(dt_program), nsteps,
                                           normals.ctypes.data, None if w is None else w.ctypes.data,
                                           None if u is None else u.ctypes.data))
    return normals, w, u


def fma_peak(precision="fp64", device=0):
    """Measured FMA instructions per second (all lanes) of the FP64 or FP32 pipe."""
    rate, ms = C.c_double(), C.c_double()
    prec = N.FP32 if precision == "fp32" else N.FP64
    N.check(N.lib.sodecl_cuda_fma_peak(device, prec, C.byref(rate), C.byref(ms)))
    return rate.value, ms.value


def sin_peak(precision="fp64", device=0):
    """Measured sine evaluations per second of the math library's sin (FP64 or
    FP32) at full occupancy, arguments within a few units of zero."""
    rate, ms = C.c_double(), C.c_double()
    prec = N.FP32 if precision == "fp32" else N.FP64
    N.check(N.lib.sodecl_cuda_sin_peak(device, prec, C.byref(rate), C.byref(ms)))
    return rate.value, ms.value
