"""Heterogeneous batches over the C ABI (sodecl_batch_* in include/sodecl_cuda.h).

    b = Batch(device=0)
    k_osc = b.add_class(system_path("kuramoto"), "rk4", neq=16, npar=17, dt=0.01)
    k_ocm = b.add_class(system_path("oculomotor"), "ie", neq=6, npar=6, dt=1e-3)
    b.compile()
    b.set_items(classes, nsteps, t0, y0_list, p_list)   # per-orbit widths follow the class
    b.run(graph=True)
    t, y, counters, passes, flags = b.results()

One persistent kernel integrates all orbits, each with its own step count,
taking them from per-class device work queues.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .api import _solver_id


def _err(b):
    n = N.lib.sodecl_batch_last_error(b, None, 0)
    buf = C.create_string_buffer(n + 1)
    N.lib.sodecl_batch_last_error(b, buf, n + 1)
    return buf.value.decode(errors="replace")


class Batch:
    def __init__(self, device=0, fmad=True, division="reciprocal"):
        self._b = C.c_void_p()
        div = N.DIV_RECIPROCAL if division == "reciprocal" else N.DIV_IEEE
        N.check(N.lib.sodecl_batch_create(int(device), 1 if fmad else 0, div, C.byref(self._b)))
        self.classes = []

    def _check(self, rc):
        if rc != N.OK:
            raise N.SodeclError(rc, _err(self._b))

    def add_class(self, system, solver, *, neq, npar, dt, nnoi=0, newton_tol=1e-7, newton_max_iter=1000,
                  lanes=0, system_src=None):
        """lanes: lanes per orbit (0 automatic, 1 one lane, 2..32 a power of two)."""
        cfg = N.ClassCfg()
        N.lib.sodecl_class_cfg_init(C.byref(cfg))
        cfg.solver, cfg.num_equat, cfg.num_params, cfg.num_noi = _solver_id(solver), neq, npar, nnoi
        cfg.dt, cfg.newton_tol, cfg.newton_max_iter = dt, newton_tol, newton_max_iter
        cfg.lanes_per_orbit = int(lanes)
        if system_src is None:
            with open(system, "rb") as f:
                system_src = f.read()
        elif isinstance(system_src, str):
            system_src = system_src.encode()
        cid = C.c_int32()
        self._check(N.lib.sodecl_batch_add_class(self._b, system_src, len(system_src), C.byref(cfg), C.byref(cid)))
        self.classes.append(dict(neq=neq, npar=npar, solver=cfg.solver, nnoi=nnoi))
        return cid.value

    def compile(self):
        self._check(N.lib.sodecl_batch_compile(self._b))
        return self

    def set_items(self, item_class, nsteps, t0, y0, params, counters=None):
        """y0/params: flat arrays packed in item order (each item's width is its
        class's neq/npar), or lists of per-item arrays."""
        cls = np.ascontiguousarray(item_class, dtype=np.int32)
        steps = np.ascontiguousarray(nsteps, dtype=np.int64)
        t = np.ascontiguousarray(t0, dtype=np.float64)
        pack = lambda a: np.ascontiguousarray(np.concatenate([np.ravel(x) for x in a]) if isinstance(a, list)  # noqa
                                              else np.ravel(a), dtype=np.float64)
        self._y, self._p = pack(y0), pack(params)
        self._cls, self._steps, self._t = cls, steps, t
        self._cnt = None if counters is None else np.ascontiguousarray(counters, dtype=np.float64)
        widths = np.array([c["neq"] for c in self.classes] or [0])[np.clip(cls, 0, max(0, len(self.classes) - 1))]
        pw = np.array([c["npar"] for c in self.classes] or [0])[np.clip(cls, 0, max(0, len(self.classes) - 1))]
        if self.classes and (self._y.size != widths.sum() or self._p.size != pw.sum()):
            raise ValueError("packed y0/params do not match the classes' widths")
        self._check(N.lib.sodecl_batch_set_items(self._b, cls.size, cls.ctypes.data, steps.ctypes.data, t.ctypes.data,
                                                 self._y.ctypes.data, self._p.ctypes.data if self._p.size else None,
                                                 None if self._cnt is None else self._cnt.ctypes.data))
        self._widths = widths
        return self

    def set_launch(self, block, blocks_per_sm=0):
        self._check(N.lib.sodecl_batch_set_launch(self._b, block, blocks_per_sm))

    def tune(self):
        """Times lanes per orbit for the automatic classes, then launch shapes,
        on the current items (every trial advances them); returns (threads per
        block, resident blocks per SM, best ms).  `lanes` gives the classes'
        lanes per orbit."""
        blk, bps, ms = C.c_int32(), C.c_int32(), C.c_double()
        self._check(N.lib.sodecl_batch_tune(self._b, C.byref(blk), C.byref(bps), C.byref(ms)))
        return blk.value, bps.value, ms.value

    @property
    def lanes(self):
        """Lanes per orbit of each class."""
        out = (C.c_int32 * max(1, len(self.classes)))()
        self._check(N.lib.sodecl_batch_class_lanes(self._b, out))
        return [int(v) for v in out[:len(self.classes)]]

    def run(self, graph=True):
        self._check(N.lib.sodecl_batch_run(self._b, 1 if graph else 0))
        return self.last_ms

    @property
    def last_ms(self):
        ms = C.c_double()
        N.lib.sodecl_batch_last_ms(self._b, C.byref(ms))
        return ms.value

    def kernel_info(self):
        r, l = C.c_int(), C.c_int()
        self._check(N.lib.sodecl_batch_kernel_info(self._b, C.byref(r), C.byref(l)))
        return {"registers": r.value, "local_bytes": l.value}

    @property
    def program_source(self):
        n = N.lib.sodecl_batch_program_source(self._b, None, 0)
        buf = C.create_string_buffer(n + 1)
        N.lib.sodecl_batch_program_source(self._b, buf, n + 1)
        return buf.value.decode(errors="replace")

    def results(self):
        """(t, y as a list of per-item arrays, counters, newton passes, flags)."""
        n = self._cls.size
        t = np.empty(n)
        y = np.empty(self._y.size)
        cnt = np.empty(n)
        passes = np.empty(n, dtype=np.int64)
        flags = np.empty(n, dtype=np.int32)
        self._check(N.lib.sodecl_batch_results(self._b, t.ctypes.data, y.ctypes.data, cnt.ctypes.data,
                                               passes.ctypes.data, flags.ctypes.data))
        ys = np.split(y, np.cumsum(self._widths)[:-1])
        return t, ys, (cnt if self._cnt is not None else None), passes, flags

    def close(self):
        if self._b:
            N.lib.sodecl_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
