"""The reference's Python entry point, sodecl.sodecl(...), over the CUDA engine.

Same signature, argument meaning and return value as the reference's
interfaces/python/sodecl.py:35-84:

    t, results = sodecl(openclplatform, opencldevice, openclkernel, initx, params,
                        sodesolver, orbits, nequat, nnoiseprocesses, dt, tspan,
                        ksteps, localgroupsize)

results has shape (orbits*nequat, records); row eq*orbits + orbit.  The
platform argument is ignored and the device is the CUDA ordinal.  Extra
keywords (precision, fmad, newton_tol, newton_max_iter, counters) expose this
library's options.

t is built as the reference builds it, numpy.arange(0, tspan + dt*ksteps,
dt*ksteps), which in floating point can hold one entry more or fewer than there
are records (tspan 0.2 with dt*ksteps 0.1: four times, three records).  With
exact_time=True, t holds one time per record instead: record r at r*dt*ksteps.
"""
from __future__ import annotations

import numpy

from . import sodecl_interface


def sodecl(openclplatform, opencldevice, openclkernel, initx, params, sodesolver, orbits, nequat, nnoiseprocesses,
           dt, tspan, ksteps, localgroupsize, *, precision=0, fmad=1, newton_tol=1e-7, newton_max_iter=1000,
           counters=None, exact_time=False):
    # t0 = 0 for every orbit; nparams from the first parameter row (sodecl.py:40-46)
    t0 = numpy.zeros(orbits)
    nparams = numpy.asarray(params)[0].size
    # flattened in C order, as the reference's flatten() calls do
    # (sodecl.py:44-46); ravel copies only what is not already contiguous
    initx = numpy.ravel(numpy.asarray(initx, dtype=numpy.float64))
    params = numpy.ravel(numpy.asarray(params, dtype=numpy.float64))

    # solver choice (sodecl.py:48-61): any noise forces Euler-Maruyama; an
    # unknown deterministic solver falls back to Euler
    if nnoiseprocesses == 0:
        if 0 < sodesolver < 5:
            solver2user = sodesolver
        else:
            print("Invalid SODE solver selected! Using Euler!")
            solver2user = 1
    else:
        solver2user = 0

    results = sodecl_interface.sodeclcall_array(
        t0, initx, params, openclplatform, opencldevice, openclkernel, solver2user, orbits, nequat, nparams,
        nnoiseprocesses, dt, tspan, ksteps, localgroupsize, precision=precision, fmad=fmad, newton_tol=newton_tol,
        newton_max_iter=newton_max_iter, counters=None if counters is None else numpy.asarray(counters, dtype=float))

    results = numpy.asarray(results)
    if results.size == 0:
        t = numpy.zeros(0) if exact_time else numpy.arange(0, tspan + dt * ksteps, dt * ksteps)
        return t, results.reshape(orbits * nequat, 0)
    results = results.reshape(orbits * nequat, int(results.shape[0] / (orbits * nequat)), order='F')

    if exact_time:
        t = numpy.arange(results.shape[1]) * (dt * ksteps)
    else:
        # time axis as the reference builds it (sodecl.py:82)
        t = numpy.arange(0, tspan + dt * ksteps, dt * ksteps)
    return t, results
