"""Regenerates the golden fixtures in this directory.

Run where the reference checkout is present (its location is the one
oracle/build.py reads, REFERENCE_ROOT there) after `python oracle/build.py`:

    python tests/golden/make_golden.py

1. oculomotor_{euler,rk,ie,im}.npy -- the reference's own known-answer arrays
   (tests/data/oculomotor_*.pkl, pinned by tests/sodecl_python_tests.py:9-179),
   re-saved as .npy: float64 (12, records), row eq*orbits + orbit.
2. ref_*.npz -- inputs and outputs of the reference's kernel sources
   (src/kernels/*.cl + examples/*.cl) compiled as C (oracle/_ref), for paths
   the reference's tests do not pin: Euler-Maruyama with Threefry noise,
   Kuramoto, implicit midpoint with varied parameters, raw Threefry words.
"""
from __future__ import annotations

import os
import pickle
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.build import REFERENCE_ROOT  # noqa: E402
from oracle.oracle import ReferenceBuild, num_chunks  # noqa: E402

OCULOMOTOR_NOMINAL = [120.0, 1.5, 0.0045, 0.05, 600.0, 9.0]
OCULOMOTOR_Y0 = [0.0, 0.0, 0.0, 0.0, 0.0, 2.0]


def convert_pickles():
    for name in ("euler", "rk", "ie", "im"):
        src = os.path.join(REFERENCE_ROOT, "tests", "data", "oculomotor_%s.pkl" % name)
        with open(src, "rb") as f:
            arr = np.asarray(pickle.load(f), dtype=np.float64)
        np.save(os.path.join(HERE, "oculomotor_%s.npy" % name), arr)


def ref_case(name, system, solver, *, neq, npar, nnoi, dt, tspan, ksteps, t0, y0, p, counters=None, orbit_offset=0):
    r = ReferenceBuild(system, solver).run(t0, y0, p, neq=neq, npar=npar, nnoi=nnoi, dt=dt, tspan=tspan,
                                           ksteps=ksteps, counters=counters, orbit_offset=orbit_offset)
    out = dict(solver=solver, neq=neq, npar=npar, nnoi=nnoi, dt=dt, tspan=tspan, ksteps=ksteps,
               nchunks=num_chunks(tspan, dt, ksteps), orbit_offset=orbit_offset, t0=np.asarray(t0, float),
               y0=np.asarray(y0, float), params=np.asarray(p, float), records=r.records, t_final=r.t,
               y_final=r.y)
    if counters is not None:
        out["counters"] = np.asarray(counters, float)
        out["counters_final"] = r.counters
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)


def make_reference_cases():
    rng = np.random.default_rng(20240501)
    # Kuramoto N=8 Euler, the CPU-runnable configuration's shape (8 orbits of 1024)
    n, N = 8, 8
    omega = rng.normal(size=N)
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(omega, (n, 1))], axis=1)
    ref_case("kuramoto_euler", "kuramoto", 1, neq=N, npar=N + 1, nnoi=0, dt=0.05, tspan=50.0, ksteps=10,
             t0=np.zeros(n), y0=rng.uniform(0, 2 * np.pi, (n, N)), p=p)
    # Kuramoto N=3 Euler-Maruyama, the shape of the reference's README run
    # (dt 0.05, tspan 50, ksteps 40); counters: non-negative integers and
    # negative non-integers (the reference draws U(-1e11, 1e11))
    n, N = 8, 3
    p = np.concatenate([np.full((n, 1), 0.2), rng.uniform(0.2, 0.4, (n, N)), rng.uniform(0.01, 0.03, (n, N))], axis=1)
    cnt = np.concatenate([np.arange(4) * 2.0 ** 20, rng.uniform(-1e11, 1e11, 4)])
    ref_case("kuramoto_se", "kuramoto", 0, neq=N, npar=2 * N + 1, nnoi=N, dt=0.05, tspan=50.0, ksteps=40,
             t0=np.zeros(n), y0=rng.uniform(-3.1416, 3.1416, (n, N)), p=p, counters=cnt, orbit_offset=5)
    # Kuramoto N=32 Euler-Maruyama (the stochastic configuration's shape), short
    n, N = 4, 32
    p = np.concatenate([rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N), (n, 1)),
                        np.repeat(rng.uniform(0, 0.5, (n, 1)), N, axis=1)], axis=1)
    ref_case("kuramoto32_se", "kuramoto", 0, neq=N, npar=2 * N + 1, nnoi=N, dt=0.01, tspan=4.0, ksteps=200,
             t0=np.zeros(n), y0=rng.uniform(0, 2 * np.pi, (n, N)), p=p,
             counters=np.arange(n) * 2.0 ** 20, orbit_offset=1000)
    # oculomotor Euler-Maruyama with two noise processes
    n = 4
    p = np.concatenate([np.tile(OCULOMOTOR_NOMINAL, (n, 1)), np.tile([0.05, 0.01], (n, 1))], axis=1)
    ref_case("oculomotor_se", "oculomotor", 0, neq=6, npar=8, nnoi=2, dt=1e-5, tspan=0.01, ksteps=100,
             t0=np.zeros(n), y0=np.tile(OCULOMOTOR_Y0, (n, 1)), p=p, counters=np.array([0.0, 1.0, 7.0, 123456789.0]))
    # oculomotor implicit midpoint / implicit Euler / RK4 with parameters within
    # +-50% of nominal, dt 1e-3 (the 2^20-orbit configuration's step), short
    n = 8
    p = np.asarray(OCULOMOTOR_NOMINAL) * rng.uniform(0.5, 1.5, (n, 6))
    for name, solver, dt in (("oculomotor_im", 4, 1e-3), ("oculomotor_ie", 3, 1e-3), ("oculomotor_rk4", 2, 1e-5)):
        ref_case(name, "oculomotor", solver, neq=6, npar=6, nnoi=0, dt=dt, tspan=1000 * dt, ksteps=100,
                 t0=np.zeros(n), y0=np.tile(OCULOMOTOR_Y0, (n, 1)), p=p)


def make_threefry_words():
    """Threefry-2x64-20 words and their (0,1) doubles from the reference's
    vendored Random123 headers (oracle/_ref/libref_threefry.so), on counters
    {orbit, draw} spanning the 64-bit range, key {0, 0xf00dcafe}."""
    import ctypes as C

    lib = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_threefry.so"))
    lib.ref_u01_open_open_64_53.restype = C.c_double
    lib.ref_u01_open_open_64_53.argtypes = [C.c_uint64]
    rng = np.random.default_rng(7)
    ctrs = [(0, 0), (1, 0), (0, 1), (12345, 678), (2 ** 20, 2 ** 40), (2 ** 63, 2 ** 64 - 1)]
    ctrs += [tuple(int(v) for v in rng.integers(0, 2 ** 63, 2, dtype=np.int64)) for _ in range(58)]
    ctr = np.array(ctrs, dtype=np.uint64)
    key = np.array([0, 0xF00DCAFE], dtype=np.uint64)
    words = np.zeros_like(ctr)
    for i in range(len(ctr)):
        c = np.ascontiguousarray(ctr[i])
        out = np.zeros(2, dtype=np.uint64)
        lib.ref_threefry2x64(C.c_void_p(c.ctypes.data), C.c_void_p(key.ctypes.data), C.c_void_p(out.ctypes.data))
        words[i] = out
    u01 = np.array([[lib.ref_u01_open_open_64_53(int(w)) for w in row] for row in words])
    np.savez_compressed(os.path.join(HERE, "threefry_words.npz"), ctr=ctr, key=key, words=words, u01=u01)


if __name__ == "__main__":
    convert_pickles()
    make_reference_cases()
    make_threefry_words()
    for f in sorted(os.listdir(HERE)):
        if f.endswith((".npy", ".npz")):
            print(f, os.path.getsize(os.path.join(HERE, f)))
