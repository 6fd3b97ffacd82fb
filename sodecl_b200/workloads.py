"""Seeded synthetic workloads of the benchmark shapes, and a command line that
runs a few launches of one of them (for profiler captures).

    python -m sodecl_b200.workloads stochastic-kuramoto --orbits 32768 --nsteps 200 --lanes 16 --block 256

Shapes (all inputs seeded; no dataset is involved):
  oculomotor-<solver>   the oculomotor model: parameters uniform within +-50 % of
                        the nominal (120, 1.5, 0.0045, 0.05, 600, 9), y0 =
                        (0, 0, 0, 0, 0, 2); default RK4, dt 1e-3, a record every 100
  stochastic-kuramoto   Kuramoto by Euler-Maruyama: N phases, K ~ U(0,5),
                        omega ~ N(0,1) shared, additive noise sigma ~ U(0,0.5) per
                        orbit, counters orbit * 2^20; dt 0.01, a record every 200
  kuramoto-<solver>     deterministic Kuramoto: N phases, K ~ U(0,5), omega ~ N(0,1)
                        shared, theta0 ~ U(0, 2 pi); dt 0.01
  uneven-batch          the persistent batch kernel over the uneven sweep: Kuramoto
                        N in {4, 16, 64} and the oculomotor model x {Euler, RK4,
                        implicit Euler}, step counts log-uniform in [100, max-steps]
  adjoint-oculomotor    loss and gradient (sodecl_cuda_adjoint) of the oculomotor
                        RK4 fit: targets from seeded true parameters + N(0, 1e-2)
                        noise, gradient at parameters within +-5 % of them; dt 1e-5
  peaks                 the measured ceilings: FMA issue rate and sine throughput,
                        FP64 and FP32 (sodecl_cuda_fma_peak, sodecl_cuda_sin_peak)
"""
from __future__ import annotations

import argparse
import json

import numpy as np

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])


def oculomotor(n, orbit_offset=0, seed=2024):
    """(t0, y0, params) of orbits [orbit_offset, orbit_offset + n)."""
    rng = np.random.default_rng([seed, orbit_offset])
    params = NOMINAL * rng.uniform(0.5, 1.5, (n, 6))
    return np.zeros(n), np.tile(Y0, (n, 1)), params


def kuramoto(n, N, seed=3, noise=False):
    """(t0, theta0, params, counters): params = [K, omega_1..N] (+ sigma_1..N,
    one sigma per orbit, with noise); counters orbit * 2^20 with noise, else None."""
    rng = np.random.default_rng(seed)
    cols = [rng.uniform(0, 5, (n, 1)), np.tile(rng.normal(size=N), (n, 1))]
    if noise:
        cols.append(np.repeat(rng.uniform(0, 0.5, (n, 1)), N, axis=1))
    params = np.concatenate(cols, axis=1)
    theta0 = rng.uniform(0, 2 * np.pi, (n, N))
    counters = np.arange(n) * 2.0 ** 20 if noise else None
    return np.zeros(n), theta0, params, counters


# the uneven sweep's classes: (system, solver, equations, parameters, dt)
UNEVEN_CLASSES = [("kuramoto", solver, N, N + 1, 0.01) for N in (4, 16, 64) for solver in ("euler", "rk4", "ie")] + \
                 [("oculomotor", solver, 6, 6, dt) for solver, dt in (("euler", 1e-6), ("rk4", 1e-5), ("ie", 1e-3))]


def uneven_batch(n, max_steps, seed=4):
    """(classes, class per orbit, step counts, y0 list, params list, generator)
    of the uneven sweep: Kuramoto N in {4, 16, 64} and the oculomotor model,
    solver in {Euler, RK4, implicit Euler} (12 classes, drawn uniformly), step
    counts log-uniform in [10^2, max_steps]."""
    rng = np.random.default_rng(seed)
    cls = rng.integers(0, len(UNEVEN_CLASSES), n).astype(np.int32)
    steps = np.exp(rng.uniform(np.log(100), np.log(max_steps), n)).astype(np.int64)
    y0, p = [], []
    for c in cls:
        system, solver, neq, npar, dt = UNEVEN_CLASSES[c]
        if system == "oculomotor":
            y0.append(Y0)
            p.append(NOMINAL * rng.uniform(0.5, 1.5, 6))
        else:
            y0.append(rng.uniform(0, 2 * np.pi, neq))
            p.append(np.concatenate([[rng.uniform(0, 5)], rng.normal(size=neq)]))
    return UNEVEN_CLASSES, cls, steps, y0, p, rng


def _batch_main(a):
    from . import system_path
    from .batch import Batch

    classes, cls, steps, y0, p, rng = uneven_batch(a.orbits, a.max_steps)
    b = Batch()
    for system, solver, neq, npar, dt in classes:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, dt=dt)
    b.compile()
    # tune on every orbit with its step count divided by 64 (trials advance
    # the items; the real ones are set below)
    b.set_items(cls, np.maximum(1, steps // 64), np.zeros(a.orbits), y0, p)
    block, bps, _ = b.tune()
    for k in range(a.launches):
        b.set_items(cls, steps, np.zeros(a.orbits), y0, p)
        ms = b.run(graph=True)
        print(json.dumps({"case": a.case, "launch": k, "ms": ms, "orbits": a.orbits, "max_steps": a.max_steps,
                          "orbit_steps": int(steps.sum()), "orbit_steps_per_s": int(steps.sum()) / (ms * 1e-3),
                          "block": block, "blocks_per_sm": bps, "lanes": b.lanes}), flush=True)


def fitting_targets(n, nsteps, ksteps, dt, seed=55, device="cuda", solver="rk4", newton_tol=1e-7):
    """(t0, y0, guess params, targets[records, 6, n]) of the oculomotor fit:
    the trajectories of seeded true parameters (integrated with `solver`)
    plus N(0, 1e-2) noise; the guess is within 5 % of the truth."""
    import torch

    from . import Integrator, system_path

    rng = np.random.default_rng(seed)
    true_p = NOMINAL * rng.uniform(0.5, 1.5, (n, 6))
    guess = true_p * rng.uniform(0.95, 1.05, (n, 6))
    y0 = np.tile(Y0, (n, 1))
    sim = Integrator(system_path("oculomotor"), solver, dt=dt, tspan=(nsteps - 0.5) * dt, ksteps=ksteps, neq=6,
                     npar=6, orbits=n, newton_tol=newton_tol)
    T = lambda x: torch.tensor(x, device=device)  # noqa: E731
    rec = torch.empty((sim.num_records, 6, n), dtype=torch.float64, device=device)
    td, yd, pd = T(np.zeros(n)), T(y0), T(true_p)
    sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=rec.data_ptr(),
               stream=torch.cuda.current_stream(device).cuda_stream)
    gen = torch.Generator(device=device).manual_seed(7)
    targets = rec + 1e-2 * torch.randn(rec.shape, dtype=torch.float64, device=device, generator=gen)
    torch.cuda.synchronize()
    sim.close()
    return np.zeros(n), y0, guess, targets


def _adjoint_main(a):
    import torch

    from . import Integrator, system_path
    from .fit import Adjoint

    dt = a.dt if a.dt is not None else 1e-5
    t0, y0, guess, targets = fitting_targets(a.orbits, a.nsteps, a.ksteps, dt)
    sim = Integrator(system_path("oculomotor"), "rk4", dt=dt, tspan=(a.nsteps - 0.5) * dt, ksteps=a.ksteps, neq=6,
                     npar=6, orbits=a.orbits)
    T = lambda x: torch.tensor(x, device="cuda")  # noqa: E731
    adj = Adjoint(sim, ckpt_every=a.ckpt_every)
    for k in range(a.launches):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        adj(T(t0), T(y0), T(guess), targets)
        e.record()
        torch.cuda.synchronize()
        print(json.dumps({"case": a.case, "launch": k, "ms": s.elapsed_time(e), "orbits": a.orbits,
                          "nsteps": a.nsteps, "ckpt_every": a.ckpt_every}), flush=True)


def _parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", help="oculomotor-<solver> | stochastic-kuramoto | kuramoto-<solver> | uneven-batch | "
                                 "adjoint-oculomotor | peaks")
    ap.add_argument("--orbits", type=int, default=1 << 15)
    ap.add_argument("--nsteps", type=int, default=200)
    ap.add_argument("--ksteps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--N", type=int, default=32, help="Kuramoto phases")
    ap.add_argument("--lanes", type=int, default=1)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--division", default="ieee", choices=["default", "ieee", "reciprocal"])
    ap.add_argument("--ckpt-every", type=int, default=0,
                    help="adjoint-oculomotor: steps per checkpoint (0: the library's choice; >= nsteps: the "
                         "forward sweep records the whole trajectory)")
    ap.add_argument("--min-blocks", type=int, default=0)
    ap.add_argument("--record-store", default="direct", choices=["direct", "pairs"])
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--max-steps", type=int, default=10000, help="uneven-batch: longest step count")
    ap.add_argument("--system-file", default=None,
                    help="oculomotor-*, kuramoto-*, stochastic-kuramoto: integrate this system file instead of "
                         "the package's (e.g. the reference's own examples/oculomotor.cl)")
    return ap.parse_args()


def main():
    import torch

    from . import Integrator, system_path

    a = _parse()
    n = a.orbits
    if a.case == "peaks":
        from . import fma_peak, sin_peak

        for prec in ("fp64", "fp32"):
            fma, fms = fma_peak(prec)
            sines, sms = sin_peak(prec)
            print(json.dumps({"case": a.case, "precision": prec, "fma_per_s": fma, "fma_ms": fms, "sin_per_s": sines,
                              "sin_ms": sms}), flush=True)
        return
    if a.case == "adjoint-oculomotor":
        return _adjoint_main(a)
    if a.case == "uneven-batch":
        return _batch_main(a)
    if a.case.startswith("oculomotor"):
        solver = a.case.split("-", 1)[1] if "-" in a.case else "rk4"
        dt = a.dt if a.dt is not None else 1e-3
        t0, y0, p = oculomotor(n)
        cnt, system, neq, nnoi = None, "oculomotor", 6, 0
    elif a.case == "stochastic-kuramoto":
        solver, dt = "se", a.dt if a.dt is not None else 0.01
        t0, y0, p, cnt = kuramoto(n, a.N, noise=True)
        system, neq, nnoi = "kuramoto", a.N, a.N
    elif a.case.startswith("kuramoto-"):
        solver, dt = a.case.split("-", 1)[1], a.dt if a.dt is not None else 0.01
        t0, y0, p, cnt = kuramoto(n, a.N)
        system, neq, nnoi = "kuramoto", a.N, 0
    else:
        raise SystemExit("unknown case " + a.case)
    sim = Integrator(a.system_file or system_path(system), solver, dt=dt, tspan=a.nsteps * dt, ksteps=a.ksteps, neq=neq,
                     npar=p.shape[1], nnoi=nnoi, orbits=n, precision=a.precision, lanes=a.lanes, block=a.block,
                     division=a.division, min_blocks=a.min_blocks, record_store=a.record_store)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    td, yd, pd = T(t0), T(y0), T(p)
    cd = T(cnt) if cnt is not None else None
    rec = torch.empty((sim.num_records, neq, n), dtype=torch.float64, device=dev)
    for k in range(a.launches):
        td.copy_(T(t0))
        yd.copy_(T(y0))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(),
                   counters=cd.data_ptr() if cd is not None else None, records=rec.data_ptr(),
                   stream=stream.cuda_stream)
        e.record(stream)
        torch.cuda.synchronize()
        ms = s.elapsed_time(e)
        print(json.dumps({"case": a.case, "launch": k, "ms": ms, "orbit_steps_per_s": n * a.nsteps / (ms * 1e-3),
                          "lanes": a.lanes, "block": a.block or 128, "orbits": n, "nsteps": a.nsteps,
                          "division": sim.division, "min_blocks": a.min_blocks,
                          "record_store": a.record_store}), flush=True)
    sim.close()


if __name__ == "__main__":
    main()
