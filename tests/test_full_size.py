"""Parity at the benchmark configurations' full sizes, through properties that
do not depend on size.

  * oculomotor RK4, 2^20 orbits, 10^4 steps, a record every 100 (the headline
    shape, at the stable step dt 1e-5 so that trajectories are comparable):
    no orbit diverges, and orbits sampled across the whole index range (first,
    middle, last, and scattered ones) match the CPU oracle run on their inputs
    alone, within the floor-based tolerance of the other parity tests;
  * stochastic Kuramoto N=32, 2^18 orbits, 2x10^4 steps, a record every 200:
    every orbit's noise counter ends exactly at counter0 + steps x 16 draws,
    and sampled orbits match the oracle run with their global orbit index (the
    noise stream's key), within the oracle's own floor.

Records stay on the device; only the sampled columns come back."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from sodecl_b200 import Integrator, system_path
from sodecl_b200.workloads import kuramoto, oculomotor

pytestmark = pytest.mark.gpu


def _launch(sim, n, t0, y0, p, cnt=None):
    import torch

    dev = torch.device("cuda", 0)
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    td, yd, pd = T(t0), T(y0), T(p)
    cd = T(cnt) if cnt is not None else None
    rec = torch.empty((sim.num_records, sim.neq, n), dtype=torch.float64, device=dev)
    sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(),
               counters=cd.data_ptr() if cd is not None else None, records=rec.data_ptr(),
               stream=torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    return rec, yd, cd


def _samples(n, k, seed):
    rng = np.random.default_rng(seed)
    return np.unique(np.r_[0, 1, n // 2, n - 2, n - 1, rng.integers(0, n, k)])


def test_headline_shape_full_size():
    from test_gpu_parity import assert_parity

    n, nsteps, ksteps, dt = 1 << 20, 10000, 100, 1e-5
    t0, y0, p = oculomotor(n)
    sim = Integrator(system_path("oculomotor"), "rk4", dt=dt, tspan=nsteps * dt, ksteps=ksteps, neq=6, npar=6,
                     orbits=n)
    assert sim.num_chunks == nsteps // ksteps
    rec, yd, _ = _launch(sim, n, t0, y0, p)
    assert bool(rec.isfinite().all())
    idx = _samples(n, 27, 1)
    got = rec[:, :, idx].cpu().numpy()
    kw = dict(neq=6, npar=6, dt=dt, ksteps=ksteps, nchunks=nsteps // ksteps)
    want = Oracle("oculomotor").run(2, t0[idx], y0[idx], p[idx], **kw).records
    alt = Oracle("oculomotor", "fp64fma").run(2, t0[idx], y0[idx], p[idx], **kw).records
    assert_parity("2^20 orbits x 10^4 steps, %d sampled" % idx.size, got, want, alt)
    sim.close()


def test_stochastic_kuramoto_full_size():
    from test_gpu_parity import assert_parity

    n, N, nsteps, ksteps, dt = 1 << 18, 32, 20000, 200, 0.01
    t0, th0, p, cnt = kuramoto(n, N, noise=True)
    sim = Integrator(system_path("kuramoto"), "se", dt=dt, tspan=nsteps * dt, ksteps=ksteps, neq=N, npar=p.shape[1],
                     nnoi=N, orbits=n, lanes=16, block=256)
    rec, _, cd = _launch(sim, n, t0, th0, p, cnt)
    # every orbit drew exactly 16 Threefry pairs per step
    np.testing.assert_array_equal(cd.cpu().numpy(), cnt + nsteps * (N // 2))
    idx = _samples(n, 3, 2)
    got = rec[:, :, idx].cpu().numpy()
    kw = dict(neq=N, npar=p.shape[1], nnoi=N, dt=dt, ksteps=ksteps, nchunks=nsteps // ksteps)
    want, alt = [], []
    for i in idx:  # one oracle run per orbit, keyed by its global index
        one = dict(counters=cnt[i:i + 1], orbit_offset=int(i), **kw)
        want.append(Oracle("kuramoto").run(0, t0[i:i + 1], th0[i:i + 1], p[i:i + 1], **one).records)
        alt.append(Oracle("kuramoto", "fp64fma").run(0, t0[i:i + 1], th0[i:i + 1], p[i:i + 1], **one).records)
    assert_parity("2^18 orbits x 2x10^4 steps, %d sampled" % idx.size, got, np.concatenate(want, axis=2),
                  np.concatenate(alt, axis=2))
    sim.close()
