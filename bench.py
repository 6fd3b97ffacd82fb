"""Throughput benchmark: orbit-steps/s of the fixed-step integrators on B200.

Workload (one "step" = one full integration of one batch of orbits):
  oculomotor model (6 states, 6 parameters), RK4, 2^20 orbits per GPU,
  parameters uniform within +-50% of the nominal values (seeded), y0 = the
  reference example's initial state, dt = 1e-3, 10^4 steps, a record every
  100 steps (101 records, [record][equation][orbit], FP64).  The system file
  is the reference's own examples/oculomotor.cl, as shipped (the staged copy
  under baseline/_ref); the package's restated file is a companion line.

  value     device-resident: inputs already in HBM, one launch per step,
            CUDA-event time of that launch (L2 flushed between steps).
  e2e       the same run through the C ABI with host buffers: upload of the
            inputs from pinned host memory + run with the records copied into
            pinned host memory, every step (wall clock of the synchronous calls).
  roofline  counted FP64 operations of the model (224 per RK4 orbit-step,
            source-level count) over the launch time, against the FP64 FMA
            issue peak measured on the same GPU by the library's
            microbenchmark (2 flops per FMA).
  cpu_baseline  the reference's kernels compiled as C (oracle/_ref), OpenMP over
            all host cores, on an orbit subsample of the same workload.
  parity    the timed launch's records of that subsample against the CPU
            baseline's: relative error over the orbits finite in both runs,
            and counts of the orbits that diverge in both or in one only;
            beside it the floor, the same measure between the CPU baseline
            and the oracle compiled with FMA contraction, and whether the
            error is within 10x the floor (the GPU parity tests' rule).

--impl reference runs only that CPU implementation of the path (rank 0), on
the cpu_baseline leg's sample: the first 2^15 orbits with all 10^4 steps per
step, so that its ms_per_step is the measured time of that sample.
Under torchrun each rank integrates its own 2^20 orbits (global orbit ids
offset by rank): weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])
RK4_OPS_PER_ORBIT_STEP = 224  # 4 x 35 (right-hand side) + 6 x 14 (stage arithmetic)
METRIC = "orbit-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--orbits", type=int, default=1 << 20)
    ap.add_argument("--nsteps", type=int, default=10000)
    ap.add_argument("--ksteps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--solver", default="rk4")
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--cpu-orbits", type=int, default=1 << 15)
    ap.add_argument("--no-extras", action="store_true", help="skip the companion measurements")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape")
    return ap.parse_args()


# the reference's own system file, staged verbatim by oracle/build.py
REFERENCE_SYSTEM = os.path.join(REPO, "baseline", "_ref", "examples", "oculomotor.cl")
PACKAGE_SYSTEM = os.path.join(REPO, "sodecl_b200", "systems", "oculomotor.cl")
REFERENCE_KURAMOTO = os.path.join(REPO, "baseline", "_ref", "examples", "kuramoto.cl")


@contextlib.contextmanager
def stdout_to_stderr():
    """Sends what native code prints to standard output (the C++ manager's
    'Compute results runtime' line, as the reference prints it) to standard
    error, so that the bench's standard output carries its JSON line alone.
    The C library's buffers are flushed before the descriptor is restored."""
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def headline_system():
    """(path, label) of the system file the headline integrates."""
    if os.path.isfile(REFERENCE_SYSTEM):
        return REFERENCE_SYSTEM, "reference examples/oculomotor.cl (unmodified)"
    return PACKAGE_SYSTEM, "sodecl_b200/systems/oculomotor.cl (the reference's file is not staged here)"


def workload(n, orbit_offset, seed=2024):
    """Seeded inputs of orbits [orbit_offset, orbit_offset + n); pure numpy
    (sodecl_b200.workloads maps no native library)."""
    from sodecl_b200.workloads import oculomotor

    return oculomotor(n, orbit_offset, seed)


def config_dict(a, n):
    """The workload; both arms print exactly this."""
    return {"workload": "oculomotor-%s-%s" % (a.solver, a.precision), "system_file": headline_system()[1],
            "orbits_per_gpu": n, "nsteps": a.nsteps, "record_every": a.ksteps, "records": a.nsteps // a.ksteps + 1,
            "dt": a.dt, "neq": 6, "npar": 6, "layout": "[record][equation][orbit]",
            "l2": "flushed between steps (256 MiB write)"}


class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_rate(n, a, cores, kind_pref="reference"):
    """(orbit-steps/s, seconds, kind, records) of the CPU implementation on the
    first n orbits."""
    from oracle.oracle import Oracle, ReferenceBuild

    t0, y0, p = workload(n, 0)
    solver = {"rk4": 2, "euler": 1, "ie": 3, "im": 4}[a.solver]
    kw = dict(neq=6, npar=6, dt=a.dt, ksteps=a.ksteps, nchunks=a.nsteps // a.ksteps, nthreads=cores)
    if kind_pref == "reference" and ReferenceBuild.available("oculomotor", solver):
        impl, kind = ReferenceBuild("oculomotor", solver), "reference"
        fn = lambda: impl.run(t0, y0, p, **kw)  # noqa: E731
    else:
        impl, kind = Oracle("oculomotor"), "port"
        fn = lambda: impl.run(solver, t0, y0, p, **kw)  # noqa: E731
    t = time.perf_counter()
    res = fn()
    secs = time.perf_counter() - t
    return n * a.nsteps / secs, secs, kind, res.records


def parity_floor(n, a, cores, cpu_records):
    """The same measure between two CPU builds of the same computation on the
    same orbits: the CPU baseline's records against the oracle compiled with
    FMA contraction.  At an unstable step the orbits that stay finite still
    amplify last-bit differences, and this is how far they carry them."""
    from oracle.oracle import Oracle

    t0, y0, p = workload(n, 0)
    solver = {"rk4": 2, "euler": 1, "ie": 3, "im": 4}[a.solver]
    fma = Oracle("oculomotor", "fp64fma").run(solver, t0, y0, p, neq=6, npar=6, dt=a.dt, ksteps=a.ksteps,
                                              nchunks=a.nsteps // a.ksteps, nthreads=cores).records
    out = records_error(fma, cpu_records)
    out["vs"] = "the oracle compiled with FMA contraction against the CPU baseline"
    return out


def records_error(got, want):
    """The GPU's records ([record][equation][orbit]) against the CPU
    implementation's on the same orbits.  Over the orbits whose records are
    all finite in both: per element |got - want| / (|want| + 1e-3 S_e), S_e
    the largest |value| of equation e among them.  An orbit that diverges
    (the configuration's step is unstable for most parameter draws) carries
    last-bit differences through its growth, so its records are not compared;
    counted instead: orbits that diverge in both, and orbits that diverge in
    one run only."""
    fin_w = np.isfinite(want).all(axis=(0, 1))
    fin_g = np.isfinite(got).all(axis=(0, 1))
    both = fin_w & fin_g
    out = {"orbits": int(both.size), "orbits_finite_in_both": int(both.sum()),
           "orbits_diverging_in_both": int((~fin_w & ~fin_g).sum()),
           "orbits_diverging_in_one": int((fin_w != fin_g).sum())}
    if both.any():
        w, g = want[:, :, both], got[:, :, both]
        scale = np.max(np.abs(w), axis=(0, 2), keepdims=True)
        e = (np.abs(g - w) / (np.abs(w) + 1e-3 * scale + 1e-300)).ravel()
        out.update({"max_rel_err": float(e.max()), "p99_rel_err": float(np.quantile(e, 0.99)),
                    "median_rel_err": float(np.median(e))})
    return out


def run_reference_arm(a, rank):
    """The reference's kernels compiled as C (oracle/_ref), OpenMP over all
    host cores, on the same sample as the cpu_baseline leg: each step
    integrates the first a.cpu_orbits orbits through all a.nsteps steps.
    ms_per_step is that sample's measured time; value is its orbit-steps/s.
    Imports nothing that maps this library's native code."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    n = min(a.cpu_orbits, a.orbits)
    for _ in range(a.warmup):
        cpu_reference_rate(256, a, cores)
    secs = []
    kind = None
    for _ in range(a.steps):
        _, sec, kind, _ = cpu_reference_rate(n, a, cores)
        secs.append(sec)
    ms = float(np.mean(secs)) * 1e3
    value = n * a.nsteps / (ms * 1e-3)
    sample = "the first %d of %d orbits, all %d steps, records every %d, per step (warm-up steps: 256 orbits)" % (
        n, a.orbits, a.nsteps, a.ksteps)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": config_dict(a, a.orbits),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference_arm(a, rank)
        return

    import torch

    import sodecl_b200
    from sodecl_b200 import Integrator, system_path

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    from sodecl_b200.sharding import max_over_ranks, shard

    # weak scaling: every rank integrates a.orbits orbits of a world x a.orbits job
    offset, n = shard(a.orbits * world, rank, world)
    t0, y0, p = workload(n, offset)
    tspan = a.nsteps * a.dt
    system_file, _ = headline_system()
    sim = Integrator(system_file, a.solver, dt=a.dt, tspan=tspan, ksteps=a.ksteps, neq=6, npar=6,
                     orbits=n, device=local_rank, precision=a.precision, block=a.block)
    nchunks = sim.num_chunks
    assert nchunks * a.ksteps == a.nsteps, (nchunks, a.ksteps, a.nsteps)
    tuned = None
    if not a.no_tune:
        # launch shape and division mode picked on copies of every orbit over
        # 1000 steps (results are identical for every choice).  All the orbits,
        # because register caps trade resident warps against spills and only
        # a launch of many waves shows which wins (with 2^17 orbits, 64
        # registers looked best and 85 is 3 % faster at 2^20); a thousand steps,
        # because by then most orbits have diverged, as over most of the run.
        # Outside the timing.
        sim.upload(t0, y0, p)
        tuned = sim.autotune(sample_orbits=n, sample_steps=1000)
    nrec = nchunks + 1
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    t0_d = torch.tensor(t0, device=dev)
    y0_d = torch.tensor(y0, device=dev)
    p_d = torch.tensor(p, device=dev)
    t_d, y_d = t0_d.clone(), y0_d.clone()
    rec_d = torch.empty((nrec, 6, n), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def one_launch():
        sim.launch(t=t_d.data_ptr(), y=y_d.data_ptr(), params=p_d.data_ptr(), records=rec_d.data_ptr(), n=n,
                   orbit_offset=offset, rec_stride=n, chunk_begin=0, chunk_end=nchunks, write_final=True,
                   stream=stream.cuda_stream)

    # ---------------- device-resident timing
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    for _ in range(a.warmup):
        t_d.copy_(t0_d)
        y_d.copy_(y0_d)
        one_launch()
    barrier()
    with ClockSampler(local_rank) as clocks:
        barrier()
        wall0 = time.perf_counter()
        for i in range(a.steps):
            t_d.copy_(t0_d)
            y_d.copy_(y0_d)
            flush.zero_()
            starts[i].record(stream)
            one_launch()
            ends[i].record(stream)
        barrier()
        wall = time.perf_counter() - wall0
    launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = float(np.mean(launch_ms))
    ms = max_over_ranks(ms, dist, dev)
    rec_last = rec_d[-1].cpu().numpy()
    # the records of the orbits the CPU baseline integrates, checked against it below
    rec_sample = rec_d[:, :, :min(a.cpu_orbits, n)].cpu().numpy() if rank == 0 and world == 1 else None
    nan_fraction = float(np.mean(~np.isfinite(rec_last).all(axis=0)))
    value = world * n * a.nsteps / (ms * 1e-3)

    # ---------------- roofline: counted FP64 ops vs measured FMA issue peak
    peaks = {prec: 2.0 * sodecl_b200.fma_peak(prec, device=local_rank)[0] / 1e12 for prec in ("fp64", "fp32")}
    peak_tflops = peaks[a.precision]
    achieved = RK4_OPS_PER_ORBIT_STEP * n * a.nsteps / (ms * 1e-3) / 1e12 if a.solver == "rk4" else None
    # DRAM bytes per launch: ncu's dram__bytes_read.sum + dram__bytes_write.sum
    # on a 2^18-orbit x 1000-step launch of the same kernel on the same system
    # file with the default 85-register cap (129.2 MB, 11 records), scaled by
    # orbits x records, which the traffic follows (it is the record stream)
    traffic = 129.2e6 * (n * nrec) / (262144 * 11) if (a.solver == "rk4" and a.precision == "fp64") else None
    algorithmic_bytes = nrec * 6 * n * 8 + n * (104 + 56)
    hbm_gbs = algorithmic_bytes / (ms * 1e-3) / 1e9
    hbm_peak = None
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            hbm_peak = float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        pass
    roofline = {"bound": "fp64" if a.precision == "fp64" else "fp32", "achieved": achieved, "peak": peak_tflops,
                "unit": "TFLOP/s", "frac": (achieved / peak_tflops) if achieved else None, "traffic": traffic,
                "algorithmic_bytes": algorithmic_bytes, "hbm_gbs": hbm_gbs,
                "hbm_frac_of_measured": (hbm_gbs / hbm_peak) if hbm_peak else None,
                "peak_source": "measured on this GPU: FMA-chain microbenchmark (sodecl_cuda_fma_peak, fastest of "
                               "7 launches), 2 flops/FMA",
                "ops_per_orbit_step": RK4_OPS_PER_ORBIT_STEP,
                "fp64_pipe_active": "52.4 % of peak (ncu sm__pipe_fp64_cycles_active, 2^18-orbit x 1000-step "
                                    "launch of this kernel on this system file, dt 1e-3); counted source ops "
                                    "understate the pipe work, exp and division expanding to many FP64 "
                                    "instructions each"}

    # ---------------- end to end through the C ABI with host buffers
    e2e = None
    h2d = (t0.nbytes + y0.nbytes + p.nbytes)
    d2h = nrec * 6 * n * 8
    if not a.no_e2e:
        del rec_d
        torch.cuda.empty_cache()
        host_t = torch.from_numpy(t0).pin_memory()
        host_y = torch.from_numpy(y0).pin_memory()
        host_p = torch.from_numpy(p).pin_memory()
        host_out = torch.empty((nrec, 6, n), dtype=torch.float64, pin_memory=True)
        from sodecl_b200 import _native as N

        def e2e_step():
            N.check(N.lib.sodecl_cuda_upload(sim.ctx, host_t.data_ptr(), host_y.data_ptr(), host_p.data_ptr(), None),
                    sim.ctx)
            sim.run_into(host_out.data_ptr(), host_out.numel())

        for _ in range(max(1, a.warmup)):
            e2e_step()
        barrier()
        w0 = time.perf_counter()
        for _ in range(a.steps):
            e2e_step()
        barrier()
        e2e_s = (time.perf_counter() - w0) / a.steps
        e2e_s = max_over_ranks(e2e_s, dist, dev)
        e2e = {"value": world * n * a.nsteps / e2e_s, "unit": METRIC, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3, "path": "sodecl_cuda_upload + sodecl_cuda_run, "
               "pinned host buffers"}
        assert np.array_equal(host_out[-1].numpy(), rec_last, equal_nan=True)

    # ---------------- the drop-in path end to end (single-GPU runs)
    e2e_dropin = None
    if not a.no_e2e and world == 1:
        with stdout_to_stderr():
            e2e_dropin = dropin_e2e(a, n, t0, y0, p, rec_last)

    # ---------------- companions: stable step, fp32, implicit midpoint
    extras = {}
    # companions on single-GPU runs only: under torchrun they would hold every
    # rank's GPU while rank 0 alone works
    if not a.no_extras and world == 1:
        def line(name, fn):
            # a companion line only: an error takes its place, the headline stands
            try:
                extras[name] = fn()
            except Exception as exc:
                extras[name] = {"error": "%s: %s" % (type(exc).__name__, exc)}
                try:
                    torch.cuda.synchronize()
                    torch.cuda.empty_cache()
                except Exception:
                    pass

        line("companions", lambda: companions(a, n, dev, stream, peaks)["companions"])
        # the ceiling of right-hand sides made of sines (the Kuramoto lines)
        sin_peaks = {}
        line("sin_peak", lambda: sin_peaks.update({prec: sodecl_b200.sin_peak(prec, device=local_rank)[0]
                                                   for prec in ("fp64", "fp32")}) or dict(sin_peaks))
        line("gradient", lambda: gradient_companion(dev))
        line("gradient_implicit_midpoint", lambda: gradient_implicit_companion(dev))
        line("uneven_batch", lambda: batch_companion(dev, sin_peaks))
        line("uneven_batch_full", lambda: batch_full_companion(sin_peaks))
        line("stochastic_kuramoto", lambda: stochastic_kuramoto_companion(dev, stream, sin_peaks))
        line("small_kuramoto", lambda: small_kuramoto_companion(dev, stream, sin_peaks))
        line("readme_case", readme_case_companion)
        line("adaptive", lambda: adaptive_companion(a, n, dev, stream))

    cpu = parity = None
    if rank == 0 and world == 1:
        cores = os.cpu_count() or 1
        v, secs, kind, cpu_records = cpu_reference_rate(min(a.cpu_orbits, n), a, cores)
        try:
            parity = records_error(rec_sample, cpu_records)
            parity["floor"] = parity_floor(min(a.cpu_orbits, n), a, cores, cpu_records)
            if "max_rel_err" in parity and "max_rel_err" in parity["floor"]:
                parity["within_10x_floor"] = bool(parity["max_rel_err"] <= max(1e-12, 10 * parity["floor"]["max_rel_err"]))
        except Exception as exc:  # a check beside the measurement: the line stands without it
            parity = {"error": "%s: %s" % (type(exc).__name__, exc)}
        parity.update({"vs": "the CPU baseline's records (%s) of the same %d orbits, all %d records"
                             % ("the reference's kernels compiled as C" if kind == "reference" else "the oracle",
                                rec_sample.shape[2], rec_sample.shape[0]),
                       "fmad": "GPU with FMA contraction (the library's default), CPU without"})
        cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
               "sample": "%d of %d orbits, all %d steps, records every %d (%.1f s)" % (min(a.cpu_orbits, n), n,
                                                                                     a.nsteps, a.ksteps, secs)}
    info = sim.kernel_info()
    if rank == 0:
        launch_info = {"parallelism": "orbits sharded, %d per GPU" % n, "block": sim.cfg.local_group_size or 128,
                       "min_blocks_per_sm": sim.cfg.min_blocks_per_sm, "division": sim.division,
                       "record_store": "pairs" if sim.cfg.record_store == 1 else "direct",
                       "autotuned": tuned is not None, "registers": info["registers"],
                       "local_bytes": info["local_bytes"], "nan_fraction_final": nan_fraction}
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32", "data": "synthetic",
               "config": config_dict(a, n), "launch": launch_info, "roofline": roofline, "cpu_baseline": cpu,
               "parity": parity,
               "e2e": e2e, "e2e_dropin": e2e_dropin, "gpu_launches": a.steps, "clocks": clocks.summary(), "wall_s_timed_region": wall,
               "launch_ms": launch_ms}
        out.update(extras)
        print(json.dumps(out), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


def dropin_e2e(a, n, t0, y0, p, rec_last, reps=5):
    """The headline through the reference's Python entry point on this
    library, sodecl_b200.sodecl.sodecl(platform, device, system file, initx,
    params, solver, orbits, nequat, nnoise, dt, tspan, ksteps, local size):
    per call a new manager (program from the on-disk cache), upload from
    pageable numpy arrays, the run, and the records in a new pageable numpy
    array -- as a user of the reference calls it, with its default launch
    shape (local size 0, no tuning).  Wall clock per call, median of `reps`
    after one untimed call; the previous call's result array is released
    outside the timed region."""
    import contextlib
    import io

    from sodecl_b200.sodecl import sodecl

    system_file, _ = headline_system()
    solver = {"euler": 1, "rk4": 2, "ie": 3, "im": 4}[a.solver]
    tspan = a.nsteps * a.dt

    def call():
        with contextlib.redirect_stdout(io.StringIO()):  # the manager prints its runtime line
            return sodecl(0, 0, system_file, y0, p, solver, n, 6, 0, a.dt, tspan, a.ksteps, 0,
                          precision=0 if a.precision == "fp64" else 1)

    _, res = call()
    secs = []
    for _ in range(reps):
        w0 = time.perf_counter()
        out = call()
        secs.append(time.perf_counter() - w0)
        # the previous call's records (5 GB of numpy) are released after the
        # clock stops: dropping them is the caller's business, not the call's
        res = out[1]
        del out
    # the last record of the drop-in run equals the device-resident run's
    same = bool(np.array_equal(res[:, -1].reshape(6, n), rec_last, equal_nan=True))
    s = float(np.median(secs))
    return {"value": n * a.nsteps / s, "unit": METRIC, "ms_per_step": s * 1e3, "ms_all": [x * 1e3 for x in secs],
            "h2d_bytes_per_step": int(t0.nbytes + y0.nbytes + p.nbytes), "d2h_bytes_per_step": int(res.nbytes),
            "records_equal_to_device_run": same,
            "path": "sodecl_b200.sodecl.sodecl -> sodecl_interface.sodeclcall_array -> sodecl::sodeclmgr -> "
                    "C ABI; pageable numpy in and out; default launch shape"}


def gradient_companion(dev, n=1 << 16, nsteps=5000, ksteps=100, dt=1e-5):
    """Gradient fitting: oculomotor RK4, 2^16 orbits, 5000 steps, records every
    100; MSE against targets from seeded true parameters + N(0, 1e-2) noise.
    Times the discrete adjoint (loss + d/d(params, y0)) against central finite
    differences of the same loss (2 x 12 perturbed copies of every orbit in one
    launch) on the same GPU, and reports their relative disagreement.  dt 1e-5:
    at the configuration's 1e-3 RK4 diverges for this model and the gradients
    are NaN."""
    import torch

    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint, finite_difference_gradient

    from sodecl_b200.workloads import fitting_targets

    _, y0, guess, targets = fitting_targets(n, nsteps, ksteps, dt, device=dev)
    kw = dict(dt=dt, tspan=(nsteps - 0.5) * dt, ksteps=ksteps, neq=6, npar=6)
    sim = Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw)
    assert sim.num_chunks * ksteps == nsteps
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    # the library's default schedule: the forward sweep records the whole
    # trajectory (n x nsteps x 25 doubles, 65.5 GB here) when it fits in half
    # the free memory; the same context then serves the other schedules
    adj = Adjoint(sim)
    sqrt_every = int(np.ceil(np.sqrt(nsteps)))
    adj_sqrt = Adjoint(sim, ckpt_every=sqrt_every)
    adj_tape = Adjoint(sim, use_tape=True, ckpt_every=nsteps)
    # the same file without calc_vjp: products from calc_jacobian + calc_jacobian_params
    src = open(system_path("oculomotor")).read().replace("void calc_vjp(", "void unused_calc_vjp(")
    sim_jac = Integrator(None, "rk4", orbits=n, system_src=src, **kw)
    adj_jac = Adjoint(sim_jac, ckpt_every=nsteps)
    wide = Adjoint(Integrator(system_path("oculomotor"), "rk4", orbits=n * 24, **kw))
    t0, y0d, gd = T(np.zeros(n)), T(y0), T(guess)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            r = fn()
            e.record()
            torch.cuda.synchronize()
            out.append(s.elapsed_time(e))
        return float(np.median(out)), r

    whole_gb = 8.0 * n * (nsteps * 25 + 7) / 1e9
    whole = whole_gb * 1e9 <= 0.5 * torch.cuda.mem_get_info(dev)[0]  # the library's test, before its first call
    ms_adj, (loss, gp, gy, flags) = timed(lambda: adj(t0, y0d, gd, targets))
    ms_sqrt, (loss_s, gp_s, gy_s, _) = timed(lambda: adj_sqrt(t0, y0d, gd, targets))
    sqrt_identical = bool(torch.equal(loss_s, loss) and torch.equal(gp_s, gp) and torch.equal(gy_s, gy))
    ms_jac, (_, gpj, _, _) = timed(lambda: adj_jac(t0, y0d, gd, targets))
    sim_jac.close()
    ms_tape, (_, gpt, gyt, _) = timed(lambda: adj_tape(t0, y0d, gd, targets), reps=1)
    ms_fd, (fp, fy) = timed(lambda: finite_difference_gradient(t0, y0d, gd, targets, wide))
    ms_fwd, _ = timed(lambda: adj(t0, y0d, gd, targets, with_gradient=False))
    # per-orbit relative differences; the model's burst non-linearity has a kink
    # at y5 = 0, so the central differences of the few orbits whose stage
    # evaluations pass within the step of it are off: report quantiles
    dp = ((gp - fp).abs().amax(1) / gp.abs().amax(1)).cpu().numpy()
    dy = ((gy - fy).abs().amax(1) / gy.abs().amax(1)).cpu().numpy()
    err_tape = ((gpt - gp).abs().amax(1) / gp.abs().amax(1)).max().item()
    err_jac = ((gpj - gp).abs().amax(1) / gp.abs().amax(1)).max().item()
    q = lambda d: {"median": float(np.median(d)), "p99": float(np.quantile(d, 0.99)),  # noqa: E731
                   "max": float(d.max()), "orbits_above_1e-4": int((d > 1e-4).sum())}
    return {"orbits": n, "nsteps": nsteps, "record_every": ksteps, "dt": dt, "adjoint_ms": ms_adj,
            "division": "IEEE in the gradient pass, reciprocal in loss-only passes (finite differences, loss_only)",
            "adjoint_jacobians_ms": ms_jac, "adjoint_tape_ms": ms_tape,
            "rel_diff_jacobians_vs_vjp": err_jac, "rel_diff_tape_vs_vjp": err_tape,
            "finite_difference_ms": ms_fd, "loss_only_ms": ms_fwd, "speedup_vs_fd": ms_fd / ms_adj,
            "schedule": ("forward sweep records the whole trajectory (%.1f GB), no recomputation" % whole_gb
                         if whole else "checkpoints every %d steps (the whole trajectory did not fit)" % sqrt_every),
            "adjoint_sqrt_checkpoints_ms": ms_sqrt, "sqrt_checkpoint_every": sqrt_every,
            "speedup_vs_fd_sqrt_checkpoints": ms_fd / ms_sqrt, "sqrt_checkpoints_identical": sqrt_identical,
            "rel_diff_vs_fd_params": q(dp), "rel_diff_vs_fd_y0": q(dy),
            "tape_overflow": int((flags != 0).sum().item()),
            "fd": "central, relative step 1e-6, 24 perturbed copies per orbit in one launch",
            "derivatives": "adjoint_ms: the system file's calc_vjp; adjoint_jacobians_ms: its calc_jacobian + "
                           "calc_jacobian_params; adjoint_tape_ms: reverse mode over sode_system"}


def gradient_implicit_companion(dev, n=1 << 16, nsteps=1000, ksteps=100, dt=1e-3, newton_tol=1e-10):
    """The same fit with implicit midpoint steps (dt 1e-3, where the model is
    stable under it): the discrete adjoint of the implicit step taken as
    solved exactly (one transposed solve with the full Jacobian per step)
    against central finite differences (24 perturbed copies in one loss-only
    launch).  Newton tolerance 1e-10 (the pass limit the reference's 1000), so
    that the converged steps the differences see are close to the exact steps
    the adjoint differentiates; orbits with a step stopped at the pass limit
    are counted and left out of the comparison (their steps are not the
    solved ones)."""
    import torch

    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint, finite_difference_gradient

    from sodecl_b200.workloads import fitting_targets

    _, y0, guess, targets = fitting_targets(n, nsteps, ksteps, dt, device=dev, solver="im", newton_tol=newton_tol)
    kw = dict(dt=dt, tspan=(nsteps - 0.5) * dt, ksteps=ksteps, neq=6, npar=6, newton_tol=newton_tol)
    sim = Integrator(system_path("oculomotor"), "im", orbits=n, **kw)
    wide_sim = Integrator(system_path("oculomotor"), "im", orbits=n * 24, **kw)
    adj, wide = Adjoint(sim), Adjoint(wide_sim)
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    t0, y0d, gd = T(np.zeros(n)), T(y0), T(guess)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            r = fn()
            e.record()
            torch.cuda.synchronize()
            out.append(s.elapsed_time(e))
        return float(np.median(out)), r

    ms_adj, (loss, gp, gy, flags) = timed(lambda: adj(t0, y0d, gd, targets))
    ms_fd, (fp, fy) = timed(lambda: finite_difference_gradient(t0, y0d, gd, targets, wide))
    ok = (flags == 0).cpu().numpy()
    dp = ((gp - fp).abs().amax(1) / gp.abs().amax(1)).cpu().numpy()[ok]
    dy = ((gy - fy).abs().amax(1) / gy.abs().amax(1)).cpu().numpy()[ok]
    q = lambda d: {"median": float(np.median(d)), "p99": float(np.quantile(d, 0.99)),  # noqa: E731
                   "max": float(d.max())}
    sim.close()
    wide_sim.close()
    return {"solver": "im", "orbits": n, "nsteps": nsteps, "record_every": ksteps, "dt": dt,
            "newton_tol": newton_tol, "adjoint_ms": ms_adj, "finite_difference_ms": ms_fd,
            "speedup_vs_fd": ms_fd / ms_adj, "rel_diff_vs_fd_params": q(dp), "rel_diff_vs_fd_y0": q(dy),
            "orbits_flagged": int((~ok).sum()), "compared": "orbits with every step converged",
            "fd": "central, relative step 1e-6, 24 perturbed copies per orbit in one launch"}


def tuning_steps(steps, scale=64):
    """Step counts for the batch tuner's trials: every orbit, each with its
    step count divided by `scale` (at least one).  Scaling the steps and not
    the orbits keeps the ratio of the longest orbit's time (the launch's
    critical path) to the total work's time (throughput) that the real launch
    has; each trial then takes about 1/scale of the launch."""
    return np.maximum(1, steps // scale)


def sine_roofline(sines, seconds, peak, basis):
    """Roofline block of a Kuramoto line: sine evaluations per second against
    the measured throughput of the math library's sin (sodecl_cuda_sin_peak,
    fastest of 7 launches at full occupancy)."""
    achieved = sines / seconds
    return {"bound": "sin", "achieved": achieved, "peak": peak, "unit": "sines/s", "frac": achieved / peak,
            "sines": basis, "peak_source": "measured on this GPU: sodecl_cuda_sin_peak (eight independent sums of "
                                           "sin(x_k - y) per thread, fastest of 7 launches)"}


def kuramoto_sines(classes, cls, steps, passes):
    """Sine evaluations of an uneven sweep's Kuramoto orbits: N^2 per
    right-hand side (Euler one per step, RK4 four), and N^2 per Newton pass of
    implicit Euler (a pass evaluates every row's N terms; where it also takes
    the band from the same sincos, or the Jacobian's cosines, those are not
    counted: a lower bound).  The oculomotor orbits evaluate no sine."""
    total = 0
    for k, (system, solver, neq, npar, dt) in enumerate(classes):
        if system != "kuramoto":
            continue
        m = cls == k
        per = {"euler": int(steps[m].sum()), "rk4": 4 * int(steps[m].sum()), "ie": int(passes[m].sum())}[solver]
        total += per * neq * neq
    return total


SINE_BASIS_BATCH = ("Kuramoto orbits only: N^2 sines per right-hand side (Euler 1, RK4 4 per step) and per implicit "
                    "Euler Newton pass (sincos counted once, cosines of the Jacobian not counted); oculomotor work "
                    "not counted: a lower bound")


def batch_companion(dev, sin_peaks, n=1 << 15, max_steps=10000, seed=4):
    """The uneven-sweep shape: orbits mixing Kuramoto N in {4, 16, 64} and the
    oculomotor model, solver per orbit in {Euler, RK4, implicit Euler}, step
    counts log-uniform in [10^2, max_steps], FP64.  The full configuration is
    2^18 orbits and steps up to 10^5; this sample (2^15 orbits, up to 10^4
    steps) keeps the default run short.  Wide classes run lanes per orbit (the
    tuner's choice per class), in the batch and in the padded launches alike.
    One persistent launch from device work queues (autotuned launch shape,
    graph replay), against the padded alternative: one launch per class
    through the single-system kernel, every orbit of a class run for that
    class's longest step count.  Tuned as the full-size line below."""
    import torch

    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.batch import Batch

    from sodecl_b200.workloads import uneven_batch

    classes, cls, steps, y0, p, rng = uneven_batch(n, max_steps, seed)
    b = Batch()
    for system, solver, neq, npar, dt in classes:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, dt=dt)
    b.compile()
    b.set_items(cls, tuning_steps(steps), np.zeros(n), y0, p)
    block, bps, _ = b.tune()
    b.set_items(cls, steps, np.zeros(n), y0, p)
    b.run(graph=True)  # capture
    times = []
    for _ in range(2):
        b.set_items(cls, steps, np.zeros(n), y0, p)
        b.set_launch(block, bps)
        times.append(b.run(graph=True))
    batch_ms = float(np.median(times))
    useful = int(steps.sum())
    _, _, _, passes, _ = b.results()
    sines = kuramoto_sines(classes, cls, steps, passes)
    # padded: per class, every orbit runs the class's longest orbit, with the
    # lanes per orbit the tuner chose for the class
    tuned_lanes = b.lanes
    padded_ms = 0.0
    stream = torch.cuda.current_stream(dev)
    for k, (system, solver, neq, npar, dt) in enumerate(classes):
        idx = np.nonzero(cls == k)[0]
        if idx.size == 0:
            continue
        m = int(steps[idx].max())
        sim = Integrator(system_path(system), solver, dt=dt, tspan=(m - 0.5) * dt, ksteps=m, neq=neq, npar=npar,
                         orbits=idx.size, lanes=tuned_lanes[k])
        td = torch.zeros(idx.size, dtype=torch.float64, device=dev)
        yd = torch.tensor(np.stack([y0[i] for i in idx]), device=dev)
        pd = torch.tensor(np.stack([p[i] for i in idx]), device=dev)
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record(stream)
        sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), stream=stream.cuda_stream)
        e_.record(stream)
        torch.cuda.synchronize()
        padded_ms += s_.elapsed_time(e_)
        sim.close()
    return {"orbits": n, "classes": len(classes), "steps": "log-uniform [100, %d]" % max_steps,
            "orbit_steps": useful, "batch_ms": batch_ms, "value": useful / (batch_ms * 1e-3), "unit": METRIC,
            "tuned_launch": {"block": block, "blocks_per_sm": bps}, "padded_per_class_ms": padded_ms,
            "speedup_vs_padded": padded_ms / batch_ms, "registers": b.kernel_info()["registers"],
            "lanes_per_class": b.lanes,
            "roofline": sine_roofline(sines, batch_ms * 1e-3, sin_peaks["fp64"], SINE_BASIS_BATCH)}


def batch_full_companion(sin_peaks, n=1 << 18, max_steps=100000, seed=4):
    """The uneven sweep at its configured size: 2^18 orbits, step counts
    log-uniform in [10^2, 10^5] (3.8e9 orbit-steps), the same 12 classes, in
    one persistent launch (CUDA graph), after the tuner has chosen lanes per
    class, the register cap and the launch shape on every orbit with its step
    count divided by 64 (tuning_steps).  One timed launch (it takes about a
    minute; the padded comparison runs on the smaller sample above)."""
    from sodecl_b200 import system_path
    from sodecl_b200.batch import Batch
    from sodecl_b200.workloads import uneven_batch

    classes, cls, steps, y0, p, rng = uneven_batch(n, max_steps, seed)
    b = Batch()
    for system, solver, neq, npar, dt in classes:
        b.add_class(system_path(system), solver, neq=neq, npar=npar, dt=dt)
    b.compile()
    b.set_items(cls, tuning_steps(steps), np.zeros(n), y0, p)
    block, bps, _ = b.tune()
    b.set_items(cls, steps, np.zeros(n), y0, p)
    b.set_launch(block, bps)
    ms = b.run(graph=True)
    _, _, _, passes, flags = b.results()
    useful = int(steps.sum())
    sines = kuramoto_sines(classes, cls, steps, passes)
    return {"orbits": n, "classes": len(classes), "steps": "log-uniform [100, %d]" % max_steps,
            "orbit_steps": useful, "batch_ms": ms, "value": useful / (ms * 1e-3), "unit": METRIC,
            "tuned_launch": {"block": block, "blocks_per_sm": bps}, "lanes_per_class": b.lanes,
            "registers": b.kernel_info()["registers"], "orbits_flagged": int((flags != 0).sum()),
            "launches_timed": 1, "roofline": sine_roofline(sines, ms * 1e-3, sin_peaks["fp64"], SINE_BASIS_BATCH)}


def stochastic_kuramoto_companion(dev, stream, sin_peaks, n=1 << 18, N=32, nsteps=2000, ksteps=200, seed=3):
    """Stochastic Kuramoto by Euler-Maruyama: N=32 phases, 2^18 orbits,
    K ~ U(0,5), omega ~ N(0,1) shared, additive noise sigma ~ U(0,0.5) per
    orbit, counters orbit * 2^20, dt=0.01, a record every 200 steps, FP64 (and
    FP32).  2000 of the full configuration's 2x10^4 steps keep the default run
    short (the rate does not depend on the step count).  One thread per orbit
    against the tuned launch (lanes per orbit for this 32-equation system),
    and the reference's own examples/kuramoto.cl (same arithmetic; without
    the per-row functions lanes per orbit need, so one thread per orbit,
    tuned).  Each line carries its roofline against the measured sine
    throughput of its precision."""
    import torch

    from sodecl_b200 import Integrator, system_path

    from sodecl_b200.workloads import kuramoto

    _, th0, p, cnt = kuramoto(n, N, seed=seed, noise=True)
    out = {}
    cases = [("one_thread_per_orbit_fp64", system_path("kuramoto"), "fp64", False),
             ("tuned_fp64", system_path("kuramoto"), "fp64", True),
             ("tuned_fp32", system_path("kuramoto"), "fp32", True)]
    if os.path.isfile(REFERENCE_KURAMOTO):
        cases.append(("reference_file_tuned_fp64", REFERENCE_KURAMOTO, "fp64", True))
    for name, path, prec, tune in cases:
        sim = Integrator(path, "se", dt=0.01, tspan=nsteps * 0.01, ksteps=ksteps, neq=N,
                         npar=2 * N + 1, nnoi=N, orbits=n, precision=prec)
        choice = None
        if tune:
            sim.upload(np.zeros(n), th0, p, cnt)
            # trials on every orbit: with one thread per orbit a register cap
            # pays only when the launch has many waves, which a sample of
            # 2^15 orbits (a fraction of one wave) does not show
            choice = sim.autotune(sample_orbits=n, sample_steps=50)
        td, yd, pd, cd = [torch.tensor(x, device=dev) for x in (np.zeros(n), th0, p, cnt)]
        rec = torch.empty((sim.num_records, N, n), dtype=torch.float64, device=dev)
        ms = []
        for it in range(3):
            td.zero_()
            yd.copy_(torch.tensor(th0, device=dev))
            cd.copy_(torch.tensor(cnt, device=dev))
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), counters=cd.data_ptr(),
                       records=rec.data_ptr(), stream=stream.cuda_stream)
            e_.record(stream)
            torch.cuda.synchronize()
            if it > 0:
                ms.append(s_.elapsed_time(e_))
        info = sim.kernel_info()
        out[name] = {"value": n * nsteps / (np.mean(ms) * 1e-3), "unit": METRIC, "ms": float(np.mean(ms)),
                     "precision": prec, "launch": choice or {"lanes": 1, "block": 128},
                     "registers": info["registers"], "local_bytes": info["local_bytes"],
                     "roofline": sine_roofline(n * nsteps * N * N, np.mean(ms) * 1e-3, sin_peaks[prec],
                                               "N^2 = %d sines per orbit-step (one right-hand side); the noise's "
                                               "Threefry words, logarithms and square roots not counted" % (N * N))}
        sim.close()
        del rec
        torch.cuda.empty_cache()
    out["config"] = {"orbits": n, "N": N, "nsteps": nsteps, "full_nsteps": 20000, "dt": 0.01, "record_every": ksteps}
    return out


# Counted source-level operations per Newton pass of the implicit midpoint on
# the reference's oculomotor file (tests/test_opcount.py): the pass that
# meets the stop test, and a full pass (Jacobian, scaling, banded solve)
IM_OPS_CONVERGED_PASS, IM_OPS_FULL_PASS = 78, 236


def companions(a, n, dev, stream, peaks):
    """Same shape, other settings: the stable step dt=1e-5 (RK4 diverges at
    1e-3 for most parameter draws), FP32, implicit midpoint -- with the
    reference's Newton settings (1e-7, up to 1000 passes) and with the stated
    1e-10 / 10 passes, which the reference's banded solve does not converge
    within (the orbits that hit the limit are counted) -- all on the
    headline's system file; and the headline itself on the package's restated
    system file (sodecl_b200/systems/oculomotor.cl: the same trajectories,
    with the burst's exp argument selected instead of branched).  Each line
    carries its counted-operation roofline against the measured FMA peak of
    its precision."""
    import torch

    from sodecl_b200 import Integrator

    out = {}
    t0, y0, p = workload(n, 0)
    system_file, _ = headline_system()
    # (name, system file, solver, dt, precision, Newton tolerance, Newton pass limit)
    cases = [("stable_dt_1e-5", system_file, a.solver, 1e-5, a.precision, 1e-7, 1000),
             ("fp32", system_file, a.solver, a.dt, "fp32", 1e-7, 1000),
             ("fp32_stable_dt_1e-5", system_file, a.solver, 1e-5, "fp32", 1e-7, 1000),
             ("package_system_file", PACKAGE_SYSTEM, a.solver, a.dt, a.precision, 1e-7, 1000),
             ("package_system_file_stable_dt_1e-5", PACKAGE_SYSTEM, a.solver, 1e-5, a.precision, 1e-7, 1000),
             ("implicit_midpoint", system_file, "im", a.dt, "fp64", 1e-7, 1000),
             ("implicit_midpoint_tol1e-10_max10", system_file, "im", a.dt, "fp64", 1e-10, 10),
             ("implicit_midpoint_fp32_tol1e-10_max10", system_file, "im", a.dt, "fp32", 1e-10, 10)]
    for name, path, solver, dt, prec, tol, maxit in cases:
        sim = Integrator(path, solver, dt=dt, tspan=a.nsteps * dt, ksteps=a.ksteps, neq=6,
                         npar=6, orbits=n, precision=prec, newton_tol=tol, newton_max_iter=maxit)
        nrec = sim.num_records
        td, yd, pd = torch.tensor(t0, device=dev), torch.tensor(y0, device=dev), torch.tensor(p, device=dev)
        tuned = None
        if solver == a.solver:
            # tuned like the headline (launch shape and division mode)
            sim.upload(t0, y0, p)
            tuned = sim.autotune(sample_orbits=n, sample_steps=1000)
        rec = torch.empty((nrec, 6, n), dtype=torch.float64, device=dev)
        passes = torch.zeros(n, dtype=torch.int64, device=dev)
        flags = torch.zeros(n, dtype=torch.int32, device=dev)
        ms = []
        for it in range(3):
            td.copy_(torch.tensor(t0, device=dev))
            yd.copy_(torch.tensor(y0, device=dev))
            passes.zero_()
            flags.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=rec.data_ptr(), n=n,
                       chunk_begin=0, chunk_end=sim.num_chunks, newton_passes=passes.data_ptr(),
                       flags=flags.data_ptr(), stream=stream.cuda_stream)
            e.record(stream)
            torch.cuda.synchronize()
            if it > 0:
                ms.append(s.elapsed_time(e))
        last = rec[-1].cpu().numpy()
        t_s = float(np.mean(ms)) * 1e-3
        entry = {"value": n * a.nsteps / t_s, "unit": METRIC, "dt": dt, "precision": prec, "solver": solver,
                 "system_file": os.path.relpath(path, REPO), "ms": t_s * 1e3,
                 "nan_fraction_final": float(np.mean(~np.isfinite(last).all(axis=0)))}
        if tuned:
            entry["launch"] = tuned
        if solver == "im":
            total_passes = float(passes.double().sum().item())
            steps = float(n) * a.nsteps
            entry["newton_passes_per_step"] = total_passes / steps
            entry["newton"] = {"tol": tol, "max_passes": maxit,
                               "orbits_at_pass_limit": float((flags & 1).bool().double().mean().item())}
            ops = IM_OPS_CONVERGED_PASS * steps + IM_OPS_FULL_PASS * max(0.0, total_passes - steps)
            basis = ("%d per converged pass + %d per full pass (tests/test_opcount.py), every step's last pass "
                     "counted as its converged one" % (IM_OPS_CONVERGED_PASS, IM_OPS_FULL_PASS))
        else:
            ops = RK4_OPS_PER_ORBIT_STEP * float(n) * a.nsteps
            basis = "%d per RK4 orbit-step (tests/test_opcount.py)" % RK4_OPS_PER_ORBIT_STEP
        achieved = ops / t_s / 1e12
        entry["roofline"] = {"bound": prec, "achieved": achieved, "peak": peaks[prec], "unit": "TFLOP/s",
                             "frac": achieved / peaks[prec], "ops": basis,
                             "peak_source": "measured %s FMA issue rate on this GPU, 2 flops/FMA" % prec}
        out[name] = entry
        sim.close()
        del rec
        torch.cuda.empty_cache()
    return {"companions": out}


def adaptive_companion(a, n, dev, stream):
    """The adaptive solver (Dormand-Prince 5(4), no reference counterpart) on
    the headline's orbits and record grid: the same 2^20 orbit draws, a record
    every 100 x 1e-3 time units, rtol 1e-6 and atol 1e-9, over 0.2 time units
    (two record intervals).  Where fixed-step RK4 at dt 1e-3 diverges for 99 %
    of the orbits, this keeps every orbit finite; reported as accepted steps
    per second and orbit-intervals per second."""
    import torch

    from sodecl_b200 import Integrator, system_path

    t0, y0, p = workload(n, 0)
    dt, ksteps, tspan = 1e-3, 100, 0.2
    sim = Integrator(system_path("oculomotor"), "dp45", dt=dt, tspan=tspan, ksteps=ksteps, neq=6, npar=6, orbits=n,
                     rtol=1e-6, atol=1e-9)
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    td, yd, pd = T(t0), T(y0), T(p)
    hd = torch.zeros(n, dtype=torch.float64, device=dev)
    rec = torch.empty((sim.num_records, 6, n), dtype=torch.float64, device=dev)
    passes = torch.zeros(n, dtype=torch.int64, device=dev)
    ms = []
    for it in range(3):
        td.copy_(T(t0))
        yd.copy_(T(y0))
        hd.zero_()
        passes.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), counters=hd.data_ptr(),
                   records=rec.data_ptr(), newton_passes=passes.data_ptr(), stream=stream.cuda_stream)
        e.record(stream)
        torch.cuda.synchronize()
        if it > 0:
            ms.append(s.elapsed_time(e))
    steps = int(passes.sum().item())
    t_ms = float(np.mean(ms))
    last = rec[-1].cpu().numpy()
    out = {"orbits": n, "dt_first_step": dt, "record_every": ksteps * dt, "tspan": tspan, "rtol": 1e-6, "atol": 1e-9,
           "ms": t_ms, "accepted_steps": steps, "accepted_steps_per_s": steps / (t_ms * 1e-3),
           "orbit_intervals_per_s": n * sim.num_chunks / (t_ms * 1e-3),
           "steps_per_orbit_median": float(np.median(passes.cpu().numpy())),
           "nan_fraction_final": float(np.mean(~np.isfinite(last).all(axis=0)))}
    sim.close()
    return out


# The reference's one published figure (its README): "Compute results runtime:
# 0.0690873 sec." for examples/kuramoto_euler_stochastic.py on an Intel Core
# i7-4790K at 4.00 GHz, Intel OpenCL CPU runtime, local group size 8.
README_PUBLISHED_S = 0.0690873


def readme_case_companion(reps=5):
    """The run the reference publishes a time for: its README's
    examples/kuramoto_euler_stochastic.py -- Kuramoto N=3 by Euler-Maruyama,
    2 orbits, dt 0.05, tspan 50, a record every 40 steps (1000 steps, 26
    records), phases U(-3.1416, 3.1416), K 0.2, omega U(0.2, 0.4), noise
    amplitudes U(0.01, 0.03) (seeded here; the script draws them unseeded) --
    on the reference's own examples/kuramoto.cl, through the reference's
    Python entry point on this library (sodecl_b200.sodecl.sodecl, a new
    manager per call, as the script makes).  'compute_results_runtime_s' is
    what the reference's line of that name times (the run loop: launches and
    record copies, sodeclmgr.cpp:951-1020), from this library's own timing of
    sodecl_cuda_run; 'call_s' is the whole call with the program from the
    cache (the reference's 'Simulation execution time', 0.589 s there,
    includes its OpenCL build)."""
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.sodecl import sodecl

    path = REFERENCE_KURAMOTO if os.path.isfile(REFERENCE_KURAMOTO) else system_path("kuramoto")
    orbits, nequat, nnoi, dt, tspan, ksteps = 2, 3, 3, 0.05, 50.0, 40
    rng = np.random.default_rng(12)
    initx = rng.uniform(-3.1416, 3.1416, (orbits, nequat))
    params = np.concatenate([np.full((orbits, 1), 0.2), rng.uniform(0.2, 0.4, (orbits, nequat)),
                             rng.uniform(0.01, 0.03, (orbits, nequat))], axis=1)
    # the run loop alone, as the reference's "Compute results runtime" line times it
    sim = Integrator(path, "se", dt=dt, tspan=tspan, ksteps=ksteps, neq=nequat, npar=params.shape[1], nnoi=nnoi,
                     orbits=orbits)
    loop_ms = []
    for _ in range(reps + 1):
        sim.upload(np.zeros(orbits), initx, params)
        sim.run()
        loop_ms.append(sim.last_run_ms()[1])
    sim.close()
    # the whole call through the reference's entry point
    call_s = []
    with stdout_to_stderr():
        for _ in range(reps + 1):
            w = time.perf_counter()
            t, res = sodecl(0, 0, path, initx, params, 0, orbits, nequat, nnoi, dt, tspan, ksteps, 0)
            call_s.append(time.perf_counter() - w)
    runtime_s = float(np.median(loop_ms[1:])) * 1e-3
    return {"system_file": "reference examples/kuramoto.cl" if path == REFERENCE_KURAMOTO else "package kuramoto.cl",
            "orbits": orbits, "N": nequat, "solver": "Euler-Maruyama", "dt": dt, "tspan": tspan, "record_every": ksteps,
            "records": int(res.shape[1]), "compute_results_runtime_s": runtime_s,
            "call_s": float(np.median(call_s[1:])), "published_s": README_PUBLISHED_S,
            "published_hardware": "Intel Core i7-4790K @ 4.00 GHz, Intel OpenCL CPU runtime (the reference's README)",
            "speedup_vs_published": README_PUBLISHED_S / runtime_s}


def small_kuramoto_companion(dev, stream, sin_peaks):
    """The plain CPU-sized case: Kuramoto N=8, 1024 orbits, K ~ U(0,5) per orbit,
    omega ~ N(0,1) shared, theta0 ~ U(0, 2 pi), explicit Euler, dt 0.05, 1000
    steps, a record every 10 (101 records), FP64.  One launch; at this size it
    is latency-bound (1024 orbits on 148 SMs), so the tuner's lanes per orbit
    (several lanes sharing one orbit's 8 rows) shorten each orbit's steps."""
    import torch

    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.workloads import kuramoto

    n, N, nsteps, ksteps, dt = 1024, 8, 1000, 10, 0.05
    t0, th0, p, _ = kuramoto(n, N, seed=11)
    out = {"orbits": n, "N": N, "nsteps": nsteps, "records": nsteps // ksteps + 1, "unit": METRIC}
    T = lambda x: torch.tensor(x, device=dev)  # noqa: E731
    for name, tune in (("one_thread_per_orbit", False), ("tuned", True)):
        sim = Integrator(system_path("kuramoto"), "euler", dt=dt, tspan=nsteps * dt, ksteps=ksteps, neq=N,
                         npar=N + 1, orbits=n)
        choice = None
        if tune:
            sim.upload(t0, th0, p)
            choice = sim.autotune(sample_orbits=n, sample_steps=200)
        td, yd, pd = T(t0), T(th0), T(p)
        rec = torch.empty((sim.num_records, N, n), dtype=torch.float64, device=dev)
        ms = []
        for it in range(4):
            td.copy_(T(t0))
            yd.copy_(T(th0))
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            sim.launch(t=td.data_ptr(), y=yd.data_ptr(), params=pd.data_ptr(), records=rec.data_ptr(),
                       stream=stream.cuda_stream)
            e.record(stream)
            torch.cuda.synchronize()
            if it > 0:
                ms.append(s.elapsed_time(e))
        sim.close()
        out[name] = {"ms": float(np.mean(ms)), "value": n * nsteps / (np.mean(ms) * 1e-3),
                     "launch": choice or {"lanes": 1, "block": 128},
                     "roofline": sine_roofline(n * nsteps * N * N, np.mean(ms) * 1e-3, sin_peaks["fp64"],
                                               "N^2 = %d sines per orbit-step (one right-hand side)" % (N * N))}
    return out


if __name__ == "__main__":
    main()
