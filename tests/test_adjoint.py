"""Discrete adjoint (model fitting): loss and d(loss)/d(params, y0) per orbit.

The GPU adjoint (sodecl_cuda_adjoint) is checked against
  * an FP64 reference gradient: forward-mode dual numbers through the same
    system file and a restatement of the steps (oracle/gradient.cpp), which is
    exact to rounding -- agreement to 1e-9 of the gradient's scale (measured:
    ~1e-15);
  * central finite differences of the GPU loss (relative step 1e-6), the
    baseline the adjoint replaces -- agreement to 1e-5, the finite differences'
    own error at that step being a few 1e-6.
All three derivative paths are exercised: the system file's own
vector-Jacobian product (calc_vjp), its analytic Jacobians (calc_jacobian +
calc_jacobian_params), and the reverse-mode tape.
The per-orbit loss is checked against the CPU oracle's records."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, reference_gradient

NOMINAL = np.array([120.0, 1.5, 0.0045, 0.05, 600.0, 9.0])
Y0 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 2.0])
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SYSTEMS = os.path.join(REPO, "sodecl_b200", "systems")


def fitting_problem(n, seed, dt=1e-5, nchunks=10, ksteps=50, noise=1e-2, solver=2):
    """Targets: trajectories of perturbed true parameters plus Gaussian noise."""
    rng = np.random.default_rng(seed)
    true_p = NOMINAL * rng.uniform(0.5, 1.5, (n, 6))
    y0 = np.tile(Y0, (n, 1))
    rec = Oracle("oculomotor").run(solver, np.zeros(n), y0, true_p, neq=6, npar=6, dt=dt, ksteps=ksteps,
                                   nchunks=nchunks).records
    targets = rec + rng.normal(0, noise, rec.shape)
    guess = true_p * rng.uniform(0.95, 1.05, (n, 6))
    return np.zeros(n), y0, guess, targets


def test_reference_gradient_matches_cpu_finite_differences():
    t0, y0, p, tg = fitting_problem(2, 0, nchunks=4, ksteps=25)
    kw = dict(neq=6, npar=6, dt=1e-5, ksteps=25, nchunks=4)
    loss, gp, gy = reference_gradient(os.path.join(SYSTEMS, "oculomotor.cl"), 2, 6, 6, 1e-5, 25, 4, t0, y0, p, tg)
    o = Oracle("oculomotor")

    def cpu_loss(pp, yy):
        rec = o.run(2, t0, yy, pp, **kw).records
        return ((rec - tg) ** 2).sum(axis=(0, 1)) / (5 * 6)

    assert np.allclose(cpu_loss(p, y0), loss, rtol=1e-13)
    for j in range(6):
        h = 1e-6 * abs(p[0, j])
        pp, pm = p.copy(), p.copy()
        pp[:, j] += h
        pm[:, j] -= h
        fd = (cpu_loss(pp, y0) - cpu_loss(pm, y0)) / (2 * h)
        assert np.allclose(fd, gp[:, j], rtol=1e-5, atol=1e-9 * np.abs(gp).max())


def oculomotor_source(products):
    """The oculomotor system file with the adjoint taking `products` from
    calc_vjp ("vjp"), from the two Jacobians ("jacobians": calc_vjp renamed
    away) or from the tape ("tape")."""
    from sodecl_b200 import system_path

    src = open(system_path("oculomotor")).read()
    if products == "jacobians":
        src = src.replace("void calc_vjp(", "void unused_calc_vjp(")
    return src


@pytest.mark.gpu
@pytest.mark.parametrize("products", ["vjp", "jacobians", "tape"])
@pytest.mark.parametrize("solver", ["rk4", "euler"])
def test_adjoint_matches_reference_gradient(solver, products):
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint

    use_tape = products == "tape"

    n, nchunks, ksteps, dt = 64, 10, 50, 1e-5 if solver == "rk4" else 1e-6
    t0, y0, p, tg = fitting_problem(n, 1, dt=dt, nchunks=nchunks, ksteps=ksteps)
    sid = 2 if solver == "rk4" else 1
    loss_r, gp_r, gy_r = reference_gradient(system_path("oculomotor"), sid, 6, 6, dt, ksteps, nchunks, t0[:8], y0[:8],
                                            p[:8], tg[:, :, :8])
    sim = Integrator(None, solver, dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps,
                     neq=6, npar=6, orbits=n, system_src=oculomotor_source(products))
    assert sim.num_chunks == nchunks
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    loss, gp, gy, flags = Adjoint(sim, use_tape=use_tape)(T(t0), T(y0), T(p), T(tg))
    loss, gp, gy = loss.cpu().numpy(), gp.cpu().numpy(), gy.cpu().numpy()
    assert not flags.any()
    np.testing.assert_allclose(loss[:8], loss_r, rtol=1e-11)
    scale_p = np.abs(gp_r).max(axis=1, keepdims=True)
    scale_y = np.abs(gy_r).max(axis=1, keepdims=True)
    assert np.max(np.abs(gp[:8] - gp_r) / scale_p) < 1e-9
    assert np.max(np.abs(gy[:8] - gy_r) / scale_y) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("products", ["vjp", "jacobians", "tape"])
@pytest.mark.parametrize("solver", ["ie", "im"])
def test_implicit_adjoint_matches_reference_gradient(solver, products):
    """Implicit Euler / midpoint at dt 1e-3: the adjoint of the exact implicit
    step (transposed solve with the full Jacobian) against dual numbers pushed
    through the reference's Newton passes.  With the passes run to 1e-12 the
    two derivatives coincide to the iteration's convergence."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint

    n, nchunks, ksteps, dt, tol = 48, 5, 20, 1e-3, 1e-12
    sid = 3 if solver == "ie" else 4
    t0, y0, p, tg = fitting_problem(n, 5, dt=dt, nchunks=nchunks, ksteps=ksteps, solver=sid)
    loss_r, gp_r, gy_r = reference_gradient(system_path("oculomotor"), sid, 6, 6, dt, ksteps, nchunks, t0[:8], y0[:8],
                                            p[:8], tg[:, :, :8], newton_tol=tol, newton_max_iter=200)
    sim = Integrator(None, solver, dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps, neq=6, npar=6,
                     orbits=n, newton_tol=tol, newton_max_iter=200, system_src=oculomotor_source(products))
    T = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    loss, gp, gy, flags = Adjoint(sim, use_tape=products == "tape")(T(t0), T(y0), T(p), T(tg))
    loss, gp, gy, flags = loss.cpu().numpy(), gp.cpu().numpy(), gy.cpu().numpy(), flags.cpu().numpy()
    assert not flags.any()
    np.testing.assert_allclose(loss[:8], loss_r, rtol=1e-9)
    err_p = np.max(np.abs(gp[:8] - gp_r) / np.abs(gp_r).max(axis=1, keepdims=True))
    err_y = np.max(np.abs(gy[:8] - gy_r) / np.abs(gy_r).max(axis=1, keepdims=True))
    print("%s/%s adjoint vs dual numbers: params %.2e, y0 %.2e" % (solver, products, err_p, err_y))
    assert err_p < 1e-7 and err_y < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["ie", "im"])
def test_implicit_adjoint_schedules_agree(solver):
    """Implicit solvers: the whole-trajectory schedule and the checkpoint
    schedules give the same loss, gradients and pass-limit flags bit for bit,
    steps stopped at the pass limit included."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint

    n, nchunks, ksteps, dt = 2000, 6, 25, 1e-3
    sid = 3 if solver == "ie" else 4
    t0, y0, p, tg = fitting_problem(n, 9, dt=dt, nchunks=nchunks, ksteps=ksteps, solver=sid)
    T = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    for max_iter in (1000, 12):  # 12 passes stop steps early (flagged)
        sim = Integrator(system_path("oculomotor"), solver, dt=dt, tspan=(nchunks * ksteps - 0.5) * dt,
                         ksteps=ksteps, neq=6, npar=6, orbits=n, newton_tol=1e-10, newton_max_iter=max_iter)
        runs = [Adjoint(sim, ckpt_every=c)(T(t0), T(y0), T(p), T(tg)) for c in (0, 1, 7, 10**6)]
        flagged = int((runs[0][3] != 0).sum())
        assert flagged > 0 if max_iter == 12 else flagged < n
        for r in runs[1:]:
            for a, b in zip(r, runs[0]):
                assert torch.equal(a, b)
        sim.close()


@pytest.mark.gpu
def test_adjoint_against_finite_differences_and_checkpoint_spacing():
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint, finite_difference_gradient

    n, nchunks, ksteps, dt = 256, 20, 25, 1e-5
    t0, y0, p, tg = fitting_problem(n, 2, dt=dt, nchunks=nchunks, ksteps=ksteps)
    kw = dict(dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps, neq=6, npar=6)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    sim = Integrator(system_path("oculomotor"), "rk4", orbits=n, **kw)
    # 500 steps: ckpt_every 500 and above leave one segment, recorded by the
    # forward sweep itself (no recomputation)
    grads = [Adjoint(sim, ckpt_every=c)(T(t0), T(y0), T(p), T(tg)) for c in (0, 1, 7, 499, 500, 10**6)]
    for g in grads[1:]:  # recomputation is exact: same loss and gradients for any spacing
        assert torch.equal(g[0], grads[0][0])
        assert torch.equal(g[1], grads[0][1]) and torch.equal(g[2], grads[0][2])
    wide = Integrator(system_path("oculomotor"), "rk4", orbits=n * 24, **kw)
    fd_p, fd_y = finite_difference_gradient(T(t0), T(y0), T(p), T(tg), Adjoint(wide))
    gp, gy = grads[0][1], grads[0][2]
    err_p = ((gp - fd_p).abs().amax(dim=1) / gp.abs().amax(dim=1)).max().item()
    err_y = ((gy - fd_y).abs().amax(dim=1) / gy.abs().amax(dim=1)).max().item()
    print("adjoint vs central differences: params %.2e, y0 %.2e" % (err_p, err_y))
    assert err_p < 1e-5 and err_y < 1e-5


@pytest.mark.gpu
def test_release_scratch_returns_the_trajectory_buffer():
    """The whole-trajectory buffer stays with the context between calls;
    release_scratch hands it back to the device, and the next call
    allocates it again and gives the same gradients."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint

    n, nchunks, ksteps, dt = 1 << 14, 10, 50, 1e-5
    t0, y0, p, tg = fitting_problem(n, 3, dt=dt, nchunks=nchunks, ksteps=ksteps)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    with Integrator(system_path("oculomotor"), "rk4", orbits=n, dt=dt, tspan=(nchunks * ksteps - 0.5) * dt,
                    ksteps=ksteps, neq=6, npar=6) as sim:
        adj = Adjoint(sim)
        first = adj(T(t0), T(y0), T(p), T(tg))
        torch.cuda.synchronize()
        held = n * nchunks * ksteps * 25 * 8  # the RK4 trajectory: state, t and three stage inputs per step
        before = torch.cuda.mem_get_info()[0]
        sim.release_scratch()
        after = torch.cuda.mem_get_info()[0]
        assert after - before >= 0.9 * held
        sim.release_scratch()  # nothing left: a no-op
        again = adj(T(t0), T(y0), T(p), T(tg))
        for a, b in zip(first[:3], again[:3]):
            assert torch.equal(a, b)


@pytest.mark.gpu
def test_torch_autograd_function_and_tape_overflow():
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint, trajectory_mse

    n, nchunks, ksteps, dt = 32, 5, 20, 1e-5
    t0, y0, p, tg = fitting_problem(n, 3, dt=dt, nchunks=nchunks, ksteps=ksteps)
    sim = Integrator(system_path("oculomotor"), "rk4", dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps,
                     neq=6, npar=6, orbits=n)
    dev = torch.device("cuda")
    params = torch.tensor(p, device=dev, requires_grad=True)
    y0t = torch.tensor(y0, device=dev, requires_grad=True)
    adj = Adjoint(sim)
    loss = trajectory_mse(params, y0t, torch.tensor(t0, device=dev), torch.tensor(tg, device=dev), adj)
    (2.0 * loss.sum()).backward()
    _, gp, gy, _ = adj(torch.tensor(t0, device=dev), torch.tensor(y0, device=dev), torch.tensor(p, device=dev),
                       torch.tensor(tg, device=dev))
    assert torch.allclose(params.grad, 2.0 * gp) and torch.allclose(y0t.grad, 2.0 * gy)
    # a tape too short for one right-hand side is reported, not silently wrong
    _, _, _, flags = Adjoint(sim, tape_entries=16, use_tape=True)(torch.tensor(t0, device=dev), torch.tensor(y0, device=dev),
                                                    torch.tensor(p, device=dev), torch.tensor(tg, device=dev))
    assert (flags.cpu().numpy() & 4).all()
    with pytest.raises(RuntimeError):
        trajectory_mse(params, y0t, torch.tensor(t0, device=dev), torch.tensor(tg, device=dev),
                       Adjoint(sim, tape_entries=16, use_tape=True))


@pytest.mark.parametrize("system,neq,npar,jacp", [("oculomotor", 6, 6, True), ("kuramoto", 8, 9, False)])
def test_system_jacobians_match_central_differences(tmp_path, system, neq, npar, jacp):
    """calc_jacobian (and calc_jacobian_params and calc_vjp where present)
    against central differences of sode_system, on the host.  Both bursts'
    branches of the oculomotor model are visited (y5 of either sign)."""
    import subprocess

    exe = str(tmp_path / "jacobian_fd")
    cmd = ["g++", "-O1", "-std=c++17", "-DNUMEQ=%d" % neq, "-DNUMPAR=%d" % npar,
           '-DSYSTEM_FILE="%s"' % os.path.join(SYSTEMS, system + ".cl"),
           os.path.join(REPO, "tests", "cpp", "jacobian_fd.cpp"), "-o", exe]
    if jacp:
        cmd[1:1] = ["-DHAS_JACP", "-DHAS_VJP"]
    subprocess.run(cmd, check=True)
    rng = np.random.default_rng(7)
    cases = []
    for k in range(16):
        if system == "oculomotor":
            y = rng.normal(0, 0.5, neq)
            y[5] = (1 if k % 2 else -1) * rng.uniform(0.1, 3.0)
            p = NOMINAL * rng.uniform(0.5, 1.5, npar)
        else:
            y = rng.uniform(0, 2 * np.pi, neq)
            p = np.concatenate([[rng.uniform(0, 5)], rng.normal(size=neq)])
        cases.append(" ".join("%.17g" % v for v in np.concatenate([y, p])))
    out = subprocess.run([exe], input="\n".join(cases) + "\n", capture_output=True, text=True, check=True).stdout
    errs = np.array([[float(v) for v in line.split()] for line in out.strip().splitlines()])
    assert errs.shape == (16, 3)
    print("%s: max rel diff J %.2e, Jp %.2e, vjp %.2e" % (system, errs[:, 0].max(), errs[:, 1].max(),
                                                          errs[:, 2].max()))
    assert errs.max() < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("use_tape", [False, True])
def test_adjoint_division_modes_bit_identical(use_tape):
    """Loss-only passes divide in the context's mode, passes with gradients in
    IEEE division; the reciprocal quotient is IEEE-rounded, so losses and
    gradients agree bit for bit across modes and passes."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint

    n, nchunks, ksteps, dt = 200, 6, 20, 1e-5
    t0, y0, p, tg = fitting_problem(n, 4, dt=dt, nchunks=nchunks, ksteps=ksteps)
    kw = dict(dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps, neq=6, npar=6, orbits=n)
    T = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    outs = []
    for d in ("ieee", "reciprocal"):
        adj = Adjoint(Integrator(system_path("oculomotor"), "rk4", division=d, **kw), use_tape=use_tape)
        full = adj(T(t0), T(y0), T(p), T(tg))
        loss_only = adj(T(t0), T(y0), T(p), T(tg), with_gradient=False)
        assert torch.equal(full[0], loss_only[0])
        outs.append(full)
    for a, b in zip(outs[0][:3], outs[1][:3]):
        assert torch.equal(a, b)


@pytest.mark.gpu
def test_gradient_fit_reduces_the_loss():
    """Model fitting end to end: Adam on log-parameters through trajectory_mse
    (one adjoint launch per iteration, the compiled programs and device
    buffers kept across iterations) pulls perturbed oculomotor parameters
    back towards the ones that made the targets."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint, trajectory_mse

    n, nchunks, ksteps, dt = 64, 10, 50, 1e-5
    t0, y0, p, tg = fitting_problem(n, 9, dt=dt, nchunks=nchunks, ksteps=ksteps, noise=0.0)
    sim = Integrator(system_path("oculomotor"), "rk4", dt=dt, tspan=(nchunks * ksteps - 0.5) * dt, ksteps=ksteps,
                     neq=6, npar=6, orbits=n)
    adj = Adjoint(sim)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    logp = torch.log(T(p)).requires_grad_(True)
    y0t, t0t, tgt = T(y0), T(t0), T(tg)
    opt = torch.optim.Adam([logp], lr=0.01)
    losses = []
    for _ in range(40):
        opt.zero_grad()
        loss = trajectory_mse(torch.exp(logp), y0t, t0t, tgt, adj)
        loss.sum().backward()
        opt.step()
        losses.append(float(loss.detach().sum()))
    print("fit: loss %.3e -> %.3e" % (losses[0], losses[-1]))
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0]  # measured: 87.1 -> 18.6


@pytest.mark.gpu
def test_adjoint_at_the_fitting_shape_against_dual_numbers():
    """The fitting configuration itself -- 2^16 orbits, 5000 RK4 steps of
    dt 1e-5, a record every 100, targets from seeded true parameters plus
    N(0, 1e-2) noise, gradient at parameters within +-5 % -- and 64 of its
    orbits (spread over the index range) against the FP64 dual-number
    reference gradient: per orbit, max |adjoint - reference| over the 12
    derivatives, relative to the largest |reference|, within 1e-6."""
    torch = pytest.importorskip("torch")
    from sodecl_b200 import Integrator, system_path
    from sodecl_b200.fit import Adjoint
    from sodecl_b200.workloads import fitting_targets

    n, nsteps, ksteps, dt = 1 << 16, 5000, 100, 1e-5
    dev = torch.device("cuda")
    t0, y0, guess, targets = fitting_targets(n, nsteps, ksteps, dt, device=dev)
    sim = Integrator(system_path("oculomotor"), "rk4", dt=dt, tspan=(nsteps - 0.5) * dt, ksteps=ksteps, neq=6,
                     npar=6, orbits=n)
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    loss, gp, gy, flags = Adjoint(sim)(T(t0), T(y0), T(guess), targets)
    assert not flags.any()
    pick = np.linspace(0, n - 1, 64).astype(int)
    tg = targets.cpu().numpy()[:, :, pick]
    loss_r, gp_r, gy_r = reference_gradient(system_path("oculomotor"), 2, 6, 6, dt, ksteps, nsteps // ksteps,
                                            t0[pick], y0[pick], guess[pick], tg)
    gp, gy = gp.cpu().numpy()[pick], gy.cpu().numpy()[pick]
    np.testing.assert_allclose(loss.cpu().numpy()[pick], loss_r, rtol=1e-9)
    err = np.maximum(np.abs(gp - gp_r).max(axis=1) / np.abs(gp_r).max(axis=1),
                     np.abs(gy - gy_r).max(axis=1) / np.abs(gy_r).max(axis=1))
    print("adjoint vs dual numbers at 2^16 x 5000, 64 orbits: max %.2e, p99 %.2e, median %.2e"
          % (err.max(), np.quantile(err, 0.99), np.median(err)))
    assert err.max() <= 1e-6
