"""The CPU oracle, pinned against the reference's own known answers.

The oracle (oracle/oracle_solvers.h) is the checker of every GPU parity test,
so it is itself checked first:
  * against the reference's golden arrays (tests/data/oculomotor_*.pkl of the
    reference, re-saved in tests/golden), with the reference test's own rule
    (numpy.isclose, tests/sodecl_python_tests.py:50) and a tight bound;
  * against fixtures produced by the reference's kernel sources compiled as C
    (tests/golden/ref_*.npz) -- bit for bit, same arithmetic, same libm;
  * against the reference's vendored Threefry on raw words and u01 doubles.
"""
import os

import numpy as np
import pytest

from oracle.oracle import (IMPLICIT_EULER, IMPLICIT_MIDPOINT, Oracle, ReferenceBuild, num_chunks, printed_dt,
                           to_reference_layout)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NOMINAL = [120.0, 1.5, 0.0045, 0.05, 600.0, 9.0]
Y0 = [0.0, 0.0, 0.0, 0.0, 0.0, 2.0]
# tests/sodecl_python_tests.py of the reference: solver, dt, ksteps (tspan 0.1, 2 orbits)
GOLDEN_CASES = {"euler": (1, 1e-8, 40000), "rk": (2, 1e-6, 400), "ie": (3, 1e-6, 400), "im": (4, 1e-6, 400)}


@pytest.fixture(scope="module")
def oculomotor():
    return Oracle("oculomotor")


@pytest.fixture(scope="module")
def kuramoto():
    return Oracle("kuramoto")


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_golden_reference_arrays(oculomotor, name):
    solver, dt, ksteps = GOLDEN_CASES[name]
    golden = np.load(os.path.join(GOLDEN, "oculomotor_%s.npy" % name))
    r = oculomotor.run(solver, np.zeros(2), np.tile(Y0, (2, 1)), np.tile(NOMINAL, (2, 1)), neq=6, npar=6, dt=dt,
                       tspan=0.1, ksteps=ksteps)
    got = to_reference_layout(r.records)
    assert got.shape == golden.shape
    assert np.isclose(got, golden).all()
    # the reference's OpenCL CPU run and this oracle differ by rounding only
    assert np.max(np.abs(got - golden) / np.maximum(np.abs(golden), 1.0)) < 1e-13


def test_record_count_matches_reference_loop():
    # 0.1/(1e-8*40000) == 250.0 -> 251 records; 0.1/(1e-6*400) > 250 -> 252
    assert num_chunks(0.1, 1e-8, 40000) + 1 == 251
    assert num_chunks(0.1, 1e-6, 400) + 1 == 252
    assert num_chunks(50, 0.05, 10) == 100
    assert num_chunks(0.0, 0.05, 10) == 0


def test_printed_dt():
    assert printed_dt(1e-8) == 1e-8
    assert printed_dt(0.0123456789) == 0.0123457
    assert printed_dt(1.0 / 3.0) == 0.333333


def _fixture(name):
    return dict(np.load(os.path.join(GOLDEN, "ref_%s.npz" % name)))


@pytest.mark.parametrize("name,system", [("kuramoto_euler", "kuramoto"), ("kuramoto_se", "kuramoto"),
                                         ("kuramoto32_se", "kuramoto"), ("oculomotor_se", "oculomotor"),
                                         ("oculomotor_im", "oculomotor"), ("oculomotor_ie", "oculomotor"),
                                         ("oculomotor_rk4", "oculomotor")])
def test_reference_build_fixtures_bit_exact(name, system):
    f = _fixture(name)
    o = Oracle(system)
    r = o.run(int(f["solver"]), f["t0"], f["y0"], f["params"], neq=int(f["neq"]), npar=int(f["npar"]),
              nnoi=int(f["nnoi"]), dt=float(f["dt"]), ksteps=int(f["ksteps"]), nchunks=int(f["nchunks"]),
              counters=f.get("counters"), orbit_offset=int(f["orbit_offset"]))
    np.testing.assert_array_equal(r.records, f["records"])
    np.testing.assert_array_equal(r.y, f["y_final"])
    np.testing.assert_array_equal(r.t, f["t_final"])
    if "counters" in f:
        np.testing.assert_array_equal(r.counters, f["counters_final"])


def test_threefry_against_vendored_random123(kuramoto):
    f = dict(np.load(os.path.join(GOLDEN, "threefry_words.npz")))
    for ctr, words, u01 in zip(f["ctr"], f["words"], f["u01"]):
        np.testing.assert_array_equal(kuramoto.threefry2x64_20(ctr, f["key"]), words)
        assert [kuramoto.u01_open_open(int(w)) for w in words] == list(u01)
    # known answer computed with the vendored header
    w = kuramoto.threefry2x64_20([0, 0], [0, 0xF00DCAFE])
    assert [int(x) for x in w] == [0x03ED3FEB0846F822, 0xE6E400C11521CD65]


def test_counter_word_conversion(kuramoto):
    assert kuramoto.counter_word(0.0) == 0
    assert kuramoto.counter_word(12345.75) == 12345
    assert kuramoto.counter_word(-1.0) == 2 ** 64 - 1
    assert kuramoto.counter_word(-2.5) == 2 ** 64 - 2
    assert kuramoto.counter_word(2.0 ** 63) == 2 ** 63
    assert kuramoto.counter_word(2.0 ** 63 + 2.0 ** 11) == 2 ** 63 + 2 ** 11


def test_noise_stream_statistics(kuramoto):
    z = kuramoto.noise_stream(3, 0.0, 4, 1.0, 20000)
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1.0) < 0.02


def test_newton_pass_limit_flags(oculomotor):
    r = oculomotor.run(IMPLICIT_MIDPOINT, np.zeros(2), np.tile(Y0, (2, 1)), np.tile(NOMINAL, (2, 1)), neq=6, npar=6,
                       dt=1e-3, tspan=0.01, ksteps=10, newton_tol=1e-14, newton_max_iter=3)
    assert (r.flags & 1).all()
    assert (r.newton_passes == 3 * 10).all()
    r = oculomotor.run(IMPLICIT_EULER, np.zeros(2), np.tile(Y0, (2, 1)), np.tile(NOMINAL, (2, 1)), neq=6, npar=6,
                       dt=1e-3, tspan=0.01, ksteps=10)
    assert not (r.flags & 1).any()
    assert (r.newton_passes > 10).all()


def test_fp32_oracle_close_to_fp64():
    o32, o64 = Oracle("oculomotor", "fp32"), Oracle("oculomotor", "fp64")
    rng = np.random.default_rng(3)
    p = np.asarray(NOMINAL) * rng.uniform(0.5, 1.5, (16, 6))
    kw = dict(neq=6, npar=6, dt=1e-5, tspan=0.01, ksteps=100)
    a = o32.run(2, np.zeros(16), np.tile(Y0, (16, 1)), p, **kw).records
    b = o64.run(2, np.zeros(16), np.tile(Y0, (16, 1)), p, **kw).records
    scale = np.abs(b).max(axis=(0, 2), keepdims=True)
    # single precision over 1000 stiff steps: ~1e-3 of each equation's scale
    assert np.max(np.abs(a - b) / scale) < 1e-2
    assert not np.array_equal(a, b)


@pytest.mark.skipif(not ReferenceBuild.available("oculomotor", 2), reason="reference build not present")
@pytest.mark.parametrize("solver", [0, 1, 2, 3, 4])
def test_restatement_equals_reference_build(oculomotor, solver):
    rng = np.random.default_rng(solver)
    n = 16
    p = np.asarray(NOMINAL) * rng.uniform(0.5, 1.5, (n, 6))
    nnoi = 2 if solver == 0 else 0
    if nnoi:
        p = np.concatenate([p, rng.uniform(0, 0.1, (n, 2))], axis=1)
    kw = dict(neq=6, npar=p.shape[1], nnoi=nnoi, dt=1e-4, tspan=0.02, ksteps=20)
    cnt = rng.uniform(-1e11, 1e11, n) if nnoi else None
    y0 = np.tile(Y0, (n, 1))
    a = oculomotor.run(solver, np.zeros(n), y0, p, counters=cnt, orbit_offset=3, **kw)
    b = ReferenceBuild("oculomotor", solver).run(np.zeros(n), y0, p, counters=cnt, orbit_offset=3, **kw)
    np.testing.assert_array_equal(a.records, b.records)


def test_oracle_build_stamp_covers_headers(tmp_path):
    """A change to an oracle header (oracle_solvers.h, oracle_prelude.h) must
    rebuild the oracle libraries, although the compiled unit only names them."""
    import shutil

    from oracle import build

    for h in os.listdir(os.path.dirname(build.__file__)):
        if h.endswith(".h"):
            shutil.copy(os.path.join(os.path.dirname(build.__file__), h), tmp_path / h)
    cmd, unit = ["gcc", "-O2"], '#include "oracle_solvers.h"\n'
    before = build.build_digest(cmd, unit, str(tmp_path))
    assert build.build_digest(cmd, unit, str(tmp_path)) == before
    with open(tmp_path / "oracle_solvers.h", "a") as f:
        f.write("\n/* edited */\n")
    assert build.build_digest(cmd, unit, str(tmp_path)) != before
