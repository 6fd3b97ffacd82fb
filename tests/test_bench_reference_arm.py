"""bench.py's reference arm on the CPU: the reference's kernels compiled as C
time a sample of the headline workload, the line carries the same `config`
as the GPU arm, and the process maps none of this library's native code (the
package loads libsodecl_cuda.so only when its API is first used)."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1", "--cpu-orbits", "256",
            "--orbits", "4096", "--nsteps", "200", "--ksteps", "100"]
sys.path.insert(0, %(repo)r)
import bench
a = bench.parse()
bench.run_reference_arm(a, 0)
maps = open("/proc/self/maps").read()
print(json.dumps({"config": bench.config_dict(a, a.orbits),
                  "mapped": sorted(set(l.split()[-1] for l in maps.splitlines() if l.endswith(".so")))}))
"""


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libref_oculomotor_rk4.so")),
                    reason="the reference's kernels are not built (oracle/build.py builds them where the reference "
                           "checkout is present)")
def test_reference_arm_maps_no_library_code():
    out = subprocess.run([sys.executable, "-c", CHILD % {"repo": REPO}], capture_output=True, text=True, timeout=300,
                         cwd=REPO)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["metric"] == "orbit-steps/s"
    assert line["config"] == probe["config"]
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # the sample's own time: 256 orbits x 200 steps per step
    assert abs(line["value"] * line["ms_per_step"] * 1e-3 - 256 * 200) < 1e-6 * 256 * 200
    mapped = [m for m in probe["mapped"] if m.startswith(REPO)]
    assert not [m for m in mapped if "sodecl_b200" in m], mapped
    assert any("oracle/_ref/libref_oculomotor_rk4.so" in m for m in mapped)


def test_bench_parity_measure():
    """The bench's parity block: relative error over the orbits finite in both
    runs, diverging orbits counted; and its CPU-to-CPU floor on a small sample
    of the headline's orbits at the stable step (the reference's kernels
    against the oracle built with FMA contraction: every orbit finite in both,
    differing in the last bits)."""
    sys.path.insert(0, REPO)
    import numpy as np

    import bench

    rng = np.random.default_rng(0)
    want = rng.uniform(1, 2, (3, 2, 5))
    got = want * (1 + 1e-12)
    want[1, 0, 3] = np.nan                 # orbit 3 diverges in the CPU run only
    got[2, 1, 4] = want[2, 1, 4] = np.inf  # orbit 4 diverges in both
    r = bench.records_error(got, want)
    assert (r["orbits"], r["orbits_finite_in_both"], r["orbits_diverging_in_both"], r["orbits_diverging_in_one"]) \
        == (5, 3, 1, 1)
    assert 0.9e-12 < r["max_rel_err"] < 1.1e-12

    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libref_oculomotor_rk4.so")):
        pytest.skip("the reference's kernels are not built")
    saved = sys.argv
    sys.argv = ["bench.py", "--nsteps", "300", "--dt", "1e-5"]
    try:
        a = bench.parse()
    finally:
        sys.argv = saved
    _, _, kind, rec = bench.cpu_reference_rate(64, a, 2)
    assert kind == "reference" and rec.shape == (4, 6, 64)
    floor = bench.parity_floor(64, a, 2, rec)
    assert floor["orbits_finite_in_both"] == 64 and 0 < floor["max_rel_err"] < 1e-9


def test_bench_keeps_native_prints_off_stdout():
    """The C++ manager prints the reference's 'Compute results runtime' line
    to standard output; inside bench.stdout_to_stderr it goes to standard
    error (C buffers flushed), so the bench's standard output is its JSON line
    alone."""
    code = r"""
import ctypes, sys
sys.argv = ["bench.py"]
sys.path.insert(0, %(repo)r)
import bench
with bench.stdout_to_stderr():
    ctypes.CDLL(None).printf(b"Compute results runtime: 0.1 sec.\n")
    print("python inside")
print('{"metric": "x"}', flush=True)
""" % {"repo": REPO}
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120, cwd=REPO)
    assert out.returncode == 0, out.stderr
    assert out.stdout == '{"metric": "x"}\n'
    assert "Compute results runtime" in out.stderr and "python inside" in out.stderr
