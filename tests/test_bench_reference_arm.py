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
