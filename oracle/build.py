"""Build the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two kinds of shared library come out of this script:

* ``oracle/_build/liboracle_<system>_<fp64|fp32>.so`` -- the plain-C
  restatement (oracle_solvers.h) compiled together with one SODECL system
  file.  Used by the tests, the smoke check and bench.py's CPU-baseline leg as
  the checker for the CUDA path.

* ``oracle/_ref/libref_<system>_<solver>.so`` -- the reference's own OpenCL C
  kernel sources (src/kernels/*.cl and examples/*.cl), concatenated in the
  order src/sodeclmgr.cpp:374-503 uses and compiled as C with ref_shim.h in
  front and ref_driver.c behind.  Only built where the reference checkout is
  present; the sources are piped to gcc and never copied into this repository.

Where the checkout is present this script also stages verbatim copies of the
reference's user-facing files (its example system files, its Python layer,
its known-answer tests and their golden data) under the git-ignored
``baseline/_ref/``, for the GPU machines, which have no checkout: the tests
run them unchanged through this library, and bench.py integrates the
reference's own oculomotor system file.

Both are built with ``-ffp-contract=off`` (x86-64 baseline has no FMA, so this
only makes the intent explicit) and OpenMP over orbits.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
SYSTEMS_DIR = os.path.join(REPO, "sodecl_b200", "systems")
# The reference checkout this recipe reads (read-only); SODECL_REFERENCE_ROOT
# overrides it.  Nothing else in the repository names this location: tests,
# smoke() and bench.py read the staged copy under baseline/_ref.
REFERENCE_ROOT = os.environ.get("SODECL_REFERENCE_ROOT", "/root/reference")
# Verbatim copies of the reference's user-facing files (system files, Python
# layer, known-answer tests and their golden data), git-ignored, so that the
# machines that run the GPU tests and the benchmark -- which have no
# reference checkout -- can run them unchanged through this library.
STAGED_ROOT = os.path.join(REPO, "baseline", "_ref")
STAGED_FILES = ["LICENSE", "examples/oculomotor.cl", "examples/kuramoto.cl", "tests/oculomotor.cl",
                "tests/kuramoto.cl", "tests/sodecl_python_tests.py", "tests/data/oculomotor_euler.pkl",
                "tests/data/oculomotor_rk.pkl", "tests/data/oculomotor_ie.pkl", "tests/data/oculomotor_im.pkl",
                "interfaces/python/sodecl.py"]

CFLAGS = ["-O2", "-std=gnu11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
          "-Wno-unused-variable", "-Wno-unused-but-set-variable"]

# solver_Type numbering (include/solver_Type.hpp:14-20 of the reference)
REF_SOLVER_FILES = {0: "stochastic_euler.cl", 1: "euler.cl", 2: "rk4.cl", 3: "ie.cl", 4: "im.cl"}
REF_SOLVER_NAMES = {0: "se", 1: "euler", 2: "rk4", 3: "ie", 4: "im"}

_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def strip_comments(src: str) -> str:
    """Source with comments blanked (string literals kept), for detection."""
    return _scan(src, lambda code: code, keep_comments=False)


def fp32_rewrite(src: str) -> str:
    """Give every unsuffixed floating literal an ``f`` suffix, outside comments
    and string literals, so a system file compiled with ``double`` defined to
    ``float`` evaluates in single precision throughout (the counterpart of
    OpenCL's -cl-single-precision-constant)."""
    return _scan(src, lambda code: _FLOAT_LIT.sub(lambda m: m.group(1) + "f", code), keep_comments=True)


def _scan(src, on_code, keep_comments):
    out, code, i, n = [], [], 0, len(src)

    def flush():
        if code:
            out.append(on_code("".join(code)))
            code.clear()

    while i < n:
        c = src[i]
        if src.startswith("//", i):
            j = src.find("\n", i)
            j = n if j < 0 else j
            flush()
            out.append(src[i:j] if keep_comments else " " * (j - i))
            i = j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            j = n if j < 0 else j + 2
            flush()
            out.append(src[i:j] if keep_comments else re.sub(r"[^\n]", " ", src[i:j]))
            i = j
        elif c in "\"'":
            j = i + 1
            while j < n and src[j] != c:
                j += 2 if src[j] == "\\" else 1
            j = min(j + 1, n)
            flush()
            out.append(src[i:j])
            i = j
        else:
            code.append(c)
            i += 1
    flush()
    return "".join(out)


def defines_function(src: str, name: str) -> bool:
    body = strip_comments(src)
    return re.search(r"\b" + name + r"\s*\([^;{]*\)\s*\{", body, re.S) is not None


def _stamp_ok(target: str, digest: str) -> bool:
    stamp = target + ".stamp"
    return os.path.exists(target) and os.path.exists(stamp) and open(stamp).read() == digest


def build_digest(cmd: list[str], source: str, header_dir: str = HERE) -> str:
    """What a build stamp records: the command, the unit, and the text of the
    oracle headers (the unit only names the headers it includes)."""
    headers = "".join(open(os.path.join(header_dir, h)).read() for h in sorted(os.listdir(header_dir))
                      if h.endswith(".h"))
    return hashlib.sha256((" ".join(cmd) + "\0" + source + "\0" + headers).encode()).hexdigest()


def _compile(source: str, target: str, extra: list[str]) -> str:
    os.makedirs(os.path.dirname(target), exist_ok=True)
    flags = CFLAGS if "-ffp-contract=fast" not in extra else [f for f in CFLAGS if f != "-ffp-contract=off"]
    cmd = ["gcc"] + flags + ["-I", HERE] + extra + ["-x", "c", "-", "-o", target, "-lm"]
    digest = build_digest(cmd, source)
    if _stamp_ok(target, digest):
        return target
    proc = subprocess.run(cmd, input=source.encode(), capture_output=True)
    if proc.returncode != 0:
        raise RuntimeError("oracle build failed for %s:\n%s" % (target, proc.stderr.decode()))
    with open(target + ".stamp", "w") as f:
        f.write(digest)
    return target


def cpu_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return any(line.startswith("flags") and " fma " in line + " " for line in f)
    except OSError:
        return False


def build_restatement(system_path: str, name: str, precision: str = "fp64", out_dir: str = BUILD_DIR) -> str:
    """Compile oracle_solvers.h with one system file into
    ``<out_dir>/liboracle_<name>_<precision>.so``.  Precisions: fp64, fp32,
    and fp64fma / fp32fma -- the same code with FMA contraction on, whose
    distance from the plain build is the noise floor the parity tests scale
    their tolerances by."""
    src = open(system_path).read()
    extra = []
    if precision.endswith("fma"):
        extra += ["-mfma", "-ffp-contract=fast"]
        base = precision[:-3]
    else:
        base = precision
    if defines_function(src, "calc_jacobian"):
        extra.append("-DORACLE_HAS_JACOBIAN")
    if defines_function(src, "sode_system_stoch"):
        extra.append("-DORACLE_HAS_STOCH")
    if base == "fp32":
        extra.append("-DORACLE_FP32")
        body = "#define double float\n" + fp32_rewrite(src) + "\n#undef double\n"
    elif base == "fp64":
        body = src
    else:
        raise ValueError(precision)
    unit = '#include "oracle_prelude.h"\n#line 1 "%s"\n%s\n#include "oracle_solvers.h"\n' % (
        os.path.basename(system_path), body)
    return _compile(unit, os.path.join(out_dir, "liboracle_%s_%s.so" % (name, precision)), extra)


def build_reference(system: str, solver: int) -> str:
    """Compile the reference's kernels for (examples/<system>.cl, solver) with
    the host loop of ref_driver.c into oracle/_ref/libref_<system>_<solver>.so."""
    kdir = os.path.join(REFERENCE_ROOT, "src", "kernels")
    parts = ['#include "ref_shim.h"\n']
    if solver == 0:
        # src/sodeclmgr.cpp:381-390
        parts.append("#define R123_USE_U01_DOUBLE 1\n#include <Random123/threefry.h>\n#include <Random123/u01.h>\n")
    parts.append(open(os.path.join(REFERENCE_ROOT, "examples", system + ".cl")).read() + "\n")
    parts.append(open(os.path.join(kdir, REF_SOLVER_FILES[solver])).read() + "\n")
    caller = "stochastic_solver_caller.cl" if solver == 0 else "solver_caller.cl"
    parts.append(open(os.path.join(kdir, caller)).read() + "\n")
    parts.append('#include "ref_driver.c"\n')
    extra = ["-I", os.path.join(REFERENCE_ROOT, "external", "include")]
    if solver == 0:
        extra.append("-DREF_STOCHASTIC")
    target = os.path.join(REF_DIR, "libref_%s_%s.so" % (system, REF_SOLVER_NAMES[solver]))
    return _compile("".join(parts), target, extra)


def build_reference_threefry() -> str:
    """The reference's vendored Threefry/u01 headers behind ref_threefry.c."""
    extra = ["-I", os.path.join(REFERENCE_ROOT, "external", "include")]
    src = open(os.path.join(HERE, "ref_threefry.c")).read()
    return _compile(src, os.path.join(REF_DIR, "libref_threefry.so"), extra)


# (system, solver) pairs of the reference that compile: Kuramoto ships no
# calc_jacobian, so only the explicit and stochastic solvers exist for it.
REFERENCE_BUILDS = [("oculomotor", s) for s in (0, 1, 2, 3, 4)] + [("kuramoto", s) for s in (0, 1, 2)]


def reference_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "src", "kernels"))


def stage_reference_inputs() -> list[str]:
    """Copy STAGED_FILES from the reference checkout to baseline/_ref,
    byte for byte (rewritten only when they differ)."""
    out = []
    for rel in STAGED_FILES:
        src = os.path.join(REFERENCE_ROOT, rel)
        dst = os.path.join(STAGED_ROOT, rel)
        data = open(src, "rb").read()
        if not os.path.exists(dst) or open(dst, "rb").read() != data:
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(dst, "wb") as f:
                f.write(data)
        out.append(dst)
    return out


def build_all(verbose: bool = False) -> list[str]:
    built = []
    for fname in sorted(os.listdir(SYSTEMS_DIR)):
        if fname.endswith(".cl"):
            for prec in ("fp64", "fp32") + (("fp64fma", "fp32fma") if cpu_has_fma() else ()):
                built.append(build_restatement(os.path.join(SYSTEMS_DIR, fname), fname[:-3], prec))
    if reference_available():
        built += stage_reference_inputs()
        for system, solver in REFERENCE_BUILDS:
            built.append(build_reference(system, solver))
        built.append(build_reference_threefry())
        # the reference's own example system files through the restatement,
        # to show the package's system files are faithful restatements
        # (with FMA contraction too: the noise floor of parity runs on them)
        for system in ("oculomotor", "kuramoto"):
            for prec in ("fp64",) + (("fp64fma",) if cpu_has_fma() else ()):
                built.append(build_restatement(os.path.join(REFERENCE_ROOT, "examples", system + ".cl"),
                                               "refsys_" + system, prec, out_dir=REF_DIR))
    if verbose:
        for b in built:
            print("built", os.path.relpath(b, REPO))
    return built


if __name__ == "__main__":
    build_all(verbose=True)
    sys.exit(0)
