"""The parity measure shared by the GPU tests.

Error measure: per element, |got - want| / (|want| + 1e-3 * S_e), S_e the
largest |value| of equation e in the run (axis 1 of a [record][equation]
[orbit] array), so values crossing zero are measured against their
equation's scale; NaN/Inf positions must agree.

Tolerance: max(rtol, 10 x the oracle's own noise floor), the floor being the
same measure between two CPU builds of the same computation (with and
without FMA contraction) on the same inputs.  Last-bit differences (CUDA's
exp/log/sin/cos against glibc's, FMA contraction) are all the GPU adds; how
far they travel is a property of the dynamics."""
import numpy as np

RTOL = 1e-12


def rel_error(got, want):
    """(max error over elements finite in both, count of NaN/Inf mismatches)."""
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    fin_w, fin_g = np.isfinite(want), np.isfinite(got)
    both = fin_w & fin_g
    axes = tuple(i for i in range(want.ndim) if i != 1)
    scale = np.max(np.where(fin_w, np.abs(want), 0.0), axis=axes, keepdims=True)
    den = np.abs(want) + 1e-3 * scale + 1e-300
    err = np.where(both, np.abs(np.where(both, got, 0) - np.where(both, want, 0)) / den, 0.0)
    return float(err.max()) if err.size else 0.0, int(np.count_nonzero(fin_w != fin_g))


def assert_parity(label, got, want, alt, rtol=RTOL):
    """got vs want within max(rtol, 10 x floor), floor = distance of `alt`
    (a second CPU build) from `want`."""
    floor, floor_nan = rel_error(alt, want)
    err, nan_mismatch = rel_error(got, want)
    tol = max(rtol, 10 * floor)
    print("%s: error %.3g (floor %.3g, tolerance %.3g), NaN mismatches %d (floor %d)"
          % (label, err, floor, tol, nan_mismatch, floor_nan))
    assert err <= tol
    assert nan_mismatch <= 10 * floor_nan
    return err
