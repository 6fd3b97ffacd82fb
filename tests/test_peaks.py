"""The measured ceilings the bench reports its roofline fractions against:
the FMA issue rate of the FP64 / FP32 pipes (sodecl_cuda_fma_peak) and the
throughput of the math library's sin (sodecl_cuda_sin_peak).  The checks are
sanity bounds: each rate is positive and plausible for one B200, FP32 beats
FP64, and a sine costs many FMAs."""
import pytest

from sodecl_b200 import _native as N


@pytest.mark.gpu
def test_fma_and_sin_peaks_are_plausible():
    import sodecl_b200

    if N.device_count() < 1:
        pytest.fail("no CUDA device")
    fma64, ms64 = sodecl_b200.fma_peak("fp64")
    fma32, _ = sodecl_b200.fma_peak("fp32")
    sin64, sms64 = sodecl_b200.sin_peak("fp64")
    sin32, _ = sodecl_b200.sin_peak("fp32")
    print("FMA/s fp64 %.3e fp32 %.3e; sin/s fp64 %.3e fp32 %.3e" % (fma64, fma32, sin64, sin32))
    # 148 SMs x 64 FP64 FMA per clock x ~2 GHz is 1.9e13
    assert 1e12 < fma64 < 3e13 and ms64 > 0
    assert fma32 > 2 * fma64
    # a double sine is a range reduction and a polynomial: dozens of instructions
    assert 1e10 < sin64 < fma64 / 8 and sms64 > 0
    assert sin32 > sin64
