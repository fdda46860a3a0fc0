"""One stack split in z over several GPUs of one process (inlm_denoise_multi,
the reference's n_gpus block mode): the owned slices, sigma0 and sigma1 must
equal the single-GPU whole job (inlm_denoise) bit for bit. Parts may share a
device, so one B200 runs two and three parts; with more GPUs the parts go to
different devices and the halos cross NVLink."""
import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, denoise_multi, synth

pytestmark = pytest.mark.gpu


def single(raw, p):
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, p)
    out, s0, s1 = g.denoise(raw)
    g.free_device()
    return out, s0, s1


def device_count():
    import ctypes
    n = ctypes.c_int(0)
    ctypes.CDLL("libcudart.so").cudaGetDeviceCount(ctypes.byref(n))
    return n.value


@pytest.mark.parametrize("mode,prec,parts", [("z-adaptive", "f32", 2), ("global", "f16", 3),
                                             ("manual", "f32", 2), ("global", "f32_fma", 2)])
def test_multi_equals_single(gpu, mode, prec, parts):
    raw = synth.small_case((48, 40, 56), seed=13)
    p = DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3), noise_mode=mode,
                          zwindow=10, sigma=(0.06, 0.05), noise_seed=4, n_samples=20000, precision=prec)
    want, w0, w1 = single(raw, p)
    ndev = device_count()
    ids = [i % ndev for i in range(parts)] if ndev > 1 else [0] * parts
    got, s0, s1 = denoise_multi(raw, p, ids)
    assert np.array_equal(s0, w0) and np.array_equal(s1, w1)
    assert np.array_equal(got, want), float(np.abs(got - want).max())


def test_multi_continuous_and_single_part(gpu):
    raw = synth.small_case((40, 36, 44), seed=3)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(2, 2, 2), noise_mode="global",
                          continuous_estimate=True, maxiterations=4, noise_seed=7, n_samples=20000)
    want, _, _ = single(raw, p)
    for ids in ([0], [0, 0, 0]):
        got, _, _ = denoise_multi(raw, p, ids)
        assert np.array_equal(got, want)


def test_multi_rejects_thin_slabs(gpu):
    from microtomodenoise_b200 import InlmError
    raw = synth.small_case((16, 24, 24), seed=1)
    p = DenoiseParameters(radius_patchspace=(3, 3, 3), radius_searchspace=(7, 7, 7), nslices=21,
                          noise_mode="manual", sigma=(0.05, 0.05))
    with pytest.raises(InlmError, match="halo"):
        denoise_multi(raw, p, [0, 0])
