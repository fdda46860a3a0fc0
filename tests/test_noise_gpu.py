"""GPU noise estimators against the reference (golden fixtures) and the oracle.

* sample positions: bit-exact (glibc rand() sequence),
* per-sample 15x15 patch std: bit-exact,
* sigma: the device EM accumulates in FP64 (the reference in float), so it is
  held to 1e-6 relative of the oracle's FP64-accumulating restatement and to
  2e-5 relative of the reference's own float result.
"""
import os
import sys

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, NoiseLevel, synth
from oracle.oracle import FilterParams

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["global", "z-adaptive"])
@pytest.mark.parametrize("mask", [0, 60])
def test_noise_vs_reference_golden(gpu, port, golden_noise, mode, mask):
    import make_golden
    vol = make_golden.noise_volume()
    key = f"{mode}_m{mask}"
    nl = NoiseLevel(20000, 15, vol.shape, seed=7)
    dp = DenoiseParameters(noise_mode=mode, zwindow=20, circular_mask_diameter=mask)
    s1 = nl.get_noiselevel(vol, dp)
    samples = nl.samples()
    assert np.array_equal(samples, golden_noise[key + "_samples"].astype(np.int64))
    ps = nl.patchstd()
    assert np.array_equal(ps, golden_noise[key + "_patchstd"])
    o64 = port.noise_from_patchstd(ps, samples, vol.shape, mode, zwindow=20, f64acc=True)
    assert np.max(np.abs(s1 / o64 - 1)) <= 1e-6
    assert np.max(np.abs(s1 / golden_noise[key + "_sigma1"] - 1)) <= 2e-5
    # second call reuses the samples (NoiseLevel::samples cache)
    vol2 = vol * np.float32(0.8)
    s2 = nl.get_noiselevel(vol2, dp)
    assert np.array_equal(nl.samples(), samples)
    assert np.max(np.abs(s2 / golden_noise[key + "_sigma2"] - 1)) <= 2e-5
    nl.close()


def test_manual_and_semimanual_modes(gpu, port):
    vol = synth.small_case((10, 40, 48), seed=2)
    nl = NoiseLevel(5000, 15, vol.shape, seed=3)
    dp = DenoiseParameters(noise_mode="manual", sigma=(0.07, 0.03))
    assert np.all(nl.get_noiselevel(vol, dp) == np.float32(0.07))
    assert np.all(nl.get_noiselevel(vol, dp) == np.float32(0.03))
    nl.close()
    nl = NoiseLevel(5000, 15, vol.shape, seed=3)
    dp = DenoiseParameters(noise_mode="semimanual", sigma=(0.05, 0.0))
    s = nl.get_noiselevel(vol, dp)
    assert np.all(s == np.float32(0.05))
    ps = nl.patchstd()
    ref_i = int(np.argmin(np.abs(ps - np.float32(0.05))))
    vol2 = vol * np.float32(0.5)
    s2 = nl.get_noiselevel(vol2, dp)
    ps2 = port.patchstd(vol2, nl.samples())
    assert np.all(s2 == ps2[ref_i]) and dp.sigma[1] == pytest.approx(float(ps2[ref_i]))
    nl.close()


def test_noise_on_device_pointer(gpu, port):
    torch = pytest.importorskip("torch")
    vol = synth.small_case((24, 48, 56), seed=5)
    nl = NoiseLevel(8000, 15, vol.shape, seed=1)
    dp = DenoiseParameters(noise_mode="z-adaptive", zwindow=10)
    t = torch.from_numpy(vol).cuda()
    torch.cuda.synchronize()
    s = nl.get_noiselevel(t.data_ptr(), dp, on_device=True)
    samples = port.draw_samples(vol.shape, 8000, 15, 0, 1)
    o = port.noise_from_patchstd(port.patchstd(vol, samples), samples, vol.shape, "z-adaptive",
                                 zwindow=10, f64acc=True)
    assert np.max(np.abs(s / o - 1)) <= 1e-6
    nl.close()


def test_whole_job_schedule(gpu, port):
    """denoise(): sigma0 on raw, iteration 1, sigma1 on its output, blend,
    iterations 2..4, all on the device; each step checked against the oracle."""
    vol = synth.spheres_volume((24, 64, 64), n_spheres=8, rmin=3, rmax=10, seed=2)
    dp = DenoiseParameters(radius_searchspace=(3, 3, 3), radius_patchspace=(1, 1, 1),
                           noise_mode="global", n_samples=20000, noise_seed=5, maxiterations=4)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, dp)
    out, s0, s1 = g.denoise(vol)
    g.free_device()
    samples = port.draw_samples(vol.shape, 20000, 15, 0, 5)
    o_s0 = port.noise_from_patchstd(port.patchstd(vol, samples), samples, vol.shape, "global",
                                    f64acc=True)
    assert np.max(np.abs(s0 / o_s0 - 1)) <= 1e-6
    p = FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))
    it1 = port.denoise_f32(vol, p, s0[None])
    o_s1 = port.noise_from_patchstd(port.patchstd(it1, samples), samples, vol.shape, "global",
                                    f64acc=True)
    assert np.max(np.abs(s1 / o_s1 - 1)) <= 1e-6
    blend = (np.float32(0.5) * s0 + (np.float32(1) - np.float32(0.5)) * s1).astype(np.float32)
    want = port.denoise_f32(vol, p, np.stack([s0, blend, blend, blend]))
    assert np.array_equal(out, want)
