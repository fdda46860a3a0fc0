"""The colour path on the GPU (inlm_rgb_denoise, the --color CLI) against the
reference's own colour job (tests/golden/rgb_small.npz, from oracle/_ref):
bit for bit with manual sigma (every saved iteration too), and within the
noise estimator's tolerance (FP64 EM sums, sigma <= 2e-5 relative) with
estimated sigma."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, color

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)
from make_golden import RGB_CASES  # noqa: E402

CLI = os.path.join(os.path.dirname(HERE), "microtomodenoise_b200", "lib", "iterNLM")


@pytest.fixture(scope="module")
def golden_rgb():
    return np.load(os.path.join(GOLDEN, "rgb_small.npz"))


def run_case(img, name):
    sr, pr, iters, mode, sig, indep, stab, avg, cont, keep = RGB_CASES[name]
    dp = DenoiseParameters(radius_searchspace=(sr[0], sr[1], 0), radius_patchspace=(pr[0], pr[1], 0),
                           nslices=1, maxiterations=iters, noise_mode=mode, sigma=sig, n_samples=2048,
                           noise_seed=3, continuous_estimate=cont)
    cp = color.ColorParameters(stabilize_variance=stab, independent_channels=indep,
                               average_channelsigma=avg)
    saved = []
    cb = (lambda it, planes: saved.append((it, np.stack(planes)))) if keep else None
    out, s_first, s_last = color.rgb_denoise(img, dp, cp, cb)
    return np.stack(out), saved, s_first, s_last


@pytest.mark.parametrize("name", ["manual_joint", "manual_indep_raw"])
def test_rgb_manual_sigma_bit_exact(gpu, golden_rgb, name):
    out, saved, s_first, s_last = run_case(list(golden_rgb["image"]), name)
    assert np.array_equal(s_first, golden_rgb[name + "/sigma_first"])
    assert np.array_equal(s_last, golden_rgb[name + "/sigma_last"])
    assert np.array_equal(out, golden_rgb[name + "/final"]), float(np.abs(out - golden_rgb[name + "/final"]).max())
    if RGB_CASES[name][-1]:
        assert [it for it, _ in saved] == list(range(1, RGB_CASES[name][2] + 1))
        assert np.array_equal(np.stack([p for _, p in saved]), golden_rgb[name + "/iterations"])


@pytest.mark.parametrize("name", ["global_joint", "global_noavg_cont", "semimanual"])
def test_rgb_estimated_sigma(gpu, golden_rgb, name):
    out, saved, s_first, s_last = run_case(list(golden_rgb["image"]), name)
    for got, key in ((s_first, "/sigma_first"), (s_last, "/sigma_last")):
        want = golden_rgb[name + key]
        assert np.max(np.abs(got / want - 1)) <= 2e-5, (key, got, want)
    ref = golden_rgb[name + "/final"]
    err = np.abs(out - ref)
    print(name, "max abs", err.max(), "mean", err.mean())
    assert err.max() <= 0.02 and err.mean() <= 1e-3


def test_cli_color(gpu, golden_rgb, tmp_path):
    PIL = pytest.importorskip("PIL.Image")
    img = golden_rgb["image"]
    (tmp_path / "in").mkdir()
    PIL.fromarray(np.moveaxis(img, 0, -1).astype(np.uint8)).save(tmp_path / "in" / "photo.tif")
    out = tmp_path / "out"
    r = subprocess.run([CLI, "-i", str(tmp_path / "in"), "-o", str(out), "--color", "-iter", "3",
                        "-search", "4", "-patch", "1", "-noise", "manual", "-sigma0", "1.2",
                        "-sigma1", "0.9"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    to8 = lambda a: np.where(np.where(a < 255, a, 255) > 0, np.where(a < 255, a, 255), 0).astype(np.uint8)
    got = np.array(PIL.open(out / "photo_denoised.tif"))
    assert np.array_equal(got, np.moveaxis(to8(golden_rgb["manual_joint/final"]), 0, -1))
    for it in range(1, 4):
        got = np.array(PIL.open(out / "denoise_iterations" / f"photo_iter{it:02d}.tif"))
        want = to8(golden_rgb["manual_joint/iterations"][it - 1])
        assert np.array_equal(got, np.moveaxis(want, 0, -1))
