"""The iterNLM command line end to end on the GPU: TIFF slices in, the
reference driver's schedule (main.cpp:311-545) through the C++ shim and the
C ABI, TIFF slices and noise files out; results checked bit for bit against
the oracle (manual sigma) and against the library's own whole-job call
(estimated sigma)."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth, tiffio
from oracle.oracle import FilterParams

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "microtomodenoise_b200", "lib", "iterNLM")


def _cli(*args):
    r = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture()
def stack(tmp_path):
    vol = synth.spheres_volume((12, 40, 48), n_spheres=6, rmin=3, rmax=9, seed=4)
    tiffio.save_stack(vol, str(tmp_path / "in"), "slice")
    return vol, tmp_path


def test_cli_manual_sigma_matches_oracle(gpu, port, stack):
    vol, tmp = stack
    out = tmp / "out"
    log = _cli("-i", tmp / "in", "-o", out, "-iter", 2, "-search", 3, "-patch", 1, "-noise", "manual",
               "-sigma0", 0.05, "-sigma1", 0.03, "-alpha", 0.5)
    assert "iteration 2 took" in log
    it1 = tiffio.read_stack(str(out / "denoise-iteration01"))
    it2 = tiffio.read_stack(str(out / "denoise-iteration02"))
    p = FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))
    s0 = np.full(12, 0.05, np.float32)
    blend = (np.float32(0.5) * s0 + np.float32(0.5) * np.full(12, 0.03, np.float32)).astype(np.float32)
    assert np.array_equal(it1, port.denoise_f32(vol, p, s0[None]))
    assert np.array_equal(it2, port.denoise_f32(vol, p, np.stack([s0, blend])))
    # noise files: "n,value" per slice
    rows = (out / "noise_vs_slice00.csv").read_text().splitlines()
    assert len(rows) == 12 and rows[0] == "0,0.05"
    assert os.path.exists(tmp / "logfile.txt")


def test_cli_estimated_noise_equals_library_whole_job(gpu, stack):
    vol, tmp = stack
    out = tmp / "out"
    _cli("-i", tmp / "in", "-o", out, "-iter", 3, "-search", 3, "-patch", 2, "-noise", "global",
         "-nsamples", 20000, "-seed", 5)
    got = tiffio.read_stack(str(out / "denoise-iteration03"))
    dp = DenoiseParameters(radius_searchspace=(3, 3, 3), radius_patchspace=(2, 2, 2),
                           noise_mode="global", n_samples=20000, noise_seed=5, maxiterations=3)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, dp)
    want, s0, s1 = g.denoise(vol)
    g.free_device()
    assert np.array_equal(got, want)
    csv0 = np.array([float(r.split(",")[1]) for r in (out / "noise_vs_slice00.csv").read_text().split()])
    assert np.allclose(csv0, s0, rtol=1e-5)


def test_cli_16bit_cleanup_and_slice_range(gpu, port, tmp_path):
    vol = synth.spheres_volume((10, 32, 36), n_spheres=5, rmin=3, rmax=8, seed=6) * 1000.0
    tiffio.save_stack(vol.astype(np.float32), str(tmp_path / "in"), "s")
    out = tmp_path / "out"
    _cli("-i", tmp_path / "in", "-o", out, "-iter", 2, "-search", 2, "-patch", 1, "-noise", "manual",
         "-sigma", 40, "-fs", 2, "-ls", 6, "--16bit", "--cleanup")
    names = sorted(n for n in os.listdir(out) if n.endswith(".tif"))
    assert names == [f"denoised{z:04d}.tif" for z in range(2, 7)]
    assert not any(n.startswith("denoise-iteration") for n in os.listdir(out))
    got = tiffio.read_stack(str(out))
    sub = vol[2:7].astype(np.float32)
    p = FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1))
    s = np.full(5, 40, np.float32)
    want = port.denoise_f32(sub, p, np.stack([s, s]))
    r = np.trunc(want.astype(np.float64) + np.copysign(0.5, want))
    assert np.array_equal(got, np.clip(r, 0, 65535).astype(np.float32))


def test_cli_resume_reads_finished_iterations(gpu, stack):
    vol, tmp = stack
    out = tmp / "out"
    args = ["-i", tmp / "in", "-o", out, "-iter", 3, "-search", 3, "-patch", 1, "-noise", "global",
            "-nsamples", 20000, "-seed", 9]
    _cli(*args)
    full = tiffio.read_stack(str(out / "denoise-iteration03"))
    shutil.rmtree(out / "denoise-iteration03")
    log = _cli(*args, "--resume")
    assert "iteration 1 read in from disk" in log and "iteration 2 read in from disk" in log
    assert "Read in noise level 0 from file" in log and "Read in noise level 1 from file" in log
    assert "iteration 3 took" in log
    got = tiffio.read_stack(str(out / "denoise-iteration03"))
    # a resumed run continues from the saved iterations and from the noise
    # files, whose six significant digits (hdcommunication.cpp:1736-1746)
    # round sigma: rebuild that continuation through the library
    csv = lambda k: np.array([float(r.split(",")[1]) for r in
                              (out / f"noise_vs_slice{k:02d}.csv").read_text().split()], np.float32)
    s0c, s1c = csv(0), csv(1)
    blend = (np.float32(0.5) * s0c + np.float32(0.5) * s1c).astype(np.float32)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_searchspace=(3, 3, 3),
                                                    radius_patchspace=(1, 1, 1)))
    g.set_sigma(blend)
    g.set_result(1, tiffio.read_stack(str(out / "denoise-iteration01")), vol)
    g.set_result(2, tiffio.read_stack(str(out / "denoise-iteration02")))
    g.Run_GaussianNoise(3)
    want = g.get_result()
    g.free_device()
    assert np.array_equal(got, want)
    assert np.max(np.abs(got - full)) < 1e-4  # and close to the uninterrupted run


def test_cli_fp16_form(gpu, stack):
    """-precision f16 runs the FP16 storage form: the same result as the
    library's FP16 form called directly (its accuracy is covered by the FP16
    tests against the FP64 oracle)."""
    vol, tmp = stack
    out = tmp / "out"
    _cli("-i", tmp / "in", "-o", out, "-iter", 2, "-search", 3, "-patch", 2, "-noise", "manual",
         "-sigma", 0.05, "-precision", "f16")
    got = tiffio.read_stack(str(out / "denoise-iteration02"))
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_searchspace=(3, 3, 3),
                                                    radius_patchspace=(2, 2, 2), precision="f16"))
    s = np.full(12, 0.05, np.float32)
    g.set_sigma(s)
    g.Run_GaussianNoise(1, vol)
    g.Run_GaussianNoise(2)
    want = g.get_result()
    g.free_device()
    assert np.array_equal(got, want)


def _iterations(out, n):
    return [tiffio.read_stack(str(out / f"denoise-iteration{k:02d}")) for k in range(1, n + 1)]


def _noise_files(out):
    return {n: (out / n).read_text() for n in sorted(os.listdir(out)) if n.startswith("noise_vs_slice")}


@pytest.mark.parametrize("split", [["-gpulist", "0,0"], ["-slab", 16]], ids=["two_parts", "z_slabs"])
def test_cli_blocks_save_every_iteration(gpu, tmp_path, split):
    """The stack split over two parts (-gpulist 0,0: the multi-GPU path on one
    device) or streamed through one device in z-slabs of 16 slices (-slab 16)
    runs the host-RAM blocks per iteration (Run_GaussianNoise_GPUBlocks,
    main.cpp:377-384, 471-478): every iteration folder and every noise file,
    --continuous included, equals the single-GPU run's."""
    vol = synth.spheres_volume((40, 32, 36), n_spheres=8, rmin=3, rmax=8, seed=2)
    tmp = tmp_path
    tiffio.save_stack(vol, str(tmp / "in"), "slice")
    args = ["-i", tmp / "in", "-iter", 4, "-search", 3, "-patch", 1, "-noise", "z-adaptive",
            "-nsamples", 20000, "-seed", 5, "--continuous"]
    _cli(*args, "-o", tmp / "one", "-gpus", 1)
    log = _cli(*args, "-o", tmp / "two", *split)
    assert ("on 2 GPUs" in log) if split[0] == "-gpulist" else ("Streaming z-slabs of 16" in log)
    for k, (a, b) in enumerate(zip(_iterations(tmp / "one", 4), _iterations(tmp / "two", 4))):
        assert np.array_equal(a, b), f"iteration {k + 1}"
    assert _noise_files(tmp / "one") == _noise_files(tmp / "two")
    assert len(_noise_files(tmp / "one")) == 3  # sigma0, sigma1 and the --continuous estimate before iteration 4


@pytest.mark.parametrize("split", [["-slab", 16], ["-gpulist", "0,0"]], ids=["z_slabs", "two_parts"])
def test_cli_blocks_match_oracle_and_resume(gpu, port, tmp_path, split):
    """Host-RAM blocks at patch radius 3, search radius 7: z-slabs of 16
    slices through one device, or two parts (slices 0-23 and 24-39, halos of
    8): every iteration bit-exact against the oracle (manual sigma); a
    --resume run continues from the saved iterations."""
    vol = synth.spheres_volume((40, 30, 34), n_spheres=8, rmin=3, rmax=8, seed=12)
    tiffio.save_stack(vol, str(tmp_path / "in"), "slice")
    args = ["-i", tmp_path / "in", "-o", tmp_path / "out", "-iter", 3, "-search", 7, "-patch", 3,
            "-noise", "manual", "-sigma0", 0.05, "-sigma1", 0.03, *split]
    _cli(*args)
    got = _iterations(tmp_path / "out", 3)
    p = FilterParams(search_radius=(7, 7, 7), patch_radius=(3, 3, 3))
    s0 = np.full(40, 0.05, np.float32)
    blend = (np.float32(0.5) * s0 + np.float32(0.5) * np.full(40, 0.03, np.float32)).astype(np.float32)
    want = port.denoise_f32(vol, p, np.stack([s0, blend, blend]), all_iters=True)
    for k in range(3):
        assert np.array_equal(got[k], want[k]), f"iteration {k + 1}"
    shutil.rmtree(tmp_path / "out" / "denoise-iteration03")
    log = _cli(*args, "--resume")
    assert "iteration 2 read in from disk" in log
    assert np.array_equal(_iterations(tmp_path / "out", 3)[2], want[2])


REFDRIVER = os.path.join(ROOT, "oracle", "_ref", "iterNLM_refdriver")


@pytest.mark.skipif(not os.path.exists(REFDRIVER), reason="reference driver not built (needs the reference tree)")
def test_reference_driver_runs_on_this_library(gpu, port, stack):
    """The reference's own main.cpp, unmodified, compiled against this
    library's C++ shim (oracle/Makefile refdriver): its whole-stack GPU flow
    (configure_device, set_sigma, Run_GaussianNoise, get_result, the TIFF
    saves) runs on this library, bit-exact against the oracle."""
    vol, tmp = stack
    out = tmp / "out"
    r = subprocess.run([REFDRIVER, "-i", str(tmp / "in"), "-o", str(out), "-iter", "2", "-search", "3",
                        "-patch", "1", "-noise", "manual", "-sigma0", "0.05", "-sigma1", "0.03"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    p = FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))
    s0 = np.full(12, 0.05, np.float32)
    blend = (np.float32(0.5) * s0 + np.float32(0.5) * np.full(12, 0.03, np.float32)).astype(np.float32)
    want = port.denoise_f32(vol, p, np.stack([s0, blend]), all_iters=True)
    got = _iterations(out, 2)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
