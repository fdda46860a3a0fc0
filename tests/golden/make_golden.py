"""Generates the golden fixtures in tests/golden/ from the reference's own CPU
code (oracle/_ref/libiternlm_ref.so, compiled from the unmodified reference
sources by `make -C oracle ref`).

    python tests/golden/make_golden.py

Fixtures:
  filter_small.npz   a 24x20x16 seeded volume, 3 iterations of the reference
                     CPU filter for every specialised patch shape, generic
                     shapes, z anisotropy; every iterate stored.
  noise_small.npz    a 72x64x40 two-phase volume: glibc-rand sample positions
                     (seed 7), per-sample patch std, and sigma for global and
                     z-adaptive modes (with and without a circular mask),
                     first and second call.
  tables.npz         search offsets, patch offsets and distance weights of
                     the reference for several radii.
  config1.json       the 128x128x64 spheres workload (p1, s5, 4 iterations,
                     global noise): reference sigma0/sigma1, sha256 of every
                     iterate and 256 sampled voxels per iterate.
  rgb_small.npz      the colour path (color_denoising.h) on a seeded 48x64 RGB
                     image: final and per-iteration planes and both sigma
                     triples for the cases in RGB_CASES.

    python tests/golden/make_golden.py rgb     # only rgb_small.npz
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import FilterParams, Reference  # noqa: E402
from microtomodenoise_b200 import synth  # noqa: E402

sys.path.insert(0, HERE)
from cases import FILTER_CASES, TABLE_CASES  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small_filter_volume() -> np.ndarray:
    return synth.small_case((16, 20, 24), seed=3)


def noise_volume() -> np.ndarray:
    rng = np.random.default_rng(11)
    vol = (rng.standard_normal((40, 64, 72)).astype(np.float32) * np.float32(0.05) + np.float32(0.5))
    vol[:, :30, :] += np.float32(0.3)
    vol[5:9] *= np.float32(1.3)   # a few slices with a different noise level
    return vol


def config1_volume() -> np.ndarray:
    return synth.spheres_volume((64, 128, 128), n_spheres=40, rmin=4, rmax=20,
                                phases=(0.2, 0.5, 0.8), background=0.5, noise_std=0.05,
                                noise_blur=1.0, seed=0)


def rgb_image() -> list:
    """A seeded 8-bit RGB test image: smooth colour gradients, a few disks and
    Poisson counts, as three float planes."""
    rng = np.random.default_rng(5)
    ny, nx = 48, 64
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float32)
    base = [40 + 2.0 * x, 60 + 3.0 * y, 120 + 40 * np.sin(x / 9.0) * np.cos(y / 7.0)]
    for cy, cx, r, v in ((14, 18, 7, 200.0), (30, 44, 9, 30.0), (36, 12, 5, 150.0)):
        m = (y - cy) ** 2 + (x - cx) ** 2 <= r * r
        for c in range(3):
            base[c] = np.where(m, v - 40 * c, base[c])
    return [np.clip(rng.poisson(np.clip(b, 1, 250)), 0, 255).astype(np.float32) for b in base]


# name: (search xy, patch xy, iterations, mode, sigma, independent, stabilize, average,
#        continuous, keep_iterations)
RGB_CASES = {
    "manual_joint": ((4, 4), (1, 1), 3, "manual", (1.2, 0.9), False, True, True, False, True),
    "manual_indep_raw": ((3, 5), (2, 1), 2, "manual", (18.0, 12.0), True, False, True, False, False),
    "global_joint": ((5, 5), (1, 1), 3, "global", (0.0, 0.0), False, True, True, False, True),
    "global_noavg_cont": ((4, 4), (2, 2), 4, "global", (0.0, 0.0), False, True, False, True, False),
    "semimanual": ((4, 4), (1, 1), 3, "semimanual", (1.0, 0.0), False, True, True, False, True),
}


def make_rgb(ref) -> None:
    img = rgb_image()
    out = {"image": np.stack(img)}
    for name, (sr, pr, iters, mode, sig, indep, stab, avg, cont, keep) in RGB_CASES.items():
        p = FilterParams(search_radius=(sr[0], sr[1], 0), patch_radius=(pr[0], pr[1], 0), nslices=1)
        fin, its, s_first, s_last = ref.rgb_job(img, p, maxiterations=iters, mode=mode, sigma=sig,
                                                seed=3, stabilize=stab, independent=indep,
                                                average=avg, continuous=cont, keep_iterations=keep)
        out[name + "/final"] = np.stack(fin)
        if its is not None:
            out[name + "/iterations"] = its
        out[name + "/sigma_first"] = s_first
        out[name + "/sigma_last"] = s_last
    np.savez_compressed(os.path.join(HERE, "rgb_small.npz"), **out)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "rgb":
        make_rgb(Reference())
        print("rgb_small.npz written to", HERE)
        return
    ref = Reference()
    # ---- filter ----
    raw = small_filter_volume()
    nz = raw.shape[0]
    sig = np.empty((3, nz), np.float32)
    sig[0] = 0.06
    sig[1] = np.linspace(0.04, 0.07, nz, dtype=np.float32)
    sig[2] = sig[1] * np.float32(0.9)
    out = {"raw": raw, "sigmas": sig}
    for name, pr, sr, nsl, an in FILTER_CASES:
        p = FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl, z_anisotropy=an)
        res, _ = ref.denoise(raw, p, sig, n_threads=4, all_iters=True)
        out[name] = res
    np.savez_compressed(os.path.join(HERE, "filter_small.npz"), **out)

    # ---- noise ----
    vol = noise_volume()
    nres = {"vol_sha": np.array(sha(vol))}
    for mode in ("global", "z-adaptive"):
        for mask in (0, 60):
            s = ref.noise_session(vol.shape, n_samples=20000, patchsize=15, seed=7)
            s1 = s.estimate(vol, mode=mode, zwindow=20, mask=mask)
            samp = s.samples()
            s2 = s.estimate(vol * np.float32(0.8), mode=mode, zwindow=20, mask=mask)
            key = f"{mode}_m{mask}"
            nres[key + "_sigma1"] = s1
            nres[key + "_sigma2"] = s2
            nres[key + "_samples"] = samp.astype(np.int32)
            nres[key + "_patchstd"] = ref.patchstd(vol, samp)
            s.close()
    np.savez_compressed(os.path.join(HERE, "noise_small.npz"), **nres)

    # ---- tables ----
    tabs = {}
    for i, (pr, sr, nsl) in enumerate(TABLE_CASES):
        p = FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl)
        pad = (sr[0] + pr[0], sr[1] + pr[1], min(nsl // 2, sr[2]) + pr[2])
        ps = (40 + 2 * pad[0], 30 + 2 * pad[1], 20 + 2 * pad[2])
        s, q, w = ref.tables(p, ps)
        tabs[f"c{i}_params"] = np.array(list(pr) + list(sr) + [nsl] + list(ps), np.int32)
        tabs[f"c{i}_search"] = s
        tabs[f"c{i}_patch"] = q
        tabs[f"c{i}_weights"] = w
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **tabs)

    # ---- config 1 ----
    vol = config1_volume()
    nzc = vol.shape[0]
    s = ref.noise_session(vol.shape, n_samples=100000, patchsize=15, seed=0)
    sigma0 = s.estimate(vol, mode="global")
    p = FilterParams(search_radius=(5, 5, 5), patch_radius=(1, 1, 1))
    it1, _ = ref.denoise(vol, p, sigma0[None, :], n_threads=8)
    sigma1_raw = s.estimate(it1, mode="global")
    alpha = np.float32(0.5)
    sigma1 = (alpha * sigma0 + (np.float32(1.0) - alpha) * sigma1_raw).astype(np.float32)
    sigmas = np.stack([sigma0, sigma1, sigma1, sigma1])
    allit, secs = ref.denoise(vol, p, sigmas, n_threads=8, all_iters=True)
    rng = np.random.default_rng(123)
    idx = rng.integers(0, vol.size, 256)
    cfg = {
        "shape_zyx": list(vol.shape),
        "input_sha256": sha(vol),
        "patch_radius": [1, 1, 1], "search_radius": [5, 5, 5], "iterations": 4, "alpha": 0.5,
        "noise": "global", "n_samples": 100000, "noise_seed": 0,
        "sigma0": [float(x) for x in sigma0], "sigma1_estimate": [float(x) for x in sigma1_raw],
        "sigma1": [float(x) for x in sigma1],
        "iterate_sha256": [sha(allit[i]) for i in range(4)],
        "sample_index": [int(i) for i in idx],
        "sample_values": [[float(allit[i].ravel()[j]) for j in idx] for i in range(4)],
        "reference_seconds_8threads": secs,
    }
    with open(os.path.join(HERE, "config1.json"), "w") as f:
        json.dump(cfg, f, indent=1)
    make_rgb(ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
