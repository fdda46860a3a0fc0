"""Seeded synthetic tomography volumes for tests and benchmarks.

The reference ships no dataset, so every workload here is generated from a
seed: spheres or a grain pack, correlated Gaussian noise, concentric z-axis
ring artefacts and a sigma drift along z. Volumes are float32 with shape
(nz, ny, nx), x fastest, as the reference stores image stacks
(iternlm_cpu.cpp:10-11).
"""
from __future__ import annotations

import numpy as np

try:  # scipy is in the image; the fallback keeps the module importable without it
    from scipy.ndimage import gaussian_filter as _gaussian_filter
except Exception:  # pragma: no cover
    _gaussian_filter = None


def gaussian_blur(vol: np.ndarray, sigma: float) -> np.ndarray:
    """Separable 3D Gaussian blur (reflective borders), float32."""
    if sigma <= 0:
        return vol.astype(np.float32, copy=True)
    if _gaussian_filter is not None:
        return _gaussian_filter(vol.astype(np.float32), sigma, mode="mirror", truncate=4.0)
    r = int(4 * sigma + 0.5)
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = vol.astype(np.float32)
    for ax in range(3):
        padw = [(0, 0)] * 3
        padw[ax] = (r, r)
        p = np.pad(out, padw, mode="reflect")
        acc = np.zeros_like(out)
        for i, kv in enumerate(k):
            sl = [slice(None)] * 3
            sl[ax] = slice(i, i + out.shape[ax])
            acc += np.float32(kv) * p[tuple(sl)]
        out = acc
    return out


def correlated_noise(shape, std: float, blur: float, rng: np.random.Generator) -> np.ndarray:
    """N(0, std^2) white noise, blurred, then rescaled back to the given std."""
    n = rng.standard_normal(shape, dtype=np.float32) * np.float32(std)
    if blur > 0:
        n = gaussian_blur(n, blur)
        s = float(n.std())
        if s > 0:
            n *= np.float32(std / s)
    return n


def _draw_sphere(vol, cz, cy, cx, r, value):
    nz, ny, nx = vol.shape
    z0, z1 = max(int(np.floor(cz - r)), 0), min(int(np.ceil(cz + r)) + 1, nz)
    y0, y1 = max(int(np.floor(cy - r)), 0), min(int(np.ceil(cy + r)) + 1, ny)
    x0, x1 = max(int(np.floor(cx - r)), 0), min(int(np.ceil(cx + r)) + 1, nx)
    if z0 >= z1 or y0 >= y1 or x0 >= x1:
        return
    zz, yy, xx = np.ogrid[z0:z1, y0:y1, x0:x1]
    m = (zz - cz) ** 2 + (yy - cy) ** 2 + (xx - cx) ** 2 <= r * r
    vol[z0:z1, y0:y1, x0:x1][m] = value


def spheres_volume(shape=(64, 128, 128), n_spheres=40, rmin=4.0, rmax=20.0,
                   phases=(0.2, 0.5, 0.8), background=0.5, noise_std=0.05, noise_blur=1.0,
                   seed=0) -> np.ndarray:
    """Random spheres on a background plus blurred Gaussian noise rescaled to
    ``noise_std`` (the 128x128x64 plain-filter workload uses the defaults)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    vol = np.full(shape, background, np.float32)
    for _ in range(n_spheres):
        r = rng.uniform(rmin, rmax)
        c = rng.uniform(0, 1, 3) * np.array([nz, ny, nx])
        _draw_sphere(vol, c[0], c[1], c[2], r, np.float32(rng.choice(phases)))
    vol += correlated_noise(shape, noise_std, noise_blur, rng)
    return vol


def grain_pack(shape, mu=np.log(12.0), sig=0.3, grain=0.7, pore=0.3, spacing_factor=1.9,
               rng=None) -> np.ndarray:
    """Dense pack of log-normal-radius spheres: centres on a cubic lattice of
    pitch ``spacing_factor`` x median radius, each jittered by up to a quarter
    pitch, radii drawn log-normal(mu, sig) and capped at 0.6 pitch (grains
    touch and overlap slightly, as in a close-packed grain pack)."""
    rng = rng if rng is not None else np.random.default_rng(0)
    nz, ny, nx = shape
    vol = np.full(shape, pore, np.float32)
    a = spacing_factor * float(np.exp(mu))
    gz, gy, gx = (np.arange(-0.5 * a, n + 0.5 * a, a) for n in shape)
    cz, cy, cx = np.meshgrid(gz, gy, gx, indexing="ij")
    cen = np.stack([cz.ravel(), cy.ravel(), cx.ravel()], 1)
    cen += rng.uniform(-0.25 * a, 0.25 * a, cen.shape)
    rad = np.minimum(rng.lognormal(mu, sig, len(cen)), 0.6 * a)
    for (c0, c1, c2), r in zip(cen, rad):
        _draw_sphere(vol, c0, c1, c2, r, np.float32(grain))
    return vol


def ring_artefacts(shape, amplitude, period) -> np.ndarray:
    """Concentric rings about the z axis through the slice centre."""
    nz, ny, nx = shape
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float32)
    rr = np.sqrt((yy - (ny - 1) / 2) ** 2 + (xx - (nx - 1) / 2) ** 2)
    ring = np.float32(amplitude) * np.sin(np.float32(2 * np.pi / period) * rr)
    return np.broadcast_to(ring.astype(np.float32), shape)


def to_uint16_unit(vol: np.ndarray) -> np.ndarray:
    """Quantise to uint16 over [0, 1] and scale back to float32."""
    q = np.clip(np.rint(np.clip(vol, 0.0, 1.0) * 65535.0), 0, 65535).astype(np.uint16)
    return (q.astype(np.float32) / np.float32(65535.0)).astype(np.float32)


def grain_pack_volume(shape=(512, 512, 512), noise_std=0.04, noise_blur=1.2, ring_amp=0.02,
                      ring_period=6.0, sigma_drift=None, seed=0, quantise=True,
                      return_clean=False):
    """Grain pack + correlated noise + ring artefacts (the 512^3 workload).

    sigma_drift=(s0, s1) makes the noise std drift linearly along z.
    return_clean=True also returns the noise- and ring-free phantom."""
    rng = np.random.default_rng(seed)
    vol = grain_pack(shape, rng=rng)
    clean = vol.copy() if return_clean else None
    if sigma_drift is None:
        vol += correlated_noise(shape, noise_std, noise_blur, rng)
    else:
        n = correlated_noise(shape, 1.0, noise_blur, rng)
        s = np.linspace(sigma_drift[0], sigma_drift[1], shape[0], dtype=np.float32)
        vol += n * s[:, None, None]
    if ring_amp:
        vol += ring_artefacts(shape, ring_amp, ring_period)
    out = to_uint16_unit(vol) if quantise else vol.astype(np.float32)
    if return_clean:
        return out, (to_uint16_unit(clean) if quantise else clean)
    return out


def small_case(shape=(16, 20, 24), seed=0, noise_std=0.05) -> np.ndarray:
    """Tiny spheres volume for unit tests (odd sizes welcome)."""
    nz, ny, nx = shape
    r = max(2.0, min(shape) / 4.0)
    return spheres_volume(shape, n_spheres=4, rmin=1.5, rmax=r, noise_std=noise_std,
                          noise_blur=1.0, seed=seed)


def rgb_photo(ny: int = 3072, nx: int = 4096, n_disks: int = 60, seed: int = 0):
    """A seeded 8-bit RGB test image: smooth colour gradients, random flat
    disks and Poisson (shot) noise on the counts, as three float32 (ny, nx)
    planes with integer values 0..255 (the colour path's input)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float32)
    base = [40 + 150 * x / nx, 60 + 120 * y / ny,
            120 + 50 * np.sin(x * (12.0 / nx)) * np.cos(y * (9.0 / ny))]
    for _ in range(n_disks):
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        r = rng.uniform(0.01, 0.06) * min(ny, nx)
        col = rng.uniform(10, 245, 3)
        y0, y1 = int(max(0, cy - r)), int(min(ny, cy + r + 1))
        x0, x1 = int(max(0, cx - r)), int(min(nx, cx + r + 1))
        m = (y[y0:y1, x0:x1] - cy) ** 2 + (x[y0:y1, x0:x1] - cx) ** 2 <= r * r
        for c in range(3):
            base[c][y0:y1, x0:x1] = np.where(m, col[c], base[c][y0:y1, x0:x1])
    return [np.clip(rng.poisson(np.clip(b, 1, 250)), 0, 255).astype(np.float32) for b in base]
