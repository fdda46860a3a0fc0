"""Batched form (one persistent kernel per iteration over many volumes, the
whole schedule captured as a CUDA graph) and the tile-configuration
autotuner. Every batched volume must equal its own single-volume run of the
same schedule bit for bit: the persistent kernel runs the same tile bodies,
and the noise estimates draw the same samples."""
import numpy as np
import pytest

from microtomodenoise_b200 import Batch, DenoiseParameters, IterativeNLM_GPU, synth
from oracle.oracle import FilterParams

pytestmark = pytest.mark.gpu


def cases():
    return [
        ((20, 40, 48), DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3),
                                         noise_mode="global", noise_seed=1)),
        ((16, 36, 70), DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(2, 2, 2),
                                         noise_mode="manual", sigma=(0.05, 0.04))),
        ((24, 33, 40), DenoiseParameters(radius_patchspace=(3, 3, 3), radius_searchspace=(2, 2, 2),
                                         noise_mode="z-adaptive", zwindow=10, noise_seed=3)),
        # patch shape without a batched body: its own launch inside the graph
        ((9, 17, 33), DenoiseParameters(radius_patchspace=(1, 1, 2), radius_searchspace=(2, 2, 2),
                                        noise_mode="global", noise_seed=4)),
        ((12, 64, 64), DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(5, 5, 5),
                                         noise_mode="global", maxiterations=2, noise_seed=5)),
        # raw staged as a slab (search radius 10): the persistent slab body
        ((14, 36, 40), DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(10, 10, 10),
                                         noise_mode="global", noise_seed=6)),
    ]


def single(raw, p):
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, p)
    out, _, _ = g.denoise(raw)
    g.free_device()
    return out


def test_batch_equals_single_volume_runs(gpu):
    cs = cases()
    raws = [synth.small_case(s, seed=10 + i) for i, (s, _) in enumerate(cs)]
    b = Batch([s for s, _ in cs], [p for _, p in cs])
    desc = b.describe()
    print(desc)
    assert "persistent nlm_batch_f32<" in desc and "own launch" in desc
    assert "persistent nlm_batch_f32<p111, raw_slab>" in desc
    outs = b.run(raws)
    assert b.last_ms > 0
    for i, ((s, p), raw, got) in enumerate(zip(cs, raws, outs)):
        want = single(raw, p)
        assert np.array_equal(got, want), f"volume {i} {s}"
    # replay with new inputs
    raws2 = [synth.small_case(s, seed=50 + i) for i, (s, _) in enumerate(cs)]
    outs2 = b.run(raws2)
    for i, ((s, p), raw, got) in enumerate(zip(cs, raws2, outs2)):
        assert np.array_equal(got, single(raw, p)), f"replay volume {i}"
    # and the first inputs again
    outs3 = b.run(raws)
    for a, c in zip(outs, outs3):
        assert np.array_equal(a, c)
    b.close()


def test_batch_device_pointers(gpu):
    torch = pytest.importorskip("torch")
    cs = cases()[:3]
    raws = [synth.small_case(s, seed=70 + i) for i, (s, _) in enumerate(cs)]
    b = Batch([s for s, _ in cs], [p for _, p in cs])
    host = b.run(raws)
    dr = [torch.from_numpy(r).cuda() for r in raws]
    do = [torch.empty_like(t) for t in dr]
    torch.cuda.synchronize()
    b.run([t.data_ptr() for t in dr], [t.data_ptr() for t in do], on_device=True)
    for h, d in zip(host, do):
        assert np.array_equal(h, d.cpu().numpy())
    b.close()


def test_autotune_keeps_results(gpu, port):
    from oracle.oracle import FilterParams
    raw = synth.small_case((16, 40, 72), seed=3)
    p = DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3))
    sig = np.full(16, 0.06, np.float32)
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, p)
    rep = g.autotune()
    print(rep)
    assert "chosen" in rep or "cached" in rep
    g.set_sigma(sig)
    g.Run_GaussianNoise(1, raw)
    got = g.get_result()
    g.free_device()
    want = port.denoise_f32(raw, FilterParams(search_radius=(3, 3, 3), patch_radius=(2, 2, 2)),
                            sig[None])
    assert np.array_equal(got, want)


def test_batch_groups_by_patch_weights(gpu):
    """Volumes of one patch shape whose weights differ (the distance-weight
    table with z anisotropy; the CPU table ignores anisotropy) run in separate
    launch groups: a group's kernel reads the weights of its first volume."""
    cs = [((16, 40, 48), DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3),
                                           noise_mode="manual", sigma=(0.05, 0.04), z_anisotropy=za,
                                           weight_table="distweight"))
          for za in (1.0, 2.0, 1.0, 0.5)]
    raws = [synth.small_case(s, seed=90 + i) for i, (s, _) in enumerate(cs)]
    b = Batch([s for s, _ in cs], [p for _, p in cs])
    desc = b.describe()
    assert desc.count("persistent nlm_batch_f32<p222") == 3, desc
    outs = b.run(raws)
    for i, ((s, p), raw, got) in enumerate(zip(cs, raws, outs)):
        assert np.array_equal(got, single(raw, p)), f"volume {i} z_anisotropy {p.z_anisotropy}"
    b.close()


def test_batch_at_config3_sizes_against_the_oracle(gpu, port):
    """The batch at the batched workload's largest sizes, pinned to the oracle
    directly rather than through the single-volume path: a 384x384x256 volume
    at patch radius 3, search radius 7 (the costliest shape of the mix), a
    256x200x160 one at patch radius 2, search radius 5 and a 64^3 one at patch
    radius 1, search radius 3 in one batch with manual sigma. Iteration 1 (one
    batched iteration) and iteration 2 (a two-iteration batch) are compared
    at 1500 seeded voxels per volume, faces and edges included, with the
    oracle's FP32 filter (bit-exact to the reference's CPU filter) evaluated
    at those voxels on the reflectively padded raw volume and previous
    iterate."""
    shapes = [(256, 384, 384), (160, 200, 256), (64, 64, 64)]
    radii = [((3, 3, 3), (7, 7, 7)), ((2, 2, 2), (5, 5, 5)), ((1, 1, 1), (3, 3, 3))]
    raws = [synth.spheres_volume(s, n_spheres=40, rmin=4, rmax=20, noise_std=0.05, seed=300 + i)
            for i, s in enumerate(shapes)]
    sig = (0.06, 0.045)

    def params(pr, sr, iters):
        return DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, noise_mode="manual",
                                 sigma=sig, maxiterations=iters)

    b1 = Batch(shapes, [params(pr, sr, 1) for pr, sr in radii])
    it1 = b1.run(raws)
    b1.close()
    b2 = Batch(shapes, [params(pr, sr, 2) for pr, sr in radii])
    it2 = b2.run(raws)
    b2.close()
    rng = np.random.default_rng(7)
    for (pr, sr), raw, o1, o2 in zip(radii, raws, it1, it2):
        nz, ny, nx = raw.shape
        p = FilterParams(search_radius=sr, patch_radius=pr)
        pad = port.padding(p)
        # seeded voxels: uniform, plus the volume's corners and face centres
        vox = list(rng.integers(0, raw.size, 1500 - 14))
        for z in (0, nz - 1):
            for y in (0, ny - 1):
                for x in (0, nx - 1):
                    vox.append((z * ny + y) * nx + x)
        for z, y, x in ((0, ny // 2, nx // 2), (nz - 1, ny // 2, nx // 2), (nz // 2, 0, nx // 2),
                        (nz // 2, ny - 1, nx // 2), (nz // 2, ny // 2, 0), (nz // 2, ny // 2, nx - 1)):
            vox.append((z * ny + y) * nx + x)
        vox = np.asarray(vox, np.int64)
        raw_pad = port.pad_reflective(raw, pad)
        s0 = np.full(nz, sig[0], np.float32)
        s1 = (np.float32(0.5) * s0 + np.float32(0.5) * np.full(nz, sig[1], np.float32)).astype(np.float32)
        want1 = port.filter_voxels(raw_pad, raw_pad, raw.shape, p, s0, vox)
        assert np.array_equal(o1.ravel()[vox], want1), f"iteration 1, shape {raw.shape}"
        want2 = port.filter_voxels(raw_pad, port.pad_reflective(o1, pad), raw.shape, p, s1, vox)
        assert np.array_equal(o2.ravel()[vox], want2), f"iteration 2, shape {raw.shape}"
