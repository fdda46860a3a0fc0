"""Small cases of the filter kernels for ncu captures (one GPU, a few GB).

    python -m microtomodenoise_b200.profile_case fast
        two iterations of a 512x512x64 grain pack, patch r2 search r5, FP16
        form: iteration 1 with the shipped proposal (k = 112 per 8^3 tile, the
        one-tile-per-CTA kernel), iteration 2 full search (the 32-wide kernel).
    python -m microtomodenoise_b200.profile_case learned
        the whole learned + FP16 job (noise estimates, 4 iterations, k = 144
        per 32x8x8 block) on a 512x512x128 grain pack, for a launch list.
    python -m microtomodenoise_b200.profile_case slab
        two exact FP32 iterations of a 256^3 grain pack at the reference's
        default geometry (patch r1, search r10, 11 slices: 3102 offsets), the
        tile kernel with raw staged as a z-offset slab.
"""
from __future__ import annotations

import sys

import numpy as np


def fast_case():
    import torch
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth
    from microtomodenoise_b200.proposal import ProposalNet, default_weights
    vol = synth.grain_pack_volume((64, 512, 512), seed=0)
    raw = torch.from_numpy(vol).cuda()
    net = ProposalNet.load(default_weights((2, 2, 2), (5, 5, 5)))
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(2, 2, 2),
                                                    radius_searchspace=(5, 5, 5), precision="f16"))
    g.set_sigma(np.full(64, 0.14, np.float32))
    g.attach_proposal(net, 112, 0.0)
    g.Run_GaussianNoise_device(1, raw.data_ptr())
    g.attach_proposal(None)
    g.Run_GaussianNoise_device(2)
    torch.cuda.synchronize()
    print("ok", g.describe())
    g.free_device()
    net.close()


def learned_case():
    import torch
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth
    from microtomodenoise_b200.proposal import ProposalNet, default_weights
    vol = synth.grain_pack_volume((128, 512, 512), seed=0)
    raw = torch.from_numpy(vol).cuda()
    out = torch.empty_like(raw)
    net = ProposalNet.load(default_weights((2, 2, 2), (5, 5, 5)))
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(2, 2, 2),
                                                    radius_searchspace=(5, 5, 5), precision="f16",
                                                    noise_mode="z-adaptive", n_samples=100000))
    g.attach_proposal(net, 144, 0.0, tiles_x=4)
    g.denoise(raw.data_ptr(), on_device=True, out=out.data_ptr())
    torch.cuda.synchronize()
    print("ok", g.describe(), g.proposal_stats())
    g.free_device()
    net.close()


def slab_case():
    import torch
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth
    vol = synth.grain_pack_volume((256, 256, 256), seed=0)
    raw = torch.from_numpy(vol).cuda()
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(1, 1, 1),
                                                    radius_searchspace=(10, 10, 10), nslices=11))
    g.set_sigma(np.full(256, 0.045, np.float32))
    g.Run_GaussianNoise_device(1, raw.data_ptr())
    g.Run_GaussianNoise_device(2)
    torch.cuda.synchronize()
    ms, n = g.filter_kernel_ms()
    print("ok", g.describe(), f"{ms:.1f} ms per launch ({n})")
    g.free_device()


if __name__ == "__main__":
    {"fast": fast_case, "learned": learned_case, "slab": slab_case}[sys.argv[1] if len(sys.argv) > 1 else "fast"]()
