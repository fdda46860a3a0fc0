"""The allocation-free two-cluster EM entry point (inlm_noise_em_noalloc).

It serves callers that cannot allocate device memory (for instance code that
runs while another thread captures a CUDA graph in global mode, or an
application whose device memory belongs to its own pool): its scratch is a
file-scope device array of the library. Here it is called through the C ABI
with inputs and outputs the test allocates, several times in a row, and its
per-window results are checked against what the regular entry point
(inlm_noise_estimate) produces for the same samples, to the noise tests'
1e-6 relative tolerance.

Kept in a file of its own, collected after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, NoiseLevel, _lib, synth

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6


def _noalloc_sigma(lib, torch, patchstd, windows, shift):
    values = torch.from_numpy(np.ascontiguousarray(patchstd, np.float32)).cuda()
    nw = len(windows)
    mean = torch.full((nw,), -1.0, dtype=torch.float32, device="cuda")
    sd = torch.full((nw,), -1.0, dtype=torch.float32, device="cuda")
    win = np.ascontiguousarray(windows, np.int64).reshape(-1)
    torch.cuda.synchronize()
    rc = lib.inlm_noise_em_noalloc(None, values.data_ptr(), len(patchstd), win.ctypes.data, nw,
                                   mean.data_ptr(), sd.data_ptr())
    _lib.check(rc, "inlm_noise_em_noalloc")
    torch.cuda.synchronize()
    m, s = mean.cpu().numpy(), sd.cpu().numpy()
    # sigma = mean + shift*std, as the estimator finishes (noiselevel.cpp:51)
    return (m + np.float32(shift) * s).astype(np.float32), m


def test_noalloc_em_matches_regular_estimate(gpu, port):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    vol = synth.small_case((24, 48, 56), seed=5)
    cases = [("z-adaptive", 10), ("global", 100), ("z-adaptive", 6)]
    for mode, zwin in cases:  # consecutive calls reuse the same static scratch
        nl = NoiseLevel(8000, 15, vol.shape, seed=1)
        dp = DenoiseParameters(noise_mode=mode, zwindow=zwin, stds_from_mean=1.0)
        want = nl.get_noiselevel(vol, dp)
        ps, samples = nl.patchstd(), nl.samples()
        nl.close()
        if mode == "global":
            windows = [[0, len(samples) - 1]]
        else:
            st, en = port.zwindows(samples, vol.shape, zwin)
            windows = np.stack([st, en], 1)
        got, mean = _noalloc_sigma(lib, torch, ps, windows, 1.0)
        assert np.all(mean > 0), "every window holds samples, so no neighbour fill is involved"
        if mode == "global":
            got = np.full(vol.shape[0], got[0], np.float32)
        rel = np.max(np.abs(got / want - 1))
        assert rel <= REL_TOL, f"{mode} window {zwin}: max relative difference {rel}"


def test_noalloc_em_rejects_oversized_requests(gpu):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    n = 2000
    values = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.empty(20000, dtype=torch.float32, device="cuda")
    # more windows than the static table holds
    many = np.zeros((16385, 2), np.int64)
    rc = lib.inlm_noise_em_noalloc(None, values.data_ptr(), n, many.ctypes.data, 16385,
                                   out.data_ptr(), out.data_ptr())
    assert rc == -1 and b"16384" in lib.inlm_last_error()
    # windows covering more samples (16384 x 2000) than the static scratch holds (16 Mi)
    cover = np.tile(np.array([[0, n - 1]], np.int64), (16384, 1))
    rc = lib.inlm_noise_em_noalloc(None, values.data_ptr(), n, cover.ctypes.data, 16384,
                                   out.data_ptr(), out.data_ptr())
    assert rc == -1 and b"static scratch" in lib.inlm_last_error()
    # a window outside the values
    bad = np.array([[0, n]], np.int64)
    rc = lib.inlm_noise_em_noalloc(None, values.data_ptr(), n, bad.ctypes.data, 1,
                                   out.data_ptr(), out.data_ptr())
    assert rc == -1


def test_noalloc_em_empty_windows_store_no_range(gpu):
    """An empty window (last < first) yields zeros whatever its indices are,
    and does not shift the scratch of the windows after it: first = 2^32,
    last = 5 would read as 0..5 if the indices were truncated to 32 bits."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    vol = synth.small_case((16, 40, 48), seed=7)
    nl = NoiseLevel(6000, 15, vol.shape, seed=2)
    nl.get_noiselevel(vol, DenoiseParameters(noise_mode="global"))
    ps = nl.patchstd()
    nl.close()
    n = len(ps)
    want, want_mean = _noalloc_sigma(lib, torch, ps, [[0, n - 1]], 1.0)
    windows = [[1 << 32, 5], [0, n - 1], [7, 6]]
    got, mean = _noalloc_sigma(lib, torch, ps, windows, 1.0)
    assert mean[0] == 0.0 and mean[2] == 0.0
    assert abs(got[1] / want[0] - 1) <= REL_TOL


def test_noalloc_em_beside_a_global_mode_capture(gpu):
    """The call enqueues kernels only, so it may run on a non-blocking stream
    while another thread captures a CUDA graph in global capture mode (where
    cudaMalloc, or a copy from pageable host memory, would invalidate the
    capture). Both the call and the capture must succeed."""
    import threading
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    vol = synth.small_case((16, 40, 48), seed=9)
    nl = NoiseLevel(6000, 15, vol.shape, seed=4)
    nl.get_noiselevel(vol, DenoiseParameters(noise_mode="global"))
    ps = nl.patchstd()
    nl.close()
    n = len(ps)
    want, _ = _noalloc_sigma(lib, torch, ps, [[0, n - 1]], 1.0)  # first call, before any capture
    values = torch.from_numpy(np.ascontiguousarray(ps, np.float32)).cuda()
    mean = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    sd = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    win = np.array([0, n - 1], np.int64)
    side = torch.cuda.Stream()  # torch creates its streams with cudaStreamNonBlocking
    x = torch.zeros(16, device="cuda")
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    capturing, called = threading.Event(), threading.Event()
    rc_box = []

    def caller():
        capturing.wait(30)
        rc_box.append(lib.inlm_noise_em_noalloc(C.c_void_p(side.cuda_stream), values.data_ptr(), n,
                                                win.ctypes.data, 1, mean.data_ptr(), sd.data_ptr()))
        called.set()

    t = threading.Thread(target=caller)
    t.start()
    with torch.cuda.graph(graph, capture_error_mode="global"):
        capturing.set()
        assert called.wait(30), "the call did not return while the capture was open"
        x.add_(1.0)
    t.join(30)
    assert rc_box == [0], lib.inlm_last_error()
    side.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 16.0
    got = (mean.cpu().numpy() + sd.cpu().numpy()).astype(np.float32)
    assert abs(got[0] / want[0] - 1) <= REL_TOL
