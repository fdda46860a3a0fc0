"""C ABI checks that need no GPU: the library loads, exports every entry point
include/inlm.h declares, reports missing devices cleanly, and its host-side
geometry and sampling equal the oracle's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, _lib
from oracle.oracle import FilterParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(inlm_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol(lib):
    decl = declared_entry_points()
    assert len(decl) >= 18
    for name in decl:
        assert hasattr(lib, name), name
    assert set(decl) == set(_lib.EXPORTS)


def test_default_params_match_reference_defaults(lib):
    p = _lib.InlmParams()
    lib.inlm_default_params(C.byref(p))
    assert p.alpha == 0.5 and p.maxiterations == 4 and p.nslices == 11
    assert list(p.search_radius) == [10, 10, 10] and list(p.patch_radius) == [1, 1, 1]
    assert p.zwindow == 100 and p.n_samples == 100000 and p.noise_patchsize == 15
    assert p.noise_mode == 0 and p.stds_from_mean == 1.0


def test_errors_are_reported_not_raised(lib):
    h = C.c_void_p()
    p = _lib.InlmParams()
    lib.inlm_default_params(C.byref(p))
    bad = (C.c_int * 3)(0, 10, 10)
    rc = lib.inlm_denoiser_create(bad, C.byref(p), C.byref(h))
    assert rc in (-1, -3)  # bad shape, or no device on this machine
    assert lib.inlm_last_error()


def _geometry(lib, dp: DenoiseParameters, nz=20):
    cp = dp.to_c()
    ns, npch = C.c_int(0), C.c_int(0)
    pad = (C.c_int * 3)()
    assert lib.inlm_geometry(C.byref(cp), nz, None, C.byref(ns), None, None, C.byref(npch), pad) == 0
    s = np.zeros(3 * ns.value, np.int32)
    q = np.zeros(3 * npch.value, np.int32)
    w = np.zeros(npch.value, np.float32)
    assert lib.inlm_geometry(C.byref(cp), nz, s.ctypes.data, C.byref(ns), q.ctypes.data,
                             w.ctypes.data, C.byref(npch), pad) == 0
    return s.reshape(-1, 3), q.reshape(-1, 3), w, tuple(pad)


@pytest.mark.parametrize("pr,sr,nsl,an", [
    ((1, 1, 1), (5, 5, 5), 11, 1.0), ((2, 2, 2), (5, 5, 5), 11, 1.0), ((3, 3, 3), (7, 7, 7), 11, 1.0),
    ((3, 3, 3), (7, 7, 7), 15, 1.0), ((1, 2, 3), (3, 4, 5), 7, 1.0), ((2, 2, 2), (2, 2, 2), 11, 2.0),
    ((1, 2, 1), (2, 2, 2), 11, 1.5), ((1, 1, 0), (2, 2, 0), 11, 1.0), ((3, 3, 1), (10, 10, 10), 11, 1.0),
])
def test_host_geometry_equals_oracle(lib, port, pr, sr, nsl, an):
    dp = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, nslices=nsl, z_anisotropy=an)
    s, q, w, pad = _geometry(lib, dp)
    fp = FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl, z_anisotropy=an)
    assert np.array_equal(s, port.search_offsets(fp))
    assert np.array_equal(q, port.patch_taps(fp))
    ow, _ = port.filter_weights(fp, 20 + 2 * pad[2])
    assert np.array_equal(w, ow)
    assert pad == port.padding(fp)


@pytest.mark.parametrize("shape,mask,seed", [((40, 64, 72), 0, 7), ((40, 64, 72), 60, 7),
                                             ((5, 33, 17), 0, 2**31 + 1), ((64, 128, 128), 0, 0)])
def test_host_sampling_equals_oracle(lib, port, shape, mask, seed):
    nz, ny, nx = shape
    n = 5000
    out = np.zeros(n, np.int64)
    rc = lib.inlm_noise_draw_samples((C.c_int * 3)(nx, ny, nz), n, 15, mask, seed, out.ctypes.data)
    assert rc == 0
    assert np.array_equal(out, port.draw_samples(shape, n, 15, mask, seed))


def test_host_sampling_matches_reference_fixture(lib, golden_noise):
    out = np.zeros(20000, np.int64)
    assert lib.inlm_noise_draw_samples((C.c_int * 3)(72, 64, 40), 20000, 15, 0, 7, out.ctypes.data) == 0
    assert np.array_equal(out, golden_noise["global_m0_samples"].astype(np.int64))


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(ImportError):
        _lib._lib_saved = _lib._lib
        try:
            _lib._lib = None
            _lib.load(str(tmp_path / "nope.so"))
        finally:
            _lib._lib = _lib._lib_saved


@pytest.mark.parametrize("pr,sr,nsl", [((1, 1, 1), (10, 10, 10), 11), ((2, 2, 2), (7, 7, 7), 11),
                                       ((1, 1, 2), (9, 9, 9), 21), ((3, 3, 3), (7, 7, 7), 15),
                                       ((2, 2, 1), (4, 6, 3), 5)])
def test_search_list_runs_z_major(lib, pr, sr, nsl):
    """The raw-slab staging of the tile kernel relies on the search offsets
    running z-major (the reference order, iternlm_prepare.cpp:102-150): a pair
    of consecutive offsets then spans at most two z offsets."""
    s, _, _, _ = _geometry(lib, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, nslices=nsl))
    z = s[:, 2]
    assert np.all(np.diff(z) >= 0)
    pairs = [z[i:i + 2] for i in range(0, len(z), 2)]
    assert max(int(p.max() - p.min()) for p in pairs) <= 1


def test_multi_gpu_entry_points_without_a_gpu(lib):
    """inlm_denoise_multi checks its arguments before it touches a device;
    inlm_device_count reports 0 devices here without failing."""
    n = C.c_int(-1)
    assert lib.inlm_device_count(C.byref(n)) == 0 and n.value >= 0
    p = _lib.InlmParams()
    lib.inlm_default_params(C.byref(p))
    shape = (C.c_int * 3)(16, 16, 32)
    buf = np.zeros(16 * 16 * 32, np.float32)
    ids = (C.c_int * 2)(0, 0)
    assert lib.inlm_denoise_multi(shape, C.byref(p), None, buf.ctypes.data, 2, ids, None, None) == -1
    assert lib.inlm_denoise_multi(shape, C.byref(p), buf.ctypes.data, buf.ctypes.data, 0, ids,
                                  None, None) == -1
    assert "n_parts" in lib.inlm_last_error().decode()
    if n.value == 0:  # valid arguments, no device: INLM_ERR_NODEVICE
        assert lib.inlm_denoise_multi(shape, C.byref(p), buf.ctypes.data, buf.ctypes.data, 2, ids,
                                      None, None) == -3


def test_blocks_entry_points_check_arguments(lib):
    """The per-iteration host-RAM engine rejects bad arguments before it
    touches a device."""
    p = _lib.InlmParams()
    lib.inlm_default_params(C.byref(p))
    h = C.c_void_p(None)
    shape = (C.c_int * 3)(16, 16, 16)
    assert lib.inlm_blocks_create(shape, C.byref(p), 0, None, 8, C.byref(h)) == -1
    assert "n_devices" in lib.inlm_last_error().decode()
    assert lib.inlm_blocks_create(shape, None, 1, None, 8, C.byref(h)) == -1
    assert lib.inlm_blocks_run_iteration(None, 1, None, None, None) == -1
    assert lib.inlm_blocks_set_sigma(None, None) == -1


def test_proposal_schedule_entry_points_check_arguments(lib):
    """The per-iteration proposal schedules reject bad arguments before they
    touch a device; the Python helper broadcasts scalars and pads the shorter
    sequence with its last entry."""
    from microtomodenoise_b200 import _schedule
    k = (C.c_int * 2)(64, 128)
    r = (C.c_float * 2)(0.0, 0.9)
    assert lib.inlm_proposal_schedule(None, 2, k, r) == -1
    assert lib.inlm_blocks_proposal_schedule(None, 2, k, r) == -1
    p = _lib.InlmParams()
    lib.inlm_default_params(C.byref(p))
    shape = (C.c_int * 3)(16, 16, 16)
    buf = np.zeros(16 ** 3, np.float32)
    assert lib.inlm_stream_denoise_sched(shape, C.byref(p), buf.ctypes.data, buf.ctypes.data, 8, None, 0, k, r,
                                         0.0, 4, None, None, None) == -1
    assert "schedule" in lib.inlm_last_error().decode()
    bad = (C.c_int * 2)(64, -1)
    assert lib.inlm_stream_denoise_sched(shape, C.byref(p), buf.ctypes.data, buf.ctypes.data, 8, None, 2, bad, r,
                                         0.0, 4, None, None, None) == -1
    badr = (C.c_float * 2)(0.0, 1.5)
    assert lib.inlm_stream_denoise_sched(shape, C.byref(p), buf.ctypes.data, buf.ctypes.data, 8, None, 2, k, badr,
                                         0.0, 4, None, None, None) == -1
    ks, rels = _schedule([128, 128, 128, 240], [0.0, 0.0, 0.0, 0.9])
    assert ks.tolist() == [128, 128, 128, 240] and np.allclose(rels, [0, 0, 0, 0.9])
    ks, rels = _schedule(208, 0.9)
    assert ks.tolist() == [208] and np.allclose(rels, [0.9])
    ks, rels = _schedule([96, 240], 0.5)
    assert ks.tolist() == [96, 240] and np.allclose(rels, [0.5, 0.5])
    assert ks.dtype == np.int32 and rels.dtype == np.float32


REF_MAIN = os.path.join(os.environ.get("INLM_REFERENCE_DIR", "/root/reference/iterNLM_v0.3"), "main.cpp")


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference sources not present")
def test_reference_driver_compiles_against_the_shim(tmp_path):
    """The reference's unmodified main.cpp compiles against this library's C++
    shim: csrc/compat provides its header names (denoise_parameters.h,
    Geometry/, Noise/, Denoiser/, Color/). It is compiled from a copy because
    a quoted include searches the source file's own directory first."""
    import shutil
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    csrc = os.path.join(root, "microtomodenoise_b200", "csrc")
    src = tmp_path / "main.cpp"
    shutil.copy(REF_MAIN, src)
    r = subprocess.run(["g++", "-fsyntax-only", "-std=c++17", "-fopenmp", "-I" + os.path.join(csrc, "compat"),
                        "-I" + csrc, "-I" + os.path.join(root, "include"), str(src)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
