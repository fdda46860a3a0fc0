"""TIFF sequence IO (the hdcom::HdCommunication reads and writes of the iterNLM
driver, Geometry/hdcommunication.cpp) and the iterNLM command line, on the CPU.

The library's own TIFF reader and writer are checked against Pillow's
independent TIFF implementation in both directions, for every sample type the
driver reads, both byte orders and both stack layouts (slice directory,
multi-page file), plus the 16-bit save's clamp-and-round rule
(Save2DTifImage_as16bit, hdcommunication.cpp:1472)."""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import gpu_available

PIL = pytest.importorskip("PIL.Image")

from microtomodenoise_b200 import _lib, tiffio  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "microtomodenoise_b200", "lib", "iterNLM")


def _vol(shape=(5, 37, 53), seed=0):
    return np.random.default_rng(seed).normal(100, 500, shape).astype(np.float32)


def _round_half_away(v):
    v = v.astype(np.float64)
    return np.trunc(v + np.copysign(0.5, v))


def _as16(v):
    r = np.minimum(np.maximum(0.0, _round_half_away(v)), 65535.0)
    r[np.isnan(v)] = 0.0  # std::max(0.f, NaN) keeps 0
    return r.astype(np.uint16)


def test_float_sequence_written_here_reads_in_pillow(tmp_path):
    vol = _vol()
    tiffio.save_stack(vol, str(tmp_path / "f32"), "denoised", z0=3)
    names = sorted(os.listdir(tmp_path / "f32"))
    assert names == [f"denoised{z:04d}.tif" for z in range(3, 8)]
    for i, n in enumerate(names):
        im = PIL.open(tmp_path / "f32" / n)
        assert im.mode == "F" and im.size == (53, 37)
        assert np.array_equal(np.array(im), vol[i])


def test_16bit_save_clamps_and_rounds_half_away(tmp_path):
    v = np.array([[-3.7, -0.5, 0.49999997, 0.5, 1.5, 2.5, 3.5, 65534.5, 65535.4, 7e4, np.nan, np.inf,
                   -np.inf, 1234.5678]], np.float32)
    tiffio.save_stack(v, str(tmp_path), "s", as_16bit=True)
    im = PIL.open(tmp_path / "s0000.tif")
    assert im.mode == "I;16"
    got = np.array(im)
    assert np.array_equal(got, _as16(v)), (got, _as16(v))
    assert list(got[0, :8]) == [0, 0, 0, 1, 2, 3, 4, 65535]


@pytest.mark.parametrize("width", [1, 3, 2048, 2049])
def test_strip_layout_edge_widths(tmp_path, width):
    """rows per strip = max(1, 2048 / width): one row per strip for wide
    slices, many strips for narrow ones."""
    vol = _vol((2, 5, width), seed=width)
    tiffio.save_stack(vol, str(tmp_path), "w")
    for z in range(2):
        assert np.array_equal(np.array(PIL.open(tmp_path / f"w{z:04d}.tif")), vol[z])
    assert np.array_equal(tiffio.read_stack(str(tmp_path)), vol)


@pytest.mark.parametrize("kind", ["F", "I;16", "L", "I;16B", "I"])
def test_pillow_written_slices_read_here(tmp_path, kind):
    base = _vol((4, 19, 23), seed=1)
    if kind == "F":
        arrs = [s for s in base]
    elif kind in ("I;16", "I;16B"):
        arrs = [np.clip(s * 30, 0, 65535).astype(np.uint16) for s in base]
    elif kind == "L":
        arrs = [np.clip(s / 4, 0, 255).astype(np.uint8) for s in base]
    else:
        arrs = [(s * 1000).astype(np.int32) for s in base]
    d = tmp_path / "seq"
    d.mkdir()
    for z, a in enumerate(arrs):
        if kind == "I;16B":
            im = PIL.frombytes("I;16B", (a.shape[1], a.shape[0]), a.astype(">u2").tobytes())
        else:
            im = PIL.fromarray(a)
        im.save(d / f"img_{z:03d}.tiff")
    (d / "notes.txt").write_text("not a slice")
    (nz, ny, nx), spp = tiffio.stack_shape(str(d))
    assert (nz, ny, nx) == (4, 19, 23) and spp == 1
    got = tiffio.read_stack(str(d))
    assert np.array_equal(got, np.stack(arrs).astype(np.float32))


def test_multipage_file_and_slice_range(tmp_path):
    vol = _vol((7, 11, 13), seed=2)
    frames = [PIL.fromarray(v) for v in vol]
    p = tmp_path / "stack.tif"
    frames[0].save(p, save_all=True, append_images=frames[1:])
    assert tiffio.stack_shape(str(p))[0] == (7, 11, 13)
    assert np.array_equal(tiffio.read_stack(str(p)), vol)
    assert np.array_equal(tiffio.read_stack(str(p), 2, 4), vol[2:5])
    # one end given: the other is that end of the stack; ranges clamp
    assert np.array_equal(tiffio.read_stack(str(p), 5, -1), vol[5:])
    assert np.array_equal(tiffio.read_stack(str(p), -1, 1), vol[:2])
    assert np.array_equal(tiffio.read_stack(str(p), 3, 99), vol[3:])


def _imagej_contiguous(path, vol, big_endian):
    """One IFD followed by every page back to back, "images=N" in the
    description: how ImageJ stores large stacks (Custom3DTifReader's layout)."""
    nz, ny, nx = vol.shape
    e = ">" if big_endian else "<"
    desc = f"ImageJ=1.53t\nimages={nz}\nslices={nz}\n\0".encode()
    n_tags = 9
    ifd_off = 8
    desc_off = ifd_off + 2 + 12 * n_tags + 4
    data_off = desc_off + len(desc)
    data_off += (-data_off) % 16
    out = bytearray(b"MM" if big_endian else b"II")
    out += struct.pack(e + "HI", 42, ifd_off)
    tags = [(256, 4, 1, nx), (257, 4, 1, ny), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1),
            (270, 2, len(desc), desc_off), (273, 4, 1, data_off), (277, 3, 1, 1), (339, 3, 1, 3)]
    out += struct.pack(e + "H", n_tags)
    for tag, typ, cnt, val in tags:
        if typ == 3:
            out += struct.pack(e + "HHIHH", tag, typ, cnt, val, 0)
        else:
            out += struct.pack(e + "HHII", tag, typ, cnt, val)
    out += struct.pack(e + "I", 0)
    out += desc
    out += b"\0" * (data_off - len(out))
    out += vol.astype(e + "f4").tobytes()
    path.write_bytes(bytes(out))


@pytest.mark.parametrize("big_endian", [False, True])
def test_imagej_contiguous_stack(tmp_path, big_endian):
    vol = _vol((6, 9, 10), seed=3)
    p = tmp_path / "ij.tif"
    _imagej_contiguous(p, vol, big_endian)
    assert tiffio.stack_shape(str(p))[0] == (6, 9, 10)
    assert np.array_equal(tiffio.read_stack(str(p)), vol)
    assert np.array_equal(tiffio.read_stack(str(p), 4, 5), vol[4:6])


def test_io_errors(tmp_path):
    with pytest.raises(_lib.InlmError) as e:
        tiffio.stack_shape(str(tmp_path / "missing"))
    assert e.value.code == -8
    (tmp_path / "empty").mkdir()
    with pytest.raises(_lib.InlmError) as e:
        tiffio.stack_shape(str(tmp_path / "empty"))
    assert "No tif-file" in str(e.value)
    (tmp_path / "junk.tif").write_bytes(b"not a tiff at all")
    with pytest.raises(_lib.InlmError):
        tiffio.read_stack(str(tmp_path / "junk.tif"))
    # compressed and RGB slices are refused, not misread
    PIL.fromarray(np.zeros((8, 8), np.uint8)).save(tmp_path / "pk.tif", compression="packbits")
    with pytest.raises(_lib.InlmError) as e:
        tiffio.read_stack(str(tmp_path / "pk.tif"))
    assert e.value.code == -7
    PIL.fromarray(np.zeros((8, 8, 3), np.uint8)).save(tmp_path / "rgb.tif")
    assert tiffio.stack_shape(str(tmp_path / "rgb.tif"))[1] == 3
    with pytest.raises(_lib.InlmError) as e:
        tiffio.read_stack(str(tmp_path / "rgb.tif"))
    assert e.value.code == -7
    # slices of different sizes in one directory
    d = tmp_path / "mixed"
    d.mkdir()
    PIL.fromarray(np.zeros((8, 8), np.float32)).save(d / "a.tif")
    PIL.fromarray(np.zeros((8, 9), np.float32)).save(d / "b.tif")
    with pytest.raises(_lib.InlmError):
        tiffio.read_stack(str(d))


def _cli(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120)


def test_cli_help_and_input_errors(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("iterNLM not built")
    r = _cli("-h")
    assert r.returncode == 0 and "usage: iterNLM" in r.stdout
    r = _cli("-i", str(tmp_path / "nothing"))
    assert r.returncode != 0 and "not found" in r.stdout
    (tmp_path / "e").mkdir()
    r = _cli("-i", str(tmp_path / "e"))
    assert r.returncode != 0 and "No tif-file" in r.stdout
    tiffio.save_stack(_vol((3, 8, 8)), str(tmp_path / "in"), "s")
    r = _cli("-i", str(tmp_path / "in"), "-gpus", "0")
    assert r.returncode != 0 and "GPU only" in r.stdout
    r = _cli("-i", str(tmp_path / "in"), "--color")
    assert r.returncode != 0 and "RGB" in r.stdout


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_cli_without_device_reports_and_fails(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("iterNLM not built")
    tiffio.save_stack(_vol((3, 8, 8)), str(tmp_path / "in"), "s")
    r = _cli("-i", str(tmp_path / "in"), "-o", str(tmp_path / "out"))
    assert r.returncode != 0
    assert "image shape: 8x8x3" in r.stdout and "No CUDA device" in r.stdout
