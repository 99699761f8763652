"""The result encoders (CPU): PFM in the format of Photon's save_pfm (src/scene/image.cpp:88-96) and PNG
of a display buffer (the image its save_png writes), checked by decoding the bytes here."""
import ctypes as C
import struct
import zlib

import numpy as np
import pytest

from photon_b200 import abi, native


def _photon_pfm(rgb):
    h, w = rgb.shape[:2]
    return f"PF\n{w} {h}\n-1.0\n".encode() + np.ascontiguousarray(rgb[::-1], "<f4").tobytes()


def _decode_png(data):
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, []
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) & 0xffffffff == crc
        chunks.append((typ, body))
        pos += 12 + n
    assert chunks[0][0] == b"IHDR" and chunks[-1][0] == b"IEND"
    w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (depth, ctype, comp, filt, inter) == (8, 6, 0, 0, 0)
    raw = zlib.decompress(b"".join(b for t, b in chunks if t == b"IDAT"))
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert (rows[:, 0] == 0).all()  # filter type none
    return np.ascontiguousarray(rows[:, 1:]).view("<u4").reshape(h, w)


@pytest.mark.parametrize("w,h", [(1, 1), (7, 3), (64, 37)])
def test_pfm_is_photons_format(w, h):
    rgb = np.random.default_rng(w * h).standard_normal((h, w, 3)).astype(np.float32)
    data = native.encode_pfm(rgb)
    assert data == _photon_pfm(rgb)
    head = f"PF\n{w} {h}\n-1.0\n".encode()
    back = np.frombuffer(data[len(head):], "<f4").reshape(h, w, 3)[::-1]
    assert np.array_equal(back, rgb)


@pytest.mark.parametrize("level", [0, 1, 6, 9])
def test_png_round_trips_the_display_buffer(level):
    rgba = np.random.default_rng(level).integers(0, 2**32, size=(29, 41), dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(_decode_png(native.encode_png(rgba, level)), rgba)


def test_encoder_size_query_and_capacity():
    lib = native.lib
    rgb = np.zeros((4, 5, 3), np.float32)
    n = C.c_size_t()
    assert lib.pt_encode_pfm(rgb.ctypes.data, 5, 4, None, 0, C.byref(n)) == abi.PT_OK
    assert n.value == len(b"PF\n5 4\n-1.0\n") + 4 * 5 * 12
    small = np.zeros(n.value - 1, np.uint8)
    assert lib.pt_encode_pfm(rgb.ctypes.data, 5, 4, small.ctypes.data, small.size, C.byref(n)) == abi.PT_ERR_INVALID
    assert lib.pt_encode_pfm(rgb.ctypes.data, 0, 4, None, 0, C.byref(n)) == abi.PT_ERR_INVALID
    rgba = np.zeros((2, 2), np.uint32)
    assert lib.pt_encode_png(rgba.ctypes.data, 2, 2, 10, None, 0, C.byref(n)) == abi.PT_ERR_INVALID


def test_file_writers_match_the_encoders(tmp_path):
    lib = native.lib
    rgb = np.random.default_rng(3).random((9, 11, 3), dtype=np.float32)
    rgba = np.random.default_rng(4).integers(0, 2**32, size=(9, 11), dtype=np.uint64).astype(np.uint32)
    pfm, png = tmp_path / "a.pfm", tmp_path / "a.png"
    assert lib.pt_write_pfm(str(pfm).encode(), 11, 9, rgb.ctypes.data) == abi.PT_OK
    assert lib.pt_write_png(str(png).encode(), 11, 9, rgba.ctypes.data) == abi.PT_OK
    assert pfm.read_bytes() == _photon_pfm(rgb)
    assert np.array_equal(_decode_png(png.read_bytes()), rgba)
    assert lib.pt_write_pfm(str(tmp_path / "missing" / "x.pfm").encode(), 11, 9, rgb.ctypes.data) == abi.PT_ERR_INVALID
