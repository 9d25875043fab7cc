"""CPU tests of the pilot's weights file (ZB3DPLT1) and of the C entry points' checks:
the Python writer and reader agree, the shipped file is intact and carries its gate,
and the loader refuses damaged, foreign or mis-sized files before any CUDA call."""
import ctypes
import os
import struct
import zlib

import numpy as np
import pytest

from zb3d import _native as N
from zb3d import pilot as P


def _load_bytes(data: bytes):
    err = N.err_buf()
    buf = ctypes.create_string_buffer(data, len(data))
    h = N.lib().zb3d_pilot_from_memory(buf, len(data), 0, err, len(err))
    return h, err.value.decode()


def test_writer_and_reader_round_trip(tmp_path):
    with np.load(P.WEIGHTS) as f:
        st = {k: f[k] for k in f.files}
    path = str(tmp_path / "w.zb3dp")
    gate = [(5.0, 640, 480, -0.2), (10.0, 640, 480, 0.03), (10.0, 320, 240, 0.1)]
    P.save_weights(path, st, gate=gate, gate_frames=3, tol=0.05)
    back = P.read_weights(path)
    assert tuple(back["arch"]) == tuple(st["arch"])
    assert back["gate_frames"] == 3
    assert np.allclose(np.array(back["gate"]), np.array(gate)) and back["tol"] == pytest.approx(0.05)
    for l in range(len(P.arch(*(int(v) for v in st["arch"])))):
        assert np.array_equal(back[f"w{l}"], st[f"w{l}"]) and np.array_equal(back[f"b{l}"], st[f"b{l}"])
    data = open(path, "rb").read()
    assert data[:8] == b"ZB3DPLT1" and struct.unpack("<I", data[8:12])[0] == 1
    assert struct.unpack("<I", data[-4:])[0] == zlib.crc32(data[:-4]) & 0xFFFFFFFF


def test_shipped_binary_matches_the_trained_weights_and_has_a_gate():
    back = P.read_weights(P.WEIGHTS_BIN)
    with np.load(P.WEIGHTS) as f:
        assert tuple(back["arch"]) == tuple(f["arch"])
        for k in f.files:
            if k.startswith(("w", "b")):
                assert np.array_equal(back[k], f[k]), k
    # one level per calibrated noise level and plane size of 1080p YUV420
    levels = {(w, h): [s for s, ww, hh, _ in back["gate"] if (ww, hh) == (w, h)] for w, h in P.GATE_SIZES}
    for (w, h), sig in levels.items():
        assert sig == list(P.GATE_SIGMAS), (w, h, sig)
    assert back["gate_frames"] >= 8 and back["tol"] == pytest.approx(0.05)


def _reseal(data: bytes) -> bytes:
    body = data[:-4]
    return body + struct.pack("<I", zlib.crc32(body) & 0xFFFFFFFF)


def test_loader_refuses_bad_files_before_any_cuda_call():
    good = open(P.WEIGHTS_BIN, "rb").read()
    h, msg = _load_bytes(b"NOTPILOT" + good[8:])
    assert not h and "not a ZB3DPLT1" in msg
    flipped = bytearray(good)
    flipped[100] ^= 1
    h, msg = _load_bytes(bytes(flipped))
    assert not h and "checksum" in msg
    v2 = bytearray(good)
    v2[8:12] = struct.pack("<I", 2)
    h, msg = _load_bytes(_reseal(bytes(v2)))
    assert not h and "version" in msg
    odd = bytearray(good)
    odd[12:16] = struct.pack("<I", 24)  # 24 hidden channels: no kernel for it
    h, msg = _load_bytes(_reseal(bytes(odd)))
    assert not h and "architecture" in msg
    short = good[:-4 - 8]
    h, msg = _load_bytes(_reseal(short + b"\0\0\0\0"))
    assert not h and "size does not match" in msg
    h, msg = _load_bytes(b"ZB3D")
    assert not h and "too short" in msg
    err = N.err_buf()
    assert not N.lib().zb3d_pilot_load(b"/nonexistent/pilot.zb3dp", 0, err, len(err))
    assert "cannot open" in err.value.decode()


def test_pilot_entry_points_reject_null_handles():
    lib = N.lib()
    assert lib.zb3d_pilot_accepts(None, 10.0, 64, 64) == 0
    assert lib.zb3d_pilot_workspace_bytes(None, 64, 64) == 0
    assert lib.zb3d_pilot_run(None, 0x10000, 64, 64, 64, 10.0, 0x10000, 64, 0x10000, None, None) == -1
    assert lib.zb3d_pilot_gate_level(None, 0, None, None, None, None) == -1
    lib.zb3d_pilot_free(None)


@pytest.mark.parametrize("v2, over, msg", [
    (0, {}, '"pilot" needs BM3Dv2'),
    (1, {"ref": True}, '"ref" must not be given'),
    (1, {"radius": 1}, '"pilot" needs radius 0'),
])
def test_create_checks_pilot_arguments(v2, over, msg):
    """A pilot handle is not dereferenced before these checks (a fake one serves)."""
    lib = N.lib()
    a = N.Args()
    lib.zb3d_args_init(ctypes.byref(a))
    vi = N.VideoInfo(N.GRAY, N.FLOAT, 32, 0, 0, 1, 64, 48, 4)
    sig = (ctypes.c_float * 1)(10.0)
    a.sigma, a.n_sigma = ctypes.cast(sig, ctypes.POINTER(ctypes.c_float)), 1
    a.pilot = 0x10000
    if over.get("ref"):
        a.ref = ctypes.pointer(vi)
    if "radius" in over:
        a.radius = over["radius"]
    err = N.err_buf()
    assert not lib.zb3d_create(ctypes.byref(vi), ctypes.byref(a), v2, err, len(err))
    assert msg in err.value.decode()
