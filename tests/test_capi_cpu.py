"""CPU-side checks of the C ABI: the library builds for sm_100a, loads
without a GPU, exports every function include/*.h declares, and its host-only
logic (bounds, messages, header peek) matches the reference."""

import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(fqxv_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_reference_api():
    names = _declared()
    for fn in ["fqxv_rans_encode", "fqxv_rans_decode", "fqxv_rans_decode_bounded", "fqxv_rans_decode_with",
               "fqxv_rans_peek_output_len", "fqxv_rans_encode_batch", "fqxv_rans_decode_batch",
               "fqxv_crc32c_batch", "fqxv_crc32c_combine", "fqxv_frame_blocks", "fqxv_read_blocks",
               "fqxv_payload_stream_locs"]:
        assert fn in names


def test_library_exports_every_declared_symbol():
    from fqxv_b200 import rans

    L = rans.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_status_messages_are_the_references(orc):
    from fqxv_b200 import rans

    for st, msg in orc.MESSAGES.items():
        assert rans.status_message(st) == msg


def test_encode_bound():
    from fqxv_b200 import rans

    assert rans.encode_bound(0, 0) == 9
    assert rans.encode_bound(0, 1) == 9
    assert rans.encode_bound(10, 0) == 9 + 512 + 128 + 20
    assert rans.encode_bound(10, 1) == 9 + 32 + 256 * 512 + 128 + 20
    assert rans.encode_bound(10, 2) == rans.encode_bound(10, 1)


def test_bound_check_happens_before_decoding():
    # lib.rs:226-231: a declared length above the bound fails without decoding
    # (so this runs without a device).
    from fqxv_b200 import rans

    bomb = b"\x00" + (1 << 31).to_bytes(8, "little") + bytes(700)
    with pytest.raises(rans.Malformed) as e:
        rans.decode_bounded(bomb, 1 << 20)
    assert e.value.status == 7
    L = rans.lib()
    n = ctypes.c_uint64(0)
    assert L.fqxv_rans_peek_output_len(ctypes.c_char_p(bomb), len(bomb), ctypes.byref(n)) == 0
    assert n.value == 1 << 31
    assert L.fqxv_rans_peek_output_len(ctypes.c_char_p(b"\x00\x01"), 2, ctypes.byref(n)) == 1


def test_status_numbering_matches_oracle():
    text = open(os.path.join(ROOT, "include", "fqxv_rans_gpu.h")).read()
    o = open(os.path.join(ROOT, "oracle", "rans_oracle.h")).read()
    pairs = dict(re.findall(r"FQXV_RANS_(E_\w+) = (\d+)", text))
    opairs = dict(re.findall(r"ORC_(E_\w+) = (\d+)", o))
    for k, v in opairs.items():
        assert pairs[k] == v, k


def _build_c_caller(tmp_path):
    """Compile tests/c/capi_roundtrip.c as strict C99 against the header and
    link it with the library; returns the executable's path."""
    import subprocess

    from fqxv_b200 import build

    lib = build.build()
    libdir = os.path.dirname(lib)
    exe = str(tmp_path / "capi_roundtrip")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c", "capi_roundtrip.c"), "-o", exe, "-L", libdir, "-lfqxv_rans_gpu",
           "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_plain_c_caller_compiles_and_links(tmp_path):
    assert os.path.exists(_build_c_caller(tmp_path))


def test_frame_tok_stream_entry_points_validate_arguments():
    """The added C-ABI calls reject bad arguments before touching a device,
    and their host-only arithmetic needs none."""
    from fqxv_b200 import rans

    L = rans.lib()
    null = ctypes.c_void_p()
    n = ctypes.c_uint64(0)
    assert L.fqxv_crc32c_batch(null, null, null, 0, null) == 16
    assert L.fqxv_frame_blocks(null, null, null, 0, 0, null, 0, null, null, ctypes.byref(n)) == 16
    sz = ctypes.c_size_t(0)
    t = ctypes.c_int(0)
    assert L.fqxv_read_blocks(null, null, 0, 0, null, null, null, ctypes.byref(sz), ctypes.byref(n),
                              ctypes.byref(t)) == 16
    assert L.fqxv_tok_encode_host(null, null, null, 0, null, 0, null, 0, null, None) == 16
    assert L.fqxv_tok_decode_host(null, null, null, 0, null, 0, null, 0, null, null, None, None) == 16
    assert L.fqxv_put_streams_host(null, null, null, 0, null, 0, null, None) == 16
    assert L.fqxv_perm_decode_host(null, null, 0, 0, null) == 16
    spans = (ctypes.c_uint64 * 4)(0, 10, 10, 5)
    assert L.fqxv_frame_blocks_bound(spans, 2, 0) == 16 * 2 + 15
    assert L.fqxv_frame_blocks_bound(spans, 2, 1) == 16 * 2 + 15 + 12


def test_added_status_messages():
    from fqxv_b200 import rans

    assert rans.status_message(33) == "corrupted fqxv data: block (crc mismatch)"
    assert rans.status_message(48) == "malformed name stream: unsupported version"
    assert rans.status_message(61) == "malformed name stream: unknown op"
    assert rans.status_message(64) == "malformed lroverlap block"
    assert rans.status_message(66) == "malformed fqxv block: permutation length mismatch"
