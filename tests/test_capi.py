"""Host-side checks of the C ABI library (no GPU compute)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from cmblensing_b200 import _native as nat
from cmblensing_b200 import build as b

HEADER = os.path.join(ROOT, "include", "lenseflow.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lf_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    b.build(verbose=False)
    return nat.load()


def test_header_symbols_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/lenseflow.h but not exported"
    assert set(syms) == set(nat.SIGNATURES), "ctypes signature table out of sync with the header"


def test_version_and_status_strings(lib):
    assert lib.lf_version() >= 100
    for s in range(0, 9):
        assert len(nat.status_string(s)) > 0
    assert nat.status_string(99) == "unknown status"


def test_plan_rejects_bad_arguments_before_touching_the_device(lib):
    h = ctypes.c_void_p()
    assert lib.lf_plan_create(ctypes.byref(h), 100, 1, 1e-3, nat.LF_F32) == nat.LF_ERR_BAD_SHAPE
    assert lib.lf_plan_create(ctypes.byref(h), 128, 4, 1e-3, nat.LF_F32) == nat.LF_ERR_BAD_SHAPE
    assert lib.lf_plan_create(ctypes.byref(h), 128, 1, 1e-3, 7) == nat.LF_ERR_BAD_DTYPE
    assert lib.lf_plan_create(ctypes.byref(h), 128, 1, -1.0, nat.LF_F32) == nat.LF_ERR_BAD_ARG
    assert lib.lf_plan_create(None, 128, 1, 1e-3, nat.LF_F32) == nat.LF_ERR_BAD_ARG
    assert not h.value


def test_null_plan_calls_return_status(lib):
    assert lib.lf_workspace_bytes(None, 4, 0) == 0
    assert lib.lf_workspace_bytes_n(None, 4, 0, 7) == 0
    assert lib.lf_lense_flow(None, None, 0, None, 0, None, 1, 7, 1, 0, None, 0, None) == nat.LF_ERR_BAD_ARG
    assert lib.lf_phi_precompute(None, None, 0, 1, None, None, None, 0, None) == nat.LF_ERR_BAD_ARG
    assert lib.lf_plan_destroy(None) == nat.LF_OK


def test_new_entry_points_validate_before_touching_the_device(lib):
    """Null plans and bad arguments come back as status codes (no device work)."""
    assert lib.lf_pp_bytes(None, 4, 7) == 0
    assert lib.lf_vjp_ckpt_workspace_bytes(None, 4, 7) == 0
    assert lib.lf_phi_precompute_pp(None, None, 0, 1, None, None, 7, None, None, 0, None) == nat.LF_ERR_BAD_ARG
    assert lib.lf_lense_flow_pp(None, None, 0, None, 0, None, 1, 7, 1, 0, None, 0, None) == nat.LF_ERR_BAD_ARG
    assert lib.lf_lense_flow_vjp_ckpt(None, None, None, 0, None, 1, 7, 1, None, None, None, 0, None, 0,
                                      None) == nat.LF_ERR_BAD_ARG
    # per-mode products: bad shapes and misaligned pointers are refused
    assert lib.lf_modes_apply(None, 0, 1, None, None, None, 1, 4, 10, 1.0, 0.0, None) == nat.LF_ERR_BAD_SHAPE
    assert lib.lf_modes_apply(None, 0, 1, None, None, None, 1, 1, 10, 1.0, 0.0, None) == nat.LF_ERR_BAD_ARG
    assert lib.lf_modes_apply(None, 0, 1, None, None, None, 0, 1, 10, 1.0, 0.0, None) == nat.LF_OK


def test_timeout_status_without_a_plan(lib):
    """No plan, no recorded timeout: the status word reads OK without touching the device."""
    assert lib.lf_timeout_status() == nat.LF_OK


def test_min_det_encoding_round_trip(lib):
    import struct
    for v in (0.7, 1.0, 1e-9, -0.3, -5.0, 3.4e38):
        bits = struct.unpack("<i", struct.pack("<f", v))[0]
        enc = bits if bits >= 0 else bits ^ 0x7FFFFFFF
        assert abs(lib.lf_decode_min_det(enc) - v) <= 1e-7 * max(1.0, abs(v))


def test_encoded_order_is_monotone():
    import struct
    vals = [-3.0, -1.0, -0.1, 0.0, 0.1, 0.5, 2.0]
    enc = []
    for v in vals:
        bits = struct.unpack("<i", struct.pack("<f", v))[0]
        enc.append(bits if bits >= 0 else bits ^ 0x7FFFFFFF)
    assert enc == sorted(enc)


def test_host_pipeline_chunk_schedule():
    """Chunk sizes of the pipelined host-buffer call: near-equal by default, validated when given."""
    from cmblensing_b200.engine import chunk_schedule
    assert chunk_schedule(64, 16) == [4] * 16
    assert chunk_schedule(5, 2) == [3, 2]
    assert chunk_schedule(3, 16) == [1, 1, 1]
    assert chunk_schedule(0, 16) == []
    assert chunk_schedule(8, 4, [1, 2, 4, 1]) == [1, 2, 4, 1]
    for bad in ([1, 2, 4], [0, 4, 4], [9, -1]):
        with pytest.raises(ValueError):
            chunk_schedule(8, 4, bad)
