"""libtga.so checks that need no GPU: it loads, exports every entry point of
include/tga.h, and its host-side code tables match the oracle's independent
restatement bit for bit."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import acq_oracle as O
import tga

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "tga.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tga_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_all_symbols():
    L = tga.lib()
    syms = _declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", tga.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (tga_\w+)", out))
    assert set(syms) <= exported, set(syms) - exported
    assert b"sm_100a" in L.tga_version()


@pytest.mark.parametrize("c", range(6), ids=O.NAMES)
def test_code_chips_match_oracle(c):
    lo, hi = O.PRN_RANGE[c]
    for prn in range(lo, hi + 1):
        mine = tga.code_chips(c, prn).astype(np.float64)
        ref = O.base_sequence(c, prn)
        assert np.array_equal(mine, ref), (c, prn)


def test_code_chips_rejects_bad_prn():
    for c, prn in [(tga.GPS, 0), (tga.GPS, 39), (tga.SBAS, 119), (tga.QZSS, 207), (tga.GALILEO, 51), (tga.L1C, 64)]:
        with pytest.raises(tga.TgaError):
            tga.code_chips(c, prn)


@pytest.mark.parametrize("c,spc,n", [
    (tga.GPS, 16368.0, 32736), (tga.GPS, 16000.0, 32000), (tga.GPS, 2046.0, 2049), (tga.GPS, 256.0, 512),
    (tga.GALILEO, 65472.0, 130944), (tga.GALILEO, 4092.0, 4095), (tga.BEIDOU, 163680.0, 327360),
    (tga.L1C, 10230.0, 20460), (tga.L1C, 10230.0, 10236), (tga.SBAS, 1023.0, 2046), (tga.QZSS, 16000.0, 1000)])
def test_resampled_code_matches_oracle(c, spc, n):
    prn = O.PRN_RANGE[c][0] + 2
    assert np.array_equal(tga.code_resampled(c, prn, spc, n).astype(np.float64), O.resampled_code(c, prn, spc, n))


def test_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    h = ctypes.c_void_p()
    rc = tga.lib().tga_create(0, ctypes.byref(h))
    assert rc == 3 and not h.value
    with pytest.raises(tga.TgaError):
        tga.Context(0)


def test_cell_count():
    o = tga.AllOptions()
    o.constellation_mask = tga.ALL
    n = ctypes.c_size_t()
    assert tga.lib().tga_all_cell_count(24, ctypes.byref(o), ctypes.byref(n)) == 0
    assert n.value == 24 * (38 + 50 + 63 + 39 + 63 + 23)
    p = np.array([1, 2], dtype=np.int32)
    o.constellation_mask = 1 << tga.SBAS
    o.prn_filter = p.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    o.n_prn_filter = 2
    assert tga.lib().tga_all_cell_count(24, ctypes.byref(o), ctypes.byref(n)) == 1  # PRN 1 invalid for SBAS
