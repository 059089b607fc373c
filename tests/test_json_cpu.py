"""The acquisition JSON (CombinedOutput, lib.rs:32-45, printed by main.rs:893
with serde_json::to_string_pretty) from tga_results_json / tga_format_f64,
pinned on the CPU against serde_json's rules:

* numbers: serde_json writes f64 with ryu's format_finite -- the shortest
  digits that round-trip, "d.0" when integral and 10^kk <= 1e16, a plain
  decimal for 1e-5 <= |x| < 1e16, otherwise "d.ddde[-]x" with no '+' and no
  leading zeros in the exponent; -0.0 keeps its sign; NaN and inf become
  null.  `ryu_format` below restates that case analysis on Python's shortest
  round-trip digits (repr), independently of the library's C code;
* layout: two-space indentation, one array element per line, `[]` for an
  empty array, fields in struct order (sv, strengths, phases, freqs,
  cn0_acr, phase_median, phase_mad, freq_median, freq_mad), Option::None
  fields omitted, `null` for a None inside cn0_acr (acquisition.rs:36-59),
  constellations in CombinedOutput order, results sorted by sv.
"""
import ctypes
import json
import math
import struct

import numpy as np
import pytest

import tga


def _fmt(v):
    buf = ctypes.create_string_buffer(64)
    assert tga.lib().tga_format_f64(ctypes.c_double(v), buf, 64) == 0
    return buf.value.decode()


def ryu_format(x):
    """serde_json / ryu format_finite of one f64 (null for NaN, inf)."""
    if math.isnan(x) or math.isinf(x):
        return "null"
    if x == 0.0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    sign = "-" if x < 0 else ""
    r = repr(abs(x))  # shortest round-trip digits
    mant, _, exp = r.partition("e")
    e = int(exp) if exp else 0
    if "." in mant:
        ip, fp = mant.split(".")
    else:
        ip, fp = mant, ""
    digits = (ip + fp).lstrip("0")
    # value = 0.digits... x 10^kk: position of the decimal point
    lead_zeros = len(ip + fp) - len((ip + fp).lstrip("0"))
    kk = len(ip) + e - lead_zeros
    digits = digits.rstrip("0") or "0"
    n = len(digits)
    k = kk - n
    if 0 <= k and kk <= 16:
        return sign + digits + "0" * k + ".0"
    if 0 < kk <= 16:
        return sign + digits[:kk] + "." + digits[kk:]
    if -5 < kk <= 0:
        return sign + "0." + "0" * (-kk) + digits
    if n == 1:
        return sign + digits + "e" + str(kk - 1)
    return sign + digits[0] + "." + digits[1:] + "e" + str(kk - 1)


FIXED = [
    (0.0, "0.0"), (-0.0, "-0.0"), (1.0, "1.0"), (100.0, "100.0"), (-2.5, "-2.5"), (4.092e6, "4092000.0"),
    (1e-5, "0.00001"), (1e-6, "1e-6"), (1.2345e-6, "1.2345e-6"), (0.000123, "0.000123"), (-1.5e-7, "-1.5e-7"),
    (1e15, "1000000000000000.0"), (1e16, "1e16"), (1.5e16, "1.5e16"), (123456789012345.6, "123456789012345.6"),
    (float(np.float32(0.1)), "0.10000000149011612"), (float(np.float32(266590.0)), "266590.0"),
    (1.0 / 3.0, "0.3333333333333333"), (5e-324, "5e-324"), (1.7976931348623157e308, "1.7976931348623157e308"),
    (float("nan"), "null"), (float("inf"), "null"), (-float("inf"), "null"),
]


@pytest.mark.parametrize("v,want", FIXED, ids=[w for _, w in FIXED])
def test_format_f64_fixed_values(v, want):
    assert ryu_format(v) == want
    assert _fmt(v) == want


def test_format_f64_random_doubles_round_trip():
    rng = np.random.default_rng(0x1CE)
    bits = rng.integers(0, 2 ** 63, size=4000, dtype=np.int64).astype(np.uint64)
    vals = [struct.unpack("<d", struct.pack("<Q", int(b)))[0] for b in bits]
    # and values on the scales the search reports (strengths, phases, Hz, dB-Hz)
    vals += list(rng.uniform(0, 1, 500)) + list(rng.uniform(-6000, 6000, 500)) + \
        [float(np.float32(v)) for v in rng.uniform(0, 3e5, 500)] + list(rng.uniform(20, 70, 200))
    for v in map(float, vals):
        s = _fmt(v)
        assert s == ryu_format(v), (v, s)
        if s != "null":
            assert float(s) == v or (v != v)


def _cells(rows):
    out = np.zeros(len(rows), dtype=tga.CELL_DTYPE)
    for i, r in enumerate(rows):
        for k, v in r.items():
            out[i][k] = v
    return out


def _json(cells, ants, mask, cn0, fpm=float("nan"), ffm=float("nan")):
    p = ctypes.c_char_p()
    nf = ctypes.c_size_t()
    a = np.ascontiguousarray(ants, dtype=np.int32)
    rc = tga.lib().tga_results_json(cells.ctypes.data_as(ctypes.c_void_p), len(cells),
                                    a.ctypes.data_as(ctypes.c_void_p), len(a), mask, int(cn0), fpm, ffm,
                                    ctypes.byref(p), ctypes.byref(nf))
    assert rc == 0
    text = ctypes.string_at(p).decode()
    tga.lib().tga_free(p)
    return text, nf.value


def _serde_pretty(obj, lvl=0):
    """serde_json::to_string_pretty of nested dicts / lists / floats / ints /
    strings / None, numbers through ryu_format."""
    pad, pad1 = "  " * lvl, "  " * (lvl + 1)
    if isinstance(obj, dict):
        if not obj:
            return "{}"
        return "{\n" + ",\n".join(pad1 + json.dumps(k) + ": " + _serde_pretty(v, lvl + 1)
                                  for k, v in obj.items()) + "\n" + pad + "}"
    if isinstance(obj, list):
        if not obj:
            return "[]"
        return "[\n" + ",\n".join(pad1 + _serde_pretty(v, lvl + 1) for v in obj) + "\n" + pad + "]"
    if obj is None:
        return "null"
    if isinstance(obj, bool):
        return "true" if obj else "false"
    if isinstance(obj, int):
        return str(obj)
    if isinstance(obj, float):
        return ryu_format(obj)
    return json.dumps(obj)


def _median(x):
    x = sorted(x)
    m = len(x) // 2
    return (x[m - 1] + x[m]) / 2.0 if len(x) % 2 == 0 else x[m]


def test_results_json_layout_matches_serde():
    # two antennas (numbers 3 and 7), GPS PRNs 12 and 2 and Galileo PRN 5;
    # GPS12 has one failed C/N0 (null), GPS02 has none valid (cn0_acr
    # omitted), f32-widened strengths, tiny and large values
    f32 = lambda v: float(np.float32(v))
    rows = [
        dict(constellation=tga.GPS, prn=12, antenna=3, signal_strength=f32(123.4), second_peak=f32(20.1),
             codephase_frac=0.25, frequency=-300.0, cn0_acr=45.123456789, cn0_valid=1),
        dict(constellation=tga.GPS, prn=12, antenna=7, signal_strength=f32(99.9), second_peak=f32(21.0),
             codephase_frac=0.2500610948191593, frequency=0.0, cn0_acr=0.0, cn0_valid=0),
        dict(constellation=tga.GPS, prn=2, antenna=3, signal_strength=f32(1e-6), second_peak=f32(1e-6),
             codephase_frac=1e-6, frequency=-6000.0, cn0_valid=0),
        dict(constellation=tga.GPS, prn=2, antenna=7, signal_strength=f32(3.0), second_peak=f32(2.0),
             codephase_frac=0.999, frequency=5700.0, cn0_valid=0),
        dict(constellation=tga.GALILEO, prn=5, antenna=3, signal_strength=f32(7.5), second_peak=f32(3.5),
             codephase_frac=0.5, frequency=300.0, cn0_acr=51.25, cn0_valid=1),
        dict(constellation=tga.GALILEO, prn=5, antenna=7, signal_strength=f32(8.5), second_peak=f32(3.25),
             codephase_frac=0.75, frequency=600.0, cn0_acr=52.0, cn0_valid=1),
    ]
    cells = _cells(rows)
    mask = 1 << tga.GPS | 1 << tga.GALILEO
    text, nf = _json(cells, [3, 7], mask, True)
    assert nf == 0

    def prn_result(sv, rs):
        r = {"sv": sv, "strengths": [x["signal_strength"] for x in rs], "phases": [x["codephase_frac"] for x in rs],
             "freqs": [x["frequency"] for x in rs]}
        cn = [x["cn0_acr"] if x["cn0_valid"] else None for x in rs]
        if any(v is not None for v in cn):
            r["cn0_acr"] = cn
        pm, fm = _median(r["phases"]), _median(r["freqs"])
        r.update(phase_median=pm, phase_mad=_median([abs(v - pm) for v in r["phases"]]), freq_median=fm,
                 freq_mad=_median([abs(v - fm) for v in r["freqs"]]))
        return r
    by = lambda c, p: [x for x in rows if x["constellation"] == c and x["prn"] == p]
    want = {"gps": {"antenna_numbers": [3, 7], "results": [prn_result("GPS02", by(tga.GPS, 2)),
                                                           prn_result("GPS12", by(tga.GPS, 12))]},
            "galileo": {"antenna_numbers": [3, 7], "results": [prn_result("GSAT05", by(tga.GALILEO, 5))]}}
    assert text == _serde_pretty(want)
    assert '"cn0_acr": [\n          45.123456789,\n          null\n        ]' in text
    assert "1e-6" in text
    # field order inside a result
    doc = json.loads(text)
    assert list(doc["gps"]["results"][1]) == ["sv", "strengths", "phases", "freqs", "cn0_acr", "phase_median",
                                              "phase_mad", "freq_median", "freq_mad"]
    assert "cn0_acr" not in doc["gps"]["results"][0]


def test_results_json_one_antenna_omits_medians_and_cn0_off():
    cells = _cells([dict(constellation=tga.SBAS, prn=131, antenna=0, signal_strength=2.0, second_peak=1.0,
                         codephase_frac=0.125, frequency=-900.0, cn0_acr=40.0, cn0_valid=1)])
    text, _ = _json(cells, [0], 1 << tga.SBAS, False)
    want = {"sbas": {"antenna_numbers": [0], "results": [{"sv": "SBAS131", "strengths": [2.0], "phases": [0.125],
                                                          "freqs": [-900.0]}]}}
    assert text == _serde_pretty(want)


def test_results_json_empty_selection():
    text, _ = _json(_cells([]), [0, 1], 1 << tga.QZSS, False)
    assert text == _serde_pretty({"qzss": {"antenna_numbers": [0, 1], "results": []}})
