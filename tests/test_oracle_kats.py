"""Pin the CPU oracle to the reference's known-answer tests.

Each test restates one reference unit test (file:line in tart-gnss-acquire)
and runs it on the oracle; the golden vectors come from tests/golden/kats.json
(extracted from the reference's test modules by tests/golden/make_golden.py).
"""
import json
import math
import os

import numpy as np
import pytest

import acq_oracle as O


@pytest.fixture(scope="module")
def kats(golden_dir):
    return json.load(open(os.path.join(golden_dir, "kats.json")))


def chips24_to_octal(bits):
    """beidou_codes.rs:212-220 / l1c_codes.rs:243-251 (0/1 chips, MSB-first)."""
    return "".join(str(4 * bits[3 * i] + 2 * bits[3 * i + 1] + bits[3 * i + 2]) for i in range(8))


def chips10_to_octal(chips):
    """sbas.rs:417-426 / qzss.rs:418-427 (+1 -> 0, -1 -> 1)."""
    b = [0 if v == 1.0 else 1 for v in chips]
    return "%d%d%d%d" % (b[0], 4 * b[1] + 2 * b[2] + b[3], 4 * b[4] + 2 * b[5] + b[6], 4 * b[7] + 2 * b[8] + b[9])


@pytest.mark.parametrize("const,key", [(O.BEIDOU, "b1c"), (O.L1C, "l1c")])
def test_weil_first_last24_octal(kats, const, key):
    # beidou_codes.rs:255-279, l1c_codes.rs:291-315
    for prn in range(1, 64):
        bits = O.weil_bits(const, prn)
        assert chips24_to_octal(bits[:24]) == kats[key + "_first24"][prn - 1], prn
        assert chips24_to_octal(bits[-24:]) == kats[key + "_last24"][prn - 1], prn


def test_sbas_qzss_first10_octal(kats):
    # sbas.rs:444-455, qzss.rs:443-454
    for i, exp in enumerate(kats["sbas_first10"]):
        assert chips10_to_octal(O.base_sequence(O.SBAS, 120 + i)[:10]) == exp
    for i, exp in enumerate(kats["qzss_first10"]):
        assert chips10_to_octal(O.base_sequence(O.QZSS, 184 + i)[:10]) == exp


def test_code_lengths_and_bipolar():
    # acquisition.rs:405-423, galileo.rs:372-398, beidou_codes.rs:283-323
    for c, n in [(O.GPS, 1023), (O.SBAS, 1023), (O.QZSS, 1023), (O.GALILEO, 4092), (O.BEIDOU, 20460), (O.L1C, 20460)]:
        lo, hi = O.PRN_RANGE[c]
        for prn in range(lo, hi + 1):
            s = O.base_sequence(c, prn)
            assert len(s) == n and set(np.unique(s)) <= {-1.0, 1.0}
    with pytest.raises(ValueError):
        O.base_sequence(O.GPS, 39)
    with pytest.raises(ValueError):
        O.base_sequence(O.SBAS, 119)


def test_boc_structure():
    # beidou_codes.rs:145-157: [+c, -c] per chip; mapping 0 -> +1 (:347-358)
    bits = O.weil_bits(O.BEIDOU, 1)
    s = O.base_sequence(O.BEIDOU, 1)
    assert np.array_equal(s[0::2], 1.0 - 2.0 * bits)
    assert np.array_equal(s[1::2], -s[0::2])


def test_legendre_residue_count():
    # beidou_codes.rs:201-206: exactly (N-1)/2 ones -> Weil code of w has balanced-ish chips
    for c in (O.BEIDOU, O.L1C):
        bits = O.weil_bits(c, 5)
        assert len(bits) == 10230


def test_resampling_lengths():
    # acquisition.rs:473-484, gold_code length == n for every n
    for n in range(1000, 1100):
        assert len(O.resampled_code(O.GPS, 5, 1000.0, n)) == n
    r = O.resampled_code(O.GPS, 1, 1023.0, 2046)
    assert np.array_equal(r[:1023], r[1023:])


# ---- ACR (acr.rs:103-169) --------------------------------------------------
@pytest.mark.parametrize("tid", [0, 1, 2, 3])
def test_acr_tables_monotonic(tid):
    t = O.acr_table(tid)
    assert len(t) >= 10 and t[0, 0] > 1.0
    assert np.all(np.diff(t[:, 0]) > 0) and np.all(np.diff(t[:, 1]) > 0)


@pytest.mark.parametrize("tid", [0, 1, 2, 3])
def test_acr_cutoff_points_saturation(tid):
    t = O.acr_table(tid)
    for r in (0.5, 1.0, float("nan")):
        assert O.estimate_cn0(r, tid) is None
    for r, c in t[::7]:
        assert O.estimate_cn0(r, tid) == c
    assert O.estimate_cn0(0.5 * (1.0 + t[0, 0]), tid) == t[0, 1]
    assert O.estimate_cn0(t[-1, 0] * 10.0, tid) == t[-1, 1]


def test_acr_gps_mid_range(kats):
    for r, c in kats["acr_gps_points"]:
        assert abs(O.estimate_cn0(r, 0) - c) < 0.3


def test_acr_interpolation_monotonic():
    t = O.acr_table(0)
    prev, r = t[0, 1], t[0, 0]
    while r < t[-1, 0]:
        r *= 1.01
        c = O.estimate_cn0(r, 0)
        assert c >= prev - 1e-9
        prev = c


# ---- stats.rs:36-60 ---------------------------------------------------------
def test_stats():
    assert O.median([1.0, 3.0, 2.0]) == 2.0
    assert O.median([1.0, 4.0, 2.0, 3.0]) == 2.5
    assert O.median([7.0]) == 7.0
    assert O.mad([1.0, 2.0, 3.0, 4.0, 5.0], 3.0) == 1.0
    assert O.mad([2.0, 2.0, 2.0], 2.0) == 0.0


# ---- observation.rs:246-320 ----------------------------------------------------
def test_unpack_and_correlate():
    assert list(O.unpack_bits(np.array([0b10101010], np.uint8))) == [1, 0, 1, 0, 1, 0, 1, 0]
    b = O.unpack_bits(np.array([0xFF, 0x00], np.uint8))
    assert list(b[:8]) == [1] * 8 and list(b[8:]) == [0] * 8
    assert abs(O.correlate_antennas([1, 0, 1, 0], [1, 0, 1, 0]) - 1.0) < 1e-12
    assert abs(O.correlate_antennas([1, 0, 1, 0], [0, 1, 0, 1]) + 1.0) < 1e-12


def test_freq_grid():
    # acquisition.rs:188-198
    fc = O.freq_grid(4.092e6, 6000.0)
    assert len(fc) == 41 and fc[0] == 4.092e6 - 6000.0 and fc[-1] == 4.092e6 + 6000.0
    assert list(O.freq_grid(100e3, 0.0)) == [100e3]
    assert len(O.freq_grid(0.0, 3000.0)) == 21


def test_real_fixture_shape(golden_dir):
    z = np.load(os.path.join(golden_dir, "tart_head.npz"))
    assert z["head"].shape == (24, 40920) and z["ones"].shape == (24,)
    assert float(z["sampling_frequency"]) == 16368000.0
    frac = z["ones"] / (int(z["row_bytes"]) * 8.0)
    assert np.all((frac > 0.44) & (frac < 0.56))


def test_gps_ca_first10_octal_is_gps_200():
    # IS-GPS-200 Table 3-Ia, first 10 chips of the C/A code in octal, PRN 1-32
    # (tables.json; the reference has no such test).  The table counts a chip
    # of logic 1 as a 1 bit, and the reference's bipolar C/A chip is +1 for
    # logic 1 (acquisition.rs:96-125: registers start at -1 = logic 1, chip =
    # -(g1 g2)), so +1 -> 1 here -- the complement of the mapping the
    # reference's SBAS / QZSS octal tests use for their tables.
    want = O.tables()["ca_first10_octal"]
    for prn in range(1, 33):
        c = O.base_sequence(O.GPS, prn)[:10]
        assert chips10_to_octal(-c) == want[prn - 1], prn


def _header_tables():
    """The product's generated table header, parsed as text."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    h = open(os.path.join(root, "tart-gnss_b200", "csrc", "gnss_tables.h")).read()

    def body(name):
        i = h.index(name)
        return h[h.index("{", i) + 1:h.index("};", i)]
    ints = lambda b: [int(x) for x in re.findall(r"-?\d+", b)]
    out = {"gps_g2_delay": ints(body("TGA_GPS_G2_DELAY")), "sbas_g2_delay": ints(body("TGA_SBAS_G2_DELAY")),
           "qzss_g2_delay": ints(body("TGA_QZSS_G2_DELAY")),
           "galileo_e1c_hex": re.findall(r'"([0-9A-F]{1023})"', body("TGA_GALILEO_E1C_HEX"))}
    for key, name in (("b1cp_weil_wp", "TGA_B1CP_WP"), ("l1cp_weil_wp", "TGA_L1CP_WP")):
        v = ints(body(name + "[63][2]"))
        out[key] = [v[2 * i:2 * i + 2] for i in range(len(v) // 2)]
    for key, name in (("acr_gps_l1_ca", "TGA_GPS_L1_CA_ACR_TABLE"), ("acr_galileo_e1c", "TGA_GALILEO_E1C_ACR_TABLE"),
                      ("acr_beidou_b1c", "TGA_BEIDOU_B1C_ACR_TABLE"), ("acr_gps_l1c", "TGA_GPS_L1C_ACR_TABLE")):
        v = [float(x) for x in re.findall(r"[-+0-9.eE]+", body(name + "["))]
        out[key] = [v[2 * i:2 * i + 2] for i in range(len(v) // 2)]
    return out


def test_oracle_tables_equal_product_header():
    """The oracle's tables (tests/golden/tables.json, read from the reference
    sources) and the product's generated header hold the same values, so a
    transcription error in either shows up here rather than passing every
    parity test on both sides."""
    mine, theirs = O.tables(), _header_tables()
    for key, v in theirs.items():
        want = mine[key] if key != "galileo_e1c_hex" else [x.upper() for x in mine[key]]
        assert v == want, key
