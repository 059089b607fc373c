#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference crate.

Run in the build container (where the reference checkout exists):
    python tests/golden/make_golden.py /path/to/tart-gnss

Outputs (committed; the GPU box never reads the reference):
* kats.json -- known-answer vectors copied from the reference's own unit
  tests: BeiDou B1C pilot first/last 24 chips in octal for PRN 1-63
  (src/beidou_codes.rs:225-253), GPS L1C pilot first/last 24 chips
  (src/l1c_codes.rs:256-289), SBAS first 10 chips (src/sbas.rs:436-442),
  QZSS first 10 chips (src/qzss.rs:437-441), and the ACR mid-range points
  (src/acr.rs:150-154).
* tables.json -- the oracle's own copy of the reference's data tables,
  read straight from its sources (the oracle does not use the product's
  generated header): G2 delays of GPS PRN 1-38 (src/acquisition.rs:84-87),
  SBAS 120-158 (src/sbas.rs:39-44) and QZSS 184-206 (src/qzss.rs:40-44);
  Weil (w, p) of the BeiDou B1C (src/beidou_codes.rs:46-63) and GPS L1C
  (src/l1c_codes.rs:45-62) pilots; the 50 Galileo E1-C hex codes
  (src/galileo_codes.rs:20-70); the four ACR tables (src/acr_tables.rs);
  and the IS-GPS-200 table of the first 10 C/A chips in octal for PRN 1-32
  (the ICD's known-answer column; the reference has no such test).
  The tables come from tart-gnss, GPL-3.0 (Cargo.toml:7), as signal
  definitions and calibration data.
* tart_head.npz -- the reference's real 24-antenna TART recording
  (data/data_2026-03-09_04_25_10.145497.hdf), reduced to what the
  acquisition search reads: per antenna the count of one-bits over the
  whole record (it sets the de-mean, acquisition.rs:285) and the first
  40920 packed bytes (= 327360 samples = two 10 ms code periods, the
  longest search window), plus the sampling rate from the file's config.
  The HDF5 `data` dataset is stored contiguous and uncompressed at the end
  of the file; its offset is checked against the JSON config.
* tart_head4096.hdf -- the same HDF5 file cut down to the first 4096 bytes
  of every antenna row: the file's own metadata (its first 6176 bytes)
  with the `data` dataspace (current and maximum dims) and the contiguous
  layout size patched to 24 x 4096, followed by the 24 row heads.  It is a
  valid HDF5 file of the reference's layout for the reader and CLI tests.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _strings(text, const):
    i = text.index(const)
    j = text.index("];", i)
    return re.findall(r'"([0-7]+)"', text[i:j])


def main(ref):
    src = os.path.join(ref, "src")
    rd = lambda f: open(os.path.join(src, f)).read()
    bds, l1c, sbas, qzss = rd("beidou_codes.rs"), rd("l1c_codes.rs"), rd("sbas.rs"), rd("qzss.rs")
    kats = {
        "b1c_first24": _strings(bds, "const REF_FIRST24"),
        "b1c_last24": _strings(bds, "const REF_LAST24"),
        "l1c_first24": _strings(l1c, "const REF_FIRST24"),
        "l1c_last24": _strings(l1c, "const REF_LAST24"),
        "sbas_first10": _strings(sbas, "const REF_FIRST10"),
        "qzss_first10": _strings(qzss, "const REF_FIRST10"),
        # acr.rs:150-154: r_A -> expected dB-Hz (+-0.3) in the GPS C/A table
        "acr_gps_points": [[4.1725, 45.0], [11.4497, 50.0]],
    }
    assert [len(kats[k]) for k in ("b1c_first24", "b1c_last24", "l1c_first24", "l1c_last24")] == [63] * 4
    assert len(kats["sbas_first10"]) == 39 and len(kats["qzss_first10"]) == 23
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, indent=1)
    write_tables(extract_tables(src))

    hdf = os.path.join(ref, "data", "data_2026-03-09_04_25_10.145497.hdf")
    raw = open(hdf, "rb").read()
    m = re.search(rb'\{[^{}]*"num_antenna"[^{}]*\}', raw)
    cfg = json.loads(m.group(0))
    n_ant = int(cfg["num_antenna"])
    row_bytes = 524288
    off = len(raw) - n_ant * row_bytes
    assert off == 6176, off
    block = np.frombuffer(raw[off:], dtype=np.uint8).reshape(n_ant, row_bytes)
    ones = np.unpackbits(block, axis=1).sum(axis=1).astype(np.int64)
    head_bytes = 327360 // 8
    np.savez_compressed(os.path.join(HERE, "tart_head.npz"), head=block[:, :head_bytes].copy(),
                        ones=ones, row_bytes=np.int64(row_bytes),
                        sampling_frequency=np.float64(cfg["sampling_frequency"]),
                        timestamp=np.bytes_(b"2026-03-09T04:25:10.145497+00:00"))
    write_hdf5_fixture(raw, block, n_ant, row_bytes, off)
    print("wrote kats.json, tart_head.npz and tart_head4096.hdf", ones[:4], off)


# IS-GPS-200 Table 3-Ia, "First 10 Chips (Octal)" of the C/A code, PRN 1-32
# (chip 1 first, MSB; a chip of logic 1 is a 1 bit)
CA_FIRST10_OCTAL = [
    "1440", "1620", "1710", "1744", "1133", "1455", "1131", "1454", "1626", "1504", "1642", "1750", "1764", "1772",
    "1775", "1776", "1156", "1467", "1633", "1715", "1746", "1763", "1063", "1706", "1743", "1761", "1770", "1774",
    "1127", "1453", "1625", "1712"]


def _array_body(text, name):
    """The text between the opening '[' of the array literal assigned to
    `name` and its closing '];' (comments removed)."""
    i = text.index(name)
    i = text.index("=", i)
    j = text.index("[", i)
    k = text.index("];", j)
    return re.sub(r"//[^\n]*", "", text[j + 1:k])


def extract_tables(src):
    rd = lambda f: open(os.path.join(src, f)).read()
    ints = lambda body: [int(x) for x in re.findall(r"-?\d+", body)]
    pairs = lambda body: [[int(a), int(b)] for a, b in re.findall(r"\(\s*(\d+)\s*,\s*(\d+)\s*\)", body)]
    fpairs = lambda body: [[float(a), float(b)] for a, b in
                           re.findall(r"\(\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\)", body)]
    t = {
        "gps_g2_delay": ints(_array_body(rd("acquisition.rs"), "CODE_DELAY_TABLE")),
        "sbas_g2_delay": ints(_array_body(rd("sbas.rs"), "CODE_DELAY_TABLE")),
        "qzss_g2_delay": ints(_array_body(rd("qzss.rs"), "CODE_DELAY_TABLE")),
        "b1cp_weil_wp": pairs(_array_body(rd("beidou_codes.rs"), "B1CP_PARAMS")),
        "l1cp_weil_wp": pairs(_array_body(rd("l1c_codes.rs"), "L1CP_PARAMS")),
        "galileo_e1c_hex": re.findall(r'"([0-9A-Fa-f]{1023})"', rd("galileo_codes.rs")),
        "ca_first10_octal": CA_FIRST10_OCTAL,
    }
    acr = rd("acr_tables.rs")
    for key, name in (("acr_gps_l1_ca", "GPS_L1_CA_ACR_TABLE"), ("acr_galileo_e1c", "GALILEO_E1C_ACR_TABLE"),
                      ("acr_beidou_b1c", "BEIDOU_B1C_ACR_TABLE"), ("acr_gps_l1c", "GPS_L1C_ACR_TABLE")):
        t[key] = fpairs(_array_body(acr, "static " + name))
    sizes = {k: len(v) for k, v in t.items()}
    assert sizes == {"gps_g2_delay": 38, "sbas_g2_delay": 39, "qzss_g2_delay": 23, "b1cp_weil_wp": 63,
                     "l1cp_weil_wp": 63, "galileo_e1c_hex": 50, "ca_first10_octal": 32, "acr_gps_l1_ca": 59,
                     "acr_galileo_e1c": 71, "acr_beidou_b1c": 79, "acr_gps_l1c": 79}, sizes
    t["provenance"] = ("tart-gnss-acquire v0.4.0 sources (GPL-3.0): signal-definition and calibration tables; "
                       "IS-GPS-200 Table 3-Ia first-10-chip octal column")
    return t


def write_tables(t):
    """tables.json with one table per line."""
    with open(os.path.join(HERE, "tables.json"), "w") as f:
        f.write("{\n" + ",\n".join("%s: %s" % (json.dumps(k), json.dumps(v)) for k, v in t.items()) + "\n}\n")


# byte offsets, inside the first 6176 bytes of the reference file, of the
# `data` dataset's dataspace dims (row length, current and maximum) and of
# its contiguous layout size
DIM_OFFSETS = (1712, 1728)
LAYOUT_SIZE_OFFSET = 1794
HEAD_ROW = 4096


def write_hdf5_fixture(raw, block, n_ant, row_bytes, off):
    import struct
    meta = bytearray(raw[:off])
    for o in DIM_OFFSETS:
        assert struct.unpack_from("<Q", meta, o)[0] == row_bytes
        assert struct.unpack_from("<Q", meta, o - 8)[0] == n_ant
        struct.pack_into("<Q", meta, o, HEAD_ROW)
    assert struct.unpack_from("<Q", meta, LAYOUT_SIZE_OFFSET)[0] == n_ant * row_bytes
    assert struct.unpack_from("<Q", meta, LAYOUT_SIZE_OFFSET - 8)[0] == off
    struct.pack_into("<Q", meta, LAYOUT_SIZE_OFFSET, n_ant * HEAD_ROW)
    with open(os.path.join(HERE, "tart_head4096.hdf"), "wb") as f:
        f.write(bytes(meta) + block[:, :HEAD_ROW].tobytes())


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/tart-gnss")
    main(sys.argv[1])
