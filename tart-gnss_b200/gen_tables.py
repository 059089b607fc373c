#!/usr/bin/env python3
"""Generate ``csrc/gnss_tables.h`` from the tart-gnss-acquire sources.

The acquisition search needs a handful of data tables that must be identical
to the ones the reference crate ships, because they are signal-definition
data (interface-control-document tables) or calibration data, not code:

* G2 delay (code-phase) tables for GPS L1 C/A PRN 1-38 (src/acquisition.rs:84-87),
  SBAS PRN 120-158 (src/sbas.rs:39-44) and QZSS PRN 184-206 (src/qzss.rs:40-44);
* Weil-code parameters (w, p) for BeiDou B1C pilot PRN 1-63
  (src/beidou_codes.rs:46-63) and GPS L1C pilot PRN 1-63 (src/l1c_codes.rs:45-62);
* Galileo E1-C primary memory codes, 50 hex strings of 1023 digits
  (src/galileo_codes.rs:20-70);
* ACR C/N0 lookup tables, r_A -> dB-Hz, for GPS/SBAS/QZSS C/A, Galileo E1-C,
  BeiDou B1C and GPS L1C (src/acr_tables.rs:23-327).

Numbers are copied as the decimal strings written in the reference, so the
C compiler rounds them to exactly the same IEEE doubles as rustc does.

Usage:  python gen_tables.py <reference_src_dir>
The generated header is committed; this script only needs re-running if the
reference tables change.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "gnss_tables.h")


def _block(text, start_pat):
    """Return the text between the first '[' after ``start_pat`` and its matching '];'."""
    i = text.index(start_pat)
    j = text.index("= [", i) if "= [" in text[i:i + 400] else text.index("= &[", i)
    j = text.index("[", j + 1) if text[j:j + 3] == "= [" else text.index("[", j + 2)
    k = text.index("];", j)
    return text[j + 1:k]


def _ints(block):
    body = re.sub(r"//[^\n]*", "", block)
    return [int(x) for x in re.findall(r"\b\d+\b", body)]


def _pairs(block):
    return [(int(a), int(b)) for a, b in re.findall(r"\(\s*(\d+)\s*,\s*(\d+)\s*\)", block)]


def _float_pairs(block):
    return re.findall(r"\(\s*([0-9.eE+-]+)\s*,\s*([0-9.eE+-]+)\s*\)", block)


def main(src):
    rd = lambda f: open(os.path.join(src, f)).read()
    acq, sbas, qzss = rd("acquisition.rs"), rd("sbas.rs"), rd("qzss.rs")
    bds, l1c, gal, acr = rd("beidou_codes.rs"), rd("l1c_codes.rs"), rd("galileo_codes.rs"), rd("acr_tables.rs")

    gps_g2 = _ints(_block(acq, "const CODE_DELAY_TABLE"))
    gps_g2 = gps_g2[:38] if len(gps_g2) > 38 else gps_g2
    sbas_g2 = _ints(_block(sbas, "const CODE_DELAY_TABLE"))
    qzss_g2 = _ints(_block(qzss, "const CODE_DELAY_TABLE"))
    b1c = _pairs(_block(bds, "const B1CP_PARAMS"))
    l1cp = _pairs(_block(l1c, "const L1CP_PARAMS"))
    gal_hex = re.findall(r'"([0-9A-Fa-f]{100,})"', gal)
    assert len(gps_g2) == 38 and len(sbas_g2) == 39 and len(qzss_g2) == 23, (len(gps_g2), len(sbas_g2), len(qzss_g2))
    assert len(b1c) == 63 and len(l1cp) == 63
    assert len(gal_hex) == 50 and all(len(h) == 1023 for h in gal_hex)

    names = ["GPS_L1_CA_ACR_TABLE", "GALILEO_E1C_ACR_TABLE", "BEIDOU_B1C_ACR_TABLE", "GPS_L1C_ACR_TABLE"]
    acr_tabs = {n: _float_pairs(_block(acr, "pub static " + n)) for n in names}

    L = []
    w = L.append
    w("/* Generated by gen_tables.py from the tart-gnss-acquire v0.4.0 sources. Do not edit. */")
    w("/* Signal-definition (ICD) and ACR calibration tables; see gen_tables.py for provenance. */")
    w("/* The values come from tart-gnss (tmolteno/tart-gnss), licensed GPL-3.0 (its Cargo.toml). */")
    w("#pragma once")
    w("#include <stdint.h>")
    w("")
    w("/* G2 delays: GPS PRN 1-38 (acquisition.rs:84), SBAS 120-158 (sbas.rs:39), QZSS 184-206 (qzss.rs:40). */")
    for nm, arr in (("TGA_GPS_G2_DELAY", gps_g2), ("TGA_SBAS_G2_DELAY", sbas_g2), ("TGA_QZSS_G2_DELAY", qzss_g2)):
        w("static const uint16_t %s[%d] = {%s};" % (nm, len(arr), ", ".join(map(str, arr))))
    w("")
    w("/* Weil (w, p): BeiDou B1C pilot (beidou_codes.rs:46), GPS L1C pilot (l1c_codes.rs:45). */")
    for nm, arr in (("TGA_B1CP_WP", b1c), ("TGA_L1CP_WP", l1cp)):
        w("static const uint16_t %s[63][2] = {" % nm)
        for i in range(0, 63, 6):
            w("  " + " ".join("{%d, %d}," % p for p in arr[i:i + 6]))
        w("};")
    w("")
    w("/* Galileo E1-C primary codes, PRN 1-50, hex MSB-first (galileo_codes.rs:20). */")
    w("static const char* const TGA_GALILEO_E1C_HEX[50] = {")
    for h in gal_hex:
        w('  "%s",' % h.upper())
    w("};")
    w("")
    w("/* ACR r_A -> C/N0 tables (acr_tables.rs): {r_A, dB-Hz} rows, ascending. */")
    for nm in names:
        rows = acr_tabs[nm]
        w("static const double TGA_%s[%d][2] = {" % (nm, len(rows)))
        for a, b in rows:
            w("  {%s, %s}," % (a, b))
        w("};")
    w("")
    open(OUT, "w").write("\n".join(L))
    print("wrote", OUT, {n: len(acr_tabs[n]) for n in names})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_tables.py <reference_src_dir>")
    main(sys.argv[1])
