#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference crate.

Run in the build container (where the reference checkout exists):
    python tests/golden/make_golden.py [/path/to/tart-gnss]

Outputs (committed; the GPU box never reads the reference):
* kats.json -- known-answer vectors copied from the reference's own unit
  tests: BeiDou B1C pilot first/last 24 chips in octal for PRN 1-63
  (src/beidou_codes.rs:225-253), GPS L1C pilot first/last 24 chips
  (src/l1c_codes.rs:256-289), SBAS first 10 chips (src/sbas.rs:436-442),
  QZSS first 10 chips (src/qzss.rs:437-441), and the ACR mid-range points
  (src/acr.rs:150-154).
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
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
