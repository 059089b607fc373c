"""The tart-gnss-acquire CLI end to end on a cut-down copy of the reference's
real TART recording: acquisition JSON (--gps --cn0) and the RFI report
(--rfi) equal what the library produces for the same rows; --benchmark
prints the reference's schema, and tga_benchmark's searches equal the
single-PRN calls they time; the engine's own flags (--precision,
--coherent-periods / --noncoh / --bin-hz, --refine) give the library's
results."""
import json
import os
import subprocess

import numpy as np
import pytest

import tga

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
FIXTURE = os.path.join(HERE, "golden", "tart_head4096.hdf")
CLI = os.path.join(HERE, "..", "tart-gnss_b200", "tart-gnss-acquire")


def _run(args):
    r = subprocess.run([CLI, "--file", FIXTURE] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip()


def test_cli_gps_acquisition_json():
    out = _run(["--gps", "--cn0"])
    o = tga.read_hdf5(FIXTURE)
    with tga.Context(0) as ctx:
        want = ctx.acquire_json(o["data"], o["sampling_frequency"], mask=1 << tga.GPS, cn0=True)
    assert out == want.strip()
    doc = json.loads(out)
    assert len(doc["gps"]["results"]) == 38 and doc["gps"]["antenna_numbers"] == list(range(24))


def test_cli_rfi_json(tmp_path):
    path = tmp_path / "rfi.json"
    r = subprocess.run([CLI, "--file", FIXTURE, "--rfi", "--output", str(path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Wrote RFI JSON to" in r.stderr
    o = tga.read_hdf5(FIXTURE)
    with tga.Context(0) as ctx:
        want = ctx.rfi_scan(o["data"], o["sampling_frequency"], as_json=True)
    assert open(path).read().strip() == want.strip()
    assert len(json.loads(want)["channels"]) == 24


def test_cli_benchmark_schema():
    doc = json.loads(_run(["--benchmark"]))
    assert [d["constellation"] for d in doc] == ["GPS", "Galileo", "BeiDou", "SBAS", "QZSS", "L1C"]
    for d in doc:
        assert list(d) == ["constellation", "prns", "setup_s", "search_s", "duration_s"]
        assert d["prns"] == 1 and d["search_s"] > 0 and d["setup_s"] >= 0
        assert abs(d["duration_s"] - d["setup_s"] - d["search_s"]) < 1e-9


def test_library_benchmark_equals_single_prn_calls():
    import numpy as np
    o = tga.read_hdf5(FIXTURE)
    bits, fs = o["data"], o["sampling_frequency"]
    with tga.Context(0) as ctx:
        entries = ctx.benchmark(bits, fs)
        assert [(e["constellation"], e["prn"]) for e in entries] == [
            (tga.GPS, 1), (tga.GALILEO, 1), (tga.BEIDOU, 1), (tga.SBAS, 120), (tga.QZSS, 184), (tga.L1C, 1)]
        ub = np.unpackbits(bits[0]).astype(np.float64) * 2 - 1
        sig_all = (ub - ub.mean()).astype(np.float32)
        for e in entries:
            per = {tga.GALILEO: int(fs * (4092.0 / 1.023e6)), tga.BEIDOU: int(fs * (10230.0 / 1.023e6)),
                   tga.L1C: int(fs * (10230.0 / 1.023e6))}.get(e["constellation"], int(fs / 1000.0))
            n = min(2 * per, len(sig_all))
            pp = 2 * np.pi / fs * np.arange(n)
            r = ctx.acquire_single(e["constellation"], sig_all[:n], pp, fs, 4.092e6, 6000.0, e["prn"], per)
            g = e["result"]
            assert (g.best_codephase, g.best_freq_idx, g.hypothesis) == (r.best_codephase, r.best_freq_idx,
                                                                         r.hypothesis)
            assert g.signal_strength == r.signal_strength and g.second_peak == r.second_peak
            assert e["search_s"] > 0


def test_cli_precision_fp16tc_same_json():
    """--precision fp16tc: the tensor-core search gives the same JSON as the
    default FP32 search (every cell equal)."""
    assert _run(["--gps", "--galileo", "--cn0", "--precision", "fp16tc"]) == _run(["--gps", "--galileo", "--cn0"])


def test_cli_noncoherent_matches_library():
    """--coherent-periods / --noncoh / --bin-hz: the non-coherent search of
    the selected constellations through tga_search_noncoherent_multi, the
    JSON fields equal to the library's cells."""
    doc = json.loads(_run(["--gps", "--sbas", "--coherent-periods", "1", "--noncoh", "2", "--bin-hz", "250"]))
    assert list(doc) == ["gps", "sbas"]
    o = tga.read_hdf5(FIXTURE)
    fs = o["sampling_frequency"]
    with tga.Context(0) as ctx:
        want = ctx.search_noncoherent_multi(o["data"], fs, [
            dict(constellation=c, center_freq=4.092e6, bin_step_hz=250.0, n_bins=49, coherent_periods=1, blocks=2)
            for c in (tga.GPS, tga.SBAS)])
    for key, cells, first in (("gps", want[0], 1), ("sbas", want[1], 120)):
        g = doc[key]
        assert g["antenna_numbers"] == list(range(24)) and g["coherent_periods"] == 1 and g["blocks"] == 2
        assert g["bin_hz"] == 250.0
        assert [r["sv"] for r in g["results"]] == sorted(r["sv"] for r in g["results"])
        for r in g["results"]:
            prn = int(r["sv"].lstrip("GPSBA"))
            rows = cells[cells["prn"] == prn]
            assert r["powers"] == rows["power"].tolist() and r["freqs"] == rows["frequency"].tolist()
            assert r["phases"] == (rows["best_codephase"] / 16368.0).tolist()
            assert np.array_equal(r["second_powers"], rows["second_power"])


def test_cli_refine_adds_refined_satellites():
    """--refine: every satellite detected on some antenna is refined from
    its strongest antenna's grid estimate (tga_fine_acquire over the two
    search periods); the default output is unchanged apart from the added
    field."""
    base = json.loads(_run(["--gps"]))
    doc = json.loads(_run(["--gps", "--refine"]))
    assert list(doc) == ["gps", "refined"] and doc["gps"] == base["gps"]
    o = tga.read_hdf5(FIXTURE)
    fs = o["sampling_frequency"]
    with tga.Context(0) as ctx:
        cells = ctx.acquire_cells(o["data"], fs, mask=1 << tga.GPS)
        tasks = []
        for prn in sorted(set(cells["prn"].tolist())):
            rows = cells[cells["prn"] == prn]
            b = rows[int(np.argmax(rows["signal_strength"]))]
            if b["signal_strength"] >= 2.0 * b["second_peak"]:
                tasks.append((tga.GPS, prn, float(b["best_codephase"]), 4.092e6 + float(b["frequency"]), 0,
                              2 * 16368))
        res, _ = ctx.fine_acquire(o["data"], fs, tasks)
    assert len(doc["refined"]) == len(tasks) > 0
    for r, t, f in zip(doc["refined"], tasks, res):
        assert r["sv"] == "GPS%02d" % t[1]
        assert r["code_phase_samples"] == f["code_phase"] and r["frequency"] == f["frequency"] - 4.092e6
        assert r["converged"] == bool(f["converged"])
