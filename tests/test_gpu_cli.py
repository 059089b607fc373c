"""The tart-gnss-acquire CLI end to end on a cut-down copy of the reference's
real TART recording: acquisition JSON (--gps --cn0) and the RFI report
(--rfi) equal what the library produces for the same rows."""
import json
import os
import subprocess

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
