"""HDF5 ingest (tga_observation_read_hdf5, Observation::from_hdf5
observation.rs:48-92) on a cut-down copy of the reference's real TART file,
and the CLI's argument handling (main.rs:61-210) where no GPU is needed."""
import os
import subprocess

import numpy as np
import pytest

import tga
from tga import TgaError

HERE = os.path.dirname(__file__)
FIXTURE = os.path.join(HERE, "golden", "tart_head4096.hdf")
CLI = os.path.join(HERE, "..", "tart-gnss_b200", "tart-gnss-acquire")


def test_reads_the_reference_layout():
    o = tga.read_hdf5(FIXTURE)
    assert o["num_antenna"] == 24 and o["row_bytes"] == 4096
    assert o["sampling_frequency"] == 16.368e6
    assert o["timestamp"] == "2026-03-09T04:25:10.145497+00:00"
    assert '"num_antenna": 24' in o["config"]
    head = np.load(os.path.join(HERE, "golden", "tart_head.npz"))["head"]
    assert np.array_equal(o["data"], head[:, :4096])


def test_missing_and_corrupt_files_fail_cleanly(tmp_path):
    with pytest.raises(TgaError):
        tga.read_hdf5(tmp_path / "missing.hdf")
    bad = tmp_path / "cut.hdf"
    bad.write_bytes(open(FIXTURE, "rb").read()[:3000])  # metadata cut short
    with pytest.raises(TgaError):
        tga.read_hdf5(bad)
    junk = tmp_path / "junk.hdf"
    junk.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(TgaError):
        tga.read_hdf5(junk)


@pytest.mark.parametrize("args,msg", [(["--rfi", "--benchmark"], "--rfi cannot be combined with --benchmark"),
                                      (["--rfi", "--i", "0", "--j", "1"], "--rfi cannot be combined with --i/--j"),
                                      (["--rfi", "--test-antennas"], "--rfi cannot be combined with --test-antennas"),
                                      (["--gps", "--precision", "fp64"], "invalid value for --precision: fp64"),
                                      (["--gps", "--noncoh", "0"], "invalid positive integer for --noncoh: 0"),
                                      (["--gps", "--coherent-periods", "x"], "invalid positive integer for"),
                                      (["--gps", "--bin-hz", "50"], "--bin-hz sets the non-coherent search's grid"),
                                      (["--gps", "--noncoh", "2", "--bin-hz", "-5"], "invalid positive float"),
                                      (["--rfi", "--noncoh", "2"], "apply to the acquisition search only"),
                                      (["--benchmark", "--refine"], "--refine applies to the acquisition search")])
def test_cli_rejects_conflicting_modes(args, msg):
    if not os.path.exists(CLI):
        pytest.skip("CLI not built")
    r = subprocess.run([CLI, "--file", FIXTURE] + args, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and msg in r.stderr
