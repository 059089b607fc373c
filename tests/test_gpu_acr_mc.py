"""ACR table Monte Carlo on the GPU (tga_acr_table) against the tables the
reference ships (acr_tables.rs, generated by examples/gen_acr_tables.rs with
the same seeds): the GPU synthesizer replays the reference generator's random
streams, and the batched search replaces the reference's acquisition."""
import os
import re

import numpy as np
import pytest

import tga

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
# (constellation, shipped table, first C/N0, last C/N0) as gen_acr_tables.rs:175-211
SPECS = [(tga.GPS, "TGA_GPS_L1_CA_ACR_TABLE", 33.0, 62.0), (tga.GALILEO, "TGA_GALILEO_E1C_ACR_TABLE", 27.0, 62.0),
         (tga.BEIDOU, "TGA_BEIDOU_B1C_ACR_TABLE", 23.0, 62.0), (tga.L1C, "TGA_GPS_L1C_ACR_TABLE", 23.0, 62.0)]


def shipped(name):
    text = open(os.path.join(HERE, "..", "tart-gnss_b200", "csrc", "gnss_tables.h")).read()
    body = text[text.index(name):]
    body = body[body.index("{") + 1: body.index("};")]
    return np.array([[float(a), float(b)] for a, b in re.findall(r"\{\s*([-0-9.eE+]+)\s*,\s*([-0-9.eE+]+)\s*\}", body)])


@pytest.mark.parametrize("c,name,lo,hi", SPECS, ids=["gps", "galileo", "beidou", "l1c"])
def test_acr_table_regenerates_the_shipped_table(c, name, lo, hi, capsys):
    want = shipped(name)
    with tga.Context(0) as ctx:
        got = ctx.acr_table(c, 1, 16.368e6, lo, hi, 0.5, 100)
    assert got.shape == want.shape
    assert np.array_equal(got[:, 1], want[:, 1])
    rounded = np.round(got[:, 0], 4)
    dev = np.abs(rounded - want[:, 0])
    rel = dev / want[:, 0]
    with capsys.disabled():
        print("\n%s: %d points, %d identical to 4 decimals, max |dr_A| %.2e (rel %.2e)"
              % (name, len(want), int((dev < 5e-5).sum()), dev.max(), rel.max()))
    assert dev.max() <= 1.0001e-4  # at most one unit in the last printed digit
    assert (dev < 5e-5).mean() >= 0.95
