"""Parity criteria shared by the GPU tests.

* code-phase sample index and Doppler bin: bit-exact whenever the oracle's
  maximum is unique, i.e. clears every other (bin, code phase) candidate by
  more than TIE_REL relative.  When two candidates tie to within TIE_REL
  (for example the +f and -f bins of a real carrier, which are equal in exact
  arithmetic) the reference's own pick depends on FP rounding order; then
  the GPU's (bin, code phase) must be one of the tied oracle maxima;
* peak metric (signal_strength) and second_peak: within REL_TOL relative;
* detection rule (the reference reports every PRN and has no threshold):
  a PRN is "acquired" on an antenna when signal_strength / second_peak >=
  DETECT_RATIO, i.e. r_A = (V^m/V^s)^2 >= 4 (about 45 dB-Hz on the GPS C/A
  ACR table).  The same rule is applied to the oracle and to the GPU.
"""
import numpy as np

REL_TOL = 1e-4
TIE_REL = 1e-5
DETECT_RATIO = 2.0


def detected(strength, second):
    return second > 0 and strength / second >= DETECT_RATIO


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def assert_cell_parity(gpu, ref, what=""):
    """gpu, ref: dicts/objects with signal_strength, second_peak, best_codephase,
    best_freq_idx (ref = oracle)."""
    g = gpu if isinstance(gpu, dict) else gpu.__dict__
    ref = dict(ref)
    ref.pop("cells", None)
    assert rel(g["signal_strength"], ref["signal_strength"]) <= REL_TOL, (what, g, ref)
    assert rel(g["second_peak"], ref["second_peak"]) <= REL_TOL, (what, g, ref)
    grid = ref.get("grid")
    unique = True
    if grid is not None:
        best = grid[ref["best_freq_idx"], ref["best_codephase"]]
        runner = np.sort(grid.ravel())[-2] if grid.size > 1 else -np.inf
        unique = runner < best * (1.0 - TIE_REL)
    if unique:
        assert g["best_codephase"] == ref["best_codephase"], (what, g, _short(ref))
        assert g["best_freq_idx"] == ref["best_freq_idx"], (what, g, _short(ref))
        assert g["frequency"] == ref["frequency"], (what, g, _short(ref))
        assert g["codephase_frac"] == ref["codephase_frac"], (what, g, _short(ref))
    else:
        v = grid[g["best_freq_idx"], g["best_codephase"]]
        assert v >= grid.max() * (1.0 - TIE_REL), (what, "GPU pick is not one of the tied maxima", g, _short(ref))
    # detection must agree, except for ratios that sit on the threshold itself
    # (within the value tolerance), where either answer is within tolerance
    ratio = ref["signal_strength"] / ref["second_peak"]
    if abs(ratio - DETECT_RATIO) > 3 * REL_TOL * DETECT_RATIO:
        assert detected(g["signal_strength"], g["second_peak"]) == detected(ref["signal_strength"], ref["second_peak"])


def _short(ref):
    return {k: v for k, v in ref.items() if k != "grid"}
