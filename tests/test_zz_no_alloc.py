"""GPU test of tga_acquire_single_static, the entry point that allocates nothing.

It exists for callers that may not call cudaMalloc while running (real-time
receiver loops, processes whose device memory belongs to another
framework's allocator, hosts that only allow memory reserved at load
time): they pass device buffers and a stream and the search uses a fixed
scratch array inside the library.  The test calls it through the C ABI
twice in a row with different satellites and checks each result against
the context-based tga_acquire_single on the same samples, with the
tolerances of the other parity tests.  This file is collected last so a
failure here never hides the other tests' results; it passes on its own in
a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

import acq_oracle as O
import tga
from parity import REL_TOL, rel
from testutil import phasepoints, quantize_bipolar_demean, synth_signal_cn0

pytestmark = pytest.mark.gpu


def _signal(c, prn, fs, cn0, flip, seed, center=4.092e6):
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    cont = synth_signal_cn0(code, period, (prn * 4099) % period, center - 1500.0, fs, cn0, seed,
                            flip).astype(np.float64)
    sig = quantize_bipolar_demean(cont)
    return sig, phasepoints(fs, len(sig)), period


def _static_call(c, sig, pp, fs, prn, period, band=6000.0, center=4.092e6):
    import torch
    d_sig = torch.from_numpy(np.ascontiguousarray(sig)).cuda()
    d_pp = torch.from_numpy(np.ascontiguousarray(pp)).cuda()
    d_out = torch.zeros(ctypes.sizeof(tga.Result), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = tga.lib().tga_acquire_single_static(c, d_sig.data_ptr(), d_pp.data_ptr(), len(sig), fs, center, band,
                                             prn, period, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    if rc != 0:
        return rc, None
    return rc, tga.Result.from_buffer_copy(d_out.cpu().numpy().tobytes())


# (constellation, PRN, sampling rate, centre frequency, C/N0, sign flip, seed):
# every code generator of the entry point's own chip kernel (C/A G2 delays
# of GPS, SBAS and QZSS, the Galileo E1-C hex codes, the BeiDou B1C and L1C
# Weil codes with the L1C 7-chip insertion) at rates whose search fits the
# scratch array
STATIC_CASES = [
    (tga.GPS, 7, 16.368e6, 4.092e6, 47.0, False, 11),
    (tga.SBAS, 133, 16.368e6, 4.092e6, 50.0, True, 12),
    (tga.QZSS, 195, 16.368e6, 4.092e6, 47.0, True, 14),
    (tga.GALILEO, 19, 4.092e6, 1.023e6, 47.0, False, 15),
    (tga.BEIDOU, 30, 2.046e6, 0.5115e6, 47.0, True, 16),
    (tga.L1C, 12, 2.046e6, 0.5115e6, 47.0, False, 17),
]


def test_static_entry_matches_context_entry_two_calls():
    with tga.Context(0) as ctx:
        for c, prn, fs, center, cn0, flip, seed in STATIC_CASES:  # calls in a row
            sig, pp, period = _signal(c, prn, fs, cn0, flip, seed, center)
            ref = ctx.acquire_single(c, sig, pp, fs, center, 6000.0, prn, period)
            assert ref.path == 0  # the context entry took the same fused search
            for _ in range(2):  # the same call twice: the scratch left behind must not matter
                rc, got = _static_call(c, sig, pp, fs, prn, period, center=center)
                assert rc == 0, (c, rc)
                assert got.prn == prn and got.path == 0
                assert got.best_codephase == ref.best_codephase and got.best_freq_idx == ref.best_freq_idx, c
                assert got.frequency == ref.frequency and got.codephase_frac == ref.codephase_frac
                assert rel(got.signal_strength, ref.signal_strength) <= REL_TOL
                assert rel(got.second_peak, ref.second_peak) <= REL_TOL
                assert got.hypothesis == ref.hypothesis


def test_static_entry_rejects_what_does_not_fit():
    fs = 16.368e6
    sig, pp, period = _signal(tga.BEIDOU, 3, fs, 45.0, False, 13)
    rc, _ = _static_call(tga.BEIDOU, sig, pp, fs, 3, period)  # 41 bins x 2 x 163680 x 8 B > 16 MiB
    assert rc == 7  # TGA_ERR_CAPACITY
    rc, _ = _static_call(tga.GPS, sig[:1000], pp[:1000], fs, 3, 16368)  # not two periods
    assert rc == 5  # TGA_ERR_UNSUPPORTED
    rc, _ = _static_call(tga.GPS, sig, pp, fs, 39, period)  # PRN out of range
    assert rc == 1  # TGA_ERR_INVALID_ARG


def test_static_entry_has_no_generic_fallback():
    # 16 MHz: no whole number of samples per chip.  The context entry answers
    # through its generic path; the static entry has only the fused search.
    fs = 16.0e6
    sig, pp, period = _signal(tga.GPS, 5, fs, 47.0, False, 18)
    with tga.Context(0) as ctx:
        ref = ctx.acquire_single(tga.GPS, sig, pp, fs, 4.092e6, 6000.0, 5, period)
    assert ref.path == 1
    rc, _ = _static_call(tga.GPS, sig, pp, fs, 5, period)
    assert rc == 5  # TGA_ERR_UNSUPPORTED
