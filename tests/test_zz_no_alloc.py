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


def _signal(c, prn, fs, cn0, flip, seed):
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    cont = synth_signal_cn0(code, period, (prn * 4099) % period, 4.092e6 - 1500.0, fs, cn0, seed,
                            flip).astype(np.float64)
    sig = quantize_bipolar_demean(cont)
    return sig, phasepoints(fs, len(sig)), period


def _static_call(c, sig, pp, fs, prn, period, band=6000.0):
    import torch
    d_sig = torch.from_numpy(np.ascontiguousarray(sig)).cuda()
    d_pp = torch.from_numpy(np.ascontiguousarray(pp)).cuda()
    d_out = torch.zeros(ctypes.sizeof(tga.Result), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = tga.lib().tga_acquire_single_static(c, d_sig.data_ptr(), d_pp.data_ptr(), len(sig), fs, 4.092e6, band,
                                             prn, period, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    if rc != 0:
        return rc, None
    return rc, tga.Result.from_buffer_copy(d_out.cpu().numpy().tobytes())


def test_static_entry_matches_context_entry_two_calls():
    fs = 16.368e6
    cases = [(tga.GPS, 7, 47.0, False, 11), (tga.SBAS, 133, 50.0, True, 12)]
    with tga.Context(0) as ctx:
        for c, prn, cn0, flip, seed in cases:  # two calls in a row
            sig, pp, period = _signal(c, prn, fs, cn0, flip, seed)
            ref = ctx.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
            rc, got = _static_call(c, sig, pp, fs, prn, period)
            assert rc == 0, rc
            assert got.prn == prn and got.path == 0
            assert got.best_codephase == ref.best_codephase and got.best_freq_idx == ref.best_freq_idx
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
