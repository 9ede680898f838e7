"""Edge cases of a core run through the TaskCore path (submit / wait /
fetch): empty and ragged buffers, a buffer shorter than one FFT, a buffer
of exactly max_run_bytes, two streams of unequal length, and one sample
past the last whole spectrum -- each against the FP64 oracle over the same
samples (TaskCoreIPP::doMaths, src/IA-32/TaskCoreIPP.cpp:355-560: the FFTs
that fit, whole spectra of core_overlapped_ffts FFTs scaled, a trailing
partial spectrum unscaled)."""
import numpy as np
import pytest

import oracle as O
from helpers import REL_TOL, oracle_run

pytestmark = pytest.mark.gpu

N, COF = 4096, 4


def _payload(nbytes, seed):
    return np.random.default_rng(seed).integers(0, 256, nbytes, dtype=np.uint8).tobytes()


def _core(gpu, max_run, nsrc=1, xp=False):
    lay = gpu.layout("vdif:8000", 1, 2, framed=False)
    sources = tuple((s, 0) for s in range(nsrc))
    cfg = gpu.make_config(lay, N, "hann", 1, COF, sources=sources,
                          xpols=((0, 1),) if xp else (), max_run_bytes=max_run)
    return gpu.Core(cfg)


def _check(auto, ra):
    assert auto.shape[0] == ra.shape[0]
    for k in range(ra.shape[0]):
        for s in range(ra.shape[1]):
            assert np.max(np.abs(auto[k, s] - ra[k, s]) / ra[k, s]) < REL_TOL, (k, s)


def test_empty_buffer_gives_no_spectrum(gpu):
    core = _core(gpu, 1 << 16)
    auto, _, _, ns = core.run([b""])
    assert ns == 0 and auto.shape[0] == 0
    # the core stays usable
    pay = _payload(N * COF // 4, 1)
    auto, _, _, ns = core.run([pay])
    assert ns == 1


def test_shorter_than_one_fft(gpu):
    core = _core(gpu, 1 << 16)
    pay = _payload(N // 4 - 4, 2)            # N - 16 samples
    auto, _, _, ns = core.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 2, pay, len(pay) * 4, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, COF)
    assert ns == nref == 0


@pytest.mark.parametrize("nsamp", [N * COF + 1, N * COF * 2 + N * 2 + 16, N * 3 + 4 * 5])
def test_ragged_buffers(gpu, nsamp):
    """Whole spectra, then a partial one of the FFTs that fit (unscaled, as
    the reference leaves it), trailing samples that fill no FFT ignored."""
    nbytes = (nsamp + 3) // 4
    pay = _payload(nbytes, nsamp)
    core = _core(gpu, 1 << 16)
    auto, _, _, ns = core.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 2, pay, nbytes * 4, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, COF)
    assert ns == nref
    _check(auto, ra)


def test_buffer_of_exactly_max_run_bytes(gpu):
    max_run = N * COF * 3 // 4               # three whole spectra
    core = _core(gpu, max_run)
    pay = _payload(max_run, 9)
    auto, _, _, ns = core.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 2, pay, max_run * 4, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, COF)
    assert ns == nref == 3
    _check(auto, ra)


def test_unequal_streams_use_the_shorter(gpu):
    """Two input buffers of different length: the run walks the samples both
    hold (the reference sizes a run by its smallest source buffer)."""
    a = _payload(N * COF * 2 // 4, 11)
    b = _payload(N * COF // 4 + 1000, 12)
    core = _core(gpu, 1 << 16, nsrc=2, xp=True)
    auto, xp, _, ns = core.run([a, b])
    m = min(len(a), len(b)) * 4
    xa = O.decode(O.FMT_VDIF, 1, 2, a, m, 0, payload_bytes=8000)
    xb = O.decode(O.FMT_VDIF, 1, 2, b, m, 0, payload_bytes=8000)
    ra, rx, _, nref = oracle_run([xa, xb], N, "hann", 1, COF, nxpols=1)
    assert ns == nref
    _check(auto, ra)
    for k in range(nref):
        norm = np.sqrt(ra[k, 0] * ra[k, 1])
        assert np.max(np.abs(xp[k, 0] - rx[k, 0]) / norm) < REL_TOL


def test_oversized_buffer_rejected(gpu):
    core = _core(gpu, 1 << 14)
    with pytest.raises(gpu.SwsError, match="max_run_bytes"):
        core.run([_payload((1 << 14) * 2, 3)])
    # still usable afterwards
    auto, _, _, ns = core.run([_payload(N * COF // 4, 4)])
    assert ns == 1
