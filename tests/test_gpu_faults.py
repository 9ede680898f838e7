"""Failure detection without a GPU fault.

The cluster kernel's receive wait (an mbarrier counting the bytes the other
CTAs of the cluster push to it) is bounded: when it runs out the kernel
sets the core's status word and finishes, and the host reports an error.
swsgpu_inject makes that happen on purpose from the host side: the next
launch's last job of every cluster sends nothing, so every receiver's wait
for it runs out.  Nothing faults, traps or hangs on the device; the tests
then check that the error reaches the caller on each path (submit/wait,
process_device + sync) and that the same core computes correct spectra
afterwards (the status word is cleared, the context stays usable).
"""
import numpy as np
import pytest

from helpers import REL_TOL, decode_channels, oracle_run, rel_err_auto, rel_err_xpol
from swspec_b200 import synth

pytestmark = pytest.mark.gpu

PREC_OF = {"fp32": 0, "tcsplit": 1, "tcsplit_all": 2}


def _c3_small(gpu, prec):
    N, cof, nfft = 16384, 8, 8
    data, info = synth.c3_stream(nfft, N=N, npairs=1, seed=77)
    lay = gpu.layout("mark5b", info["nchan"], 2)
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 0), (0, 1)), xpols=((0, 1),),
                          max_run_bytes=len(data), samplingfreq=64e6, precision=PREC_OF[prec])
    return cfg, data, info, N, cof


def _check_against_oracle(auto, xp, data, info, N, cof):
    s = decode_channels(data, info["fmt"], info["nchan"], 2, [0, 1], info["nsamp"])
    ra, rx, _, n = oracle_run(s, N, "hann", 1, cof, nxpols=1)
    assert n == auto.shape[0]
    assert rel_err_auto(auto, ra) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


@pytest.mark.parametrize("prec", ["fp32", "tcsplit"])
def test_dropped_exchange_fails_the_wait_then_recovers(gpu, prec):
    cfg, data, info, N, cof = _c3_small(gpu, prec)
    core = gpu.Core(cfg)
    core.inject(gpu.INJECT_DROP_EXCHANGE)
    with pytest.raises(gpu.SwsError, match="ECUDA: a device-side wait .* gave up"):
        core.run([data])
    # the injection is one-shot and the status word was cleared by the failed wait
    auto, xp, _, ns = core.run([data])
    assert ns == 1
    _check_against_oracle(auto, xp, data, info, N, cof)


def test_dropped_exchange_reported_by_sync_on_process_device(gpu):
    import torch
    cfg, data, info, N, cof = _c3_small(gpu, "fp32")
    lay = cfg.layout[0]
    core = gpu.Core(cfg)
    S = N // 2 + 1
    raw = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda()
    pay = len(data) // lay.frame_bytes * (lay.frame_bytes - lay.header_bytes)
    d_auto = torch.zeros(2, S, device="cuda")
    d_xpol = torch.zeros(1, S, 2, device="cuda")
    core.inject(gpu.INJECT_DROP_EXCHANGE)
    core.process_device([raw.data_ptr()], pay, 1, 1, d_auto.data_ptr(), d_xpol.data_ptr())
    with pytest.raises(gpu.SwsError, match="gave up"):
        core.sync()
    core.process_device([raw.data_ptr()], pay, 1, 1, d_auto.data_ptr(), d_xpol.data_ptr())
    core.sync()
    auto = d_auto.cpu().numpy()[None]
    xp = d_xpol.cpu().numpy()
    xp = (xp[..., 0] + 1j * xp[..., 1])[None]
    _check_against_oracle(auto, xp, data, info, N, cof)


def test_inject_rejects_unknown_kind_and_four_step(gpu):
    cfg, _, _, _, _ = _c3_small(gpu, "fp32")
    core = gpu.Core(cfg)
    with pytest.raises(gpu.SwsError, match="EINVAL"):
        core.inject(7)
    lay = gpu.layout("vdif:8000", 1, 8)
    big = gpu.Core(gpu.make_config(lay, 1 << 20, max_run_bytes=1 << 22))
    with pytest.raises(gpu.SwsError, match="four-step"):
        big.inject(gpu.INJECT_DROP_EXCHANGE)
