"""Batched uneven streams through one CUDA graph, and the autotuner.

Cores of different FFT lengths (cluster and four-step paths) and bit depths
are recorded into one graph (swsgpu_batch_*); a replay must give the same
spectra, bit for bit, as each core's own process_device run (the kernels
are deterministic without phase-cal), every core's spectra must meet the
FP64 oracle, and the autotuned four-step split must stay within the parity
bars of the four-step tests."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, oracle_run
from swspec_b200.workloads import StreamSpec, stream_payload
from test_gpu_bigfft import _check_auto, _fp32_run

pytestmark = pytest.mark.gpu

# (N, bits, FFTs per run): every plan family and both bit depths
MIX = [(4096, 2, 16), (20000, 1, 3), (131072, 2, 2), (1 << 18, 1, 2), (1 << 20, 2, 2), (3_200_000, 1, 2)]


def _spec(i, N, nbit, cof):
    run_bytes = (N * cof * nbit // 8 + 7) // 8 * 8
    return StreamSpec(i, N, nbit, 16e6, 1.0, 1, (3.1e6,), run_bytes, cof, 1)


def _core(gpu, spec, autotune=False):
    lay = gpu.layout("vdif:8000", 1, spec.nbit, framed=False)
    cfg = gpu.make_config(lay, spec.fft_points, "hann", 1, spec.core_overlapped_ffts,
                          max_run_bytes=spec.run_bytes, samplingfreq=spec.samplingfreq,
                          autotune=autotune)
    return gpu.Core(cfg)


def test_batch_graph_equals_eager(gpu):
    specs = [_spec(i, *m) for i, m in enumerate(MIX)]
    cores = [_core(gpu, s) for s in specs]
    raws, outs_e, outs_b = [], [], []
    for s, c in zip(specs, cores):
        pay = np.frombuffer(stream_payload(s), dtype=np.uint8)
        raws.append(torch.from_numpy(pay.copy()).cuda())
        ns, _, _ = c.run_shape(s.run_bytes)
        outs_e.append(torch.zeros(ns, 1, c.S, dtype=torch.float32, device="cuda"))
        outs_b.append(torch.zeros(ns, 1, c.S, dtype=torch.float32, device="cuda"))
    for s, c, r, o in zip(specs, cores, raws, outs_e):
        c.process_device([r.data_ptr()], s.run_bytes, 1, 1, o.data_ptr())
    torch.cuda.synchronize()
    b = gpu.Batch(cores)
    for i, (s, r, o) in enumerate(zip(specs, raws, outs_b)):
        b.set(i, [r.data_ptr()], s.run_bytes, 1, 1, o.data_ptr())
    k = b.launch()                     # eager pass + graph recording
    torch.cuda.synchronize()
    assert k >= 4 * len(cores)
    for e, o in zip(outs_e, outs_b):
        assert torch.equal(e, o)
    st = torch.cuda.Stream()
    for rep in range(2):               # graph replays
        for o in outs_b:
            o.zero_()
        torch.cuda.synchronize()
        b.launch(st.cuda_stream)
        st.synchronize()
        for e, o in zip(outs_e, outs_b):
            assert torch.equal(e, o), rep
    b.close()
    # every core of the batch against the FP64 oracle: per bin at the 2e-6
    # bar with 16 FFTs per spectrum; with 2 or 3 FFTs (chi-square spectra
    # with bins near zero, and at the longer lengths an FP32 rounding noise
    # that the reference's own FP32 arithmetic shares) at the four-step
    # tests' bars, relative to max(bin, median bin) and to the FP32 CPU
    # restatement of doMaths
    for s, got in zip(specs, outs_b):
        x = O.decode(O.FMT_VDIF, 1, s.nbit, stream_payload(s), s.samples_per_run, 0, payload_bytes=8000)
        ra, _, _, nref = oracle_run([x], s.fft_points, "hann", 1, s.core_overlapped_ffts)
        g = got.cpu().numpy()
        assert g.shape[0] == nref, s.fft_points
        if s.core_overlapped_ffts >= 16:
            assert np.max(np.abs(g[0, 0] - ra[0, 0]) / ra[0, 0]) < REL_TOL, s.fft_points
        else:
            r32, _, _, _ = _fp32_run([x], s.fft_points, "hann", 1, s.core_overlapped_ffts)
            _check_auto(g[0, 0], ra[0, 0], r32[0, 0], per_bin=False)


def test_batch_rejects_unset_and_duplicate(gpu):
    s = _spec(0, 4096, 2, 4)
    c = _core(gpu, s)
    with pytest.raises(gpu.SwsError):
        gpu.Batch([c, c])
    b = gpu.Batch([c])
    with pytest.raises(gpu.SwsError, match="no work"):
        b.launch()
    b.close()


def test_autotune_four_step(gpu):
    """2^20, 1-bit: every candidate split is timed, the fastest kept; the
    result stays within the four-step parity bars; a later core of the same
    length and bits starts from the tuned split."""
    N, cof = 1 << 20, 3
    s = _spec(0, N, 1, cof)
    s.run_bytes = (N * (cof + 1) // 8 + 7) // 8 * 8
    c = _core(gpu, s, autotune=True)
    info = c.plan_info()
    assert "tuned" in info and "four-step" in info, info
    pay = stream_payload(s)
    auto, _, _, ns = c.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 1, pay, s.samples_per_run, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, cof)
    r32, _, _, _ = _fp32_run([x], N, "hann", 1, cof)
    assert ns == nref
    _check_auto(auto[0, 0], ra[0, 0], r32[0, 0])
    c2 = _core(gpu, s)
    assert c2.plan_info() == info
    # a cluster length with one plan keeps it
    c3 = _core(gpu, _spec(1, 65536, 2, 2))
    assert "candidate 0 of 1" in c3.autotune()


# cluster plans per length, as the autotuner numbers them
CLUSTER_CANDIDATES = {4096: 3, 20000: 2, 131072: 2}


@pytest.mark.parametrize("N,k", [(N, k) for N, n in CLUSTER_CANDIDATES.items() for k in range(n)])
def test_every_cluster_candidate(gpu, N, k):
    """Each cluster plan the autotuner may choose (cluster size, threads per
    CTA, radix order), pinned through plan_candidate: 16 FFTs of a 2-bit
    stream against the FP64 oracle at the 2e-6 bar in every bin."""
    s = _spec(k, N, 2, 16)
    lay = gpu.layout("vdif:8000", 1, 2, framed=False)
    cfg = gpu.make_config(lay, N, "hann", 1, 16, max_run_bytes=s.run_bytes, samplingfreq=s.samplingfreq,
                          plan_candidate=k)
    c = gpu.Core(cfg)
    info = c.plan_info()
    assert f"candidate {k} of {CLUSTER_CANDIDATES[N]}" in info and "cluster" in info, info
    pay = stream_payload(s)
    auto, _, _, ns = c.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 2, pay, s.samples_per_run, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, 16)
    assert ns == nref == 1
    assert np.max(np.abs(auto[0, 0] - ra[0, 0]) / ra[0, 0]) < REL_TOL, info
    c.close()


def test_autotune_cluster_plans(gpu):
    """N = 4096, 2-bit: the three cluster plans are timed on one run of
    max_run_bytes, the fastest is kept and meets the bar; a later core of
    the same length, bits and form starts from it; a pinned candidate
    beyond the list is refused."""
    N, cof = 4096, 64
    s = _spec(0, N, 2, cof)
    c = _core(gpu, s, autotune=True)
    info = c.plan_info()
    assert "tuned" in info and "of 3" in info, info
    pay = stream_payload(s)
    auto, _, _, ns = c.run([pay])
    x = O.decode(O.FMT_VDIF, 1, 2, pay, s.samples_per_run, 0, payload_bytes=8000)
    ra, _, _, nref = oracle_run([x], N, "hann", 1, cof)
    assert ns == nref == 1
    assert np.max(np.abs(auto[0, 0] - ra[0, 0]) / ra[0, 0]) < REL_TOL
    assert _core(gpu, s).plan_info() == info
    lay = gpu.layout("vdif:8000", 1, 2, framed=False)
    with pytest.raises(gpu.SwsError, match="beyond"):
        gpu.Core(gpu.make_config(lay, N, "hann", 1, cof, max_run_bytes=s.run_bytes, plan_candidate=3))
