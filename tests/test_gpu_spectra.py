"""GPU parity: spectra of the CUDA core vs the FP64 oracle (restated doMaths).

Each case runs one core run (one raw buffer per stream) through the C ABI
(swsgpu_submit / wait / fetch) and compares every auto spectrum, cross
spectrum and phase-cal vector with the FP64 restatement of
TaskCoreIPP::doMaths on the same decoded samples.
"""
import numpy as np
import pytest

from helpers import REL_TOL, decode_channels, fill_zone, oracle_run, payload_of, rel_err_auto, rel_err_xpol
from swspec_b200 import synth

pytestmark = pytest.mark.gpu

# the plain FP32 form and the two tensor-core split forms (tcgen05 levels
# 2-3 with an FP32 level 1, or all three local levels)
PRECS = ["fp32", "tcsplit", "tcsplit_all"]
PREC_OF = {"fp32": 0, "tcsplit": 1, "tcsplit_all": 2}


def _mark5b_noise(nchan, nbit, nframes_m5b, seed, mbps=1024):
    spf = synth.mark5b_samples_per_frame(nchan, nbit)
    T = spf * nframes_m5b
    rng = np.random.default_rng(seed)
    sig = rng.standard_normal((nchan, T))
    return synth.mark5b_stream(sig, nbit, mbps), T


@pytest.mark.parametrize("prec", PRECS)
def test_c1_like_auto_single_channel(gpu, prec):
    """16 ch x 2 bit Mark5B, channel 1 only, N=32768 Hann, 16 FFTs per spectrum
    (the default buffer plan's core run), tone at +3.1 MHz; both FFT forms."""
    N, cof = 32768, 16
    precision = PREC_OF[prec]
    data, info = synth.c1_stream(0, frames=int(np.ceil(N * cof / 2500)) + 1, N=N)
    lay = gpu.layout("mark5b", 16, 2)
    run_bytes_payload = N * cof * 4
    nfr = run_bytes_payload // 10000 + 1
    raw = data[: nfr * 10016]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 0),), max_run_bytes=len(raw),
                          precision=precision)
    core = gpu.Core(cfg)
    auto, _, _, ns = core.run([raw])
    samples = decode_channels(raw, info["fmt"], 16, 2, [0], nfr * 2500)
    ref, _, _, nref = oracle_run(samples, N, "hann", 1, cof)
    assert ns == nref == 1
    err = rel_err_auto(auto, ref)
    assert err < REL_TOL, err


@pytest.mark.parametrize("prec", PRECS)
def test_c3_like_dual_pol_cross(gpu, prec):
    """Mark5B-2048-16-2, 8 subband pairs (c, c+8), N=65536, XX/YY/XY*; both
    the plain FP32 form and the tensor-core split form meet the bar."""
    N, cof, nfft = 65536, 16, 16
    precision = PREC_OF[prec]
    data, info = synth.c3_stream(nfft, N=N)
    lay = gpu.layout("mark5b", 16, 2)
    pairs = [(c, c + 8) for c in range(8)]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=tuple((0, c) for c in range(16)),
                          xpols=pairs, max_run_bytes=len(data), samplingfreq=64e6,
                          precision=precision)
    core = gpu.Core(cfg)
    nsamp = info["nsamp"]
    auto, xp, _, ns = core.run([data])
    assert ns == 1
    samples = decode_channels(data, info["fmt"], 16, 2, range(16), nsamp)
    worst = 0.0
    for k, (i, j) in enumerate(pairs):
        ra, rx, _, n = oracle_run([samples[i], samples[j]], N, "hann", 1, cof, nxpols=1)
        assert n == 1
        worst = max(worst, rel_err_auto(auto[:, i], ra[:, 0]), rel_err_auto(auto[:, j], ra[:, 1]),
                    rel_err_xpol(xp[:, k], rx[:, 0], ra[:, 0], ra[:, 1]))
    assert worst < REL_TOL, worst
    # the synthesised cross-correlation is rho = 0.3 at 0.7 rad; 2-bit
    # quantisation at +-0.98 sigma scales |rho| by ~0.88 (Van Vleck)
    rho = np.mean(xp[0, 0, 100:-100] / np.sqrt(auto[0, 0, 100:-100] * auto[0, 8, 100:-100]))
    assert abs(abs(rho) - 0.3 * 0.88) < 0.02 and abs(abs(np.angle(rho)) - 0.7) < 0.1


@pytest.mark.parametrize("overlap,cof", [(2, 7), (1, 5), (4, 9)])
def test_two_files_overlap_partial(gpu, overlap, cof):
    """Two input files (streams), channel 3 of each, cross-pol, overlapped FFTs,
    spectrum hop and a trailing unscaled partial spectrum."""
    N = 4096
    d1, T = _mark5b_noise(8, 2, 12, 11)
    d2, _ = _mark5b_noise(8, 2, 12, 12)
    lay = gpu.layout("mark5b", 8, 2)
    cfg = gpu.make_config(lay, N, "cosine2", overlap, cof, sources=((0, 2), (1, 2)),
                          xpols=((0, 1),), max_run_bytes=len(d1))
    core = gpu.Core(cfg)
    auto, xp, _, ns = core.run([d1, d2])
    s1 = decode_channels(d1, "Mark5B-1024-8-2", 8, 2, [2], T)[0]
    s2 = decode_channels(d2, "Mark5B-1024-8-2", 8, 2, [2], T)[0]
    ra, rx, _, nref = oracle_run([s1, s2], N, "cosine2", overlap, cof, nxpols=1)
    assert ns == nref and ns >= 2
    assert rel_err_auto(auto, ra) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


@pytest.mark.parametrize("nbit,nchan,window", [(1, 16, "none"), (1, 32, "cosine"),
                                               (2, 4, "hamming"), (2, 1, "blackman")])
def test_bit_depths_and_windows(gpu, nbit, nchan, window):
    """Integrated spectra (32 FFTs) at the 2e-6 max-relative bar.  FP32 FFT
    error is absolute, so the bar is meant for integrated spectra; the
    short-integration case below checks the error against the spectrum level."""
    N, cof = 8192, 32
    spf = synth.mark5b_samples_per_frame(nchan, nbit)
    nfr = N * cof // spf + 1
    d, T = _mark5b_noise(nchan, nbit, nfr, 21 + nbit + nchan,
                         mbps=1024 if nchan * nbit >= 8 else 256)
    lay = gpu.layout("mark5b", nchan, nbit)
    ch = nchan - 1
    cfg = gpu.make_config(lay, N, window, 1, cof, sources=((0, ch),), max_run_bytes=len(d))
    core = gpu.Core(cfg)
    auto, _, _, ns = core.run([d])
    fmt = f"Mark5B-{1024 if nchan * nbit >= 8 else 256}-{nchan}-{nbit}"
    s = decode_channels(d, fmt, nchan, nbit, [ch], T)
    ra, _, _, nref = oracle_run(s, N, window, 1, cof)
    assert ns == nref
    assert rel_err_auto(auto, ra) < REL_TOL


def test_vdif_8bit_blackmanharris(gpu):
    """VDIF 8-bit single channel (dynamic-range configuration's format)."""
    N, cof = 20000, 3
    spf = 8000
    rng = np.random.default_rng(1005)
    x = rng.standard_normal(spf * 9)
    codes = synth.quantize_vdif_8bit(x, 24.0)
    payload = synth.pack_codes(codes[None, :], 8)
    data = synth.vdif_frames(payload, 8000, 1, 8, 8000)
    lay = gpu.layout("vdif:8000", 1, 8)
    cfg = gpu.make_config(lay, N, "blackmanharris", 1, cof, max_run_bytes=len(data))
    core = gpu.Core(cfg)
    auto, _, _, ns = core.run([data])
    s = decode_channels(data, "VDIF_8000-512-1-8", 1, 8, [0], spf * 9)
    ra, _, _, nref = oracle_run(s, N, "blackmanharris", 1, cof)
    assert ns == nref
    assert rel_err_auto(auto, ra) < REL_TOL


def test_pcal_fold(gpu):
    """Phase-cal folding (offset 15625 Hz at 32 Msps: rotator period 2048,
    32 tone bins) on every FFT, comb amplitude 5% of sigma."""
    N, cof, fs, off = 32768, 4, 32e6, 15625.0
    spf = 2500
    nfr = N * cof // spf + 2
    T = nfr * spf
    rng = np.random.default_rng(7)
    comb = synth.pcal_comb(T, fs, 1e6, off, 0.05, rng.uniform(0, 2 * np.pi, 16))
    sig = rng.standard_normal((16, T)) + comb[None, :]
    data = synth.mark5b_stream(sig, 2, 1024)
    lay = gpu.layout("mark5b", 16, 2)
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 4),), max_run_bytes=len(data),
                          extract_pcal=True, pcal_tonebins=32, pcal_rotatorlen=2048,
                          samplingfreq=fs, pcal_offset_hz=off)
    core = gpu.Core(cfg)
    auto, _, pc, ns = core.run([data])
    s = decode_channels(data, "Mark5B-1024-16-2", 16, 2, [4], T)
    ra, _, rp, nref = oracle_run(s, N, "hann", 1, cof,
                                 pcal=dict(tonebins=32, rotatorlen=2048, fs=fs, offset=off))
    assert ns == nref
    assert rel_err_auto(auto, ra) < REL_TOL
    scale = np.max(np.abs(rp))
    assert np.max(np.abs(pc - rp)) / scale < 1e-6


def test_short_integration_level_relative(gpu):
    """One FFT per spectrum, rectangular window: per-FFT spectra are as
    accurate as the FP32 CPU restatement of the reference core on the same
    samples (error measured against the spectrum's mean level, since single
    FFTs have near-empty bins)."""
    import oracle as O
    N = 8192
    d, T = _mark5b_noise(16, 1, 9, 5)
    lay = gpu.layout("mark5b", 16, 1)
    cfg = gpu.make_config(lay, N, "none", 1, 1, sources=((0, 7),), max_run_bytes=len(d))
    core = gpu.Core(cfg)
    auto, _, _, ns = core.run([d])
    s = decode_channels(d, "Mark5B-1024-16-1", 16, 1, [7], T)
    ra, _, _, nref = oracle_run(s, N, "none", 1, 1)
    assert ns == nref == T // N
    lvl = ra.mean(axis=-1, keepdims=True)
    err = np.max(np.abs(auto - ra) / lvl)
    r32, _, _, _ = O.domaths(O.make_cfg(N, core_overlapped_ffts=1, window=O.W_NONE), s, fp64=False)
    err_cpu32 = np.max(np.abs(r32 - ra) / lvl)
    # the GPU packs two real frames into one complex FFT, whose FP32 rounding
    # scales with the pair's combined norm: allow sqrt(2) times the CPU error
    assert err <= max(np.sqrt(2.0) * 1.1 * err_cpu32, 1e-6), (err, err_cpu32)


@pytest.mark.parametrize("prec", ["tcsplit", "tcsplit_all"])
@pytest.mark.parametrize("N", [8192, 16384])
def test_tcsplit_two_files_overlap(gpu, N, prec):
    """Tensor-core forms on the remaining Q=4096 plans, overlapped FFTs, two files."""
    d1, T = _mark5b_noise(8, 2, 40, 51)
    d2, _ = _mark5b_noise(8, 2, 40, 52)
    lay = gpu.layout("mark5b", 8, 2)
    cof = 2 * (T // N) - 1
    cfg = gpu.make_config(lay, N, "hann", 2, cof, sources=((0, 1), (1, 6)), xpols=((0, 1),),
                          max_run_bytes=len(d1), precision=PREC_OF[prec])
    core = gpu.Core(cfg)
    auto, xp, _, ns = core.run([d1, d2])
    s1 = decode_channels(d1, "Mark5B-1024-8-2", 8, 2, [1], T)[0]
    s2 = decode_channels(d2, "Mark5B-1024-8-2", 8, 2, [6], T)[0]
    ra, rx, _, nref = oracle_run([s1, s2], N, "hann", 2, cof, nxpols=1)
    assert ns == nref
    assert rel_err_auto(auto, ra) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


def test_tcsplit_rejected_without_plan(gpu):
    cfg = gpu.make_config(gpu.layout("vdif:8000", 1, 8), 20000, precision=gpu.PREC_TCSPLIT)
    with pytest.raises(gpu.SwsError, match="tensor-core"):
        gpu.Core(cfg)


@pytest.mark.parametrize("prec", PRECS)
def test_blanked_mark5b_frames(gpu, prec):
    """Fill-pattern zones (trailing, whole frame, leading, interior) through
    the whole path: blanked sample-times enter the FFTs and the phase-cal
    fold as zeros, interior fill decodes as data (blanker_mark5.c:126-200)."""
    N, cof, fs, off = 16384, 5, 32e6, 15625.0
    nfr = N * cof // 2500 + 3
    rng = np.random.default_rng(404)
    comb = synth.pcal_comb(nfr * 2500, fs, 1e6, off, 0.05, rng.uniform(0, 6.28, 16))
    data = synth.mark5b_stream(rng.standard_normal((16, nfr * 2500)) + comb[None, :], 2, 1024)
    for f, a, b in [(2, 6000, 10000), (5, 0, 10000), (8, 0, 4000), (11, 2000, 3000), (20, 4, 9996)]:
        data = fill_zone(data, f, a, b, 10016, 16)
    lay = gpu.layout("mark5b", 16, 2)
    precision = PREC_OF[prec]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 2), (0, 9)), xpols=((0, 1),),
                          max_run_bytes=len(data), extract_pcal=True, pcal_tonebins=32,
                          pcal_rotatorlen=2048, samplingfreq=fs, pcal_offset_hz=off, precision=precision)
    core = gpu.Core(cfg)
    auto, xp, pc, ns = core.run([data])
    s = decode_channels(data, "Mark5B-1024-16-2", 16, 2, [2, 9], nfr * 2500)
    assert np.count_nonzero(s[0][5 * 2500:6 * 2500]) == 0 and np.count_nonzero(s[0][11 * 2500:12 * 2500]) > 2000
    ra, rx, rp, nref = oracle_run(s, N, "hann", 1, cof, nxpols=1,
                                  pcal=dict(tonebins=32, rotatorlen=2048, fs=fs, offset=off))
    assert ns == nref
    assert rel_err_auto(auto[:, 0], ra[:, 0]) < REL_TOL and rel_err_auto(auto[:, 1], ra[:, 1]) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL
    assert np.max(np.abs(pc - rp)) / np.max(np.abs(rp)) < 1e-6


def test_blanked_vdif_frames(gpu):
    """VDIF 2-bit, 4 channels: frames with the invalid bit set and frames
    whose first or last payload word is fill are blanked whole.  128 frames
    = 125 FFTs = 5 whole spectra (no single-FFT partial spectrum, whose
    near-empty bins make relative errors meaningless)."""
    N, cof = 8192, 25
    spf = 8000 * 8 // (4 * 2)
    nfr = 128
    rng = np.random.default_rng(405)
    codes = synth.quantize_vdif_2bit(rng.standard_normal((4, nfr * spf)), 0.98)
    payload = synth.pack_codes(codes, 2)
    data = synth.vdif_frames(payload, 8000, 4, 2, 4000, invalid={3, 64})
    data = fill_zone(data, 5, 0, 8, 8032, 32)
    data = fill_zone(data, 90, 7992, 8000, 8032, 32)
    lay = gpu.layout("vdif:8000", 4, 2)
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 1), (0, 3)), xpols=((0, 1),),
                          max_run_bytes=len(data))
    core = gpu.Core(cfg)
    auto, xp, _, ns = core.run([data])
    s = decode_channels(data, "VDIF_8000-64-4-2", 4, 2, [1, 3], nfr * spf)
    assert all(np.count_nonzero(s[0][f * spf:(f + 1) * spf]) == 0 for f in (3, 5, 64, 90))
    ra, rx, _, nref = oracle_run(s, N, "hann", 1, cof, nxpols=1)
    assert ns == nref == 5
    assert rel_err_auto(auto[:, 0], ra[:, 0]) < REL_TOL and rel_err_auto(auto[:, 1], ra[:, 1]) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


@pytest.mark.parametrize("nchan,nbit,N", [(4, 2, 16384), (2, 2, 65536), (8, 1, 16384), (4, 1, 65536),
                                          (2, 1, 65536), (8, 2, 16384)])
def test_vdif_fractional_word_sample_times(gpu, nchan, nbit, N):
    """Multi-channel VDIF whose sample-times fill 1/R of a 32-bit word (R
    consecutive FFT phases per word: R = 2 .. 16) at cluster sizes R
    divides, so the corner turn transposes R phases at once; a frame with
    fill at its end is blanked whole.  Two channels and their cross
    spectrum, two whole spectra of 4 FFTs, against the FP64 oracle."""
    cof = 4
    spf = 8000 * 8 // (nchan * nbit)
    T = N * cof * 2
    nfr = -(-T // spf)
    rng = np.random.default_rng(nchan * 100 + nbit * 10 + N % 97)
    x = rng.standard_normal((nchan, nfr * spf))
    codes = synth.quantize_vdif_2bit(x, 0.98) if nbit == 2 else synth.quantize_vdif_1bit(x)
    data = synth.vdif_frames(synth.pack_codes(codes, nbit), 8000, nchan, nbit, 4000)
    data = fill_zone(data, 2, 7992, 8000, 8032, 32)
    pay = T * nchan * nbit // 8                      # exactly two spectra's samples
    run = data[:(pay // 8000) * 8032 + (32 + pay % 8000 if pay % 8000 else 0)]
    lay = gpu.layout("vdif:8000", nchan, nbit)
    chans = [1, nchan - 1]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, chans[0]), (0, chans[1])), xpols=((0, 1),),
                          max_run_bytes=len(run))
    core = gpu.Core(cfg)
    auto, xp, _, ns = core.run([run])
    s = decode_channels(data, f"VDIF_8000-64-{nchan}-{nbit}", nchan, nbit, chans, T)
    assert np.count_nonzero(s[0][2 * spf:3 * spf]) == 0
    ra, rx, _, nref = oracle_run(s, N, "hann", 1, cof, nxpols=1)
    assert ns == nref == 2
    assert rel_err_auto(auto[:, 0], ra[:, 0]) < REL_TOL and rel_err_auto(auto[:, 1], ra[:, 1]) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


def test_pcal_tones_known_answer(gpu):
    """Tone phasors on the GPU (PCal.cpp:654-678 final step, FP64) equal the
    FP64 oracle's from the same folded samples, and reproduce the PCal
    library's known answer (PCal.cpp:861-951: tones
    sin(pi n (f_off + t spacing)/BW + t 5 deg) -> phase -90 + 5 t degrees).
    The reference checks 0.1 degree on float samples (pinned in the oracle
    tests); an 8-bit stream of a comb that repeats every rotator period
    carries a periodic quantisation error that no averaging removes (0.17
    degree at 24 codes per unit), so the phase bar here is 0.5 degree."""
    import oracle as O
    bw, fs, spacing, off = 16e6, 32e6, 1e6, 15625.0
    tonebins, rotatorlen = int(fs / spacing), int(fs / np.gcd(int(fs), int(off)))
    ntones, N, cof = int(bw / spacing), 65536, 8
    spf = 8000
    nfr = N * cof // spf + 1
    n = np.arange(nfr * spf, dtype=np.float64)
    x = np.zeros(nfr * spf)
    for t in range(ntones):
        x += 0.5 * np.sin(np.pi * n * (off + t * spacing) / bw + np.deg2rad(5.0 * t))
    codes = synth.quantize_vdif_8bit(x, 24.0)
    data = synth.vdif_frames(synth.pack_codes(codes[None, :], 8), 8000, 1, 8, 4000)
    lay = gpu.layout("vdif:8000", 1, 8)
    cfg = gpu.make_config(lay, N, "hann", 1, cof, max_run_bytes=len(data), extract_pcal=True,
                          pcal_tonebins=tonebins, pcal_rotatorlen=rotatorlen, samplingfreq=fs,
                          pcal_offset_hz=off, pcal_ntones=ntones)
    core = gpu.Core(cfg)
    _, _, pc, ns = core.run([data])
    tones = core.tones[0, 0]
    ph = np.rad2deg(np.angle(tones))
    want = -90.0 + 5.0 * np.arange(ntones)
    d = (ph - want + 180) % 360 - 180
    assert np.max(np.abs(d)) < 0.5, d
    s = decode_channels(data, "VDIF_8000-256-1-8", 1, 8, [0], nfr * spf)
    _, _, rp, nref = oracle_run(s, N, "hann", 1, cof,
                                pcal=dict(tonebins=tonebins, rotatorlen=rotatorlen, fs=fs, offset=off))
    assert ns == nref == 1
    ref = O.pcal_tones(rp[0, 0], float(N * cof), ntones)
    assert np.max(np.abs(tones - ref)) / np.max(np.abs(ref)) < 1e-6
    # phasor = amplitude / 2 in decoded units: 0.5 / 2 * 24 / 256
    assert np.allclose(np.abs(tones), 0.25 * 24.0 / 256.0, rtol=2e-2)


def test_group_runs_chunked_and_per_run(gpu):
    """A 10-run output group submitted run by run: header-free runs at
    consecutive payload offsets are collected into one device chunk per
    launch; a break in the offsets flushes the open chunk (4 + 6 runs);
    framed runs go one per launch.  All three give the FP64 oracle's
    combined spectrum."""
    import oracle as O
    N, cof, nrun, frames_per_run = 4096, 12, 10, 20
    run_pay = frames_per_run * 10000          # 50000 sample-times: 12 whole FFTs
    data, info = synth.c3_stream(123, N=N)
    pay = np.frombuffer(payload_of(data, info["fmt"]), dtype=np.uint8)
    fr = np.frombuffer(data, dtype=np.uint8).reshape(-1, 10016)
    S = N // 2 + 1

    def core_for(framed):
        lay = gpu.layout("mark5b", 16, 2, framed=framed)
        cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 1), (0, 9)), xpols=((0, 1),),
                              max_run_bytes=frames_per_run * 10016, samplingfreq=64e6, runs_per_output=nrun)
        return gpu.Core(cfg)

    def collect(core, runs, offsets):
        auto = np.zeros((1, 2, S), np.float32)
        xp = np.zeros((1, 1, S, 2), np.float32)
        for r, (buf, off) in enumerate(zip(runs, offsets)):
            core.set_sizes([len(buf)])
            core.submit([np.frombuffer(buf, dtype=np.uint8)], payload_offsets=[off])
            assert core.wait() == (1 if r == len(runs) - 1 else 0)
        core.fetch_into(auto, xp)
        return auto[0], xp[0, 0, :, 0] + 1j * xp[0, 0, :, 1]

    runs = [pay[r * run_pay:(r + 1) * run_pay].tobytes() for r in range(nrun)]
    a1, x1 = collect(core_for(False), runs, [r * run_pay for r in range(nrun)])
    # a jump after run 3 (a multiple of the 10000-byte payload keeps the frame phase)
    a2, x2 = collect(core_for(False), runs, [r * run_pay + (0 if r < 4 else 10_000_000) for r in range(nrun)])
    framed = [fr[r * frames_per_run:(r + 1) * frames_per_run].tobytes() for r in range(nrun)]
    a3, x3 = collect(core_for(True), framed, [0] * nrun)
    ra = np.zeros((2, S))
    rx = np.zeros(S, complex)
    for r in range(nrun):
        s = [O.decode(O.FMT_MARK5B, 16, 2, runs[r], run_pay // 4, c, payload_bytes=10000) for c in (1, 9)]
        aa, xx, _, n = oracle_run(s, N, "hann", 1, cof, nxpols=1)
        assert n == 1
        ra += aa[0]
        rx += xx[0, 0]
    for a, x in ((a1, x1), (a2, x2), (a3, x3)):
        assert np.max(np.abs(a - ra) / ra) < REL_TOL
        assert np.max(np.abs(x - rx) / np.sqrt(ra[0] * ra[1])) < REL_TOL
    assert np.max(np.abs(a1 - a2) / a1) < 1e-6 and np.max(np.abs(a1 - a3) / a1) < 1e-6


def test_group_chunks_alternate_streams(gpu):
    """Two 10-run output groups of 8 MiB runs: the submit path collects up
    to 4 runs per device chunk (32 MiB; the group's last chunks shrink:
    4, 3, 1, 1, 1), and consecutive chunks run on alternating streams with
    their own scratch buffers, their spectrum sums and phase-cal folds added
    in submission order.  Both groups' combined spectra and phase-cal
    vectors match the FP64 oracle, and a chunk's input region is refilled
    only after its decode."""
    N, cof, nrun = 4096, 512, 10
    run = N * cof * 4                         # 16 channels x 2 bit: 4 bytes per sample-time
    rng = np.random.default_rng(77)
    pay = rng.integers(0, 256, size=2 * nrun * run, dtype=np.uint8)
    w = pay.view(np.uint32)
    w[w == 0x11223344] ^= 1                   # no mark5access fill words
    S = N // 2 + 1
    lay = gpu.layout("mark5b", 16, 2, framed=False)
    # phase-cal: 64 tone bins, rotator period 4096 at 64 Msps (15625 Hz offset)
    pc_args = dict(tonebins=64, rotatorlen=4096, fs=64e6, offset=15625.0)
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 3), (0, 12)), xpols=((0, 1),),
                          max_run_bytes=run, samplingfreq=64e6, runs_per_output=nrun,
                          extract_pcal=True, pcal_tonebins=64, pcal_rotatorlen=4096, pcal_offset_hz=15625.0)
    core = gpu.Core(cfg)
    core.set_sizes([run])
    outs = []
    for g in range(2):
        auto = np.zeros((1, 2, S), np.float32)
        xp = np.zeros((1, 1, S, 2), np.float32)
        pc = np.zeros((1, 2, 64, 2), np.float32)
        for r in range(nrun):
            off = (g * nrun + r) * run
            core.submit([pay[off:off + run]], payload_offsets=[off])
            assert core.wait() == (1 if r == nrun - 1 else 0)
        core.fetch_into(auto, xp, pc)
        outs.append((auto[0], xp[0, 0, :, 0] + 1j * xp[0, 0, :, 1], pc[0, :, :, 0] + 1j * pc[0, :, :, 1]))
    core.close()
    for g, (a, x, p) in enumerate(outs):
        ra = np.zeros((2, S))
        rx = np.zeros(S, complex)
        rp = np.zeros((2, 64), complex)
        for r in range(nrun):
            off = (g * nrun + r) * run
            s = [O_decode(pay[off:off + run].tobytes(), run // 4, c) for c in (3, 12)]
            aa, xx, pp, n = oracle_run(s, N, "hann", 1, cof, nxpols=1, pcal=pc_args)
            assert n == 1
            ra += aa[0]
            rx += xx[0, 0]
            rp += pp[0]
        assert np.max(np.abs(a - ra) / ra) < REL_TOL, g
        assert np.max(np.abs(x - rx) / np.sqrt(ra[0] * ra[1])) < REL_TOL, g
        assert np.max(np.abs(p - rp)) / np.max(np.abs(rp)) < 1e-6, g


@pytest.mark.parametrize("fmt,ntrack,N,prec,fill", [("MKIV1_2-512-8-2", 32, 4096, "fp32", False),
                                                     ("VLBA1_4-512-8-2", 64, 4096, "fp32", False),
                                                     ("MKIV1_2-512-8-2", 32, 8192, "tcsplit_all", False),
                                                     ("MKIV1_2-512-8-2", 32, 4096, "fp32", True),
                                                     ("VLBA1_4-512-8-2", 64, 4096, "fp32", True),
                                                     ("VLBA1_1-512-32-2", 64, 4096, "fp32", True)])
def test_track_format_spectra(gpu, fmt, ntrack, N, prec, fill):
    """VLBA / Mark4 track-words through the track turn, the corner turn and
    the FFT: auto spectra of two channels and their cross spectrum (16 FFTs)
    against the FP64 oracle on mark5access's decode of the same bytes
    (Mark4 header track-words blanked, VLBA modulation removed); with `fill`,
    fill-pattern regions planted at zone ends blank whole track-words through
    the blank bitmap as mark5access blanks them."""
    import oracle as O
    from helpers import plant_track_fill
    info = O.m5_format_info(fmt)
    nchan, nbit = info["nchan"], info["nbit"]
    fanout = ntrack // (nchan * nbit)
    cof = 16
    nfr = -(-N * cof // (20000 * fanout))
    rng = np.random.default_rng(N + ntrack)
    pay = rng.integers(0, 256, size=nfr * 2500 * ntrack, dtype=np.uint8).tobytes()
    if fill:
        pay = plant_track_fill(pay, ntrack, limit=N * cof * nchan * nbit // 8)
    lay = gpu.layout(("vlba:" if fmt.startswith("VLBA") else "mark4:") + str(ntrack), nchan, nbit)
    chans = [1, nchan - 2]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=tuple((0, c) for c in chans), xpols=((0, 1),),
                          max_run_bytes=N * cof * nchan * nbit // 8, precision=PREC_OF[prec])
    core = gpu.Core(cfg)
    run = pay[:N * cof * nchan * nbit // 8]            # exactly one spectrum's samples
    auto, xp, _, ns = core.run([run])
    dec, _ = O.m5_unpack(fmt, pay, nfr * 20000 * fanout)
    if fill:
        assert (dec[chans[0], :N * cof] == 0.0).any()
    ra, rx, _, nref = oracle_run([dec[c, :N * cof] for c in chans], N, "hann", 1, cof, nxpols=1)
    assert ns == nref == 1
    assert rel_err_auto(auto, ra) < REL_TOL
    assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL


def test_submit_out_matches_fetch(gpu):
    """swsgpu_submit_out (the run's output buffers given with the run, as
    TaskCore::run takes them) delivers the same spectra, bit for bit, as
    submit + fetch: into page-locked arrays by the run's own device copies,
    into pageable arrays through the staging buffer at wait; fetch after it
    is refused.  Two 6-run groups of 1 MiB runs (chunks of 3, 1, 1, 1)."""
    import torch
    N, cof, nrun = 4096, 64, 6
    run = N * cof * 4
    rng = np.random.default_rng(91)
    pay = rng.integers(0, 256, size=2 * nrun * run, dtype=np.uint8)
    w = pay.view(np.uint32)
    w[w == 0x11223344] ^= 1
    S = N // 2 + 1
    lay = gpu.layout("mark5b", 16, 2, framed=False)
    got = {}
    for mode in ("fetch", "pinned", "pageable"):
        cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=((0, 3), (0, 12)), xpols=((0, 1),),
                              max_run_bytes=run, samplingfreq=64e6, runs_per_output=nrun)
        core = gpu.Core(cfg)
        core.set_sizes([run])
        for g in range(2):
            if mode == "pinned":
                a = torch.zeros((1, 2, S), dtype=torch.float32, pin_memory=True).numpy()
                x = torch.zeros((1, 1, S, 2), dtype=torch.float32, pin_memory=True).numpy()
            else:
                a = np.zeros((1, 2, S), np.float32)
                x = np.zeros((1, 1, S, 2), np.float32)
            for r in range(nrun):
                off = (g * nrun + r) * run
                core.submit([pay[off:off + run]], payload_offsets=[off],
                            dest=None if mode == "fetch" else (a, x))
                assert core.wait() == (1 if r == nrun - 1 else 0)
            if mode == "fetch":
                core.fetch_into(a, x)
            else:
                with pytest.raises(gpu.SwsError, match="submit_out"):
                    core.fetch_into(np.zeros_like(a), np.zeros_like(x))
            got.setdefault(mode, []).append((a.copy(), x.copy()))
        core.close()
    for mode in ("pinned", "pageable"):
        for g in range(2):
            assert np.array_equal(got[mode][g][0], got["fetch"][g][0]), (mode, g)
            assert np.array_equal(got[mode][g][1], got["fetch"][g][1]), (mode, g)
    assert np.all(got["fetch"][0][0] > 0)


def O_decode(buf: bytes, nsamp: int, chan: int):
    import oracle as O
    return O.decode(O.FMT_MARK5B, 16, 2, buf, nsamp, chan, payload_bytes=10000)


@pytest.mark.parametrize("N,nbit,fmt,nchan", [(65536, 2, "mark5b", 16), (1 << 20, 8, "vdif:8000", 1)])
def test_workspace_size_covers_allocations(gpu, N, nbit, fmt, nchan):
    """swsgpu_workspace_size predicts the device memory a first
    process_device call takes (codes, bitmaps, partial spectra, four-step
    scratch): within 10 % + 64 MB above and at least half of it."""
    import torch
    lay = gpu.layout(fmt, nchan, nbit, framed=False)
    run_bytes, nruns = 8 << 20, 4
    src = ((0, 0), (0, 1)) if nchan > 1 else ((0, 0),)
    xp = ((0, 1),) if nchan > 1 else ()
    cfg = gpu.make_config(lay, N, "hann", 1, 1, sources=src, xpols=xp, max_run_bytes=run_bytes,
                          samplingfreq=32e6, runs_per_output=nruns)
    core = gpu.Core(cfg)
    ws = core.workspace_size(run_bytes, nruns)
    raw = torch.randint(0, 256, (run_bytes * nruns,), dtype=torch.uint8, device="cuda")
    per_run = run_bytes * 8 // (nchan * nbit) // N
    S = N // 2 + 1
    d_auto = torch.zeros(max(1, per_run) * len(src), S, device="cuda")
    d_xpol = torch.zeros(max(1, per_run) * max(1, len(xp)), S, 2, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    core.process_device([raw.data_ptr()], run_bytes, nruns, nruns, d_auto.data_ptr(),
                        d_xpol.data_ptr() if xp else 0)
    torch.cuda.synchronize()
    used = free0 - torch.cuda.mem_get_info()[0]
    core.close()
    assert used <= ws * 1.1 + (64 << 20), (used, ws)
    assert ws >= used // 2, (used, ws)


@pytest.mark.parametrize("fmt,nchan,nbit,N,prec", [("raw_signed", 1, 8, 32768, "fp32"),
                                                   ("raw_signed", 1, 8, 65536, "tcsplit"),
                                                   ("raw_unsigned", 8, 2, 16384, "fp32"),
                                                   ("raw_signed", 1, 2, 8192, "fp32")])
def test_raw_sampler_spectra(gpu, fmt, nchan, nbit, N, prec):
    """Raw sampler data (the reference's default SourceFormat) through the
    corner turn and the FFT: Gaussian noise plus a tone, quantised to the
    format's codes; auto spectra of two channels (or one) and their cross
    spectrum vs the FP64 oracle."""
    import oracle as O
    rng = np.random.default_rng(N + nchan)
    cof = 6
    nsamp = N * cof
    t = np.arange(nsamp)
    sig = rng.standard_normal((nchan, nsamp)) + 0.3 * np.cos(2 * np.pi * 0.123 * t)[None, :]
    if nbit == 8:
        q = np.clip(np.round(sig * 20), -128, 127).astype(np.int16)
        codes = (q & 0xFF).astype(np.uint8) if fmt == "raw_signed" else (q + 128).astype(np.uint8)
        raw = codes.T.reshape(-1).tobytes()          # sample-time major, channel minor
    else:
        # 2-bit codes (sign, magnitude) at +-0.98 sigma; map_rev order {+1, -1, +H, -H}
        mag = (np.abs(sig) > 0.98).astype(np.uint8)
        code = ((sig < 0).astype(np.uint8) | (mag << 1))
        if nchan == 1:
            c4 = code[0].reshape(-1, 4)
            raw = ((c4[:, 0] << 6) | (c4[:, 1] << 4) | (c4[:, 2] << 2) | c4[:, 3]).astype(np.uint8).tobytes()
        else:
            cb = code.T.reshape(nsamp, nchan // 4, 4)
            raw = (cb[..., 0] | (cb[..., 1] << 2) | (cb[..., 2] << 4) | (cb[..., 3] << 6)).astype(np.uint8).tobytes()
    lay = gpu.layout(fmt, nchan, nbit)
    chans = [0] if nchan == 1 else [1, nchan - 2]
    cfg = gpu.make_config(lay, N, "hann", 1, cof, sources=tuple((0, c) for c in chans),
                          xpols=((0, 1),) if len(chans) == 2 else (), max_run_bytes=len(raw),
                          precision=PREC_OF[prec])
    core = gpu.Core(cfg)
    auto, xp, _, ns = core.run([raw])
    ofmt = O.FMT_RAW_SIGNED if fmt == "raw_signed" else O.FMT_RAW_UNSIGNED
    samples = [O.decode(ofmt, nchan, nbit, raw, nsamp, c) for c in chans]
    ra, rx, _, nref = oracle_run(samples, N, "hann", 1, cof, nxpols=len(chans) - 1)
    assert ns == nref == 1
    assert rel_err_auto(auto, ra) < REL_TOL
    if len(chans) == 2:
        assert rel_err_xpol(xp[:, 0], rx[:, 0], ra[:, 0], ra[:, 1]) < REL_TOL
