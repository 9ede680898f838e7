"""CPU: the oracle pinned against the reference's own code and known answers.

* decode restatement == mark5access (golden fixtures made from the reference's
  mark5access, and the live oracle/_ref build when present);
* windows == the formulas written in the reference (Cosine, Cosine2:
  TaskCoreIPP.cpp:576-586; Hann: TaskCoreMKL.cpp:53 / TaskCoreFFTW.cpp:65);
* FFT == numpy float64 and a naive long-double DFT;
* doMaths loop == a numpy restatement; frame schedule and scaling rules;
* PCal known answer of src/IA-32/PhaseCal/PCal.cpp:904-948 (tone phases
  -90 + 5*t degrees within 0.1 degree).
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import fill_zone
from swspec_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_decode_matches_golden_mark5b():
    z = np.load(os.path.join(GOLDEN, "mark5b_decode.npz"))
    raw = z["raw"].tobytes()
    pay = synth.strip_headers(raw, 10016, 16)
    nsamp = int(z["nsamp"])
    for c in range(16):
        ref = z["decoded"][c]
        # blanked: payload bytes 6000..10000 of frame 1 -> sample-times 1500..2500
        assert np.all(ref[2500 + 1500: 2500 + 2500] == 0)
        assert np.count_nonzero(ref[2500: 2500 + 1500] == 0) == 0
        mine = O.decode(O.FMT_MARK5B, 16, 2, pay, nsamp, c, payload_bytes=10000)
        assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))
        # without the blanker only the fill zone differs
        plain = O.decode(O.FMT_MARK5B, 16, 2, pay, nsamp, c)
        ok = ref != 0
        assert np.array_equal(plain[ok].view(np.uint32), ref[ok].view(np.uint32))


def test_decode_matches_golden_vdif():
    z = np.load(os.path.join(GOLDEN, "vdif_decode.npz"))
    raw = z["raw"].tobytes()
    pay = synth.strip_headers(raw, 8032, 32)
    ref = z["decoded"][0]
    assert np.all(ref[8000:16000] == 0)  # invalid frame blanked by mark5access
    inv = O.vdif_invalid_bits(raw, 8032)
    assert list(inv) == [0, 1, 0]
    mine = O.decode(O.FMT_VDIF, 1, 8, pay, int(z["nsamp"]), 0, payload_bytes=8000, frame_invalid=inv)
    assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))




@pytest.mark.skipif(O.ref() is None, reason="mark5access not built from the reference sources")
def test_blanker_matches_live_mark5access():
    """Fill zones of every shape (whole, leading, trailing, interior, 8-byte
    edges, 32-bit stragglers) and VDIF invalid/fill frames, decoded by the
    restated blankers and by mark5access itself."""
    rng = np.random.default_rng(404)
    data = synth.mark5b_stream(rng.standard_normal((16, 30 * 2500)), 2, 1024)
    zones = [(2, 6000, 10000), (5, 0, 10000), (8, 0, 4000), (11, 2000, 3000), (20, 4, 9996),
             (22, 8, 10000), (24, 0, 9992), (26, 0, 8), (27, 9992, 10000), (28, 0, 4004), (29, 5996, 10000)]
    for f, a, b in zones:
        data = fill_zone(data, f, a, b, 10016, 16)
    ref, _ = O.m5_decode("Mark5B-1024-16-2", data, 30 * 2500)
    pay = synth.strip_headers(data, 10016, 16)
    for c in range(16):
        mine = O.decode(O.FMT_MARK5B, 16, 2, pay, 30 * 2500, c, payload_bytes=10000)
        assert np.array_equal(mine.view(np.uint32), ref[c].view(np.uint32)), c
    spf = 8000
    codes = synth.quantize_vdif_2bit(rng.standard_normal((4, 8 * spf)), 0.98)
    vd = synth.vdif_frames(synth.pack_codes(codes, 2), 8000, 4, 2, 4000, invalid={3})
    vd = fill_zone(vd, 5, 0, 8, 8032, 32)
    vd = fill_zone(vd, 6, 7992, 8000, 8032, 32)
    vref, _ = O.m5_decode("VDIF_8000-64-4-2", vd, 8 * spf)
    inv = O.vdif_invalid_bits(vd, 8032)
    vpay = synth.strip_headers(vd, 8032, 32)
    for c in range(4):
        mine = O.decode(O.FMT_VDIF, 4, 2, vpay, 8 * spf, c, payload_bytes=8000, frame_invalid=inv)
        assert np.array_equal(mine.view(np.uint32), vref[c].view(np.uint32)), c
        assert np.count_nonzero(mine[3 * spf:7 * spf].reshape(4, spf), axis=1).tolist() == [0, spf, 0, 0]


def test_decode_matches_test_unpacker_pattern():
    z = np.load(os.path.join(GOLDEN, "unpacker_pattern.npz"))
    pat = z["pattern"].tobytes()
    for c in range(16):
        assert np.array_equal(O.decode(O.FMT_MARK5B, 16, 2, pat, 2500, c), z["m5b_16ch"][c])
    for c in range(8):
        assert np.array_equal(O.decode(O.FMT_MARK5B, 8, 2, pat, 5000, c), z["m5b_8ch"][c])


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
@pytest.mark.parametrize("nchan,nbit,mbps", [(16, 2, 1024), (32, 1, 1024), (2, 2, 256),
                                             (8, 1, 1024)])
def test_decode_matches_live_mark5access(nchan, nbit, mbps):
    spf = synth.mark5b_samples_per_frame(nchan, nbit)
    rng = np.random.default_rng(nchan * 10 + nbit)
    raw = synth.mark5b_stream(rng.standard_normal((nchan, spf * 3)), nbit, mbps)
    ref, _ = O.m5_decode(f"Mark5B-{mbps}-{nchan}-{nbit}", raw, spf * 2)
    pay = synth.strip_headers(raw, 10016, 16)
    for c in range(nchan):
        assert np.array_equal(O.decode(O.FMT_MARK5B, nchan, nbit, pay, spf * 2, c), ref[c])


def test_windows_pinned_formulas():
    n = 1000
    i = np.arange(n, dtype=np.float64)
    c = np.cos(np.pi * (i - 0.5 * n + 0.5) / n)
    assert np.array_equal(O.window(O.W_COSINE2, n), (c * c).astype(np.float32))
    assert np.array_equal(O.window(O.W_COSINE, n), c.astype(np.float32))
    s = np.sin(np.pi * i / (n - 1))
    assert np.allclose(O.window(O.W_HANN, n), (s * s).astype(np.float32), atol=6e-8)
    assert np.all(O.window(O.W_NONE, n) == 1)


@pytest.mark.parametrize("n", [8, 30, 125, 4096, 20000])
def test_fft64_vs_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    r = O.fft64(x)
    assert np.max(np.abs(r - np.fft.fft(x))) / np.max(np.abs(r)) < 1e-13


def test_fft64_vs_longdouble_dft():
    n = 60
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    k = np.arange(n, dtype=np.longdouble)
    ang = -2 * np.pi * np.outer(k, k) / n
    ref = (np.cos(ang) * x.real - np.sin(ang) * x.imag) + 1j * (np.sin(ang) * x.real + np.cos(ang) * x.imag)
    ref = ref.sum(axis=1)
    assert np.max(np.abs(O.fft64(x) - ref.astype(np.complex128))) < 1e-12


@pytest.mark.parametrize("overlap,cof,nfr", [(1, 4, 9), (2, 7, 9), (3, 4, 5)])
def test_domaths_vs_numpy(overlap, cof, nfr):
    N = 1024
    rng = np.random.default_rng(overlap * 100 + cof)
    s = [rng.standard_normal(N * nfr).astype(np.float32) for _ in range(2)]
    cfg = O.make_cfg(N, overlap=overlap, core_overlapped_ffts=cof, num_sources=2, num_xpols=1,
                     window=O.W_HANN)
    a, xp, _, ns = O.domaths(cfg, s)
    starts, spec, ns2, part = O.schedule(cfg, N * nfr)
    assert ns == ns2
    w = O.window(O.W_HANN, N).astype(np.float64)
    ra = np.zeros((ns, 2, N // 2 + 1))
    rx = np.zeros((ns, N // 2 + 1), complex)
    for st, sp in zip(starts, spec):
        X = [np.fft.rfft(s[i][st:st + N].astype(np.float64) * w) for i in range(2)]
        for i in range(2):
            ra[sp, i] += np.abs(X[i]) ** 2
        rx[sp] += X[0] * np.conj(X[1])
    full = ns - part
    ra[:full] /= cof
    rx[:full] /= cof
    assert np.allclose(a, ra, rtol=1e-12)
    assert np.allclose(xp[:, 0], rx, rtol=1e-12, atol=1e-9)


def test_schedule_spectrum_hop():
    """After core_overlapped_ffts FFTs the source pointer hops by
    raw_fullfft - raw_overlap (TaskCoreIPP.cpp:506-511)."""
    cfg = O.make_cfg(1000, overlap=2, core_overlapped_ffts=3)
    starts, spec, ns, part = O.schedule(cfg, 4000)
    assert list(starts) == [0, 500, 1000, 2000, 2500, 3000]
    assert list(spec) == [0, 0, 0, 1, 1, 1] and ns == 2 and not part


def test_fp32_baseline_close_to_fp64():
    N = 4096
    rng = np.random.default_rng(9)
    s = [rng.standard_normal(N * 6).astype(np.float32)]
    cfg = O.make_cfg(N, core_overlapped_ffts=6, nthreads=3)
    a64, _, _, _ = O.domaths(cfg, s)
    a32, _, _, _ = O.domaths(cfg, s, fp64=False)
    assert np.max(np.abs(a32 - a64) / a64) < 1e-4


def test_pcal_known_answer():
    """PCal.cpp:861-951: tones sin(pi (n + off)(f_off + t*spacing)/BW + t*5deg)
    extracted with phase -90 + 5*t degrees, within 0.1 degree."""
    bw, fs = 16e6, 32e6
    spacing, off = 1e6, 10e3
    tonebins, rotatorlen = int(fs / spacing), int(fs / np.gcd(int(fs), int(off)))
    ntones = int(bw / spacing)
    N = rotatorlen * 20
    n = np.arange(N, dtype=np.float64)
    x = np.zeros(N)
    for t in range(ntones):
        x += np.sin(np.pi * n * (off + t * spacing) / bw + np.deg2rad(5.0 * t))
    cfg = O.make_cfg(N, core_overlapped_ffts=1, extract_pcal=True, pcal_tonebins=tonebins,
                     pcal_rotatorlen=rotatorlen, samplingfreq=fs, pcaloffsethz=off)
    _, _, pc, _ = O.domaths(cfg, [x.astype(np.float32)])
    tones = O.pcal_tones(pc[0, 0], N, ntones)
    ph = np.rad2deg(np.angle(tones))
    want = -90.0 + 5.0 * np.arange(ntones)
    d = (ph - want + 180) % 360 - 180
    assert np.max(np.abs(d)) < 0.1, d


# ---- raw sampler formats: the oracle against the reference's own unpackers ----

def _raw_ref_or_skip():
    import oracle as O
    if O.ref_unpack() is None:
        pytest.skip("reference unpackers not built (oracle/_ref/libunpackref.so)")
    return O


@pytest.mark.parametrize("fmt,nchan", [("signed", 1), ("signed", 4), ("signed", 3), ("unsigned", 2),
                                       ("unsigned", 8)])
def test_raw_8bit_matches_reference_unpacker(fmt, nchan):
    O = _raw_ref_or_skip()
    rng = np.random.default_rng(nchan)
    nsamp = 4096
    pay = rng.integers(0, 256, nsamp * nchan + 64, dtype=np.uint8).tobytes()
    f = O.FMT_RAW_SIGNED if fmt == "signed" else O.FMT_RAW_UNSIGNED
    kind = O.RAW_SIGNED_8 if fmt == "signed" else O.RAW_UNSIGNED_8
    for c in range(nchan):
        ours = O.decode(f, nchan, 8, pay, nsamp, c)
        ref = O.ref_unpack_raw(kind, 8, nchan, pay, nsamp, c)
        assert np.array_equal(ours, ref), (fmt, nchan, c)


@pytest.mark.parametrize("nchan,increasing", [(4, True), (8, True), (16, True), (8, False), (16, False)])
def test_raw_2bit_matches_reference_unpacker(nchan, increasing):
    O = _raw_ref_or_skip()
    rng = np.random.default_rng(100 + nchan)
    nsamp = 4096
    pay = rng.integers(0, 256, nsamp * nchan // 4 + 64, dtype=np.uint8).tobytes()
    for c in range(nchan):
        # ChannelOrderIncreasing = no reads channel c where the increasing order has nchan-1-c
        oc = c if increasing else nchan - 1 - c
        ours = O.decode(O.FMT_RAW_SIGNED, nchan, 2, pay, nsamp, oc)
        ref = O.ref_unpack_raw(O.RAW_TWOBIT, 2, nchan, pay, nsamp, c, increasing)
        assert np.array_equal(ours, ref), (nchan, increasing, c)


def test_raw_2bit_single_channel_layout():
    """One-channel 2-bit data: four samples per byte, oldest in the MSBs.  The
    reference's table lookup reads a defined entry only for the first sample
    of each byte (DataUnpackers.cpp:280-284); those agree exactly, and the
    whole layout is checked against a direct restatement."""
    O = _raw_ref_or_skip()
    rng = np.random.default_rng(7)
    nsamp = 4096
    raw = rng.integers(0, 256, nsamp // 4 + 64, dtype=np.uint8)
    pay = raw.tobytes()
    ours = O.decode(O.FMT_RAW_UNSIGNED, 1, 2, pay, nsamp, 0)
    ref = O.ref_unpack_raw(O.RAW_TWOBIT_1CH, 2, 1, pay, nsamp, 0)
    assert np.array_equal(ours[0::4], ref[0::4])
    lv = np.array([1.0, -1.0, 3.3359, -3.3359], dtype=np.float32)
    t = np.arange(nsamp)
    want = lv[(raw[t // 4] >> (6 - 2 * (t % 4))) & 3]
    assert np.array_equal(ours, want)


# ---- the PCal extractor library (src/IA-32/PhaseCal/PCal.cpp) ----

def _pcal_test_signal(n, bw, spacing, offset, ntones, sampleoffset):
    """The library's own test signal (PCal.cpp:896-906): tones at offset +
    t*spacing with phases -90 deg + 5 deg * t."""
    t = np.arange(n, dtype=np.float64) + sampleoffset
    x = np.zeros(n)
    for k in range(ntones):
        x += np.sin(np.pi * t * (offset + k * spacing) / bw + k * np.pi * 5 / 180)
    return x.astype(np.float32)


@pytest.mark.parametrize("bw,spacing,offset,kind", [(8e6, 1e6, 0, 1), (8e6, 1e6, 10000, 3)])
def test_pcallib_known_answer(bw, spacing, offset, kind):
    """The library's known answer (PCal.cpp:879-948): tone phases -90 + 5 t
    degrees, after a gap re-entered with adjustSampleOffset."""
    import oracle as O
    p = O.PcalLib(bw, spacing, offset, 0)
    assert p.kind == kind
    n, prime = 160000, 3
    x = _pcal_test_signal(n, bw, spacing, offset, p.ntones, 0)
    p.extract(x)
    p.adjust(n + prime)
    y = _pcal_test_signal(n, bw, spacing, offset, p.ntones, n + prime)   # the stream after the gap
    p.extract(y)
    tones, used = p.final()
    assert used == 2 * n
    first = 1 if offset == 0 else 0      # the DC tone of the zero-offset comb has no power
    ph = np.rad2deg(np.angle(tones[first:]))
    want = -90.0 + 5.0 * np.arange(first, p.ntones)
    d = (ph - want + 180) % 360 - 180
    assert np.max(np.abs(d)) < 0.5, d


def test_pcallib_shifting_matches_direct_restatement():
    """Shifting (chosen when the rotator period is not a multiple of the bin
    count): per full rotator period only floor(R/N)*N rotated samples are
    added (PCal.cpp:451-462); the restated C against a direct numpy model,
    over a call with a tail and a second call."""
    import oracle as O
    bw, spacing, offset = 8e6, 1e6, 128000
    p = O.PcalLib(bw, spacing, offset, 5)
    assert p.kind == 2 and p.nbins == 16
    R, N = 125, 16
    rng = np.random.default_rng(3)
    x1 = rng.standard_normal(R * 7 + 40).astype(np.float32)
    x2 = rng.standard_normal(R * 3 + 70).astype(np.float32)
    p.extract(x1)
    p.extract(x2)
    tones, used = p.final()
    fs = 2 * bw
    rot = np.exp(1j * 2 * np.pi * (-offset / fs) * np.arange(2 * R)).astype(np.complex64).astype(np.complex128)
    acc = np.zeros(2 * N, complex)
    pi, ri = 5 % N, 5 % R
    for x in (x1, x2):
        tail = len(x) % R
        end = len(x) - tail
        for n in range(end):
            j = n % R
            if j < (R // N) * N:
                acc[pi + j % N] += x[n] * rot[ri + j]
        for m in range(tail):
            acc[pi + m % N] += x[end + m] * rot[ri + m]
        ri = (ri + tail) % R
        pi = (pi + tail % N) % N
    b = acc[:N] + acc[N:]
    dft = np.fft.fft(b) / N
    want = dft[:p.ntones]
    assert used == len(x1) + len(x2)
    assert np.max(np.abs(tones - want)) < 1e-9 * np.max(np.abs(want))


def _track_zones(frame: bytes, ntrack: int, mark4: bool) -> np.ndarray:
    """Blanked track-words of one VLBA payload / Mark4 frame by the rules the
    GPU's frame-validity kernel restates (blanker_mark5.c:126-280): 32 KiB
    zones judged by the fill pattern at their two ends, a binary search for
    the boundary with the 32-bit straggler check, Mark4's first zone after
    the header and its later zones examined 20 * ntrack / 8 words late, and
    a track-word blanked by its first byte."""
    tb, nword = ntrack // 8, len(frame) // 8
    w64 = np.frombuffer(frame, "<u8")
    w32 = np.frombuffer(frame, "<u4")
    F64, F32, big = 0x1122334411223344, 0x11223344, 1 << 30

    def first(b, e, invalid):
        n = e - b
        i, r, st = n // 2, n - 1, n // 4
        while st > 0:
            if (int(w64[b + i]) == F64) == invalid:
                r, i = i, i - st
            else:
                i += st
            st >>= 1
        r = 8 * (b + r)
        if invalid and int(w32[r // 4 - 1]) == F32:
            r -= 4
        if not invalid and int(w32[r // 4 - 2]) == F32:
            r += 4
        return r

    zones, b = [], 0
    while b < nword:
        e = min(b + 4096, nword)
        if mark4 and b == 0:
            b = 20 * tb
        s_ok, e_ok = int(w64[b]) != F64, int(w64[e - 1]) != F64
        r = [0, big] if s_ok and e_ok else [big, 0] if not (s_ok or e_ok) else \
            [0, first(b, e, True)] if s_ok else [first(b, e, False), big]
        if mark4 and not zones:
            r[0] = max(r[0], 160 * tb)
        zones.append(r)
        b += 4096
    m = np.arange(20000) * tb
    lo = np.array([zones[k][0] for k in m >> 15])
    hi = np.array([zones[k][1] for k in m >> 15])
    return (m < lo) | (m >= hi)


@pytest.mark.parametrize("fmt,ntrack", [("VLBA1_1-128-8-2", 16), ("VLBA1_4-512-8-2", 64), ("VLBA1_4-64-2-1", 8),
                                        ("MKIV1_2-512-8-2", 32), ("MKIV1_2-1024-16-2", 64)])
def test_track_zone_blanking_matches_live_mark5access(fmt, ntrack):
    """VLBA / Mark4 fill-pattern zones: the rules above against mark5access's
    own header-free unpack of planted frames (the blanked track-words decode
    to 0.0 in every channel)."""
    from helpers import plant_track_fill
    if O.ref() is None:
        pytest.skip("mark5access (oracle/_ref) not built")
    info = O.m5_format_info(fmt)
    fanout = ntrack // (info["nchan"] * info["nbit"])
    frame = 2500 * ntrack
    rng = np.random.default_rng(ntrack + 3)
    pay = plant_track_fill(rng.integers(0, 256, 3 * frame, dtype=np.uint8).tobytes(), ntrack)
    ref, nref = O.m5_unpack(fmt, pay, 3 * 20000 * fanout)
    seen = (ref[0] == 0.0).reshape(3, 20000, fanout).all(axis=2)
    want = np.stack([_track_zones(pay[f * frame:(f + 1) * frame], ntrack, fmt.startswith("MKIV"))
                     for f in range(3)])
    assert np.array_equal(seen, want)
    assert nref == int((~want).sum()) * fanout
