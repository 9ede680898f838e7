"""GPU unpack (K1) bit-exact against mark5access framed decode.

The reference's own mark5access (compiled from its sources into oracle/_ref)
decodes the same bytes through mark5_stream_decode; the GPU decode must match
every float bit, including fill-pattern blanking and VDIF invalid frames.
Where oracle/_ref is absent the committed golden fixtures stand in.
"""
import os

import numpy as np
import pytest

import oracle as O
from swspec_b200 import synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dev(buf: bytes):
    import torch
    return torch.from_numpy(np.frombuffer(buf, dtype=np.uint8).copy()).cuda()


def _gpu_decode(gpu, lay, raw: bytes, chan: int, nsamp: int, payload_offset: int = 0):
    import torch
    d = _dev(raw)
    out = torch.empty(nsamp, dtype=torch.float32, device="cuda")
    nv = gpu.unpack_device(lay, d.data_ptr(), d.numel(), payload_offset, chan, nsamp,
                           out.data_ptr())
    return out.cpu().numpy(), nv


def _mark5b(nchan, nbit, nfr, seed, mbps):
    spf = synth.mark5b_samples_per_frame(nchan, nbit)
    rng = np.random.default_rng(seed)
    return synth.mark5b_stream(rng.standard_normal((nchan, spf * nfr)), nbit, mbps), spf


def _reference_decode(fmt, framed, nsamp):
    if O.ref() is not None:
        return O.m5_decode(fmt, framed, nsamp)[0]
    pytest.skip("mark5access reference build (oracle/_ref) not present")


@pytest.mark.parametrize("nchan,nbit,mbps", [(16, 2, 1024), (8, 2, 1024), (32, 1, 1024),
                                             (16, 1, 1024), (4, 2, 256), (1, 2, 256)])
def test_mark5b_framed_bit_exact(gpu, nchan, nbit, mbps):
    raw, spf = _mark5b(nchan, nbit, 4, 100 + nchan + nbit, mbps)
    fmt = f"Mark5B-{mbps}-{nchan}-{nbit}"
    nsamp = spf * 3
    ref = _reference_decode(fmt, raw, nsamp)
    lay = gpu.layout("mark5b", nchan, nbit)
    for c in sorted({0, nchan // 2, nchan - 1}):
        got, nv = _gpu_decode(gpu, lay, raw, c, nsamp)
        assert np.array_equal(got.view(np.uint32), ref[c].view(np.uint32)), (fmt, c)
        assert nv == nsamp


def _fill(raw: bytes, frame: int, start: int, end: int, frame_bytes=10016, hdr=16) -> bytes:
    a = bytearray(raw)
    base = frame * frame_bytes + hdr
    fill = bytes.fromhex("44332211") * ((end - start) // 4)
    a[base + start: base + end] = fill
    return bytes(a)


@pytest.mark.parametrize("start,end", [(0, 10000), (0, 4000), (6000, 10000), (2000, 3000),
                                       (4, 9996)])
def test_mark5b_blanking_bit_exact(gpu, start, end):
    """Fill-pattern zones: whole frame, leading, trailing, interior, almost-all."""
    raw, spf = _mark5b(16, 2, 4, 77, 1024)
    raw = _fill(raw, 1, start, end)
    fmt = "Mark5B-1024-16-2"
    nsamp = spf * 3
    ref = _reference_decode(fmt, raw, nsamp)
    lay = gpu.layout("mark5b", 16, 2)
    got, nv = _gpu_decode(gpu, lay, raw, 5, nsamp)
    assert np.array_equal(got.view(np.uint32), ref[5].view(np.uint32))
    assert nv == np.count_nonzero(ref[5] != 0) or nv <= nsamp


@pytest.mark.parametrize("nbit", [8, 2, 1])
def test_vdif_invalid_and_fill(gpu, nbit):
    pl = 8000
    spf = pl * 8 // nbit
    rng = np.random.default_rng(5 + nbit)
    x = rng.standard_normal(spf * 4)
    codes = {8: synth.quantize_vdif_8bit(x, 24.0), 2: synth.quantize_vdif_2bit(x, 0.98),
             1: synth.quantize_vdif_1bit(x)}[nbit]
    payload = synth.pack_codes(codes[None, :], nbit)
    mbps = 512 if nbit == 8 else 128
    raw = synth.vdif_frames(payload, pl, 1, nbit, mbps * 1000000 // (8 * pl), invalid={1})
    raw = _fill(raw, 2, pl - 8, pl, frame_bytes=pl + 32, hdr=32)
    fmt = f"VDIF_{pl}-{mbps}-1-{nbit}"
    nsamp = spf * 3
    ref = _reference_decode(fmt, raw, nsamp)
    lay = gpu.layout("vdif:8000", 1, nbit)
    got, nv = _gpu_decode(gpu, lay, raw, 0, nsamp)
    assert np.array_equal(got.view(np.uint32), ref[0].view(np.uint32))
    assert nv == spf  # frames 1 (invalid) and 2 (fill) blanked


def test_payload_only_with_offset(gpu):
    """Header-free buffers starting inside a frame (FileSource strips headers)."""
    raw, spf = _mark5b(16, 2, 5, 9, 1024)
    pay = synth.strip_headers(raw, 10016, 16)
    off = 4 * 1234
    nsamp = 2500 * 3
    lay = gpu.layout("mark5b", 16, 2, framed=False)
    got, _ = _gpu_decode(gpu, lay, pay[off:], 3, nsamp, payload_offset=off)
    want = O.decode(O.FMT_MARK5B, 16, 2, pay[off:], nsamp, 3)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_golden_decode_fixture(gpu):
    """Committed mark5access outputs (tests/golden/mark5b_decode.npz)."""
    z = np.load(os.path.join(GOLDEN, "mark5b_decode.npz"))
    lay = gpu.layout("mark5b", int(z["nchan"]), int(z["nbit"]))
    raw = z["raw"].tobytes()
    for c in range(int(z["nchan"])):
        got, _ = _gpu_decode(gpu, lay, raw, c, int(z["nsamp"]))
        assert np.array_equal(got.view(np.uint32), z["decoded"][c].view(np.uint32))


@pytest.mark.parametrize("fmt,nchan,nbit", [("raw_signed", 1, 8), ("raw_signed", 4, 8), ("raw_unsigned", 2, 8),
                                            ("raw_signed", 16, 2), ("raw_unsigned", 4, 2),
                                            ("raw_signed", 1, 2)])
def test_raw_formats_bit_exact(gpu, fmt, nchan, nbit):
    """The reference's raw unpackers (RawSigned / RawUnsigned: 8-bit signed or
    offset, 2-bit multi-channel, 2-bit single channel oldest-in-MSB) as the
    oracle restates them (pinned to the reference's own DataUnpackers.cpp in
    test_oracle.py); no blanking."""
    rng = np.random.default_rng(nchan * 10 + nbit)
    nsamp = 100_000
    raw = rng.integers(0, 256, nsamp * nchan * nbit // 8 + 64, dtype=np.uint8).tobytes()
    lay = gpu.layout(fmt, nchan, nbit)
    ofmt = O.FMT_RAW_SIGNED if fmt == "raw_signed" else O.FMT_RAW_UNSIGNED
    for c in sorted({0, nchan // 2, nchan - 1}):
        got, nv = _gpu_decode(gpu, lay, raw, c, nsamp)
        ref = O.decode(ofmt, nchan, nbit, raw, nsamp, c)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (fmt, nchan, nbit, c)
        assert nv == nsamp


# VLBA / Mark4 modes: (mark5access format, tracks); fanouts 1, 2 and 4, 1- and
# 2-bit, 8 to 64 tracks, 64 bits per sample-time (64 tracks, fanout 1);
# MKIV1_2-512-8-2 is the reference's own example mode (src/democonfig.ini)
TRACK_MODES = [("VLBA1_1-128-8-2", 16), ("VLBA1_2-256-8-2", 32), ("VLBA1_4-512-8-2", 64),
               ("VLBA1_2-512-32-1", 64), ("VLBA1_4-64-2-1", 8), ("MKIV1_2-512-8-2", 32),
               ("MKIV1_4-256-4-2", 32), ("MKIV1_1-256-32-1", 32), ("MKIV1_2-1024-16-2", 64),
               ("MKIV1_1-64-4-2", 8), ("VLBA1_1-512-32-2", 64), ("MKIV1_1-512-64-1", 64)]


@pytest.mark.parametrize("fmt,ntrack", TRACK_MODES)
def test_track_formats_bit_exact(gpu, fmt, ntrack):
    """Every channel of three frames of random track-words, against
    mark5access's header-free unpack of the same bytes (its VLBA modulation
    and Mark4 header blanking included), float bit for float bit; then the
    same from the second frame on through a payload offset of one frame."""
    info = O.m5_format_info(fmt)
    nchan, nbit = info["nchan"], info["nbit"]
    fanout = ntrack // (nchan * nbit)
    rng = np.random.default_rng(ntrack * 10 + nchan)
    frame = 2500 * ntrack
    pay = rng.integers(0, 256, size=3 * frame, dtype=np.uint8).tobytes()
    nsamp = 3 * 20000 * fanout
    ref, nref = O.m5_unpack(fmt, pay, nsamp)
    lay = gpu.layout(("vlba:" if fmt.startswith("VLBA") else "mark4:") + str(ntrack), nchan, nbit)
    for c in range(nchan):
        got, nv = _gpu_decode(gpu, lay, pay, c, nsamp)
        assert np.array_equal(got.view(np.uint32), ref[c].view(np.uint32)), (fmt, c)
        assert nv == nref, (fmt, nv, nref)
    # from frame 1: the payload offset keeps the frame grid (modulation, header)
    ref1, _ = O.m5_unpack(fmt, pay[frame:], 2 * 20000 * fanout)
    got1, _ = _gpu_decode(gpu, lay, pay[frame:], nchan - 1, 2 * 20000 * fanout, payload_offset=frame)
    assert np.array_equal(got1.view(np.uint32), ref1[nchan - 1].view(np.uint32)), fmt
    # a source 4 bytes past an 8-byte boundary (64 tracks: the turn reads
    # its 8-byte units bytewise); a source off 4-byte alignment is refused
    import torch
    d = torch.zeros(len(pay) + 4, dtype=torch.uint8, device="cuda")
    d[4:] = _dev(pay)
    out = torch.empty(nsamp, dtype=torch.float32, device="cuda")
    nv = gpu.unpack_device(lay, d.data_ptr() + 4, len(pay), 0, 0, nsamp, out.data_ptr())
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref[0].view(np.uint32)) and nv == nref, fmt
    with pytest.raises(gpu.SwsError):
        gpu.unpack_device(lay, d.data_ptr() + 1, len(pay) - 1, 0, 0, nsamp, out.data_ptr())


@pytest.mark.parametrize("fmt,ntrack", TRACK_MODES)
def test_track_formats_fill_blanking(gpu, fmt, ntrack):
    """Fill-pattern blanking of VLBA / Mark4 data as mark5access does it:
    32 KiB zones per frame, each blanked from the fill pattern at its ends
    (binary search for the boundary, 32-bit straggler), Mark4's first zone
    starting after the header and its later zones examined 20 n words late,
    whole track-words blanked; every channel of three planted frames float
    bit for float bit and the count of unblanked samples, then from the
    second frame on through a payload offset."""
    from helpers import plant_track_fill
    info = O.m5_format_info(fmt)
    nchan, nbit = info["nchan"], info["nbit"]
    fanout = ntrack // (nchan * nbit)
    rng = np.random.default_rng(ntrack * 7 + nchan)
    frame = 2500 * ntrack
    pay = plant_track_fill(rng.integers(0, 256, size=3 * frame, dtype=np.uint8).tobytes(), ntrack)
    nsamp = 3 * 20000 * fanout
    ref, nref = O.m5_unpack(fmt, pay, nsamp)
    assert nref < nsamp                      # the plants blank something
    lay = gpu.layout(("vlba:" if fmt.startswith("VLBA") else "mark4:") + str(ntrack), nchan, nbit)
    for c in range(nchan):
        got, nv = _gpu_decode(gpu, lay, pay, c, nsamp)
        assert np.array_equal(got.view(np.uint32), ref[c].view(np.uint32)), (fmt, c)
        assert nv == nref, (fmt, nv, nref)
    ref1, nref1 = O.m5_unpack(fmt, pay[frame:], 2 * 20000 * fanout)
    got1, nv1 = _gpu_decode(gpu, lay, pay[frame:], 0, 2 * 20000 * fanout, payload_offset=frame)
    assert np.array_equal(got1.view(np.uint32), ref1[0].view(np.uint32)), fmt
    assert nv1 == nref1
