"""Seeded synthetic VLBI streams (Mark5B and VDIF) for tests and benchmarks.

The reference's own test recording is not available, so every workload is a
seeded synthetic stream with the shapes of the benchmark configurations:

* Mark5B frames: 16-byte header (sync word 0xABADDEED, frame number within
  the second, BCD MJD/seconds/fraction; layout read by mark5access
  mark5_format_mark5b.c:139-189) followed by a 10000-byte payload.
* VDIF frames: 32-byte header (seconds from epoch, frame number, frame
  length in 8-byte units, log2(nchan), bits-1; format_vdif.c:2811-2826)
  followed by the payload.

Quantisation follows the mark5access level tables: Mark5B 2-bit codes are
(sign, magnitude) bit pairs with level[s + 2m] = {-H, +1, -1, +H}; VDIF 2-bit
codes index {-H, -1, +1, +H}; VDIF 8-bit is offset binary (2b-255)/256.
Thresholds at +-0.98 sigma (the "standard" 2-bit thresholds).
"""
from __future__ import annotations

import numpy as np

MARK5B_SYNC = 0xABADDEED
MARK5B_HEADER = 16
MARK5B_PAYLOAD = 10000
VDIF_HEADER = 32


# ----------------------------------------------------------------------------
# quantisers (value -> code) and packing
# ----------------------------------------------------------------------------

def quantize_mark5b_2bit(x: np.ndarray, thresh: float) -> np.ndarray:
    """Mark5B 2-bit code (bit0 = sign, bit1 = magnitude) for real samples."""
    s = (x >= 0).astype(np.uint8)
    m = (np.abs(x) >= thresh)
    # level[s + 2m] = {-H, +1, -1, +H}: negative small -> s=0,m=1 ; positive small -> s=1,m=0
    # negative large -> s=0,m=0 ; positive large -> s=1,m=1
    mag = np.where(s == 1, m, ~m).astype(np.uint8)
    return (s | (mag << 1)).astype(np.uint8)


def quantize_mark5b_1bit(x: np.ndarray) -> np.ndarray:
    """Mark5B 1-bit code: level {+1, -1}[bit]."""
    return (x < 0).astype(np.uint8)


def quantize_vdif_2bit(x: np.ndarray, thresh: float) -> np.ndarray:
    """VDIF 2-bit code indexing {-H, -1, +1, +H}."""
    c = np.where(x < -thresh, 0, np.where(x < 0, 1, np.where(x < thresh, 2, 3)))
    return c.astype(np.uint8)


def quantize_vdif_1bit(x: np.ndarray) -> np.ndarray:
    return (x >= 0).astype(np.uint8)


def quantize_vdif_8bit(x: np.ndarray, lsb_sigma: float) -> np.ndarray:
    """Offset-binary 8-bit code b with value (2b-255)/256; x in units of sigma,
    lsb_sigma = code steps per sigma.  Clips to [0, 255]."""
    b = np.floor(x * lsb_sigma / 2.0 + 128.0)
    return np.clip(b, 0, 255).astype(np.uint8)


def pack_codes(codes: np.ndarray, nbit: int) -> bytes:
    """Pack codes[nchan, T] into a payload: sample-time t occupies nchan*nbit
    bits from bit t*nchan*nbit, channel c at bit offset c*nbit, LSB-first."""
    nchan, T = codes.shape
    if nbit == 8:
        return np.ascontiguousarray(codes.T).astype(np.uint8).tobytes()
    bits_per_t = nchan * nbit
    assert (T * bits_per_t) % 8 == 0
    # bit matrix [T, nchan*nbit]
    bm = np.zeros((T, bits_per_t), dtype=np.uint8)
    for c in range(nchan):
        for b in range(nbit):
            bm[:, c * nbit + b] = (codes[c] >> b) & 1
    flat = bm.reshape(-1)
    return np.packbits(flat, bitorder="little").tobytes()


# ----------------------------------------------------------------------------
# framing
# ----------------------------------------------------------------------------

def _bcd(v: int, ndig: int) -> int:
    out = 0
    for i in range(ndig):
        out |= (v % 10) << (4 * i)
        v //= 10
    return out


def mark5b_frames(payload: bytes, mbps: int, mjd: int = 57000, sec: int = 100) -> bytes:
    """Wrap a payload stream (multiple of 10000 bytes) into Mark5B frames."""
    assert len(payload) % MARK5B_PAYLOAD == 0
    nfr = len(payload) // MARK5B_PAYLOAD
    frames_per_sec = mbps * 1000000 // (8 * MARK5B_PAYLOAD)
    out = np.empty((nfr, MARK5B_HEADER + MARK5B_PAYLOAD), dtype=np.uint8)
    pl = np.frombuffer(payload, dtype=np.uint8).reshape(nfr, MARK5B_PAYLOAD)
    out[:, MARK5B_HEADER:] = pl
    hdr = np.zeros((nfr, 4), dtype=np.uint32)
    for f in range(nfr):
        s = sec + f // frames_per_sec
        fn = f % frames_per_sec
        frac = (fn * 10000) // frames_per_sec  # 0.1 ms units
        hdr[f, 0] = MARK5B_SYNC
        hdr[f, 1] = (0xF00F << 16) | (fn & 0x7FFF)
        hdr[f, 2] = (_bcd(mjd % 1000, 3) << 20) | _bcd(s, 5)
        hdr[f, 3] = _bcd(frac, 4) << 16
    out[:, :MARK5B_HEADER] = hdr.view(np.uint8).reshape(nfr, MARK5B_HEADER)
    return out.tobytes()


def vdif_frames(payload: bytes, payload_bytes: int, nchan: int, nbit: int, frames_per_sec: int,
                sec: int = 1000000, epoch: int = 30, invalid: set | None = None, thread: int = 0) -> bytes:
    """Wrap a payload stream into VDIF frames with 32-byte headers (thread id
    in bits 16-25 of word 3)."""
    assert len(payload) % payload_bytes == 0
    nfr = len(payload) // payload_bytes
    fb = VDIF_HEADER + payload_bytes
    out = np.empty((nfr, fb), dtype=np.uint8)
    out[:, VDIF_HEADER:] = np.frombuffer(payload, dtype=np.uint8).reshape(nfr, payload_bytes)
    hdr = np.zeros((nfr, 8), dtype=np.uint32)
    log2nchan = int(np.log2(nchan))
    for f in range(nfr):
        s = sec + f // frames_per_sec
        fn = f % frames_per_sec
        w0 = s & 0x3FFFFFFF
        if invalid and f in invalid:
            w0 |= 1 << 31
        hdr[f, 0] = w0
        hdr[f, 1] = (epoch << 24) | (fn & 0xFFFFFF)
        hdr[f, 2] = (log2nchan << 24) | (fb // 8)
        hdr[f, 3] = ((nbit - 1) << 26) | ((thread & 0x3FF) << 16) | 0x4142  # station id "AB"
    out[:, :VDIF_HEADER] = hdr.view(np.uint8).reshape(nfr, VDIF_HEADER)
    return out.tobytes()


def strip_headers(framed: bytes, frame_bytes: int, header_bytes: int) -> bytes:
    a = np.frombuffer(framed, dtype=np.uint8).reshape(-1, frame_bytes)
    return a[:, header_bytes:].tobytes()


# ----------------------------------------------------------------------------
# signal recipes of the benchmark configurations
# ----------------------------------------------------------------------------

def gaussian_tone(rng: np.random.Generator, T: int, fs: float, tone_hz: float, amp: float,
                  phase: float = 0.0, t0: int = 0) -> np.ndarray:
    n = np.arange(t0, t0 + T, dtype=np.float64)
    return rng.standard_normal(T) + amp * np.cos(2 * np.pi * tone_hz / fs * n + phase)


def correlated_pair(rng: np.random.Generator, nframes: int, N: int, rho: float, phi: float):
    """Unit-variance real x, y with cross-spectrum rho*exp(i*phi) per bin,
    synthesised frame by frame in the frequency domain (frame-aligned)."""
    S = N // 2 + 1
    shape = (nframes, S)
    X = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    W = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    Y = rho * np.exp(1j * phi) * X + np.sqrt(1 - rho * rho) * W
    x = np.fft.irfft(X, n=N, axis=1)
    y = np.fft.irfft(Y, n=N, axis=1)
    x /= x.std()
    y /= y.std()
    return x.reshape(-1), y.reshape(-1)


def mark5b_stream(chan_signals: np.ndarray, nbit: int, mbps: int, thresh: float = 0.98,
                  framed: bool = True) -> bytes:
    """Quantise real signals[nchan, T] (unit sigma) into a Mark5B stream.
    T must fill whole 10000-byte payloads."""
    if nbit == 2:
        codes = quantize_mark5b_2bit(chan_signals, thresh)
    else:
        codes = quantize_mark5b_1bit(chan_signals)
    payload = pack_codes(codes, nbit)
    return mark5b_frames(payload, mbps) if framed else payload


def mark5b_samples_per_frame(nchan: int, nbit: int) -> int:
    return MARK5B_PAYLOAD * 8 // (nchan * nbit)


def c1_stream(seconds_or_frames: float, seed: int = 1001, fs: float = 32e6, nchan: int = 16,
              N: int = 32768, frames: int | None = None) -> tuple[bytes, dict]:
    """Plain method: 16 ch x 32 Msps 2-bit Mark5B; noise + CW at +3.1 MHz with
    20 dB per-bin SNR (Hann) on every channel."""
    spf = mark5b_samples_per_frame(nchan, 2)
    T = int(round(seconds_or_frames * fs)) if frames is None else frames * spf
    T = (T // spf) * spf
    rng = np.random.default_rng(seed)
    amp = np.sqrt(6.0 * 100.0 / N)
    sig = np.stack([gaussian_tone(rng, T, fs, 3.1e6, amp, phase=0.3 * c) for c in range(nchan)])
    sig /= np.sqrt(1.0 + amp * amp / 2.0)
    data = mark5b_stream(sig, 2, int(fs * nchan * 2 / 1e6))
    return data, dict(nsamp=T, fs=fs, nchan=nchan, nbit=2, fmt=f"Mark5B-{int(fs*nchan*2/1e6)}-{nchan}-2")


def c3_stream(nframes: int, seed: int = 1003, N: int = 65536, npairs: int = 8,
              rho: float = 0.3, phi: float = 0.7) -> tuple[bytes, dict]:
    """Dual-pol cross-spectra: 2 pol x 8 subbands at 64 Msps 2-bit
    (Mark5B-2048-16-2); channel c (X) pairs with c+8 (Y)."""
    fs = 64e6
    nchan = 2 * npairs
    rng = np.random.default_rng(seed)
    T = nframes * N
    spf = mark5b_samples_per_frame(nchan, 2)
    Tpad = ((T + spf - 1) // spf) * spf
    sig = np.zeros((nchan, Tpad))
    for p in range(npairs):
        x, y = correlated_pair(rng, nframes, N, rho, phi)
        sig[p, :T] = x
        sig[p + npairs, :T] = y
    if Tpad > T:
        sig[:, T:] = rng.standard_normal((nchan, Tpad - T))
    mbps = int(fs * nchan * 2 / 1e6)
    data = mark5b_stream(sig, 2, mbps)
    return data, dict(nsamp=Tpad, fs=fs, nchan=nchan, nbit=2, fmt=f"Mark5B-{mbps}-{nchan}-2")


def pcal_comb(T: int, fs: float, spacing: float, offset: float, amp: float, phases: np.ndarray,
              t0: int = 0) -> np.ndarray:
    """Sum of tones at k*spacing + offset (k = 0..len(phases)-1), FP64 phase."""
    n = np.arange(t0, t0 + T, dtype=np.float64)
    out = np.zeros(T)
    for k, ph in enumerate(phases):
        f = k * spacing + offset
        if f >= fs / 2:
            break
        out += amp * np.cos(2 * np.pi * ((f * n) % fs) / fs + ph)
    return out
