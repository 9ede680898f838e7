"""Device-side generator of the benchmark streams (same recipe as synth.py).

Benchmark inputs are hundreds of MB; building them with numpy takes minutes,
so this module synthesises them on the GPU with torch (input preparation
only -- nothing here is part of the measured spectrometer path).  The recipe
matches synth.c3_stream: per 65536-sample frame, complex Gaussian spectra X,
Y = rho e^{i phi} X + sqrt(1 - rho^2) W, inverse real FFT, unit variance,
2-bit Mark5B quantisation at +-0.98 sigma, framed with valid Mark5B headers.
"""
from __future__ import annotations

import numpy as np
import torch

from . import synth


def _bcd(v: int, ndig: int) -> int:
    return synth._bcd(v, ndig)


def mark5b_headers(nfr: int, mbps: int, mjd: int = 57000, sec: int = 100) -> np.ndarray:
    fps = mbps * 1000000 // (8 * synth.MARK5B_PAYLOAD)
    f = np.arange(nfr)
    s = sec + f // fps
    fn = f % fps
    frac = (fn * 10000) // fps
    hdr = np.zeros((nfr, 4), dtype=np.uint32)
    hdr[:, 0] = synth.MARK5B_SYNC
    hdr[:, 1] = (0xF00F << 16) | (fn & 0x7FFF)
    bcd_s = np.array([_bcd(int(x), 5) for x in np.unique(s)], dtype=np.uint64)
    lut = dict(zip(np.unique(s).tolist(), bcd_s.tolist()))
    hdr[:, 2] = np.array([(_bcd(mjd % 1000, 3) << 20) | lut[int(x)] for x in s], dtype=np.uint32)
    hdr[:, 3] = np.array([_bcd(int(x), 4) << 16 for x in frac], dtype=np.uint32)
    return hdr


def quantize_mark5b_2bit(x: torch.Tensor, thresh: float = 0.98) -> torch.Tensor:
    s = (x >= 0)
    m = x.abs() >= thresh
    mag = torch.where(s, m, ~m)
    return s.to(torch.int32) | (mag.to(torch.int32) << 1)


def c3_framed(nsamp_time: int, N: int = 65536, npairs: int = 8, rho: float = 0.3,
              phi: float = 0.7, seed: int = 1003, device: str = "cuda") -> tuple[torch.Tensor, int]:
    """Framed Mark5B-2048-16-2 bytes on the device holding at least
    nsamp_time sample-times (whole frames).  Returns (uint8 tensor, nframes)."""
    nchan = 2 * npairs
    spf = synth.mark5b_samples_per_frame(nchan, 2)
    nfr = (nsamp_time + spf - 1) // spf
    T = nfr * spf
    nfft = (T + N - 1) // N
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    S = N // 2 + 1
    words = torch.zeros(nfft * N, dtype=torch.int64, device=device)
    c = complex(rho * np.cos(phi), rho * np.sin(phi))
    for p in range(npairs):
        X = torch.complex(torch.randn(nfft, S, generator=g, device=device),
                          torch.randn(nfft, S, generator=g, device=device))
        W = torch.complex(torch.randn(nfft, S, generator=g, device=device),
                          torch.randn(nfft, S, generator=g, device=device))
        Y = c * X + np.sqrt(1 - rho * rho) * W
        x = torch.fft.irfft(X, n=N, dim=1).reshape(-1)
        y = torch.fft.irfft(Y, n=N, dim=1).reshape(-1)
        x = x / x.std()
        y = y / y.std()
        words |= quantize_mark5b_2bit(x).to(torch.int64) << (2 * p)
        words |= quantize_mark5b_2bit(y).to(torch.int64) << (2 * (p + npairs))
        del X, W, Y, x, y
    # low 32 bits as int32 (two's complement wrap of the packed word)
    payload = (words[:T] & 0xFFFFFFFF).to(torch.int32).reshape(nfr, spf)
    frames = torch.empty(nfr, 4 + spf, dtype=torch.int32, device=device)
    mbps = 2 * nchan * 64  # 64 Msps x nchan x 2 bits
    hdr = torch.from_numpy(mark5b_headers(nfr, mbps).view(np.int32)).to(device)
    frames[:, :4] = hdr
    frames[:, 4:] = payload
    return frames.reshape(-1).view(torch.uint8), nfr


def _chunks(T: int, chunk: int = 1 << 24):
    for t0 in range(0, T, chunk):
        yield t0, min(chunk, T - t0)


def mark5b_payload(T: int, nchan: int, fs: float, seed: int, tone_hz: float = 0.0, tone_amp: float = 0.0,
                   comb: tuple | None = None, device: str = "cuda") -> torch.Tensor:
    """Header-free Mark5B payload (nchan 2-bit channels, +-0.98 sigma
    thresholds) of T sample-times on the device: seeded unit Gaussian noise
    per channel, plus a CW tone in channel 0 (tone_hz, amplitude tone_amp in
    sigma) and/or a phase-cal comb in every channel, comb = (spacing_hz,
    offset_hz, amp_sigma, phases): tones at k spacing + offset below fs/2,
    FP64 phase, periodic in fs / gcd(fs, offset) samples, so one period is
    computed and tiled.  nchan * 2 = 32 bits per sample-time."""
    assert nchan * 2 == 32
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty(T, dtype=torch.int32, device=device)
    period = None
    if comb is not None:
        spacing, offset, amp, phases = comb
        per = int(round(fs / np.gcd(int(fs), int(offset))))
        n = torch.arange(per, dtype=torch.float64, device=device)
        period = torch.zeros(per, dtype=torch.float64, device=device)
        for k, ph in enumerate(phases):
            f = k * spacing + offset
            if f >= fs / 2:
                break
            period += amp * torch.cos(2 * np.pi * torch.remainder(f * n, fs) / fs + ph)
        period = period.to(torch.float32)
    for t0, L in _chunks(T):
        w = torch.zeros(L, dtype=torch.int64, device=device)
        add = None
        if period is not None:
            idx = torch.remainder(torch.arange(t0, t0 + L, device=device), period.numel())
            add = period[idx]
        for c in range(nchan):
            x = torch.randn(L, generator=g, device=device)
            if add is not None:
                x += add
            if c == 0 and tone_amp:
                n = torch.arange(t0, t0 + L, dtype=torch.float64, device=device)
                x += (tone_amp * torch.cos(2 * np.pi * torch.remainder(tone_hz * n, fs) / fs)).to(torch.float32)
            w |= quantize_mark5b_2bit(x).to(torch.int64) << (2 * c)
        out[t0:t0 + L] = (w & 0xFFFFFFFF).to(torch.int32)
    return out.view(torch.uint8)


def vdif8_carrier_payload(T: int, fs: float, seed: int, f0: float, drift_hz_s: float, snr_bin_db: float,
                          N: int, lsb_sigma: float = 24.0, device: str = "cuda") -> torch.Tensor:
    """Header-free single-channel 8-bit VDIF payload (offset binary, code
    b = floor(x lsb_sigma / 2 + 128) clipped to [0, 255], so lsb_sigma / 2
    codes per sigma) of T samples:
    unit Gaussian noise plus a carrier snr_bin_db above the per-bin noise
    floor of an N-point FFT, at f0 drifting drift_hz_s, FP64 phase."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    A = float(np.sqrt(4 * 10 ** (snr_bin_db / 10) * 2.0 / N))  # equivalent noise bandwidth 2 bins
    out = torch.empty(T, dtype=torch.uint8, device=device)
    for t0, L in _chunks(T):
        t = torch.arange(t0, t0 + L, dtype=torch.float64, device=device) / fs
        cyc = torch.remainder(f0 * t + 0.5 * drift_hz_s * t * t, 1.0)
        x = torch.randn(L, generator=g, device=device) + (A * torch.cos(2 * np.pi * cyc)).to(torch.float32)
        out[t0:t0 + L] = torch.clamp(torch.floor(x * (lsb_sigma / 2.0) + 128.0), 0, 255).to(torch.uint8)
    return out
