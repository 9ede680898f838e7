"""Batched uneven streams: per-stream FFT length, bit depth, bandwidth,
integration and tones drawn from a seed, each sized by the reference's
buffer plan (src/swspectrometer.cpp:166-231) into one core run per step.

Streams are single-channel VDIF payload (header-free, 8000-byte frames) of
1 or 2 bits at fs = 2 x bandwidth; FFT lengths come from {4096, 20000,
2^17, 2^20, 3,200,000}, bandwidths from 4-32 MHz, integrations from
0.1-10 s (clamped so that int(fs T / N) >= 1), and 0-3 tones each.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .settings import from_ini_values

LENGTHS = (4096, 20000, 1 << 17, 1 << 20, 3_200_000)


@dataclasses.dataclass
class StreamSpec:
    index: int
    fft_points: int
    nbit: int
    bandwidth_hz: float
    integration_s: float
    ntones: int
    tone_hz: tuple
    run_bytes: int            # payload bytes of one core run
    core_overlapped_ffts: int
    runs_per_spectrum: int

    @property
    def samplingfreq(self) -> float:
        return 2.0 * self.bandwidth_hz

    @property
    def samples_per_run(self) -> int:
        return self.run_bytes * 8 // self.nbit


def c4_streams(n: int = 64, seed: int = 2000, max_run_mb: int = 64) -> list[StreamSpec]:
    out = []
    for i in range(n):
        rng = np.random.default_rng(seed + i)
        N = int(rng.choice(LENGTHS))
        nbit = int(rng.choice([1, 2]))
        bw = float(rng.integers(4, 33)) * 1e6
        fs = 2.0 * bw
        T = float(10.0 ** rng.uniform(-1.0, 1.0))
        T = max(T, 1.000001 * N / fs)
        ntones = int(rng.integers(0, 4))
        tones = tuple(float(rng.uniform(0.05, 0.95) * bw) for _ in range(ntones))
        s = from_ini_values(fft_points=N, fft_integ_seconds=T, fft_overlap_factor=1, BandwidthHz=bw,
                            bits_per_sample=nbit, source_channels=1, MaxSourceBufferMB=max_run_mb)
        out.append(StreamSpec(i, N, nbit, bw, T, ntones, tones, int(s.rawbuf_size),
                              int(s.core_overlapped_ffts), max(1, int(s.max_buffers_per_spectrum))))
    return out


def stream_payload(spec: StreamSpec, rng: np.random.Generator | None = None) -> bytes:
    """One run of the stream: seeded unit noise plus its tones, quantised
    (VDIF 2-bit at +-0.98 sigma, or 1-bit), header-free payload."""
    from . import synth
    rng = rng or np.random.default_rng(9000 + spec.index)
    T = spec.samples_per_run
    x = rng.standard_normal(T)
    t = np.arange(T, dtype=np.float64) / spec.samplingfreq
    for f in spec.tone_hz:
        x += 0.3 * np.cos(2 * np.pi * f * t)
    codes = synth.quantize_vdif_2bit(x, 0.98) if spec.nbit == 2 else synth.quantize_vdif_1bit(x)
    return synth.pack_codes(codes[None, :], spec.nbit)
