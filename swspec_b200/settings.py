"""Derived spectrometer settings, as src/swspectrometer.cpp:166-231 computes them.

Mirrors swspect_settings_t (src/Settings.h:59-159).  Used by the tests and the
benchmark to size runs exactly as the reference's main() does; the C++ host
(swspec_b200/host/settings.cpp) carries the same derivation for the
drop-in TaskCore path.
"""
from __future__ import annotations

import dataclasses
import math

PLATFORM_MAX_RAW_BUF_SIZE_MB = 32  # INTEL_IPP build (src/Settings.h:30-31)


def _gcd(a: int, b: int) -> int:
    # Helpers::gcd (src/Helpers.cpp:150-162)
    while True:
        a = a % b
        if a == 0:
            return b
        b = b % a
        if b == 0:
            return a


@dataclasses.dataclass
class Settings:
    num_cores: int = 1
    max_rawbuf_size: int = PLATFORM_MAX_RAW_BUF_SIZE_MB * 1024 * 1024
    fft_points: int = 320000
    fft_integ_seconds: float = 20.0
    fft_overlap_factor: int = 2
    wf_type: str = "cosine2"
    samplingfreq: float = 16e6
    pcaloffsethz: float = 10e3
    pcalharmonicshz: float = 1e6
    bits_per_sample: int = 8
    source_channels: int = 1
    use_channel_file1: int = 0       # 0-based after main() decrements it
    use_channel_file2: int = 0
    extract_PCal: bool = False
    calc_Xpol: bool = False
    num_sources: int = 1
    # derived
    averaged_ffts: int = 0
    fft_overlap_points: int = 0
    fft_ssb_points: int = 0
    rawbytes_per_channelsample: float = 0.0
    raw_fullfft_bytes: int = 0
    raw_overlap_bytes: int = 0
    pcal_tonebins: int = 0
    pcal_rotatorlen: int = 0
    pcal_pulses_per_fft: int = 0
    max_spectra_per_buffer: int = 0
    max_specffts_per_buffer: int = 0
    max_buffers_per_spectrum: int = 0
    rawbuf_size: int = 0
    core_averaged_ffts: int = 0
    core_overlapped_ffts: int = 0

    def derive(self) -> "Settings":
        fs = float(_f32(self.samplingfreq))
        N = self.fft_points
        # swsfloat_t arithmetic, truncated to int on assignment
        self.averaged_ffts = int(_f32(_f32(fs * _f32(self.fft_integ_seconds)) / N))
        self.fft_overlap_points = N // self.fft_overlap_factor
        self.fft_ssb_points = N // 2 + 1
        self.rawbytes_per_channelsample = (self.bits_per_sample * self.source_channels) / 8.0
        self.raw_fullfft_bytes = int(N * self.rawbytes_per_channelsample)
        self.raw_overlap_bytes = int(self.fft_overlap_points * self.rawbytes_per_channelsample)
        if self.extract_PCal:
            self.pcal_tonebins = int(fs / self.pcalharmonicshz)
            self.pcal_rotatorlen = int(fs / _gcd(int(fs), int(self.pcaloffsethz)))
            self.pcal_pulses_per_fft = N // self.pcal_rotatorlen
            if N % self.pcal_rotatorlen != 0:
                self.extract_PCal = False
        self.max_rawbuf_size = self.max_rawbuf_size // self.num_cores
        tent = self.raw_fullfft_bytes * self.averaged_ffts
        if tent > self.max_rawbuf_size:
            self.max_spectra_per_buffer = 0
            self.max_specffts_per_buffer = 1
            self.max_buffers_per_spectrum = self.averaged_ffts
            tent = self.raw_fullfft_bytes
            while tent <= self.max_rawbuf_size and self.max_buffers_per_spectrum % 2 == 0:
                tent *= 2
                self.max_buffers_per_spectrum //= 2
                self.max_specffts_per_buffer *= 2
        else:
            self.max_spectra_per_buffer = 1
            self.max_specffts_per_buffer = self.averaged_ffts
            self.max_buffers_per_spectrum = 0
            while 2 * tent <= self.max_rawbuf_size:
                tent *= 2
                self.max_spectra_per_buffer *= 2
        self.rawbuf_size = tent
        self.core_averaged_ffts = self.max_specffts_per_buffer
        f = self.fft_overlap_factor
        self.core_overlapped_ffts = f * self.max_specffts_per_buffer - (f - 1)
        return self


def _f32(x: float) -> float:
    import numpy as np
    return float(np.float32(x))


def from_ini_values(**kw) -> Settings:
    """Settings from INI-style values (BandwidthHz -> fs = 2*BW, MaxSourceBufferMB
    -> bytes/2 per the double-buffer rule of swspectrometer.cpp:104-106)."""
    s = Settings()
    if "MaxSourceBufferMB" in kw:
        s.max_rawbuf_size = int(kw.pop("MaxSourceBufferMB")) * 1024 * 1024 // 2
    if "BandwidthHz" in kw:
        s.samplingfreq = float(kw.pop("BandwidthHz")) * 2.0
    for k, v in kw.items():
        setattr(s, k, v)
    return s.derive()
