"""Shared test helpers: oracle runs and error metrics."""
from __future__ import annotations

import os

import numpy as np

import oracle as O
from swspec_b200 import synth

# Spectral parity bar: max relative error vs the FP64 oracle.
REL_TOL = 2e-6


def payload_of(framed: bytes, fmt: str) -> bytes:
    if fmt.startswith("Mark5B"):
        return synth.strip_headers(framed, 10016, 16)
    pl = int(fmt.split("_")[1].split("-")[0])
    return synth.strip_headers(framed, pl + 32, 32)


def decode_channels(framed: bytes, fmt: str, nchan: int, nbit: int, chans, nsamp: int):
    """Oracle decode of a framed stream with mark5access's blanking (fill
    zones; VDIF frames with the invalid bit)."""
    if fmt.startswith("Mark5B"):
        ofmt, pb, inv = O.FMT_MARK5B, 10000, None
    else:
        ofmt, pb = O.FMT_VDIF, int(fmt.split("_")[1].split("-")[0])
        inv = O.vdif_invalid_bits(framed, pb + 32)
    pay = payload_of(framed, fmt)
    return [O.decode(ofmt, nchan, nbit, pay, nsamp, c, payload_bytes=pb, frame_invalid=inv) for c in chans]


def oracle_run(samples, N, window, overlap, cof, nxpols=0, pcal=None):
    cfg = O.make_cfg(N, overlap=overlap, core_overlapped_ffts=cof, num_sources=len(samples),
                     num_xpols=nxpols, window=O.WINDOW_NAMES[window], nthreads=os.cpu_count() or 1)
    if pcal:
        cfg.extract_pcal = 1
        cfg.pcal_tonebins, cfg.pcal_rotatorlen = pcal["tonebins"], pcal["rotatorlen"]
        cfg.samplingfreq, cfg.pcaloffsethz = pcal["fs"], pcal["offset"]
    return O.domaths(cfg, samples)


def rel_err_auto(gpu: np.ndarray, ref: np.ndarray) -> float:
    return float(np.max(np.abs(gpu.astype(np.float64) - ref) / np.abs(ref)))


def rel_err_xpol(gpu: np.ndarray, ref: np.ndarray, ai: np.ndarray, aj: np.ndarray) -> float:
    return float(np.max(np.abs(gpu.astype(np.complex128) - ref) / np.sqrt(ai * aj)))


def fill_zone(raw: bytes, frame: int, start: int, end: int, frame_bytes: int, hdr: int) -> bytes:
    """Overwrite payload bytes [start, end) of a frame with the mark5 fill
    pattern 0x11223344 (little-endian words), as a recorder marks lost data."""
    a = bytearray(raw)
    base = frame * frame_bytes + hdr
    a[base + start: base + end] = bytes.fromhex("44332211") * ((end - start) // 4)
    return bytes(a)
