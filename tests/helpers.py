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


def track_fill_plants(ntrack: int):
    """Fill-pattern regions (frame, start, end) of a header-free VLBA payload
    or whole Mark4 frames (2500 * ntrack bytes) that exercise mark5access's
    32 KiB blanking zones (blanker_mark5.c:126-280): zone 0 filled to its end
    from a byte 4 past a 64-bit word (the 32-bit straggler check; at 64
    tracks the range boundary falls inside a track-word), the second frame's
    start (through the Mark4 header), its zone 1 whole, the first frame's
    zone 1 from a mid point to its end on the 32 KiB grid (Mark4 examines
    that zone 20 * ntrack / 8 words late and so blanks nothing there), a fill
    that touches neither end of its zone (not blanked) and the third frame's
    end."""
    frame = 2500 * ntrack
    z0e = min(32768, frame)
    plants = [(0, 4 + 8 * (z0e // 24), z0e), (1, 0, 8 * (z0e // 40) + 4), (2, 4000, 8000),
              (2, frame - 8004, frame)]
    if frame > 65536:
        plants.append((0, 32768 + 7820, 65536))
    if frame > 32768:
        plants.append((1, 32768, min(65536, frame)))
    return plants


def plant_track_fill(pay: bytes, ntrack: int, limit: int | None = None) -> bytes:
    """`pay` with track_fill_plants(ntrack) written in; with `limit`, only the
    plants whose zone (and the Mark4 blanker's shifted view of it) lies
    inside the first `limit` bytes."""
    frame = 2500 * ntrack
    for f, a, b in track_fill_plants(ntrack):
        if (f + 1) * frame > len(pay):
            continue
        z = a >> 15
        if limit is not None and f * frame + min((z + 1) * 32768 + 20 * ntrack, frame) > limit:
            continue
        pay = fill_zone(pay, f, a, b, frame, 0)
    return pay
