"""ctypes front end of the CPU oracle (test infrastructure only).

Loads oracle/liboracle.so (this directory's C restatement of the IPP core) and,
when present, oracle/_ref/libm5ref.so (the reference's own mark5access built
from its sources).  Only tests, the smoke check and the CPU-baseline leg of
the benchmark import this module; the GPU product never does.

Dispatcher-level behaviour (splitting the sample stream into core runs and
adding per-run partial spectra) follows src/TaskDispatcher.cpp:92-247 and
TaskCoreIPP::combineResults (src/IA-32/TaskCoreIPP.cpp:311-349).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None
_uref = None

W_NONE, W_COSINE, W_COSINE2, W_HAMMING, W_HANN, W_BLACKMAN, W_BLACKMANHARRIS = range(7)
WINDOW_NAMES = {"none": 0, "cosine": 1, "cosine2": 2, "hamming": 3, "hann": 4, "blackman": 5,
                "blackmanharris": 6}


class OrcCfg(C.Structure):
    _fields_ = [("fft_points", C.c_int), ("overlap", C.c_int),
                ("core_overlapped_ffts", C.c_int), ("num_sources", C.c_int),
                ("num_xpols", C.c_int), ("window", C.c_int), ("extract_pcal", C.c_int),
                ("pcal_tonebins", C.c_int), ("pcal_rotatorlen", C.c_int),
                ("samplingfreq", C.c_double), ("pcaloffsethz", C.c_double),
                ("nthreads", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        _lib.orc_decode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_int,
                                    C.c_void_p]
        _lib.orc_decode_blanked.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_int,
                                            C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        _lib.orc_decode_blanked.restype = C.c_int64
        _lib.orc_window.argtypes = [C.c_int, C.c_int, C.c_void_p]
        _lib.orc_fft64.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        _lib.orc_domaths64.argtypes = [C.POINTER(OrcCfg), C.c_void_p, C.c_int64, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        _lib.orc_domaths32.argtypes = [C.POINTER(OrcCfg), C.c_void_p, C.c_int64, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        _lib.orc_schedule.argtypes = [C.POINTER(OrcCfg), C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib.orc_pcal_tones.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
    return _lib


def ref():
    """The reference's mark5access (None when it was not built)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libm5ref.so")
        if not os.path.exists(path):
            return None
        _ref = C.CDLL(path)
        _ref.m5ref_decode.argtypes = [C.c_char_p, C.c_void_p, C.c_uint, C.c_int, C.c_int,
                                      C.c_void_p, C.POINTER(C.c_int)]
        _ref.m5ref_unpack.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        _ref.m5ref_format_info.argtypes = [C.c_char_p] + [C.POINTER(C.c_int)] * 6
        _ref.m5ref_frame_time.argtypes = [C.c_char_p, C.c_void_p, C.c_uint, C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    return _ref


# ----------------------------------------------------------------------------
# decoding
# ----------------------------------------------------------------------------

FMT_MARK5B, FMT_VDIF, FMT_RAW_SIGNED, FMT_RAW_UNSIGNED = 0, 1, 2, 3


def decode(fmt: int, nchan: int, nbit: int, payload: bytes, nsamp: int, chan: int,
           payload_bytes: int | None = None, frame_invalid=None) -> np.ndarray:
    """Samples of one channel of a header-free payload stream.  With
    payload_bytes (frame payload size; the stream starts at a frame) the
    mark5access blanking rules apply; frame_invalid holds VDIF header
    invalid bits per frame."""
    buf = np.frombuffer(payload, dtype=np.uint8)
    out = np.empty(nsamp, dtype=np.float32)
    if payload_bytes is None:
        rc = lib().orc_decode(fmt, nchan, nbit, buf.ctypes.data, nsamp, chan, out.ctypes.data)
        assert rc == 0
        return out
    inv = None
    if frame_invalid is not None:
        inv = np.ascontiguousarray(frame_invalid, dtype=np.uint8)
    rc = lib().orc_decode_blanked(fmt, nchan, nbit, buf.ctypes.data, len(buf), payload_bytes,
                                  None if inv is None else inv.ctypes.data, nsamp, chan, out.ctypes.data)
    assert rc >= 0
    return out


def vdif_invalid_bits(framed: bytes, frame_bytes: int) -> np.ndarray:
    """Invalid bit (word 0, bit 31) of every VDIF frame header."""
    a = np.frombuffer(framed, dtype=np.uint8).reshape(-1, frame_bytes)
    w0 = a[:, :4].copy().view(np.uint32)[:, 0]
    return ((w0 >> 31) & 1).astype(np.uint8)


def ref_unpack():
    """The reference's raw-data unpackers (src/IA-32/DataUnpackers.cpp, built
    with oracle/unpack_shim.cpp into _ref/libunpackref.so), or None."""
    global _uref
    if _uref is None:
        path = os.path.join(HERE, "_ref", "libunpackref.so")
        if not os.path.exists(path):
            return None
        _uref = C.CDLL(path)
        _uref.refunpack_raw.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_long, C.c_int]
        _uref.refunpack_raw.restype = C.c_long
    return _uref


RAW_SIGNED_8, RAW_UNSIGNED_8, RAW_TWOBIT, RAW_TWOBIT_1CH = range(4)


def ref_unpack_raw(kind: int, nbit: int, nchan: int, payload: bytes, count: int, chan: int,
                   increasing: bool = True) -> np.ndarray:
    """count samples of channel chan through the reference's own unpacker of
    the given kind (count is rounded up to the unpackers' 8/16-sample unroll)."""
    L = ref_unpack()
    buf = np.frombuffer(payload, dtype=np.uint8)
    n = (count + 15) // 16 * 16
    out = np.zeros(n + 16, dtype=np.float32)
    got = L.refunpack_raw(kind, nbit, nchan, int(increasing), buf.ctypes.data, out.ctypes.data, n, chan)
    assert got == n, got
    return out[:count]


class PcalLib:
    """The reference's PCal extractor classes (src/IA-32/PhaseCal/PCal.cpp)
    as restated in C: kind 0 = PCal::getNew's choice, 1 Trivial, 2 Shifting,
    3 ImplicitShift."""

    def __init__(self, bandwidth_hz, spacing_hz, offset_hz, sampleoffset=0, kind=0):
        L = lib()
        L.orc_pcallib_new.restype = C.c_void_p
        L.orc_pcallib_new.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int64, C.c_int]
        L.orc_pcallib_free.argtypes = [C.c_void_p]
        L.orc_pcallib_clear.argtypes = [C.c_void_p]
        L.orc_pcallib_adjust.argtypes = [C.c_void_p, C.c_int64]
        L.orc_pcallib_extract.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_pcallib_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        L.orc_pcallib_final.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_pcallib_final.restype = C.c_uint64
        self.L = L
        self.h = L.orc_pcallib_new(bandwidth_hz, spacing_hz, int(offset_hz), int(sampleoffset), kind)
        k, nb, nt = C.c_int(), C.c_int(), C.c_int()
        L.orc_pcallib_info(self.h, C.byref(k), C.byref(nb), C.byref(nt))
        self.kind, self.nbins, self.ntones = k.value, nb.value, nt.value

    def extract(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        self.L.orc_pcallib_extract(self.h, x.ctypes.data, len(x))

    def adjust(self, sampleoffset):
        self.L.orc_pcallib_adjust(self.h, int(sampleoffset))

    def clear(self):
        self.L.orc_pcallib_clear(self.h)

    def final(self):
        out = np.zeros(2 * self.ntones)
        n = self.L.orc_pcallib_final(self.h, out.ctypes.data)
        return out[0::2] + 1j * out[1::2], int(n)

    def __del__(self):
        try:
            self.L.orc_pcallib_free(self.h)
        except Exception:
            pass


def m5_format_info(fmt: str) -> dict:
    r = ref()
    vals = [C.c_int() for _ in range(6)]
    rc = r.m5ref_format_info(fmt.encode(), *[C.byref(v) for v in vals])
    assert rc == 0, fmt
    keys = ["nchan", "nbit", "framebytes", "payloadoffset", "framesamples", "samplegranularity"]
    return dict(zip(keys, [v.value for v in vals]))


def m5_decode(fmt: str, framed: bytes, nsamp: int) -> tuple[np.ndarray, int]:
    """mark5access framed decode -> float32[nchan, nsamp], return value."""
    r = ref()
    info = m5_format_info(fmt)
    out = np.zeros((info["nchan"], nsamp), dtype=np.float32)
    buf = np.frombuffer(framed, dtype=np.uint8).copy()
    off = C.c_int()
    rc = r.m5ref_decode(fmt.encode(), buf.ctypes.data, len(buf), nsamp, info["nchan"],
                        out.ctypes.data, C.byref(off))
    return out, rc


def m5_frame_time(fmt: str, framed: bytes) -> tuple[int, int, float, int]:
    """(mjd, second, ns, frame offset) of the first frame mark5access finds."""
    r = ref()
    mjd, sec, ns, off = C.c_int(), C.c_int(), C.c_double(), C.c_int()
    buf = np.frombuffer(framed, dtype=np.uint8).copy()
    rc = r.m5ref_frame_time(fmt.encode(), buf.ctypes.data, len(buf), C.byref(mjd), C.byref(sec), C.byref(ns),
                            C.byref(off))
    if rc != 0:
        raise RuntimeError(f"mark5access found no frame time ({rc})")
    return mjd.value, sec.value, ns.value, off.value


def m5_unpack(fmt: str, payload: bytes, nsamp: int) -> tuple[np.ndarray, int]:
    r = ref()
    info = m5_format_info(fmt)
    out = np.zeros((info["nchan"], nsamp), dtype=np.float32)
    # mark5_unpack moves on to the frame after the last sample it decodes
    # and runs the blanker there: zero bytes of one frame (at most 64 tracks
    # x 2520 bytes) past the payload keep those reads inside the buffer
    buf = np.zeros(len(payload) + 64 * 2520, dtype=np.uint8)
    buf[:len(payload)] = np.frombuffer(payload, dtype=np.uint8)
    rc = r.m5ref_unpack(fmt.encode(), buf.ctypes.data, nsamp, info["nchan"], out.ctypes.data)
    return out, rc


# ----------------------------------------------------------------------------
# windows, FFT
# ----------------------------------------------------------------------------

def window(wtype: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    lib().orc_window(wtype, n, out.ctypes.data)
    return out


def fft64(x: np.ndarray) -> np.ndarray:
    xin = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(xin)
    lib().orc_fft64(len(xin), xin.ctypes.data, out.ctypes.data)
    return out


# ----------------------------------------------------------------------------
# doMaths over one buffer
# ----------------------------------------------------------------------------

def make_cfg(N, overlap=1, core_overlapped_ffts=1, num_sources=1, num_xpols=0, window=W_HANN,
             extract_pcal=False, pcal_tonebins=0, pcal_rotatorlen=0, samplingfreq=32e6,
             pcaloffsethz=10e3, nthreads=1) -> OrcCfg:
    return OrcCfg(N, overlap, core_overlapped_ffts, num_sources, num_xpols, window,
                  int(bool(extract_pcal)), pcal_tonebins, pcal_rotatorlen, samplingfreq,
                  pcaloffsethz, nthreads)


def schedule(cfg: OrcCfg, nsamp: int):
    ns, part = C.c_int(), C.c_int()
    nf = lib().orc_schedule(C.byref(cfg), nsamp, None, None, 0, C.byref(ns), C.byref(part))
    starts = np.zeros(max(nf, 1), dtype=np.int64)
    spec = np.zeros(max(nf, 1), dtype=np.int32)
    lib().orc_schedule(C.byref(cfg), nsamp, starts.ctypes.data, spec.ctypes.data, nf,
                       C.byref(ns), C.byref(part))
    return starts[:nf], spec[:nf], ns.value, bool(part.value)


def domaths(cfg: OrcCfg, samples: list[np.ndarray], fp64: bool = True):
    """One core run.  Returns (auto[nspec, nsrc, S], xpol[nspec, nxp, S] complex,
    pcal[nspec, nsrc, tonebins] complex, nspec)."""
    N = cfg.fft_points
    S = N // 2 + 1
    nsamp = min(len(s) for s in samples)
    _, _, nspec, _ = schedule(cfg, nsamp)
    dt = np.float64 if fp64 else np.float32
    srcs = [np.ascontiguousarray(s, dtype=np.float32) for s in samples]
    ptrs = (C.c_void_p * len(srcs))(*[s.ctypes.data for s in srcs])
    na = max(nspec, 1) * cfg.num_sources * S
    auto = np.zeros(na, dtype=dt)
    xpol = np.zeros(max(nspec, 1) * max(cfg.num_xpols, 1) * S * 2, dtype=dt)
    pcal = np.zeros(max(nspec, 1) * cfg.num_sources * max(cfg.pcal_tonebins, 1) * 2, dtype=dt)
    fn = lib().orc_domaths64 if fp64 else lib().orc_domaths32
    n = fn(C.byref(cfg), ptrs, nsamp, auto.ctypes.data, xpol.ctypes.data, pcal.ctypes.data)
    auto = auto[: n * cfg.num_sources * S].reshape(n, cfg.num_sources, S)
    xp = xpol[: n * cfg.num_xpols * S * 2].reshape(n, cfg.num_xpols, S, 2)
    xp = xp[..., 0] + 1j * xp[..., 1]
    tb = cfg.pcal_tonebins
    pc = pcal[: n * cfg.num_sources * tb * 2].reshape(n, cfg.num_sources, tb, 2)
    pc = pc[..., 0] + 1j * pc[..., 1]
    return auto, xp, pc, n


def pcal_tones(bins: np.ndarray, nfolded: float, ntones: int) -> np.ndarray:
    b = np.ascontiguousarray(np.stack([bins.real, bins.imag], -1).reshape(-1), dtype=np.float64)
    out = np.zeros(2 * ntones)
    lib().orc_pcal_tones(len(bins), b.ctypes.data, float(nfolded), ntones, out.ctypes.data)
    return out[0::2] + 1j * out[1::2]
