"""ctypes binding of libswsgpu.so (include/swsgpu.h).

The native library is the product; this module only marshals arguments.  It
refuses to run without the library: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libswsgpu.so")

FMT_MARK5B, FMT_VDIF, FMT_RAW_SIGNED, FMT_RAW_UNSIGNED, FMT_VLBA, FMT_MARK4 = 0, 1, 2, 3, 4, 5
WIN = {"none": 0, "cosine": 1, "cosine2": 2, "hamming": 3, "hann": 4, "blackman": 5,
       "blackmanharris": 6}
PREC_FP32, PREC_TCSPLIT, PREC_TCSPLIT_ALL = 0, 1, 2
PLAN_DEFAULT, PLAN_CLUSTER, PLAN_FOURSTEP = 0, 1, 2
INJECT_NONE, INJECT_DROP_EXCHANGE = 0, 1
MAX_SOURCES = 64
MAX_STREAMS = 2

ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ETIMEOUT", -4: "ENODEV", -5: "ESTATE",
          -6: "ETOOBIG"}


class Layout(C.Structure):
    _fields_ = [("format", C.c_int), ("nchan", C.c_int), ("nbit", C.c_int),
                ("frame_bytes", C.c_int), ("header_bytes", C.c_int)]


class Config(C.Structure):
    _fields_ = [("layout", Layout * MAX_STREAMS), ("num_streams", C.c_int),
                ("fft_points", C.c_int), ("overlap", C.c_int), ("window", C.c_int),
                ("precision", C.c_int), ("core_overlapped_ffts", C.c_int),
                ("num_sources", C.c_int), ("source_stream", C.c_int * MAX_SOURCES),
                ("source_channel", C.c_int * MAX_SOURCES), ("num_xpols", C.c_int),
                ("xpol_pair", (C.c_int * 2) * MAX_SOURCES), ("extract_pcal", C.c_int),
                ("pcal_tonebins", C.c_int), ("pcal_rotatorlen", C.c_int),
                ("samplingfreq", C.c_double), ("pcal_offset_hz", C.c_double),
                ("max_run_bytes", C.c_size_t), ("runs_per_output", C.c_int),
                ("pcal_ntones", C.c_int), ("autotune", C.c_int), ("plan_family", C.c_int),
                ("plan_candidate", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [("auto_out", C.c_void_p), ("xpol_out", C.c_void_p), ("pcal_out", C.c_void_p),
                ("tones_out", C.c_void_p)]


class SwsError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libswsgpu.so; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SwsError(f"{LIB_PATH} is not built; run swspec_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.swsgpu_create.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(C.c_void_p)]
        L.swsgpu_destroy.argtypes = [C.c_void_p]
        L.swsgpu_last_error.argtypes = [C.c_void_p]
        L.swsgpu_last_error.restype = C.c_char_p
        L.swsgpu_run_shape.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.swsgpu_submit.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_int64)]
        L.swsgpu_submit_out.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                        C.POINTER(C.c_int64), C.POINTER(Outputs)]
        L.swsgpu_wait.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.swsgpu_fetch.argtypes = [C.c_void_p, C.POINTER(Outputs)]
        L.swsgpu_process_device.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t, C.c_int,
                                            C.c_int, C.POINTER(Outputs), C.c_void_p]
        L.swsgpu_workspace_size.argtypes = [C.c_void_p, C.c_size_t, C.c_int,
                                            C.POINTER(C.c_size_t)]
        L.swsgpu_unpack_device.argtypes = [C.POINTER(Layout), C.c_void_p, C.c_size_t, C.c_int64,
                                           C.c_int, C.c_int64, C.c_void_p, C.POINTER(C.c_int64),
                                           C.c_void_p]
        L.swsgpu_last_launch_count.argtypes = [C.c_void_p]
        L.swsgpu_unpack_device_noalloc.argtypes = [C.POINTER(Layout), C.c_void_p, C.c_size_t,
                                                   C.c_int64, C.c_int, C.c_int64, C.c_void_p,
                                                   C.POINTER(C.c_int64), C.c_void_p]
        L.swsgpu_device_ok.argtypes = [C.c_int]
        L.swsgpu_profile.argtypes = [C.c_void_p, C.c_int]
        L.swsgpu_profile_read.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.swsgpu_autotune.argtypes = [C.c_void_p, C.c_int]
        L.swsgpu_plan_info.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.swsgpu_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        L.swsgpu_batch_set.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_size_t, C.c_int,
                                       C.c_int, C.POINTER(Outputs)]
        L.swsgpu_batch_launch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        L.swsgpu_batch_destroy.argtypes = [C.c_void_p]
        L.swsgpu_batch_destroy.restype = None
        L.swsgpu_host_register.argtypes = [C.c_void_p, C.c_size_t]
        L.swsgpu_host_unregister.argtypes = [C.c_void_p]
        L.swsgpu_sync.argtypes = [C.c_void_p, C.c_void_p]
        L.swsgpu_pcal_create.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int64, C.c_int, C.c_int,
                                         C.POINTER(C.c_void_p)]
        L.swsgpu_pcal_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        L.swsgpu_pcal_clear.argtypes = [C.c_void_p]
        L.swsgpu_pcal_adjust_offset.argtypes = [C.c_void_p, C.c_int64]
        L.swsgpu_pcal_extract.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.swsgpu_pcal_final.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]
        L.swsgpu_pcal_destroy.argtypes = [C.c_void_p]
        L.swsgpu_pcal_destroy.restype = None
        L.swsgpu_pcal_delay.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double]
        L.swsgpu_pcal_delay.restype = C.c_double
        L.swsgpu_inject.argtypes = [C.c_void_p, C.c_int]
        _lib = L
    return _lib


def _check(rc: int, h=None) -> None:
    if rc != 0:
        msg = lib().swsgpu_last_error(h).decode()
        raise SwsError(f"{ERRORS.get(rc, rc)}: {msg}")


def layout(fmt: str, nchan: int, nbit: int, framed: bool = True) -> Layout:
    """Layout of a Mark5B or VDIF stream ("mark5b" / "vdif:<payload>"), of
    header-free raw sampler data ("raw_signed" / "raw_unsigned"), or of a
    track format ("vlba:<tracks>": header-free payload; "mark4:<tracks>":
    whole frames) of 20000 track-words per frame."""
    if fmt.lower().startswith(("vlba", "mark4")):
        ntrack = int(fmt.split(":")[1])
        return Layout(FMT_VLBA if fmt.lower().startswith("vlba") else FMT_MARK4, nchan, nbit, 2500 * ntrack, 0)
    if fmt.lower().startswith("raw"):
        code = FMT_RAW_SIGNED if fmt.lower() == "raw_signed" else FMT_RAW_UNSIGNED
        return Layout(code, nchan, nbit, 8192, 0)
    if fmt.lower().startswith("mark5b"):
        return Layout(FMT_MARK5B, nchan, nbit, 10016 if framed else 10000, 16 if framed else 0)
    payload = int(fmt.split(":")[1]) if ":" in fmt else 8000
    return Layout(FMT_VDIF, nchan, nbit, payload + (32 if framed else 0), 32 if framed else 0)


def make_config(lay: Layout, N: int, window="hann", overlap=1, core_overlapped_ffts=1,
                sources=((0, 0),), xpols=(), precision=PREC_FP32, max_run_bytes=1 << 24,
                extract_pcal=False, pcal_tonebins=0, pcal_rotatorlen=0, samplingfreq=32e6,
                pcal_offset_hz=10e3, layout2: Layout | None = None,
                runs_per_output: int = 1, pcal_ntones: int = 0, autotune: bool = False,
                plan_family: int = 0, plan_candidate: int = 0) -> Config:
    c = Config()
    c.layout[0] = lay
    c.layout[1] = layout2 if layout2 is not None else lay
    c.num_streams = 1 + max(s for s, _ in sources)
    c.fft_points = N
    c.overlap = overlap
    c.window = WIN[window] if isinstance(window, str) else int(window)
    c.precision = precision
    c.core_overlapped_ffts = core_overlapped_ffts
    c.num_sources = len(sources)
    for i, (st, ch) in enumerate(sources):
        c.source_stream[i] = st
        c.source_channel[i] = ch
    c.num_xpols = len(xpols)
    for i, (a, b) in enumerate(xpols):
        c.xpol_pair[i][0] = a
        c.xpol_pair[i][1] = b
    c.extract_pcal = int(bool(extract_pcal))
    c.pcal_tonebins = pcal_tonebins
    c.pcal_rotatorlen = pcal_rotatorlen
    c.samplingfreq = samplingfreq
    c.pcal_offset_hz = pcal_offset_hz
    c.max_run_bytes = max_run_bytes
    c.runs_per_output = runs_per_output
    c.pcal_ntones = pcal_ntones
    c.autotune = int(bool(autotune))
    c.plan_family = plan_family
    c.plan_candidate = plan_candidate
    return c


class Core:
    """One GPU spectrometer core (a TaskCore's compute half)."""

    def __init__(self, cfg: Config, device: int = 0):
        self.cfg = cfg
        self.h = C.c_void_p()
        _check(lib().swsgpu_create(C.byref(cfg), device, C.byref(self.h)))
        self.S = cfg.fft_points // 2 + 1

    def close(self):
        if self.h:
            lib().swsgpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_shape(self, nbytes: int):
        ns, nf, part = C.c_int(), C.c_int(), C.c_int()
        _check(lib().swsgpu_run_shape(self.h, nbytes, C.byref(ns), C.byref(nf), C.byref(part)),
               self.h)
        return ns.value, nf.value, bool(part.value)

    def last_launches(self) -> int:
        return lib().swsgpu_last_launch_count(self.h)

    def profile(self, enable: bool) -> None:
        _check(lib().swsgpu_profile(self.h, int(enable)), self.h)

    def profile_read(self) -> tuple[int, float]:
        n, ms = C.c_int(), C.c_double()
        _check(lib().swsgpu_profile_read(self.h, C.byref(n), C.byref(ms)), self.h)
        return n.value, ms.value

    def submit(self, raws: list, payload_offsets=None, dest=None) -> None:
        """swsgpu_submit; with dest = (auto, xpol, pcal, tones) arrays (None
        for any not wanted) swsgpu_submit_out, which writes a completed run's
        spectra there (page-locked arrays get the device copies directly)."""
        n = len(raws)
        # argument arrays kept across calls: a run's submit is on the
        # per-run critical path of the host loop
        if getattr(self, "_sub_n", 0) != n:
            self._sub_n = n
            self._sub_ptrs = (C.c_void_p * n)()
            self._sub_sizes = (C.c_size_t * n)(*self._sizes)
            self._sub_offs = (C.c_int64 * n)()
        for i, r in enumerate(raws):
            self._sub_ptrs[i] = int(r) if isinstance(r, int) else r.ctypes.data
            self._sub_offs[i] = payload_offsets[i] if payload_offsets else 0
        if dest is None:
            _check(lib().swsgpu_submit(self.h, self._sub_ptrs, self._sub_sizes, self._sub_offs), self.h)
            return
        # the destination descriptor is rebuilt only when other arrays come
        # (the arrays are kept referenced, so identity means same memory)
        prev = getattr(self, "_dest_arrays", None)
        if prev is None or len(prev) != len(dest) or any(a is not b for a, b in zip(dest, prev)):
            self._dest_arrays = tuple(dest)
            key = tuple(None if a is None else a.ctypes.data for a in (tuple(dest) + (None,) * 4)[:4])
            self._dest = Outputs(*key)
            self._dest_ref = C.byref(self._dest)
        _check(lib().swsgpu_submit_out(self.h, self._sub_ptrs, self._sub_sizes, self._sub_offs,
                                       self._dest_ref), self.h)

    def set_sizes(self, sizes: list[int]) -> None:
        self._sizes = list(sizes)
        self._sub_n = 0

    def wait(self, timeout_ms: int = 60000) -> int:
        if getattr(self, "_wait_ns", None) is None:
            self._wait_ns = C.c_int()
            self._wait_ref = C.byref(self._wait_ns)
        _check(lib().swsgpu_wait(self.h, timeout_ms, self._wait_ref), self.h)
        return self._wait_ns.value

    def fetch_into(self, auto: np.ndarray, xpol: np.ndarray | None = None,
                   pcal: np.ndarray | None = None, tones: np.ndarray | None = None) -> None:
        out = Outputs(auto.ctypes.data, None if xpol is None else xpol.ctypes.data,
                      None if pcal is None else pcal.ctypes.data,
                      None if tones is None else tones.ctypes.data)
        _check(lib().swsgpu_fetch(self.h, C.byref(out)), self.h)

    def run(self, raws: list, payload_offsets=None, timeout_ms: int = 60000):
        """One core run from host bytes (submit + wait + fetch).  Returns
        (auto, xpol, pcal, nspectra); tone phasors (when configured) are left
        in self.tones as complex128 [nspectra][num_sources][pcal_ntones]."""
        n = len(raws)
        arrs = [np.frombuffer(r, dtype=np.uint8) if not isinstance(r, np.ndarray) else r
                for r in raws]
        ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
        sizes = (C.c_size_t * n)(*[a.nbytes for a in arrs])
        offs = (C.c_int64 * n)(*(payload_offsets or [0] * n))
        _check(lib().swsgpu_submit(self.h, ptrs, sizes, offs), self.h)
        ns = C.c_int()
        _check(lib().swsgpu_wait(self.h, timeout_ms, C.byref(ns)), self.h)
        nspec = ns.value
        c = self.cfg
        auto = np.zeros((nspec, c.num_sources, self.S), dtype=np.float32)
        xpol = np.zeros((nspec, max(c.num_xpols, 1), self.S, 2), dtype=np.float32)
        pcal = np.zeros((nspec, c.num_sources, max(c.pcal_tonebins, 1), 2), dtype=np.float32)
        tones = np.zeros((nspec, c.num_sources, max(c.pcal_ntones, 1), 2), dtype=np.float64)
        out = Outputs(auto.ctypes.data, xpol.ctypes.data, pcal.ctypes.data, tones.ctypes.data)
        _check(lib().swsgpu_fetch(self.h, C.byref(out)), self.h)
        self.tones = tones[:, :, : c.pcal_ntones, 0] + 1j * tones[:, :, : c.pcal_ntones, 1]
        xp = xpol[:, : c.num_xpols, :, 0] + 1j * xpol[:, : c.num_xpols, :, 1]
        pc = pcal[:, :, : c.pcal_tonebins, 0] + 1j * pcal[:, :, : c.pcal_tonebins, 1]
        return auto, xp, pc, nspec

    def sync(self, stream: int = 0) -> None:
        """Wait for the stream and raise if a kernel of an earlier call on
        this core gave up a bounded device-side wait (swsgpu_sync)."""
        _check(lib().swsgpu_sync(self.h, C.c_void_p(stream or None)), self.h)

    def inject(self, kind: int) -> None:
        """One-shot host-side fault injection for the next launch (swsgpu_inject)."""
        _check(lib().swsgpu_inject(self.h, kind), self.h)

    def plan_info(self) -> str:
        buf = C.create_string_buffer(256)
        _check(lib().swsgpu_plan_info(self.h, buf, 256), self.h)
        return buf.value.decode()

    def autotune(self, iterations: int = 3) -> str:
        _check(lib().swsgpu_autotune(self.h, iterations), self.h)
        return self.plan_info()

    def workspace_size(self, run_bytes: int, nruns: int) -> int:
        """Device bytes the core allocates for process_device of nruns runs."""
        n = C.c_size_t()
        _check(lib().swsgpu_workspace_size(self.h, run_bytes, nruns, C.byref(n)), self.h)
        return n.value

    def process_device(self, d_raw_ptrs: list[int], run_bytes: int, nruns: int,
                       runs_per_output: int, d_auto: int, d_xpol: int = 0, d_pcal: int = 0,
                       stream: int = 0, d_tones: int = 0) -> None:
        n = len(d_raw_ptrs)
        ptrs = (C.c_void_p * n)(*d_raw_ptrs)
        out = Outputs(d_auto, d_xpol or None, d_pcal or None, d_tones or None)
        _check(lib().swsgpu_process_device(self.h, ptrs, run_bytes, nruns, runs_per_output,
                                           C.byref(out), C.c_void_p(stream or None)), self.h)


class Batch:
    """Many cores' runs recorded as one CUDA graph (swsgpu_batch_*)."""

    def __init__(self, cores: list):
        self.cores = list(cores)
        arr = (C.c_void_p * len(cores))(*[c.h.value for c in cores])
        self.b = C.c_void_p()
        _check(lib().swsgpu_batch_create(arr, len(cores), C.byref(self.b)))

    def set(self, i: int, d_raw_ptrs: list[int], run_bytes: int, nruns: int, runs_per_output: int,
            d_auto: int, d_xpol: int = 0, d_pcal: int = 0, d_tones: int = 0) -> None:
        n = len(d_raw_ptrs)
        ptrs = (C.c_void_p * n)(*d_raw_ptrs)
        out = Outputs(d_auto, d_xpol or None, d_pcal or None, d_tones or None)
        _check(lib().swsgpu_batch_set(self.b, i, ptrs, run_bytes, nruns, runs_per_output, C.byref(out)))

    def launch(self, stream: int = 0) -> int:
        k = C.c_int()
        _check(lib().swsgpu_batch_launch(self.b, C.c_void_p(stream or None), C.byref(k)))
        return k.value

    def close(self) -> None:
        if self.b:
            lib().swsgpu_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def unpack_device(lay: Layout, d_raw: int, nbytes: int, payload_offset: int, chan: int,
                  nsamp: int, d_out: int, stream: int = 0) -> int:
    nv = C.c_int64()
    rc = lib().swsgpu_unpack_device(C.byref(lay), d_raw, nbytes, payload_offset, chan, nsamp,
                                    d_out, C.byref(nv), C.c_void_p(stream or None))
    _check(rc)
    return nv.value


def unpack_device_noalloc(lay: Layout, d_raw: int, nbytes: int, payload_offset: int, chan: int,
                          nsamp: int, d_out: int, stream: int = 0) -> int:
    """swsgpu_unpack_device_noalloc: the same decode with the library's fixed
    scratch array instead of per-call device allocations."""
    nv = C.c_int64()
    rc = lib().swsgpu_unpack_device_noalloc(C.byref(lay), d_raw, nbytes, payload_offset, chan,
                                            nsamp, d_out, C.byref(nv), C.c_void_p(stream or None))
    if rc != 0:
        raise SwsError(f"{ERRORS.get(rc, rc)}: swsgpu_unpack_device_noalloc failed")
    return nv.value


class PcalExtractor:
    """The reference's PCal extractor library on the GPU (swsgpu_pcal_*)."""

    def __init__(self, bandwidth_hz: float, spacing_hz: float, offset_hz: int, sampleoffset: int = 0,
                 kind: int = 0, device: int = 0):
        self.h = C.c_void_p()
        _check(lib().swsgpu_pcal_create(bandwidth_hz, spacing_hz, int(offset_hz), int(sampleoffset), kind,
                                        device, C.byref(self.h)))
        k, nb, nt = C.c_int(), C.c_int(), C.c_int()
        _check(lib().swsgpu_pcal_info(self.h, C.byref(k), C.byref(nb), C.byref(nt)))
        self.kind, self.nbins, self.ntones = k.value, nb.value, nt.value

    def extract(self, d_samples: int, n: int, stream: int = 0) -> None:
        _check(lib().swsgpu_pcal_extract(self.h, d_samples, n, C.c_void_p(stream or None)))

    def adjust(self, sampleoffset: int) -> None:
        _check(lib().swsgpu_pcal_adjust_offset(self.h, int(sampleoffset)))

    def clear(self) -> None:
        _check(lib().swsgpu_pcal_clear(self.h))

    def final(self, stream: int = 0):
        out = np.zeros(2 * self.ntones)
        n = C.c_uint64()
        _check(lib().swsgpu_pcal_final(self.h, out.ctypes.data, C.byref(n), C.c_void_p(stream or None)))
        return out[0::2] + 1j * out[1::2], int(n.value)

    def close(self) -> None:
        if self.h:
            lib().swsgpu_pcal_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pcal_delay(tone_mhz, phase, band_center_mhz: float, band_valid_mhz: float) -> float:
    """swsgpu_pcal_delay: tone-phase delay in ns (m5pcal.c calcDelay)."""
    f = np.ascontiguousarray(tone_mhz, dtype=np.int32)
    ph = np.ascontiguousarray(phase, dtype=np.float64)
    return lib().swsgpu_pcal_delay(len(f), f.ctypes.data, ph.ctypes.data, band_center_mhz, band_valid_mhz)
