"""Benchmark: input Gsamples/s of unpack -> window -> FFT -> integrate.

Workload (dual-polarisation cross-spectra): one Mark5B-2048-16-2 stream,
2 polarisations x 8 subbands of 32 MHz (64 Msps, 2-bit), X/Y correlated
Gaussian noise (rho = 0.3, 0.7 rad), real FFT N = 65536, Hann window, no
overlap, XX / YY / XY* for the 8 pairs integrated over 1 s (976 FFTs) with
the reference's default 32 MiB buffer plan: 4 MiB core runs of 16 FFTs,
61 runs combined per spectrum.  One step = one integration = 1.02e9 input
samples (16 channels x 976 x 65536); inputs are synthetic (seeded) and 256 MB
per step, larger than L2, so consecutive steps re-read HBM.

Lines printed (rank 0, one JSON line):
  value : device-resident input, the C ABI's process_device path, CUDA
          events on the launching stream, max over ranks.
  e2e   : the TaskCore path with host buffers: per 4 MiB run swsgpu_submit
          (H2D inside) + swsgpu_wait, device-side combining of the 61 runs,
          one fetch (D2H) per spectrum.
  roofline of the dominant kernel (FFT + accumulate) from its event-timed
  launches; cpu_baseline from the FP32 CPU restatement on host cores.

--impl reference times the reference's CPU core restatement (FP32, all host
threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 65536
NCHAN = 16
NPAIRS = 8
FS = 64e6
RUN_BYTES = 4 * 1024 * 1024           # default plan's raw buffer (payload bytes)
RUNS_PER_SPECTRUM = 61
CORE_FFTS = 16
FFTS_PER_STEP = RUNS_PER_SPECTRUM * CORE_FFTS          # 976
SAMPLES_PER_STEP = FFTS_PER_STEP * N * NCHAN
CONFIG = {"workload": "dual-pol cross-spectra: Mark5B-2048-16-2, 8 subband pairs, "
                      "N=65536 Hann, XX/YY/XY* over 1 s (976 FFTs), 32 MiB buffer plan",
          "fft_points": N, "channels": NCHAN, "pairs": NPAIRS, "bits": 2, "sample_rate": FS,
          "integration_s": 1.0, "ffts_per_spectrum": FFTS_PER_STEP,
          "run_bytes": RUN_BYTES, "runs_per_spectrum": RUNS_PER_SPECTRUM,
          "l2": "inputs larger than L2 (256 MB per step)"}
METRIC = "input Gsamples/s unpack->FFT->integrate"


def pinned_np(shape, dtype):
    """A zeroed page-locked host array (the GPU core's device-to-host copies
    land in it directly)."""
    import torch
    return torch.zeros(shape, dtype=dtype, pin_memory=True).numpy()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        time.sleep(0.15)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------
def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback"}


def fp32_peak(device: int) -> float | None:
    try:
        L = C.CDLL(os.path.join(ROOT, "libfp32probe.so"))
        v = C.c_double()
        if L.sws_probe_fp32_tflops(device, C.byref(v)) == 0:
            return v.value
    except OSError:
        pass
    return None


def cpu_payload(seed: int = 5):
    """One integration's packed Mark5B payload (61 runs of 4 MiB): random
    2-bit codes; the CPU core's speed does not depend on their values."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, RUNS_PER_SPECTRUM * RUN_BYTES, dtype=np.uint8)


def cpu_step(O, payload, pool, cores: int, npairs: int = NPAIRS) -> int:
    """One step of the workload on the CPU restatement of the reference core
    (TaskCoreIPP::doMaths, src/IA-32/TaskCoreIPP.cpp:355-560): decode the used
    channels from the packed payload (mark5access tables, one channel per
    thread), then for every 4 MiB run and subband pair the FP32 doMaths of 16
    FFTs (windowed real-input FFT, |X|^2 and X.Y* accumulation).  As the
    reference's NumCPUCores cores do, each thread takes whole core runs.
    Returns the input samples processed."""
    nsamp = RUNS_PER_SPECTRUM * RUN_BYTES // 4          # 16 ch x 2 bit = 4 bytes per sample-time
    chans = [c for p in range(npairs) for c in (p, p + NPAIRS)]
    dec = dict(zip(chans, pool.map(lambda c: O.decode(O.FMT_MARK5B, NCHAN, 2, payload, nsamp, c), chans)))
    cfg = O.make_cfg(N, core_overlapped_ffts=CORE_FFTS, num_sources=2, num_xpols=1,
                     window=O.W_HANN, nthreads=1)
    per_run = CORE_FFTS * N

    def core_run(task):
        r, p = task
        O.domaths(cfg, [dec[p][r * per_run:(r + 1) * per_run], dec[p + NPAIRS][r * per_run:(r + 1) * per_run]],
                  fp64=False)

    list(pool.map(core_run, [(r, p) for r in range(RUNS_PER_SPECTRUM) for p in range(npairs)]))
    return len(chans) * RUNS_PER_SPECTRUM * per_run


def cpu_baseline(seconds_budget: float = 12.0) -> dict:
    """The CPU restatement on all host cores over whole steps of the
    workload (packed payload in, spectra out) until the budget is spent."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    payload = cpu_payload()
    samples = 0
    steps = 0
    with ThreadPoolExecutor(max_workers=cores) as pool:
        t0 = time.perf_counter()
        while True:
            samples += cpu_step(O, payload, pool, cores)
            steps += 1
            if time.perf_counter() - t0 > seconds_budget:
                break
        dt = time.perf_counter() - t0
    return {"value": samples / dt / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": "port",
            "sample": f"{steps} whole step(s) of the workload (1 s integration, 16 channels, "
                      f"{samples / 1e6:.0f} Msamples) from packed Mark5B bytes: mark5access decode + "
                      "FP32 restatement of TaskCoreIPP::doMaths (real-input FFT), one core run per thread",
            "seconds": dt}


def reference_arm(args) -> None:
    """The reference's CPU core, restated (its IPP build cannot be compiled:
    Intel IPP is closed and absent), on all host cores: every step is one
    whole step of the workload, timed as it runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    payload = cpu_payload()
    times = []
    with ThreadPoolExecutor(max_workers=cores) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            n = cpu_step(O, payload, pool, cores)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    v = n / (ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": v, "unit": "Gsamples/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": CONFIG,
            "cpu_baseline": {"value": v, "unit": "Gsamples/s", "cores": cores, "kind": "port",
                             "sample": "every step is one whole step of the workload (1 s integration, "
                                       "16 channels) from packed Mark5B bytes: mark5access decode + FP32 C "
                                       "restatement of TaskCoreIPP::doMaths (real-input FFT), all host threads"},
            "e2e": {"value": v, "unit": "Gsamples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def parity_check(gpu, synth, O, raw_host: bytes, precision: int) -> dict:
    """Max relative errors of one full integration (976 FFTs) of pair 0 vs
    the FP64 oracle, through the TaskCore path (61 submits)."""
    import numpy as np
    lay = gpu.layout("mark5b", NCHAN, 2, framed=False)
    cfg = gpu.make_config(lay, N, "hann", 1, CORE_FFTS, sources=((0, 0), (0, NPAIRS)),
                          xpols=((0, 1),), precision=precision, max_run_bytes=RUN_BYTES,
                          samplingfreq=FS, runs_per_output=RUNS_PER_SPECTRUM)
    core = gpu.Core(cfg)
    core.set_sizes([RUN_BYTES])
    pay = np.frombuffer(raw_host, dtype=np.uint8)
    for r in range(RUNS_PER_SPECTRUM):
        core.submit([pay[r * RUN_BYTES:(r + 1) * RUN_BYTES]], payload_offsets=[r * RUN_BYTES])
        ns = core.wait()
    S = N // 2 + 1
    auto = np.zeros((1, 2, S), np.float32)
    xp = np.zeros((1, 1, S, 2), np.float32)
    core.fetch_into(auto, xp)
    core.close()
    nsamp = RUNS_PER_SPECTRUM * RUN_BYTES // 4
    s = [O.decode(O.FMT_MARK5B, NCHAN, 2, raw_host, nsamp, c) for c in (0, NPAIRS)]
    ra = np.zeros((2, S))
    rx = np.zeros(S, complex)
    for r in range(RUNS_PER_SPECTRUM):
        cfgo = O.make_cfg(N, core_overlapped_ffts=CORE_FFTS, num_sources=2, num_xpols=1,
                          window=O.W_HANN)
        a, x, _, n = O.domaths(cfgo, [v[r * CORE_FFTS * N:(r + 1) * CORE_FFTS * N] for v in s])
        ra += a[0]
        rx += x[0, 0]
    xc = xp[0, 0, :, 0] + 1j * xp[0, 0, :, 1]
    e_auto = float(np.max(np.abs(auto[0] - ra) / ra))
    e_xpol = float(np.max(np.abs(xc - rx) / np.sqrt(ra[0] * ra[1])))
    e_rms = float(np.sqrt(np.mean(((auto[0] - ra) / ra) ** 2)))
    return {"max_rel_err_auto": e_auto, "max_rel_err_xpol": e_xpol, "rms_rel_err_auto": e_rms,
            "bar": 2e-6, "pair": "subband 0 (channels 1 and 9), one full 1 s integration",
            "spectra_checked": int(ns)}


def gpu_arm(args) -> None:
    import numpy as np
    import torch

    from swspec_b200 import gpu, synth, synth_gpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from swspec_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    world, rank = reps.world, reps.rank

    names = {gpu.PREC_FP32: "fp32", gpu.PREC_TCSPLIT: "tcsplit", gpu.PREC_TCSPLIT_ALL: "tcsplit_all"}
    precisions = [gpu.PREC_FP32]
    if args.plan != "fourstep" and tc_available(gpu):
        if args.precision == "auto":
            precisions = [gpu.PREC_TCSPLIT_ALL, gpu.PREC_TCSPLIT, gpu.PREC_FP32]
        elif args.precision != "fp32":
            precisions = [{"tcsplit": gpu.PREC_TCSPLIT, "tcsplit_all": gpu.PREC_TCSPLIT_ALL}[args.precision],
                          gpu.PREC_FP32]
    headline = precisions[0]

    # ---- input: one integration of framed Mark5B on the device ----
    payload_needed = RUNS_PER_SPECTRUM * RUN_BYTES
    d_raw, nfr = synth_gpu.c3_framed(payload_needed // 4 + 2500, N=N, npairs=NPAIRS,
                                     seed=1003 + rank)
    torch.cuda.synchronize()
    S = N // 2 + 1
    d_auto = torch.zeros(NCHAN, S, dtype=torch.float32, device="cuda")
    d_xpol = torch.zeros(NPAIRS, S, 2, dtype=torch.float32, device="cuda")
    # a dedicated stream: its handle is what the library launches on and
    # what the timing events are recorded on
    stream = torch.cuda.Stream()
    lay = gpu.layout("mark5b", NCHAN, 2)
    sources = tuple((0, c) for c in range(NCHAN))
    pairs = tuple((c, c + NPAIRS) for c in range(NPAIRS))

    family = {"auto": gpu.PLAN_DEFAULT, "cluster": gpu.PLAN_CLUSTER, "fourstep": gpu.PLAN_FOURSTEP}[args.plan]

    def make_core(prec, framed=True, rpo=1):
        cfg = gpu.make_config(lay if framed else gpu.layout("mark5b", NCHAN, 2, framed=False), N,
                              "hann", 1, CORE_FFTS, sources=sources, xpols=pairs, precision=prec,
                              max_run_bytes=RUN_BYTES, samplingfreq=FS, runs_per_output=rpo,
                              plan_family=family, autotune=family == gpu.PLAN_FOURSTEP)
        return gpu.Core(cfg, device=local)

    # a second core on its own stream with its own outputs: consecutive
    # integrations alternate between the two, so one integration's unpack
    # and reduction run beside the other's FFT grid (the SMs no 16-CTA
    # cluster fits on), as the reference's dispatcher runs NumCPUCores cores
    stream2 = torch.cuda.Stream()
    d_auto2 = torch.zeros_like(d_auto)
    d_xpol2 = torch.zeros_like(d_xpol)

    def step(core, second=False):
        st, a, x = (stream2, d_auto2, d_xpol2) if second else (stream, d_auto, d_xpol)
        core.process_device([d_raw.data_ptr()], RUN_BYTES, RUNS_PER_SPECTRUM, RUNS_PER_SPECTRUM,
                            a.data_ptr(), x.data_ptr(), 0, st.cuda_stream)

    barrier = reps.barrier
    max_over_ranks = reps.max

    forms = {}
    launches_per_step = 0
    clocks = None
    for prec in precisions:
        name = names[prec]
        core = make_core(prec)
        core2 = make_core(prec)
        plan_desc = core.plan_info()
        for i in range(args.warmup):
            step(core)
            step(core2, True)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev2 = torch.cuda.Event(enable_timing=True)
        evb = torch.cuda.Event()
        with ClockSampler(local) as cs:
            # one core: every integration after the previous one
            ev0.record(stream)
            for _ in range(args.steps):
                step(core)
            ev1.record(stream)
            # two cores on two streams, integrations alternating
            stream2.wait_event(ev1)
            for i in range(args.steps):
                step(core2 if i % 2 else core, bool(i % 2))
            evb.record(stream2)
            stream.wait_event(evb)
            ev2.record(stream)
            stream.synchronize()
            torch.cuda.synchronize()
        barrier()
        ms1 = max_over_ranks(ev0.elapsed_time(ev1))
        ms = max_over_ranks(ev1.elapsed_time(ev2))
        launches_per_step = core.last_launches()
        # dominant kernel timing (separate pass, events around each launch)
        core.profile(True)
        for _ in range(max(2, min(args.steps, 5))):
            step(core)
        nk, kms = core.profile_read()
        core.profile(False)
        core.sync(stream.cuda_stream)   # raises if a bounded device wait of any step gave up
        core2.sync(stream2.cuda_stream)
        core.close()
        core2.close()
        value = SAMPLES_PER_STEP * args.steps * world / (ms * 1e-3) / 1e9
        value1 = SAMPLES_PER_STEP * args.steps * world / (ms1 * 1e-3) / 1e9
        forms[name] = {"value": value, "ms_per_step": ms / args.steps, "plan": plan_desc,
                       "one_core": {"value": value1, "ms_per_step": ms1 / args.steps},
                       "kernel_ms_per_launch": kms / max(nk, 1), "kernel_launches": nk,
                       "launches_per_step": launches_per_step, "clocks": cs.summary()}
        if prec == headline:
            clocks = cs.summary()
        log(f"[{name}] {value:.3f} Gsamples/s two cores ({value1:.3f} one core), {ms / args.steps:.3f} ms/step, "
            f"FFT kernel {kms / max(nk, 1):.3f} ms/launch")

    # the headline is the fastest form (every form meets the parity bar; all are reported)
    headline = max(precisions, key=lambda p: forms[names[p]]["value"])
    clocks = forms[names[headline]]["clocks"]

    # ---- e2e: TaskCore path, host buffers, per-run submit/wait ----
    pay_dev = d_raw.view(nfr, 10016)[:, 16:].reshape(-1)[:payload_needed]
    host = torch.empty(payload_needed, dtype=torch.uint8, pin_memory=True)
    host.copy_(pay_dev)
    torch.cuda.synchronize()
    core = make_core(headline, framed=False, rpo=RUNS_PER_SPECTRUM)
    core.set_sizes([RUN_BYTES])
    # output buffers handed to the run, as TaskCore::run takes them, page-locked
    auto_h = pinned_np((1, NCHAN, S), torch.float32)
    xpol_h = pinned_np((1, NPAIRS, S, 2), torch.float32)
    base = host.data_ptr()

    def e2e_step():
        for r in range(RUNS_PER_SPECTRUM):
            core.submit([base + r * RUN_BYTES], payload_offsets=[r * RUN_BYTES], dest=(auto_h, xpol_h))
            core.wait()

    # K cores, one integration each, their runs interleaved: each core's
    # next run is submitted as soon as its previous run's input has landed,
    # so the other cores' copies are already queued behind it
    K = max(2, args.e2e_cores)
    extra = [make_core(headline, framed=False, rpo=RUNS_PER_SPECTRUM) for _ in range(K - 1)]
    for c in extra:
        c.set_sizes([RUN_BYTES])
    group = [(core, (auto_h, xpol_h))] + [(c, (pinned_np((1, NCHAN, S), torch.float32),
                                              pinned_np((1, NPAIRS, S, 2), torch.float32))) for c in extra]

    def e2e_group():
        for c, d in group:
            c.submit([base], payload_offsets=[0], dest=d)
        for r in range(1, RUNS_PER_SPECTRUM + 1):
            for c, d in group:
                c.wait()
                if r < RUNS_PER_SPECTRUM:
                    c.submit([base + r * RUN_BYTES], payload_offsets=[r * RUN_BYTES], dest=d)

    for _ in range(max(1, args.warmup)):
        e2e_step()
        e2e_group()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e1_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    ngroup = (args.steps + K - 1) // K
    t0 = time.perf_counter()
    for _ in range(ngroup):
        e2e_group()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    core.close()
    for c in extra:
        c.close()
    e2e1_val = SAMPLES_PER_STEP * args.steps * world / e2e1_s / 1e9
    e2e_val = SAMPLES_PER_STEP * K * ngroup * world / e2e_s / 1e9
    # the cores' spectra of the same input (expected: bit for bit)
    cores_agree = all(np.array_equal(auto_h, d[0]) and np.array_equal(xpol_h, d[1]) for _, d in group[1:])
    d2h = auto_h.nbytes + xpol_h.nbytes
    log(f"[e2e] {e2e_val:.3f} Gsamples/s {K} cores ({e2e1_val:.3f} one core)")

    # ---- parity of the headline form on this workload ----
    parity = None
    if rank == 0 and not args.no_parity:
        import oracle as O
        parity = parity_check(gpu, synth, O, host.numpy().tobytes(), headline)
        log(f"[parity] {parity}")

    if rank != 0:
        reps.close()
        return

    hl = forms[names[headline]]
    peaks = measured_peaks()
    # the roofline of the dominant kernel (k_spectra: FFT + accumulate) is the
    # slower of the packed-input-plus-spectra bytes at HBM bandwidth and the
    # 5 N log2 N flops per channel FFT at the form's arithmetic peak
    flops_per_launch = 5.0 * N * math.log2(N) * NCHAN * FFTS_PER_STEP
    bytes_per_launch = (SAMPLES_PER_STEP * 2 / 8            # packed 2-bit input
                        + (NCHAN + 2 * NPAIRS) * 4 * (N // 2 + 1))  # spectra written
    kern_s = hl["kernel_ms_per_launch"] * 1e-3
    p32 = fp32_peak(local)
    achieved_tf = flops_per_launch / kern_s / 1e12
    hbm = {"achieved_gbs": bytes_per_launch / kern_s / 1e9, "peak_gbs": peaks["hbm_gbs"],
           "frac": bytes_per_launch / kern_s / 1e9 / peaks["hbm_gbs"],
           "t_min_ms": bytes_per_launch / (peaks["hbm_gbs"] * 1e9) * 1e3,
           "peak_source": f"HBM copy, {peaks['source']}"}
    if headline == gpu.PREC_FP32:
        roof = {"bound": "fp32", "achieved": achieved_tf, "peak": p32, "unit": "TFLOP/s",
                "frac": achieved_tf / p32 if p32 else None,
                "t_min_ms": flops_per_launch / (p32 * 1e12) * 1e3 if p32 else None,
                "peak_source": "FP32 FMA issue, measured on this GPU by fp32_probe.cu "
                               "(MEASURED_PEAKS.json holds no FP32 figure)"}
    else:
        tp = peaks["bf16_tflops"]
        levels = 3 if headline == gpu.PREC_TCSPLIT_ALL else 2
        # tcgen05.mma work actually issued: per pair FFT, 16 CTAs x levels x
        # 2 tiles x 4 K-steps of M=128, N=64, K=16
        mma_flops = FFTS_PER_STEP * NPAIRS * 16 * levels * 8 * 2.0 * 128 * 64 * 16
        roof = {"bound": "tensor", "achieved": achieved_tf, "peak": tp, "unit": "TFLOP/s",
                "frac": achieved_tf / tp, "t_min_ms": flops_per_launch / (tp * 1e12) * 1e3,
                "peak_source": f"dense bf16/f16 tensor burst, {peaks['source']}",
                "mma_issued": {"tflops": mma_flops / kern_s / 1e12, "frac": mma_flops / kern_s / 1e12 / tp,
                               "flops_per_launch": mma_flops,
                               "note": "split-precision GEMM work issued (hi/lo operands, K = 64)"}}
    roof["hbm"] = hbm
    # DRAM bytes of one k_spectra launch on this workload, from ncu captures
    # (dram__bytes_read.sum + dram__bytes_write.sum): the 2-bit codes read
    # plus the per-item partial spectra that k_reduce combines
    traffic = {gpu.PREC_FP32: (257874176 + 215790080,
                               "ncu section capture of one k_spectra launch of this workload "
                               "(dram__bytes_read.sum + dram__bytes_write.sum)")}
    t = traffic.get(headline)
    roof["traffic"] = t[0] if t else None
    roof["traffic_source"] = t[1] if t else None
    roof["kernel"] = "k_spectra (cluster FFT + accumulate), " + names[headline] + " form"
    roof["flops_per_launch"] = flops_per_launch
    roof["algorithmic_bytes_per_launch"] = bytes_per_launch
    roof["fp32_peak_tflops"] = p32
    cpu = cpu_baseline() if (world == 1 and not args.no_cpu) else None
    line = {"metric": METRIC, "value": hl["value"], "unit": "Gsamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": hl["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if headline == gpu.PREC_FP32 else "f16x2-split/f32",
            "data": "synthetic", "config": CONFIG,
            "precision": names[headline],
            "cores": "value: two cores on two streams, consecutive integrations alternating; "
                     "forms[*].one_core: one core on one stream",
            "forms": forms, "clocks": clocks,
            "tc_over_fp32": {n: forms[n]["value"] / forms["fp32"]["value"] for n in forms if n != "fp32"} or None,
            "e2e": {"value": e2e_val, "unit": "Gsamples/s",
                    "h2d_bytes_per_step": RUNS_PER_SPECTRUM * RUN_BYTES,
                    "d2h_bytes_per_step": d2h,
                    "path": "swsgpu_submit_out/wait per 4 MiB run (TaskCore path, the run given its "
                            "output buffers), device combine, spectra copied into pinned host arrays; "
                            f"{K} cores with one integration each, runs interleaved",
                    "cores": K, "one_core": e2e1_val, "cores_agree": cores_agree},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": roof, "cpu_baseline": cpu, "parity": parity}
    print(json.dumps(line), flush=True)
    reps.close()


def tc_available(gpu) -> bool:
    try:
        cfg = gpu.make_config(gpu.layout("mark5b", NCHAN, 2), N, precision=gpu.PREC_TCSPLIT,
                              max_run_bytes=1 << 20)
        c = gpu.Core(cfg)
        c.close()
        return True
    except gpu.SwsError:
        return False


def c4_cpu_baseline(specs, seconds_per_length: float = 3.0) -> dict:
    """The CPU restatement of the reference core (mark5access VDIF decode +
    FP32 TaskCoreIPP::doMaths) on all host cores, per FFT length and bit
    depth of the mix over a bounded sample of whole FFTs, combined as the
    time the step's samples of each length would take at its rate."""
    from collections import Counter
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    share = Counter()
    for s in specs:
        share[(s.fft_points, s.nbit)] += s.samples_per_run
    rng = np.random.default_rng(7)
    rates, nfft = {}, 0
    t_all = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as pool:
        for N, nbit in sorted(share):
            seg = rng.integers(0, 256, N * nbit // 8, dtype=np.uint8).tobytes()
            cfg = O.make_cfg(N, core_overlapped_ffts=1, num_sources=1, window=O.W_HANN, nthreads=1)

            def job(_):
                x = O.decode(O.FMT_VDIF, 1, nbit, seg, N, 0, payload_bytes=8000)
                O.domaths(cfg, [x], fp64=False)
                return N

            samples = 0
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < seconds_per_length:
                samples += sum(pool.map(job, range(cores)))
                nfft += cores
            rates[(N, nbit)] = samples / (time.perf_counter() - t0)
    t_step = sum(share[k] / rates[k] for k in share)
    return {"value": sum(share.values()) / t_step / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": "port",
            "sample": f"{nfft} whole FFTs over the mix's {len(share)} (length, bits) classes, about "
                      f"{seconds_per_length:.0f} s each on all threads (mark5access VDIF decode + FP32 "
                      "restatement of TaskCoreIPP::doMaths); the step's samples of each class at that "
                      "class's rate",
            "seconds": time.perf_counter() - t_all}


def c4_arm(args) -> None:
    """Batched uneven streams: 64 single-channel streams of mixed FFT length
    (4096 .. 3.2M), bit depth, bandwidth and integration, one core run each
    per step, all recorded in one CUDA graph and issued with one launch."""
    import torch

    from swspec_b200 import gpu
    from swspec_b200.replicas import Replicas
    from swspec_b200.workloads import c4_streams
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    specs = c4_streams(64, seed=2000)
    cores, raws, outs = [], [], []
    g = torch.Generator(device="cuda")
    g.manual_seed(2000 + reps.rank)
    t_tune = time.perf_counter()
    for s in specs:
        lay = gpu.layout("vdif:8000", 1, s.nbit, framed=False)
        cfg = gpu.make_config(lay, s.fft_points, "hann", 1, s.core_overlapped_ffts, max_run_bytes=s.run_bytes,
                              samplingfreq=s.samplingfreq, autotune=True)
        c = gpu.Core(cfg, device=local)
        cores.append(c)
        raws.append(torch.randint(0, 256, (s.run_bytes,), dtype=torch.uint8, device="cuda", generator=g))
        ns, _, _ = c.run_shape(s.run_bytes)
        outs.append(torch.zeros(max(ns, 1), 1, c.S, dtype=torch.float32, device="cuda"))
    t_tune = time.perf_counter() - t_tune
    b = gpu.Batch(cores)
    for i, (s, r, o) in enumerate(zip(specs, raws, outs)):
        b.set(i, [r.data_ptr()], s.run_bytes, 1, 1, o.data_ptr())
    st = torch.cuda.Stream()
    kernels = b.launch(st.cuda_stream)   # eager pass + graph recording
    for _ in range(args.warmup):
        b.launch(st.cuda_stream)
    torch.cuda.synchronize()
    reps.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as cs:
        ev0.record(st)
        for _ in range(args.steps):
            b.launch(st.cuda_stream)
        ev1.record(st)
        st.synchronize()
    reps.barrier()
    ms = reps.max(ev0.elapsed_time(ev1)) / args.steps
    samples = sum(s.samples_per_run for s in specs)
    bytes_in = sum(s.run_bytes for s in specs)
    value = samples * reps.world / (ms * 1e-3) / 1e9
    b.close()

    # ---- e2e: every stream's run from pinned host memory through its own
    # core's submit / wait / fetch (the TaskCore path), all cores in flight
    # as the reference's dispatcher runs its cores, then joins each ----
    import numpy as np
    hosts, houts = [], []
    for s, c, r in zip(specs, cores, raws):
        h = torch.empty(s.run_bytes, dtype=torch.uint8, pin_memory=True)
        h.copy_(r)
        hosts.append(h)
        ns, _, _ = c.run_shape(s.run_bytes)
        houts.append(pinned_np((max(ns, 1), 1, c.S), torch.float32))
        c.set_sizes([s.run_bytes])
    torch.cuda.synchronize()

    def e2e_step():
        for c, h, o in zip(cores, hosts, houts):
            c.submit([h.data_ptr()], dest=(o,))
        for c in cores:
            c.wait()

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    reps.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = reps.max(time.perf_counter() - t0)
    reps.barrier()
    e2e_val = samples * args.steps * reps.world / e2e_s / 1e9
    d2h = sum(o.nbytes for o in houts)
    log(f"[c4 e2e] {e2e_val:.3f} Gsamples/s")
    if reps.rank == 0:
        from collections import Counter
        peaks = measured_peaks()
        achieved = bytes_in / (ms * 1e-3) / 1e9
        line = {"metric": METRIC, "value": value, "unit": "Gsamples/s", "n_gpus": reps.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched uneven streams: 64 single-channel VDIF streams, one core run "
                                       "each per step, one CUDA graph launch per step",
                           "lengths": dict(Counter(s.fft_points for s in specs)),
                           "bits": dict(Counter(s.nbit for s in specs)),
                           "samples_per_step": samples, "bytes_per_step": bytes_in,
                           "l2": "inputs larger than L2 (%.0f MB per step)" % (bytes_in / 1e6),
                           "autotune_s": t_tune},
                "clocks": cs.summary(), "gpu_launches": kernels * args.steps, "graph_launches_per_step": 1,
                "e2e": {"value": e2e_val, "unit": "Gsamples/s", "h2d_bytes_per_step": bytes_in,
                        "d2h_bytes_per_step": d2h,
                        "path": "swsgpu_submit_out/wait per stream from pinned host buffers into pinned output "
                                "arrays, all 64 cores submitted before the waits (one outstanding run per core)"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                             "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                             "note": "packed input bytes per step over the step time"},
                "cpu_baseline": c4_cpu_baseline(specs) if (reps.world == 1 and not args.no_cpu) else None}
        print(json.dumps(line), flush=True)
    reps.close()


# one integration per step, device-resident header-free payload, the
# reference's buffer plan (runs of core_ffts FFTs combined on the device)
SPEC_WORKLOADS = {
    "c1": dict(desc="plain method: Mark5B-1024-16-2, channel 1 only, N=32768 Hann, 1 s (976 FFTs), "
                    "2 MiB runs x 61", fmt="mark5b", nchan=16, nbit=2, N=32768, window="hann", fs=32e6,
               core_ffts=16, run_bytes=2 << 20, runs=61, sources=((0, 0),), xpols=(), pcal=None,
               signal="Gaussian noise, CW tone at +3.1 MHz in channel 1 at 20 dB per FFT bin, +-0.98 sigma 2-bit"),
    "c2": dict(desc="spacecraft-tone tracking: Mark5B-1024-16-2, 16 channels, N=3,200,000 cosine2, 10 s "
                    "(100 FFTs), 51.2 MB runs x 25, phase-cal 32 bins / 3200 rotator, 16 tones",
               fmt="mark5b", nchan=16, nbit=2, N=3_200_000, window="cosine2", fs=32e6, core_ffts=4,
               run_bytes=51_200_000, runs=25, sources=tuple((0, c) for c in range(16)), xpols=(),
               pcal=dict(tonebins=32, rotatorlen=3200, offset=10e3, ntones=16),
               signal="Gaussian noise plus a phase-cal comb (1 MHz spacing, +10 kHz, 5 % of sigma, seeded "
                      "phases) in every channel, +-0.98 sigma 2-bit"),
    "c5": dict(desc="dynamic range: VDIF 8-bit 1 channel 64 Msps, N=2^22 Blackman-Harris, 5 s (76 FFTs), "
                    "16 MiB runs x 19", fmt="vdif:8000", nchan=1, nbit=8, N=1 << 22, window="blackmanharris",
               fs=64e6, core_ffts=4, run_bytes=16 << 20, runs=19, sources=((0, 0),), xpols=(), pcal=None,
               signal="Gaussian noise plus a carrier at 12.3456 MHz 50 dB over the per-bin floor drifting "
                      "1 Hz/s, 8-bit offset binary at 24 codes per sigma"),
    "vlba": dict(desc="VLBA track format: VLBA1_2-512-8-2 (32 tracks, fanout 2, 8 channels 2-bit, 32 Msps), "
                      "header-free payload, N=65536 Hann, 1.016 s (992 FFTs), 4 MiB runs x 31",
                 fmt="vlba:32", m5fmt="VLBA1_2-512-8-2", nchan=8, nbit=2, N=65536, window="hann", fs=32e6,
                 core_ffts=32, run_bytes=4 << 20, runs=31, sources=tuple((0, c) for c in range(8)), xpols=(),
                 pcal=None, signal="uniform random track-words (every sample code equally likely)"),
}


def spec_payload(name: str, w: dict, seed: int):
    """The workload's whole step of header-free payload on the device."""
    import numpy as np

    from swspec_b200 import synth_gpu
    T = w["run_bytes"] * w["runs"] * 8 // (w["nbit"] * w["nchan"])
    if name == "vlba":
        import torch
        g = torch.Generator(device="cuda")
        g.manual_seed(1006 + seed)
        return torch.randint(0, 256, (w["run_bytes"] * w["runs"],), dtype=torch.uint8, device="cuda", generator=g)
    if name == "c1":
        # Hann: 20 dB per-bin SNR <=> A^2 N / (6 sigma^2) = 100
        return synth_gpu.mark5b_payload(T, 16, w["fs"], 1001 + seed, tone_hz=3.1e6,
                                        tone_amp=float(np.sqrt(6 * 100.0 / w["N"])))
    if name == "c2":
        phases = np.random.default_rng(1002 + seed).uniform(0, 2 * np.pi, 16)
        return synth_gpu.mark5b_payload(T, 16, w["fs"], 1002 + seed, comb=(1e6, 10e3, 0.05, phases))
    # 4-term Blackman-Harris (equivalent noise bandwidth about 2 bins): 50 dB
    # over the per-bin floor <=> A = sigma sqrt(4e5 * 2 / N); sigma = 24 codes
    return synth_gpu.vdif8_carrier_payload(T, w["fs"], 1005 + seed, 12.3456e6, 1.0, 50.0, w["N"], lsb_sigma=48.0)


def spec_cpu_baseline(w: dict, payload, seconds_budget: float = 12.0) -> dict:
    """The CPU restatement of the reference core (FP32 TaskCoreIPP::doMaths
    after the mark5access decode of the packed bytes) on all host cores over
    a bounded sample of the workload: each thread takes whole FFTs of one
    source, as many as the budget allows."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    N, ns = w["N"], len(w["sources"])
    nbit, nchan = w["nbit"], w["nchan"]
    if "m5fmt" in w:
        return track_cpu_baseline(w, payload, seconds_budget)
    fmt = O.FMT_MARK5B if w["fmt"] == "mark5b" else O.FMT_VDIF
    bpt = nbit * nchan // 8                          # payload bytes per sample-time
    nfft_avail = len(payload) // (N * bpt)
    cfg = O.make_cfg(N, core_overlapped_ffts=1, num_sources=1, window=O.WINDOW_NAMES[w["window"]], nthreads=1)
    kw = {"payload_bytes": 8000} if fmt == O.FMT_VDIF else {}

    def job(k):
        f, src = k % nfft_avail, w["sources"][(k // nfft_avail) % ns][1]
        seg = payload[f * N * bpt:(f + 1) * N * bpt].tobytes()
        x = O.decode(fmt, nchan, nbit, seg, N, src, **kw)
        O.domaths(cfg, [x], fp64=False)
        return N

    samples, k = 0, 0
    with ThreadPoolExecutor(max_workers=cores) as pool:
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < seconds_budget:
            samples += sum(pool.map(job, range(k, k + cores)))
            k += cores
        dt = time.perf_counter() - t0
    return {"value": samples / dt / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": "port",
            "sample": f"{k} FFTs of N = {N} from the workload's packed bytes (mark5access decode + FP32 "
                      "restatement of TaskCoreIPP::doMaths), one FFT per thread at a time",
            "seconds": dt}


def track_cpu_baseline(w: dict, payload, seconds_budget: float = 12.0) -> dict:
    """VLBA / Mark4 on the CPU: mark5access's own unpack (built from the
    reference sources) of N sample-times of every channel from a frame
    boundary, then the FP32 restatement of TaskCoreIPP::doMaths on each
    channel, on all host cores over a bounded sample."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    N, nchan, nbit = w["N"], w["nchan"], w["nbit"]
    ntrack = int(w["fmt"].split(":")[1])
    frame = 2500 * ntrack
    need = N * nchan * nbit // 8
    nseg = (len(payload) - need) // frame
    cfg = O.make_cfg(N, core_overlapped_ffts=1, num_sources=1, window=O.WINDOW_NAMES[w["window"]], nthreads=1)

    def job(k):
        seg = payload[(k % nseg) * frame:(k % nseg) * frame + need].tobytes()
        dec, _ = O.m5_unpack(w["m5fmt"], seg, N)
        for c in range(nchan):
            O.domaths(cfg, [dec[c]], fp64=False)
        return N * nchan

    samples, k = 0, 0
    with ThreadPoolExecutor(max_workers=cores) as pool:
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < seconds_budget:
            samples += sum(pool.map(job, range(k, k + cores)))
            k += cores
        dt = time.perf_counter() - t0
    return {"value": samples / dt / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": "reference",
            "sample": f"{k} blocks of N = {N} sample-times x {nchan} channels: mark5access's header-free "
                      "unpack (the reference's own decoder library) + the FP32 restatement of "
                      "TaskCoreIPP::doMaths per channel",
            "seconds": dt}


def spec_arm(args) -> None:
    import torch

    from swspec_b200 import gpu
    from swspec_b200.replicas import Replicas
    w = SPEC_WORKLOADS[args.workload]
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    lay = gpu.layout(w["fmt"], w["nchan"], w["nbit"], framed=False)
    pc = w["pcal"] or {}
    prec = {"auto": gpu.PREC_FP32, "fp32": gpu.PREC_FP32, "tcsplit": gpu.PREC_TCSPLIT,
            "tcsplit_all": gpu.PREC_TCSPLIT}[args.precision]
    cfg = gpu.make_config(lay, w["N"], w["window"], 1, w["core_ffts"], sources=w["sources"], xpols=w["xpols"],
                          precision=prec,
                          max_run_bytes=w["run_bytes"], samplingfreq=w["fs"], runs_per_output=w["runs"],
                          extract_pcal=bool(pc), pcal_tonebins=pc.get("tonebins", 0),
                          pcal_rotatorlen=pc.get("rotatorlen", 0), pcal_offset_hz=pc.get("offset", 10e3),
                          pcal_ntones=pc.get("ntones", 0), autotune=args.candidate < 0,
                          plan_family=gpu.PLAN_FOURSTEP if args.candidate >= 0 else gpu.PLAN_DEFAULT,
                          plan_candidate=max(args.candidate, 0))
    core = gpu.Core(cfg, device=local)
    raw = spec_payload(args.workload, w, reps.rank)
    assert raw.numel() == w["run_bytes"] * w["runs"]
    torch.cuda.synchronize()
    S = w["N"] // 2 + 1
    ns = len(w["sources"])
    d_auto = torch.zeros(ns, S, dtype=torch.float32, device="cuda")
    d_pcal = torch.zeros(ns, max(pc.get("tonebins", 1), 1), 2, dtype=torch.float32, device="cuda")
    d_tones = torch.zeros(ns, max(pc.get("ntones", 1), 1), 2, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()

    def step():
        core.process_device([raw.data_ptr()], w["run_bytes"], w["runs"], w["runs"], d_auto.data_ptr(), 0,
                            d_pcal.data_ptr() if pc else 0, st.cuda_stream, d_tones.data_ptr() if pc else 0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    reps.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as cs:
        ev0.record(st)
        for _ in range(args.steps):
            step()
        ev1.record(st)
        st.synchronize()
    reps.barrier()
    ms = reps.max(ev0.elapsed_time(ev1)) / args.steps
    launches = core.last_launches()
    core.profile(True)
    for _ in range(3):
        step()
    nk, kms = core.profile_read()
    core.profile(False)
    core.sync(st.cuda_stream)   # raises if a bounded device wait of any step gave up
    samples = w["runs"] * w["core_ffts"] * w["N"] * ns
    value = samples * reps.world / (ms * 1e-3) / 1e9

    # ---- e2e: TaskCore path from pinned host memory, one submit per run ----
    import numpy as np
    host = torch.empty(raw.numel(), dtype=torch.uint8, pin_memory=True)
    host.copy_(raw)
    torch.cuda.synchronize()
    ecore = gpu.Core(cfg, device=local)
    ecore.set_sizes([w["run_bytes"]])
    # output buffers handed to the run (TaskCore::run's out / pcal), page-locked
    auto_h = pinned_np((1, ns, S), torch.float32)
    pcal_h = pinned_np((1, ns, max(pc.get("tonebins", 1), 1), 2), torch.float32) if pc else None
    tones_h = pinned_np((1, ns, max(pc.get("ntones", 1), 1), 2), torch.float64) if pc else None
    base = host.data_ptr()

    def e2e_step():
        for r in range(w["runs"]):
            ecore.submit([base + r * w["run_bytes"]], payload_offsets=[r * w["run_bytes"]],
                         dest=(auto_h, None, pcal_h, tones_h))
            ecore.wait()

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    reps.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = reps.max(time.perf_counter() - t0)
    ecore.close()
    e2e_val = samples * args.steps * reps.world / e2e_s / 1e9
    d2h = auto_h.nbytes + (pcal_h.nbytes + tones_h.nbytes if pc else 0)
    cpu = None
    if reps.rank == 0 and reps.world == 1 and not args.no_cpu:
        cpu = spec_cpu_baseline(w, host.numpy())
    if reps.rank == 0:
        peaks = measured_peaks()
        kern_s = kms / max(nk, 1) * 1e-3
        bytes_in = w["run_bytes"] * w["runs"]
        flops = 5.0 * w["N"] * math.log2(w["N"]) * w["core_ffts"] * w["runs"] * ns
        p32 = fp32_peak(local)
        line = {"metric": METRIC, "value": value, "unit": "Gsamples/s", "n_gpus": reps.world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic: " + w["signal"],
                "precision": {gpu.PREC_FP32: "fp32", gpu.PREC_TCSPLIT: "tcsplit"}[prec],
                "config": {"workload": w["desc"], "fft_points": w["N"], "sources": ns,
                           "samples_per_step": samples, "bytes_per_step": bytes_in,
                           "l2": "inputs larger than L2 (%.0f MB per step)" % (bytes_in / 1e6),
                           "plan": core.plan_info()},
                "clocks": cs.summary(), "gpu_launches": launches * args.steps,
                "e2e": {"value": e2e_val, "unit": "Gsamples/s", "h2d_bytes_per_step": w["run_bytes"] * w["runs"],
                        "d2h_bytes_per_step": d2h,
                        "path": "swsgpu_submit_out/wait per run from pinned host memory (TaskCore path, the "
                                "run given its output buffers), device combine, spectra into pinned host arrays"},
                "roofline": {"bound": "fp32", "achieved": flops / (ms * 1e-3) / 1e12, "peak": p32,
                             "unit": "TFLOP/s", "frac": flops / (ms * 1e-3) / 1e12 / p32 if p32 else None,
                             "traffic": None, "scope": "whole step (every kernel of the step)",
                             "peak_source": "FP32 FMA issue, measured on this GPU by fp32_probe.cu",
                             "hbm": {"achieved_gbs": bytes_in / (ms * 1e-3) / 1e9, "peak_gbs": peaks["hbm_gbs"],
                                     "frac": bytes_in / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"]},
                             "fft_kernel_ms_per_launch": kern_s * 1e3, "fft_kernel_launches_per_step": nk / 3},
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    core.close()
    reps.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp32", "tcsplit", "tcsplit_all"])
    ap.add_argument("--e2e-cores", type=int, default=2,
                    help="cores of the end-to-end leg, one integration each, runs interleaved (>= 2)")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--plan", default="auto", choices=["auto", "cluster", "fourstep"],
                    help="FFT path for the cross-spectra workload (auto: cluster kernel)")
    ap.add_argument("--candidate", type=int, default=-1,
                    help="c2/c5: pin four-step split k of the length's candidates instead of autotuning")
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5", "vlba"],
                    help="c3: dual-pol cross-spectra (the default line); c1: plain single channel; "
                         "c2: 3.2M-point spectra with phase-cal tones; c4: batched uneven streams; "
                         "c5: 2^22-point 8-bit dynamic range")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "c4":
        c4_arm(args)
    elif args.workload in SPEC_WORKLOADS:
        spec_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
