"""The drop-in, proven against the reference's own interface.

swspec_b200/refcore/Makefile builds the reference's own spectrometer program
-- its main (src/swspectrometer.cpp), TaskDispatcher, FileSource (with
mark5access), FileSink, Buffer, IniParser and LogFile, compiled from the
reference sources -- with TaskDispatcher.h selecting TaskCoreCUDA
(swspec_b200/refcore/TaskCoreCUDA.cpp), a subclass of the reference's
abstract TaskCore (src/TaskCore.h:36-89) over libswsgpu.so.  These tests run
that program on recordings and compare the spectrum files it writes with
the FP64 oracle over the same core-run schedule.

The reference's framed FileSource::read (src/FileSource.cpp:185-210) always
reads the rest of the current frame, however little room the buffer has
left: a raw buffer that is not a whole number of frame payloads is overrun
(heap memory past it is overwritten) and the next buffer starts at the next
frame.  The Mk5B settings below therefore give buffers of whole frames
(N = 20000: 640000-byte buffers, 64 payloads of 10000 bytes).

Its FileSource::open (src/FileSource.cpp:127-159) steps back one header
length from the current offset after locateFirstHeader; for VDIF and iBOB
that function reads no header, so the step goes before byte 0, the stream's
failbit is set and every later read fails: the program hands one buffer that
the file never filled to the cores and stops.  The reference program is
therefore run here on Mk5B and on the headerless RawSigned format; iBOB and
VDIF files go through this package's own front end (tests/test_host.py).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from test_host import _ini, _model_runs, _pcal_signal_files, _settings
from swspec_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "swspec_b200", "refcore", "_ref", "swspectrometer_cuda")


def _run(tmp_path, ini, files, precision):
    assert os.path.exists(EXE), "reference program with the GPU core not built (swspec_b200/refcore/Makefile)"
    env = dict(os.environ, SWSGPU_PRECISION=precision)
    r = subprocess.run([EXE, ini] + files, capture_output=True, text=True, timeout=300, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "TaskCoreCUDA 0:" in r.stderr and "runs" in r.stderr, r.stderr[-2000:]
    return r


def test_reference_dispatcher_mk5b_combined_spectra(tmp_path, gpu):
    """Two Mk5B files (channels 3 and 12 of 16, 2-bit), cross-pol and PCal,
    each spectrum summed over 3 core runs: the reference's dispatcher writes
    2 spectra per file, the cross spectrum with the half length its
    combineResults sets (TaskCoreIPP.cpp:333), and phase-cal vectors."""
    N, fs = 20000, 32e6
    files = _pcal_signal_files(tmp_path, 450, fs, 77)
    body = f"""[Spectrometer]
NumCPUCores = 1
FFTpoints = {N}
FFTIntegrationTimeSec = 0.015
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = Mk5B
BitsPerSample = 2
SourceChannels = 16
UseFile1Channel = 3
UseFile2Channel = 12
DoCrossPolarization = yes
ExtractPCal = yes
PCalOffsetHz = 200000
MaxSourceBufferMB = 1
BaseFilename1 = r_%channel%
"""
    ini = _ini(tmp_path, body)
    s = _settings(ini, 2)
    rawbuf, cof = s["rawbuf_size"], s["core_overlapped_ffts"]
    assert rawbuf % 10000 == 0 and s["max_buffers_per_spectrum"] == 3, s
    _run(tmp_path, ini, files, "fp32")
    pays = [synth.strip_headers((tmp_path / f).read_bytes(), 10016, 16) for f in files]
    pcal = dict(tonebins=32, rotatorlen=160, fs=fs, offset=200e3)
    runs = _model_runs(pays, rawbuf, N, 1, cof, [2, 11], 16, pcal=pcal, xpol=True)
    ngroup = len(runs) // 3
    assert ngroup == 2
    groups = [[sum(r[i][0] for r in runs[3 * g:3 * g + 3]) for i in range(3)] for g in range(ngroup)]
    S = N // 2 + 1
    a = [np.fromfile(tmp_path / f"r_{c}_swspec.bin", dtype=np.float32).reshape(-1, S) for c in (3, 12)]
    pc = [np.fromfile(tmp_path / f"r_{c}_pcal.bin", dtype=np.float32).reshape(-1, 32, 2) for c in (3, 12)]
    xp = np.fromfile(tmp_path / "r_3_xpol_swspec.bin", dtype=np.float32).reshape(-1, S)
    assert a[0].shape[0] == a[1].shape[0] == pc[0].shape[0] == xp.shape[0] == ngroup
    for g, (ra, rx, rp) in enumerate(groups):
        for k in range(2):
            assert np.max(np.abs(a[k][g] - ra[k]) / ra[k]) < 2e-6
            pcc = pc[k][g, :, 0] + 1j * pc[k][g, :, 1]
            assert np.max(np.abs(pcc - rp[k])) / np.max(np.abs(rp[k])) < 1e-6
        norm = np.sqrt(ra[0] * ra[1])
        # the first half of the interleaved cross spectrum, as the reference writes it
        ri = np.stack([rx[0].real, rx[0].imag], -1).reshape(-1)[:S]
        ni = np.repeat(norm, 2)[:S]
        assert np.max(np.abs(xp[g] - ri) / ni) < 2e-6
    assert (tmp_path / "r_3_runlog.txt").exists() and (tmp_path / "r_3_starttiming.txt").exists()


def _raw8_file(path, nbytes, seed, tone):
    """Headerless capture of signed 8-bit samples, two channels interleaved
    (a tone in channel 0)."""
    rng = np.random.default_rng(seed)
    n = nbytes // 2
    t = np.arange(n)
    x = rng.standard_normal((n, 2)) * 20
    x[:, 0] += tone * np.cos(2 * np.pi * 0.0711 * t)
    q = np.clip(np.round(x), -128, 127).astype(np.int8).reshape(-1).view(np.uint8)
    path.write_bytes(q.tobytes())
    return q.tobytes()


@pytest.mark.parametrize("precision", ["tcsplit", "tcsplit_all", "fp32"])
def test_reference_dispatcher_raw8_spectra_per_buffer(tmp_path, gpu, precision):
    """Two RawSigned files (signed 8-bit, two channels; channel 1 of the first
    and channel 2 of the second), cross-pol, N = 8192: whole spectra per core
    run written straight from the cores' output buffers
    (TaskDispatcher.cpp:172-191), on each GPU form.  The buffer that meets
    the end of file is read but not processed."""
    N = 8192
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.006144
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = RawSigned
BitsPerSample = 8
SourceChannels = 2
UseFile1Channel = 1
UseFile2Channel = 2
DoCrossPolarization = yes
MaxSourceBufferMB = 1
BaseFilename1 = b_%channel%
""")
    s = _settings(ini, 2)
    rawbuf, cof, nsp = s["rawbuf_size"], s["core_overlapped_ffts"], s["max_spectra_per_buffer"]
    assert nsp >= 1 and s["max_buffers_per_spectrum"] == 0, s
    pays = [_raw8_file(tmp_path / f"in{k}.raw", 4 * rawbuf + 1000, 30 + k, 8.0 * (k + 1)) for k in range(2)]
    _run(tmp_path, ini, ["in0.raw", "in1.raw"], precision)
    S = N // 2 + 1
    nbuf = len(pays[0]) // rawbuf
    ra_all, rx_all = [], []
    for b in range(nbuf):
        smp = [O.decode(O.FMT_RAW_SIGNED, 2, 8, p[b * rawbuf:(b + 1) * rawbuf], rawbuf // 2, c)
               for p, c in zip(pays, (0, 1))]
        cfg = O.make_cfg(N, core_overlapped_ffts=cof, num_sources=2, num_xpols=1, window=O.W_HANN,
                         nthreads=os.cpu_count() or 1)
        ra, rx, _, n = O.domaths(cfg, smp)
        ra_all.append(ra[:nsp])
        rx_all.append(rx[:nsp, 0])
    ra = np.concatenate(ra_all)
    rx = np.concatenate(rx_all)
    a0 = np.fromfile(tmp_path / "b_1_swspec.bin", dtype=np.float32).reshape(-1, S)
    a1 = np.fromfile(tmp_path / "b_2_swspec.bin", dtype=np.float32).reshape(-1, S)
    xp = np.fromfile(tmp_path / "b_1_xpol_swspec.bin", dtype=np.float32).reshape(-1, S, 2)
    assert a0.shape[0] == a1.shape[0] == xp.shape[0] == ra.shape[0] == nbuf * nsp
    assert np.max(np.abs(a0 - ra[:, 0]) / ra[:, 0]) < 2e-6
    assert np.max(np.abs(a1 - ra[:, 1]) / ra[:, 1]) < 2e-6
    xc = xp[..., 0] + 1j * xp[..., 1]
    assert np.max(np.abs(xc - rx) / np.sqrt(ra[:, 0] * ra[:, 1])) < 2e-6
