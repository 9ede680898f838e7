"""The drop-in, proven against the reference's own interface.

swspec_b200/refcore/Makefile builds the reference's own spectrometer program
-- its main (src/swspectrometer.cpp), TaskDispatcher, FileSource (with
mark5access), FileSink, Buffer, IniParser and LogFile, compiled from the
reference sources -- with TaskDispatcher.h selecting TaskCoreCUDA
(swspec_b200/refcore/TaskCoreCUDA.cpp), a subclass of the reference's
abstract TaskCore (src/TaskCore.h:36-89) over libswsgpu.so.  These tests run
that program on Mark5B files and compare the spectrum files it writes with
the FP64 oracle over the same core-run schedule.
"""
import os
import subprocess

import numpy as np
import pytest

from test_host import PCAL, _ini, _model_runs, _pcal_signal_files
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


@pytest.mark.parametrize("precision", ["fp32", "tcsplit"])
def test_reference_dispatcher_drives_gpu_core(tmp_path, gpu, precision):
    """Two Mk5B files (channels 3 and 12 of 16, 2-bit), cross-pol and PCal,
    each spectrum summed over 3 core runs (MaxSourceBufferMB = 1): the
    reference's dispatcher loop writes 2 spectra per file, the cross spectrum
    with the half length its combineResults sets, and phase-cal vectors."""
    N, fs = 4096, 32e6
    files = _pcal_signal_files(tmp_path, 197, fs, 77)
    ini = _ini(tmp_path, f"""[Spectrometer]
NumCPUCores = 1
FFTpoints = {N}
FFTIntegrationTimeSec = 0.00615
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
PCalOffsetHz = 15625
MaxSourceBufferMB = 1
BaseFilename1 = r_%channel%
""")
    if precision == "tcsplit":
        # the split form exists for N = 8192 .. 65536
        ini = _ini(tmp_path, open(ini).read().replace(f"FFTpoints = {N}", "FFTpoints = 8192")
                   .replace("0.00615", "0.0123"))
        N = 8192
    _run(tmp_path, ini, files, precision)
    rawbuf = 262144 if N == 4096 else 524288
    cof = rawbuf * 8 // (2 * 16) // N
    pays = [synth.strip_headers((tmp_path / f).read_bytes(), 10016, 16) for f in files]
    runs = _model_runs(pays, rawbuf, N, 1, cof, [2, 11], 16, pcal=PCAL, xpol=True)
    ngroup = len(runs) // 3
    assert ngroup >= 1
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
