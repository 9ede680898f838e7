"""The C++ host: settings derivation, INI semantics, and (GPU) the whole
drop-in path -- swspectrometer_gpu reading Mark5B files through FileSource,
TaskCoreCUDA, TaskDispatcher and FileSink -- against the FP64 oracle run over
the same core-run schedule (src/TaskDispatcher.cpp:92-247)."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from swspec_b200 import synth
from swspec_b200.settings import from_ini_values

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "swspec_b200", "swspectrometer_gpu")


def _ini(tmp_path, body: str) -> str:
    p = tmp_path / "run.ini"
    p.write_text(body)
    return str(p)


def _settings(ini: str, ninputs: int = 1) -> dict:
    r = subprocess.run([EXE, "--print-settings", ini, str(ninputs)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_settings_match_reference_derivation(tmp_path):
    ini = _ini(tmp_path, """[Spectrometer]
FFTpoints = 65536
FFTIntegrationTimeSec = 1
FFToverlapFactor = 1
BandwidthHz = 32e6
SourceFormat = Mark5B-2048-16-2
UseFile1Channel = 1
WindowType = Hann
BaseFilename1 = out_%fftpoints%_%channel%
""")
    s = _settings(ini)
    assert s["gpu_autotune"] == 0            # off unless asked for
    py = from_ini_values(fft_points=65536, fft_integ_seconds=1.0, fft_overlap_factor=1,
                         BandwidthHz=32e6, bits_per_sample=2, source_channels=16)
    for k in ["averaged_ffts", "raw_fullfft_bytes", "rawbuf_size", "max_buffers_per_spectrum",
              "max_specffts_per_buffer", "core_overlapped_ffts", "fft_ssb_points"]:
        assert s[k] == getattr(py, k), k
    assert s["basefilename1"] == "out_65536_1" and s["wf_type"] == 4


def test_ini_parser_semantics(tmp_path):
    """Whitespace anywhere is dropped, / ' # start comments, first duplicate wins,
    integers go through atof, unknown windows fall back to Cosine2."""
    ini = _ini(tmp_path, """# comment line
[Spectrometer]
FFT points = 3 2 768   # spaces removed
FFTpoints = 1024
FFTIntegrationTimeSec = 0.5
FFToverlapFactor = 2.9
BandwidthHz = 16e6 ' trailing comment
SourceFormat = Mark5B-1024-16-2
WindowType = Triangle
ExtractPCal = yes
PCalOffsetHz = 15625
MaxSourceBufferMB = 64
GpuAutotune = yes
BaseFilename1 = plain
""")
    s = _settings(ini)
    assert s["gpu_autotune"] == 1            # GPU-core key, absent from the reference's settings
    assert s["fft_points"] == 32768          # 'FFT points' == 'FFTpoints', first wins
    assert s["wf_type"] == 2                 # unknown -> Cosine2
    py = from_ini_values(fft_points=32768, fft_integ_seconds=0.5, fft_overlap_factor=2,
                         BandwidthHz=16e6, bits_per_sample=2, source_channels=16,
                         MaxSourceBufferMB=64, extract_PCal=True, pcaloffsethz=15625)
    assert s["core_overlapped_ffts"] == py.core_overlapped_ffts
    assert s["rawbuf_size"] == py.rawbuf_size
    assert s["pcal_rotatorlen"] == 2048 and s["pcal_tonebins"] == 32 and s["extract_PCal"] == 1


def test_xpol_needs_two_inputs(tmp_path):
    ini = _ini(tmp_path, """[Spectrometer]
FFTpoints = 4096
SourceFormat = Mark5B-1024-16-2
DoCrossPolarization = yes
BaseFilename1 = x
""")
    assert _settings(ini, 1)["calc_Xpol"] == 0
    assert _settings(ini, 2)["calc_Xpol"] == 1


def _model_runs(payloads, rawbuf, N, overlap, cof, chans, nchan, pcal=None, xpol=False):
    """FP64 oracle over the dispatcher's buffers: rawbuf payload bytes each;
    the buffer that meets the end of file is read but not processed, so only
    whole buffers run (TaskDispatcher.cpp:170-243)."""
    nbuf = min(len(p) for p in payloads) // rawbuf
    runs = []
    for b in range(nbuf):
        samples = [O.decode(O.FMT_MARK5B, nchan, 2, p[b * rawbuf:(b + 1) * rawbuf], rawbuf * 8 // (2 * nchan), c)
                   for p, c in zip(payloads, chans)]
        cfg = O.make_cfg(N, overlap=overlap, core_overlapped_ffts=cof, num_sources=len(samples),
                         num_xpols=1 if xpol else 0, window=O.W_HANN)
        if pcal:
            cfg.extract_pcal = 1
            cfg.pcal_tonebins, cfg.pcal_rotatorlen = pcal["tonebins"], pcal["rotatorlen"]
            cfg.samplingfreq, cfg.pcaloffsethz = pcal["fs"], pcal["offset"]
        runs.append(O.domaths(cfg, samples))
    return runs


def _pcal_signal_files(tmp_path, nfr, fs, seed):
    rng = np.random.default_rng(seed)
    names = []
    for k in range(2):
        comb = synth.pcal_comb(nfr * 2500, fs, 1e6, 15625.0, 0.05, rng.uniform(0, 6.28, 16))
        sig = rng.standard_normal((16, nfr * 2500)) + comb[None, :]
        (tmp_path / f"in{k}.m5b").write_bytes(synth.mark5b_stream(sig, 2, 1024))
        names.append(f"in{k}.m5b")
    return names


def _run_cli(tmp_path, ini, files):
    # paths stay relative: '/' starts a comment in the reference's INI syntax
    r = subprocess.run([EXE, ini] + files, capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-3000:]
    return r


PCAL = dict(tonebins=32, rotatorlen=2048, fs=32e6, offset=15625.0)


@pytest.mark.gpu
@pytest.mark.parametrize("on_device,fixlen", [(True, True), (False, False)])
def test_cli_multi_buffer_spectra(tmp_path, gpu, on_device, fixlen):
    """Two Mark5B files (channels 3 and 12), cross-pol and PCal, each spectrum
    summed over 3 core runs of 16 FFTs (averaged_ffts 48 > 512 KiB buffers);
    7 whole buffers -> 2 spectra, the 7th run and the partial 8th buffer
    dropped as the reference drops them."""
    N, fs = 4096, 32e6
    files = _pcal_signal_files(tmp_path, 197, fs, 77)
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.00615
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = Mark5B-1024-16-2
UseFile1Channel = 3
UseFile2Channel = 12
DoCrossPolarization = yes
ExtractPCal = yes
PCalOffsetHz = 15625
MaxSourceBufferMB = 1
GpuCombineOnDevice = {"yes" if on_device else "no"}
FixXpolLength = {"yes" if fixlen else "no"}
BaseFilename1 = s_%channel%
""")
    s = _settings(ini, 2)
    assert (s["averaged_ffts"], s["max_buffers_per_spectrum"], s["core_overlapped_ffts"], s["rawbuf_size"]) == \
        (48, 3, 16, 262144), s
    _run_cli(tmp_path, ini, files)
    pays = [synth.strip_headers((tmp_path / f).read_bytes(), 10016, 16) for f in files]
    runs = _model_runs(pays, s["rawbuf_size"], N, 1, 16, [2, 11], 16, pcal=PCAL, xpol=True)
    assert len(runs) == 7 and all(r[3] == 1 for r in runs)
    groups = [[sum(r[i][0] for r in runs[g:g + 3]) for i in range(3)] for g in (0, 3)]
    S = N // 2 + 1
    a = [np.fromfile(tmp_path / f"s_{c}_swspec.bin", dtype=np.float32).reshape(-1, S) for c in (3, 12)]
    pc = [np.fromfile(tmp_path / f"s_{c}_pcal.bin", dtype=np.float32).reshape(-1, 32, 2) for c in (3, 12)]
    xraw = np.fromfile(tmp_path / "s_3_xpol_swspec.bin", dtype=np.float32)
    xp = xraw.reshape(-1, S, 2) if fixlen else xraw.reshape(-1, S)
    assert a[0].shape[0] == a[1].shape[0] == pc[0].shape[0] == xp.shape[0] == 2
    for g, (ra, rx, rp) in enumerate(groups):
        for k in range(2):
            assert np.max(np.abs(a[k][g] - ra[k]) / ra[k]) < 2e-6
            pcc = pc[k][g, :, 0] + 1j * pc[k][g, :, 1]
            assert np.max(np.abs(pcc - rp[k])) / np.max(np.abs(rp[k])) < 1e-6
        norm = np.sqrt(ra[0] * ra[1])
        if fixlen:
            xc = xp[g, :, 0] + 1j * xp[g, :, 1]
            assert np.max(np.abs(xc - rx[0]) / norm) < 2e-6
        else:
            # half of the interleaved cross spectrum, as the reference writes it
            ri = np.stack([rx[0].real, rx[0].imag], -1).reshape(-1)[:S]
            ni = np.repeat(norm, 2)[:S]
            assert np.max(np.abs(xp[g] - ri) / ni) < 2e-6
    assert (tmp_path / "s_3_runlog.txt").exists() and (tmp_path / "s_3_starttiming.txt").exists()
    assert "second" in (tmp_path / "s_3_starttiming.txt").read_text()


@pytest.mark.gpu
@pytest.mark.parametrize("sink", ["binary", "ascii"])
def test_cli_spectra_per_buffer_overlap(tmp_path, gpu, sink):
    """One file, 50% overlap, several whole spectra per buffer plus the
    unscaled trailing partial spectrum of each buffer; binary sink and the
    reference's ASCII layout (FileSink.cpp:80-102)."""
    N, fs = 8192, 32e6
    files = _pcal_signal_files(tmp_path, 140, fs, 5)[:1]
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.0013
FFToverlapFactor = 2
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = Mark5B-1024-16-2
UseFile1Channel = 7
MaxSourceBufferMB = 1
SinkFormat = {sink}
BaseFilename1 = o_%fftpoints%
""")
    s = _settings(ini, 1)
    assert s["max_buffers_per_spectrum"] == 0 and s["max_spectra_per_buffer"] >= 2, s
    _run_cli(tmp_path, ini, files)
    pay = synth.strip_headers((tmp_path / files[0]).read_bytes(), 10016, 16)
    runs = _model_runs([pay], s["rawbuf_size"], N, 2, s["core_overlapped_ffts"], [6], 16)
    if sink == "binary":
        ref = np.concatenate([r[0][:, 0, :] for r in runs])
        got = np.fromfile(tmp_path / "o_8192_swspec.bin", dtype=np.float32).reshape(-1, N // 2 + 1)
        assert got.shape == ref.shape, (got.shape, ref.shape)
        assert np.max(np.abs(got - ref) / ref) < 2e-6
        return
    # one data set per written buffer: every other float, then the buffer's
    # second float as "Nyquist"; 12 significant digits
    sets = (tmp_path / "o_8192_swspec.bin").read_text().split("// --------------------- DATA SET TIMESTAMP")[1:]
    assert len(sets) == len(runs)
    for text, r in zip(sets, runs):
        vals = np.array([float(v) for v in text.splitlines()[2:] if v.strip()])
        flat = r[0][:, 0, :].reshape(-1)
        npair = flat.size // 2
        ref = np.concatenate([flat[0:2 * npair:2], flat[1:2]])
        assert vals.shape == ref.shape
        assert np.max(np.abs(vals - ref) / ref) < 2e-6


@pytest.mark.gpu
def test_cli_multithread_vdif_selects_one_thread(tmp_path, gpu):
    """A VDIF recording with two interleaved threads (frames alternate between
    thread 0 and thread 1, each its own signal): VdifThread = 1 keeps that
    thread's frames only, which then form one contiguous stream (two whole
    512 KiB buffers of 32 spectra each; the third meets the end of file)."""
    N, cof = 8192, 8
    rng = np.random.default_rng(61)
    nfr = 140
    frames = []
    codes_by_thread = []
    for th in range(2):
        pay = rng.integers(0, 256, nfr * 8000, dtype=np.uint8).tobytes()
        codes_by_thread.append(pay)
        frames.append(np.frombuffer(synth.vdif_frames(pay, 8000, 1, 2, 4000, thread=th),
                                    dtype=np.uint8).reshape(nfr, -1))
    inter = np.stack(frames, axis=1).reshape(-1).tobytes()   # t0 f0, t1 f0, t0 f1, ...
    (tmp_path / "mt.vdif").write_bytes(inter)
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.002048
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = VDIF_8000-64-1-2
VdifThread = 1
MaxSourceBufferMB = 1
BaseFilename1 = v
""")
    s = _settings(ini, 1)
    rawbuf = s["rawbuf_size"]
    assert rawbuf == 524288 and s["max_spectra_per_buffer"] == 32, s
    _run_cli(tmp_path, ini, ["mt.vdif"])
    pay1 = codes_by_thread[1]
    nbuf = len(pay1) // rawbuf
    ref = []
    for b in range(nbuf):
        x = O.decode(O.FMT_VDIF, 1, 2, pay1[b * rawbuf:(b + 1) * rawbuf], rawbuf * 4, 0)
        cfg = O.make_cfg(N, core_overlapped_ffts=s["core_overlapped_ffts"], num_sources=1, window=O.W_HANN)
        ra, _, _, n = O.domaths(cfg, [x])
        ref.append(ra[:, 0])
    ref = np.concatenate(ref)
    got = np.fromfile(tmp_path / "v_swspec.bin", dtype=np.float32).reshape(-1, N // 2 + 1)
    assert got.shape == ref.shape == (64, N // 2 + 1), (got.shape, ref.shape)
    assert np.max(np.abs(got - ref) / ref) < 2e-6


def _ibob_file(path, nframes, seed, tone):
    """iBOB capture: frames of a 4-byte sequence header and 4096 bytes of
    signed 8-bit samples, two channels interleaved (a tone in channel 0).
    Returns the payload bytes."""
    rng = np.random.default_rng(seed)
    n = nframes * 2048
    t = np.arange(n)
    x = rng.standard_normal((n, 2)) * 20
    x[:, 0] += tone * np.cos(2 * np.pi * 0.0711 * t)
    q = np.clip(np.round(x), -128, 127).astype(np.int8).reshape(nframes, 4096).view(np.uint8)
    hdr = np.zeros((nframes, 4), np.uint8)
    hdr[:, 0] = 0x5E
    hdr[:, 3] = (np.arange(nframes) + 1) & 0xFF
    path.write_bytes(np.concatenate([hdr, q], axis=1).tobytes())
    return q.reshape(-1).tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["tcsplit", "tcsplit_all", "fp32"])
def test_cli_ibob_spectra_per_buffer(tmp_path, gpu, precision):
    """Two iBOB files (signed 8-bit, two channels; channel 1 of the first and
    channel 2 of the second), cross-pol, N = 8192, on each GPU form: the
    4-byte headers are stripped (src/FileSource.cpp:53-57, 185-210) and the
    payloads form one contiguous stream, whole spectra per buffer."""
    N = 8192
    pays = [_ibob_file(tmp_path / f"in{k}.ibob", 500, 30 + k, 8.0 * (k + 1)) for k in range(2)]
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.006144
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = iBob
BitsPerSample = 8
SourceChannels = 2
UseFile1Channel = 1
UseFile2Channel = 2
DoCrossPolarization = yes
MaxSourceBufferMB = 1
GpuPrecision = {precision}
BaseFilename1 = b_%channel%
""")
    s = _settings(ini, 2)
    rawbuf, cof, nsp = s["rawbuf_size"], s["core_overlapped_ffts"], s["max_spectra_per_buffer"]
    assert nsp >= 1 and s["max_buffers_per_spectrum"] == 0, s
    _run_cli(tmp_path, ini, ["in0.ibob", "in1.ibob"])
    S = N // 2 + 1
    nbuf = len(pays[0]) // rawbuf
    assert nbuf >= 4
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


@pytest.mark.gpu
def test_cli_mark4_spectra_per_buffer(tmp_path, gpu):
    """A Mark4 recording in the reference's own example mode
    (MKIV1_2-512-8-2: 32 tracks, 8 channels, 2-bit, fanout 2) through the
    front end (frames read whole after 1000 leading bytes) and the GPU core:
    channel 3's spectra, four per buffer, against the FP64 oracle on
    mark5access's decode of the same frames (header track-words blanked)."""
    from test_frontend import _track_file
    N = 8192
    data, pay = _track_file("MKIV", 32, 60, 1000, 12)
    (tmp_path / "in.m4").write_bytes(data)
    ini = _ini(tmp_path, f"""[Spectrometer]
FFTpoints = {N}
FFTIntegrationTimeSec = 0.004096
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = MKIV1_2-512-8-2
UseFile1Channel = 3
MaxSourceBufferMB = 1
BaseFilename1 = m4_%channel%
""")
    s = _settings(ini, 1)
    rawbuf, cof, nsp = s["rawbuf_size"], s["core_overlapped_ffts"], s["max_spectra_per_buffer"]
    assert nsp >= 1 and s["max_buffers_per_spectrum"] == 0, s
    _run_cli(tmp_path, ini, ["in.m4"])
    S = N // 2 + 1
    nbuf = len(pay) // rawbuf
    assert nbuf >= 3
    per_buf = rawbuf * 8 // 16                       # samples per channel in a buffer
    dec, _ = O.m5_unpack("MKIV1_2-512-8-2", pay, nbuf * per_buf)
    ra = []
    for b in range(nbuf):
        cfg = O.make_cfg(N, core_overlapped_ffts=cof, num_sources=1, window=O.W_HANN, nthreads=os.cpu_count() or 1)
        a, _, _, n = O.domaths(cfg, [dec[2, b * per_buf:(b + 1) * per_buf]])
        ra.append(a[:nsp, 0])
    ra = np.concatenate(ra)
    got = np.fromfile(tmp_path / "m4_3_swspec.bin", dtype=np.float32).reshape(-1, S)
    assert got.shape[0] == ra.shape[0] == nbuf * nsp
    assert np.max(np.abs(got - ra) / ra) < 2e-6
