"""The C++ front end's FileSource alone (no GPU): swspectrometer_gpu
--read-source reads a recording into buffers of the INI's raw buffer size
and writes the payload bytes it delivered.  Covers the framed read
(src/FileSource.cpp:185-210) and the faults the reference logs and reads
past: a frame header without the Mark5B sync word (:401-427), a file that
ends inside a frame, a start time that is not a BCD time (:338-339), leading
bytes before the first frame, and no frame at all."""
import json
import os
import subprocess

import numpy as np
import pytest

from swspec_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "swspec_b200", "swspectrometer_gpu")
FRAME = 10016

INI = """[Spectrometer]
FFTpoints = 4096
FFTIntegrationTimeSec = 0.00615
FFToverlapFactor = 1
BandwidthHz = 16e6
WindowType = Hann
SourceFormat = {fmt}
UseFile1Channel = 1
MaxSourceBufferMB = 1
BaseFilename1 = fe
"""


def _read(tmp_path, data: bytes, fmt="Mark5B-1024-16-2", extra=""):
    (tmp_path / "in.bin").write_bytes(data)
    ini = tmp_path / "fe.ini"
    ini.write_text(INI.format(fmt=fmt) + extra)
    out = tmp_path / "out.bin"
    r = subprocess.run([EXE, "--read-source", str(ini), str(tmp_path / "in.bin"), str(out)],
                       capture_output=True, text=True, timeout=120)
    info = json.loads(r.stdout) if r.returncode == 0 else None
    got = out.read_bytes() if out.exists() else b""
    return r, info, got


def _mark5b(nfr, seed=3):
    rng = np.random.default_rng(seed)
    pay = rng.integers(0, 256, nfr * 10000, dtype=np.uint8).tobytes()
    return synth.mark5b_frames(pay, 1024), pay


def _settings(tmp_path, fmt="Mark5B-1024-16-2"):
    ini = tmp_path / "s.ini"
    ini.write_text(INI.format(fmt=fmt))
    r = subprocess.run([EXE, "--print-settings", str(ini), "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_payloads_in_order_and_buffer_sizes(tmp_path):
    data, pay = _mark5b(60)
    r, info, got = _read(tmp_path, data)
    assert r.returncode == 0, r.stderr
    rawbuf = _settings(tmp_path)["rawbuf_size"]
    assert got == pay
    assert all(n == rawbuf for n in info["buffers"][:-1]) and sum(info["buffers"]) == len(pay)
    assert info["frames"] == 60 and info["bad_sync_frames"] == 0
    assert "mismatch" not in r.stderr and "ends inside" not in r.stderr


def test_leading_garbage_before_the_first_frame(tmp_path):
    data, pay = _mark5b(12)
    junk = bytes(np.random.default_rng(1).integers(0, 256, 1234, dtype=np.uint8))
    r, info, got = _read(tmp_path, junk + data)
    assert r.returncode == 0, r.stderr
    assert got == pay
    assert "first Mark5B frame at byte 1234" in r.stderr


def test_corrupted_sync_word_is_reported_and_read_past(tmp_path):
    data, pay = _mark5b(12)
    a = bytearray(data)
    for k in (4, 9):
        a[k * FRAME:k * FRAME + 4] = b"\x00\x11\x22\x33"
    r, info, got = _read(tmp_path, bytes(a))
    assert r.returncode == 0, r.stderr
    # the payloads still arrive, as the reference keeps reading
    assert got == pay
    assert info["bad_sync_frames"] == 2
    assert f"mismatch in frame 4 at byte {4 * FRAME}" in r.stderr
    assert f"mismatch in frame 9 at byte {9 * FRAME}" in r.stderr


def test_file_truncated_inside_a_frame(tmp_path):
    data, pay = _mark5b(12)
    cut = 7 * FRAME + 16 + 4321          # 4321 payload bytes of frame 7
    r, info, got = _read(tmp_path, data[:cut])
    assert r.returncode == 0, r.stderr
    assert got == pay[:7 * 10000 + 4321]
    assert sum(info["buffers"]) == 7 * 10000 + 4321
    assert "ends inside frame 7 after 4321 of 10000 payload bytes" in r.stderr


def test_truncated_inside_a_header(tmp_path):
    data, pay = _mark5b(12)
    r, info, got = _read(tmp_path, data[:5 * FRAME + 9])
    assert r.returncode == 0, r.stderr
    assert got == pay[:5 * 10000] and info["frames"] == 5


def test_bad_bcd_start_time_is_reported(tmp_path):
    data, pay = _mark5b(4)
    a = bytearray(data)
    a[8:12] = np.array([0x123A5678], dtype="<u4").tobytes()   # digit 0xA
    r, info, got = _read(tmp_path, bytes(a))
    assert r.returncode == 0, r.stderr
    assert got == pay
    assert "not a valid BCD time (digits 1 2 3 10 5 6 7 8)" in r.stderr
    timing = (tmp_path / "out.bin.starttiming.txt").read_text()
    assert "First frame at byte 0" in timing


def test_good_bcd_start_time(tmp_path):
    data, _ = _mark5b(4)
    r, _, _ = _read(tmp_path, data)
    timing = (tmp_path / "out.bin.starttiming.txt").read_text()
    assert "MJD(mod 1000) 0 second 100" in timing      # synth: MJD 57000, second 100
    assert "BCD" not in r.stderr


def test_no_mark5b_frame_fails_open(tmp_path):
    junk = bytes(np.random.default_rng(2).integers(0, 256, 50000, dtype=np.uint8))
    r, info, _ = _read(tmp_path, junk)
    assert r.returncode != 0 and "no Mark5B frame found" in r.stderr


def test_ibob_headers_stripped(tmp_path):
    rng = np.random.default_rng(4)
    nfr = 300
    pay = rng.integers(0, 256, (nfr, 4096), dtype=np.uint8)
    hdr = np.zeros((nfr, 4), np.uint8)
    hdr[:, 3] = (np.arange(nfr) + 1) & 0xFF
    r, info, got = _read(tmp_path, np.concatenate([hdr, pay], 1).tobytes(), fmt="iBob",
                         extra="BitsPerSample = 8\nSourceChannels = 2\n")
    assert r.returncode == 0, r.stderr
    assert got == pay.tobytes() and info["frames"] == nfr


def test_vdif_thread_selection(tmp_path):
    rng = np.random.default_rng(6)
    nfr = 40
    pays = [rng.integers(0, 256, nfr * 8000, dtype=np.uint8).tobytes() for _ in range(2)]
    fr = [np.frombuffer(synth.vdif_frames(p, 8000, 1, 2, 4000, thread=t), np.uint8).reshape(nfr, -1)
          for t, p in enumerate(pays)]
    inter = np.stack(fr, axis=1).reshape(-1).tobytes()
    r, info, got = _read(tmp_path, inter, fmt="VDIF_8000-64-1-2", extra="VdifThread = 1\n")
    assert r.returncode == 0, r.stderr
    assert got == pays[1]


def _time_words(digits, tb: int) -> np.ndarray:
    """BCD nibbles as header track-words: four per nibble, most significant
    bit first, all tracks of a track-word carrying the bit."""
    out = np.zeros(4 * len(digits) * tb, np.uint8)
    for i, d in enumerate(digits):
        for b in range(4):
            if (d >> b) & 1:
                out[(4 * i + 3 - b) * tb:(4 * i + 4 - b) * tb] = 0xFF
    return out


def _track_file(kind: str, ntrack: int, nfr: int, lead: int, seed: int, digits=None):
    """A VLBA (20160 track-words per frame: sync, time code, payload of
    20000, 64 trailing) or Mark4 (20000 per frame: 64 auxiliary, sync, time
    code, data) recording after `lead` bytes of other data; returns the file
    and the payload stream the GPU core takes.  `digits`: the time code's
    BCD digits (12 for VLBA, 13 for Mark4) in every frame's header."""
    tb = ntrack // 8
    rng = np.random.default_rng(seed)
    frames, payload = [], []
    for _ in range(nfr):
        if kind == "VLBA":
            hdr = np.zeros(64 * tb, np.uint8)
            if digits is not None:
                hdr[:48 * tb] = _time_words(digits, tb)
            data = rng.integers(0, 256, 20000 * tb, dtype=np.uint8)
            fr = np.concatenate([np.full(32 * tb, 0xFF, np.uint8), hdr, data,
                                 np.zeros(64 * tb, np.uint8)])
            payload.append(data)
        else:
            hdr = np.zeros(64 * tb, np.uint8)
            if digits is not None:
                hdr[:52 * tb] = _time_words(digits, tb)
            data = rng.integers(0, 256, 19840 * tb, dtype=np.uint8)
            fr = np.concatenate([np.zeros(64 * tb, np.uint8), np.full(32 * tb, 0xFF, np.uint8),
                                 hdr, data])
            payload.append(fr)
        frames.append(fr)
    head = rng.integers(0, 200, lead, dtype=np.uint8)
    return np.concatenate([head] + frames).tobytes(), np.concatenate(payload).tobytes()


def test_vlba_frames_headers_removed(tmp_path):
    data, pay = _track_file("VLBA", 32, 6, 1000, 8)
    r, info, got = _read(tmp_path, data, fmt="VLBA1_2-256-8-2")
    assert r.returncode == 0, r.stderr
    assert got == pay
    assert "leading bytes skipped" in r.stderr


def test_mark4_frames_read_whole(tmp_path):
    data, pay = _track_file("MKIV", 16, 5, 0, 9)
    r, info, got = _read(tmp_path, data, fmt="MKIV1_1-256-8-2")
    assert r.returncode == 0, r.stderr
    assert got == pay


def _pin_time(fmt, data, offset, check):
    """The same header through mark5access (oracle/_ref), where it was built."""
    import oracle as O
    if O.ref() is None:
        return
    mjd, sec, ns, off = O.m5_frame_time(fmt, data)
    assert off == offset and check(mjd, sec, ns), (mjd, sec, ns, off)


def test_vlba_start_time_code(tmp_path):
    """The first VLBA frame's time code (MJD mod 1000, second of day, 0.1 ms)
    in the start-timing file, each bit the majority of its track-word."""
    data, pay = _track_file("VLBA", 32, 4, 3000, 9, digits=[1, 2, 3, 4, 5, 6, 7, 8, 1, 2, 3, 4])
    r, info, got = _read(tmp_path, data, fmt="VLBA1_2-256-8-2")
    assert r.returncode == 0, r.stderr
    assert got == pay
    timing = (tmp_path / "out.bin.starttiming.txt").read_text()
    assert "First frame at byte 3000: MJD(mod 1000) 123 second 45678 + 1234 x 0.1 ms" in timing
    assert "BCD" not in r.stderr
    _pin_time("VLBA1_2-256-8-2", data, 3000, lambda mjd, sec, ns: (mjd % 1000, sec, ns) == (123, 45678, 1.234e8))


def test_mark4_start_time_code(tmp_path):
    """Mark4: year digit, day of year and time of day (12:34:56 = second
    45296); a day above 366 is reported."""
    data, pay = _track_file("MKIV", 32, 4, 0, 10, digits=[6, 1, 2, 3, 1, 2, 3, 4, 5, 6, 0, 0, 0])
    r, info, got = _read(tmp_path, data, fmt="MKIV1_2-512-8-2")
    assert r.returncode == 0, r.stderr
    timing = (tmp_path / "out.bin.starttiming.txt").read_text()
    assert "First frame at byte 0: year digit 6 day 123 second 45296" in timing
    assert "BCD" not in r.stderr
    # mark5access: MJD 51543 + 365 y + day + (y + 3) // 4 (decade 0), its frame pointer at the sync word
    _pin_time("MKIV1_2-512-8-2", data, 64 * 4,
              lambda mjd, sec, ns: (mjd, sec, ns) == (51543 + 365 * 6 + 123 + 9 // 4, 45296, 0.0))
    data, _ = _track_file("MKIV", 32, 4, 0, 10, digits=[6, 3, 9, 9, 1, 2, 3, 4, 5, 6, 0, 0, 0])
    r, _, _ = _read(tmp_path, data, fmt="MKIV1_2-512-8-2")
    assert r.returncode == 0, r.stderr
    assert "not a valid BCD time (digits 6 3 9 9 1 2 3 4 5 6 0 0 0)" in r.stderr


@pytest.mark.parametrize("fmt,nchan,nbit", [("MKIV1_2-512-8-2", 8, 2), ("VLBA1_1-512-32-2", 32, 2),
                                             ("MKIV1_1-512-64-1", 64, 1)])
def test_track_format_settings(tmp_path, fmt, nchan, nbit):
    s = _settings(tmp_path, fmt=fmt)
    assert s["source_channels"] == nchan and s["bits_per_sample"] == nbit
