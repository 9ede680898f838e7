"""Regenerate the golden fixtures from the reference's own mark5access.

Run in the development container, where the reference sources are present
and oracle/Makefile has compiled them into oracle/_ref/libm5ref.so:

    python tests/golden/make_golden.py

Fixtures:
  mark5b_decode.npz   framed Mark5B-1024-16-2 stream (3 frames, one with a
                      trailing fill-pattern zone) and mark5access's
                      mark5_stream_decode output for every channel.
  vdif_decode.npz     VDIF_8000-512-1-8 stream with an invalid frame, decoded.
  unpacker_pattern.npz  the byte pattern of mark5access examples/test_unpacker.c
                      (data[i] = (i%11) + 2*(i%121)) unpacked header-free as
                      Mark5B-1024-16-2 and Mark5B-1024-8-2 (mark5_unpack).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from swspec_b200 import synth  # noqa: E402


def main():
    O.build()
    assert O.ref() is not None, "oracle/_ref/libm5ref.so missing"
    rng = np.random.default_rng(20260101)
    # Mark5B with a trailing fill-pattern zone in frame 1 (payload bytes
    # 6000..10000); mark5access's blanker finds it by binary search
    spf = 2500
    sig = rng.standard_normal((16, spf * 4))
    raw = bytearray(synth.mark5b_stream(sig, 2, 1024))
    base = 10016 + 16
    raw[base + 6000: base + 10000] = bytes.fromhex("44332211") * 1000
    raw = bytes(raw)
    nsamp = spf * 3
    dec, rc = O.m5_decode("Mark5B-1024-16-2", raw, nsamp)
    np.savez_compressed(os.path.join(HERE, "mark5b_decode.npz"),
                        raw=np.frombuffer(raw, dtype=np.uint8), decoded=dec, nchan=16, nbit=2,
                        nsamp=nsamp, rc=rc)
    # VDIF 8-bit, frame 1 invalid
    x = rng.standard_normal(8000 * 3)
    payload = synth.pack_codes(synth.quantize_vdif_8bit(x, 24.0)[None, :], 8)
    vraw = synth.vdif_frames(payload, 8000, 1, 8, 8000, invalid={1})
    vdec, vrc = O.m5_decode("VDIF_8000-512-1-8", vraw, 8000 * 3)
    np.savez_compressed(os.path.join(HERE, "vdif_decode.npz"),
                        raw=np.frombuffer(vraw, dtype=np.uint8), decoded=vdec, nsamp=8000 * 3,
                        rc=vrc)
    # test_unpacker.c byte pattern, header-free unpack
    pat = np.array([(i % 11) + 2 * (i % 121) for i in range(10000)], dtype=np.uint8).tobytes()
    u16, _ = O.m5_unpack("Mark5B-1024-16-2", pat, 2500)
    u8, _ = O.m5_unpack("Mark5B-1024-8-2", pat, 5000)
    np.savez_compressed(os.path.join(HERE, "unpacker_pattern.npz"),
                        pattern=np.frombuffer(pat, dtype=np.uint8), m5b_16ch=u16, m5b_8ch=u8)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
