"""The decode entry point that allocates no device memory.

swsgpu_unpack_device_noalloc serves callers that cannot allocate device
memory where they decode (an acquisition thread that must not stall on the
synchronisation cudaMalloc/cudaFree can imply, an application whose memory
manager owns all device allocations, a process that reserves its memory once).
It keeps its scratch in a fixed array inside the library, shared by all calls,
so these tests call it twice in a row on different streams of data -- the
second call must not see the first call's scratch contents -- and compare each
result bit for bit with the allocating entry point, swsgpu_unpack_device.
"""
import numpy as np
import pytest

from swspec_b200 import synth

pytestmark = pytest.mark.gpu


def _both(gpu, lay, raw: bytes, chan: int, nsamp: int, payload_offset: int = 0):
    import torch
    d = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda()
    ref = torch.full((nsamp,), 7.0, dtype=torch.float32, device="cuda")
    got = torch.full((nsamp,), -7.0, dtype=torch.float32, device="cuda")
    n_ref = gpu.unpack_device(lay, d.data_ptr(), d.numel(), payload_offset, chan, nsamp,
                              ref.data_ptr())
    n_got = gpu.unpack_device_noalloc(lay, d.data_ptr(), d.numel(), payload_offset, chan, nsamp,
                                      got.data_ptr())
    return ref.cpu().numpy(), n_ref, got.cpu().numpy(), n_got


def test_noalloc_matches_allocating_entry_on_two_calls(gpu):
    # call 1: Mark5B 16 ch x 2 bit, frame 1 ends in fill pattern (blanked)
    rng = np.random.default_rng(31)
    raw = bytearray(synth.mark5b_stream(rng.standard_normal((16, 2500 * 4)), 2, 1024))
    base = 10016 + 16
    raw[base + 7000: base + 10000] = bytes.fromhex("44332211") * 750
    lay1 = gpu.layout("mark5b", 16, 2)
    ref1, nr1, got1, ng1 = _both(gpu, lay1, bytes(raw), 5, 2500 * 3)
    assert np.array_equal(got1.view(np.uint32), ref1.view(np.uint32))
    assert ng1 == nr1 < 2500 * 3
    # call 2: VDIF 8-bit, no blanking, more samples
    x = rng.standard_normal(8000 * 5)
    payload = synth.pack_codes(synth.quantize_vdif_8bit(x, 24.0)[None, :], 8)
    vraw = synth.vdif_frames(payload, 8000, 1, 8, 8000)
    lay2 = gpu.layout("vdif:8000", 1, 8)
    ref2, nr2, got2, ng2 = _both(gpu, lay2, vraw, 0, 8000 * 4)
    assert np.array_equal(got2.view(np.uint32), ref2.view(np.uint32))
    assert ng2 == nr2 == 8000 * 4


def test_noalloc_rejects_more_frames_than_its_scratch_holds(gpu):
    import torch
    lib = gpu.lib()
    lay = gpu.layout("mark5b", 16, 2)
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    max_frames = 16384  # SWSGPU_NOALLOC_MAX_FRAMES
    nsamp = 2500 * (max_frames + 1)
    import ctypes as C
    nv = C.c_int64()
    rc = lib.swsgpu_unpack_device_noalloc(C.byref(lay), d.data_ptr(), 2 ** 40, 0, 0, nsamp,
                                          out.data_ptr(), C.byref(nv), None)
    assert rc == -6  # SWSGPU_ETOOBIG


def test_noalloc_allocates_nothing_after_the_warm_up_call(gpu):
    """After one warm-up call per device (which loads the scratch array),
    further calls leave the device's free memory unchanged."""
    import torch
    rng = np.random.default_rng(5)
    raw = synth.mark5b_stream(rng.standard_normal((16, 2500 * 6)), 2, 1024)
    d = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda()
    out = torch.empty(2500 * 5, dtype=torch.float32, device="cuda")
    lay = gpu.layout("mark5b", 16, 2)
    gpu.unpack_device_noalloc(lay, d.data_ptr(), d.numel(), 0, 3, 2500 * 5, out.data_ptr())
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for chan in range(16):
        gpu.unpack_device_noalloc(lay, d.data_ptr(), d.numel(), 0, chan, 2500 * 5, out.data_ptr())
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0

