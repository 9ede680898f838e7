"""CPU: the C ABI library loads and exports every entry point the header declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(swsgpu_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared("swsgpu.h")
    for n in ["swsgpu_create", "swsgpu_submit", "swsgpu_wait", "swsgpu_fetch", "swsgpu_destroy",
              "swsgpu_process_device", "swsgpu_unpack_device", "swsgpu_last_error"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from swspec_b200 import gpu
    lib = gpu.lib()  # loads without a GPU
    for n in _declared("swsgpu.h"):
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", gpu.LIB_PATH], capture_output=True,
                         text=True).stdout
    for n in _declared("swsgpu.h"):
        assert re.search(rf"\bT {n}\b", out), n


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from swspec_b200 import gpu
    cfg = gpu.make_config(gpu.layout("mark5b", 16, 2), 32768)
    with pytest.raises(gpu.SwsError):
        gpu.Core(cfg)


def test_create_rejects_bad_config():
    from swspec_b200 import gpu
    cfg = gpu.make_config(gpu.layout("mark5b", 16, 2), 32768, overlap=3)
    with pytest.raises(gpu.SwsError, match="EINVAL|ENODEV"):
        gpu.Core(cfg)


def test_noalloc_source_names_no_allocation_call():
    """The allocation-free decode entry's source file calls no allocator."""
    src = open(os.path.join(ROOT, "swspec_b200", "csrc", "noalloc.cu")).read()
    code = re.sub(r"//.*", "", src)
    for name in ("cudaMalloc", "cudaMallocAsync", "cudaFree", "cudaMallocHost", "cudaMallocManaged"):
        assert not re.search(rf"\b{name}\s*\(", code), name


def test_pcal_delay_recovers_a_known_delay():
    """swsgpu_pcal_delay (m5pcal.c calcDelay, host code): tones 1 MHz apart
    with phases 2 pi f tau wrapped to (-pi, pi] give back tau in ns, and a
    band-edge cut drops the tones outside the valid band."""
    import numpy as np
    from swspec_b200 import gpu
    f = np.arange(1, 16, dtype=np.int32)
    for tau_ns in (37.0, -120.5, 0.0):
        ph = np.angle(np.exp(2j * np.pi * f * 1e6 * tau_ns * 1e-9))
        assert abs(gpu.pcal_delay(f, ph, 8.0, 20.0) - tau_ns) < 1e-9
    ph = np.angle(np.exp(2j * np.pi * f * 1e6 * 55e-9))
    ph[0] += 1.0                                        # a corrupted edge tone, excluded below
    assert abs(gpu.pcal_delay(f, ph, 8.0, 6.5) - 55.0) < 1e-9
    assert gpu.pcal_delay(f[:1], ph[:1], 8.0, 20.0) == 0.0
