"""GPU parity of the phase-cal extractor library (src/IA-32/PhaseCal/PCal.cpp):
the device extractor (swsgpu_pcal_*) against the oracle's restatement of the
same classes, over calls with partial periods, a gap re-entered through
adjustSampleOffset, and the library's own known answer."""
import numpy as np
import pytest

import oracle as O
from test_oracle import _pcal_test_signal

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()


@pytest.mark.parametrize("bw,spacing,offset,kind", [(8e6, 1e6, 0, 1), (8e6, 1e6, 10000, 3),
                                                    (8e6, 1e6, 128000, 2), (16e6, 1e6, 10000, 3)])
def test_pcallib_matches_oracle(gpu, bw, spacing, offset, kind):
    rng = np.random.default_rng(int(offset) + 7)
    g = gpu.PcalExtractor(bw, spacing, offset, 11)
    o = O.PcalLib(bw, spacing, offset, 11)
    assert (g.kind, g.nbins, g.ntones) == (o.kind, o.nbins, o.ntones) and g.kind == kind
    chunks = [rng.standard_normal(n).astype(np.float32) * 3 for n in (1_000_003, 77, 2_500_000 + 13)]
    for i, x in enumerate(chunks):
        if i == 2:
            g.adjust(5_000_041)
            o.adjust(5_000_041)
        d = _dev(x)
        g.extract(d.data_ptr(), len(x))
        o.extract(x)
    tg, ng = g.final()
    to, no = o.final()
    assert ng == no == sum(len(x) for x in chunks)
    assert np.max(np.abs(tg - to)) < 1e-9 * np.max(np.abs(to)), (tg, to)
    # finalized: further extraction is refused until clear()
    with pytest.raises(gpu.SwsError, match="ESTATE"):
        g.extract(_dev(chunks[1]).data_ptr(), 77)
    g.clear()
    g.extract(_dev(chunks[1]).data_ptr(), 77)


@pytest.mark.parametrize("bw,spacing,offset", [(8e6, 1e6, 0), (8e6, 1e6, 10000)])
def test_pcallib_known_answer_on_gpu(gpu, bw, spacing, offset):
    """PCal.cpp:879-948: tone phases -90 + 5 t degrees, with a gap."""
    g = gpu.PcalExtractor(bw, spacing, offset, 0)
    n, prime = 160000, 3
    x = _pcal_test_signal(n, bw, spacing, offset, g.ntones, 0)
    y = _pcal_test_signal(n, bw, spacing, offset, g.ntones, n + prime)
    g.extract(_dev(x).data_ptr(), n)
    g.adjust(n + prime)
    g.extract(_dev(y).data_ptr(), n)
    tones, used = g.final()
    assert used == 2 * n
    first = 1 if offset == 0 else 0
    ph = np.rad2deg(np.angle(tones[first:]))
    want = -90.0 + 5.0 * np.arange(first, g.ntones)
    d = (ph - want + 180) % 360 - 180
    assert np.max(np.abs(d)) < 0.5, d
