"""Repeated execs replay a captured CUDA graph (from the second exec on the
same buffers and direction): the replayed results must equal the first,
directly launched exec's, for pass-by-pass plans (plain and split) and for
the batch queue; changing buffers or direction must not reuse a graph of
other buffers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from tests.gpu_util import from_device, rand_complex, to_device  # noqa: E402


def _execs(plan, xd, outs, directions):
    res = []
    for out, d in zip(outs, directions):
        out.view(torch.uint8).fill_(0xFF)
        plan.exec_ptr(xd.data_ptr(), out.data_ptr(), d, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        plan.check_status()
        res.append(from_device(out).copy())
    return res


@pytest.mark.parametrize("prec,shape,batch", [(mc.PREC_FP16, (1 << 16,), 4),
                                              (mc.PREC_SPLIT, (1 << 16,), 4),
                                              (mc.PREC_FP16, (256, 512), 2)])
def test_graph_replay_matches_direct(prec, shape, batch):
    n = int(np.prod(shape))
    x = rand_complex((batch, n), seed=5)
    f16 = True
    flags = mc.FLAG_INPUT_F16 if prec == mc.PREC_SPLIT else mc.FLAG_NONE
    xd = to_device(x, f16)
    odt = torch.complex64 if prec == mc.PREC_SPLIT else torch.complex32
    o1 = torch.empty(n * batch, dtype=odt, device="cuda")
    o2 = torch.empty(n * batch, dtype=odt, device="cuda")
    with mc.Plan(shape, batch, prec, flags) as p:
        seq = [(o1, mc.FORWARD)] * 4 + [(o2, mc.FORWARD)] * 3 + [(o1, mc.INVERSE)] * 3 + [(o1, mc.FORWARD)]
        r = _execs(p, xd, [s[0] for s in seq], [s[1] for s in seq])
    fwd = [r[i] for i, s in enumerate(seq) if s[1] == mc.FORWARD]
    inv = [r[i] for i, s in enumerate(seq) if s[1] == mc.INVERSE]
    for y in fwd[1:]:
        assert np.array_equal(y, fwd[0])
    for y in inv[1:]:
        assert np.array_equal(y, inv[0])
    assert not np.array_equal(fwd[0], inv[0])


def test_graph_replay_batch_queue():
    descs, off = [], 0
    for shape, count in (((256,), 3), ((8192,), 2), ((128, 256), 1)):
        nn = int(np.prod(shape))
        for _ in range(count):
            descs.append((shape, 1, off, off))
            off += nn
    x = rand_complex((off,), seed=9)
    xd = to_device(x, True)
    out = torch.empty(off, dtype=torch.complex32, device="cuda")
    with mc.Plan(descs=descs, precision=mc.PREC_FP16) as p:
        assert p.info().launches == 1
        r = _execs(p, xd, [out] * 4, [mc.FORWARD] * 4)
    for y in r[1:]:
        assert np.array_equal(y, r[0])


@pytest.mark.parametrize("prec,shape,batch", [(mc.PREC_FP16, (64, 128, 256), 2),
                                              (mc.PREC_SPLIT, (256, 512), 3),
                                              (mc.PREC_FP16, (1 << 24,), 1)])
def test_dependent_launch_matches_stream_order(prec, shape, batch, monkeypatch):
    """A plan's later passes start by programmatic dependent launch (their
    setup overlapping the previous pass); with MCFFT_PDL=0 every pass runs
    in plain stream order.  Both must give identical outputs, directly and
    replayed from the captured graph (3D: three passes; 1D 2^24: three
    passes, the last one per transform)."""
    f16 = prec == mc.PREC_FP16
    x = rand_complex((batch,) + shape, seed=len(shape) + batch)
    xd = to_device(x, f16)
    n = int(np.prod(shape)) * batch
    res = {}
    for pdl in ("1", "0"):
        monkeypatch.setenv("MCFFT_PDL", pdl)
        monkeypatch.setenv("MCFFT_AUTOTUNE", "0")
        with mc.Plan(shape, batch, prec) as p:
            assert p.info().num_passes >= 2
            outs = [torch.empty(n, dtype=torch.complex32 if f16 else torch.complex64, device="cuda")
                    for _ in range(3)]
            res[pdl] = _execs(p, xd, [outs[0], outs[0], outs[0]], [mc.FORWARD] * 3)
    for y in res["1"] + res["0"]:
        assert np.array_equal(y, res["1"][0])
