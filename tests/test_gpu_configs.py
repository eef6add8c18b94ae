"""Parity at the stated benchmark configurations, at their full sizes and
inputs (tests/workloads.py), every transform checked: the CUDA path through
the C ABI against the FP64 oracle on identical storage-rounded inputs, the
error norms reduced in FP64 on the GPU (mcfftErrorNorms) per transform.

Tolerances (rel-L2 = ||y - y_ref|| / ||y_ref|| of each transform):
  plain FP16 form   <= 1e-3
  split hi+lo form  <= 2e-6  (round trips: <= 4e-6, two transforms)
The GPU norm reduction itself is checked against the oracle's long-double
reduction first.  Outputs are NaN-poisoned before every exec.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests import workloads as W  # noqa: E402
from tests.gpu_util import from_device, rounded, to_device  # noqa: E402

PLAIN_TOL = 1e-3
SPLIT_TOL = 2e-6


def _ref_device(ref: np.ndarray) -> torch.Tensor:
    flat = np.ascontiguousarray(ref.reshape(-1), dtype=np.complex128)
    return torch.from_numpy(flat.view(np.float64)).cuda()


def _exec(plan, xd, out_f16, direction=mc.FORWARD):
    info = plan.info()
    out = torch.empty(info.elements, dtype=torch.complex32 if out_f16 else torch.complex64,
                      device="cuda")
    out.view(torch.uint8).fill_(0xFF)  # NaN poison
    plan.exec_ptr(xd.data_ptr(), out.data_ptr(), direction, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.check_status()
    return out, info


def _norms(y, out_f16, ref, seg_off, scales):
    rd = _ref_device(ref)
    res = mc.error_norms(y.data_ptr(), out_f16, rd.data_ptr(), seg_off, scales,
                         torch.cuda.current_stream().cuda_stream)
    del rd
    return res


def _worst(res):
    return max(r["rel_l2"] for r in res), max(r["max_rel"] for r in res)


# ------------------------------------------------------------------ checker


@pytest.mark.parametrize("f16", [True, False])
def test_gpu_norms_match_oracle(f16):
    """mcfftErrorNorms against the oracle's long-double norms and the
    reference harness metric, on uneven segments with per-segment scales."""
    rng = np.random.default_rng(5)
    sizes = [1, 17, 4096, 5000, 65536 + 3]
    seg_off = np.concatenate([[0], np.cumsum(sizes)]).tolist()
    scales = [0, -3, 2, -10, 5]
    total = seg_off[-1]
    y = rng.standard_normal(total) + 1j * rng.standard_normal(total)
    yr = rounded(y, f16)
    ref = yr.copy()
    for i, s in enumerate(scales):
        a, b = seg_off[i], seg_off[i + 1]
        ref[a:b] = yr[a:b] * 2.0 ** s + 1e-3 * (rng.standard_normal(b - a) + 1j * rng.standard_normal(b - a))
    yd = to_device(y, f16)
    res = _norms(yd, f16, ref, seg_off, scales)
    for i, s in enumerate(scales):
        a, b = seg_off[i], seg_off[i + 1]
        rel, mx = oracle.error_norms(yr[a:b] * 2.0 ** s, ref[a:b])
        ge = oracle.get_error(yr[a:b] * 2.0 ** s, ref[a:b])
        assert abs(res[i]["rel_l2"] - rel) <= 1e-12 * max(rel, 1e-300) + 1e-15, (i, res[i], rel)
        assert abs(res[i]["max_rel"] - mx) <= 1e-12 * max(mx, 1e-300) + 1e-15, (i, res[i], mx)
        assert abs(res[i]["get_error"] - ge) <= 1e-9 * max(ge, 1e-300) + 1e-15, (i, res[i], ge)


# ----------------------------------------------------------- c2: 2^20 x 64


@pytest.mark.parametrize("form", ["plain", "split", "split_fp32"])
def test_c2_every_transform(form):
    dims, batch, seed, _ = W.CONFIGS["c2"]
    n = dims[0]
    x = W.uniform((batch, n), seed)
    # FP16 input in the plain form and the split form with FLAG_INPUT_F16;
    # FP32 input in the split form's FP32 in / FP32 out case
    in16 = form != "split_fp32"
    xr = rounded(x, in16)
    xd = to_device(x, in16)
    del x
    if form == "plain":
        p = mc.Plan(dims, batch, mc.PREC_FP16)
    elif form == "split":
        p = mc.Plan(dims, batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16)
    else:
        p = mc.Plan(dims, batch, mc.PREC_SPLIT)
    with p:
        y, info = _exec(p, xd, form == "plain")
    ref = oracle.fft1d(xr)
    del xr
    seg = [i * n for i in range(batch + 1)]
    # the plain form's output carries 2^scale_log2: undo it before comparing
    res = _norms(y, form == "plain", ref, seg, [-info.scale_log2] * batch)
    rel, mx = _worst(res)
    assert rel < (PLAIN_TOL if form == "plain" else SPLIT_TOL), (rel, mx)
    # the GPU reduction agrees with the CPU one on a transform
    rel0, _ = oracle.error_norms(from_device(y[:n]) * 2.0 ** -info.scale_log2, ref[0])
    assert abs(rel0 - res[0]["rel_l2"]) <= 1e-9 * rel0


# ------------------------------------------------------- c3: 1024^2 x 16


@pytest.mark.parametrize("variant", ["uniform", "wide"])
@pytest.mark.parametrize("form", ["plain", "split"])
def test_c3_every_transform(form, variant):
    dims, batch, seed, _ = W.CONFIGS["c3"]
    gen = W.uniform if variant == "uniform" else W.wide_range
    x = gen((batch,) + dims, seed)
    f16 = form == "plain"  # split: FP32 input split into hi + lo
    xr = rounded(x, f16)
    xd = to_device(x, f16)
    with mc.Plan(dims, batch, mc.PREC_FP16 if f16 else mc.PREC_SPLIT) as p:
        y, info = _exec(p, xd, f16)
    ref = oracle.fftnd(xr, list(dims))
    npt = int(np.prod(dims))
    res = _norms(y, f16, ref, [i * npt for i in range(batch + 1)], [-info.scale_log2] * batch)
    rel, mx = _worst(res)
    assert rel < (PLAIN_TOL if f16 else SPLIT_TOL), (rel, mx)


# ----------------------------------------------------------- c4: 256^3


def test_c4_split_forward_inverse_roundtrip():
    dims, _, seed, _ = W.CONFIGS["c4"]
    x = W.plane_waves(seed=seed)
    xr = rounded(x, False)
    xd = to_device(x, False)
    npt = int(np.prod(dims))
    with mc.Plan(dims, 1, mc.PREC_SPLIT) as p:
        y, _ = _exec(p, xd, False)
        z, _ = _exec(p, y, False, direction=mc.INVERSE)
    ref = oracle.fftnd(xr, list(dims))
    fwd = _norms(y, False, ref, [0, npt], None)[0]
    assert fwd["rel_l2"] < SPLIT_TOL, fwd
    # inverse of exactly what the forward wrote
    ref_inv = oracle.fftnd(from_device(y).reshape((1,) + dims), list(dims), sign=+1)
    inv = _norms(z, False, ref_inv, [0, npt], None)[0]
    assert inv["rel_l2"] < SPLIT_TOL, inv
    # round trip: inverse(forward(x)) / N against x
    rt = _norms(z, False, xr * npt, [0, npt], None)[0]
    assert rt["rel_l2"] < 2 * SPLIT_TOL, rt


def test_c4_plain_forward():
    dims, _, seed, _ = W.CONFIGS["c4"]
    x = W.plane_waves(seed=seed)
    xr = rounded(x, True)
    xd = to_device(x, True)
    with mc.Plan(dims, 1, mc.PREC_FP16) as p:
        y, info = _exec(p, xd, True)
    ref = oracle.fftnd(xr, list(dims))
    res = _norms(y, True, ref, [0, int(np.prod(dims))], [-info.scale_log2])[0]
    assert res["rel_l2"] < PLAIN_TOL, res


# ------------------------------------------------------ c5: uneven batch


def _uneven_ref(shapes, offs, xr):
    """The oracle per transform, batched over equal shapes."""
    ref = np.empty_like(xr)
    by_shape = {}
    for i, s in enumerate(shapes):
        by_shape.setdefault(s, []).append(i)
    for s, idx in by_shape.items():
        npt = int(np.prod(s))
        stack = np.stack([xr[offs[i]:offs[i] + npt] for i in idx]).reshape((len(idx),) + s)
        out = oracle.fftnd(stack, list(s)).reshape(len(idx), npt)
        for j, i in enumerate(idx):
            ref[offs[i]:offs[i] + npt] = out[j]
    return ref


@pytest.mark.parametrize("order", ["draw", "sorted"])
@pytest.mark.parametrize("form", ["plain", "split"])
def test_c5_every_transform(form, order):
    shapes, offs, total = W.uneven_layout(order)
    x = W.uneven_input(total)
    xr = rounded(x, True)
    xd = to_device(x, True)
    descs = [(s, 1, o, o) for s, o in zip(shapes, offs)]
    if form == "plain":
        p = mc.Plan(descs=descs, precision=mc.PREC_FP16)
    else:
        p = mc.Plan(descs=descs, precision=mc.PREC_SPLIT, flags=mc.FLAG_INPUT_F16)
    with p:
        y, info = _exec(p, xd, form == "plain")
        assert info.launches == 1
    ref = _uneven_ref(shapes, offs, xr)
    seg = offs + [total]
    scales = [int(np.log2(np.prod(s))) if form == "plain" else 0 for s in shapes]
    res = _norms(y, form == "plain", ref, seg, scales)
    rel, mx = _worst(res)
    assert rel < (PLAIN_TOL if form == "plain" else SPLIT_TOL), (rel, mx)
