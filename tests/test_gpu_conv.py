"""GPU tests of the tensor-core 3x3x3 convolutions (k_conv.cu) against a plain
PyTorch FP64 reference on the CPU, computed from the same BF16-rounded inputs
and weights.  Tolerances: FP32-accumulated channel-0 output and weight
gradients within 1e-4 of max|ref|; BF16 outputs within BF16 rounding
(2^-8 relative) plus 1e-3 of max|ref|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
F = torch.nn.functional

PAIRS = [(16, 16), (16, 32), (32, 32), (32, 16)]


@pytest.fixture(autouse=True)
def _gpu(lib):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float64)


def _wt(w):
    """[27][cin][cout] -> torch conv3d weight (cout, cin, 3, 3, 3) over (j, k, i)."""
    cin, cout = w.shape[1], w.shape[2]
    return w.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2).contiguous()


def _ref_conv(x, w, b):
    """x (C, ny, nz, nx) -> (cout, ny, nz, nx), FP64."""
    y = F.conv3d(x[None], _wt(w), b, padding=1)
    return y[0]


def _data(cin, cout, nx, ny, nz, seed):
    g = torch.Generator().manual_seed(seed)
    x = _bf(torch.randn((cin, ny, nz, nx), generator=g, dtype=torch.float64))
    w = _bf(torch.randn((27, cin, cout), generator=g, dtype=torch.float64) * (2.0 / (27 * cin)) ** 0.5)
    b = torch.randn((cout,), generator=g, dtype=torch.float64) * 0.1
    return x, w, b


def _close_bf16(ours, ref):
    scale = float(ref.abs().max())
    err = (ours.double() - ref).abs()
    assert float((err - 4e-3 * ref.abs()).max()) <= 1e-3 * scale


@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("nx,ny,nz", [(200, 5, 4), (128, 3, 6), (260, 40, 8)])
def test_conv_forward(cin, cout, nx, ny, nz):
    from hicar_b200 import learned as L
    x, w, b = _data(cin, cout, nx, ny, nz, seed=cin * 100 + cout + nx)
    ref = _ref_conv(x, w, b)
    xa = L.to_act(x)
    out, out0 = L.conv3(xa, w.float().cuda(), b.float().cuda(), nx, ny, nz, cin, cout, want_out0=True)
    torch.cuda.synchronize()
    assert float((out0.double().cpu() - ref[0]).abs().max()) <= 1e-4 * float(ref.abs().max())
    _close_bf16(L.from_act(out, nx).cpu(), ref)
    # the halo and the x padding stay zero
    o = out.float().cpu()
    assert not o[0].any() and not o[-1].any() and not o[:, 0].any() and not o[:, -1].any()
    assert not o[:, :, :, 0].any() and not o[:, :, :, nx + 1:].any()


def test_conv_epilogue_skip_relu_mask():
    from hicar_b200 import learned as L
    cin, cout, nx, ny, nz = 16, 16, 150, 4, 3
    x, w, b = _data(cin, cout, nx, ny, nz, seed=7)
    g = torch.Generator().manual_seed(8)
    skip = _bf(torch.randn((cout, ny, nz, nx), generator=g, dtype=torch.float64))
    mask = _bf(torch.randn((cout, ny, nz, nx), generator=g, dtype=torch.float64))
    ref = torch.where(mask > 0, torch.relu(_ref_conv(x, w, b) + skip), torch.zeros(()).double())
    out, _ = L.conv3(L.to_act(x), w.float().cuda(), b.float().cuda(), nx, ny, nz, cin, cout, skip=L.to_act(skip),
                     mask=L.to_act(mask), relu=True)
    _close_bf16(L.from_act(out, nx).cpu(), ref)


@pytest.mark.parametrize("cin,cout", PAIRS)
def test_conv_data_gradient(cin, cout):
    """transpose=True is the data gradient: dx = conv^T(dy)."""
    from hicar_b200 import learned as L
    nx, ny, nz = 170, 4, 5
    x, w, _ = _data(cin, cout, nx, ny, nz, seed=11 + cin + cout)
    g = torch.Generator().manual_seed(12)
    dy = _bf(torch.randn((cout, ny, nz, nx), generator=g, dtype=torch.float64))
    ref = F.conv_transpose3d(dy[None], _wt(w), padding=1)[0]
    out, out0 = L.conv3(L.to_act(dy), w.float().cuda(), None, nx, ny, nz, cin, cout, transpose=True,
                        want_out0=True)
    assert float((out0.double().cpu() - ref[0]).abs().max()) <= 1e-4 * float(ref.abs().max())
    _close_bf16(L.from_act(out, nx).cpu(), ref)


@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("nx,ny,nz", [(200, 5, 4), (300, 13, 7)])
def test_conv_weight_gradient(cin, cout, nx, ny, nz):
    from hicar_b200 import learned as L
    x, w, _ = _data(cin, cout, nx, ny, nz, seed=21 + cin + cout)
    g = torch.Generator().manual_seed(22)
    dy = _bf(torch.randn((cout, ny, nz, nx), generator=g, dtype=torch.float64))
    wt = _wt(w).requires_grad_(True)
    bt = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    (F.conv3d(x[None], wt, bt, padding=1)[0] * dy).sum().backward()
    ref_w = wt.grad.permute(2, 3, 4, 1, 0).reshape(27, cin, cout)
    dw, db = L.conv3_wgrad(L.to_act(x), L.to_act(dy), nx, ny, nz, cin, cout)
    dw, db = dw.double().cpu(), db.double().cpu()
    assert float((dw - ref_w).abs().max()) <= 1e-4 * float(ref_w.abs().max())
    assert float((db - bt.grad).abs().max()) <= 1e-4 * float(bt.grad.abs().max())


def test_act_layout_round_trip():
    from hicar_b200 import learned as L
    x = torch.randn((16, 3, 4, 130))
    a = L.to_act(x)
    assert a.shape == (5, 6, 2, L.act_pitch(130), 8)
    np.testing.assert_array_equal(L.from_act(a, 130).cpu().numpy(), x.to(torch.bfloat16).float().numpy())
