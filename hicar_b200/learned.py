"""Learned preconditioner for the wind solver: host side of the tensor-core
convolutions and the 3-level U-Net (hicar_b200/csrc/k_conv.cu, k_unet.cu).

Activation tensors live in the library's "act layout" (BF16, channel groups of
8, zero halo): `to_act` / `from_act` convert (C, ny, nz, nx) float tensors to
and from it.  Convolution weights are FP32 [27][cin][cout] with tap
t = (dj+1)*9 + (dk+1)*3 + (di+1)."""
from __future__ import annotations

import ctypes as C

from . import _capi


def _torch():
    import torch
    return torch


def act_pitch(nx: int) -> int:
    return ((nx + 127) // 128) * 128 + 2


def act_empty(nx: int, ny: int, nz: int, ch: int, device="cuda"):
    """Zeroed act-layout tensor, shape (ny+2, nz+2, ch/8, PX, 8), BF16."""
    torch = _torch()
    if ch % 8:
        raise ValueError("channel count must be a multiple of 8")
    return torch.zeros((ny + 2, nz + 2, ch // 8, act_pitch(nx), 8), dtype=torch.bfloat16, device=device)


def to_act(x, device="cuda"):
    """(C, ny, nz, nx) float tensor -> act-layout BF16 tensor."""
    torch = _torch()
    ch, ny, nz, nx = x.shape
    out = act_empty(nx, ny, nz, ch, device)
    out[1:ny + 1, 1:nz + 1, :, 1:nx + 1, :] = (
        x.to(device=device, dtype=torch.float32).reshape(ch // 8, 8, ny, nz, nx).permute(2, 3, 0, 4, 1)
        .to(torch.bfloat16))
    return out


def from_act(a, nx: int):
    """act-layout tensor -> (C, ny, nz, nx) float32 tensor (same device)."""
    torch = _torch()
    ny, nz, g = a.shape[0] - 2, a.shape[1] - 2, a.shape[2]
    v = a[1:ny + 1, 1:nz + 1, :, 1:nx + 1, :].to(torch.float32)  # (ny, nz, G, nx, 8)
    return v.permute(2, 4, 0, 1, 3).reshape(g * 8, ny, nz, nx).contiguous()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def conv3(x_act, w, bias, nx, ny, nz, cin, cout, *, skip=None, mask=None, relu=False, transpose=False,
          want_out=True, want_out0=False, stream=None):
    """One tensor-core 3x3x3 convolution (transpose=True: its data-gradient form,
    cout -> cin channels).  Returns (out_act or None, out0 or None)."""
    torch = _torch()
    co = cin if transpose else cout
    out = act_empty(nx, ny, nz, co, x_act.device) if want_out else None
    out0 = torch.empty((ny, nz, nx), dtype=torch.float32, device=x_act.device) if want_out0 else None
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = _capi.load().hicarw_nn_conv3(cin, cout, nx, ny, nz, _ptr(x_act), _ptr(w), _ptr(bias), _ptr(skip),
                                      _ptr(mask), int(relu), int(transpose), _ptr(out), _ptr(out0), C.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"hicarw_nn_conv3 failed ({rc})")
    return out, out0


def conv3_wgrad(x_act, dy_act, nx, ny, nz, cin, cout, stream=None):
    """(dW [27][cin][cout], db [cout]) of one convolution, FP32."""
    torch = _torch()
    dw = torch.zeros((27, cin, cout), dtype=torch.float32, device=x_act.device)
    db = torch.zeros((cout,), dtype=torch.float32, device=x_act.device)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = _capi.load().hicarw_nn_conv3_wgrad(cin, cout, nx, ny, nz, _ptr(x_act), _ptr(dy_act), _ptr(dw), _ptr(db),
                                            C.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"hicarw_nn_conv3_wgrad failed ({rc})")
    return dw, db
