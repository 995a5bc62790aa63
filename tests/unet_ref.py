"""Plain PyTorch (CPU, FP64) restatement of the learned preconditioner's U-Net
(hicar_b200/csrc/k_unet.cu), used by the GPU tests as the checker of its
forward pass and of the gradients of its backward pass.

`q` rounds a stored activation to BF16 as the device does (the device keeps
every activation tensor in BF16 and accumulates in FP32); for gradients it is
the identity (straight-through), so autograd gives the gradient of the same
network in exact arithmetic.  Tensors are (C, ny, nz, nx)."""
import torch

F = torch.nn.functional

# (cin, cout, level) of convolutions a..g
SPEC = [(16, 16, 0), (16, 32, 1), (32, 32, 2), (32, 32, 2), (32, 16, 1), (16, 16, 0), (16, 16, 0)]

# stencil offsets (dk, dj, di) of coefficients A..O
OFF = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 1), (1, 0, -1),
       (-1, 0, 1), (-1, 0, -1), (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0)]


def split(params):
    """flat FP32 parameter vector -> [(W [27][cin][cout], b [cout])] (weights then bias per conv)."""
    out, o = [], 0
    for cin, cout, _ in SPEC:
        w = params[o:o + 27 * cin * cout].reshape(27, cin, cout)
        o += 27 * cin * cout
        b = params[o:o + cout]
        o += cout
        out.append((w, b))
    assert o == params.numel()
    return out


def wt(w):
    cin, cout = w.shape[1], w.shape[2]
    return w.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2)


def q(x, on=True):
    if not on:
        return x
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


def conv(x, w, b):
    return F.conv3d(x[None], wt(w), b, padding=1)[0]


def pool(x):
    c, ny, nz, nx = x.shape
    x = F.pad(x, (0, nx % 2, 0, 0, 0, ny % 2))
    return 0.25 * (x[:, 0::2, :, 0::2] + x[:, 1::2, :, 0::2] + x[:, 0::2, :, 1::2] + x[:, 1::2, :, 1::2])


def up(x, ny, nx):
    return x.repeat_interleave(2, dim=1).repeat_interleave(2, dim=3)[:, :ny, :, :nx]


def forward(params, x0, bf16=True):
    """O_0 (ny, nz, nx) of features x0 (16, ny, nz, nx)."""
    (wa, ba), (wb, bb), (wc, bc), (wd, bd), (we, be), (wf, bf), (wg, bg) = [
        (q(w, bf16), b) for w, b in split(params)]
    ny, nz, nx = x0.shape[1:]
    ny1, nx1 = (ny + 1) // 2, (nx + 1) // 2
    e0 = q(torch.relu(conv(x0, wa, ba)), bf16)
    p1 = q(pool(e0), bf16)
    e1 = q(torch.relu(conv(p1, wb, bb)), bf16)
    p2 = q(pool(e1), bf16)
    e2 = q(torch.relu(conv(p2, wc, bc)), bf16)
    f2 = q(torch.relu(conv(e2, wd, bd)), bf16)
    u1 = q(up(f2, ny1, nx1) + e1, bf16)
    d1 = q(torch.relu(conv(u1, we, be)), bf16)
    u0 = q(up(d1, ny, nx), bf16)
    d0 = q(torch.relu(conv(u0, wf, bf) + e0), bf16)
    return (conv(d0, wg, bg) + x0)[0]


def apply_interior(coefs, x):
    """A x on the interior cells (zero outside); coefs (15, ny, nz, nx), x (ny, nz, nx)."""
    ny, nz, nx = x.shape
    xp = F.pad(x, (1, 1, 1, 1, 1, 1))
    y = torch.zeros_like(x)
    for s, (dk, dj, di) in enumerate(OFF):
        y = y + coefs[s] * xp[1 + dj:1 + dj + ny, 1 + dk:1 + dk + nz, 1 + di:1 + di + nx]
    return y


def loss_and_grad(params, x0, target, bf16=True):
    p = params.clone().requires_grad_(True)
    o = forward(p, x0, bf16)
    loss = ((o - target) ** 2).mean()
    loss.backward()
    return float(loss.detach()), p.grad.detach(), o.detach()


def residual_loss_and_grad(params, x0, coefs, rhat, bf16=True):
    """mean((A z - rhat)^2), z = O_0 / coef_A, and its parameter gradient."""
    p = params.clone().requires_grad_(True)
    o = forward(p, x0, bf16)
    res = apply_interior(coefs, o / coefs[0]) - rhat
    loss = (res ** 2).mean()
    loss.backward()
    return float(loss.detach()), p.grad.detach()
