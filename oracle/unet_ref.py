"""CPU checker (test infrastructure) of the learned pseudo-Hessian U-Net.

The reference has no learned component, so this is not a restatement of
reference code: it is the same network as denise-sh_b200/dsh/nn.py written
with PyTorch CPU operators in FP32, with the GPU path's BF16 rounding points
(inputs, weights, every stored activation) reproduced, so the GPU forward
pass and the gradients of its hand-written backward pass can be compared
with CPU autograd.  Only tests import it.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

BASE = 32


_ROUND = True


def _bf(t):
    return t.to(torch.bfloat16).to(torch.float32) if _ROUND else t


class _RoundST(torch.autograd.Function):
    """BF16 rounding in the forward pass, identity in the backward pass."""

    @staticmethod
    def forward(ctx, x):
        return _bf(x)

    @staticmethod
    def backward(ctx, g):
        return g


class _RoundGrad(torch.autograd.Function):
    """Identity in the forward pass, BF16 rounding of the gradient in the
    backward pass (the GPU path feeds BF16 output gradients to its GEMMs)."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        return _bf(g)


def _conv(x, w, b, cin, cout):
    """x [B][cin][H][W]; w [cout][9*cin] tap-major (k = tap*cin + c, tap = (dy+1)*3 + (dx+1))."""
    wk = w.view(cout, 3, 3, cin).permute(0, 3, 1, 2)           # [cout][cin][ky][kx]
    z = _RoundGrad.apply(F.conv2d(x, _RoundST.apply(wk), b, padding=1))
    return _RoundST.apply(F.relu(z))


def forward(state, x_nhwc, B, H, W, rounding=True):
    """state: dict of numpy FP32 parameters (UNet.state()); x_nhwc [B*H*W][8]
    (already BF16-representable).  Returns (prediction [B*H*W], parameter tensors).
    rounding=False gives the same network in plain FP32 (no BF16 rounding)."""
    global _ROUND
    _ROUND = rounding
    params = {k: torch.tensor(v, dtype=torch.float32, requires_grad=True) for k, v in state.items()}
    c = [BASE, 2 * BASE, 4 * BASE, 8 * BASE]
    x = torch.tensor(np.asarray(x_nhwc, np.float32)).view(B, H, W, -1).permute(0, 3, 1, 2)
    k = 0

    def conv(inp, cin, cout):
        nonlocal k
        out = _conv(inp, params[f"w{k}"], params[f"b{k}"], cin, cout)
        k += 1
        return out

    enc = []
    inp, cin = x, x.shape[1]
    for l in range(4):
        a = conv(inp, cin, c[l])
        bb = conv(a, c[l], c[l])
        enc.append(bb)
        if l < 3:
            inp, cin = F.max_pool2d(bb, 2), c[l]
    low = enc[3]
    for l in (2, 1, 0):
        u = F.interpolate(low, scale_factor=2, mode="nearest")
        d = conv(u, c[l + 1], c[l])
        cat = torch.cat([enc[l], d], dim=1)
        d = conv(cat, 2 * c[l], c[l])
        low = conv(d, c[l], c[l])
    out = torch.einsum("bchw,c->bhw", low, params["hw"]) + params["hb"][0]
    return out.reshape(-1), params


def gradients(state, x_nhwc, B, H, W, dout, rounding=True):
    """Parameter gradients of sum(pred * dout) (weights [cout][9cin])."""
    out, params = forward(state, x_nhwc, B, H, W, rounding)
    (out * torch.tensor(np.asarray(dout, np.float32))).sum().backward()
    return out.detach().numpy(), {k: v.grad.numpy() for k, v in params.items()}
