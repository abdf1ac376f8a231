"""Learned pseudo-Hessian preconditioner: a 4-level U-Net whose every
convolution, pooling, activation, loss and optimiser step runs in the
in-tree CUDA library ``libdsh_nn.so`` (include/dsh_nn.h): 3x3 convolutions
are im2col + a tcgen05/TMA BF16 GEMM with FP32 accumulation in tensor
memory.  PyTorch only provides device memory and the stream.

Network (NHWC, H and W divisible by 8):
    enc1 conv(8->32) conv(32->32) | pool | enc2 conv(32->64) conv(64->64) | pool
    enc3 conv(64->128) conv(128->128) | pool | bottom conv(128->256) conv(256->256)
    up + conv(256->128), concat enc3, conv(256->128) conv(128->128)
    up + conv(128->64),  concat enc2, conv(128->64)  conv(64->64)
    up + conv(64->32),   concat enc1, conv(64->32)   conv(32->32)
    head 1x1 conv(32->1)
3x3 convolutions are zero-padded and followed by ReLU; weights are FP32
masters with BF16 operand copies, activations BF16, gradients FP32.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NN_LIB_PATH = os.path.join(PKG_DIR, "libdsh_nn.so")
BASE = 32
RED_BLOCKS = 296     # DSH_NN_RED_BLOCKS: row chunks of the fixed-order gradient reductions
IN_CH = 8            # 4 input maps padded to 8 channels (72-element rows, 16-byte aligned)

_nn = None


def nnlib() -> C.CDLL:
    global _nn
    if _nn is None:
        if not os.path.exists(NN_LIB_PATH):
            raise FileNotFoundError(f"{NN_LIB_PATH} not built (make -C denise-sh_b200/csrc)")
        L = C.CDLL(NN_LIB_PATH)
        v, i, ll, f = C.c_void_p, C.c_int, C.c_longlong, C.c_float
        L.dsh_nn_gemm.argtypes = [i, i, i, v, ll, v, ll, v, v, ll, v, i, i, v, i, v, v]
        L.dsh_nn_set_wait_limit.argtypes = [ll]
        L.dsh_nn_im2col.argtypes = [v, i, i, i, i, v, ll, v]
        L.dsh_nn_im2col_t.argtypes = [v, i, i, i, i, v, ll, v]
        L.dsh_nn_transpose.argtypes = [v, ll, i, v, ll, v]
        L.dsh_nn_prep_weights.argtypes = [v, i, i, v, ll, v, ll, v]
        L.dsh_nn_to_bf16.argtypes = [v, v, ll, v]
        L.dsh_nn_relu_bwd.argtypes = [v, v, v, v, ll, v]
        L.dsh_nn_add.argtypes = [v, v, ll, v]
        L.dsh_nn_maxpool_fwd.argtypes = [v, i, i, i, i, v, v, v]
        L.dsh_nn_maxpool_bwd.argtypes = [v, v, i, i, i, i, v, v]
        L.dsh_nn_upsample_fwd.argtypes = [v, i, i, i, i, v, v]
        L.dsh_nn_upsample_bwd.argtypes = [v, i, i, i, i, v, v]
        L.dsh_nn_concat.argtypes = [v, i, v, i, ll, v, v]
        L.dsh_nn_split.argtypes = [v, i, i, ll, v, v, v]
        L.dsh_nn_head_fwd.argtypes = [v, ll, i, v, v, v, v]
        L.dsh_nn_head_bwd.argtypes = [v, v, ll, i, v, v, v, v, v, v]
        L.dsh_nn_colsum.argtypes = [v, ll, i, v, v, v]
        L.dsh_nn_mse.argtypes = [v, v, v, ll, f, v, v, v]
        L.dsh_nn_adam.argtypes = [v, v, v, v, i, i, i, f, f, f, f, i, v]
        _nn = L
    return _nn


class NNError(RuntimeError):
    pass


def _ck(rc, what):
    if rc != 0:
        raise NNError(f"{what}: error {rc}")


def _p(t):
    return None if t is None else t.data_ptr()


def _rup(x, m):
    return (x + m - 1) // m * m


def set_wait_limit(polls: int = 0):
    """Poll limit of the tensor-core GEMM's mbarrier waits (0 = default);
    an expired wait is reported through Ctx.check (DSH_NN_ERR_TIMEOUT)."""
    _ck(nnlib().dsh_nn_set_wait_limit(int(polls)), "dsh_nn_set_wait_limit")


class Ctx:
    """Stream, error word and scratch shared by the layers."""

    def __init__(self, torch, device="cuda"):
        self.torch = torch
        self.device = device
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.stream = None
        self._ws = {}

    @property
    def st(self):
        return self.stream

    def scratch(self, name, numel, dtype):
        t = self._ws.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = self.torch.empty(int(numel * 1.0), dtype=dtype, device=self.device)
            self._ws[name] = t
        return t[:numel]

    def gemm(self, M, N, K, A, lda, B, ldb, c32=None, c16=None, ldc=None, bias=None, relu=False, splits=1,
             accumulate=False):
        torch = self.torch
        ldc = ldc or N
        part = None
        if splits > 1 or accumulate:
            part = self.scratch("part", max(splits, 1) * M * ldc, torch.float32)
        _ck(nnlib().dsh_nn_gemm(M, N, K, _p(A), lda, _p(B), ldb, _p(c32), _p(c16), ldc, _p(bias), int(relu),
                                splits, _p(part), int(accumulate), _p(self.err), self.st), "dsh_nn_gemm")

    def check(self):
        self.torch.cuda.synchronize()
        e = int(self.err.item())
        if e:
            raise NNError(f"tensor-core GEMM reported {e} (a bounded wait expired)")


class Conv3x3:
    """3x3 same-padded convolution + ReLU on the tensor cores."""

    def __init__(self, ctx, cin, cout, rng):
        torch = ctx.torch
        self.ctx, self.cin, self.cout = ctx, cin, cout
        self.K = 9 * cin
        self.ldk = _rup(self.K, 8)
        self.ldf = _rup(9 * cout, 8)
        std = math.sqrt(2.0 / self.K)
        w = (rng.standard_normal((cout, self.K)) * std).astype(np.float32)
        self.w = torch.from_numpy(w).to(ctx.device)
        self.b = torch.zeros(cout, dtype=torch.float32, device=ctx.device)
        self.wb = torch.zeros(cout * self.ldk, dtype=torch.bfloat16, device=ctx.device)
        self.wf = torch.zeros(cin * self.ldf, dtype=torch.bfloat16, device=ctx.device)
        self.gwt = torch.zeros(self.K * cout, dtype=torch.float32, device=ctx.device)    # [9cin][cout]
        self.gb = torch.zeros(cout, dtype=torch.float32, device=ctx.device)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.prep()

    def prep(self):
        _ck(nnlib().dsh_nn_prep_weights(_p(self.w), self.cout, self.cin, _p(self.wb), self.ldk, _p(self.wf), self.ldf,
                                        self.ctx.st), "prep_weights")

    def forward(self, x, B, H, W, y):
        """x bf16 [P][cin] -> y bf16 [P][cout] (ReLU applied)."""
        ctx = self.ctx
        P = B * H * W
        col = ctx.scratch("col", P * self.ldk, ctx.torch.bfloat16)
        _ck(nnlib().dsh_nn_im2col(_p(x), B, H, W, self.cin, _p(col), self.ldk, ctx.st), "im2col")
        ctx.gemm(P, self.cout, self.K, col, self.ldk, self.wb, self.ldk, c16=y, bias=self.b, relu=True)

    def backward(self, x, y, dy, B, H, W, dx=None):
        """dy float [P][cout] (gradient of the ReLU output, overwritten) ->
        weight / bias gradients accumulated, dx float [P][cin] if given."""
        ctx, torch = self.ctx, self.ctx.torch
        P = B * H * W
        dz = ctx.scratch("dz16", P * self.cout, torch.bfloat16)
        _ck(nnlib().dsh_nn_relu_bwd(_p(dy), _p(y), _p(dz), _p(dy), P * self.cout, ctx.st), "relu_bwd")
        red = ctx.scratch("red", RED_BLOCKS * (self.cout + 1), torch.float32)
        _ck(nnlib().dsh_nn_colsum(_p(dy), P, self.cout, _p(self.gb), _p(red), ctx.st), "colsum")
        # weight gradient (transposed): colT [9cin][P] . dzT [cout][P]^T, split over P
        ldp = _rup(P, 8)                      # 16-byte row pitch for the tensor-map operands
        colT = ctx.scratch("colT", self.K * ldp, torch.bfloat16)
        _ck(nnlib().dsh_nn_im2col_t(_p(x), B, H, W, self.cin, _p(colT), ldp, ctx.st), "im2col_t")
        dzT = ctx.scratch("dzT", self.cout * ldp, torch.bfloat16)
        _ck(nnlib().dsh_nn_transpose(_p(dz), P, self.cout, _p(dzT), ldp, ctx.st), "transpose")
        splits = max(1, min(64, P // 8192))
        ctx.gemm(self.K, self.cout, P, colT, ldp, dzT, ldp, c32=self.gwt, splits=splits, accumulate=True)
        if dx is not None:
            col = ctx.scratch("col", P * self.ldf, torch.bfloat16)
            _ck(nnlib().dsh_nn_im2col(_p(dz), B, H, W, self.cout, _p(col), self.ldf, ctx.st), "im2col")
            ctx.gemm(P, self.cin, 9 * self.cout, col, self.ldf, self.wf, self.ldf, c32=dx)

    def params(self):
        return [(self.w, self.mw, self.vw, self.gwt, self.cout, self.K, 1), (self.b, self.mb, self.vb, self.gb, 1,
                                                                          self.cout, 0)]

    def zero_grad(self):
        self.gwt.zero_()
        self.gb.zero_()


class UNet:
    """The pseudo-Hessian U-Net on one device; buffers sized for (B, H, W)."""

    def __init__(self, torch, seed=0, device="cuda"):
        self.torch = torch
        self.ctx = Ctx(torch, device)
        rng = np.random.default_rng(seed)
        c = [BASE, 2 * BASE, 4 * BASE, 8 * BASE]
        cv = lambda a, b: Conv3x3(self.ctx, a, b, rng)
        self.enc = [[cv(IN_CH, c[0]), cv(c[0], c[0])], [cv(c[0], c[1]), cv(c[1], c[1])],
                    [cv(c[1], c[2]), cv(c[2], c[2])], [cv(c[2], c[3]), cv(c[3], c[3])]]
        # decoder level l (2, 1, 0): up-conv c[l+1] -> c[l], then two convs on the concatenation
        self.dec = {l: [cv(c[l + 1], c[l]), cv(2 * c[l], c[l]), cv(c[l], c[l])] for l in (2, 1, 0)}
        self.hw = torch.from_numpy((rng.standard_normal(c[0]) * math.sqrt(1.0 / c[0])).astype(np.float32)).to(device)
        self.hb = torch.zeros(1, dtype=torch.float32, device=device)
        self.ghw, self.ghb = torch.zeros_like(self.hw), torch.zeros_like(self.hb)
        self.mhw, self.vhw = torch.zeros_like(self.hw), torch.zeros_like(self.hw)
        self.mhb, self.vhb = torch.zeros_like(self.hb), torch.zeros_like(self.hb)
        self.step_count = 0
        self.shape = None
        self.target = "log_h"            # meaning of the output, one of TARGETS

    def layers(self):
        out = [l for lev in self.enc for l in lev]
        for k in (2, 1, 0):
            out += self.dec[k]
        return out

    def _alloc(self, B, H, W):
        if self.shape == (B, H, W):
            return
        torch, dev = self.torch, self.ctx.device
        self.shape = (B, H, W)
        c = [BASE, 2 * BASE, 4 * BASE, 8 * BASE]
        P = [B * (H >> l) * (W >> l) for l in range(4)]
        bf = lambda n: torch.empty(n, dtype=torch.bfloat16, device=dev)
        self.a = {}
        for l in range(4):
            self.a[f"e{l}a"] = bf(P[l] * c[l])
            self.a[f"e{l}b"] = bf(P[l] * c[l])
            if l < 3:
                self.a[f"p{l}"] = bf(P[l + 1] * c[l])
                self.a[f"arg{l}"] = torch.empty(P[l + 1] * c[l], dtype=torch.uint8, device=dev)
        for l in (2, 1, 0):
            self.a[f"u{l}"] = bf(P[l] * c[l + 1])         # upsampled input
            self.a[f"d{l}a"] = bf(P[l] * c[l])            # up-conv output
            self.a[f"cat{l}"] = bf(P[l] * 2 * c[l])
            self.a[f"d{l}b"] = bf(P[l] * c[l])
            self.a[f"d{l}c"] = bf(P[l] * c[l])
        self.out = torch.empty(P[0], dtype=torch.float32, device=dev)
        self.P, self.C = P, c

    def forward(self, x16, B, H, W):
        """x16 bf16 [B*H*W][8] -> prediction float [B*H*W] (self.out)."""
        self._alloc(B, H, W)
        a, P, c, st = self.a, self.P, self.C, self.ctx.st
        L = nnlib()
        self.x16 = x16
        inp = x16
        for l in range(4):
            h, w = H >> l, W >> l
            self.enc[l][0].forward(inp, B, h, w, a[f"e{l}a"])
            self.enc[l][1].forward(a[f"e{l}a"], B, h, w, a[f"e{l}b"])
            if l < 3:
                _ck(L.dsh_nn_maxpool_fwd(_p(a[f"e{l}b"]), B, h, w, c[l], _p(a[f"p{l}"]), _p(a[f"arg{l}"]), st), "pool")
                inp = a[f"p{l}"]
        low = a["e3b"]
        for l in (2, 1, 0):
            h, w = H >> l, W >> l
            _ck(L.dsh_nn_upsample_fwd(_p(low), B, h // 2, w // 2, c[l + 1], _p(a[f"u{l}"]), st), "upsample")
            d = self.dec[l]
            d[0].forward(a[f"u{l}"], B, h, w, a[f"d{l}a"])
            _ck(L.dsh_nn_concat(_p(a[f"e{l}b"]), c[l], _p(a[f"d{l}a"]), c[l], P[l], _p(a[f"cat{l}"]), st), "concat")
            d[1].forward(a[f"cat{l}"], B, h, w, a[f"d{l}b"])
            d[2].forward(a[f"d{l}b"], B, h, w, a[f"d{l}c"])
            low = a[f"d{l}c"]
        _ck(L.dsh_nn_head_fwd(_p(a["d0c"]), P[0], c[0], _p(self.hw), _p(self.hb), _p(self.out), st), "head")
        return self.out

    def backward(self, dout):
        """dout float [P0] = dLoss/dprediction; accumulates every parameter gradient."""
        torch = self.torch
        B, H, W = self.shape
        a, P, c, st = self.a, self.P, self.C, self.ctx.st
        L = nnlib()
        f32 = lambda n: torch.empty(n, dtype=torch.float32, device=self.ctx.device)
        g = f32(P[0] * c[0])
        red = self.ctx.scratch("red", RED_BLOCKS * (c[0] + 1), torch.float32)
        _ck(L.dsh_nn_head_bwd(_p(dout), _p(a["d0c"]), P[0], c[0], _p(self.hw), _p(g), _p(self.ghw), _p(self.ghb),
                              _p(red), st), "head_bwd")
        skip = {}
        for l in (0, 1, 2):
            h, w = H >> l, W >> l
            d = self.dec[l]
            g_b = f32(P[l] * c[l])
            d[2].backward(a[f"d{l}b"], a[f"d{l}c"], g, B, h, w, dx=g_b)
            g_cat = f32(P[l] * 2 * c[l])
            d[1].backward(a[f"cat{l}"], a[f"d{l}b"], g_b, B, h, w, dx=g_cat)
            g_skip, g_up = f32(P[l] * c[l]), f32(P[l] * c[l])
            _ck(L.dsh_nn_split(_p(g_cat), c[l], c[l], P[l], _p(g_skip), _p(g_up), st), "split")
            skip[l] = g_skip
            g_u = f32(P[l] * c[l + 1])
            d[0].backward(a[f"u{l}"], a[f"d{l}a"], g_up, B, h, w, dx=g_u)
            g = f32(P[l + 1] * c[l + 1])
            _ck(L.dsh_nn_upsample_bwd(_p(g_u), B, h // 2, w // 2, c[l + 1], _p(g), st), "upsample_bwd")
        # g: gradient of e3b (bottom output)
        for l in (3, 2, 1, 0):
            h, w = H >> l, W >> l
            e = self.enc[l]
            inp = self.x16 if l == 0 else a[f"p{l - 1}"]
            g_a = f32(P[l] * c[l])
            e[1].backward(a[f"e{l}a"], a[f"e{l}b"], g, B, h, w, dx=g_a)
            if l == 0:
                e[0].backward(inp, a["e0a"], g_a, B, h, w, dx=None)
                break
            g_in = f32(P[l] * c[l - 1])
            e[0].backward(inp, a[f"e{l}a"], g_a, B, h, w, dx=g_in)
            # input of level l is the pooled output of level l-1: route, then add the skip gradient
            g = f32(P[l - 1] * c[l - 1])
            _ck(L.dsh_nn_maxpool_bwd(_p(g_in), _p(a[f"arg{l - 1}"]), B, H >> (l - 1), W >> (l - 1), c[l - 1], _p(g),
                                     st), "pool_bwd")
            _ck(L.dsh_nn_add(_p(g), _p(skip[l - 1]), P[l - 1] * c[l - 1], st), "add")

    def zero_grad(self):
        for l in self.layers():
            l.zero_grad()
        self.ghw.zero_()
        self.ghb.zero_()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        L, st = nnlib(), self.ctx.st
        groups = []
        for l in self.layers():
            groups += l.params()
        groups += [(self.hw, self.mhw, self.vhw, self.ghw, 1, self.hw.numel(), 0),
                   (self.hb, self.mhb, self.vhb, self.ghb, 1, 1, 0)]
        for w, m, v, g, rows, cols, tr in groups:
            _ck(L.dsh_nn_adam(_p(w), _p(m), _p(v), _p(g), rows, cols, tr, lr, b1, b2, eps, self.step_count, st),
                "adam")
        for l in self.layers():
            l.prep()

    def loss_grad(self, target, mask=None):
        """MSE against target float [P0]: returns (loss tensor [1], grad [P0])."""
        torch = self.torch
        n = self.P[0]
        grad = torch.empty(n, dtype=torch.float32, device=self.ctx.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.ctx.device)
        count = float(n if mask is None else int(mask.sum().item()))
        _ck(nnlib().dsh_nn_mse(_p(self.out), _p(target), _p(mask), n, count, _p(grad), _p(loss), self.ctx.st), "mse")
        return loss, grad

    def state(self):
        """FP32 parameters as numpy arrays (for the CPU check and checkpoints)."""
        out = {}
        for k, l in enumerate(self.layers()):
            out[f"w{k}"] = l.w.cpu().numpy()
            out[f"b{k}"] = l.b.cpu().numpy()
        out["hw"] = self.hw.cpu().numpy()
        out["hb"] = self.hb.cpu().numpy()
        return out

    def load_state(self, st):
        """Inverse of state(): FP32 parameters from numpy arrays."""
        torch = self.torch
        for k, l in enumerate(self.layers()):
            l.w.copy_(torch.from_numpy(np.asarray(st[f"w{k}"], np.float32)))
            l.b.copy_(torch.from_numpy(np.asarray(st[f"b{k}"], np.float32)))
            l.prep()
        self.hw.copy_(torch.from_numpy(np.asarray(st["hw"], np.float32)))
        self.hb.copy_(torch.from_numpy(np.asarray(st["hb"], np.float32)))

    def grads(self):
        """Accumulated gradients as numpy arrays (weights [cout][9cin])."""
        out = {}
        for k, l in enumerate(self.layers()):
            out[f"w{k}"] = l.gwt.view(l.K, l.cout).t().contiguous().cpu().numpy()
            out[f"b{k}"] = l.gb.cpu().numpy()
        out["hw"] = self.ghw.cpu().numpy()
        out["hb"] = self.ghb.cpu().numpy()
        return out


def pack_inputs(torch, g, ws, wr, vs, device="cuda"):
    """Network input bf16 [B*H*W][8] from per-sample maps [B][H][W]: raw
    gradient / max|g|, log10 of the energies relative to their maxima / 8,
    (vs - 300) / 100, zero padding channels."""
    g, ws, wr, vs = (np.asarray(a, np.float32) for a in (g, ws, wr, vs))
    if g.ndim == 2:
        g, ws, wr, vs = g[None], ws[None], wr[None], vs[None]
    B, H, W = g.shape
    x = np.zeros((B, H, W, IN_CH), np.float32)
    for b in range(B):
        x[b, ..., 0] = g[b] / max(float(np.abs(g[b]).max()), 1e-30)
        x[b, ..., 1] = np.log10(np.maximum(ws[b] / max(float(ws[b].max()), 1e-30), 1e-8)) / 8.0
        x[b, ..., 2] = np.log10(np.maximum(wr[b] / max(float(wr[b].max()), 1e-30), 1e-8)) / 8.0
        x[b, ..., 3] = (vs[b] - 300.0) / 100.0
    return torch.from_numpy(x.reshape(-1, IN_CH)).to(device).to(torch.bfloat16)


def hessian_target(h):
    """Training target: log10 of the Hessian diagonal relative to its maximum, / 8."""
    h = np.asarray(h, np.float64)
    return (np.log10(np.maximum(h / max(float(h.max()), 1e-300), 1e-8)) / 8.0).astype(np.float32)


def hessian_from_prediction(pred):
    """Inverse of hessian_target (up to the unknown scale)."""
    return np.power(10.0, 8.0 * np.asarray(pred, np.float64)).astype(np.float32)


# What the network's output stands for:
#   "log_h"          hessian_target(H) itself
#   "log_h_over_ws"  hessian_target(H) minus input channel 1 (log10 Ws / max Ws, / 8):
#                    the correction to the forward energy Ws, which carries most of
#                    the pseudo-Hessian's dynamic range (the vs kernel correlates
#                    forward strains, and strain ~ particle velocity / vs)
TARGETS = ("log_h", "log_h_over_ws")


def residual_targets(torch, xs, ts):
    """Training targets of the "log_h_over_ws" mode from (inputs, hessian_target) pairs."""
    return [t - x.view(-1, IN_CH)[:, 1].float() for x, t in zip(xs, ts)]


def prediction_to_hessian(torch, target, out, x16, shape):
    """Pseudo-Hessian (up to scale) from the network output of a `target` mode network."""
    pred = out.float()
    if target == "log_h_over_ws":
        pred = pred + x16.view(-1, IN_CH)[:, 1].float()
    elif target != "log_h":
        raise ValueError(target)
    return hessian_from_prediction(pred.cpu().numpy().reshape(shape))
