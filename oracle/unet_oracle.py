"""CPU oracle of the warm-start U-Net (test infrastructure only).

A float64 numpy restatement of the network that `csrc/unet.cu` trains on
the GPU, with its forward pass, loss and backward pass, used to check the
GPU kernels' outputs and parameter gradients.  The reference has no such
network (it is this library's learned warm start); what is restated
here is the architecture and the parameter layout of `csrc/unet.cu`:

  e1a = relu(conv(x, 2->16)),  e1 = relu(conv(e1a, 16->16))           H
  e2a = relu(conv(pool(e1), 16->32)), e2 = relu(conv(e2a, 32->32))    H/2
  e3a = relu(conv(pool(e2), 32->64)), e3 = relu(conv(e3a, 64->64))    H/4
  e4a = relu(conv(pool(e3), 64->128)), e4 = relu(conv(e4a, 128->128)) H/8
  u3 = relu(conv(up(e4), 128->64)); d3a = relu(conv([u3, e3], 128->64)); d3 = relu(conv(d3a, 64->64))
  u2 = relu(conv(up(d3), 64->32));  d2a = relu(conv([u2, e2], 64->32));  d2 = relu(conv(d2a, 32->32))
  u1 = relu(conv(up(d2), 32->16));  d1a = relu(conv([u1, e1], 32->16));  d1 = relu(conv(d1a, 16->16))
  s = b + sum_c w_c d1_c, y = relu(s)                                  (1x1 head)

conv = 3x3, zero padding 1; pool = 2x2 max (gradient to the first maximum
in row-major order); up = nearest 2x.  Parameters (float32 master copy):
for each conv in the order above its weights [cout][cin][3][3] then its
bias [cout]; then the head's 16 weights and its bias.  Convolution and head
weights act through their BF16 rounding (round to nearest even), biases in
float32.  Loss = mean squared error of the unclamped s against the target
(the clamp applies to the returned initial image only).
"""
from __future__ import annotations

import numpy as np

# (cout, cin_a, cin_b, upsample_a, level)
CONVS = [(16, 2, 0, 0, 0), (16, 16, 0, 0, 0), (32, 16, 0, 0, 1), (32, 32, 0, 0, 1), (64, 32, 0, 0, 2),
         (64, 64, 0, 0, 2), (128, 64, 0, 0, 3), (128, 128, 0, 0, 3), (64, 128, 0, 1, 2), (64, 64, 64, 0, 2),
         (64, 64, 0, 0, 2), (32, 64, 0, 1, 1), (32, 32, 32, 0, 1), (32, 32, 0, 0, 1), (16, 32, 0, 1, 0),
         (16, 16, 16, 0, 0), (16, 16, 0, 0, 0)]
# source of input a of conv i: -1 network input, ('pool', l), or k = output of conv k - 1
SRC_A = [-1, 1, ("pool", 0), 3, ("pool", 1), 5, ("pool", 2), 7, 8, 9, 10, 11, 12, 13, 14, 15, 16]
SRC_B = {9: 6, 12: 4, 15: 2}  # concat partner: e3, e2, e1


def layout():
    """Offsets (w_off, b_off) per conv, head weight / bias offsets, total."""
    off, out = 0, []
    for cout, ca, cb, _, _ in CONVS:
        w = off
        off += cout * (ca + cb) * 9
        out.append((w, off))
        off += cout
    head_w = off
    return out, head_w, head_w + 16, head_w + 17


def bf16(a):
    """Round float32 values to BF16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3x3(x, w, bias=None):
    """x [n][ci][H][W], w [co][ci][3][3] -> [n][co][H][W]."""
    n, ci, H, W = x.shape
    xp = np.zeros((n, ci, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((n, w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oc,nchw->nohw", w[:, :, ky, kx], xp[:, :, ky:ky + H, kx:kx + W])
    if bias is not None:
        out += bias[None, :, None, None]
    return out


def conv3x3_grads(x, w, g):
    """Gradients of conv3x3(x, w) for the output gradient g: (dx, dw, db)."""
    n, ci, H, W = x.shape
    xp = np.zeros((n, ci, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    dw = np.zeros_like(w)
    dxp = np.zeros_like(xp)
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", g, xp[:, :, ky:ky + H, kx:kx + W])
            dxp[:, :, ky:ky + H, kx:kx + W] += np.einsum("oc,nohw->nchw", w[:, :, ky, kx], g)
    return dxp[:, :, 1:-1, 1:-1], dw, g.sum(axis=(0, 2, 3))


def pool(x):
    n, c, H, W = x.shape
    return x.reshape(n, c, H // 2, 2, W // 2, 2).max(axis=(3, 5))


def pool_grad(x, g):
    blocks = [x[:, :, 0::2, 0::2], x[:, :, 0::2, 1::2], x[:, :, 1::2, 0::2], x[:, :, 1::2, 1::2]]
    am = np.zeros(blocks[0].shape, int)
    best = blocks[0].copy()
    for k in range(1, 4):
        better = blocks[k] > best
        am[better] = k
        best = np.where(better, blocks[k], best)
    out = np.zeros_like(x)
    for k, (dy, dx) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1)]):
        out[:, :, dy::2, dx::2] = np.where(am == k, g, 0.0)
    return out


def up(x):
    return x.repeat(2, axis=2).repeat(2, axis=3)


def up_grad(g):
    n, c, H, W = g.shape
    return g.reshape(n, c, H // 2, 2, W // 2, 2).sum(axis=(3, 5))


class UNetOracle:
    """round_bf16=False keeps the weights in float64 (for finite-difference
    checks of the oracle itself); the GPU network corresponds to True."""

    def __init__(self, params, round_bf16=True):
        self.p = np.asarray(params, np.float32 if round_bf16 else np.float64)
        self.rnd = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
        self.lay, self.hw, self.hb, self.n = layout()
        assert self.p.size == self.n

    def _w(self, i):
        cout, ca, cb, _, _ = CONVS[i]
        w0, b0 = self.lay[i]
        w = self.rnd(self.p[w0:b0]).reshape(cout, ca + cb, 3, 3)
        return w, self.p[b0:b0 + cout].astype(np.float64)

    def forward(self, x):
        """The clamped initial image [n][H][W]."""
        act = [np.asarray(x, np.float64)]
        pools = {}
        self.inp = []
        for i, (cout, ca, cb, ups, lv) in enumerate(CONVS):
            if i in (2, 4, 6):
                l = (i - 2) // 2
                pools[l] = pool(act[2 + 2 * l])
            s = SRC_A[i]
            a = act[0] if s == -1 else pools[s[1]] if isinstance(s, tuple) else act[s]
            if ups:
                a = up(a)
            inp = np.concatenate([a, act[SRC_B[i]]], axis=1) if cb else a
            self.inp.append(inp)
            w, b = self._w(i)
            act.append(np.maximum(conv3x3(inp, w, b), 0.0))
        self.act, self.pools = act, pools
        hwt = self.rnd(self.p[self.hw:self.hb])
        self.pre = self.p[self.hb].astype(np.float64) + np.einsum("c,nchw->nhw", hwt, act[17])
        return np.maximum(self.pre, 0.0)

    def loss_and_grad(self, x, target):
        self.forward(x)
        t = np.asarray(target, np.float64).reshape(self.pre.shape)
        d = self.pre - t
        loss = float(np.mean(d * d))
        gp = 2.0 * d / d.size
        grad = np.zeros(self.n)
        hwt = self.rnd(self.p[self.hw:self.hb])
        grad[self.hw:self.hb] = np.einsum("nhw,nchw->c", gp, self.act[17])
        grad[self.hb] = gp.sum()
        gact = [np.zeros_like(a) for a in self.act]
        gpool = {l: np.zeros_like(p) for l, p in self.pools.items()}
        gact[17] = hwt[None, :, None, None] * gp[:, None]
        for i in range(16, -1, -1):
            cout, ca, cb, ups, lv = CONVS[i]
            g = np.where(self.act[i + 1] > 0, gact[i + 1], 0.0)
            w, _ = self._w(i)
            dx, dw, db = conv3x3_grads(self.inp[i], w, g)
            w0, b0 = self.lay[i]
            grad[w0:b0] = dw.reshape(-1)
            grad[b0:b0 + cout] = db
            if i > 0:
                da = dx[:, :ca]
                if ups:
                    da = up_grad(da)
                s = SRC_A[i]
                if isinstance(s, tuple):
                    gpool[s[1]] += da
                else:
                    gact[s] += da
                if cb:
                    gact[SRC_B[i]] += dx[:, ca:]
            if i in (2, 4, 6):
                l = (i - 2) // 2
                gact[2 + 2 * l] += pool_grad(self.act[2 + 2 * l], gpool[l])
        return loss, grad
