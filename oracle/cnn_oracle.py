"""CPU oracle of the learned warm-start network (TEST INFRASTRUCTURE ONLY: imported by
tests/ to check the CUDA forward and backward kernels).

The network: per 20 x 20 tile, six 3x3 convolutions with zero padding at the tile edge
(2 -> 32, 32 -> 32 x 4, 32 -> 1), ReLU after the first five, output = the centre
16 x 16.  Parameters in one vector, layer by layer: W [9 taps][co][ci] then b [co];
tap t has offset (t // 3 - 1, t % 3 - 1) in (y, x).  Loss = mean over all outputs of
(y - t)^2.

With ``bf16=True`` the oracle rounds where the GPU kernels round (weights, every
layer's post-ReLU activation, every layer's output gradient) and accumulates in FP64;
with ``bf16=False`` it is the exact FP64 network (used for finite-difference checks of
the oracle's own backward pass).
"""
from __future__ import annotations

import numpy as np

LAYERS = [(2, 32), (32, 32), (32, 32), (32, 32), (32, 32), (32, 1)]  # (ci, co)
T = 20


def nparams():
    return sum(9 * co * ci + co for ci, co in LAYERS)


def bf16_round(a):
    """Round to bfloat16 (nearest even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def unpack(theta):
    out, o = [], 0
    for ci, co in LAYERS:
        W = theta[o:o + 9 * co * ci].reshape(9, co, ci)
        o += 9 * co * ci
        b = theta[o:o + co]
        o += co
        out.append((W, b))
    return out


def _shift(Ap, tap):
    dy, dx = tap // 3 - 1, tap % 3 - 1
    return Ap[:, 1 + dy:1 + dy + T, 1 + dx:1 + dx + T, :]


def _pad(A):
    return np.pad(A, ((0, 0), (1, 1), (1, 1), (0, 0)))


def forward(x, theta, bf16=True):
    """x: [n][400][2] -> (y [n][256], activations A_0..A_5 as [n][20][20][c])."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    n = x.shape[0]
    A = rnd(x.reshape(n, T, T, 2))
    acts = [A]
    params = unpack(np.asarray(theta, dtype=np.float64))
    for l, (W, b) in enumerate(params):
        Wr = rnd(W)
        Ap = _pad(acts[-1])
        Z = np.zeros((n, T, T, Wr.shape[1])) + b[None, None, None, :]
        for tap in range(9):
            Z += np.einsum("nyxc,oc->nyxo", _shift(Ap, tap), Wr[tap], optimize=True)
        if l < len(params) - 1:
            acts.append(rnd(np.maximum(Z, 0.0)))
        else:
            y = Z[:, 2:18, 2:18, 0].reshape(n, 256)
    return y, acts


def rweights(ir0, geom):
    """Radial stencil weights [n][16] (w-, w+) of the 16 cell columns of each sample."""
    i = np.asarray(ir0, dtype=np.float64)[:, None] + np.arange(16)[None, :] + 1.0
    if geom == 1:
        return (2 * i - 2) / (2 * i - 1), (2 * i) / (2 * i - 1)
    return np.ones_like(i), np.ones_like(i)


def residual(y, x, ir0, geom, bf16=True):
    """rho [n][14][14] = L(y) + db channel of x on the interior cells."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    n = y.shape[0]
    Y = y.reshape(n, 16, 16)
    x1 = rnd(x.reshape(n, T, T, 2)[..., 1])[:, 3:17, 3:17]
    wm, wp = rweights(ir0, geom)
    wm, wp = wm[:, None, 1:15], wp[:, None, 1:15]
    L = wm * Y[:, 1:15, 0:14] + wp * Y[:, 1:15, 2:16] + Y[:, 0:14, 1:15] + Y[:, 2:16, 1:15] - 4 * Y[:, 1:15, 1:15]
    return L + x1


def gradients(x, t, theta, bf16=True, ir0=None, lam=0.0, geom=1):
    """Loss and gradient (parameter-vector layout).  Loss = mean (y - t)^2 plus, with
    ir0 given, lam * mean rho^2 over the 14 x 14 interior cells (rho = residual())."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    n = x.shape[0]
    y, acts = forward(x, theta, bf16)
    d = y - t.reshape(n, 256)
    loss = float(np.mean(d * d))
    gy = (2.0 / (256 * n) * d).reshape(n, 16, 16)
    if ir0 is not None and lam > 0:
        rho = residual(y, x, ir0, geom, bf16)
        loss += lam * float(np.mean(rho * rho))
        gr = 2.0 * lam / (196 * n) * rho
        wm, wp = rweights(ir0, geom)
        wm, wp = wm[:, None, 1:15], wp[:, None, 1:15]
        gy[:, 1:15, 1:15] += -4 * gr
        gy[:, 1:15, 0:14] += wm * gr
        gy[:, 1:15, 2:16] += wp * gr
        gy[:, 0:14, 1:15] += gr
        gy[:, 2:16, 1:15] += gr
    params = unpack(np.asarray(theta, dtype=np.float64))
    dZ = np.zeros((n, T, T, 1))
    dZ[:, 2:18, 2:18, 0] = gy
    dZ = rnd(dZ)
    grads = [None] * len(params)
    for l in range(len(params) - 1, -1, -1):
        W, b = params[l]
        Ap = _pad(acts[l])
        dW = np.zeros_like(W)
        for tap in range(9):
            dW[tap] = np.einsum("nyxo,nyxc->oc", dZ, _shift(Ap, tap), optimize=True)
        grads[l] = (dW, dZ.sum(axis=(0, 1, 2)))
        if l > 0:
            Wr = rnd(W)
            dZp = _pad(dZ)
            dA = np.zeros_like(acts[l])
            for tap in range(9):
                # dA[q] += dZ[q - off(tap)] W[tap]  (the flipped tap reads q - off)
                dA += np.einsum("nyxo,oc->nyxc", _shift(dZp, 8 - tap), Wr[tap], optimize=True)
            dZ = rnd(dA * (acts[l] > 0))
    g = np.concatenate([np.concatenate([dW.ravel(), db.ravel()]) for dW, db in grads])
    return loss, g


def layer_slices():
    """(start, end) of every layer's W and b in the parameter vector."""
    out, o = [], 0
    for ci, co in LAYERS:
        out.append(((o, o + 9 * co * ci), (o + 9 * co * ci, o + 9 * co * ci + co)))
        o += 9 * co * ci + co
    return out
