"""CPU oracle for the tensor-core MLP -- TEST INFRASTRUCTURE ONLY.

The learned warm start has no counterpart in the reference; this numpy restatement of the
library's network (csrc/mlp.cu) is what its GPU kernels are checked against. It rounds to
bfloat16 exactly where the GPU stores bfloat16 (inputs, weights, hidden activations, the
backward's gradients) and accumulates in float64 where the GPU accumulates in float32, so the
two agree to accumulation order and the occasional bfloat16 rounding that order flips.

Network: H_0 = bf16(X); Z_l = H_{l-1} bf16(W_l)^T + b_l; H_l = bf16(gelu(Z_l)) between layers;
out = Z_L. Loss = mean (out - T)^2. Backward: G_L = bf16(2 (out - T) / count);
dW_l = G_l^T H_{l-1}; db_l = column sums of G_l; G_{l-1} = bf16((G_l bf16(W_l)) * gelu'(Z_{l-1})).
Parameters flat, per layer W (out x in, row-major) then b.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(np.shape(x))


def gelu(z):
    z = np.asarray(z, dtype=np.float64)
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    z = np.asarray(z, dtype=np.float64)
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params, dims):
    out, off = [], 0
    for l in range(len(dims) - 1):
        n_in, n_out = dims[l], dims[l + 1]
        W = np.asarray(params[off:off + n_in * n_out], dtype=np.float64).reshape(n_out, n_in)
        off += n_in * n_out
        b = np.asarray(params[off:off + n_out], dtype=np.float64)
        off += n_out
        out.append((W, b))
    return out


def forward(params, dims, X, rounding=True):
    """(out float32, Zs, Hs): the forward pass; rounding=False keeps every value in float64."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params, dims)
    H = rnd(np.asarray(X, dtype=np.float32))
    Hs, Zs = [H], []
    for l, (W, b) in enumerate(layers):
        Wr = rnd(W.astype(np.float32)) if rounding else W
        bb = b.astype(np.float32).astype(np.float64) if rounding else b
        Z = np.asarray(H, np.float64) @ np.asarray(Wr, np.float64).T + bb
        if rounding:
            Z = Z.astype(np.float32)
        if l + 1 < len(layers):
            Zs.append(Z)
            g = gelu(Z)
            H = rnd(g.astype(np.float32)) if rounding else g
            Hs.append(H)
        else:
            return Z, Zs, Hs


def loss_grad(params, dims, X, T, rounding=True):
    """(loss, flat gradient) of the mean squared error."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    out, Zs, Hs = forward(params, dims, X, rounding)
    T = np.asarray(T, dtype=np.float64)
    e = np.asarray(out, np.float64) - T
    loss = float(np.mean(e * e))
    layers = unpack(params, dims)
    G = 2.0 * e / e.size
    G = rnd(G.astype(np.float32)) if rounding else G
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        Gd = np.asarray(G, np.float64)
        grads[l] = (Gd.T @ np.asarray(Hs[l], np.float64), Gd.sum(axis=0))
        if l == 0:
            break
        dH = Gd @ np.asarray(rnd(W.astype(np.float32)) if rounding else W, np.float64)
        G = dH * gelu_grad(Zs[l - 1])
        G = rnd(G.astype(np.float32)) if rounding else G
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat.astype(np.float64)


def init_params(dims, seed=0):
    """Seeded parameters in the flat layout (uniform +-1/sqrt(fan_in))."""
    rng = np.random.default_rng(seed)
    parts = []
    for l in range(len(dims) - 1):
        a = 1.0 / math.sqrt(dims[l])
        parts.append(rng.uniform(-a, a, dims[l + 1] * dims[l]))
        parts.append(rng.uniform(-a, a, dims[l + 1]))
    return np.concatenate(parts).astype(np.float32)
