"""The tensor-core GEMM (tcgen05) and the warm-start MLP on the GPU, through the C ABI: the GEMM
against numpy on the same bfloat16 values (exact for an identity operand), the network's forward
pass, loss and every parameter's gradient against the CPU oracle (oracle/mlp_oracle.py), and a
training run that fits a teacher network."""
import numpy as np
import pytest

import mlp_oracle as MO
from rumb import _lib

pytestmark = pytest.mark.gpu


def _bf(rng, shape, scale=1.0):
    x = (rng.standard_normal(shape) * scale).astype(np.float32)
    return _lib.to_bf16_bits(x), MO.bf16(x)


def test_gemm_identity_is_exact(ctx):
    rng = np.random.default_rng(0)
    A = _lib.to_bf16_bits(np.eye(128, dtype=np.float32))
    Bb, Bf = _bf(rng, (128, 128))
    C = _lib.gemm_bf16(ctx, A, Bb)                  # C = I . B^T
    np.testing.assert_array_equal(C, Bf.T)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 320), (384, 256, 1024), (512, 1024, 384)])
def test_gemm_matches_numpy(ctx, M, N, K):
    rng = np.random.default_rng(M + N + K)
    Ab, Af = _bf(rng, (M, K))
    Bb, Bf = _bf(rng, (N, K))
    C = _lib.gemm_bf16(ctx, Ab, Bb)
    ref = Af.astype(np.float64) @ Bf.astype(np.float64).T
    # float32 accumulation of exact bfloat16 products: error ~ K * 2^-24 * sum |a b|
    bound = 4 * K * 2.0 ** -24 * (np.abs(Af).astype(np.float64) @ np.abs(Bf).astype(np.float64).T) + 1e-6
    assert np.all(np.abs(C - ref) <= bound)


def test_gemm_rejects_unpadded_shapes(ctx):
    with pytest.raises(_lib.RumbError, match="multiples of 128"):
        _lib.gemm_bf16(ctx, np.zeros((100, 64), np.uint16), np.zeros((128, 64), np.uint16))


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("dims,rows", [([301, 256, 256, 301], 200), ([37, 130, 5], 300)])
def test_mlp_matches_oracle(ctx, dims, rows):
    rng = np.random.default_rng(7)
    p = MO.init_params(dims, seed=3)
    X = rng.uniform(0, 1, (rows, dims[0])).astype(np.float32)
    T = rng.uniform(0, 1, (rows, dims[-1])).astype(np.float32)
    net = _lib.MLP(ctx, dims, seed=0)
    net.set_params(p)
    np.testing.assert_array_equal(net.get_params(), p)
    out = net.forward(X)
    ref_out, _, _ = MO.forward(p, dims, X)
    assert _rel(out, ref_out) <= 5e-3
    loss, g = net.loss_grad(X, T)
    ref_loss, ref_g = MO.loss_grad(p, dims, X, T)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    off = 0
    for l in range(len(dims) - 1):                  # every layer's dW and db
        nw = dims[l] * dims[l + 1]
        assert _rel(g[off:off + nw], ref_g[off:off + nw]) <= 2e-2, ("W", l)
        off += nw
        assert _rel(g[off:off + dims[l + 1]], ref_g[off:off + dims[l + 1]]) <= 2e-2, ("b", l)
        off += dims[l + 1]
    net.close()


def test_mlp_training_fits_a_teacher(ctx):
    dims = [64, 256, 256, 32]
    rng = np.random.default_rng(11)
    teacher = MO.init_params(dims, seed=5)
    X = rng.uniform(-1, 1, (1024, dims[0])).astype(np.float32)
    T = MO.forward(teacher, dims, X)[0].astype(np.float32)
    net = _lib.MLP(ctx, dims, seed=1)
    before, _ = net.loss_grad(X, T, want_grad=False)
    after = net.train(X, T, epochs=60, batch=256, lr=2e-3, seed=0)
    check, _ = net.loss_grad(X, T, want_grad=False)
    assert after < 0.1 * before and check < 0.1 * before
    net.close()
