"""Tensor-core (tcgen05) kernels of the volume-move surrogate, against FP64 numpy.

* the BF16 GEMM (C = A B^T, FP32 accumulation in TMEM) on ragged shapes;
* MLP gradients (forward + backward kernels) against the FP64 oracle in
  tests/mlp_oracle.py with the same BF16 rounding points;
* training reduces the loss on a learnable synthetic target.
"""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle as mo
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

pytestmark = pytest.mark.gpu

FP = C.POINTER(C.c_float)


def lib():
    L = _lib.lib()
    L.lcmc_gemm_bf16.argtypes = [FP, FP, FP, C.c_int, C.c_int, C.c_int]
    L.lcmc_mlp_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
    L.lcmc_mlp_destroy.argtypes = [C.c_void_p]
    L.lcmc_mlp_num_params.argtypes = [C.c_void_p]
    L.lcmc_mlp_gradients.argtypes = [C.c_void_p, FP, FP, C.c_int, FP, FP]
    L.lcmc_mlp_get_params.argtypes = [C.c_void_p, FP]
    L.lcmc_mlp_train.argtypes = [C.c_void_p, FP, FP, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64, FP]
    L.lcmc_mlp_predict.argtypes = [C.c_void_p, FP, C.c_int, FP]
    return L


def fp(a):
    return a.ctypes.data_as(FP)


# the last shape is the surrogate's first layer on a training batch of 8192 samples
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 128, 256), (300, 200, 4224), (128, 4224, 512),
                                   (8192, 128, 4224)])
def test_gemm_tensor_cores(M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = rng.normal(size=(N, K)).astype(np.float32)
    Cm = np.zeros((M, N), dtype=np.float32)
    rc = lib().lcmc_gemm_bf16(fp(A), fp(B), fp(Cm), M, N, K)
    assert rc == 0, rc
    want = mo.bf16(A) @ mo.bf16(B).T
    err = np.abs(Cm - want).max() / np.abs(want).max()
    assert err < 1e-5, err


def test_mlp_gradients_match_fp64_oracle():
    L = lib()
    n_in, n = 4097, 256
    h = C.c_void_p()
    assert L.lcmc_mlp_create(n_in, 128, 512, 11, C.byref(h)) == 0
    try:
        npar = L.lcmc_mlp_num_params(h)
        params = np.zeros(npar, dtype=np.float32)
        assert L.lcmc_mlp_get_params(h, fp(params)) == 0
        rng = np.random.default_rng(3)
        x = rng.normal(size=(n, n_in)).astype(np.float32)
        t = rng.normal(size=n).astype(np.float32)
        g = np.zeros(npar, dtype=np.float32)
        loss = C.c_float()
        assert L.lcmc_mlp_gradients(h, fp(x), fp(t), n, fp(g), C.byref(loss)) == 0
        want, wloss = mo.gradients(params, x, t.astype(np.float64), n_in)
        assert abs(loss.value - wloss) <= 1e-3 * wloss
        # BF16 activations of the backward pass (dZ) bound the agreement at ~1e-2
        rel = np.linalg.norm(g - want) / np.linalg.norm(want)
        cos = float(np.dot(g, want) / (np.linalg.norm(g) * np.linalg.norm(want)))
        print(f"MLP gradient: relative L2 error {rel:.2e}, cosine {cos:.6f}")
        assert rel < 2e-2 and cos > 0.9998
    finally:
        L.lcmc_mlp_destroy(h)


def test_mlp_training_reduces_loss():
    L = lib()
    n_in, n = 4097, 4096
    rng = np.random.default_rng(5)
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    w = np.zeros(n_in)
    w[:64] = rng.normal(size=64) / 8.0
    t = (np.tanh(x @ w) + 0.3 * x[:, -1]).astype(np.float32)
    h = C.c_void_p()
    assert L.lcmc_mlp_create(n_in, 128, 512, 12, C.byref(h)) == 0
    try:
        y0 = np.zeros(n, dtype=np.float32)
        assert L.lcmc_mlp_predict(h, fp(x), n, fp(y0)) == 0
        loss0 = float(np.mean((y0 - t) ** 2))
        fl = C.c_float()
        assert L.lcmc_mlp_train(h, fp(x), fp(t), n, 8, 256, 1e-3, 1, C.byref(fl)) == 0
        y1 = np.zeros(n, dtype=np.float32)
        assert L.lcmc_mlp_predict(h, fp(x), n, fp(y1)) == 0
        loss1 = float(np.mean((y1 - t) ** 2))
        print(f"MLP training loss {loss0:.4f} -> {loss1:.4f} (last epoch {fl.value:.4f})")
        assert loss1 < 0.2 * loss0
    finally:
        L.lcmc_mlp_destroy(h)


def test_bounded_wait_gives_up_cleanly():
    """With the mbarrier wait limit at one try, the GEMM's first wait gives up:
    the kernel sets its error flag, drains its MMAs (full bound), frees its
    TMEM and returns, and the call reports LCMC_ETIMEOUT; nothing faults or
    hangs.  With the default limit back, the next call computes the product."""
    L = lib()
    rng = np.random.default_rng(5)
    M, N, K = 256, 256, 1024
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    c = np.zeros((M, N), dtype=np.float32)
    try:
        assert L.lcmc_set_wait_limit(1) == 0
        assert L.lcmc_gemm_bf16(fp(a), fp(b), fp(c), M, N, K) == _lib.ETIMEOUT
    finally:
        L.lcmc_set_wait_limit(0)
    assert L.lcmc_gemm_bf16(fp(a), fp(b), fp(c), M, N, K) == 0
    ab = a.astype(np.float64)
    bb = b.astype(np.float64)
    want = mo.bf16(ab) @ mo.bf16(bb).T
    assert np.max(np.abs(c - want)) <= 1e-3 * np.max(np.abs(want))
