"""The network on the tcgen05 tensor cores (TMEM accumulators, shared-memory
operands, TMA-loaded feature tiles): the dense forward and the fused training
step (forward, loss, backward) against the CUDA-core kernels and the float64
oracle.

Tolerances: T within 2e-3 of the CUDA-core forward (max; 1e-4 mean) and 5e-3
of the float64 network; gradients within 2e-2 relative L2 error of the
CUDA-core backward and of the float64 oracle (the tensor-core backward rounds
dY to bfloat16 where it enters a product), cosine > 0.999."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu


def _features(r, n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    lf = rng.normal(size=(n, 3))
    lf = (lf / np.linalg.norm(lf, axis=1, keepdims=True)).astype(np.float32)
    return r.mlp_encode(pos, lf)


@pytest.mark.parametrize("n", [1, 1000, 300_001])
def test_tcgen05_forward_matches_cuda_core_forward(cuda_device, n):
    s = scenes.small(81, n=24, image=16, m=8)
    with B.Renderer(0) as r:
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        rng = np.random.default_rng(3)
        P = rng.normal(0, 0.1, M.N_PARAMS).astype(np.float32)
        r.mlp_set_params(P)
        X = _features(r, n, 5)
        T_tc = r.mlp_forward_tc(X)
        r.mlp_set_tensor_cores(False)  # the CUDA-core forward as the reference
        _, _, T_cc = r.mlp_loss_grad(X, np.zeros(n, np.float32))
        r.mlp_set_tensor_cores(True)
        _, _, T_tr = r.mlp_loss_grad(X, np.zeros(n, np.float32))  # training's forward: tcgen05
        assert np.array_equal(T_tr, T_tc)
        d = np.abs(T_tc - T_cc)
        print(f"n={n}: tcgen05 vs CUDA cores max {d.max():.2e} mean {d.mean():.2e}")
        assert np.all(np.isfinite(T_tc)) and d.max() < 2e-3 and d.mean() < 1e-4
        if n <= 1000:
            _, _, T64 = M.forward_backward(P, M.bf16(X), np.zeros(n))
            assert np.abs(T_tc - T64).max() < 5e-3


@pytest.mark.parametrize("n", [7, 384, 1000, 40_000])
def test_tcgen05_training_step_matches_cuda_cores_and_oracle(cuda_device, n):
    """Partial tiles (n not a multiple of 128) and several tiles per CTA
    (40,000 rows = 313 tiles on 148 SMs) accumulate the weight gradients in
    TMEM across tiles."""
    s = scenes.small(82, n=24, image=16, m=8)
    with B.Renderer(0) as r:
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        rng = np.random.default_rng(n)
        P = rng.normal(0, 0.15, M.N_PARAMS).astype(np.float32)
        r.mlp_set_params(P)
        X = _features(r, n, 9)
        t = rng.uniform(0, 1, n).astype(np.float32)
        loss_tc, g_tc, T_tc = r.mlp_loss_grad(X, t)
        r.mlp_set_tensor_cores(False)
        loss_cc, g_cc, T_cc = r.mlp_loss_grad(X, t)
        r.mlp_set_tensor_cores(True)
        assert np.all(np.isfinite(g_tc)) and np.all(np.isfinite(T_tc))
        assert np.abs(T_tc - T_cc).max() < 2e-3
        assert abs(loss_tc - loss_cc) <= 2e-3 * loss_cc + 1e-7
        rel = np.linalg.norm(g_tc - g_cc) / np.linalg.norm(g_cc)
        cos = float(g_tc @ g_cc / (np.linalg.norm(g_tc) * np.linalg.norm(g_cc)))
        print(f"n={n}: tensor-core vs CUDA-core gradient relative L2 {rel:.2e}, cosine {cos:.6f}")
        assert rel < 2e-2 and cos > 0.999
        if n <= 1000:
            _, og, _ = M.forward_backward(P, M.bf16(X), t)
            rel64 = np.linalg.norm(g_tc - og) / np.linalg.norm(og)
            assert rel64 < 2e-2, rel64
