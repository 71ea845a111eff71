"""Learned form, training side: the device forward/backward against the float64
oracle, the input encoding, a training run's gain over the method without a
shadow model, and checkpoints."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu


def small_renderer(seed=51, n=40):
    s = scenes.small(seed, n=n, image=64, m=16, kind="blobs")
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    return s, r


def test_mlp_gradients_match_float64_oracle(cuda_device):
    _, r = small_renderer()
    rng = np.random.default_rng(3)
    P = rng.normal(0, 0.15, M.N_PARAMS).astype(np.float32)
    r.mlp_set_params(P)
    X = rng.uniform(-1, 1, (384, M.K_IN)).astype(np.float32)
    X[:, M.K_USED:] = 0
    t = rng.uniform(0, 1, 384).astype(np.float32)
    loss, g, T = r.mlp_loss_grad(X, t)
    oloss, og, oT = M.forward_backward(P, M.bf16(X), t)
    assert np.max(np.abs(T - oT)) < 5e-3
    assert abs(loss - oloss) <= 1e-3 * oloss + 1e-7
    rel = np.linalg.norm(g - og) / np.linalg.norm(og)
    cos = float(g @ og / (np.linalg.norm(g) * np.linalg.norm(og)))
    print(f"gradient: relative L2 error {rel:.2e}, cosine {cos:.6f}")
    assert rel < 2e-2 and cos > 0.9995


def test_mlp_encoding_matches_oracle(cuda_device):
    s, r = small_renderer()
    rng = np.random.default_rng(4)
    pos = rng.uniform(0, 1, (500, 3)).astype(np.float32)
    lf = rng.normal(size=(500, 3))
    lf = (lf / np.linalg.norm(lf, axis=1, keepdims=True)).astype(np.float32)
    got = r.mlp_encode(pos, lf)
    ref = M.bf16(M.encode(pos, lf, (0, 0, 0), (1, 1, 1)))
    # one bfloat16 ulp, plus the phase error of a float32 position at 128 half-cycles
    ulp = np.abs(ref) * 2.0 ** -7
    assert np.all(np.abs(got - ref) <= ulp + 1e-3)
    assert np.mean(got == ref) > 0.97


def test_mlp_training_gains_over_no_shadow_model(cuda_device):
    _, r = small_renderer(52, n=48)
    rep = r.mlp_train(B.mlp_options(samples_log2=17, epochs=8, batch=1024, lr=3e-3))
    print("mlp training report:", rep)
    assert rep["holdout_rmse"] < 0.5 * rep["initial_rmse"]
    assert rep["holdout_rmse"] < 0.5 * rep["unlit_rmse"] and rep["holdout_rmse"] < rep["mean_rmse"]


def test_mlp_checkpoint_roundtrip_and_corruption(cuda_device, tmp_path):
    _, r = small_renderer()
    rng = np.random.default_rng(5)
    P = rng.normal(0, 0.1, M.N_PARAMS).astype(np.float32)
    r.mlp_set_params(P)
    path = tmp_path / "net.bmlp"
    r.mlp_save(path)
    _, r2 = small_renderer()
    r2.mlp_load(path)
    assert np.array_equal(r2.mlp_params(), P)
    data = bytearray(path.read_bytes())
    data[100] ^= 0xFF
    bad = tmp_path / "bad.bmlp"
    bad.write_bytes(bytes(data))
    with pytest.raises(B.BeamsError) as e:
        r2.mlp_load(bad)
    assert e.value.status == 6  # CONFIG
