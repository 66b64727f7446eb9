"""The schedule MLP: the float64 oracle against finite differences (CPU), and the CUDA training kernels against
the oracle (GPU)."""
import numpy as np
import pytest

import oracle as O
import pytrav as T

F, H = 10, 32


def _problem(kind, n, seed):
    rng = np.random.default_rng(seed)
    Oo = T.MLP_OUTPUTS[kind]
    p = T.mlp_init(kind, seed).astype(np.float64) if False else None
    x = rng.normal(size=(n, F))
    y = rng.integers(0, Oo, n).astype(np.int32)
    return Oo, x, y


def _init64(kind, seed):
    rng = np.random.default_rng(seed)
    Oo = T.MLP_OUTPUTS[kind]
    sizes = [H * F, H, H * H, H, Oo * H, Oo]
    return np.concatenate([rng.normal(scale=0.3, size=s) for s in sizes])


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_gradient_matches_finite_differences(kind):
    Oo, x, y = _problem(kind, 7, 3)
    p = _init64(kind, 5)
    loss, g = O.mlp_loss_grad(F, H, Oo, p, x, y)
    rng = np.random.default_rng(1)
    for i in rng.choice(len(p), 40, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        lp, _ = O.mlp_loss_grad(F, H, Oo, p + e, x, y, want_grad=False)
        lm, _ = O.mlp_loss_grad(F, H, Oo, p - e, x, y, want_grad=False)
        assert abs((lp - lm) / 2e-6 - g[i]) < 1e-6 + 1e-5 * abs(g[i]), i
    assert loss > 0


def test_param_layout_counts_match_library():
    for kind, Oo in ((0, 2), (1, 6)):
        assert T.mlp_param_count(kind) == H * F + H + H * H + H + Oo * H + Oo
        assert len(T.mlp_init(kind)) == T.mlp_param_count(kind)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1])
def test_cuda_gradient_matches_oracle(kind):
    Oo, x, y = _problem(kind, 1000, 11)
    p64 = _init64(kind, 12)
    want_loss, want = O.mlp_loss_grad(F, H, Oo, p64, x, y)
    loss, g = T.mlp_loss_grad(kind, p64.astype(np.float32), x.astype(np.float32), y)
    # fp32 kernels against the float64 oracle: relative 2e-3 of the largest gradient entry
    assert abs(loss - want_loss) < 1e-4 * max(1.0, abs(want_loss))
    assert np.max(np.abs(g - want)) < 2e-3 * np.max(np.abs(want))


@pytest.mark.gpu
def test_cuda_training_fits_a_separable_rule():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(4096, F)).astype(np.float32)
    y = (x[:, 1] - x[:, 2] > 0.3).astype(np.int32)  # a push/pull-like threshold rule
    p0 = T.mlp_init(0, 7)
    loss0, _ = T.mlp_loss_grad(0, p0, x, y)
    p, loss = T.mlp_train(0, p0, x, y, epochs=300, lr=1e-2)
    assert loss < 0.25 * loss0
    l64, _ = O.mlp_loss_grad(F, H, 2, p.astype(np.float64), x.astype(np.float64), y, want_grad=False)
    assert abs(l64 - loss) < 1e-3
