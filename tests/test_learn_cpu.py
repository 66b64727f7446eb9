"""Host logic of the learned schedule (pytrav.learn), on the CPU: the abstention rule the kernels apply, the
trace labels, the margin pick, and the learned split's features and choice.  The networks here have constant
outputs (last layer's weights zero), so every logit is known."""
import json
import types

import numpy as np
import pytest

import pytrav as T
from pytrav import learn

F, H = 10, 32


def constant_net(kind, logits):
    """Parameters of a network whose output logits are `logits` for every input."""
    O = T.MLP_OUTPUTS[kind]
    assert len(logits) == O
    rng = np.random.default_rng(kind)
    p = np.concatenate([rng.normal(size=H * F), rng.normal(size=H), rng.normal(size=H * H), rng.normal(size=H),
                        np.zeros(O * H), np.asarray(logits, np.float64)])
    assert len(p) == learn.mlp_param_count(kind)
    return p.astype(np.float32)


def test_abstention_keeps_the_plain_option_unless_the_margin_is_cleared():
    p = constant_net(1, [0.0, 0.3, 0.1, -1.0, -1.0, -1.0])  # width x4 beats the plain x1 by 0.3
    X = np.zeros((3, F), np.float32)
    assert (learn.choose(1, p, X, 0.0) == 1).all()
    assert (learn.choose(1, p, X, 0.25) == 1).all()
    assert (learn.choose(1, p, X, 0.5) == 0).all()
    # BFS: the plain option is Beamer's direction, the last feature
    q = constant_net(0, [0.2, 0.0])  # top-down preferred by 0.2
    Xb = np.zeros((2, F), np.float32)
    Xb[1, 9] = 1.0  # Beamer says bottom-up here
    assert learn.choose(0, q, Xb, 0.1).tolist() == [0, 0]
    assert learn.choose(0, q, Xb, 0.5).tolist() == [0, 1]  # abstains: keeps Beamer's choice
    assert learn.plain_option(0, Xb).tolist() == [0, 1]
    assert learn.plain_option(1, Xb).tolist() == [0, 0]


def test_trace_labels_leave_the_plain_option_only_when_clearly_faster():
    assert learn.margin_label([10.0, 9.6], 0) == 0  # 4% faster: a near tie stays plain
    assert learn.margin_label([10.0, 9.4], 0) == 1  # 6% faster
    assert learn.margin_label([9.0, 10.0, 8.0], 1) == 2
    assert learn.margin_label([np.inf, 5.0], 0) == 1  # the plain option was never timed


def test_margin_pick_minimises_the_traced_cost():
    p = constant_net(1, [0.0, 0.3, -1.0, -1.0, -1.0, -1.0])
    X = np.zeros((2, F), np.float32)
    cost = np.array([[1.0, 5.0, 9, 9, 9, 9], [1.0, 5.0, 9, 9, 9, 9]])  # deviating to x4 costs more here
    best, table = learn.pick_margin(1, p, X, cost)
    assert best >= 0.5 and table["by_margin"][str(best)] == pytest.approx(2.0)
    assert table["plain"] == pytest.approx(2.0)
    cost2 = np.array([[5.0, 1.0, 9, 9, 9, 9]] * 2)  # deviating pays: the smallest margin that deviates wins
    best2, table2 = learn.pick_margin(1, p, X, cost2)
    assert best2 <= 0.25 and table2["by_margin"][str(best2)] == pytest.approx(2.0)


def test_split_features_are_scale_free_except_the_size_input():
    a = learn.split_features(1 << 20, 16 << 20, 5000, 0.5, 0.1)
    b = learn.split_features(1 << 22, 16 << 22, 5000, 0.5, 0.1)
    assert np.isfinite(a).all() and np.isfinite(b).all()
    assert a[0] == pytest.approx(b[0]) and a[3] == pytest.approx(b[3]) and a[4] == pytest.approx(b[4])
    assert b[2] > a[2]  # log2 E
    c = learn.split_features(1 << 20, 16 << 20, 5000, 0.05, 0.1)  # mean weight below delta
    assert c[3] < 0.0 < a[3]


def test_split_choice_follows_the_network_and_its_margin(tmp_path):
    g = types.SimpleNamespace(V=1 << 20, E=16 << 20, max_out_degree=5000, mean_weight=0.5)
    assert learn.split_scale(g, 0.1, str(tmp_path)) == 1.0  # no split network: the caller's delta
    logits = [0.0, 0.4, -1.0, -5.0, -5.0, -5.0]  # delta / 2 preferred by 0.4
    constant_net(1, logits).tofile(tmp_path / "sssp_split.f32")
    for margin, want in ((0.0, learn.SPLITS[1]), (0.25, learn.SPLITS[1]), (1.0, 1.0)):
        (tmp_path / "sssp_split.json").write_text(json.dumps({"margin": margin}))
        assert learn.split_scale(g, 0.1, str(tmp_path)) == want, margin
    np.zeros(7, np.float32).tofile(tmp_path / "sssp_split.f32")
    with pytest.raises(ValueError):
        learn.split_scale(g, 0.1, str(tmp_path))


def test_shipped_networks_load_with_their_margins():
    for kind in (0, 1):
        p = learn.load(kind)
        assert p is not None and len(p) == learn.mlp_param_count(kind) and np.isfinite(p).all()
        assert learn.load_margin(kind) in learn.MARGINS
    p, margin = learn.load_split()
    assert p is not None and np.isfinite(p).all() and margin in learn.MARGINS
