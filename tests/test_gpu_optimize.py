"""The graph optimisation pass on the GPU (trav_el_optimize, trav_el_gpu_transactions) against the oracle.

The device pass must give the oracle's arrays exactly (its sorts are stable, so the order is defined), and the
transaction count must equal the oracle's, which the CPU suite pins to the reference's own functions.
"""
import os

import numpy as np
import pytest

import oracle as O
import pytrav as T

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


CASES = [
    # (V, E, weight levels, segment)
    (50, 2000, 3, 0),
    (250000, 20011, 8, 65536),
    (1000, 31, 2, 7),
    (1000, 32, 2, 100),
    (1000, 33, 2, 0),
    (7, 500, 1, 2),       # all weights equal: ties resolved by edge order
    (300000, 400000, 1000, 1 << 12),
]


@pytest.mark.parametrize("V,E,levels,segment", CASES)
def test_el_optimize_equals_oracle(V, E, levels, segment):
    rng = np.random.default_rng(V + E)
    s = rng.integers(0, V, E).astype(np.int32)
    d = rng.integers(0, V, E).astype(np.int32)
    w = (rng.integers(0, levels, E) / max(levels - 1, 1)).astype(np.float32)
    s[: E // 20] = d[: E // 20]   # loops
    w[: E // 7] *= -0.0            # some weights become -0.0 (read as +0.0)
    ws, wd, ww = O.el_optimize(s, d, w, segment=segment)
    ts, td, tw = _dev(s), _dev(d), _dev(w)
    n = T.el_optimize(ts, td, tw, V, segment)
    assert n == len(ws)
    assert np.array_equal(ts[:n].cpu().numpy(), ws)
    assert np.array_equal(td[:n].cpu().numpy(), wd)
    assert np.array_equal(tw[:n].cpu().numpy().view(np.uint32), ww.view(np.uint32))


@pytest.mark.parametrize("E", [0, 1, 31, 32, 33, 64, 1000, 100003])
@pytest.mark.parametrize("elem", [1, 4, 8, 16])
def test_gpu_transactions_equal_oracle(E, elem):
    rng = np.random.default_rng(E * 7 + elem)
    V = 5000
    s = np.sort(rng.integers(0, V, E)).astype(np.int32)   # sorted sources share segments
    d = rng.integers(0, V, E).astype(np.int32)
    got = T.el_gpu_transactions(_dev(s), _dev(d), V, elem) if E else 0
    assert got == O.gpu_transactions(s, d, elem)


def test_fixture_through_the_device_pass(golden):
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "el_optimize.npz"))
    meta = golden[0]["optimize"]
    ts, td, tw = _dev(f["src"]), _dev(f["dst"]), _dev(f["w"])
    assert T.el_gpu_transactions(ts, td, meta["V"], 4) == meta["transactions_before"]["4"]
    n = T.el_optimize(ts, td, tw, meta["V"], meta["segment"])
    assert n == meta["E_after"]
    got = sorted(zip(ts[:n].cpu().numpy().tolist(), td[:n].cpu().numpy().tolist(), tw[:n].cpu().numpy().tolist()))
    ref = sorted(zip(f["ref_src"].tolist(), f["ref_dst"].tolist(), f["ref_w"].tolist()))
    assert got == ref


def test_host_arrays_take_the_same_path():
    rng = np.random.default_rng(8)
    V, E = 90000, 50000
    s = rng.integers(0, V, E).astype(np.int32)
    d = rng.integers(0, V, E).astype(np.int32)
    w = (rng.integers(0, 4, E) / 3).astype(np.float32)
    ws, wd, ww = O.el_optimize(s, d, w, segment=1 << 14)
    hs, hd, hw = s.copy(), d.copy(), w.copy()
    n = T.el_optimize(hs, hd, hw, V, 1 << 14)
    assert n == len(ws) and np.array_equal(hs[:n], ws) and np.array_equal(hd[:n], wd)
    assert np.array_equal(hw[:n].view(np.uint32), ww.view(np.uint32))
    assert T.el_gpu_transactions(s, d, V, 8) == O.gpu_transactions(s, d, 8)


def test_el_optimize_rejects_bad_input():
    import torch

    s = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    d = torch.tensor([1, 2], dtype=torch.int32, device="cuda")
    w = torch.tensor([0.5, 0.5], dtype=torch.float32, device="cuda")
    with pytest.raises(T.TravError):
        T.el_optimize(s, d, w, 4, 0)          # id 5 out of range
    with pytest.raises(T.TravError):
        T.el_optimize(s, d, w, 8, -1)         # negative segment
    with pytest.raises(T.TravError):
        T.el_optimize(s, d, -w, 8, 0)         # negative weights
