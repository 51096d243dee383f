"""The warm-start network's CPU oracle itself: bf16 rounding against torch's
conversion, GELU derivative and backward pass against central differences."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000) * 10 ** rng.uniform(-8, 8, 10000), [0.0, -0.0, 1.0, 65504.0]])
    ours = mo.bf16(x)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(ours, ref)


def test_gelu_grad_central_difference():
    z = np.linspace(-6, 6, 241)
    h = 1e-6
    fd = (mo.gelu(z + h) - mo.gelu(z - h)) / (2 * h)
    assert np.abs(fd - mo.gelu_grad(z)).max() < 1e-8


@pytest.mark.parametrize("skip", [False, True])
def test_backward_matches_central_differences(monkeypatch, skip):
    """With bf16 rounding switched off the oracle's gradients are exact."""
    monkeypatch.setattr(mo, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    rng = np.random.default_rng(1)
    B, n_in, hid, n_out = 6, 5, 7, 4
    x = rng.standard_normal((B, n_in))
    Ws = [rng.standard_normal((hid, n_in)) * 0.5, rng.standard_normal((hid, hid)) * 0.5,
          rng.standard_normal((n_out, hid + (n_in if skip else 0))) * 0.5]
    bs = [rng.standard_normal(hid) * 0.1, rng.standard_normal(hid) * 0.1, rng.standard_normal(n_out) * 0.1]
    y = rng.standard_normal((B, n_out))
    _, loss, dWs, dbs = mo.forward_backward(x, Ws, bs, y, n_out, skip=skip)
    h = 1e-6
    for l in range(3):
        for (i, j) in [(0, 0), (1, 2), (Ws[l].shape[0] - 1, Ws[l].shape[1] - 1)]:
            Wp = [w.copy() for w in Ws]
            Wm = [w.copy() for w in Ws]
            Wp[l][i, j] += h
            Wm[l][i, j] -= h
            fd = (mo.forward_backward(x, Wp, bs, y, n_out, skip=skip)[1] - mo.forward_backward(x, Wm, bs, y, n_out, skip=skip)[1]) / (2 * h)
            assert fd == pytest.approx(dWs[l][i, j], rel=1e-5, abs=1e-9)
        bp = [b.copy() for b in bs]
        bm = [b.copy() for b in bs]
        bp[l][0] += h
        bm[l][0] -= h
        fd = (mo.forward_backward(x, Ws, bp, y, n_out, skip=skip)[1] - mo.forward_backward(x, Ws, bm, y, n_out, skip=skip)[1]) / (2 * h)
        assert fd == pytest.approx(dbs[l][0], rel=1e-5, abs=1e-9)
