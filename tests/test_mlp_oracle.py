"""The CPU restatement of the learned initial guess (oracle/mlp_oracle.py) and
the network's host-side set-up, without a GPU: BF16 rounding, the FP64
gradients against finite differences, the output encoding of the field
(continuous across the 180-degree azimuth ambiguity) and gm_mlp_init."""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import mlp_oracle as M
from helpers import random_net


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-3, 1000), [0.0, -0.0, 1.0, 3.0e38]])
    x = x.astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(M.bf16(x), want)


def test_fp64_gradients_match_finite_differences():
    rng = np.random.default_rng(2)
    net = random_net(2)
    p = M.params(net)
    X = rng.normal(0, 1, (16, M.IN))
    X[:, 120:] = 0.0
    Y = rng.normal(0, 1, (16, M.OUT))
    _, g = M.loss_and_grads(p, X, Y, quantize=False)
    h = 1e-6
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        arr = p[name]
        flat = arr.reshape(-1)
        n = flat.size if name != "b3" else M.OUT
        for i in rng.choice(n, size=min(12, n), replace=False):
            if name == "w1" and i % M.IN >= 120:
                continue
            keep = flat[i]
            flat[i] = keep + h
            lp, _ = M.loss_and_grads(p, X, Y, quantize=False)
            flat[i] = keep - h
            lm, _ = M.loss_and_grads(p, X, Y, quantize=False)
            flat[i] = keep
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[i]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(fd), (name, i, fd, an)


def test_field_encoding_round_trip():
    """Models -> the 9 outputs -> models: B, gamma, phi (modulo 180) and the
    other parameters come back; azimuths either side of 0 / 180 map to
    neighbouring outputs."""
    rng = np.random.default_rng(3)
    m = H.truth_models(2000, rng)
    m[:, 1] = rng.uniform(10, 3000, len(m))
    m[:, 4] = np.maximum(m[:, 4], 1e-3)   # within the damping's range check
    back = M.outputs_to_models(M.targets(m), H.GUESS, (1,) * 11)
    for i in (0, 1, 2, 3, 4, 7, 8):
        np.testing.assert_allclose(back[:, i], m[:, i], rtol=1e-9, atol=1e-9)
    assert np.max(H.angle_diff(back[:, 5], m[:, 5], 360)) < 1e-7
    assert np.max(H.angle_diff(back[:, 6], m[:, 6], 180)) < 1e-7
    a = np.array([[20, 1000, 0, 0.03, 0.1, 60, 0.01, 0.3, 0.7, 0, 1],
                  [20, 1000, 0, 0.03, 0.1, 60, 179.99, 0.3, 0.7, 0, 1]], dtype=float)
    t = M.targets(a)
    assert np.abs(t[0] - t[1]).max() < 1.0


def test_fixed_parameters_come_from_the_guess():
    y = M.targets(H.truth_models(10, np.random.default_rng(4)))
    fix = (1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 1)
    m = M.outputs_to_models(y, H.GUESS, fix)
    assert (m[:, 7] == H.GUESS[7]).all() and (m[:, 8] == H.GUESS[8]).all()
    assert (m[:, 9] == H.GUESS[9]).all() and (m[:, 10] == H.GUESS[10]).all()


def test_mlp_init_on_the_host():
    net = G.mlp_new(30, 7)
    a = net.arrays()
    assert net.nl == 30 and net.steps == 0 and net.abi_version == G.ABI_VERSION
    assert (a["w1"][:, 120:] == 0).all() and (a["in_scale"][:120] == 1).all() and (a["in_scale"][120:] == 0).all()
    # uniform weights of variance 2 / fan-in; the output layer a tenth of that scale
    assert abs(a["w1"][:, :120].var() * 120 / 2 - 1) < 0.05
    assert abs(a["w2"].var() * 256 / 2 - 1) < 0.05
    assert abs(a["w3"].var() * 256 / 2 * 100 - 1) < 0.2
    assert (a["b1"] == 0).all() and (a["b2"] == 0).all()
    same = G.mlp_new(30, 7).arrays()
    np.testing.assert_array_equal(a["w2"], same["w2"])
    with pytest.raises(G.GmError):
        G.mlp_new(33)


def test_fp64_gradients_match_torch_autograd():
    """The restatement's backward pass (without the BF16 roundings) against
    torch's automatic differentiation of the same network in FP64."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    p = M.params(random_net(9))
    X = rng.normal(0, 1, (64, M.IN))
    X[:, 120:] = 0.0
    Y = rng.normal(0, 1, (64, M.OUT))
    loss, g = M.loss_and_grads(p, X, Y, quantize=False)
    t = {k: torch.tensor(p[k], dtype=torch.float64, requires_grad=True) for k in ("w1", "b1", "w2", "b2", "w3")}
    t["b3"] = torch.tensor(p["b3"][:M.OUT], dtype=torch.float64, requires_grad=True)
    gelu = lambda z: 0.5 * z * (1 + torch.tanh(np.sqrt(2.0 / np.pi) * (z + 0.044715 * z ** 3)))
    h1 = gelu(torch.tensor(X) @ t["w1"].T + t["b1"])
    h2 = gelu(h1 @ t["w2"].T + t["b2"])
    out = h2 @ t["w3"].T + t["b3"]
    lt = ((out - torch.tensor(Y)) ** 2).mean()
    lt.backward()
    assert lt.item() == pytest.approx(loss, rel=1e-12)
    for k in t:
        np.testing.assert_allclose(g[k], t[k].grad.numpy(), rtol=1e-9, atol=1e-12, err_msg=k)
