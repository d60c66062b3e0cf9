"""CPU: the network oracle (oracle/cnn_oracle.py) pinned before it checks the GPU kernels.

The learned warm start has no counterpart in the reference, so the convolution and its
adjoints are pinned against torch's CPU conv3d and autograd (float64), and the composed
U-Net gradient against central differences of its own loss.
"""
import numpy as np
import pytest
import torch

from oracle import cnn_oracle as C


@pytest.mark.parametrize("s", [1, 2])
@pytest.mark.parametrize("shape", [(2, 3, 5, 6, 7), (1, 2, 8, 4, 4)])
def test_conv3d_and_adjoints_match_torch(s, shape):
    rng = np.random.default_rng(7 + s)
    N, Ci = shape[:2]
    Co = 4
    x = rng.normal(size=shape)
    w = rng.normal(size=(Co, Ci, 3, 3, 3))
    b = rng.normal(size=Co)
    xt, wt, bt = (torch.tensor(a, requires_grad=True) for a in (x, w, b))
    y = torch.nn.functional.conv3d(xt, wt, bt, stride=s, padding=1)
    yo = C.conv3d(x, w, b, s)
    assert yo.shape == tuple(y.shape)
    assert np.allclose(yo, y.detach().numpy(), rtol=1e-12, atol=1e-12)
    assert np.allclose(C.conv3d(x, w, b, s, relu=True), np.maximum(y.detach().numpy(), 0), atol=1e-12)
    dy = rng.normal(size=yo.shape)
    y.backward(torch.tensor(dy))
    assert np.allclose(C.conv3d_bwd_data(dy, w, x.shape, s), xt.grad.numpy(), atol=1e-11)
    dw, db = C.conv3d_bwd_weight(x, dy, s)
    assert np.allclose(dw, wt.grad.numpy(), atol=1e-11)
    assert np.allclose(db, bt.grad.numpy(), atol=1e-11)


def test_upsample_cell2node_adjoints():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(2, 3, 2, 3, 4))
    y = rng.normal(size=(2, 3, 4, 6, 8))
    assert np.isclose(np.sum(C.upsample2(x) * y), np.sum(x * C.upsample2_bwd(y)))
    xt = torch.tensor(x)
    assert np.array_equal(C.upsample2(x), torch.nn.functional.interpolate(xt, scale_factor=2, mode="nearest").numpy())
    cells = rng.normal(size=(2, 3, 3, 2, 4))
    nodes = rng.normal(size=(2, 4 * 3 * 5, 3))
    assert np.isclose(np.sum(C.cell2node(cells) * nodes), np.sum(cells * C.cell2node_bwd(nodes, 3, 2, 4)))
    # a constant cell field is reproduced at every node
    const = np.broadcast_to(np.array([1.0, -2.0, 0.5]).reshape(1, 3, 1, 1, 1), (1, 3, 3, 2, 4))
    assert np.allclose(C.cell2node(np.ascontiguousarray(const)), np.array([1.0, -2.0, 0.5]))


def _tiny_net(rng, ch=(2, 2, 4, 4)):
    c1, c2, c3, c4 = ch
    spec = [("c1a", 8, c1), ("c1b", c1, c1), ("c2a", c1, c2), ("c2b", c2, c2), ("c3a", c2, c3), ("c4a", c3, c4),
            ("d3", c4 + c3 + c4, c3), ("d2", c3 + c2, c2), ("d1", c2 + c1, c1), ("out", c1, 3)]
    W = {n: rng.normal(size=(co, ci, 3, 3, 3)) * np.sqrt(2.0 / (ci * 27)) for n, ci, co in spec}
    B = {n: rng.normal(size=co) * 0.1 for n, ci, co in spec}
    return W, B


def test_unet_gradient_central_differences():
    rng = np.random.default_rng(11)
    W, B = _tiny_net(rng)
    x = rng.normal(size=(1, 8, 8, 8, 8))
    t = rng.normal(size=(1, 9 * 9 * 9, 3))
    loss, dW, dB = C.unet_loss_grad(W, B, x, t)
    h = 1e-6
    for name in ("c1a", "c2a", "c4a", "d3", "d1", "out"):
        for _ in range(2):
            idx = tuple(int(rng.integers(n)) for n in W[name].shape)
            W[name][idx] += h
            lp = C.unet_loss_grad(W, B, x, t)[0]
            W[name][idx] -= 2 * h
            lm = C.unet_loss_grad(W, B, x, t)[0]
            W[name][idx] += h
            fd = (lp - lm) / (2 * h)
            assert abs(fd - dW[name][idx]) < 1e-6 * max(1.0, abs(fd)), (name, idx, fd, dW[name][idx])
        k = int(rng.integers(B[name].shape[0]))
        B[name][k] += h
        lp = C.unet_loss_grad(W, B, x, t)[0]
        B[name][k] -= 2 * h
        lm = C.unet_loss_grad(W, B, x, t)[0]
        B[name][k] += h
        assert abs((lp - lm) / (2 * h) - dB[name][k]) < 1e-6 * max(1.0, abs(dB[name][k]))


def test_features_and_guess_small():
    nel = (4, 4, 8)
    rng = np.random.default_rng(5)
    E = rng.uniform(0.1, 1.0, size=np.prod(nel))
    nn = 5 * 5 * 9
    f = np.zeros(nn * 3)
    f[3 * 7 + 1] = -2.0
    f[3 * 8] = 1.0
    mask = np.zeros(nn, dtype=np.uint8)
    mask[:9] = 7
    F1 = C.features(nel, 1, E, f, mask)
    F2 = C.features(nel, 2, E, f, mask)
    # pooling keeps the total force (over max |f|) and the block-mean stiffness
    assert np.allclose(F1[1:4].sum(axis=(1, 2, 3)), F2[1:4].sum(axis=(1, 2, 3)))
    assert np.allclose(F1[1:4].sum(axis=(1, 2, 3)), [0.5, -1.0, 0.0])
    assert np.allclose(F2[0] ** 3, (F1[0] ** 3).reshape(2, 2, 2, 2, 4, 2).mean(axis=(1, 3, 5)))
    assert np.allclose(F2[5, :, 0, 0], [-0.5, 0.5]) and np.allclose(F1[7, 0, 0, :], (2 * np.arange(8) + 1) / 8 - 1)
    # a linear coarse field is interpolated exactly
    cn = np.array([[i + 2 * j - k, 1.0, j] for j in range(3) for i in range(3) for k in range(5)], dtype=np.float64)
    g = C.guess(nel, 2, cn.reshape(-1), None).reshape(-1, 3)
    fine = np.array([[i / 2 + j - k / 2, 1.0, j / 2] for j in range(5) for i in range(5) for k in range(9)])
    assert np.allclose(g, fine)
