"""numpy restatement of the learned warm start's network operations (float64).

TEST INFRASTRUCTURE ONLY: the checker of the library's convolution kernels and of the
network's gradients (tests/test_cnn_gpu.py); the library never imports it.  The network is
a form of this library with no counterpart in the reference, so these restate the plain
definitions: 3x3x3 convolution with zero padding 1 and stride s, its exact adjoints with
respect to input and weights, nearest 2x upsampling, channel concatenation, channel means,
cell-to-node averaging and the mean-squared error, the composed U-Net, the input features
and the interpolated guess.  tests/test_cnn_oracle.py pins the convolution against torch's
CPU conv3d and the composed gradient against central differences.

Layout: [N][C][X][Y][Z]; weights [Cout][Cin][3][3][3].
"""
from __future__ import annotations

import numpy as np


def _out(n, s):
    return (n - 1) // s + 1


def conv3d(x, w, b, s=1, relu=False):
    N, C, X, Y, Z = x.shape
    Co = w.shape[0]
    Xo, Yo, Zo = _out(X, s), _out(Y, s), _out(Z, s)
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    y = np.broadcast_to(b.reshape(1, Co, 1, 1, 1), (N, Co, Xo, Yo, Zo)).astype(np.float64).copy()
    for tx in range(3):
        for ty in range(3):
            for tz in range(3):
                sl = xp[:, :, tx:tx + s * (Xo - 1) + 1:s, ty:ty + s * (Yo - 1) + 1:s, tz:tz + s * (Zo - 1) + 1:s]
                y += np.einsum("oc,ncxyz->noxyz", w[:, :, tx, ty, tz], sl)
    return np.maximum(y, 0.0) if relu else y


def conv3d_bwd_data(dy, w, xshape, s=1):
    N, C, X, Y, Z = xshape
    Xo, Yo, Zo = dy.shape[2:]
    dxp = np.zeros((N, C, X + 2, Y + 2, Z + 2))
    for tx in range(3):
        for ty in range(3):
            for tz in range(3):
                dxp[:, :, tx:tx + s * (Xo - 1) + 1:s, ty:ty + s * (Yo - 1) + 1:s, tz:tz + s * (Zo - 1) + 1:s] += \
                    np.einsum("oc,noxyz->ncxyz", w[:, :, tx, ty, tz], dy)
    return dxp[:, :, 1:-1, 1:-1, 1:-1]


def conv3d_bwd_weight(x, dy, s=1):
    N, C, X, Y, Z = x.shape
    Co = dy.shape[1]
    Xo, Yo, Zo = dy.shape[2:]
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    dw = np.zeros((Co, C, 3, 3, 3))
    for tx in range(3):
        for ty in range(3):
            for tz in range(3):
                sl = xp[:, :, tx:tx + s * (Xo - 1) + 1:s, ty:ty + s * (Yo - 1) + 1:s, tz:tz + s * (Zo - 1) + 1:s]
                dw[:, :, tx, ty, tz] = np.einsum("noxyz,ncxyz->oc", dy, sl)
    return dw, dy.sum(axis=(0, 2, 3, 4))


def upsample2(x):
    return x.repeat(2, axis=2).repeat(2, axis=3).repeat(2, axis=4)


def upsample2_bwd(dy):
    N, C, X2, Y2, Z2 = dy.shape
    return dy.reshape(N, C, X2 // 2, 2, Y2 // 2, 2, Z2 // 2, 2).sum(axis=(3, 5, 7))


def _node_cells(X, Y, Z):
    """For each node (structured-mesh order k + nz*(i + nx*j)) the list of adjacent cells."""
    nx, ny, nz = X + 1, Y + 1, Z + 1
    out = []
    for j in range(ny):
        for i in range(nx):
            for k in range(nz):
                cells = [(i + a, j + b, k + c) for a in (-1, 0) for b in (-1, 0) for c in (-1, 0)
                         if 0 <= i + a < X and 0 <= j + b < Y and 0 <= k + c < Z]
                out.append(cells)
    return out


def cell2node(cells):
    """[N][3][X][Y][Z] -> [N][nodes][3] (mean of adjacent cells)."""
    N, _, X, Y, Z = cells.shape
    nc = _node_cells(X, Y, Z)
    out = np.zeros((N, len(nc), 3))
    for m, cl in enumerate(nc):
        for (cx, cy, cz) in cl:
            out[:, m, :] += cells[:, :, cx, cy, cz]
        out[:, m, :] /= len(cl)
    return out


def cell2node_bwd(dnode, X, Y, Z):
    N = dnode.shape[0]
    nc = _node_cells(X, Y, Z)
    dcell = np.zeros((N, 3, X, Y, Z))
    for m, cl in enumerate(nc):
        for (cx, cy, cz) in cl:
            dcell[:, :, cx, cy, cz] += dnode[:, m, :] / len(cl)
    return dcell


def mse(pred, target):
    d = pred - target
    return float(np.mean(d * d)), 2.0 * d / d.size


def relu_bwd(y, dy):
    return np.where(y > 0, dy, 0.0)


def unet_loss_grad(W, B, x, target):
    """The warm-start U-Net (encoder c1a c1b | c2a(s2) c2b | c3a(s2) | c4a(s2), decoder
    d3 d2 d1 on [up2(lower), skip] concatenations - d3's also carries the channel mean of
    c4a broadcast over the grid - linear 3-channel output, outputs averaged to nodes) and
    the node MSE against ``target`` [N, nodes, 3].  W, B: dicts of weights/biases by layer
    name.  Returns (loss, dW, dB)."""
    st = {"c2a": 2, "c3a": 2, "c4a": 2}
    a = {}
    a["c1a"] = conv3d(x, W["c1a"], B["c1a"], 1, True)
    a["c1b"] = conv3d(a["c1a"], W["c1b"], B["c1b"], 1, True)
    a["c2a"] = conv3d(a["c1b"], W["c2a"], B["c2a"], 2, True)
    a["c2b"] = conv3d(a["c2a"], W["c2b"], B["c2b"], 1, True)
    a["c3a"] = conv3d(a["c2b"], W["c3a"], B["c3a"], 2, True)
    a["c4a"] = conv3d(a["c3a"], W["c4a"], B["c4a"], 2, True)
    gctx = a["c4a"].mean(axis=(2, 3, 4))
    a["cat3"] = np.concatenate([upsample2(a["c4a"]), a["c3a"],
                                np.broadcast_to(gctx[:, :, None, None, None], a["c3a"].shape[:1] + gctx.shape[1:2]
                                                + a["c3a"].shape[2:])], axis=1)
    a["d3"] = conv3d(a["cat3"], W["d3"], B["d3"], 1, True)
    a["cat2"] = np.concatenate([upsample2(a["d3"]), a["c2b"]], axis=1)
    a["d2"] = conv3d(a["cat2"], W["d2"], B["d2"], 1, True)
    a["cat1"] = np.concatenate([upsample2(a["d2"]), a["c1b"]], axis=1)
    a["d1"] = conv3d(a["cat1"], W["d1"], B["d1"], 1, True)
    out = conv3d(a["d1"], W["out"], B["out"], 1, False)
    X, Y, Z = x.shape[2:]
    nodes = cell2node(out)
    loss, gn = mse(nodes, target)
    dW, dB = {}, {}
    g = cell2node_bwd(gn, X, Y, Z)

    def back(name, xin, gy, relu_out=None):
        if relu_out is not None:
            gy = relu_bwd(relu_out, gy)
        dW[name], dB[name] = conv3d_bwd_weight(xin, gy, st.get(name, 1))
        return conv3d_bwd_data(gy, W[name], xin.shape, st.get(name, 1))

    g = back("out", a["d1"], g)
    g = back("d1", a["cat1"], g, a["d1"])
    c = a["d2"].shape[1]
    g_d2, g_e1 = upsample2_bwd(g[:, :c]), g[:, c:]
    g = back("d2", a["cat2"], g_d2, a["d2"])
    c = a["d3"].shape[1]
    g_d3, g_e2 = upsample2_bwd(g[:, :c]), g[:, c:]
    g = back("d3", a["cat3"], g_d3, a["d3"])
    c, c3 = a["c4a"].shape[1], a["c3a"].shape[1]
    g_e4, g_e3 = upsample2_bwd(g[:, :c]), g[:, c:c + c3]
    V4 = np.prod(a["c4a"].shape[2:])
    g_e4 = g_e4 + (g[:, c + c3:].sum(axis=(2, 3, 4)) / V4)[:, :, None, None, None]
    g_e3 = g_e3 + back("c4a", a["c3a"], g_e4, a["c4a"])
    g_e2 = g_e2 + back("c3a", a["c2b"], g_e3, a["c3a"])
    g = back("c2b", a["c2a"], g_e2, a["c2b"])
    g_e1 = g_e1 + back("c2a", a["c1b"], g, a["c2a"])
    g = back("c1b", a["c1a"], g_e1, a["c1b"])
    back("c1a", x, g, a["c1a"])
    return loss, dW, dB


def features(nel, P, E, f, node_mask):
    """Network input [8, X/P, Y/P, Z/P] of one sample: E^(1/3) of the block mean; forces
    of the closed node box of each block (nodes shared with a neighbouring block count
    half per shared axis) over max |f|; constrained fraction of the 24 corner DOFs;
    cell-centre coordinates scaled to (-1, 1)."""
    FX, FY, FZ = nel
    X, Y, Z = FX // P, FY // P, FZ // P
    nx, nz = FX + 1, FZ + 1
    Eb = E.reshape(FX, FY, FZ).reshape(X, P, Y, P, Z, P).mean(axis=(1, 3, 5))
    out = np.zeros((8, X, Y, Z))
    out[0] = np.cbrt(Eb)
    out[5] = ((2 * np.arange(X) + 1) / X - 1)[:, None, None]
    out[6] = ((2 * np.arange(Y) + 1) / Y - 1)[None, :, None]
    out[7] = ((2 * np.arange(Z) + 1) / Z - 1)[None, None, :]
    fm = np.abs(f).max()
    fs = 1.0 / fm if fm > 0 else 0.0
    fn = f.reshape(-1, 3)
    mask = np.zeros(fn.shape[0], dtype=np.int64) if node_mask is None else node_mask.astype(np.int64)
    bits = (mask & 1) + ((mask >> 1) & 1) + ((mask >> 2) & 1)
    for cx in range(X):
        for cy in range(Y):
            for cz in range(Z):
                s = np.zeros(3)
                for a in range(P + 1):
                    i = P * cx + a
                    wa = 0.5 if (a in (0, P) and 0 < i < FX) else 1.0
                    for b in range(P + 1):
                        j = P * cy + b
                        wb = wa * (0.5 if (b in (0, P) and 0 < j < FY) else 1.0)
                        for d in range(P + 1):
                            k = P * cz + d
                            w = wb * (0.5 if (d in (0, P) and 0 < k < FZ) else 1.0)
                            s += w * fn[k + nz * (i + nx * j)]
                out[1:4, cx, cy, cz] = s * fs
                ncon = 0
                for a in (0, 1):
                    for b in (0, 1):
                        for d in (0, 1):
                            ncon += bits[P * (cz + d) + nz * (P * (cx + a) + nx * P * (cy + b))]
                out[4, cx, cy, cz] = ncon / 24.0
    return out


def guess(nel, P, coarse_nodes, node_mask):
    """Trilinear interpolation of the nodal field of the mesh nel / P onto the mesh nel,
    zero where node_mask has the component's bit."""
    FX, FY, FZ = nel
    X, Y, Z = FX // P, FY // P, FZ // P
    c = coarse_nodes.reshape(Y + 1, X + 1, Z + 1, 3)  # node k + nz (i + nx j): j slowest
    out = np.zeros((FY + 1, FX + 1, FZ + 1, 3))
    for j in range(FY + 1):
        j0 = min(j // P, Y - 1)
        tj = (j - P * j0) / P
        for i in range(FX + 1):
            i0 = min(i // P, X - 1)
            ti = (i - P * i0) / P
            for k in range(FZ + 1):
                k0 = min(k // P, Z - 1)
                tk = (k - P * k0) / P
                s = np.zeros(3)
                for a in (0, 1):
                    for b in (0, 1):
                        for d in (0, 1):
                            w = (ti if a else 1 - ti) * (tj if b else 1 - tj) * (tk if d else 1 - tk)
                            s += w * c[j0 + b, i0 + a, k0 + d]
                out[j, i, k] = s
    out = out.reshape(-1, 3)
    if node_mask is not None:
        for e in range(3):
            out[(node_mask.astype(np.int64) >> e) & 1 == 1, e] = 0.0
    return out.reshape(-1)
