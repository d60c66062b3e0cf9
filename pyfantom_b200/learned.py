"""Learned warm start for the MGCG solve: a small 3D U-Net run by the library's own kernels.

The network maps what the solver is given - the element stiffness E, the nodal load f and
the Dirichlet mask - to the displacement field, on a cell grid.  Its output is used as the
initial guess of the preconditioned CG (``MultiGrid(..., warm_start=LearnedWarmStart(net))``):
the guess is interpolated to the mesh, zeroed on constrained DOFs and scaled by the
energy-optimal factor alpha = (x0.b) / (x0.K x0), so its energy error is never larger than
that of the zero start; the plain MGCG then runs to the same tolerance from it.  A mesh
finer than the training grid is seen through block pooling (``pool=P``: the cell grid has
nel / P cells) and the prediction is interpolated back trilinearly.

Architecture (``channels=(c1, c2, c3, c4)``, default (16, 32, 64, 48), 571,859 parameters),
every convolution 3x3x3 with zero padding 1, ReLU after all but the last:

    input 8 ch   -> c1a(c1) -> c1b(c1) = e1                   [X, Y, Z]
    e1 -stride 2-> c2a(c2) -> c2b(c2) = e2                    [X/2 ...]
    e2 -stride 2-> c3a(c3) = e3                               [X/4 ...]
    e3 -stride 2-> c4a(c4) = e4                               [X/8 ...]
    [up2(e4), e3, g] -> d3(c3);  [up2(d3), e2] -> d2(c2);  [up2(d2), e1] -> d1(c1) -> out(3)

where g is the channel mean of e4 broadcast over the grid.  The inputs are E^(1/3), the
load, the Dirichlet fraction and the cell-centre coordinates; the coordinates and the
global context g let the field at one end of the mesh depend on a load at the other,
beyond the roughly 40-cell receptive field of the convolutions.

Cell outputs become nodal displacements by averaging the adjacent cells.  Two training
losses are available.  ``energy`` (the default) is what the CG pays for: the relative
energy error left after the energy-optimal scaling, 1 - (b.y)^2 / ((y.Ky) b.u) by the
Rayleigh-Ritz principle, evaluated with one stiffness matvec per sample
(``pf_cnn_energy_loss_f64``).  ``mse`` is the mean-squared error against solver
displacements normalised to unit RMS per sample.  Forward, backward (input and weight
gradients), the losses and the Adam update are the ``pf_cnn_*`` kernels; torch only
holds the buffers.  This form has no counterpart in the reference.
"""
from __future__ import annotations

import ctypes
import math
import os
import time

import numpy as np
import torch

from . import _lib
from ._tensor import as_cuda, device

__all__ = ["WarmStartNet", "LearnedWarmStart", "EnergyLoss", "make_dataset", "random_edge_load",
           "cantilever_constraints", "edge_load_rhs", "DEFAULT_WEIGHTS"]

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_unet_64x32x32.npz")
N_IN = 8


def _p(t):
    return _lib.ptr(t)


class WarmStartNet:
    """The U-Net, its flat float32 parameters, Adam state and activation buffers."""

    def __init__(self, channels=(16, 32, 64, 48), seed: int = 0, tensor_cores: bool = True):
        c1, c2, c3, c4 = (int(c) for c in channels)
        # convolutions on the tensor cores (BF16 operands, FP32 accumulation) or on the
        # CUDA cores in FP32 (the exact path the gradient checks use)
        self.tensor_cores = bool(tensor_cores)
        self.channels = (c1, c2, c3, c4)
        # name, Cin, Cout, stride, relu
        self.layers = [
            ("c1a", N_IN, c1, 1, 1), ("c1b", c1, c1, 1, 1),
            ("c2a", c1, c2, 2, 1), ("c2b", c2, c2, 1, 1),
            ("c3a", c2, c3, 2, 1), ("c4a", c3, c4, 2, 1),
            ("d3", c4 + c3 + c4, c3, 1, 1), ("d2", c3 + c2, c2, 1, 1), ("d1", c2 + c1, c1, 1, 1),
            ("out", c1, 3, 1, 0),
        ]
        self.spec = {}
        off = 0
        for name, ci, co, s, r in self.layers:
            nw = co * ci * 27
            self.spec[name] = (ci, co, s, r, off, off + nw)
            off += nw + co
        self.n_params = off
        rng = np.random.default_rng(seed)
        p = np.zeros(off, dtype=np.float32)
        for name, ci, co, s, r in self.layers:
            _, _, _, _, ow, ob = self.spec[name]
            fan_in = ci * 27
            bound = math.sqrt(6.0 / fan_in) if r else math.sqrt(1.0 / fan_in)
            p[ow:ob] = rng.uniform(-bound, bound, size=ob - ow)
        dev = device()
        self.params = torch.from_numpy(p).to(dev)
        self.grad = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        wmax = max(co * ci for _, ci, co, _, _ in self.layers)
        self._wwork = torch.empty(int(_lib.load().pf_cnn_conv3d_bwd_weight_workspace(wmax, 1)), dtype=torch.float32,
                                  device=dev)
        self._tc_err = torch.zeros(1, dtype=torch.int32, device=dev)
        self._tc_work = {}
        self._bufs = {}

    def tensor_core_errors(self):
        """Number of tensor-core convolutions that gave up waiting since the last call
        (0 in normal operation; their outputs were not written).  Reads one device int."""
        e = int(self._tc_err.item())
        self._tc_err.zero_()
        return e

    # ---- parameters -----------------------------------------------------------------
    def w(self, name):
        _, _, _, _, ow, ob = self.spec[name]
        return self.params[ow:ob]

    def b(self, name):
        ci, co, _, _, ow, ob = self.spec[name]
        return self.params[ob:ob + co]

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), channels=np.array(self.channels))

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, tensor_cores: bool = True):
        z = np.load(path)
        net = cls(channels=tuple(int(c) for c in z["channels"]), tensor_cores=tensor_cores)
        if z["params"].shape[0] != net.n_params:
            raise ValueError("weight file does not match the architecture")
        net.params.copy_(torch.from_numpy(z["params"]))
        return net

    # ---- buffers --------------------------------------------------------------------
    def _buffers(self, N, X, Y, Z):
        key = (N, X, Y, Z)
        if key in self._bufs:
            return self._bufs[key]
        if X % 8 or Y % 8 or Z % 8:
            raise ValueError("the network needs a cell grid divisible by 8 along every axis")
        c1, c2, c3, c4 = self.channels
        dev = device()
        s1, s2, s3, s4 = (X, Y, Z), (X // 2, Y // 2, Z // 2), (X // 4, Y // 4, Z // 4), (X // 8, Y // 8, Z // 8)

        def t(c, s):
            return torch.empty((N, c) + s, dtype=torch.float32, device=dev)

        b = dict(c1a=t(c1, s1), c1b=t(c1, s1), c2a=t(c2, s2), c2b=t(c2, s2), c3a=t(c3, s3), c4a=t(c4, s4),
                 cat3=t(c4 + c3 + c4, s3), d3=t(c3, s3), cat2=t(c3 + c2, s2), d2=t(c2, s2), cat1=t(c2 + c1, s1),
                 d1=t(c1, s1), out=t(3, s1), up3=t(c4, s3), up2=t(c3, s2), up1=t(c2, s1),
                 nodes=torch.empty((N, (X + 1) * (Y + 1) * (Z + 1) * 3), dtype=torch.float32, device=dev),
                 gctx=torch.empty((N, c4), dtype=torch.float32, device=dev))
        # gradient buffers
        for k in ("c1a", "c1b", "c2a", "c2b", "c3a", "c4a", "cat3", "d3", "cat2", "d2", "cat1", "d1", "out", "up3",
                  "up2", "up1", "nodes", "gctx"):
            b["g_" + k] = torch.empty_like(b[k])
        b["mse"] = torch.empty(int(_lib.load().pf_cnn_mse_workspace(b["nodes"].numel())), dtype=torch.float64,
                               device=dev)
        self._bufs[key] = b
        return b

    # ---- forward --------------------------------------------------------------------
    def _conv(self, name, x, y):
        ci, co, s, r, _, _ = self.spec[name]
        N, _, X, Y, Z = x.shape
        L = _lib.load()
        if self.tensor_cores:
            _lib.check(L.pf_cnn_conv3d_fwd_tc(_p(x), N, ci, X, Y, Z, _p(self.w(name)), _p(self.b(name)), co, s, r,
                                              _p(y), _p(self._tc_err), _lib.stream()))
        else:
            _lib.check(L.pf_cnn_conv3d_fwd_f32(_p(x), N, ci, X, Y, Z, _p(self.w(name)), _p(self.b(name)), co, s, r,
                                               _p(y), _lib.stream()))

    def _up_cat(self, src, up, cat, c_off_skip, skip):
        """cat[:, :C] = up2(src), cat[:, c_off_skip:c_off_skip + Cskip] = skip."""
        L = _lib.load()
        N, C, X, Y, Z = src.shape
        V = cat.shape[2] * cat.shape[3] * cat.shape[4]
        if N == 1:  # the first C channels of cat are contiguous
            _lib.check(L.pf_cnn_upsample2_f32(C, X, Y, Z, _p(src), _p(cat), 0, _lib.stream()))
        else:
            _lib.check(L.pf_cnn_upsample2_f32(N * C, X, Y, Z, _p(src), _p(up), 0, _lib.stream()))
            _lib.check(L.pf_cnn_copy_channels_f32(N, C, V, _p(up), cat.shape[1], 0, 0, 0, _p(cat), _lib.stream()))
        _lib.check(L.pf_cnn_copy_channels_f32(N, skip.shape[1], V, _p(skip), cat.shape[1], c_off_skip, 0, 0, _p(cat),
                                              _lib.stream()))

    def forward(self, x):
        """Cell outputs [N, 3, X, Y, Z] for inputs [N, 8, X, Y, Z] (buffers are reused)."""
        N, C, X, Y, Z = x.shape
        if C != N_IN or x.dtype != torch.float32 or not x.is_contiguous():
            raise ValueError("input must be a contiguous float32 tensor [N, 8, X, Y, Z]")
        b = self._buffers(N, X, Y, Z)
        c1, c2, c3, c4 = self.channels
        L = _lib.load()
        self._conv("c1a", x, b["c1a"])
        self._conv("c1b", b["c1a"], b["c1b"])
        self._conv("c2a", b["c1b"], b["c2a"])
        self._conv("c2b", b["c2a"], b["c2b"])
        self._conv("c3a", b["c2b"], b["c3a"])
        self._conv("c4a", b["c3a"], b["c4a"])
        self._up_cat(b["c4a"], b["up3"], b["cat3"], c4, b["c3a"])
        V4, V3 = b["c4a"][0, 0].numel(), b["c3a"][0, 0].numel()
        _lib.check(L.pf_cnn_channel_sum_f32(N, c4, V4, _p(b["c4a"]), c4, 0, 1.0 / V4, _p(b["gctx"]), _lib.stream()))
        _lib.check(L.pf_cnn_channel_bcast_f32(N, c4, V3, _p(b["gctx"]), 1.0, c4 + c3 + c4, c4 + c3, 0, _p(b["cat3"]),
                                              _lib.stream()))
        self._conv("d3", b["cat3"], b["d3"])
        self._up_cat(b["d3"], b["up2"], b["cat2"], c3, b["c2b"])
        self._conv("d2", b["cat2"], b["d2"])
        self._up_cat(b["d2"], b["up1"], b["cat1"], c2, b["c1b"])
        self._conv("d1", b["cat1"], b["d1"])
        self._conv("out", b["d1"], b["out"])
        self._x = x
        return b["out"]

    def predict_nodes(self, x):
        """Nodal displacements [N, nodes * 3] (node order of the structured mesh)."""
        out = self.forward(x)
        N, _, X, Y, Z = out.shape
        b = self._buffers(N, X, Y, Z)
        _lib.check(_lib.load().pf_cnn_cell2node_f32(N, X, Y, Z, _p(out), _p(b["nodes"]), 0, _lib.stream()))
        return b["nodes"]

    # ---- backward -------------------------------------------------------------------
    def _wgrad(self, name, x, dy):
        ci, co, s, _, ow, ob = self.spec[name]
        N, _, X, Y, Z = x.shape
        L = _lib.load()
        if self.tensor_cores:
            key = (name, N, X, Y, Z)
            if key not in self._tc_work:
                n = int(L.pf_cnn_conv3d_bwd_weight_tc_workspace(N, ci, X, Y, Z, co, s))
                self._tc_work[key] = torch.empty(n, dtype=torch.float32, device=device())
            _lib.check(L.pf_cnn_conv3d_bwd_weight_tc(_p(x), _p(dy), N, ci, X, Y, Z, co, s, _p(self.grad[ow:ob]),
                                                     _p(self.grad[ob:ob + co]), _p(self._tc_work[key]),
                                                     _p(self._tc_err), _lib.stream()))
        else:
            _lib.check(L.pf_cnn_conv3d_bwd_weight_f32(_p(x), _p(dy), N, ci, X, Y, Z, co, s, _p(self.grad[ow:ob]),
                                                      _p(self.grad[ob:ob + co]), _p(self._wwork), _lib.stream()))

    def _dgrad(self, name, dy, xshape, dx, accumulate=0):
        ci, co, s, _, _, _ = self.spec[name]
        N, _, X, Y, Z = xshape
        L = _lib.load()
        if self.tensor_cores:
            _lib.check(L.pf_cnn_conv3d_bwd_data_tc(_p(dy), N, ci, X, Y, Z, _p(self.w(name)), co, s, accumulate,
                                                   _p(dx), _p(self._tc_err), _lib.stream()))
        else:
            _lib.check(L.pf_cnn_conv3d_bwd_data_f32(_p(dy), N, ci, X, Y, Z, _p(self.w(name)), co, s, accumulate,
                                                    _p(dx), _lib.stream()))

    def _relu_bwd(self, y, dy):
        _lib.check(_lib.load().pf_cnn_relu_bwd_f32(y.numel(), _p(y), _p(dy), _lib.stream()))

    def _split_cat(self, gcat, gup, src_shape, gsrc, c_off_skip, gskip):
        """gsrc = up2^T(gcat[:, :C]); gskip = gcat[:, c_off_skip:c_off_skip + Cskip] (overwrites both)."""
        L = _lib.load()
        N, C, X, Y, Z = src_shape
        V = gcat.shape[2] * gcat.shape[3] * gcat.shape[4]
        if N == 1:
            _lib.check(L.pf_cnn_upsample2_f32(C, X, Y, Z, _p(gcat), _p(gsrc), 1, _lib.stream()))
        else:
            _lib.check(L.pf_cnn_copy_channels_f32(N, C, V, _p(gcat), gcat.shape[1], 0, 0, 1, _p(gup), _lib.stream()))
            _lib.check(L.pf_cnn_upsample2_f32(N * C, X, Y, Z, _p(gup), _p(gsrc), 1, _lib.stream()))
        _lib.check(L.pf_cnn_copy_channels_f32(N, gskip.shape[1], V, _p(gcat), gcat.shape[1], c_off_skip, 0, 1,
                                              _p(gskip), _lib.stream()))

    def backward(self, g_out):
        """Parameter gradient (into ``self.grad``) for the output gradient [N, 3, X, Y, Z]
        of the last ``forward``."""
        x = self._x
        N, _, X, Y, Z = x.shape
        b = self._buffers(N, X, Y, Z)
        c1, c2, c3, c4 = self.channels
        L = _lib.load()
        self._wgrad("out", b["d1"], g_out)
        self._dgrad("out", g_out, b["d1"].shape, b["g_d1"])
        self._relu_bwd(b["d1"], b["g_d1"])
        self._wgrad("d1", b["cat1"], b["g_d1"])
        self._dgrad("d1", b["g_d1"], b["cat1"].shape, b["g_cat1"])
        self._split_cat(b["g_cat1"], b["g_up1"], b["d2"].shape, b["g_d2"], c2, b["g_c1b"])
        self._relu_bwd(b["d2"], b["g_d2"])
        self._wgrad("d2", b["cat2"], b["g_d2"])
        self._dgrad("d2", b["g_d2"], b["cat2"].shape, b["g_cat2"])
        self._split_cat(b["g_cat2"], b["g_up2"], b["d3"].shape, b["g_d3"], c3, b["g_c2b"])
        self._relu_bwd(b["d3"], b["g_d3"])
        self._wgrad("d3", b["cat3"], b["g_d3"])
        self._dgrad("d3", b["g_d3"], b["cat3"].shape, b["g_cat3"])
        self._split_cat(b["g_cat3"], b["g_up3"], b["c4a"].shape, b["g_c4a"], c4, b["g_c3a"])
        # global context: g = mean_v(e4) broadcast into cat3[:, c4 + c3:]
        V4, V3 = b["c4a"][0, 0].numel(), b["c3a"][0, 0].numel()
        _lib.check(L.pf_cnn_channel_sum_f32(N, c4, V3, _p(b["g_cat3"]), c4 + c3 + c4, c4 + c3, 1.0, _p(b["g_gctx"]),
                                            _lib.stream()))
        _lib.check(L.pf_cnn_channel_bcast_f32(N, c4, V4, _p(b["g_gctx"]), 1.0 / V4, c4, 0, 1, _p(b["g_c4a"]),
                                              _lib.stream()))
        # encoder: each level's gradient collects the skip path and the path below
        self._relu_bwd(b["c4a"], b["g_c4a"])
        self._wgrad("c4a", b["c3a"], b["g_c4a"])
        self._dgrad("c4a", b["g_c4a"], b["c3a"].shape, b["g_c3a"], accumulate=1)
        self._relu_bwd(b["c3a"], b["g_c3a"])
        self._wgrad("c3a", b["c2b"], b["g_c3a"])
        self._dgrad("c3a", b["g_c3a"], b["c2b"].shape, b["g_c2b"], accumulate=1)
        self._relu_bwd(b["c2b"], b["g_c2b"])
        self._wgrad("c2b", b["c2a"], b["g_c2b"])
        self._dgrad("c2b", b["g_c2b"], b["c2a"].shape, b["g_c2a"])
        self._relu_bwd(b["c2a"], b["g_c2a"])
        self._wgrad("c2a", b["c1b"], b["g_c2a"])
        self._dgrad("c2a", b["g_c2a"], b["c1b"].shape, b["g_c1b"], accumulate=1)
        self._relu_bwd(b["c1b"], b["g_c1b"])
        self._wgrad("c1b", b["c1a"], b["g_c1b"])
        self._dgrad("c1b", b["g_c1b"], b["c1a"].shape, b["g_c1a"])
        self._relu_bwd(b["c1a"], b["g_c1a"])
        self._wgrad("c1a", x, b["g_c1a"])
        return self.grad

    def loss_and_grad(self, x, target, loss_out):
        """Forward, node MSE against ``target`` [N, nodes * 3] into the device double
        ``loss_out`` (a 1-element float64 tensor view), and backward."""
        nodes = self.predict_nodes(x)
        N, _, X, Y, Z = x.shape
        b = self._buffers(N, X, Y, Z)
        L = _lib.load()
        _lib.check(L.pf_cnn_mse_f32(nodes.numel(), _p(nodes), _p(target), _p(b["g_nodes"]), _p(loss_out), _p(b["mse"]),
                                    _lib.stream()))
        _lib.check(L.pf_cnn_cell2node_f32(N, X, Y, Z, _p(b["g_nodes"]), _p(b["g_out"]), 1, _lib.stream()))
        return self.backward(b["g_out"])

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        _lib.check(_lib.load().pf_cnn_adam_f32(self.n_params, _p(self.params), _p(self.grad), _p(self.m), _p(self.v),
                                               lr, b1, b2, eps, self.step, _lib.stream()))

    def eval_loss(self, inputs, targets, batch=8):
        """Mean node MSE over a data set (forward only)."""
        S = inputs.shape[0]
        losses = torch.zeros(S // batch, dtype=torch.float64, device=inputs.device)
        L = _lib.load()
        for it in range(S // batch):
            xb = inputs[it * batch:(it + 1) * batch]
            yb = targets[it * batch:(it + 1) * batch]
            nodes = self.predict_nodes(xb)
            N, _, X, Y, Z = xb.shape
            b = self._buffers(N, X, Y, Z)
            _lib.check(L.pf_cnn_mse_f32(nodes.numel(), _p(nodes), _p(yb), None, _p(losses[it:it + 1]), _p(b["mse"]),
                                        _lib.stream()))
        return float(losses.mean())

    def energy_loss_and_grad(self, x, idx, energy, loss_out):
        """Forward, the energy-deficit loss of each sample (``energy``: an EnergyLoss over
        the data set, ``idx``: the samples' indices in it) into ``loss_out`` [N], and
        backward."""
        nodes = self.predict_nodes(x)
        N, _, X, Y, Z = x.shape
        b = self._buffers(N, X, Y, Z)
        for s, i in enumerate(idx):
            energy.sample(int(i), nodes[s], b["g_nodes"][s], loss_out[s:s + 1])
        _lib.check(_lib.load().pf_cnn_cell2node_f32(N, X, Y, Z, _p(b["g_nodes"]), _p(b["g_out"]), 1, _lib.stream()))
        return self.backward(b["g_out"])

    def eval_energy(self, inputs, energy, batch=8):
        """Mean energy deficit over a data set (forward only)."""
        S = inputs.shape[0]
        losses = torch.zeros(S, dtype=torch.float64, device=inputs.device)
        for it in range(S // batch):
            xb = inputs[it * batch:(it + 1) * batch]
            nodes = self.predict_nodes(xb)
            b = self._buffers(*xb.shape[:1], *xb.shape[2:])
            for s in range(batch):
                k = it * batch + s
                energy.sample(k, nodes[s], b["g_nodes"][s], losses[k:k + 1])
        return float(losses[:(S // batch) * batch].mean())

    # ---- training -------------------------------------------------------------------
    def fit(self, inputs, targets, epochs=20, batch=8, lr=1e-3, lr_final=1e-4, seed=0, log=None, energy=None):
        """Adam over ``inputs`` [S, 8, X, Y, Z] (device float32) on the node MSE against
        ``targets`` [S, nodes * 3], or on the energy deficit when ``energy`` (an EnergyLoss
        over the same samples) is given; cosine learning-rate decay from lr to lr_final.
        Returns the mean loss of every epoch."""
        S = inputs.shape[0]
        steps = S // batch
        gen = torch.Generator().manual_seed(seed)
        per = batch if energy is not None else 1
        losses = torch.zeros(epochs * steps * per, dtype=torch.float64, device=inputs.device)
        hist = []
        total = epochs * steps
        for ep in range(epochs):
            perm_h = torch.randperm(S, generator=gen)
            perm = perm_h.to(inputs.device)
            t0 = time.time()
            for it in range(steps):
                k = ep * steps + it
                idx = perm[it * batch:(it + 1) * batch]
                xb = inputs.index_select(0, idx)
                if energy is not None:
                    self.energy_loss_and_grad(xb, perm_h[it * batch:(it + 1) * batch].tolist(), energy,
                                              losses[k * per:(k + 1) * per])
                else:
                    yb = targets.index_select(0, idx)
                    self.loss_and_grad(xb, yb, losses[k:k + 1])
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * k / total))
                self.adam(lr=lr_k)
            hist.append(float(losses[ep * steps * per:(ep + 1) * steps * per].mean()))
            if self.tensor_cores and self.tensor_core_errors():
                raise RuntimeError("a tensor-core convolution gave up waiting during this epoch")
            if log is not None:
                log(f"epoch {ep + 1}/{epochs} loss {hist[-1]:.5f} ({time.time() - t0:.1f} s)")
        return hist


def random_edge_load(nel, rng):
    """A unit load of random direction spread uniformly over one of the 8 box edges that
    do not lie on the clamped face x = 0.  Returns (node ids, forces [n, 3])."""
    nelx, nely, nelz = nel
    nx, nz = nelx + 1, nelz + 1
    edges = []
    for j in (0, nely):  # edges along z on the face x = nelx
        edges.append([(nelx, j, k) for k in range(nelz + 1)])
    for k in (0, nelz):  # edges along y on the face x = nelx
        edges.append([(nelx, j, k) for j in range(nely + 1)])
    for j in (0, nely):  # edges along x
        for k in (0, nelz):
            edges.append([(i, j, k) for i in range(1, nelx + 1)])
    e = edges[int(rng.integers(len(edges)))]
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    ids = np.array([k + nz * (i + nx * j) for (i, j, k) in e], dtype=np.int64)
    return ids, np.tile(d / len(ids), (len(ids), 1))


def cantilever_constraints(nel):
    """DOF indices of the clamped face x = 0 of a structured H8 mesh."""
    nx, ny, nz = (n + 1 for n in nel)
    J, K = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    fixed = (K + nz * nx * J).reshape(-1)
    return (fixed[:, None] * 3 + np.arange(3)).reshape(-1)


def edge_load_rhs(nel, seed):
    """Load vector of ``random_edge_load`` drawn from ``default_rng(seed)``."""
    nx, ny, nz = (n + 1 for n in nel)
    ids, F = random_edge_load(nel, np.random.default_rng(seed))
    f = np.zeros(3 * nx * ny * nz)
    f[(ids[:, None] * 3 + np.arange(3)).reshape(-1)] = F.reshape(-1)
    return f


class EnergyLoss:
    """Per-sample energy-deficit loss over a data set of cantilever problems sharing one
    mesh and constraint set (``kern``): E [S, elements] and f [S, dof] device doubles,
    compliances c [S] (host floats)."""

    def __init__(self, kern, E, f, c):
        self.kern, self.E, self.f, self.c = kern, E, f, [float(v) for v in c]
        n = f.shape[1]
        dev = f.device
        self.y = torch.empty(n, dtype=torch.float64, device=dev)
        self.ky = torch.empty(n, dtype=torch.float64, device=dev)
        self.work = torch.empty(int(_lib.load().pf_cnn_energy_loss_workspace()), dtype=torch.float64, device=dev)

    def sample(self, i, nodes, grad, loss_out):
        """loss_out = deficit of the nodal prediction ``nodes`` (float32) for sample i;
        grad (float32, nodes' layout) = its gradient."""
        L = _lib.load()
        k = self.kern
        Ei, fi = self.E[i], self.f[i]
        _lib.check(L.pf_cnn_guess_f64(ctypes.byref(k._grid), 1, _p(nodes), k._mask_ptr(), _p(self.y), _lib.stream()))
        _lib.check(L.pf_matvec_f64(k._op, _p(Ei), _p(self.y), k._mask_ptr(), _p(self.ky), _lib.stream()))
        _lib.check(L.pf_cnn_energy_loss_f64(self.y.numel(), _p(self.y), _p(self.ky), _p(fi), self.c[i], _p(grad),
                                            _p(loss_out), _p(self.work), _lib.stream()))


def make_dataset(n_samples, nel=(64, 32, 32), seed0=1000, n_level=4, tol=1e-8, log=None, keep_problems=False):
    """(inputs [S, 8, X, Y, Z], targets [S, nodes * 3], solve statistics) from cold-start
    FP64 MGCG solves of cantilevers clamped at x = 0 with seeded smoothed-random densities
    (sigma 2, SIMP p = 3) and a random edge load (sample i uses seed seed0 + i).  With
    ``keep_problems`` the statistics also hold ``energy``, an EnergyLoss over the samples."""
    from .geom import CuStructuredMesh3D
    from .physics import LinearElasticity
    from .solvers import MultiGrid
    from .stiffness import StructuredStiffnessKernel
    from .workloads import simp_E, smoothed_density

    nelx, nely, nelz = nel
    mesh = CuStructuredMesh3D(nelx, nely, nelz, nelx, nely, nelz, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    kern.set_constraints(cantilever_constraints(nel))
    sol = MultiGrid(mesh, kern, maxiter=2000, tol=tol, n_smooth=2, omega=0.6, n_level=n_level)
    D = kern.shape[0]
    inputs = torch.empty((n_samples, N_IN, nelx, nely, nelz), dtype=torch.float32, device=device())
    targets = torch.empty((n_samples, D), dtype=torch.float32, device=device())
    g = _lib.make_grid(nel)
    work = torch.zeros(1, dtype=torch.int32, device=device())
    its, res, comp = [], [], []
    if keep_problems:
        Es = torch.empty((n_samples, nelx * nely * nelz), dtype=torch.float64, device=device())
        fs = torch.empty((n_samples, D), dtype=torch.float64, device=device())
    t0 = time.time()
    for s in range(n_samples):
        E = as_cuda(simp_E(smoothed_density(nel, seed0 + s)), torch.float64)
        f = as_cuda(edge_load_rhs(nel, seed0 + s), torch.float64)
        U, r = sol.solve(f, rho=E, use_last=False)
        if sol.last_info["status"] != "PF_OK":
            raise RuntimeError(f"training solve {seed0 + s} ended with {sol.last_info['status']} at residual {r:.3e}")
        its.append(sol.last_info["iterations"])
        res.append(r)
        comp.append(float(torch.dot(f, U)))
        if keep_problems:
            Es[s].copy_(E)
            fs[s].copy_(f)
        _lib.check(_lib.load().pf_cnn_features_f32(ctypes.byref(g), 1, _p(E), _p(f), kern._mask_ptr(), _p(work),
                                                   _p(inputs[s]), _lib.stream()))
        targets[s].copy_(U / U.square().mean().sqrt())
        if log is not None and (s + 1) % 250 == 0:
            log(f"dataset {s + 1}/{n_samples} ({time.time() - t0:.1f} s, mean iterations {np.mean(its):.1f})")
    stats = dict(iterations=its, residuals=res, compliances=comp, seconds=time.time() - t0)
    if keep_problems:
        stats["energy"] = EnergyLoss(kern, Es, fs, comp)
    return inputs, targets, stats


class LearnedWarmStart:
    """Initial guess of the MGCG from the network (see the module docstring).

    ``pool`` = P sets the network's cell grid to nel / P (each count divisible by 8 P).
    ``with_previous``: in a sequence of solves (the SIMP loop, where the solver reuses the
    last solution), offer both the network's guess and the previous solution and start
    from the one with the lower energy (``guess(..., prev=...)``).
    After every guess, ``last`` holds {alpha, residual}: the energy-optimal scale and the
    relative residual ||b - K x0|| / ||b|| of the scaled guess (read back only when
    ``read_stats``)."""

    def __init__(self, net: WarmStartNet, pool: int = 1, read_stats: bool = True, with_previous: bool = False):
        self.net = net
        self.pool = int(pool)
        self.read_stats = read_stats
        self.with_previous = bool(with_previous)
        self.last = None
        self.x0 = None
        self._scratch = {}

    def _buf(self, n, kern):
        key = (n, kern.nel)
        if key not in self._scratch:
            dev = device()
            nel = kern.nel
            P = self.pool
            cells = (1, N_IN, nel[0] // P, nel[1] // P, nel[2] // P)
            self._scratch = {key: dict(
                x0=torch.empty(n, dtype=torch.float64, device=dev), kx=torch.empty(n, dtype=torch.float64, device=dev),
                kp=torch.empty(n, dtype=torch.float64, device=dev), xs=torch.empty(n, dtype=torch.float64, device=dev),
                sel=torch.empty(int(_lib.load().pf_cnn_guess_select_workspace()), dtype=torch.float64, device=dev),
                feat=torch.empty(cells, dtype=torch.float32, device=dev),
                work=torch.zeros(1, dtype=torch.int32, device=dev),
                scale=torch.empty(int(_lib.load().pf_cnn_energy_scale_workspace()), dtype=torch.float64, device=dev))}
        return self._scratch[key]

    def guess(self, kern, rhs, prev=None):
        """Scaled initial guess for K(rho) u = rhs with the kernel's current rho.  With
        ``prev`` (the previous solution of a sequence of solves, e.g. the last SIMP
        iteration's displacements) the guess is whichever of the network's prediction and
        ``prev``, each energy-optimally scaled, has the lower energy."""
        L = _lib.load()
        n = rhs.shape[0]
        b = self._buf(n, kern)
        g = kern._grid
        _lib.check(L.pf_cnn_features_f32(ctypes.byref(g), self.pool, _p(kern.rho), _p(rhs), kern._mask_ptr(),
                                         _p(b["work"]), _p(b["feat"]), _lib.stream()))
        nodes = self.net.predict_nodes(b["feat"])
        _lib.check(L.pf_cnn_guess_f64(ctypes.byref(g), self.pool, _p(nodes), kern._mask_ptr(), _p(b["x0"]),
                                      _lib.stream()))
        _lib.check(L.pf_matvec_f64(kern._op, _p(kern.rho), _p(b["x0"]), kern._mask_ptr(), _p(b["kx"]), _lib.stream()))
        if prev is not None:
            prev = as_cuda(prev, torch.float64)
            _lib.check(L.pf_matvec_f64(kern._op, _p(kern.rho), _p(prev), kern._mask_ptr(), _p(b["kp"]),
                                       _lib.stream()))
            _lib.check(L.pf_cnn_guess_select_f64(n, _p(b["x0"]), _p(b["kx"]), _p(prev), _p(b["kp"]), _p(rhs),
                                                 _p(b["xs"]), _p(b["sel"]), _lib.stream()))
            self.x0 = b["xs"]
            if self.read_stats:
                a, which, ea, eb = b["sel"][-4:].tolist()
                self.last = dict(alpha=a, choice="previous" if which else "network", energy_network=ea,
                                 energy_previous=eb)
            return b["xs"]
        _lib.check(L.pf_cnn_energy_scale_f64(n, _p(b["x0"]), _p(b["kx"]), _p(rhs), _p(b["scale"]), _lib.stream()))
        self.x0 = b["x0"]
        if self.read_stats:
            a, r = b["scale"][-2:].tolist()
            self.last = dict(alpha=a, residual=r)
        return b["x0"]


class LearnedCoarseSpace:
    """Learned coarse-grid correction of the MGCG (``MultiGrid(..., coarse_correction=...)``):
    the network's predicted displacement field, interpolated to the mesh and zeroed on
    constrained DOFs, spans a three-column deflation space Q (one column per displacement
    component).  The solver starts from x0 = x + Q G^-1 Q^T (b - K x) with G = Q^T K Q, the
    energy-optimal correction of its start inside span(Q), and keeps every search direction
    K-orthogonal to Q (deflated PCG), so the part of the error the network predicts is
    removed once and does not come back through the V-cycle.  ``pool`` as in
    ``LearnedWarmStart``.  No counterpart in the reference."""

    def __init__(self, net: WarmStartNet, pool: int = 1):
        self.net = net
        self.pool = int(pool)
        self._scratch = {}

    def field(self, kern, rhs):
        """Nodal field (float64, one value per DOF) for K(rho) u = rhs with the kernel's
        current rho and constraints."""
        L = _lib.load()
        n = rhs.shape[0]
        key = (n, kern.nel)
        if key not in self._scratch:
            dev = device()
            nel = kern.nel
            P = self.pool
            self._scratch = {key: dict(
                y=torch.empty(n, dtype=torch.float64, device=dev),
                feat=torch.empty((1, N_IN, nel[0] // P, nel[1] // P, nel[2] // P), dtype=torch.float32, device=dev),
                work=torch.zeros(1, dtype=torch.int32, device=dev))}
        b = self._scratch[key]
        g = kern._grid
        _lib.check(L.pf_cnn_features_f32(ctypes.byref(g), self.pool, _p(kern.rho), _p(rhs), kern._mask_ptr(),
                                         _p(b["work"]), _p(b["feat"]), _lib.stream()))
        nodes = self.net.predict_nodes(b["feat"])
        _lib.check(L.pf_cnn_guess_f64(ctypes.byref(g), self.pool, _p(nodes), kern._mask_ptr(), _p(b["y"]),
                                      _lib.stream()))
        return b["y"]
