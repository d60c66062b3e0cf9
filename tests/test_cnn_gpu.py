"""GPU: the learned warm start's kernels against the CPU oracle, the network gradient,
training, and what the trained network gains over the zero start.

float32 kernels are compared with the float64 oracle at a relative tolerance of 1e-5
(max-norm), the composed U-Net gradient at 1e-4 (it sums over 10 layers in float32).
Every device array handed to the library is bound to a name: a temporary would be freed
before the call runs and its memory handed to the next allocation.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from oracle import cnn_oracle as C
from pyfantom_b200 import _lib
from pyfantom_b200 import learned

pytestmark = pytest.mark.gpu
P = _lib.ptr
S = _lib.stream


def lib():
    return _lib.load()


def f32(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def relerr(a, b):
    a = a.detach().cpu().double().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def normal32(rng, size):
    """float32-representable draws, so exact kernels compare exactly."""
    return rng.normal(size=size).astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("stride", [1, 2])
@pytest.mark.parametrize("shape,co", [((2, 3, 5, 6, 7), 10), ((1, 16, 8, 8, 8), 8), ((3, 9, 4, 3, 6), 3)])
def test_conv_forward_and_adjoints(stride, shape, co):
    rng = np.random.default_rng(stride * 100 + co)
    N, ci, X, Y, Z = shape
    x, w, b = normal32(rng, shape), normal32(rng, (co, ci, 3, 3, 3)), normal32(rng, co)
    xt, wt, bt = f32(x), f32(w), f32(b)
    ref = C.conv3d(x, w, b, stride)
    y = torch.empty(ref.shape, dtype=torch.float32, device="cuda")
    for relu in (0, 1):
        _lib.check(lib().pf_cnn_conv3d_fwd_f32(P(xt), N, ci, X, Y, Z, P(wt), P(bt), co, stride, relu, P(y), S()))
        assert relerr(y, np.maximum(ref, 0) if relu else ref) < 1e-5
    dy = normal32(rng, ref.shape)
    dyt = f32(dy)
    dx = torch.empty(shape, dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_conv3d_bwd_data_f32(P(dyt), N, ci, X, Y, Z, P(wt), co, stride, 0, P(dx), S()))
    gx = C.conv3d_bwd_data(dy, w, shape, stride)
    assert relerr(dx, gx) < 1e-5
    _lib.check(lib().pf_cnn_conv3d_bwd_data_f32(P(dyt), N, ci, X, Y, Z, P(wt), co, stride, 1, P(dx), S()))
    assert relerr(dx, 2 * gx) < 1e-5
    work = torch.empty(int(lib().pf_cnn_conv3d_bwd_weight_workspace(ci, co)), dtype=torch.float32, device="cuda")
    dw = torch.empty((co, ci, 3, 3, 3), dtype=torch.float32, device="cuda")
    db = torch.empty(co, dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_conv3d_bwd_weight_f32(P(xt), P(dyt), N, ci, X, Y, Z, co, stride, P(dw), P(db), P(work),
                                                  S()))
    gw, gb = C.conv3d_bwd_weight(x, dy, stride)
    assert relerr(dw, gw) < 1e-5
    assert relerr(db, gb) < 1e-5


def bf16(a):
    """a rounded to BF16 (round to nearest even), back as float64."""
    return torch.as_tensor(np.asarray(a, np.float32)).to(torch.bfloat16).double().numpy()


@pytest.mark.parametrize("stride", [1, 2])
@pytest.mark.parametrize("shape,co", [((2, 3, 5, 6, 7), 10), ((1, 16, 8, 8, 8), 16), ((3, 9, 4, 3, 6), 3),
                                      ((1, 8, 17, 9, 13), 64), ((2, 160, 4, 4, 8), 48), ((1, 32, 16, 8, 8), 32)])
def test_conv_tensor_core_kernels(stride, shape, co):
    """The tcgen05 implicit-GEMM kernels (forward, input gradient, weight gradient): equal to
    the oracle's convolution of the BF16-rounded operands to FP32 summation accuracy (1e-5
    of the largest entry), and to the FP32 convolution within BF16 rounding (1e-2).  Shapes
    cover K = 27 Cin not a multiple of the 16-wide MMA step (Cin 3, 9) or the 64-wide chunk,
    output channels padded up to 16 (3, 10, 48), several 128-row tiles with a ragged last
    one, weight gradients over several voxel ranges, and both strides."""
    rng = np.random.default_rng(stride * 1000 + co + shape[1])
    N, ci, X, Y, Z = shape
    x, w, b = normal32(rng, shape), normal32(rng, (co, ci, 3, 3, 3)), normal32(rng, co)
    xt, wt, bt = f32(x), f32(w), f32(b)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref_r = C.conv3d(bf16(x), bf16(w), b, stride)
    ref = C.conv3d(x, w, b, stride)
    y = torch.full(ref.shape, float("nan"), dtype=torch.float32, device="cuda")
    for relu in (0, 1):
        _lib.check(lib().pf_cnn_conv3d_fwd_tc(P(xt), N, ci, X, Y, Z, P(wt), P(bt), co, stride, relu, P(y), P(err),
                                              S()))
        assert int(err.item()) == 0
        assert relerr(y, np.maximum(ref_r, 0) if relu else ref_r) < 1e-5
        assert relerr(y, np.maximum(ref, 0) if relu else ref) < 1e-2
    dy = normal32(rng, ref.shape)
    dyt = f32(dy)
    dx = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_conv3d_bwd_data_tc(P(dyt), N, ci, X, Y, Z, P(wt), co, stride, 0, P(dx), P(err), S()))
    assert int(err.item()) == 0
    gx_r = C.conv3d_bwd_data(bf16(dy), bf16(w), shape, stride)
    assert relerr(dx, gx_r) < 1e-5
    assert relerr(dx, C.conv3d_bwd_data(dy, w, shape, stride)) < 1e-2
    _lib.check(lib().pf_cnn_conv3d_bwd_data_tc(P(dyt), N, ci, X, Y, Z, P(wt), co, stride, 1, P(dx), P(err), S()))
    assert relerr(dx, 2 * gx_r) < 1e-5
    # weight gradient: split over voxel ranges, ranges summed in order
    nwork = int(lib().pf_cnn_conv3d_bwd_weight_tc_workspace(N, ci, X, Y, Z, co, stride))
    work = torch.empty(nwork, dtype=torch.float32, device="cuda")
    dw = torch.full((co, ci, 3, 3, 3), float("nan"), dtype=torch.float32, device="cuda")
    db = torch.full((co,), float("nan"), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_conv3d_bwd_weight_tc(P(xt), P(dyt), N, ci, X, Y, Z, co, stride, P(dw), P(db), P(work),
                                                 P(err), S()))
    assert int(err.item()) == 0
    gw_r, _ = C.conv3d_bwd_weight(bf16(x), bf16(dy), stride)
    assert relerr(dw, gw_r) < 1e-5
    assert relerr(db, bf16(dy).sum(axis=(0, 2, 3, 4))) < 1e-5
    gw, _ = C.conv3d_bwd_weight(x, dy, stride)
    assert relerr(dw, gw) < 1e-2


def test_conv_rejects_bad_stride():
    t = torch.zeros(8, device="cuda")
    assert lib().pf_cnn_conv3d_fwd_f32(P(t), 1, 1, 2, 2, 2, P(t), P(t), 1, 3, 0, P(t), S()) == _lib.PF_BAD_ARG


def test_elementwise_kernels():
    rng = np.random.default_rng(1)
    x = normal32(rng, (2, 3, 2, 3, 4))
    xt = f32(x)
    up = torch.empty((2, 3, 4, 6, 8), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_upsample2_f32(6, 2, 3, 4, P(xt), P(up), 0, S()))
    assert relerr(up, C.upsample2(x)) == 0.0
    g = normal32(rng, (2, 3, 4, 6, 8))
    gt = f32(g)
    dn = torch.empty((2, 3, 2, 3, 4), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_upsample2_f32(6, 2, 3, 4, P(gt), P(dn), 1, S()))
    assert relerr(dn, C.upsample2_bwd(g)) < 1e-6
    # channel scatter / gather / accumulate
    src, dst = normal32(rng, (2, 3, 5)), normal32(rng, (2, 7, 5))
    srct, dt = f32(src), f32(dst)
    _lib.check(lib().pf_cnn_copy_channels_f32(2, 3, 5, P(srct), 7, 2, 1, 0, P(dt), S()))
    want = dst.copy()
    want[:, 2:5] += src
    assert relerr(dt, want) < 1e-6
    back = torch.empty((2, 3, 5), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_copy_channels_f32(2, 3, 5, P(dt), 7, 2, 0, 1, P(back), S()))
    assert torch.equal(back, dt[:, 2:5])
    assert lib().pf_cnn_copy_channels_f32(2, 3, 5, P(dt), 4, 2, 0, 0, P(back), S()) == _lib.PF_BAD_ARG
    # channel sums and broadcasts (the network's global context)
    wide = normal32(rng, (2, 6, 7))
    wt = f32(wide)
    cs = torch.empty((2, 3), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_channel_sum_f32(2, 3, 7, P(wt), 6, 2, 0.5, P(cs), S()))
    assert relerr(cs, 0.5 * wide[:, 2:5].sum(axis=2)) < 1e-6
    gv = normal32(rng, (2, 3))
    gvt = f32(gv)
    _lib.check(lib().pf_cnn_channel_bcast_f32(2, 3, 7, P(gvt), 2.0, 6, 1, 1, P(wt), S()))
    want = wide.copy()
    want[:, 1:4] += 2.0 * gv[:, :, None]
    assert relerr(wt, want) < 1e-6
    assert lib().pf_cnn_channel_sum_f32(2, 3, 7, P(wt), 4, 2, 1.0, P(cs), S()) == _lib.PF_BAD_ARG
    # cell -> node and back
    cells = normal32(rng, (2, 3, 3, 2, 4))
    ct = f32(cells)
    nodes = torch.empty((2, 4 * 3 * 5 * 3), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_cell2node_f32(2, 3, 2, 4, P(ct), P(nodes), 0, S()))
    assert relerr(nodes, C.cell2node(cells).reshape(2, -1)) < 1e-6
    gn = normal32(rng, (2, 60, 3))
    gnt = f32(gn)
    gc = torch.empty((2, 3, 3, 2, 4), dtype=torch.float32, device="cuda")
    _lib.check(lib().pf_cnn_cell2node_f32(2, 3, 2, 4, P(gnt), P(gc), 1, S()))
    assert relerr(gc, C.cell2node_bwd(gn, 3, 2, 4)) < 1e-6
    # relu backward
    y, dy = normal32(rng, 1000), normal32(rng, 1000)
    yt, dyt = f32(y), f32(dy)
    _lib.check(lib().pf_cnn_relu_bwd_f32(1000, P(yt), P(dyt), S()))
    assert relerr(dyt, C.relu_bwd(y, dy)) == 0.0


def test_mse_and_adam():
    rng = np.random.default_rng(2)
    n = 100003
    p, t = normal32(rng, n), normal32(rng, n)
    pt, tt = f32(p), f32(t)
    g = torch.empty(n, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float64, device="cuda")
    work = torch.empty(int(lib().pf_cnn_mse_workspace(n)), dtype=torch.float64, device="cuda")
    _lib.check(lib().pf_cnn_mse_f32(n, P(pt), P(tt), P(g), P(loss), P(work), S()))
    ref_l, ref_g = C.mse(p, t)
    assert abs(float(loss) - ref_l) < 1e-6 * ref_l
    assert relerr(g, ref_g) < 1e-5
    # two Adam steps against the textbook update
    w, gr = normal32(rng, 1000), normal32(rng, (2, 1000))
    wt, m, v = f32(w), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    mw, vw = np.zeros(1000), np.zeros(1000)
    for k in (1, 2):
        gk = f32(gr[k - 1])
        _lib.check(lib().pf_cnn_adam_f32(1000, P(wt), P(gk), P(m), P(v), 1e-2, 0.9, 0.999, 1e-8, k, S()))
        mw = 0.9 * mw + 0.1 * gr[k - 1]
        vw = 0.999 * vw + 0.001 * gr[k - 1] ** 2
        w = w - 1e-2 * (mw / (1 - 0.9 ** k)) / (np.sqrt(vw / (1 - 0.999 ** k)) + 1e-8)
    assert relerr(wt, w) < 1e-5


@pytest.mark.parametrize("pool", [1, 2])
def test_features_guess_and_scale(pool):
    nel = (8, 4, 8)
    rng = np.random.default_rng(pool)
    nn = 9 * 5 * 9
    E = rng.uniform(1e-3, 1.0, size=int(np.prod(nel)))
    f = np.zeros(nn * 3)
    f[rng.choice(nn * 3, 12, replace=False)] = rng.normal(size=12)
    mask = np.zeros(nn, dtype=np.uint8)
    mask[rng.choice(nn, 20, replace=False)] = rng.integers(1, 8, size=20).astype(np.uint8)
    g = _lib.make_grid(nel)
    X, Y, Z = (n // pool for n in nel)
    out = torch.empty((8, X, Y, Z), dtype=torch.float32, device="cuda")
    work = torch.zeros(1, dtype=torch.int32, device="cuda")
    Et, ft = torch.as_tensor(E, device="cuda"), torch.as_tensor(f, device="cuda")
    mt = torch.as_tensor(mask, device="cuda")
    _lib.check(lib().pf_cnn_features_f32(ctypes.byref(g), pool, P(Et), P(ft), P(mt), P(work), P(out), S()))
    assert relerr(out, C.features(nel, pool, E, f, mask)) < 1e-6
    cn = normal32(rng, (X + 1) * (Y + 1) * (Z + 1) * 3)
    cnt = f32(cn)
    x0 = torch.empty(nn * 3, dtype=torch.float64, device="cuda")
    _lib.check(lib().pf_cnn_guess_f64(ctypes.byref(g), pool, P(cnt), P(mt), P(x0), S()))
    assert relerr(x0, C.guess(nel, pool, cn, mask)) < 1e-12
    bad = _lib.make_grid((6, 4, 8))
    assert lib().pf_cnn_guess_f64(ctypes.byref(bad), 4, P(cnt), P(mt), P(x0), S()) == _lib.PF_BAD_ARG
    # energy-optimal scale
    x = rng.normal(size=2000)
    kx, b = rng.normal(size=2000), rng.normal(size=2000)
    kx = np.abs(kx) * np.sign(x)  # x.Kx > 0
    xt = torch.as_tensor(x, device="cuda")
    kxt, bt = torch.as_tensor(kx, device="cuda"), torch.as_tensor(b, device="cuda")
    sw = torch.empty(int(lib().pf_cnn_energy_scale_workspace()), dtype=torch.float64, device="cuda")
    _lib.check(lib().pf_cnn_energy_scale_f64(2000, P(xt), P(kxt), P(bt), P(sw), S()))
    alpha = x.dot(b) / x.dot(kx)
    assert relerr(xt, alpha * x) < 1e-13
    assert abs(float(sw[-2]) - alpha) < 1e-13 * abs(alpha)
    assert abs(float(sw[-1]) - np.linalg.norm(b - alpha * kx) / np.linalg.norm(b)) < 1e-12


def test_energy_loss_kernel():
    rng = np.random.default_rng(9)
    n = 5000
    A = rng.normal(size=(50, n)) / 10
    y, u = rng.normal(size=n), rng.normal(size=n)
    # K = A^T A + I restricted to a random subspace is SPD; only Ky and b = Ku enter
    ky = A.T @ (A @ y) + y
    b = A.T @ (A @ u) + u
    c = float(b @ u)
    yt, kyt, bt = (torch.as_tensor(v, device="cuda") for v in (y, ky, b))
    grad = torch.empty(n, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float64, device="cuda")
    work = torch.empty(int(lib().pf_cnn_energy_loss_workspace()), dtype=torch.float64, device="cuda")
    _lib.check(lib().pf_cnn_energy_loss_f64(n, P(yt), P(kyt), P(bt), c, P(grad), P(loss), P(work), S()))
    a, q = b @ y, y @ ky
    assert abs(float(loss) - (1 - a * a / (q * c))) < 1e-12
    assert relerr(grad, -2 * a / (q * c) * (b - a / q * ky)) < 1e-6
    assert 0.0 <= float(loss) <= 1.0


@pytest.mark.parametrize("tc", [False, True])
def test_network_gradient_matches_oracle(tc):
    """The composed U-Net loss and parameter gradient against the float64 oracle: 1e-4 of
    each layer's largest entry with the FP32 convolutions.  With the tensor-core
    convolutions (BF16 operands; each kernel matches the oracle to 1e-5 on BF16-representable
    operands, test_conv_tensor_core_kernels) the rounding compounds over the ten layers of
    the backward pass and cancels in the weight-gradient sums: the loss to 1e-3 and each
    layer's gradient to 0.15 in the 2-norm (measured, deterministic: 0.3 % to 9 %, the
    stride-2 layers largest), pointing the same way (cosine above 0.99)."""
    net = learned.WarmStartNet(channels=(4, 4, 8, 8), seed=3, tensor_cores=tc)
    tl, tg = (1e-3, 0.15) if tc else (1e-5, 1e-4)
    err = (lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))) if tc else relerr
    rng = np.random.default_rng(4)
    N, X, Y, Z = 2, 8, 8, 16
    x = normal32(rng, (N, 8, X, Y, Z))
    t = normal32(rng, (N, (X + 1) * (Y + 1) * (Z + 1), 3))
    xt, tt = f32(x), f32(t.reshape(N, -1))
    loss = torch.empty(1, dtype=torch.float64, device="cuda")
    net.loss_and_grad(xt, tt, loss)
    W = {n: net.w(n).double().cpu().numpy().reshape(net.spec[n][1], net.spec[n][0], 3, 3, 3) for n in net.spec}
    B = {n: net.b(n).double().cpu().numpy() for n in net.spec}
    ref_loss, dW, dB = C.unet_loss_grad(W, B, x, t)
    assert abs(float(loss) - ref_loss) < tl * ref_loss
    g = net.grad.double().cpu().numpy()
    for n in net.spec:
        ci, co, _, _, ow, ob = net.spec[n]
        assert err(g[ow:ob], dW[n].reshape(-1)) < tg, n
        assert err(g[ob:ob + co], dB[n]) < tg, n
        if tc:
            a, b = g[ow:ob], dW[n].reshape(-1)
            assert a @ b / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.99, n
    # single-sample path (upsampling straight into the concatenation)
    x1, t1 = f32(x[:1]), f32(t[:1].reshape(1, -1))
    net.loss_and_grad(x1, t1, loss)
    ref_loss, dW, dB = C.unet_loss_grad(W, B, x[:1], t[:1])
    g = net.grad.double().cpu().numpy()
    assert abs(float(loss) - ref_loss) < tl * ref_loss
    for n in ("c1a", "c4a", "d3", "out"):
        ci, co, _, _, ow, ob = net.spec[n]
        assert err(g[ow:ob], dW[n].reshape(-1)) < tg, n
    assert not tc or net.tensor_core_errors() == 0


def test_training_reduces_loss():
    inputs, targets, stats = learned.make_dataset(48, nel=(16, 8, 8), seed0=1000, n_level=2)
    assert np.isfinite(targets.cpu().numpy()).all()
    assert max(stats["residuals"]) <= 1e-8
    net = learned.WarmStartNet(channels=(8, 8, 16, 16), seed=0)
    hist = net.fit(inputs, targets, epochs=25, batch=4, lr=2e-3, lr_final=2e-4, seed=0)
    assert hist[-1] < 0.75 * hist[0], hist
    # the energy deficit (1 - cos^2 in the energy inner product) falls as well
    inputs, targets, stats = learned.make_dataset(48, nel=(16, 8, 8), seed0=1000, n_level=2, keep_problems=True)
    net = learned.WarmStartNet(channels=(8, 8, 16, 16), seed=0)
    d0 = net.eval_energy(inputs, stats["energy"], batch=4)
    hist = net.fit(inputs, targets, epochs=25, batch=4, lr=2e-3, lr_final=2e-4, seed=0, energy=stats["energy"])
    d1 = net.eval_energy(inputs, stats["energy"], batch=4)
    assert 0.0 <= d1 < 0.85 * d0, (d0, d1, hist)


def _held_out(nel, seed, n_level, ws, precision="fp64", cc=None):
    from pyfantom_b200.geom import CuStructuredMesh3D
    from pyfantom_b200.physics import LinearElasticity
    from pyfantom_b200.solvers import MultiGrid
    from pyfantom_b200.stiffness import StructuredStiffnessKernel
    from pyfantom_b200.workloads import simp_E, smoothed_density
    mesh = CuStructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    kern.set_constraints(learned.cantilever_constraints(nel))
    f = torch.as_tensor(learned.edge_load_rhs(nel, seed), device="cuda")
    E = torch.as_tensor(simp_E(smoothed_density(nel, seed)), device="cuda")
    sol = MultiGrid(mesh, kern, maxiter=2000, tol=1e-8, n_smooth=2, omega=0.6, n_level=n_level,
                    precision=precision, warm_start=ws, coarse_correction=cc)
    U, res = sol.solve(f, rho=E, use_last=False)
    assert sol.last_info["status"] == "PF_OK"
    return sol.last_info["iterations"], res, U, f


@pytest.mark.skipif(not os.path.exists(learned.DEFAULT_WEIGHTS), reason="no trained weights in the package")
def test_trained_network_gains_over_zero_start():
    """The committed network (trained with the energy loss on 64x32x32 cantilevers, seeds
    1000..2999) on held-out seeds.  What it gains: its scaled guess carries a large share of
    the solution's energy (energy deficit 1 - f.x0 / f.u well below 1, the value of the zero
    start and of an untrained network).  The MGCG from it meets the same tolerance, gives the
    same compliance and takes no more iterations than from zero (the iteration saving of
    such a guess is small at this deficit; the counts are printed)."""
    net = learned.WarmStartNet.load()
    ws = learned.LearnedWarmStart(net)
    raw = learned.LearnedWarmStart(learned.WarmStartNet(seed=0))
    d_trained, d_raw, its = [], [], []
    for seed in (5000, 5001, 5002, 5003):
        it0, r0, U0, f = _held_out((64, 32, 32), seed, 4, None)
        c0 = float(f.dot(U0))
        it1, r1, U1, _ = _held_out((64, 32, 32), seed, 4, ws)
        d_trained.append(1.0 - float(f.dot(ws.x0)) / c0)
        _held_out((64, 32, 32), seed, 4, raw)
        d_raw.append(1.0 - float(f.dot(raw.x0)) / c0)
        assert r0 <= 1e-8 and r1 <= 1e-8
        assert abs(float(f.dot(U1)) - c0) < 1e-8 * abs(c0)
        assert it1 <= it0 + 2, (it0, it1)
        its.append((it0, it1))
    print("iterations zero/learned", its, "energy deficit trained", d_trained, "untrained", d_raw)
    assert np.mean(d_trained) < 0.7, d_trained
    assert min(d_raw) > 0.9, d_raw


@pytest.mark.skipif(not os.path.exists(learned.DEFAULT_WEIGHTS), reason="no trained weights in the package")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_learned_coarse_space_gains_iterations(precision):
    """The committed network as a coarse-grid correction (LearnedCoarseSpace: deflation of
    the PCG by its predicted field) on held-out 64x32x32 cantilevers, seeds 5000..5003: every
    solve takes fewer iterations than the plain MGCG from zero and the mean ratio is below
    0.9 (the oracle's deflated PCG with the network field takes 51/62, 42/63, 49/62 and
    49/63 in FP64), with the same tolerance met and the same compliance."""
    net = learned.WarmStartNet.load()
    cs = learned.LearnedCoarseSpace(net)
    ratios, its = [], []
    for seed in (5000, 5001, 5002, 5003):
        it0, r0, U0, f = _held_out((64, 32, 32), seed, 4, None, precision)
        c0 = float(f.dot(U0))
        it1, r1, U1, _ = _held_out((64, 32, 32), seed, 4, None, precision, cc=cs)
        assert r0 <= 1e-8 and r1 <= 1e-8
        assert abs(float(f.dot(U1)) - c0) < 1e-8 * abs(c0)
        assert it1 < it0, (seed, it0, it1)
        ratios.append(it1 / it0)
        its.append((it0, it1))
    print("iterations plain/coarse-space", its)
    assert np.mean(ratios) < 0.9, its
