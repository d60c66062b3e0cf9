"""Train the learned warm start on solver-generated data and save its weights.

    python -m pyfantom_b200.train_warmstart [--samples 2000] [--epochs 30] [--loss energy|mse] [--out FILE]

Data: ``samples`` cold-start FP64 MGCG solves (tol 1e-8) of 64x32x32 cantilevers clamped
at x = 0, seeded smoothed-random densities and random edge loads (seeds 1000, 1001, ...).
Validation: 64 held-out samples (seeds 5000...).  The epoch count is lowered when the
measured epoch time would exceed ``--budget`` seconds.  One JSON line summarises the run,
including the mean MGCG iterations from the zero start and from the learned guess on 16
held-out problems.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from . import learned


def held_out_gain(net, nel, seeds, n_level=4, pool=1):
    """Mean MGCG iterations to 1e-8 from the zero start and from the learned guess, and the
    guess's mean relative residual, on held-out cantilevers."""
    from .geom import CuStructuredMesh3D
    from .physics import LinearElasticity
    from .solvers import MultiGrid
    from .stiffness import StructuredStiffnessKernel
    from .workloads import simp_E, smoothed_density
    mesh = CuStructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    kern.set_constraints(learned.cantilever_constraints(nel))
    ws = learned.LearnedWarmStart(net, pool=pool)
    zero = MultiGrid(mesh, kern, maxiter=2000, tol=1e-8, n_smooth=2, omega=0.6, n_level=n_level)
    warm = MultiGrid(mesh, kern, maxiter=2000, tol=1e-8, n_smooth=2, omega=0.6, n_level=n_level, warm_start=ws)
    it0, it1, gr, de = [], [], [], []
    for s in seeds:
        f = torch.as_tensor(learned.edge_load_rhs(nel, s), device="cuda")
        E = torch.as_tensor(simp_E(smoothed_density(nel, s)), device="cuda")
        U0, _ = zero.solve(f, rho=E, use_last=False)
        c0 = float(torch.dot(f, U0))
        warm.solve(f, rho=E, use_last=False)
        it0.append(zero.last_info["iterations"])
        it1.append(warm.last_info["iterations"])
        gr.append(ws.last["residual"])
        de.append(1.0 - float(torch.dot(f, ws.x0)) / c0)  # energy error of the scaled guess / that of zero
    return dict(iterations_zero=float(np.mean(it0)), iterations_learned=float(np.mean(it1)),
                guess_residual=float(np.mean(gr)), guess_energy_deficit=float(np.mean(de)),
                seeds=[int(s) for s in seeds])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=2000)
    ap.add_argument("--val", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=5e-5)
    ap.add_argument("--budget", type=float, default=900.0, help="seconds of training at most")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--loss", choices=("energy", "mse"), default="energy")
    ap.add_argument("--out", default=learned.DEFAULT_WEIGHTS)
    a = ap.parse_args(argv)

    def log(m):
        print(m, file=sys.stderr, flush=True)

    nel = (64, 32, 32)
    t0 = time.time()
    keep = a.loss == "energy"
    xs, ys, st = learned.make_dataset(a.samples, nel, seed0=1000, log=log, keep_problems=keep)
    xv, yv, sv = learned.make_dataset(a.val, nel, seed0=5000, keep_problems=keep)
    en, env = st.get("energy"), sv.get("energy")
    t_data = time.time() - t0
    net = learned.WarmStartNet(seed=a.seed)
    # time a fraction of an epoch to size the run
    torch.cuda.synchronize()
    t1 = time.time()
    probe = min(a.samples, 20 * a.batch)
    learned.WarmStartNet(seed=a.seed).fit(xs[:probe], ys[:probe], epochs=1, batch=a.batch, lr=a.lr, energy=en)
    torch.cuda.synchronize()
    per_epoch = (time.time() - t1) * a.samples / probe
    epochs = max(1, min(a.epochs, int(a.budget / per_epoch)))
    log(f"data {t_data:.1f} s; ~{per_epoch:.1f} s per epoch; training {epochs} epochs")
    def val_loss():
        return net.eval_energy(xv, env) if keep else net.eval_loss(xv, yv)

    val0 = val_loss()
    t2 = time.time()
    hist = net.fit(xs, ys, epochs=epochs, batch=a.batch, lr=a.lr, lr_final=a.lr_final, seed=a.seed, log=log,
                   energy=en)
    torch.cuda.synchronize()
    t_train = time.time() - t2
    val = val_loss()
    net.save(a.out)
    gain = held_out_gain(net, nel, seeds=range(5000, 5016))
    print(json.dumps(dict(loss=a.loss, samples=a.samples, grid=list(nel), params=net.n_params, epochs=epochs,
                          batch=a.batch,
                          data_seconds=round(t_data, 1), train_seconds=round(t_train, 1),
                          mean_solve_iterations=float(np.mean(st["iterations"])), train_loss=hist,
                          val_loss_init=val0, val_loss=val, held_out=gain, out=a.out)))


if __name__ == "__main__":
    main()
