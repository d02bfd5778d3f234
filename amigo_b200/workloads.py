"""Small, self-contained workloads that exercise every kernel of the
library once or a few times; used for profiler captures of single kernels.

    python -m amigo_b200.workloads simp2d [nx ny]   # KKT assembly, factor, solve, IPM vectors
    python -m amigo_b200.workloads cartpole [N]     # one whole IPM solve
    python -m amigo_b200.workloads simp3d [nx ny nz [fp32|fp64]]
                                   # 3D KKT factor (tensor-core updates in
                                   # fp32) and solve
"""
import sys
import time

import numpy as np
import torch


def simp2d(nx=64, ny=32, reps=2):
    from . import linalg
    from .ipm import InteriorPointOptimizer
    from .problems.simp2d import Simp2D
    dev = torch.device("cuda", 0)
    m = Simp2D(nx, ny)
    dm = m.device_model(dev)
    K = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, device=dev)
    ldl = linalg.SparseLDL(K, order=linalg.OrderingType.AMD)
    opt = InteriorPointOptimizer(m.mult, m.lower, m.upper, device=dev)
    opt.relax_bounds()
    x = torch.from_numpy(m.initial_point()).to(dev)
    v = opt.create_opt_vector(x)
    opt.initialize_multipliers_and_slacks(0.1, None, v)
    g = torch.zeros(m.n, dtype=torch.float64, device=dev)
    diag = torch.zeros_like(g)
    res = torch.zeros_like(g)
    px = torch.zeros_like(g)
    kp = torch.zeros_like(g)
    upd = opt.create_opt_vector()
    tmp = opt.create_opt_vector()
    primal = torch.from_numpy(~m.mult).to(dev).double()
    for _ in range(reps):
        t = time.perf_counter()
        dm.gradient(v.x, 1.0, g)
        dm.hessian(v.x, 1.0, K.vals)
        opt.compute_diagonal(v, diag)
        diag.add_(primal, alpha=1e-8)
        K.add_diagonal(diag)
        ldl.factor()
        inertia = ldl.get_inertia()
        opt.compute_residual(0.1, v, g, res)
        px.copy_(res)
        ldl.solve_device(px)
        K.mult(px, kp)
        opt.compute_update(0.1, v, px, upd)
        ax, xi, az, zi = opt.compute_max_step(0.99, v, upd)
        opt.apply_step_update(ax, az, v, upd, tmp)
        opt.compute_kkt_error_mu(0.1, v, g)
        torch.cuda.synchronize()
        print("simp2d %dx%d n=%d inertia=%s step %.2f ms" %
              (nx, ny, m.n, inertia, 1e3 * (time.perf_counter() - t)))


def cartpole(N=100):
    from . import ipm_driver
    from .problems.cartpole import CartPole
    m = CartPole(N=N, seed=0)
    B = ipm_driver.DeviceBackend(ipm_driver.CartPoleProblem(m, "cuda:0"), m, "cuda:0")
    r = ipm_driver.solve(B)
    print("cartpole N=%d: %d iterations, objective %.12g, kkt %.3e, %.3f s" %
          (N, r["iterations"], r["objective"], r["kkt_error"], r["time_s"]))


def simp3d(nx=16, ny=8, nz=8, precision="fp32", reps=2):
    from . import linalg
    from .problems.simp3d import Simp3D
    dev = torch.device("cuda", 0)
    m = Simp3D(nx, ny, nz)
    dm = m.device_model(dev)
    K = linalg.CSRMat(m.n, m.n, m.rowp, m.cols, device=dev)
    ldl = linalg.SparseLDL(K, order=linalg.OrderingType.AMD, precision=precision)
    x = torch.from_numpy(m.initial_point()).to(dev)
    dm.hessian(x, 1.0, K.vals)
    d = torch.from_numpy(np.where(~m.mult, 1.0, 0.0)).to(dev)
    K.add_diagonal(d)
    b = torch.ones(m.n, dtype=torch.float64, device=dev)
    for _ in range(reps):
        t = time.perf_counter()
        ldl.factor()
        xs = b.clone()
        ldl.solve_device(xs)
        torch.cuda.synchronize()
        print("simp3d %dx%dx%d n=%d %s inertia=%s %.2f ms" %
              (nx, ny, nz, m.n, precision, ldl.get_inertia(),
               1e3 * (time.perf_counter() - t)))


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "simp2d"
    args = [int(a) for a in sys.argv[2:] if a.isdigit()]
    if which == "simp2d":
        simp2d(*args)
    elif which == "cartpole":
        cartpole(*args)
    elif which == "simp3d":
        prec = sys.argv[5] if len(sys.argv) > 5 else "fp32"
        simp3d(*[int(a) for a in sys.argv[2:5]], precision=prec)
    else:
        raise SystemExit("unknown workload " + which)
