"""GPU parity of the IPM vector kernels against the reference's own
include/interior_point_backend.h (compiled into oracle/_ref).

Elementwise kernels are compiled without FMA contraction and must match the
reference bit for bit; max-step must match bit for bit including the argmin
indices; sums may differ by summation order (rtol 1e-12), maxima/minima are
exact.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def make_problem(n, seed, inf_frac=0.3):
    r = np.random.RandomState(seed)
    mult = r.rand(n) < 0.4
    lower = r.randn(n) - 2.0
    upper = lower + 0.5 + 4 * r.rand(n)
    lower[r.rand(n) < inf_frac] = -np.inf
    upper[r.rand(n) < inf_frac] = np.inf
    lower[mult] = r.randn(mult.sum())  # lbh for multipliers
    return mult, lower, upper


def make_state(opt, seed):
    r = np.random.RandomState(seed)
    v = opt.create_opt_vector()
    v.x.copy_(torch.from_numpy(r.randn(opt.n)))
    v.duals.copy_(torch.from_numpy(0.1 + r.rand(2 * opt.np_)))
    v.slacks.copy_(torch.from_numpy(0.05 + r.rand(2 * opt.np_)))
    return v


def host(v):
    return [v.x.cpu().numpy(), v.zl.cpu().numpy(), v.zu.cpu().numpy(),
            v.sl.cpu().numpy(), v.su.cpu().numpy()]


@pytest.fixture(params=[(1, 7), (5000, 1), (200003, 2)])
def setup(request, oracle_ref):
    from amigo_b200.ipm import InteriorPointOptimizer
    n, seed = request.param
    mult, lower, upper = make_problem(n, seed)
    opt = InteriorPointOptimizer(mult, lower, upper, device="cuda:0")
    ref = oracle_ref.RefIPM(opt.pidx.cpu().numpy(), opt.cidx.cpu().numpy(),
                            opt.lbx.cpu().numpy(), opt.ubx.cpu().numpy(),
                            opt.lbh.cpu().numpy())
    v = make_state(opt, seed + 100)
    return opt, ref, v, np.random.RandomState(seed + 200)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def test_elementwise_bit_exact(setup):
    opt, ref, v, r = setup
    st = host(v)
    n = opt.n
    mu = 0.137
    grad = r.randn(n)
    res = dev(np.zeros(n))
    opt.compute_residual(mu, v, dev(grad), res)
    assert np.array_equal(res.cpu().numpy(), ref.compute_residual(mu, st, grad))
    diag = dev(np.zeros(n))
    opt.compute_diagonal(v, diag)
    assert np.array_equal(diag.cpu().numpy(), ref.compute_diagonal(st, n))
    px = r.randn(n)
    upd = opt.create_opt_vector()
    opt.compute_update(mu, v, dev(px), upd)
    dzl, dzu = ref.compute_bound_dual_step(mu, st, px)
    assert np.array_equal(upd.zl.cpu().numpy(), dzl)
    assert np.array_equal(upd.zu.cpu().numpy(), dzu)
    ax, xi, az, zi = opt.compute_max_step(0.995, v, upd)
    assert (ax, xi, az, zi) == ref.compute_max_step(0.995, st, px, dzl, dzu)
    tmp = opt.create_opt_vector()
    tmp.copy(v)
    opt.apply_step_update(0.3, 0.7, v, upd, tmp)
    want = ref.apply_step(0.3, 0.7, st, px, dzl, dzu)
    for got, w in zip(host(tmp), want):
        assert np.array_equal(got, w)
    w = opt.create_opt_vector()
    w.copy(v)
    opt.reset_bound_multipliers(mu, 1e10, w)
    zl, zu = ref.reset_bound_multipliers(mu, 1e10, st)
    assert np.array_equal(w.zl.cpu().numpy(), zl)
    assert np.array_equal(w.zu.cpu().numpy(), zu)
    dst = opt.create_opt_vector()
    dst.copy(v)
    opt.compute_affine_start_point(1e-2, v, upd, dst)
    zl, zu = ref.compute_affine_start_point(1e-2, st, dzl, dzu)
    assert np.array_equal(dst.zl.cpu().numpy(), zl)
    assert np.array_equal(dst.zu.cpu().numpy(), zu)


def test_reductions(setup):
    opt, ref, v, r = setup
    st = host(v)
    mu = 0.05
    grad = r.randn(opt.n)
    px = r.randn(opt.n)
    s, cnt, mn = ref.compute_complementarity(st)
    avg = s / cnt if cnt > 0 else 0.0
    xi = max(0.0, min(1.0, mn / avg)) if avg > 0 else 1.0
    gavg, gxi = opt.compute_complementarity(v)
    assert gavg == pytest.approx(avg, rel=1e-12, abs=0)
    assert gxi == pytest.approx(xi, rel=1e-12, abs=0)
    d, p, c = opt.compute_kkt_error_mu(mu, v, dev(grad))
    assert (d, p, c) == ref.compute_kkt_error(mu, st, grad)
    assert opt.compute_barrier_log_sum(mu, v) == pytest.approx(
        ref.compute_barrier_log_sum(mu, st), rel=1e-12, abs=1e-300)
    assert opt.compute_barrier_dphi_direct(mu, v, dev(grad), dev(px)) == \
        pytest.approx(ref.compute_barrier_dphi(mu, st, grad, px), rel=1e-11,
                      abs=1e-300)
    assert opt.compute_constraint_violation_1norm(v, dev(grad)) == pytest.approx(
        ref.compute_constraint_violation_1norm(st, grad), rel=1e-12, abs=0)
    assert opt.compute_max_comp_deviation(v, mu) == \
        ref.compute_max_comp_deviation(st, mu)
    assert opt.compute_complementarity_sq(v) == pytest.approx(
        ref.compute_complementarity_sq(st, 0.0), rel=1e-12, abs=0)


def test_max_step_ties_and_empty(oracle_ref):
    from amigo_b200.ipm import InteriorPointOptimizer
    n = 4096
    mult = np.zeros(n, bool)
    lower = np.zeros(n)
    upper = np.full(n, np.inf)
    opt = InteriorPointOptimizer(mult, lower, upper, device="cuda:0")
    v = opt.create_opt_vector()
    v.slacks.fill_(1.0)
    v.duals.fill_(1.0)
    upd = opt.create_opt_vector()
    # no blocking direction -> (1, -1, 1, -1)
    assert opt.compute_max_step(0.99, v, upd) == (1.0, -1, 1.0, -1)
    # identical blocking ratios everywhere -> the first index wins
    upd.x.fill_(-2.0)
    upd.duals.fill_(-4.0)
    ax, xi, az, zi = opt.compute_max_step(0.99, v, upd)
    assert (xi, zi) == (0, 0)
    assert ax == -0.99 * 1.0 / -2.0 and az == -0.99 * 1.0 / -4.0


def test_initialize_and_relax(oracle_ref):
    from amigo_b200.ipm import InteriorPointOptimizer
    n = 3001
    mult, lower, upper = make_problem(n, 9)
    opt = InteriorPointOptimizer(mult, lower, upper, device="cuda:0")
    lbx0, ubx0 = opt.lbx.cpu().numpy(), opt.ubx.cpu().numpy()
    opt.relax_bounds()
    lbx, ubx = opt.lbx.cpu().numpy(), opt.ubx.cpu().numpy()
    fin = np.isfinite(lbx0)
    d = np.minimum(1e-4, 1e-8 * np.maximum(1.0, np.abs(lbx0[fin])))
    assert np.array_equal(lbx[fin], lbx0[fin] - d)
    fin = np.isfinite(ubx0)
    d = np.minimum(1e-4, 1e-8 * np.maximum(1.0, np.abs(ubx0[fin])))
    assert np.array_equal(ubx[fin], ubx0[fin] + d)
    v = opt.create_opt_vector()
    v.x.copy_(torch.from_numpy(np.random.RandomState(3).randn(n) * 3))
    opt.initialize_multipliers_and_slacks(0.1, None, v)
    x = v.x.cpu().numpy()[opt.pidx.cpu().numpy()]
    assert np.all(x[np.isfinite(lbx)] > lbx[np.isfinite(lbx)])
    assert np.all(x[np.isfinite(ubx)] < ubx[np.isfinite(ubx)])
    sl = v.sl.cpu().numpy()
    assert np.array_equal(sl[np.isfinite(lbx)], (x - lbx)[np.isfinite(lbx)])
    assert np.all(v.zl.cpu().numpy()[np.isfinite(lbx)] == 1.0)


def test_reductions_on_two_streams_at_once():
    """The reductions' block partials live in a scratch array per stream:
    two problems reduced on two streams whose kernels overlap give the same
    values as each alone on the default stream."""
    from amigo_b200.ipm import InteriorPointOptimizer
    probs = []
    for seed in (11, 12):
        mult, lower, upper = make_problem(300000, seed)
        opt = InteriorPointOptimizer(mult, lower, upper, device="cuda:0")
        v = make_state(opt, seed + 100)
        g = dev(np.random.RandomState(seed).randn(opt.n))
        probs.append((opt, v, g))
    alone = [opt.compute_kkt_error_mu(0.05, v, g) + opt.compute_complementarity(v)
             for opt, v, g in probs]
    import threading
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    torch.cuda.synchronize()
    outs = [[], []]

    def work(i):
        opt, v, g = probs[i]
        with torch.cuda.stream(streams[i]):
            for rep in range(20):
                outs[i].append(opt.compute_kkt_error_mu(0.05, v, g) +
                               opt.compute_complementarity(v))

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    for i in range(2):
        assert len(outs[i]) == 20 and all(o == alone[i] for o in outs[i])
