"""The allocation-free step-length entry point (ab_ipm_max_step_noalloc).

Callers that cannot let a library allocate device memory use this variant:
its reduction scratch is a fixed array compiled into the library instead of
a buffer from cudaMalloc.  The test calls it through the C ABI and checks
that it returns exactly what ab_ipm_max_step returns (both are
deterministic: bit-identical values and indices), on two calls in a row
that reuse the shared array, and that sizes beyond its limit are refused.
This file is collected last so that a failing run stops after every other
test; it passes alone in a fresh process as well as after the others.
"""
import ctypes

import numpy as np
import pytest
import torch

from amigo_b200 import _lib


def problem(np_, seed):
    r = np.random.RandomState(seed)
    lbx = np.where(r.rand(np_) < 0.8, -1.0 - r.rand(np_), -np.inf)
    ubx = np.where(r.rand(np_) < 0.6, 1.0 + r.rand(np_), np.inf)
    d = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to(
        "cuda:0", dt)
    t = dict(pidx=d(np.arange(np_, dtype=np.int32), torch.int32),
             cidx=d(np.zeros(1, np.int32), torch.int32),
             lbx=d(lbx), ubx=d(ubx), lbh=d(np.zeros(1)),
             zl=d(0.1 + r.rand(np_)), zu=d(0.1 + r.rand(np_)),
             sl=d(0.05 + r.rand(np_)), su=d(0.05 + r.rand(np_)),
             px=d(r.randn(np_)), dzl=d(r.randn(np_)), dzu=d(r.randn(np_)))
    P = _lib.IpmProblem(np_, np_, 0, t["pidx"].data_ptr(), t["cidx"].data_ptr(),
                        t["lbx"].data_ptr(), t["ubx"].data_ptr(),
                        t["lbh"].data_ptr())
    S = _lib.IpmState(t["px"].data_ptr(), t["zl"].data_ptr(), t["zu"].data_ptr(),
                      t["sl"].data_ptr(), t["su"].data_ptr())
    return P, S, t


def run(name, P, S, t, tau):
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    iout = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = getattr(_lib.lib(), name)(ctypes.byref(P), ctypes.byref(S), tau,
                                   t["px"].data_ptr(), t["dzl"].data_ptr(),
                                   t["dzu"].data_ptr(), out.data_ptr(),
                                   iout.data_ptr(), stream)
    assert rc == 0, (name, rc)
    torch.cuda.synchronize()
    return out.cpu().numpy(), iout.cpu().numpy()


# 8192 * 256 fills the static array: every block partial is written and read
@pytest.mark.gpu
@pytest.mark.parametrize("np_", [1, 1000, 300001, 8192 * 256])
def test_noalloc_matches_allocating_entry_point(np_):
    for call, seed in enumerate((5, 6)):  # two calls in a row share the array
        P, S, t = problem(np_, seed + np_)
        want_v, want_i = run("ab_ipm_max_step", P, S, t, 0.99)
        got_v, got_i = run("ab_ipm_max_step_noalloc", P, S, t, 0.99)
        assert np.array_equal(got_v, want_v), (call, got_v, want_v)
        assert np.array_equal(got_i, want_i), (call, got_i, want_i)


@pytest.mark.gpu
def test_noalloc_rejects_oversize():
    P, S, t = problem(8, 1)
    P.np = 8192 * 256 + 1  # beyond the static scratch (never launched)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    iout = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    rc = _lib.lib().ab_ipm_max_step_noalloc(
        ctypes.byref(P), ctypes.byref(S), 0.99, t["px"].data_ptr(),
        t["dzl"].data_ptr(), t["dzu"].data_ptr(), out.data_ptr(),
        iout.data_ptr(), None)
    assert rc == -6


def test_noalloc_checks_arguments_like_allocating_entry_point():
    """Both entry points reject the same malformed arguments (no launch is
    reached, so this runs without a GPU)."""
    P, S = _lib.IpmProblem(), _lib.IpmState()
    P.n, P.np, P.nc = 4, 0, 4   # constraints without their index/bound arrays
    out = (ctypes.c_double * 2)()
    iout = (ctypes.c_int * 2)()
    for name in ("ab_ipm_max_step", "ab_ipm_max_step_noalloc"):
        rc = getattr(_lib.lib(), name)(ctypes.byref(P), ctypes.byref(S), 0.99,
                                       None, None, None, out, iout, None)
        assert rc == -1, (name, rc)
