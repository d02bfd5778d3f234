"""Bit-exact parity of the host symbolic analysis (CPU only).

The product's ordering + supernode partition must equal the reference
SparseLDL's private arrays (include/sparse_ldl.h:2204-2358) exactly: against
the committed golden fixtures (generated from the reference by
tests/golden/make_golden.py) and, when oracle/_ref is built, against the
reference itself on further patterns.
"""
import os

import numpy as np
import pytest

from amigo_b200 import linalg
from matrices import csr_arrays, kkt_matrix, ldl_unit_matrix, poisson_2d

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldl_golden.npz")
KEYS = ("node_ptr", "node_to_var", "children_ptr", "children", "contrib_ptr",
        "contrib_rows", "invperm")


def golden_cases():
    z = np.load(GOLD)
    names = sorted({k.split("/")[0] for k in z.files})
    return z, names


def test_golden_symbolic_bit_exact():
    z, names = golden_cases()
    assert len(names) == 22
    for name in names:
        rp, ci = z[name + "/rowp"], z[name + "/cols"]
        n = len(rp) - 1
        got = linalg.analyze(n, rp, ci, int(z[name + "/order"]))
        for k in KEYS:
            np.testing.assert_array_equal(got[k], z[name + "/" + k],
                                          err_msg="%s %s" % (name, k))


def _patterns():
    mats = []
    for i in range(7):
        mats.append(ldl_unit_matrix(i)[0])
    for n in (10, 20, 50):
        mats.append(poisson_2d(n)[0])
    for s, (a, b) in enumerate([(50, 30), (500, 300), (2000, 1500)]):
        mats.append(kkt_matrix(a, b, 100 + s))
    # unsorted column indices inside rows
    M = kkt_matrix(300, 200, 7, sort=False)
    mats.append(M)
    return mats


@pytest.mark.parametrize("order", ["NATURAL", "AMD", "NESTED_DISSECTION"])
def test_symbolic_matches_reference(oracle_ref, order):
    for M in _patterns():
        n, rp, ci, _ = csr_arrays(M)
        want = oracle_ref.RefSparseLDL(n, rp, ci, order=order).symbolic()
        got = linalg.analyze(n, rp, ci, linalg.OrderingType[order])
        assert got["num_nodes"] == want["num_nodes"]
        for k in KEYS:
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_amd_permutation_matches_reference(oracle_ref):
    for M in _patterns():
        n, rp, ci, _ = csr_arrays(M)
        perm, iperm = oracle_ref.order(n, rp, ci, "AMD")
        got = linalg.analyze(n, rp, ci, linalg.OrderingType.AMD)
        np.testing.assert_array_equal(got["invperm"], iperm)


def test_empty_and_tiny():
    got = linalg.analyze(1, np.array([0, 1]), np.array([0]))
    assert got["num_nodes"] == 1
    np.testing.assert_array_equal(got["node_ptr"], [0, 1])
    got = linalg.analyze(2, np.array([0, 1, 2]), np.array([0, 1]))  # two roots
    assert got["num_nodes"] >= 1
    assert got["children_ptr"][-1] == got["num_nodes"]


def test_bad_arguments():
    with pytest.raises(Exception):
        linalg.analyze(2, np.array([0, 1, 2]), np.array([0, 5]))
    with pytest.raises(Exception):
        linalg.analyze(2, np.array([0, 1, 2]), np.array([0, 1]),
                       linalg.OrderingType.MULTI_COLOR)


def _config_pattern(name):
    """KKT sparsity patterns of the benchmarked configurations: the cart-pole
    collocation problem (N = 100), the 2D SIMP 128 x 64 and the 3D SIMP
    48 x 24 x 24 compliance KKTs."""
    if name == "cartpole_N100":
        from amigo_b200.problems.cartpole import CartPole
        m = CartPole(N=100, seed=0)
    elif name == "simp2d_128x64":
        from amigo_b200.problems.simp2d import Simp2D
        m = Simp2D(128, 64)
    else:
        from amigo_b200.problems.simp3d import Simp3D
        m = Simp3D(48, 24, 24)
    return m.n, m.rowp, m.cols


@pytest.mark.parametrize("name", ["cartpole_N100", "simp2d_128x64", "simp3d_48x24x24"])
def test_config_patterns_match_reference(oracle_ref, name):
    """Ordering, elimination tree, supernodes and contribution rows of the
    benchmarked KKT patterns equal the reference SparseLDL's (AMD, its
    default ordering here) bit for bit."""
    n, rp, ci = _config_pattern(name)
    want = oracle_ref.RefSparseLDL(n, rp, ci, order="AMD").symbolic()
    got = linalg.analyze(n, rp, ci, linalg.OrderingType.AMD)
    assert got["num_nodes"] == want["num_nodes"]
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want[k], err_msg="%s %s" % (name, k))


def test_mem_estimate_from_symbolic_analysis():
    """The workspace estimate (ab_ldl_mem_estimate) covers the fronts'
    static sizes times the delay growth, halves the front pool for FP32
    fronts, and grows with the number of right-hand sides; no GPU needed."""
    M = kkt_matrix(500, 300, 5)
    n, rp, ci, _ = csr_arrays(M)
    S = linalg.analyze(n, rp, ci, linalg.OrderingType.AMD)
    f = (np.diff(S["node_ptr"]) + np.diff(S["contrib_ptr"])).astype(np.int64)
    fronts = 8 * np.sum(f * f + 32 * f)
    e64 = linalg.mem_estimate(n, rp, ci, precision=64, delay_growth=2.0)
    e64_1 = linalg.mem_estimate(n, rp, ci, precision=64, delay_growth=1.0)
    e32 = linalg.mem_estimate(n, rp, ci, precision=32, delay_growth=2.0)
    e64_4 = linalg.mem_estimate(n, rp, ci, precision=64, delay_growth=2.0, nrhs=4)
    assert e64 >= 2 * fronts and e64_1 >= fronts
    assert e32 < e64 and e64 - e32 >= fronts * 0.99
    assert e64_4 > e64
