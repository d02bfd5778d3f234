"""Generate tests/golden/ldl_golden.npz from the reference's own SparseLDL.

Run in a checkout where oracle/_ref/libamigo_ref.so has been built from the
reference sources (oracle/build_ref.sh):

    python tests/golden/make_golden.py

For every case it records the reference's symbolic arrays (node_ptr,
node_to_var, children_ptr, children, contrib_ptr, contrib_rows, invperm),
the inertia, the per-node pivot/delay counts and the solution of
K x = K 1 (ustab, pivot_tol, delay_growth as stated per case).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from matrices import csr_arrays, kkt_matrix, ldl_unit_matrix, poisson_2d  # noqa: E402
from oracle import ref  # noqa: E402


def cases():
    out = []
    for i in range(7):
        M, _ = ldl_unit_matrix(i)
        for order in ("NATURAL", "AMD"):
            out.append(("unit%d_%s" % (i, order), M, order, 0.4))
    for n in (10, 20):
        M, _ = poisson_2d(n)
        for order in ("NATURAL", "AMD"):
            out.append(("poisson%d_%s" % (n, order), M, order, 0.4))
    for seed, (npr, nc) in enumerate([(120, 80), (400, 300)]):
        M = kkt_matrix(npr, nc, seed + 11)
        for order in ("AMD", "NESTED_DISSECTION"):
            out.append(("kkt%d_%s" % (npr + nc, order), M, order, 0.01))
    return out


def main():
    data = {}
    for name, M, order, ustab in cases():
        n, rp, ci, v = csr_arrays(M)
        L = ref.RefSparseLDL(n, rp, ci, order=order, ustab=ustab)
        sym = L.symbolic()
        assert L.factor(v) == 0
        npos, nneg = L.inertia()
        npiv, ndel = L.node_pivots()
        b = M @ np.ones(n)
        x = L.solve(b)
        data[name + "/rowp"] = rp
        data[name + "/cols"] = ci
        data[name + "/vals"] = v
        data[name + "/order"] = np.array(ref.ORDER[order])
        data[name + "/ustab"] = np.array(ustab)
        for k in ("node_ptr", "node_to_var", "children_ptr", "children",
                  "contrib_ptr", "contrib_rows", "invperm"):
            data[name + "/" + k] = np.asarray(sym[k], dtype=np.int32)
        data[name + "/inertia"] = np.array([npos, nneg], dtype=np.int32)
        data[name + "/npiv"] = npiv
        data[name + "/ndel"] = ndel
        data[name + "/x"] = x
    np.savez_compressed(os.path.join(HERE, "ldl_golden.npz"), **data)
    print("wrote", len(cases()), "cases")


if __name__ == "__main__":
    main()
