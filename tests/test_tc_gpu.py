"""The tensor-core (tcgen05, 3xTF32) Schur update against an FP64 product of
the same FP32 inputs: lower(C) -= A B^T.  Bar: max error <= 2e-6 relative to
max(|C|, |A||B|^T) (FP32 accuracy: the split drops only the lo*lo term),
strict upper triangle untouched, no timeout status."""
import numpy as np
import pytest
import torch

from amigo_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,kw", [(128, 31), (300, 17), (517, 31), (64, 1)])
def test_tc_syrk_matches_fp64(n, kw):
    g = torch.Generator(device="cuda").manual_seed(n * 100 + kw)
    ld = n + 3
    A = torch.randn(kw, ld, device="cuda", generator=g)     # column j = A[j]
    B = torch.randn(kw, ld, device="cuda", generator=g)
    C = torch.randn(n, ld, device="cuda", generator=g)      # column c = C[c]
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    C0 = C.clone()
    _lib.call("ab_tc_syrk_tf32x3", n, kw, A.data_ptr(), ld, B.data_ptr(), ld,
              C.data_ptr(), ld, st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    a = A[:, :n].double().T           # n x kw
    b = B[:, :n].double().T
    want = C0[:, :n].double().T - a @ b.T   # rows x cols
    got = C[:, :n].double().T
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"))
    scale = max(C0.abs().max().item(), (a.abs() @ b.abs().T).max().item())
    assert (got - want)[low].abs().max().item() <= 2e-6 * scale
    assert torch.equal(got[~low], C0[:, :n].double().T[~low])
    # padding rows beyond n untouched
    assert torch.equal(C[:, n:], C0[:, n:])
