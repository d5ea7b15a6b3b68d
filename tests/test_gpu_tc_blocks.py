"""The tensor-core building blocks on their own: split-bf16 forward GEMM
D = Q C^T and adjoint GEMM G = DCDV Q through the same 128B-swizzled
shared-memory layouts, descriptors and TMEM reads as the MSE kernel.

Tolerance: three-term split bf16 keeps ~16 significant bits; the largest
element error relative to the largest element must stay below 1e-4."""
import ctypes as C

import numpy as np
import pytest

import plastimatch_b200 as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [16, 48, 80, 96])
def test_tc_forward_and_adjoint_gemm(N):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(N)
    q = rng.uniform(0, 0.3, (128, 64)).astype(np.float32)
    c = rng.normal(0, 3.0, (N, 64)).astype(np.float32)
    dc = rng.normal(0, 100.0, (128, 128)).astype(np.float32)
    tq, tc_, td = (torch.from_numpy(a).cuda() for a in (q, c, dc))
    d_out = torch.zeros(128 * N, device="cuda")
    g_out = torch.zeros(128 * 64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    f = P.lib().b200bsp_internal_tc_selftest
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
    rc = f(tq.data_ptr(), tc_.data_ptr(), td.data_ptr(), N, d_out.data_ptr(),
           g_out.data_ptr(), err.data_ptr())
    assert rc == 0 and int(err.item()) == 0
    D = d_out.cpu().numpy().reshape(128, N)
    G = g_out.cpu().numpy().reshape(128, 64)
    Dref = q.astype(np.float64) @ c.astype(np.float64).T
    # adjoint: G[r][m] = sum_v dcdv[r][v] * Q[v][m] (Q rows = voxels)
    Gref = dc.astype(np.float64) @ q.astype(np.float64)
    assert np.abs(D - Dref).max() <= 1e-4 * np.abs(Dref).max()
    assert np.abs(G - Gref).max() <= 1e-4 * np.abs(Gref).max()
