"""GPU test of aces_xgemm_static, the contraction entry point that allocates
no device memory.

It serves callers that cannot call cudaMalloc when they need a product --
hosts whose device memory belongs to their own allocator, or code that must
not stall on an allocation.  Its scratch is a fixed static device array, so
the test checks (a) that it reproduces aces_xgemm (the allocating entry
point, same FP64 kernels) to the FP64 tolerance of the other XGEMM tests, on
two calls in a row with shapes that use the scratch for operand copies and
split-K partials, (b) that those calls request no device memory from the
library's allocator (aces_pool_stats), and (c) that a request beyond the
array is refused with a status code.  This file is collected last (tests/test_zz_*) and also passes
on its own in a fresh process.
"""
import numpy as np
import pytest

import acesb200 as ab

pytestmark = pytest.mark.gpu

SHAPES = [  # m, n, k, transa, transb
    (300, 200, 513, "N", "T"),   # both operands copied into the scratch, split-K partials
    (20, 900, 2000, "T", "N"),   # thin product with split-K partials in the scratch
    (129, 7, 1000, "N", "N"),
    (37, 53, 29, "T", "T"),      # low-rank path (no split-K)
]


def _operands(m, n, k, ta, tb, seed):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn((m, k) if ta == "N" else (k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n) if tb == "N" else (n, k), generator=g, dtype=torch.float64)
    C0 = torch.randn((m, n), generator=g, dtype=torch.float64)
    return A, B, C0


def _run(lib, fn, m, n, k, ta, tb, A, B, C0):
    dA = A.T.contiguous().cuda()
    dB = B.T.contiguous().cuda()
    dC = C0.T.contiguous().cuda()
    fn(ta, tb, m, n, k, 0.9, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0], -0.4,
       dC.data_ptr(), m)
    return dC.cpu().T


def test_static_scratch_matches_allocating_entry_point():
    lib = ab.load()
    for rep in range(2):          # two calls in a row: the shared array is reused
        for idx, (m, n, k, ta, tb) in enumerate(SHAPES):
            A, B, C0 = _operands(m, n, k, ta, tb, 100 * rep + idx)
            ref = _run(lib, lib.xgemm, m, n, k, ta, tb, A, B, C0)
            out = _run(lib, lib.xgemm_static, m, n, k, ta, tb, A, B, C0)
            err = (out - ref).abs().max().item()
            assert err <= 1e-12 * max(1.0, ref.abs().max().item()) * np.sqrt(k), (m, n, k, err)
            # and directly against an FP64 product on the host
            opA = A if ta == "N" else A.T
            opB = B if tb == "N" else B.T
            exact = 0.9 * opA @ opB - 0.4 * C0
            err = (out - exact).abs().max().item()
            assert err <= 1e-12 * max(1.0, exact.abs().max().item()) * np.sqrt(k), (m, n, k, err)


def test_static_scratch_requests_no_device_memory():
    """The defining property: across calls of every shape above (after one
    warm-up call per shape, which also looks up the array's address), the
    library's allocator sees no request at all -- neither a cached block nor a
    cudaMalloc -- while the allocating entry point does request scratch."""
    import torch
    lib = ab.load()
    ops = []
    for idx, (m, n, k, ta, tb) in enumerate(SHAPES):
        A, B, C0 = _operands(m, n, k, ta, tb, 7 + idx)
        dA, dB = A.T.contiguous().cuda(), B.T.contiguous().cuda()
        dC = C0.T.contiguous().cuda()
        ops.append((m, n, k, ta, tb, dA, A.shape[0], dB, B.shape[0], dC))

    def call(fn, op):
        m, n, k, ta, tb, dA, lda, dB, ldb, dC = op
        fn(ta, tb, m, n, k, 1.0, dA.data_ptr(), lda, dB.data_ptr(), ldb, 0.0, dC.data_ptr(), m)

    for op in ops:
        call(lib.xgemm_static, op)
    torch.cuda.synchronize()
    before = lib.pool_stats()
    for _ in range(2):
        for op in ops:
            call(lib.xgemm_static, op)
    torch.cuda.synchronize()
    after = lib.pool_stats()
    assert after[:2] == before[:2], (before, after)
    call(lib.xgemm, ops[0])       # transa = 'N': the allocating path copies op(A)
    assert lib.pool_stats()[0] > after[0]


def test_static_scratch_rejects_requests_beyond_its_size():
    import torch
    lib = ab.load()
    m, k = 2048, 1024          # op(A) copy alone needs 2^21 doubles > 2^20
    A = torch.zeros((m, k), dtype=torch.float64, device="cuda")
    B = torch.zeros((k, 8), dtype=torch.float64, device="cuda")
    C = torch.zeros((m, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(ab.AcesError) as e:
        lib.xgemm_static("N", "N", m, 8, k, 1.0, A.data_ptr(), m, B.data_ptr(), k, 0.0,
                         C.data_ptr(), m)
    assert e.value.status == -1
