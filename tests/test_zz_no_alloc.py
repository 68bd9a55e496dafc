"""The allocation-free PCG entry point (lcs_pcg_solve_noalloc) against the regular one.

It exists for callers that cannot allocate device memory while they run -- cudaMalloc and
cudaFree synchronise the whole device, which a fixed-latency loop cannot afford, and a host
that hands all device memory to its own pool allocator leaves none to allocate -- so it keeps
its working vectors in one static device array of the library.  This file is named to be
collected last; it needs nothing from the other tests and also passes on its own in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from luisacomputesimulator_b200 import _capi as A
from luisacomputesimulator_b200.collision import ptr, stream
from luisacomputesimulator_b200.linear import ConjugateGradientSolver, make_bsr
from tests.gpu_util import dev, host
from tests.test_gpu_pcg import contact_system

pytestmark = pytest.mark.gpu


def _solve_noalloc(n, diag, Ab, Bb, b, x, opts):
    st = A.PcgStats()
    rc = A.load().lcs_pcg_solve_noalloc(n, ptr(diag), C.byref(Ab), C.byref(Bb), ptr(b), ptr(x), C.byref(opts),
                                        C.byref(st), stream())
    return rc, st


def test_noalloc_pcg_matches_regular_solve_twice_in_a_row():
    sc, diag_h, Ah, Bh, b_h = contact_system()
    n = sc.num_verts
    diag, b = dev(diag_h), dev(b_h)
    Ab = make_bsr(n, dev(Ah[0]), dev(Ah[1]), dev(Ah[2]))
    Bb = make_bsr(n, dev(Bh[0]), dev(Bh[1]), dev(Bh[2]))
    ref = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    st_ref = ConjugateGradientSolver(n).device_solve(diag, Ab, Bb, b, ref, max_iter=300, rel_tol=1e-4,
                                                     check_every=1)
    opts = A.PcgOpts(300, 1e-4, 1e-10, 1, 0)
    for call in range(2):  # the shared static array keeps the previous call's contents
        x = torch.full((n, 4), 7.0, dtype=torch.float32, device="cuda")
        rc, st = _solve_noalloc(n, diag, Ab, Bb, b, x, opts)
        assert rc == 0, A.load().lcs_last_error()
        assert st.iterations == st_ref["iterations"]
        assert st.rel_residual <= 1e-4
        np.testing.assert_allclose(host(x)[:, :3], host(ref)[:, :3], rtol=1e-6,
                                   atol=1e-6 * float(np.abs(host(ref)).max()))


def test_noalloc_rejects_systems_above_its_limit():
    n = 65536 + 1
    z = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    d = torch.zeros((n, 3, 4), dtype=torch.float32, device="cuda")
    rc, _ = _solve_noalloc(n, d, A.Bsr(n, None, None, None), A.Bsr(n, None, None, None), z, z,
                           A.PcgOpts(10, 1e-4, 1e-10, 1, 0))
    assert rc == 3  # LCS_ERR_CAPACITY
    assert b"65536" in A.load().lcs_last_error()


def test_noalloc_call_allocates_no_device_memory():
    sc, diag_h, Ah, Bh, b_h = contact_system()
    n = sc.num_verts
    diag, b = dev(diag_h), dev(b_h)
    Ab = make_bsr(n, dev(Ah[0]), dev(Ah[1]), dev(Ah[2]))
    Bb = make_bsr(n, dev(Bh[0]), dev(Bh[1]), dev(Bh[2]))
    x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    opts = A.PcgOpts(300, 1e-4, 1e-10, 1, 0)
    assert _solve_noalloc(n, diag, Ab, Bb, b, x, opts)[0] == 0  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _solve_noalloc(n, diag, Ab, Bb, b, x, opts)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_defaults_and_rejected_flags_follow_the_regular_solve():
    sc, diag_h, Ah, Bh, b_h = contact_system()
    n = sc.num_verts
    diag, b = dev(diag_h), dev(b_h)
    Ab = make_bsr(n, dev(Ah[0]), dev(Ah[1]), dev(Ah[2]))
    Bb = make_bsr(n, dev(Bh[0]), dev(Bh[1]), dev(Bh[2]))
    lib = A.load()
    # opts NULL: the regular solve's defaults (100 iterations, checks every 25)
    x0 = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    x1 = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    s0, s1 = A.PcgStats(), A.PcgStats()
    solver = ConjugateGradientSolver(n)
    assert lib.lcs_pcg_solve(solver.h, ptr(diag), C.byref(Ab), C.byref(Bb), ptr(b), ptr(x0), None, C.byref(s0),
                             stream()) == 0
    assert lib.lcs_pcg_solve_noalloc(n, ptr(diag), C.byref(Ab), C.byref(Bb), ptr(b), ptr(x1), None, C.byref(s1),
                                     stream()) == 0
    assert s1.iterations == s0.iterations and s1.iterations % 25 == 0
    for flag in (A.LCS_PCG_PLAIN, A.LCS_PCG_ROWS, A.LCS_PCG_SINGLE_REDUCTION):
        rc, _ = _solve_noalloc(n, diag, Ab, Bb, b, x1, A.PcgOpts(100, 1e-4, 1e-10, 1, flag))
        assert rc == 1  # LCS_ERR_INVALID
