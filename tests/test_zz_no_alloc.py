"""The allocation-free dot product (gb_dot_noalloc) against gb_vec_dot.

gb_dot_noalloc serves callers that cannot allocate device memory once they run
(applications whose device memory belongs to their own pool allocator from
start-up, loops that cannot take cudaMalloc's device-wide synchronisation). It
uses a fixed file-scope scratch array instead of allocating, so this test
checks, through the C-ABI, that two calls in a row
agree with the context-based gb_vec_dot within the tolerance of the other dot
tests (1e-13 relative to sum |a_i b_i|), and that sizes beyond the scratch
capacity are rejected. This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 4096 * 2048


def test_dot_noalloc_matches_vec_dot_twice():
    import torch

    from gascoignelib_b200.build import build_library
    from gascoignelib_b200.native import GB_EINVAL, GB_OK, Context, lib
    from gascoignelib_b200.problem import Level, Problem

    build_library()
    L = lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(21)
    with Context(0) as ctx:
        # n = 274,625: same partition as gb_vec_dot; n = 2,000,003: a larger grid
        for n in (274_625, 2_000_003):
            idx = np.arange(n, dtype=np.int64)
            lv = Level(n=n, B=1, rowptr=np.arange(n + 1, dtype=np.int64), col=idx,
                       diag=idx, val=np.ones(n), dirichlet=np.zeros(0, np.int64))
            P = Problem(dim=1, levels=[lv], transfers=[], rhs=np.zeros(n))
            fl = 0
            assert n <= MAX_N
            ctx.load_problem(P)
            va, vb = ctx.vec(), ctx.vec()
            for call in range(2):
                a = rng.standard_normal(n)
                b = rng.standard_normal(n)
                ctx.upload(fl, va, a)
                ctx.upload(fl, vb, b)
                ref = ctx.dot(fl, va, vb)
                ta = torch.from_numpy(a).to(dev)
                tb = torch.from_numpy(b).to(dev)
                out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
                rc = L.gb_dot_noalloc(C.c_void_p(ta.data_ptr()), C.c_void_p(tb.data_ptr()),
                                      n, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
                assert rc == GB_OK
                got = out.item()
                scale = float(np.abs(a * b).sum())
                assert abs(got - ref) <= 1e-13 * scale, (got, ref)
                assert abs(got - float(a @ b)) <= 1e-13 * scale
                if n <= 296 * 2048:
                    assert got == ref  # same partition as gb_vec_dot: same bits
            ctx.free(va)
            ctx.free(vb)
        # beyond the scratch capacity: rejected before touching memory
        t = torch.zeros(4, dtype=torch.float64, device=dev)
        rc = L.gb_dot_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()),
                              MAX_N + 1, C.c_void_p(t.data_ptr()), C.c_void_p(stream))
        assert rc == GB_EINVAL
