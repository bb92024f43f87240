"""Failure detection on the GPU, in the forms that fault, trap or hang no GPU.

The reference aborts on CUDA errors (cuda/check_cuda.h:28-67) and has no
bounded device waits; this library returns status codes instead:
- a device-side wait that runs out (the grid barriers of the multi-CTA cycle,
  made to wait for CTAs that do not exist) ends the kernel, the call returns
  GB_ETIMEOUT and the context stays usable;
- a NaN or Inf in the right-hand side or in the matrix values ends the solve
  with the reference's CGInfo outcome (Common/cginfo.cc:201-255: NaN passes
  none of its tests, so the status stays "running" until the Krylov memory is
  used up), checked against the oracle's restatement, and the flexible solver
  stops at once with GB_ENOTCONV;
- a failing device allocation (host-side fault injection in the library's
  allocator) returns GB_ENOMEM and leaks no device memory.
"""
import os

import numpy as np
import pytest

from gascoignelib_b200.native import (GB_ENOMEM, GB_ETIMEOUT, GB_FP32, GB_FP64, Context,
                                      GBError, lib)
from gascoignelib_b200.problem import seeded_inputs, structured_problem
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _problem(refine):
    kappa, rhs = seeded_inputs(3, 1, refine)
    return structured_problem(3, 1, refine, kappa, rhs)


def test_bounded_wait_runs_out_and_the_context_recovers():
    # the multi-CTA cycle with software grid barriers covers the levels below
    # the finest: 33^3 finest, its 17^3 level above the single-CTA levels
    P = _problem(5)
    old = os.environ.get("GB_MID")
    os.environ["GB_MID"] = "1"
    try:
        ctx = Context(0)
    finally:
        if old is None:
            os.environ.pop("GB_MID", None)
        else:
            os.environ["GB_MID"] = old
    try:
        ctx.load_problem(P)
        ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-300, maxiter=20)
        l = P.nlevels - 1
        x, b = ctx.vec(), ctx.vec()
        ctx.upload(l, b, P.rhs)
        ref = ctx.fgmres(x, b, GB_FP32)
        assert ref["status_name"] == "converged"
        u_ref = ctx.download(l, x)
        L = lib()
        # every barrier waits for one CTA that does not exist, at most 20 ms
        assert L.gb_set_wait_limit(ctx.h, 20_000_000, 1) == 0
        with pytest.raises(GBError) as e:
            ctx.fgmres(x, b, GB_FP32)
        assert e.value.code == GB_ETIMEOUT
        # the flag is cleared: the next solve with the default bound succeeds
        assert L.gb_set_wait_limit(ctx.h, 1_000_000_000, 0) == 0
        info = ctx.fgmres(x, b, GB_FP32)
        assert info["status_name"] == "converged"
        assert info["iterations"] == ref["iterations"]
        assert np.array_equal(ctx.download(l, x), u_ref)
    finally:
        ctx.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_rhs_gives_the_reference_outcome(ctx, bad):
    P = _problem(3)
    ctx.load_problem(P)
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    rhs = P.rhs.copy()
    rhs[100] = bad
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, rhs)
    info = ctx.gmres(x, b)
    _, io = Oracle(P).gmres(rhs, vmax=21, tol=1e-8)
    assert info["status_name"] == io["status"] == "running"
    assert info["iterations"] == io["iterations"]
    assert np.isnan(info["firstresidual"]) and np.isnan(io["firstresidual"])
    # the flexible solver stops at its first residual test, as exploded
    fi = ctx.fgmres(x, b, GB_FP32, check=False)
    assert fi["status_name"] == "exploded"
    assert fi["iterations"] == 0
    # the context is unharmed: a finite right-hand side solves
    ctx.upload(l, b, P.rhs)
    assert ctx.fgmres(x, b, GB_FP32)["status_name"] == "converged"
    ctx.free(x)
    ctx.free(b)


def test_nonfinite_matrix_value_gives_the_reference_outcome(ctx):
    P = _problem(3)
    F = P.levels[-1]
    good = F.val.copy()
    i = int(F.diag[F.n // 2] + 1)   # an off-diagonal entry of an interior row
    F.val = good.copy()
    F.val[i] = np.nan
    ctx.load_problem(P)
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    _, io = Oracle(P).gmres(vmax=21, tol=1e-8)
    assert info["status_name"] == io["status"]
    assert info["iterations"] == io["iterations"]
    assert ctx.fgmres(x, b, GB_FP64, check=False)["status_name"] != "converged"
    F.val = good
    ctx.load_problem(P)
    ctx.upload(l, b, P.rhs)
    assert ctx.gmres(x, b)["status_name"] == "converged"
    ctx.free(x)
    ctx.free(b)


def test_failed_allocation_returns_enomem_and_leaks_nothing():
    import torch
    L = lib()
    P = _problem(4)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    # the context's own set-up allocations
    assert L.gb_debug_fail_alloc(1) == 0
    with pytest.raises(GBError) as e:
        Context(0)
    assert e.value.code == GB_ENOMEM
    # an allocation in the middle of the upload of the levels
    assert L.gb_debug_fail_alloc(0) == 0
    ctx = Context(0)
    try:
        assert L.gb_debug_fail_alloc(5) == 0
        with pytest.raises(GBError) as e:
            ctx.load_problem(P)
        assert e.value.code == GB_ENOMEM
        assert L.gb_debug_fail_alloc(0) == 0
        # still usable: the whole upload and a solve succeed
        ctx.load_problem(P)
        ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-300, maxiter=100)
        l = P.nlevels - 1
        x, b = ctx.vec(), ctx.vec()
        ctx.upload(l, b, P.rhs)
        assert ctx.fgmres(x, b, GB_FP32)["status_name"] == "converged"
    finally:
        L.gb_debug_fail_alloc(0)
        ctx.close()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    # lazily loaded kernel code may stay resident; the levels (tens of MB) may not
    assert free1 >= free0 - (64 << 20), (free0, free1)
