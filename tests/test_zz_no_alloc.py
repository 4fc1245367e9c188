"""The allocation-free Poisson solve (oracle_b200_poisson_solve_noalloc).

It exists for callers that cannot call cudaMalloc when they need a solve, for
example a process whose own allocator already holds the GPU's memory, or a
framework whose memory pool must stay the only owner of device memory.  Its
working memory is one fixed array per device, so these tests check that it
gives the same answer as the plan-based oracle_b200_poisson_solve, call after
call, and that it rejects grids that do not fit in that array.

This file is collected last on purpose: run on its own, in a fresh process, it
must pass too.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup():
    from oraclev8_b200 import _lib as L
    from oracle import lh82 as O
    lib = L.load()
    nx, ny, nz = 128, 96, 32
    Lx, Ly, Lz = nx * 20e3, ny * 20e3, 16e3
    z, rho0, th0 = O.build_base_state(nz, Lz)
    return L, lib, (nx, ny, nz, Lx, Ly, Lz), np.ascontiguousarray(rho0), th0


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_solve_matches_plan_solve_on_consecutive_calls(precision):
    from oraclev8_b200._plan import Plan, PlanSpec
    L, lib, (nx, ny, nz, Lx, Ly, Lz), rho0, th0 = _setup()
    dtype = torch.float64 if precision == "fp64" else torch.float32
    tol = 1e-12 if precision == "fp64" else 1e-5
    plan = Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=precision,
                         projection=True))
    grid = L.GridDesc(nx, ny, nz, Lx, Ly, Lz, plan.prec)
    rng = np.random.default_rng(2024)
    for call in range(2):
        d = torch.as_tensor(rng.standard_normal((nx, ny, nz)) * (1e-5 * (call + 1)),
                            dtype=dtype, device="cuda")
        ref = plan.poisson_solve(d)
        out = torch.full_like(d, float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.oracle_b200_poisson_solve_noalloc(
            ctypes.byref(grid), rho0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(out.data_ptr()), _stream())
        assert rc == 0, lib.oracle_b200_last_error()
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        err = float((out - ref).abs().max() / ref.abs().max())
        assert err <= tol, (call, err)


def test_noalloc_rejects_grids_beyond_its_scratch():
    L, lib, _, _, _ = _setup()
    nx = ny = 512
    nz = 64
    from oracle import lh82 as O
    rho0 = np.ascontiguousarray(O.build_base_state(nz, 16e3)[1])
    grid = L.GridDesc(nx, ny, nz, nx * 5e3, ny * 5e3, 16e3, L.OB_PREC_F64)
    d = torch.zeros((nx, ny, nz), dtype=torch.float64, device="cuda")
    rc = lib.oracle_b200_poisson_solve_noalloc(
        ctypes.byref(grid), rho0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), _stream())
    assert rc == L.OB_ERR_ARG
    assert b"at most" in lib.oracle_b200_last_error()
