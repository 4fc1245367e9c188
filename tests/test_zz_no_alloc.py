"""The allocation-free Poisson solve (oracle_b200_poisson_solve_noalloc).

It exists for callers that cannot call cudaMalloc when they need a solve, for
example a process whose own allocator already holds the GPU's memory, or a
framework whose memory pool must stay the only owner of device memory.  Its
working memory is one fixed array per device, so these tests check that it
gives the same answer as the plan-based oracle_b200_poisson_solve and as the
oracle's Poisson solve, call after call; that it rejects grids that do not fit
in that array; that it refuses a capturing stream without breaking the
capture; and, in a fresh process, what its first call reserves.

This file is collected last on purpose: run on its own, in a fresh process, it
must pass too.
"""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
# FP32 against the FP64 oracle: single-precision input rounding amplified by
# the long-wave modes of the vertical solve (about 1/(k Lz)^2 = 650 at this
# grid's longest wave) stays well under this bound.
TOL = {"fp64": 1e-12, "fp32": 1e-3}
TOL_PLAN = {"fp64": 1e-12, "fp32": 1e-5}


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


def _oracle_solve(d, dims, rho0):
    from oracle import lh82 as O
    nx, ny, nz, Lx, Ly, Lz = dims
    return O.Poisson(nx, ny, nz, Lx, Ly, Lz).solve(d, rho0, O.rho_half_levels(rho0))[0]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_solve_matches_plan_solve_and_oracle_on_consecutive_calls(precision):
    from oraclev8_b200._plan import Plan, PlanSpec
    L, lib, dims, rho0, th0 = _setup()
    nx, ny, nz, Lx, Ly, Lz = dims
    dtype = torch.float64 if precision == "fp64" else torch.float32
    plan = Plan(PlanSpec(nx, ny, nz, Lx, Ly, Lz, rho0, th0, precision=precision,
                         projection=True))
    grid = L.GridDesc(nx, ny, nz, Lx, Ly, Lz, plan.prec)
    rng = np.random.default_rng(2024)
    for call in range(2):
        dh = rng.standard_normal((nx, ny, nz)) * (1e-5 * (call + 1))
        d = torch.as_tensor(dh, dtype=dtype, device="cuda")
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
        assert err <= TOL_PLAN[precision], (call, err)
        # the oracle solves the same (rounded) source in FP64
        phi = _oracle_solve(d.double().cpu().numpy(), dims, rho0)
        err_o = float(np.max(np.abs(out.double().cpu().numpy() - phi)) / np.max(np.abs(phi)))
        assert err_o <= TOL[precision], (call, err_o)


def test_noalloc_rejects_grids_beyond_its_scratch():
    L, lib, _, _, _ = _setup()
    from oracle import lh82 as O
    # 256 x 256 x 32 in FP64 needs two 16.9 MB half-spectrum buffers: over 32 MiB
    nx = ny = 256
    nz = 32
    rho0 = np.ascontiguousarray(O.build_base_state(nz, 16e3)[1])
    grid = L.GridDesc(nx, ny, nz, nx * 5e3, ny * 5e3, 16e3, L.OB_PREC_F64)
    d = torch.zeros((nx, ny, nz), dtype=torch.float64, device="cuda")
    rc = lib.oracle_b200_poisson_solve_noalloc(
        ctypes.byref(grid), rho0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), _stream())
    assert rc == L.OB_ERR_ARG
    assert b"at most" in lib.oracle_b200_last_error()


def test_noalloc_refuses_a_capturing_stream_and_the_capture_survives():
    L, lib, dims, rho0, _ = _setup()
    nx, ny, nz, Lx, Ly, Lz = dims
    grid = L.GridDesc(nx, ny, nz, Lx, Ly, Lz, L.OB_PREC_F64)
    d = torch.zeros((nx, ny, nz), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(d)
    x = torch.zeros(16, device="cuda")
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc = lib.oracle_b200_poisson_solve_noalloc(
            ctypes.byref(grid), rho0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(out.data_ptr()), _stream())
        x.add_(1.0)
    assert rc == L.OB_ERR_ARG
    assert b"captur" in lib.oracle_b200_last_error()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert float(x.min()) == 2.0 and float(x.max()) == 2.0
    del g


_FRESH = r"""
import ctypes, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from oraclev8_b200 import _lib as L
from oracle import lh82 as O
nx, ny, nz = 128, 96, 32
Lx, Ly, Lz = nx * 20e3, ny * 20e3, 16e3
z, rho0, th0 = O.build_base_state(nz, Lz)
rho0 = np.ascontiguousarray(rho0)
lib = L.load()
grid = L.GridDesc(nx, ny, nz, Lx, Ly, Lz, L.OB_PREC_F64)
rng = np.random.default_rng(7)
dh = rng.standard_normal((nx, ny, nz)) * 1e-5
d = torch.as_tensor(dh, device="cuda")
out = torch.full_like(d, float("nan"))
st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
rp = rho0.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
free = [torch.cuda.mem_get_info()[0]]
for _ in range(2):
    rc = lib.oracle_b200_poisson_solve_noalloc(ctypes.byref(grid), rp, ctypes.c_void_p(d.data_ptr()),
                                               ctypes.c_void_p(out.data_ptr()), st)
    assert rc == 0, lib.oracle_b200_last_error()
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
phi = O.Poisson(nx, ny, nz, Lx, Ly, Lz).solve(dh, rho0, O.rho_half_levels(rho0))[0]
err = float(np.max(np.abs(out.cpu().numpy() - phi)) / np.max(np.abs(phi)))
print(json.dumps({"free": free, "err": err}))
"""


def test_noalloc_first_call_in_a_fresh_process():
    """The first call on a device is the one that may load the library's module
    (and with it the fixed array): record free device memory before it, check
    that it reserves no more than the module and the 32 MiB array, that the
    second call reserves nothing, and that both results match the oracle."""
    import json
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    r = subprocess.run([sys.executable, "-c", _FRESH, str(ROOT)], capture_output=True,
                       text=True, timeout=600, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    rep = json.loads(r.stdout.strip().splitlines()[-1])
    f0, f1, f2 = rep["free"]
    assert f0 - f1 <= 256 << 20, rep  # module image + the 32 MiB array
    assert f2 == f1, rep
    assert rep["err"] <= TOL["fp64"], rep
