"""cfd_block_gs_static: the block Gauss-Seidel entry point that allocates no
device memory (scratch in one static device array of the library).

It runs the same level-scheduled sweeps with the same kernels as
cfd_block_gs, so on the same system its solution and RMS must agree bit for
bit with cfd_block_gs (which is itself bit-exact against the reference's
MC_Iterative_Block_LU_Jacobi_CRS, MATH/src/MC_Iterative_Jacobi.c:346).  The
system lives in caller-owned device arrays (torch tensors here) and is passed
through the C ABI as raw device pointers.  Calls are made back to back, on
systems of different sizes, to show that nothing left in the static array by
one call changes the next.  This file is named to be collected last so it also
runs after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, capi
from tests._util import make_case, params_from

pytestmark = pytest.mark.gpu


def _system(n, seed):
    """Roe Jacobian system of an n^3-hex tet cube, plus cfd_block_gs results."""
    m, cfg, Q = make_case(n=n, seed=seed)
    out = {}
    with Euler3DGPU(m, params_from(cfg)) as s:
        s.set_state(Q)
        s.begin_iteration(0)
        s.Apply_Boundary_Condition(0)
        s.Compute_Residual(1)
        s.Compute_DeltaT(0)
        s.Compute_Jacobian(1, 0)
        IA, JA, IAU = s.get_block_pattern()
        A, B, _ = s.get_system()
        for sweeps, direction in ((6, 0), (5, 2)):
            rms = s.MC_Iterative_Block_LU_Jacobi_CRS(sweeps, direction)
            out[(sweeps, direction)] = (s.get_system()[2].copy(), rms)
    return dict(n=m.nnode, IA=IA, JA=JA, IAU=IAU, A=A, B=B, expect=out)


def _static_gs(torch, sysd, sweeps, direction):
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(sysd[k])).to(dev) for k in ("IA", "JA", "IAU", "A", "B")}
    X = torch.full((sysd["n"], 5), float("nan"), dtype=torch.float64, device=dev)  # must be cleared by the call
    torch.cuda.synchronize()
    rms = C.c_double()
    code = capi.lib.cfd_block_gs_static(sysd["n"], t["IA"].data_ptr(), t["JA"].data_ptr(), t["IAU"].data_ptr(),
                                        t["A"].data_ptr(), t["B"].data_ptr(), X.data_ptr(), sweeps, direction,
                                        None, C.byref(rms))
    capi.check(code, "cfd_block_gs_static")
    torch.cuda.synchronize()
    return X.cpu().numpy(), rms.value


def test_static_block_gs_matches_allocating_entry_point(gpu_available):
    import torch

    big = _system(20, 11)  # 9261 block rows
    small = _system(6, 3)  # 343 block rows
    assert big["n"] <= capi.GS_STATIC_MAX_ROWS
    for sysd in (big, small, big):
        for (sweeps, direction), (x_ref, rms_ref) in sysd["expect"].items():
            for _ in range(2):  # two calls in a row on the same system
                x, rms = _static_gs(torch, sysd, sweeps, direction)
                np.testing.assert_array_equal(x, x_ref)
                assert rms == rms_ref


def test_static_block_gs_rejects_too_many_rows(gpu_available):
    import torch

    dev = torch.device("cuda:0")
    n = capi.GS_STATIC_MAX_ROWS + 1
    IA = torch.zeros(2, dtype=torch.int32, device=dev)
    buf = torch.zeros(25, dtype=torch.float64, device=dev)
    rms = C.c_double()
    # rejected from the size alone, before any device array is read
    code = capi.lib.cfd_block_gs_static(n, IA.data_ptr(), IA.data_ptr(), IA.data_ptr(), buf.data_ptr(),
                                        buf.data_ptr(), buf.data_ptr(), 1, 0, None, C.byref(rms))
    assert code == -9  # CFD_ERR_RANGE
    assert b"static scratch capacity" in capi.lib.cfd_last_error()


def _call_raw(torch, n, IA, JA, IAU, nnzb):
    """Call cfd_block_gs_static on a caller-built pattern (host lists) with
    device buffers sized for it; returns the status code."""
    dev = torch.device("cuda:0")
    t = lambda a: torch.tensor(a, dtype=torch.int32, device=dev)  # noqa: E731
    dIA, dJA, dIAU = t(IA), t(JA), t(IAU)
    A = torch.zeros((max(nnzb, 1), 5, 5), dtype=torch.float64)
    for r, k in enumerate(IAU):
        if 0 <= k < nnzb:
            A[k] = torch.eye(5, dtype=torch.float64)  # identity diagonal blocks: a solvable system
    A = A.to(dev)
    B = torch.zeros(n * 5, dtype=torch.float64, device=dev)
    X = torch.zeros(n * 5, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rms = C.c_double()
    return capi.lib.cfd_block_gs_static(n, dIA.data_ptr(), dJA.data_ptr(), dIAU.data_ptr(), A.data_ptr(),
                                        B.data_ptr(), X.data_ptr(), 1, 0, None, C.byref(rms))


def test_static_block_gs_rejects_bad_patterns_before_any_launch(gpu_available):
    """The caller's pattern is validated on the host, so each malformed one
    below returns CFD_ERR_ARG without a kernel ever indexing through it.  Every
    device buffer is allocated at the size the (bad) pattern itself claims, so
    the host-side copies stay inside them."""
    import torch

    # a valid 3-row tridiagonal pattern: rows {0,1}, {0,1,2}, {1,2}
    IA = [0, 2, 5, 7]
    JA = [0, 1, 0, 1, 2, 1, 2]
    IAU = [0, 3, 6]
    assert _call_raw(torch, 3, IA, JA, IAU, 7) == 0
    cases = {
        "IA not starting at 0": ([1, 2, 5, 7], JA, IAU),
        "IA decreasing": ([0, 5, 2, 7], JA, IAU),
        "empty row": ([0, 2, 2, 7], JA, IAU),
        "JA out of range": (IA, [0, 1, 0, 1, 3, 1, 2], IAU),
        "negative JA": (IA, [0, -1, 0, 1, 2, 1, 2], IAU),
        "IAU outside its row": (IA, JA, [0, 5, 6]),
        "IAU past the pattern": (IA, JA, [0, 3, 9]),
        "IAU not on the diagonal": (IA, JA, [1, 3, 6]),
    }
    for what, (ia, ja, iau) in cases.items():
        code = _call_raw(torch, 3, ia, ja, iau, len(ja))
        assert code == -1, what  # CFD_ERR_ARG
    # after the rejections the entry point still solves a real system
    sysd = _system(6, 3)
    (x_ref, rms_ref) = sysd["expect"][(6, 0)]
    x, rms = _static_gs(torch, sysd, 6, 0)
    np.testing.assert_array_equal(x, x_ref)


def test_static_block_gs_allocates_no_device_memory(gpu_available):
    """After the first call on the device, further calls leave the device's
    free memory exactly unchanged: the entry point reaches no allocator (all
    buffers of this test are created before the measured calls)."""
    import torch

    sysd = _system(12, 5)
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(sysd[k])).to(dev) for k in ("IA", "JA", "IAU", "A", "B")}
    X = torch.empty((sysd["n"], 5), dtype=torch.float64, device=dev)
    rms = C.c_double()

    def call():
        code = capi.lib.cfd_block_gs_static(sysd["n"], t["IA"].data_ptr(), t["JA"].data_ptr(),
                                            t["IAU"].data_ptr(), t["A"].data_ptr(), t["B"].data_ptr(),
                                            X.data_ptr(), 6, 0, None, C.byref(rms))
        capi.check(code, "cfd_block_gs_static")

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    np.testing.assert_array_equal(X.cpu().numpy(), sysd["expect"][(6, 0)][0])
