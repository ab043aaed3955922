"""fcu_solve_csr_cg_noalloc: the allocation-free CSR PCG entry point.

Collected last on purpose (file name), so it runs both alone in a fresh
process and after every other test has used the library. Everything goes
through the C ABI: the library's fcu_solve_csr_cg (host arrays, through a
context) is the comparison, the no-alloc entry point gets device arrays on
the current torch stream. The matrix is the 7-point Laplacian that
crates/fenics-solver/src/gpu.rs:1610-1663 solves with solve_csr_cg_gpu, and
the CPU oracle's restatement of cg.rs:40-149 checks the solution.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-9
MAX_ITER = 1000


def _laplacian_csr(nx):
    """7-point Laplacian on nx^3 points as u32 CSR with sorted columns."""
    import scipy.sparse as sp
    e = np.ones(nx)
    t = sp.diags([-e[:-1], 2.0 * e, -e[:-1]], [-1, 0, 1])
    i = sp.identity(nx)
    a = (sp.kron(sp.kron(t, i), i) + sp.kron(sp.kron(i, t), i) + sp.kron(sp.kron(i, i), t)).tocsr()
    a.sort_indices()
    return (a.indptr.astype(np.uint32), a.indices.astype(np.uint32), a.data.astype(np.float64),
            1.0 / a.diagonal())


def _ptr(a):
    return C.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())


def _existing(fcu, ctx, rp, ci, v, inv, b, x0=None):
    lib = fcu._abi.lib()
    n = len(b)
    x = np.zeros(n)
    info = fcu._abi.SolveInfo()
    rc = lib.fcu_solve_csr_cg(ctx.h, n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(inv), _ptr(b),
                              _ptr(x0) if x0 is not None else None, RTOL, MAX_ITER, _ptr(x), C.byref(info))
    assert rc == 0, lib.fcu_last_error(ctx.h)
    return x, info


def _noalloc(fcu, n, dev, b, x, x0=None, max_iter=MAX_ITER):
    import torch
    lib = fcu._abi.lib()
    info = fcu._abi.SolveInfo()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fcu_solve_csr_cg_noalloc(n, _ptr(dev["rp"]), _ptr(dev["ci"]), _ptr(dev["v"]), _ptr(dev["inv"]),
                                      _ptr(b), _ptr(x0) if x0 is not None else None, RTOL, max_iter, _ptr(x),
                                      C.byref(info), C.c_void_p(stream))
    return rc, info


def _close(a, b):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) <= 1e-12 * scale


@pytest.fixture(scope="module")
def system():
    import torch
    rp, ci, v, inv = _laplacian_csr(20)
    dev = {"rp": torch.from_numpy(rp.view(np.int32)).cuda(), "ci": torch.from_numpy(ci.view(np.int32)).cuda(),
           "v": torch.from_numpy(v).cuda(), "inv": torch.from_numpy(inv).cuda()}
    return rp, ci, v, inv, dev


def test_noalloc_matches_existing_entry_two_calls(fcu, ctx, system):
    import torch
    rp, ci, v, inv, dev = system
    n = len(inv)
    rng = np.random.default_rng(7)
    rhs = [np.ones(n), rng.standard_normal(n)]
    want = [_existing(fcu, ctx, rp, ci, v, inv, b) for b in rhs]
    for (b, (x_ref, info_ref)) in zip(rhs, want):
        bd = torch.from_numpy(b).cuda()
        xd = torch.full((n,), 3.0, dtype=torch.float64, device="cuda")  # stale output must not matter
        rc, info = _noalloc(fcu, n, dev, bd, xd)
        assert rc == 0, fcu._abi.lib().fcu_last_error(None)
        assert info.status == 0
        assert info.iterations == info_ref.iterations
        assert info.rel_residual < RTOL
        assert _close(xd.cpu().numpy(), x_ref)


def test_noalloc_matches_oracle_cg(fcu, system):
    """x and the iteration count against the oracle's CG (cg.rs:40-149) on the
    same Laplacian (symmetric, so its CSR arrays are its CSC arrays)."""
    import torch
    import oracle as O
    rp, ci, v, inv, dev = system
    n = len(inv)
    A = O.Csc(n, rp.astype(np.int64), ci.astype(np.int64), v)
    b = np.random.default_rng(11).standard_normal(n)
    x_o, it_o, _ = O.solve_cg(A, b, None, RTOL, MAX_ITER)
    for _ in range(2):
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        rc, info = _noalloc(fcu, n, dev, torch.from_numpy(b).cuda(), xd)
        assert rc == 0, fcu._abi.lib().fcu_last_error(None)
        assert abs(info.iterations - it_o) <= 1
        x = xd.cpu().numpy()
        assert np.linalg.norm(x - x_o) <= 1e-8 * np.linalg.norm(x_o)


def test_noalloc_allocates_no_device_memory(fcu, system):
    import torch
    rp, ci, v, inv, dev = system
    n = len(inv)
    bd = torch.ones(n, dtype=torch.float64, device="cuda")
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(fcu, n, dev, bd, xd)  # first call may load the module
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, _ = _noalloc(fcu, n, dev, bd, xd)
    assert rc == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0


def test_noalloc_initial_guess_in_place_and_zero_rhs(fcu, ctx, system):
    import torch
    rp, ci, v, inv, dev = system
    n = len(inv)
    b = np.linspace(-1.0, 2.0, n)
    x0 = np.sin(np.arange(n) * 0.01)
    x_ref, info_ref = _existing(fcu, ctx, rp, ci, v, inv, b, x0)
    xd = torch.from_numpy(x0.copy()).cuda()
    rc, info = _noalloc(fcu, n, dev, torch.from_numpy(b).cuda(), xd, x0=xd)  # x0 aliases x
    assert rc == 0
    assert info.iterations == info_ref.iterations
    assert _close(xd.cpu().numpy(), x_ref)
    # gpu.rs:1169-1180: b = 0 -> x = 0, Ok, no iterations
    xd = torch.ones(n, dtype=torch.float64, device="cuda")
    rc, info = _noalloc(fcu, n, dev, torch.zeros(n, dtype=torch.float64, device="cuda"), xd)
    assert rc == 0 and info.iterations == 0
    assert float(xd.abs().max()) == 0.0
    # iteration limit: Ok with the residual reported (gpu.rs semantics)
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc, info = _noalloc(fcu, n, dev, torch.ones(n, dtype=torch.float64, device="cuda"), xd, max_iter=5)
    assert rc == 0 and info.iterations == 5 and info.rel_residual > RTOL


def test_noalloc_rejects_bad_arguments(fcu, system):
    import torch
    lib = fcu._abi.lib()
    rp, ci, v, inv, dev = system
    n = len(inv)
    bd = torch.ones(n, dtype=torch.float64, device="cuda")
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    # beyond the scratch capacity: rejected before any pointer is read
    big = fcu._abi.FCU_NOALLOC_MAX_N + 1
    rc, _ = _noalloc(fcu, big, dev, bd, xd)
    assert rc == fcu._abi.FCU_ERR_BAD_ARG
    assert b"capacity" in lib.fcu_last_error(None)
    # host arrays are not staged
    rc, _ = _noalloc(fcu, n, dev, np.ones(n), xd)
    assert rc == fcu._abi.FCU_ERR_BAD_ARG
    assert b"device pointer" in lib.fcu_last_error(None)
    # out-of-range column index
    ci_bad = dev["ci"].clone()
    ci_bad[5] = n
    bad = dict(dev, ci=ci_bad)
    rc, _ = _noalloc(fcu, n, bad, bd, xd)
    assert rc == fcu._abi.FCU_ERR_BAD_ARG
    assert b"out of range" in lib.fcu_last_error(None)
    # a valid call right after the rejected ones still solves
    rc, info = _noalloc(fcu, n, dev, bd, xd)
    assert rc == 0 and info.rel_residual < RTOL
