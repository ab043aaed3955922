"""The persistent PCG loop on 3x3-block systems.

Mixed-precision elasticity solves on the tiled operator run as one
cooperative launch per stretch between residual replacements, with grid
barriers instead of kernel boundaries; FP64 solves keep the per-iteration
kernel graph unless FCU_PERSISTENT=2 (one launch per solve). These tests hold
the loop in both precisions to the oracle's CG (cg.rs:40-149 restated) and to
the graph, in child processes with FCU_PERSISTENT=2 (the loop for both) and
FCU_PERSISTENT=0 (the graph for both), on:
  * a beam whose 64-row tiles give most CTAs no tile at all and the one
    loaded CTA fewer tiles than ring stages (its producer runs iterations
    ahead of the consumers);
  * the 16x4x4 beam of the elasticity CG parity test;
  * the 200x50x50 beam in FP64, where a CTA's share exceeds the 32 tile
    descriptors its producer warp holds at once.
All calls go through the C ABI (libfenics_cuda.so).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/fenics-rs_b200")
import fenics_cuda as fcu
dims, out = json.loads(sys.argv[1]), sys.argv[2]
ctx = fcu.Context(0)
m = fcu.box_beam(4.0, 1.0, 1.0, *dims)
cv = np.nonzero(m.coords[:, 0] < 1e-6)[0]
dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
V = fcu.FunctionSpace(ctx, m, fcu.FCU_SPACE_P1_VEC3)
M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
b = V.body_force([0.0, 0.0, -7.8e4])
M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
res = {}
for name, prec in (("fp64", fcu.FCU_FP64), ("mixed", fcu.FCU_MIXED)):
    x, info = M.pcg(b, tol=1e-8, max_iter=100000, precision=prec)
    np.save(out + "_" + name + ".npy", x)
    res[name] = [int(info.iterations), int(info.outer_updates), int(info.status)]
print(json.dumps(res))
'''.replace("ROOT", repr(ROOT))


def _child(dims, tmp_path, mode):
    env = dict(os.environ, FCU_PERSISTENT=mode)
    out = str(tmp_path / ("mode" + mode))
    r = subprocess.run([sys.executable, "-c", CHILD, json.dumps(list(dims)), out], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    return res, {k: np.load(out + "_" + k + ".npy") for k in ("fp64", "mixed")}


def _system(fcu, ctx, dims):
    m = fcu.box_beam(4.0, 1.0, 1.0, *dims)
    cv = np.nonzero(m.coords[:, 0] < 1e-6)[0]
    dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
    V = fcu.FunctionSpace(ctx, m, fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    b = V.body_force([0.0, 0.0, -7.8e4])
    M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
    return m, dofs, V, M, b


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("dims", [(2, 1, 1), (16, 4, 4)])
def test_persistent_matches_oracle_and_graph(fcu, ctx, dims, tmp_path):
    om = O.box_beam(4.0, 1.0, 1.0, *dims)
    dofs = O.clamp_dofs(om)
    K = O.assemble_elasticity_3d(om, 210e9, 0.3)
    f = O.body_force_3d(om, [0.0, 0.0, -7.8e4])
    Kb, fb = O.apply_dirichlet_bc(K, f, dofs, np.zeros(len(dofs)))
    x_o, it_o, _ = O.solve_cg(Kb, fb, None, 1e-8, 20000)
    p_info, p_x = _child(dims, tmp_path, "2")
    g_info, g_x = _child(dims, tmp_path, "0")
    A = Kb.to_scipy()
    for name in ("fp64", "mixed"):
        x, it, it_g = p_x[name], p_info[name][0], g_info[name][0]
        assert p_info[name][2] == 0 and g_info[name][2] == 0
        print(f"{dims} {name}: persistent {it} it ({p_info[name][1]} replacements), "
              f"graph {it_g} it, oracle {it_o} it; |x - x_graph| {_rel(x, g_x[name]):.2e}, "
              f"|x - x_oracle| {_rel(x, x_o):.2e}")
        assert np.linalg.norm(fb - A @ x) / np.linalg.norm(fb) < 1e-8
        assert _rel(x, x_o) <= 1e-6
        assert _rel(x, g_x[name]) <= 1e-6
        if name == "fp64":
            # the same recurrence as cg.rs and as the graph; p.Ap and r.z are
            # summed over other CTA groupings, so counts may differ by round-off
            assert abs(it - it_o) <= max(3, 0.02 * it_o)
            assert abs(it - it_g) <= max(2, 0.01 * it_g)
        else:
            # the FP32 operator's iteration count follows its rounding order
            # (4,393-4,844 at 200x50x50 over builds of the graph path)
            assert abs(it - it_g) <= max(3, 0.15 * it_g)
    # in this process (default policy) the mixed solve is the persistent one
    m, dofs2, V, M, b = _system(fcu, ctx, dims)
    xm, infom = M.pcg(b, tol=1e-8, max_iter=100000, precision=fcu.FCU_MIXED)
    assert infom.iterations == p_info["mixed"][0] and np.array_equal(xm, p_x["mixed"])


def test_persistent_iteration_limit_and_restart(fcu, ctx):
    m, dofs, V, M, b = _system(fcu, ctx, (16, 4, 4))
    # cg.rs: the limit without convergence is an error (status 3,
    # FCU_ERR_NO_CONVERGENCE); x holds the iterate
    x7, info = M.pcg(b, tol=1e-12, max_iter=7, precision=fcu.FCU_MIXED, raise_on_error=False)
    assert info.iterations == 7 and info.status == 3
    # continuing from the iterate gives the same solution as one solve
    x_full, _ = M.pcg(b, tol=1e-9, max_iter=100000, precision=fcu.FCU_MIXED)
    x_cont, info_c = M.pcg(b, x0=x7, tol=1e-9, max_iter=100000, precision=fcu.FCU_MIXED)
    assert info_c.status == 0 and _rel(x_cont, x_full) <= 1e-6
    # an exact initial guess converges at iteration 0
    x0, info0 = M.pcg(b, x0=x_full, tol=1e-6, max_iter=100, precision=fcu.FCU_MIXED)
    assert info0.iterations == 0 and np.array_equal(x0, x_full)


def test_time_pcg_runs_its_iteration_count(fcu, ctx):
    m, dofs, V, M, b = _system(fcu, ctx, (16, 4, 4))
    for prec, w in ((fcu.FCU_MIXED, 4), (fcu.FCU_FP64, 8)):
        ms, by = M.time_pcg(prec, iterations=50, reps=2)
        n, nnzb = M.n, V.nnz // 9
        per_it = nnzb * (9 * w + 4) + 4 * (n // 3 + 1) + n * (3 * w + 24 + 3 * w + 16 + 2 * w)
        assert ms > 0 and by == pytest.approx(50 * per_it, rel=1e-12)
    # the solver is usable afterwards
    x, info = M.pcg(b, tol=1e-8, max_iter=100000, precision=fcu.FCU_MIXED)
    assert info.status == 0


def test_persistent_large_share_matches_graph(fcu, ctx, tmp_path):
    dims = (200, 50, 50)
    p_info, p_x = _child(dims, tmp_path, "2")
    g_info, g_x = _child(dims, tmp_path, "0")
    for name in ("fp64", "mixed"):
        it, it_g = p_info[name][0], g_info[name][0]
        print(f"{dims} {name}: persistent {it} it, graph {it_g} it, |x - x_graph| {_rel(p_x[name], g_x[name]):.2e}")
        assert p_info[name][2] == 0
        assert _rel(p_x[name], g_x[name]) <= 1e-6
        assert abs(it - it_g) <= max(3, (0.01 if name == "fp64" else 0.15) * it_g)


def test_bounded_waits_give_up_and_report(fcu, ctx):
    """The waits the loop and the tiled SpMV rely on are bounded: a grid
    barrier whose arrival count is never reached and an mbarrier nothing
    arrives at each give up after their polls and say so, while the same
    waits with their condition met pass; the context stays usable (a solve
    follows). No wait is left unbounded and nothing traps."""
    import ctypes as C
    lib = fcu._abi.lib()
    res = (C.c_int * 4)()
    for polls in (64, 4096):
        assert lib.fcu_check_wait_limits(ctx.h, polls, res) == 0, lib.fcu_last_error(ctx.h)
        assert list(res) == [0, 1, 0, 1], (polls, list(res))
    assert lib.fcu_check_wait_limits(ctx.h, 0, res) == fcu._abi.FCU_ERR_BAD_ARG
    assert lib.fcu_check_wait_limits(ctx.h, (1 << 20) + 1, res) == fcu._abi.FCU_ERR_BAD_ARG
    om = O.box_beam(4.0, 1.0, 1.0, 8, 2, 2)
    V = fcu.FunctionSpace(ctx, fcu.Mesh(om.coords, om.cells), fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    dofs = O.clamp_dofs(om)
    b = V.body_force([0.0, 0.0, -7.8e4])
    M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
    x, info = M.pcg(b, tol=1e-8, max_iter=10000, precision=fcu.FCU_MIXED)
    assert info.status == 0
    M.close()
    V.close()
