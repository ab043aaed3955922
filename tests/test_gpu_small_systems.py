"""fcu_pcg on small scalar systems started from zero runs as a single
instance of the batched kernel (one launch). The same solves on the
per-iteration graph (FCU_SMALL_BATCHED=0, read once per process, hence the
subprocesses) must agree: same statuses, iteration counts within 2, and
solutions within 1e-7 relative L2 at a 1e-12 residual tolerance (the two
paths sum in different orders; cg.rs:40-149 semantics either way); the
batched results repeat bit for bit.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_SCRIPT = r"""
import json, sys
import numpy as np
sys.path[:0] = [ROOT, PKG]
import fenics_cuda as fcu
import oracle as O
ctx = fcu.Context(0)
out = []
def solve(A, b, tol, prec, tag, max_iter=5000):
    x, it, res = None, -1, None
    try:
        x, it, res = fcu.solve_cg(A, b, None, tol, max_iter, ctx, precision=prec)
        st = 0
    except fcu.CgError as e:
        st = e.code
    out.append({"tag": tag, "status": st, "it": int(it),
                "x": None if x is None else [float(v) for v in x]})
om = O.unit_square(40, 40)
rng = np.random.default_rng(3)
A = O.assemble_stiffness_2d(om, np.exp(rng.standard_normal(om.nc)))
b = O.assemble_rhs_2d(om, lambda x, y: np.sin(4 * x) + y * y)
bd = O.boundary_dofs_2d(om)
Ab, bb = O.apply_dirichlet_bc(A, b, bd, np.zeros(len(bd)))
for name, prec in (("fp64", fcu.FCU_FP64), ("mixed", fcu.FCU_MIXED)):
    solve(Ab, bb, 1e-12, prec, "p1_" + name)
    solve(Ab, bb, 1e-12, prec, "p1_" + name + "_again")
m3 = O.unit_cube(4, 4, 4)
cd, ev = O.p2_dofmap(m3)
nd = m3.nv + len(ev)
A3 = O.assemble_p2_stiffness_3d(m3, cd, nd, None)
b3 = np.cos(np.arange(nd) * 0.1)
bd3 = O.p2_boundary_dofs(m3)
A3b, b3b = O.apply_dirichlet_bc(A3, b3, bd3, np.zeros(len(bd3)))
solve(A3b, b3b, 1e-12, fcu.FCU_FP64, "p2_fp64")
solve(Ab, bb, 1e-12, fcu.FCU_FP64, "limit", max_iter=10)  # FCU_ERR_NO_CONVERGENCE on both paths
print(json.dumps(out))
"""


def _run(flag):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = f"ROOT = {root!r}; PKG = {os.path.join(root, 'fenics-rs_b200')!r}\n" + _SCRIPT
    env = dict(os.environ, FCU_SMALL_BATCHED=flag)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return {d["tag"]: d for d in json.loads(r.stdout.strip().splitlines()[-1])}


def test_batched_small_systems_agree_with_graph_path():
    on, off = _run("1"), _run("0")
    assert on.keys() == off.keys()
    for tag in on:
        a, b = on[tag], off[tag]
        assert a["status"] == b["status"], tag
        if a["x"] is None:
            continue
        assert abs(a["it"] - b["it"]) <= 2, (tag, a["it"], b["it"])
        xa, xb = np.asarray(a["x"]), np.asarray(b["x"])
        assert np.linalg.norm(xa - xb) <= 1e-7 * max(np.linalg.norm(xb), 1e-300), tag
    assert on["limit"]["status"] == 3
    for name in ("fp64", "mixed"):
        assert on["p1_" + name]["x"] == on["p1_" + name + "_again"]["x"]
        assert on["p1_" + name]["it"] == on["p1_" + name + "_again"]["it"]
