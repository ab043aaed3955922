"""Adjoint sensitivities through the forward/backward pair (ElasticityAdjoint):
vector-P1 elasticity on a box with E_e = E0 * theta_e^3 (E0 = 1, nu = 0.3),
clamped at x = 0, unit downward traction on the x = L face; objectives the
compliance f^T u and the mean u_z over the vertices of the cells that touch
x = L.

The reference point is the oracle with direct solves (scipy SuperLU):
its adjoint gradient (the same formula, restated on the CPU) and central
finite differences of J with h = 1e-6 on 32 random cells. With direct
solves the difference quotient at h = 1e-6 stays within ~4e-7 of
max |dJ/dtheta| (J is then exact to a few ulps); with an iterative solve at
tolerance tau the quotient would carry ~tau |J| / h of noise instead.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

E0, NU = 1.0, 0.3


def _problem(nx=8, ny=3, nz=3, L=3.0, seed=21):
    m = O.box_beam(L, 1.0, 1.0, nx, ny, nz)
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0.01, 1.0, m.nc)
    verts, cells, _ = O.boundary_facets_3d(m)
    tip = np.all(np.abs(m.coords[verts][..., 0] - L) < 1e-9, axis=1)
    facets = verts[tip]
    f = O.surface_traction_3d(m, facets, lambda x, y, z: (0.0 * x, 0.0 * x, -1.0 + 0.0 * x))
    dofs = O.clamp_dofs(m)
    tipv = np.unique(m.cells[cells[tip]])
    c = np.zeros(3 * m.nv)
    c[3 * tipv + 2] = 1.0 / len(tipv)
    return m, theta, f, dofs, c


def _direct(m, theta, f, dofs, rhs):
    import scipy.sparse.linalg as spl
    A = O.assemble_elasticity_3d(m, E0, NU, E0 * theta ** 3)
    Ab, bb = O.apply_dirichlet_bc(A, rhs, dofs, np.zeros(len(dofs)))
    return spl.spsolve(Ab.to_scipy().tocsc(), bb)


def _J(m, theta, f, dofs, c):
    u = _direct(m, theta, f, dofs, f)
    return float(np.dot(c, u))


@pytest.mark.parametrize("objective", ["compliance", "tip_uz"])
def test_adjoint_gradient_vs_oracle_and_fd(fcu, ctx, objective):
    m, theta, f, dofs, c = _problem()
    cvec = f if objective == "compliance" else c
    adj = fcu.ElasticityAdjoint(fcu.Mesh(m.coords, m.cells), NU, f, dofs,
                                objective="compliance" if objective == "compliance" else c,
                                ctx=ctx, E0=E0, tol=1e-13, precision=fcu.FCU_FP64)
    J = adj.forward(theta)
    g = adj.backward()
    # forward value against the direct solve
    u = _direct(m, theta, f, dofs, f)
    assert abs(J - np.dot(cvec, u)) <= 1e-9 * abs(J)
    # the CPU restatement of the same adjoint, with direct-solve u and lambda
    lam = u if objective == "compliance" else _direct(m, theta, f, dofs, c)
    g_ref = O.adjoint_grad(m, NU, E0, theta, u, lam)
    scale = np.max(np.abs(g_ref))
    assert np.max(np.abs(g - g_ref)) <= 1e-6 * scale
    # central finite differences on random cells
    rng = np.random.default_rng(4)
    h = 1e-6
    for e in rng.choice(m.nc, 32, replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[e] += h
        tm[e] -= h
        fd = (_J(m, tp, f, dofs, cvec) - _J(m, tm, f, dofs, cvec)) / (2 * h)
        assert abs(fd - g[e]) <= 1e-6 * scale
    if objective == "compliance":
        # dJ/dtheta_e = -3 theta_e^2 E0 u_e^T K_e^1 u_e <= 0: stiffening lowers the compliance
        assert np.all(g <= 1e-15 * scale)
    adj.close()


def test_adjoint_backward_scales_and_requires_forward(fcu, ctx):
    m, theta, f, dofs, c = _problem(6, 2, 2)
    adj = fcu.ElasticityAdjoint(fcu.Mesh(m.coords, m.cells), NU, f, dofs, objective=c, ctx=ctx, tol=1e-12)
    with pytest.raises(RuntimeError):
        adj.backward()
    adj.forward(theta)
    g1 = adj.backward()
    g2 = adj.backward(2.5)
    assert np.allclose(g2, 2.5 * g1, rtol=1e-12, atol=0.0)
    assert adj.adjoint_info.iterations > 0
    adj.close()
