"""Stress recovery (fcu_element_stresses, fcu_vertex_von_mises) against the
oracle's restatement of compute_element_stresses / compute_vertex_von_mises
(elasticity.rs:230-360) and a numpy restatement of the per-cell tensors, on a
perturbed box with one degenerate cell appended (four coplanar corners of a
hexahedron face), which must give zeros and be left out of the vertex
averages."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

E, NU = 210e9, 0.3


def _mesh():
    m = O.box_beam(3.0, 1.0, 1.0, 6, 3, 3)
    rng = np.random.default_rng(31)
    inner = np.all((m.coords > 1e-9) & (m.coords < m.coords.max(axis=0) - 1e-9), axis=1)
    m.coords[inner] += rng.uniform(-0.05, 0.05, (inner.sum(), 3))
    flat = np.array([[0, 1, 7, 8]], np.int64)   # z = 0 face of the first hexahedron
    return O.Mesh(m.coords, np.concatenate([m.cells, flat])), rng


def _numpy_tensors(m, u):
    lam = (E * NU) / ((1 + NU) * (1 - 2 * NU))
    mu = E / (2 * (1 + NU))
    nc = m.cells.shape[0]
    st = np.zeros((nc, 3, 3))
    ep = np.zeros((nc, 3, 3))
    for c in range(nc):
        v = m.coords[m.cells[c]]
        J = (v[1:] - v[0]).T
        if abs(np.linalg.det(J)) < 1e-14:
            continue
        G = np.linalg.inv(J).T
        g = np.vstack([-G.sum(axis=1), G.T])      # rows: gradients of the four basis functions
        un = u.reshape(-1, 3)[m.cells[c]]          # 4 x 3
        gu = un.T @ g                              # du_i/dx_j
        e = 0.5 * (gu + gu.T)
        ep[c] = e
        st[c] = lam * np.trace(e) * np.eye(3) + 2 * mu * e
    return st, ep


def test_element_and_vertex_stresses_match_oracle(fcu, ctx):
    m, rng = _mesh()
    u = rng.normal(scale=1e-3, size=3 * m.nv)
    fm = fcu.Mesh(m.coords, m.cells)
    s = fcu.compute_element_stresses(fm, u, fcu.ElasticMaterial(E, NU), ctx)
    cv, vv = O.von_mises(m, u, E, NU)
    scale = np.max(np.abs(cv))
    assert np.max(np.abs(s.von_mises - cv)) <= 1e-12 * scale
    st, ep = _numpy_tensors(m, u)
    assert np.max(np.abs(s.stress - st)) <= 1e-12 * np.max(np.abs(st))
    assert np.max(np.abs(s.strain - ep)) <= 1e-12 * np.max(np.abs(ep))
    assert np.max(np.abs(s.trace - np.trace(st, axis1=1, axis2=2))) <= 1e-12 * np.max(np.abs(st))
    # the degenerate cell: StressState::default()
    assert s.von_mises[-1] == 0.0 and np.all(s.stress[-1] == 0.0) and s.trace[-1] == 0.0
    vvm = fcu.compute_vertex_von_mises(fm, s, ctx)
    assert np.max(np.abs(vvm - vv)) <= 1e-12 * scale


def test_stresses_on_device_arrays_and_rigid_motion(fcu, ctx):
    import torch
    m, rng = _mesh()
    fm = fcu.Mesh(m.coords, m.cells)
    V = fcu.FunctionSpace(ctx, fm, fcu.FCU_SPACE_P1_VEC3)
    # a rigid motion (translation + small rotation) has no strain and no stress
    w = np.array([1e-3, -2e-3, 5e-4])
    u = (np.cross(np.broadcast_to(w, m.coords.shape), m.coords) + np.array([0.1, 0.2, -0.3])).ravel()
    vm = torch.empty(m.cells.shape[0], dtype=torch.float64, device="cuda")
    V.element_stresses(E, NU, torch.from_numpy(u).cuda(), von_mises=vm)
    assert float(vm.abs().max()) <= 1e-9 * E * 1e-3
    out = torch.empty(m.nv, dtype=torch.float64, device="cuda")
    V.vertex_von_mises(vm, out=out)
    assert float(out.abs().max()) <= 1e-9 * E * 1e-3
    with pytest.raises(fcu.FcuError):
        V.element_stresses(E, 0.5, u)   # ElasticMaterial::new rejects nu = 0.5
    V.close()
