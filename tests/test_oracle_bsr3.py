"""The oracle's restatement of the block CSR operators (gpu.rs:434-1141)
against independent computations (scipy BSR products, dense solves) and the
reference's own BSR3 test (gpu.rs:1666-1760: PCG to 1e-9 within 500
iterations on the 15^3-node case)."""
import numpy as np

import oracle as O
from bsr3_cases import synthetic_bsr3


def test_bsr3_spmv_and_inverse_blocks():
    nn, rp, ci, va, dinv = synthetic_bsr3(6)
    import scipy.sparse as sp
    B = sp.bsr_matrix((va.reshape(-1, 3, 3), ci, rp), shape=(3 * nn, 3 * nn))
    x = np.arange(3 * nn) % 17 * 0.1   # the reference's x_in
    assert np.max(np.abs(O.bsr3_spmv(nn, rp, ci, va, x) - B @ x)) <= 1e-12
    assert np.max(np.abs(O.bsr3_block_inverse(nn, rp, ci, va) - dinv)) <= 1e-15


def test_bsr3_pcg_reference_case():
    nn, rp, ci, va, dinv = synthetic_bsr3(15)
    b = np.ones(3 * nn)
    x, it, rel = O.solve_bsr3_pcg(nn, rp, ci, va, dinv, b, None, 1e-9, 500)
    assert rel < 1e-9 and it < 500
    assert np.linalg.norm(b - O.bsr3_spmv(nn, rp, ci, va, x)) / np.linalg.norm(b) < 2e-9
    z, it0, rel0 = O.solve_bsr3_pcg(nn, rp, ci, va, dinv, np.zeros(3 * nn))
    assert it0 == 0 and rel0 == 0.0 and not z.any()


def test_bsr3_jacobi_smooth_converges_and_zero_start():
    nn, rp, ci, va, dinv = synthetic_bsr3(5)
    r = np.sin(np.arange(3 * nn))
    # zero_initial_z: the first sweep is z = D^-1 r
    z0 = O.bsr3_jacobi_smooth(nn, rp, ci, va, dinv, r, np.zeros(3 * nn), 1, 0.8, True)
    assert np.array_equal(z0, O.bsr3_apply_dinv(dinv, r))
    # from z = 0 the explicit first sweep gives omega D^-1 r
    z1 = O.bsr3_jacobi_smooth(nn, rp, ci, va, dinv, r, np.zeros(3 * nn), 1, 0.8, False)
    assert np.allclose(z1, 0.8 * O.bsr3_apply_dinv(dinv, r), rtol=1e-15, atol=0)
    zz = np.full(3 * nn, 2.0)
    assert np.array_equal(O.bsr3_jacobi_smooth(nn, rp, ci, va, dinv, r, zz, 0, 0.8, True), zz)
    # diagonally dominant: the sweeps converge to A^-1 r
    A = np.stack([O.bsr3_spmv(nn, rp, ci, va, e) for e in np.eye(3 * nn)], axis=1)
    ex = np.linalg.solve(A, r)
    z40 = O.bsr3_jacobi_smooth(nn, rp, ci, va, dinv, r, np.zeros(3 * nn), 40, 1.0, True)
    assert np.linalg.norm(z40 - ex) < 1e-6 * np.linalg.norm(ex)


def test_multi_gpu_row_split_reassembles_the_product():
    # spmv_bsr3_multi_gpu's split (gpu.rs:662-771): each range's rows, computed
    # with the range's blocks and a row pointer that empties the other rows,
    # reassemble the full product for 1-4 parts (host logic; no GPU needed)
    import fenics_cuda as fcu
    nn, rp, ci, va, _ = synthetic_bsr3(5)
    x = np.cos(np.arange(3 * nn))
    full = O.bsr3_spmv(nn, rp, ci, va, x)
    for parts in (1, 2, 3, 4):
        y = np.zeros(3 * nn)
        split = fcu.bsr3_row_split(nn, rp, parts)
        assert [(a, b) for a, b, *_ in split] == [(i * -(-nn // parts), min((i + 1) * -(-nn // parts), nn))
                                                 for i in range(parts) if i * -(-nn // parts) < nn]
        for r0, r1, sub, b0, b1 in split:
            assert len(sub) == nn + 1 and sub[0] == 0 and sub[-1] == b1 - b0
            part = O.bsr3_spmv(nn, sub, ci[b0:b1], va[9 * b0:9 * b1], x)
            assert not part[:3 * r0].any() and not part[3 * r1:].any()
            y[3 * r0:3 * r1] = part[3 * r0:3 * r1]
        assert np.array_equal(y, full)
