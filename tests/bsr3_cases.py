"""Block CSR test inputs shared by the oracle and GPU tests."""
import numpy as np


def synthetic_bsr3(nx=15):
    """The reference's own BSR3 case (gpu.rs:1666-1741): an nx^3 grid of nodes,
    each coupled to itself and its six neighbours; diagonal block
    [[18, 1, .5], [1, 18, .5], [.5, .5, 18]], off-diagonal blocks -2 I, block
    columns sorted, inverse diagonal blocks in closed form."""
    n_nodes = nx * nx * nx
    diag = np.array([18.0, 1.0, 0.5, 1.0, 18.0, 0.5, 0.5, 0.5, 18.0])
    det = 18.0 * (18.0 * 18.0 - 0.25) - 1.0 * (18.0 - 0.25) + 0.5 * (0.5 - 9.0)
    inv = np.array([(18.0 * 18.0 - 0.25) / det, -(18.0 - 0.25) / det, (0.5 - 9.0) / det,
                    -(18.0 - 0.25) / det, (18.0 * 18.0 - 0.25) / det, -(9.0 - 0.5) / det,
                    (0.5 - 9.0) / det, -(9.0 - 0.5) / det, (18.0 * 18.0 - 1.0) / det])
    off = np.array([-2.0, 0.0, 0.0, 0.0, -2.0, 0.0, 0.0, 0.0, -2.0])
    row_ptr, cols, vals = [0], [], []
    for z in range(nx):
        for y in range(nx):
            for x in range(nx):
                i = (z * nx + y) * nx + x
                nb = [i]
                if x > 0:
                    nb.append(i - 1)
                if x + 1 < nx:
                    nb.append(i + 1)
                if y > 0:
                    nb.append(i - nx)
                if y + 1 < nx:
                    nb.append(i + nx)
                if z > 0:
                    nb.append(i - nx * nx)
                if z + 1 < nx:
                    nb.append(i + nx * nx)
                for j in sorted(nb):
                    cols.append(j)
                    vals.append(diag if j == i else off)
                row_ptr.append(len(cols))
    return (n_nodes, np.array(row_ptr, np.uint32), np.array(cols, np.uint32), np.concatenate(vals),
            np.tile(inv, n_nodes))
