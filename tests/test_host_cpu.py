"""CPU-only checks of the host side: mesh generators against the oracle, and
the C-ABI library loading with every symbol include/fenics_cuda.h declares.
No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "fenics_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fcu_[a-z0-9_]+)\s*\(", txt)))


def test_generators_match_oracle_bitwise(fcu):
    for nx, ny in ((1, 1), (4, 4), (7, 3)):
        a, b = fcu.unit_square(nx, ny), O.unit_square(nx, ny)
        assert np.array_equal(a.coords, b.coords) and np.array_equal(a.cells, b.cells)
    for args in ((1.0, 1.0, 1.0, 1, 1, 1), (4.0, 1.0, 1.0, 8, 2, 2), (3.0, 1.0, 1.0, 5, 3, 2)):
        a, b = fcu.box_beam(*args), O.box_beam(*args)
        assert np.array_equal(a.coords, b.coords) and np.array_equal(a.cells, b.cells)


def test_library_exports_every_declared_symbol(fcu):
    from fenics_cuda import _abi
    lib = ctypes.CDLL(_abi.SO)
    syms = _header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert sorted(_abi.SIGNATURES) == syms


def test_material_validation(fcu):
    import pytest
    with pytest.raises(ValueError):
        fcu.ElasticMaterial(1.0, 0.5)
    m = fcu.ElasticMaterial(210e9, 0.3)
    assert abs(m.lame_mu() - 210e9 / 2.6) < 1e-3


def test_vector_bc_arrays(fcu):
    bc = fcu.VectorDirichletBC([(3, 0.0), (4, 1.5)])
    d, v = bc.arrays()
    assert d.tolist() == [3, 4] and v.tolist() == [0.0, 1.5]


def test_concat_meshes_layout(fcu):
    """A batch's concatenated mesh: disjoint vertex ranges, renumbered cells,
    and a boundary that is the union of the instances' boundaries."""
    parts = [O.unit_square(n, n) for n in (3, 5, 2)]
    mesh, offs = fcu.concat_meshes([fcu.Mesh(p.coords, p.cells) for p in parts])
    assert offs.tolist() == [0, 16, 52, 61]
    assert mesh.nv == 61 and mesh.nc == sum(p.cells.shape[0] for p in parts)
    for p, o, c0 in zip(parts, offs[:-1], np.cumsum([0] + [q.cells.shape[0] for q in parts])[:-1]):
        assert np.array_equal(mesh.coords[o:o + p.coords.shape[0]], p.coords)
        assert np.array_equal(mesh.cells[c0:c0 + p.cells.shape[0]], p.cells + o)
    om = O.Mesh(mesh.coords, mesh.cells)
    want = np.concatenate([O.boundary_dofs_2d(p) + o for p, o in zip(parts, offs[:-1])])
    assert np.array_equal(O.boundary_dofs_2d(om), want)
    with pytest.raises(ValueError):
        fcu.concat_meshes([])


def test_package_imports_without_torch():
    """The product package allocates and copies device memory through the
    library's own C ABI (DeviceArray), so it imports and loads with torch
    unavailable, as a Rust caller would run it."""
    import subprocess
    import sys
    code = ("import sys; sys.modules['torch'] = None\n"
            "sys.path.insert(0, %r)\n"
            "import fenics_cuda as f\n"
            "f._abi.lib()\n"
            "assert f.DeviceArray and f.device_count() >= 0\n"
            "bad = [m for m in sys.modules if m == 'torch' or m.startswith('torch.')]\n"
            "assert all(sys.modules[m] is None for m in bad), bad\n"
            "print('ok')\n") % os.path.join(ROOT, "fenics-rs_b200")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr


def test_profile_summaries_give_traffic():
    """Every profile summary bench.py reads a roofline's DRAM traffic from
    exists and states it per launch."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for name in ("spmv_bsr3_fp32_elasticity_c2.txt", "spmv_bsr3_fp64_elasticity_c2.txt",
                 "pcg_persistent_fp32_elasticity_c2.txt", "spmv_bsr3_fp32_elasticity_c2p.txt"):
        t = bench._profile_traffic(name)
        assert t is not None and t > 0, name
