"""CPU checks of the Rust binding crate (crates/fenics-cuda) against the C ABI.

There is no Rust toolchain in this image, so the crate is not compiled here.
These tests read its raw bindings (src/ffi.rs) as text and check them against
include/fenics_cuda.h: every declared function is bound under the same name
with the same number of arguments, each argument and return type maps to the
C type's Rust equivalent, the status/space/precision constants carry the
header's values, and the fcu_solve_info struct has the header's fields in the
header's order. The safe wrappers in src/lib.rs may only call functions that
ffi.rs binds.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fenics_cuda.h")
CRATE = os.path.join(ROOT, "crates", "fenics-cuda")

# C parameter / return type -> the Rust type ffi.rs must use for it
C_TO_RUST = {
    "int": "c_int",
    "int64_t": "i64",
    "size_t": "usize",
    "double": "f64",
    "void": "()",
    "const char*": "*const c_char",
    "char*": "*mut c_char",
    "void*": "*mut c_void",
    "const void*": "*const c_void",
    "void**": "*mut *mut c_void",
    "const double*": "*const f64",
    "double*": "*mut f64",
    "const int64_t*": "*const i64",
    "int64_t*": "*mut i64",
    "const uint32_t*": "*const u32",
    "uint32_t*": "*mut u32",
    "uint32_t": "u32",
    "int*": "*mut c_int",
    "fcu_ctx": "fcu_ctx",
    "fcu_mesh": "fcu_mesh",
    "fcu_space": "fcu_space",
    "fcu_matrix": "fcu_matrix",
    "fcu_transient": "fcu_transient",
    "fcu_ctx*": "*mut fcu_ctx",
    "fcu_mesh*": "*mut fcu_mesh",
    "fcu_space*": "*mut fcu_space",
    "fcu_matrix*": "*mut fcu_matrix",
    "fcu_transient*": "*mut fcu_transient",
    "fcu_solve_info*": "*mut fcu_solve_info",
    "fcu_inner_solve": "fcu_inner_solve",
}


def _strip_c_comments(txt):
    return re.sub(r"/\*.*?\*/", "", txt, flags=re.S)


def _c_type(decl):
    """'const double* vals' -> 'const double*'"""
    decl = " ".join(decl.split())
    m = re.match(r"^(.*?)([A-Za-z_][A-Za-z0-9_]*)$", decl)
    t = m.group(1).strip() if m else decl
    return t.replace(" *", "*")


def header_functions():
    txt = _strip_c_comments(open(HEADER).read())
    txt = re.sub(r"typedef[^;]*;", "", txt)
    out = {}
    for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_ \*]*?)\b(fcu_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", txt, flags=re.S):
        ret = _c_type(m.group(1) + " x")
        args = [a.strip() for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(2)] = (ret, [_c_type(a) for a in args])
    return out


def header_defines():
    txt = open(HEADER).read()
    return {k: int(v) for k, v in re.findall(r"#define\s+(FCU_[A-Z0-9_]+)\s+(-?\d+)", txt)}


def _split_top(s):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "(<[":
            depth += 1
        elif ch in ")>]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return [p.strip() for p in parts if p.strip()]


def ffi_functions():
    txt = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    txt = re.sub(r"//[^\n]*", "", txt)
    block = txt[txt.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (fcu_[a-z0-9_]+)\s*\((.*?)\)\s*(->\s*([^;]+))?;", block, flags=re.S):
        args = []
        for a in _split_top(m.group(2)):
            name, ty = a.split(":", 1)
            args.append(" ".join(ty.split()))
        ret = " ".join(m.group(4).split()) if m.group(4) else "()"
        out[m.group(1)] = (ret, args)
    return out


def test_ffi_binds_every_header_function_with_matching_types():
    h = header_functions()
    r = ffi_functions()
    assert len(h) >= 60
    assert sorted(h) == sorted(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    for name, (cret, cargs) in h.items():
        rret, rargs = r[name]
        assert len(cargs) == len(rargs), name
        assert C_TO_RUST[cret] == rret, (name, cret, rret)
        for i, (ca, ra) in enumerate(zip(cargs, rargs)):
            assert C_TO_RUST[ca] == ra, (name, i, ca, ra)


def test_ffi_constants_match_header():
    d = header_defines()
    txt = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    consts = {k: int(v) for k, v in re.findall(r"pub const (FCU_[A-Z0-9_]+): \w+ = (-?\d+);", txt)}
    want = {k: v for k, v in d.items() if k != "FENICS_CUDA_H"}
    assert consts == want


def test_ffi_solve_info_layout_matches_header():
    ctext = _strip_c_comments(open(HEADER).read())
    body = re.search(r"typedef struct \{(.*?)\} fcu_solve_info;", ctext, flags=re.S).group(1)
    cfields = [(_c_type(f)) for f in body.split(";") if f.strip()]
    cnames = [f.split()[-1] for f in body.split(";") if f.strip()]
    rtext = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    rbody = re.search(r"pub struct fcu_solve_info \{(.*?)\}", rtext, flags=re.S).group(1)
    rfields = re.findall(r"pub (\w+): ([\w:]+),", rbody)
    assert [n for n, _ in rfields] == cnames
    assert [C_TO_RUST[c] for c in cfields] == [t for _, t in rfields]


def test_safe_wrappers_call_only_bound_functions():
    lib = open(os.path.join(CRATE, "src", "lib.rs")).read()
    called = set(re.findall(r"ffi::(fcu_[a-z0-9_]+)\s*\(", lib))
    assert called, "lib.rs calls no ffi function"
    assert called <= set(ffi_functions())
    # the reference signatures the crate is a drop-in for
    for sig in ("pub fn assemble_stiffness_2d(mesh: &TriangleMesh) -> SparseColMat<usize, f64>",
                "pub fn assemble_stiffness_3d(mesh: &TetrahedronMesh) -> SparseColMat<usize, f64>",
                "pub fn assemble_elasticity_stiffness_3d(mesh: &TetrahedronMesh, mat: &ElasticMaterial)",
                "pub fn apply_dirichlet_bc(a: &SparseColMat<usize, f64>, b: &[f64], bc: &DirichletBC)",
                "pub fn solve_cg(", "pub fn solve_csr_cg_gpu(", "pub fn boundary_dofs_2d(mesh: &TriangleMesh)",
                "pub fn assemble_elasticity_body_force_3d(mesh: &TetrahedronMesh, f_body: [f64; 3])"):
        assert sig in lib, sig


def test_crate_manifest_and_build_script():
    toml = open(os.path.join(CRATE, "Cargo.toml")).read()
    assert 'name = "fenics-cuda"' in toml and 'links = "fenics_cuda"' in toml
    build = open(os.path.join(CRATE, "build.rs")).read()
    assert "rustc-link-lib=dylib=fenics_cuda" in build


def test_integration_reexports_exist_in_crate():
    """Every item the integration recipe re-exports from the crate
    (`pub use fenics_cuda::{...}`) is defined public in src/lib.rs."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    doc = open(os.path.join(root, "INTEGRATION.md")).read()
    lib = open(os.path.join(root, "crates", "fenics-cuda", "src", "lib.rs")).read()
    names = set()
    for block in re.findall(r"pub use fenics_cuda::\{([^}]*)\}", doc):
        names.update(n.strip() for n in block.split(",") if n.strip())
    assert len(names) >= 15
    defined = set(re.findall(r"^pub (?:fn|struct|enum) (\w+)", lib, flags=re.M))
    assert not sorted(names - defined), sorted(names - defined)
