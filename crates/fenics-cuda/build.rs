//! Links libfenics_cuda.so, built by `python fenics-rs_b200/build.py`
//! (nvcc, sm_100a). Set FENICS_CUDA_LIB_DIR to the directory that holds it
//! (fenics-rs_b200/fenics_cuda in the CUDA repository).
fn main() {
    let dir = std::env::var("FENICS_CUDA_LIB_DIR")
        .expect("set FENICS_CUDA_LIB_DIR to the directory holding libfenics_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=fenics_cuda");
    println!("cargo:rerun-if-env-changed=FENICS_CUDA_LIB_DIR");
}
