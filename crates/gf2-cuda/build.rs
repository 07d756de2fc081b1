//! Links libgf2cuda.so (built by `python gf2_b200/build.py`, nvcc for sm_100a).
//! GF2CUDA_LIB_DIR names the folder that holds the library.
fn main() {
    println!("cargo:rerun-if-env-changed=GF2CUDA_LIB_DIR");
    if std::env::var_os("CARGO_FEATURE_CUDA").is_none() {
        return;
    }
    let dir = std::env::var("GF2CUDA_LIB_DIR")
        .expect("set GF2CUDA_LIB_DIR to the folder of libgf2cuda.so (gf2_b200/ in the gf2cuda tree)");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=gf2cuda");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
}
