// Links libsph_cuda.so (built by `python -m ultraballpit_b200.build`, nvcc,
// -gencode arch=compute_100a,code=sm_100a). The library links the CUDA
// runtime statically and needs only the NVIDIA driver at run time.
fn main() {
    let dir = std::env::var("SPH_CUDA_LIB_DIR")
        .expect("set SPH_CUDA_LIB_DIR to the directory holding libsph_cuda.so (ultraballpit_b200/lib)");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=sph_cuda");
    println!("cargo:rerun-if-env-changed=SPH_CUDA_LIB_DIR");
}
