// Links libprimus_gpu.so (built by primus_b200/build.py: nvcc, sm_100a, CUDA
// runtime linked statically, so only the NVIDIA driver is needed at run time).
// PRIMUS_GPU_LIB_DIR names the directory holding it; the rpath lets test and
// bench binaries find it without LD_LIBRARY_PATH.
fn main() {
    let dir = std::env::var("PRIMUS_GPU_LIB_DIR")
        .expect("set PRIMUS_GPU_LIB_DIR to the directory that holds libprimus_gpu.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=primus_gpu");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
    println!("cargo:rerun-if-env-changed=PRIMUS_GPU_LIB_DIR");
    println!("cargo:rerun-if-changed={dir}/libprimus_gpu.so");
}
