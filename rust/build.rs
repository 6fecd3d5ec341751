// Links the crate against libspecspars.so and the CUDA runtime.  This replaces the reference's cxx_build
// block and MKL link lines (build.rs:18-35 of the reference crate): nothing is compiled here, the library is
// built by `python -m spec_spars_b200.build` (nvcc, sm_100a).
// SPEC_SPARS_B200_LIB names the directory of libspecspars.so; by default the package directory next to
// this crate.  CUDA_LIB_DIR names the directory of libcudart.so (default /usr/local/cuda/lib64).
use std::env;
use std::path::PathBuf;

fn main() {
    let lib_dir = match env::var("SPEC_SPARS_B200_LIB") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..").join("spec_spars_b200"),
    };
    let cuda_dir = env::var("CUDA_LIB_DIR").unwrap_or_else(|_| "/usr/local/cuda/lib64".to_string());
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-search=native={}", cuda_dir);
    println!("cargo:rustc-link-lib=dylib=specspars");
    println!("cargo:rustc-link-lib=dylib=cudart");
    // let binaries find the library at run time without LD_LIBRARY_PATH
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
    println!("cargo:rerun-if-env-changed=SPEC_SPARS_B200_LIB");
    println!("cargo:rerun-if-env-changed=CUDA_LIB_DIR");
}
