//! Links libpencil_b200.so (built in-tree by `pencil_b200/_build.py`, next to
//! this crate) and the CUDA runtime for device allocations.
//! PENCIL_B200_LIB_DIR overrides the library directory, CUDA_HOME the
//! toolkit (default /usr/local/cuda).

use std::env;
use std::path::PathBuf;

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("cargo sets CARGO_MANIFEST_DIR"));
    let lib_dir = env::var("PENCIL_B200_LIB_DIR")
        .map(PathBuf::from)
        .unwrap_or_else(|_| manifest.join("..").join("pencil_b200"));
    let cuda = env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
    println!("cargo:rustc-link-lib=dylib=pencil_b200");
    println!("cargo:rustc-link-search=native={}/lib64", cuda);
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rerun-if-env-changed=PENCIL_B200_LIB_DIR");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
}
