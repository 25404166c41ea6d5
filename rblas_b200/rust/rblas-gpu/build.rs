//! Links librblas_b200.so (built with `python -m rblas_b200._build`).
//! RBLAS_B200_LIB_DIR names the directory that holds it; by default the
//! package directory two levels up from this crate.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("RBLAS_B200_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..").join(".."),
    };
    println!("cargo:rerun-if-env-changed=RBLAS_B200_LIB_DIR");
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=rblas_b200");
    // find the library at run time without LD_LIBRARY_PATH
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir.display());
}
