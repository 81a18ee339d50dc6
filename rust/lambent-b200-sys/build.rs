//! Links liblambent_b200.so.  The library is built from lambent_b200/csrc (make) and found through
//! LAMBENT_B200_LIB_DIR, or the repository layout when the crate sits at rust/lambent-b200-sys.
use std::env;
use std::path::PathBuf;

fn main() {
    println!("cargo:rerun-if-env-changed=LAMBENT_B200_LIB_DIR");
    let dir = match env::var("LAMBENT_B200_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => {
            let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
            manifest.join("..").join("..").join("lambent_b200")
        }
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=lambent_b200");
    // the CUDA runtime the library itself links against
    if let Ok(cuda) = env::var("CUDA_HOME") {
        println!("cargo:rustc-link-search=native={}/lib64", cuda);
    }
}
