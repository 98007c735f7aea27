//! Builds or locates libmorphogen_gpu.so and links it.
//!
//! The reference's build.rs runs nvcc to emit PTX that cudarc loads at run
//! time (crates/morphogen-gpu-dpf/build.rs:1-85).  Here the CUDA code is the
//! sm_100a library of this repository: with MORPHOGEN_B200_LIB_DIR set, the
//! prebuilt library in that directory is linked; otherwise build.rs compiles
//! morphogen_b200/csrc/*.cu with nvcc (the same flags as
//! morphogen_b200/build.py) into OUT_DIR and links that.
use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    println!("cargo:rerun-if-env-changed=MORPHOGEN_B200_LIB_DIR");
    println!("cargo:rerun-if-env-changed=NVCC");
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
    let repo = manifest.join("..").join("..");
    let csrc = repo.join("morphogen_b200").join("csrc");
    let include = repo.join("include");

    let lib_dir = match env::var("MORPHOGEN_B200_LIB_DIR") {
        Ok(dir) => PathBuf::from(dir),
        Err(_) => {
            let out = PathBuf::from(env::var("OUT_DIR").unwrap());
            let nvcc = env::var("NVCC").unwrap_or_else(|_| "/usr/local/cuda/bin/nvcc".to_string());
            let sources = ["mg_kernels.cu", "mg_api.cu", "mg_server.cu", "mg_noalloc.cu"];
            for s in sources.iter() {
                println!("cargo:rerun-if-changed={}", csrc.join(s).display());
            }
            let status = Command::new(&nvcc)
                .args(["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17"])
                .args(["-Xcompiler", "-fPIC,-O2", "-shared", "-cudart", "static"])
                .arg("-I")
                .arg(&include)
                .arg("-I")
                .arg(&csrc)
                .arg("-o")
                .arg(out.join("libmorphogen_gpu.so"))
                .args(sources.iter().map(|s| csrc.join(s)))
                .status()
                .expect("running nvcc (set NVCC, or MORPHOGEN_B200_LIB_DIR to a prebuilt library)");
            assert!(status.success(), "nvcc failed building libmorphogen_gpu.so");
            out
        }
    };
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-lib=dylib=morphogen_gpu");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
}
