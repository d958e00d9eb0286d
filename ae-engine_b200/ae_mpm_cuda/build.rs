// build.rs -- compiles the CUDA sources with nvcc for sm_100a into a static library, the way
// ae_cpp_kernel/build.rs compiles cpp/simd_kernels.cpp with the cc crate.
use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    let csrc = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../csrc");
    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = env::var("NVCC").unwrap_or_else(|_| "nvcc".to_string());
    let sources = [
        "radix_sort.cu",
        "mpm_world.cu",
        "ae_mpm_api.cu",
        "ae_mpm_server.cu",
        "ae_mpm_noalloc.cu",
        "ae_mpm_lod.cu",
        "ae_mpm_ck.cu",
    ];
    let mut objects = Vec::new();
    for src in sources.iter() {
        let obj = out.join(src.replace(".cu", ".o"));
        // the CK-MPM kernels round every operation separately, as Rust's f32 arithmetic does
        let extra: &[&str] = match *src {
            "ae_mpm_ck.cu" => &["--fmad=false"],
            "ae_mpm_api.cu" => &["-Xcompiler", "-fopenmp"],
            _ => &[],
        };
        let status = Command::new(&nvcc)
            .args(["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo", "-Xptxas", "-v"])
            .args(extra)
            .args(["-Xcompiler", "-fPIC", "-c"])
            .arg(csrc.join(src))
            .arg("-o")
            .arg(&obj)
            .status()
            .expect("nvcc not found: set NVCC or put CUDA 12.9 on PATH");
        assert!(status.success(), "nvcc failed on {}", src);
        println!("cargo:rerun-if-changed={}", csrc.join(src).display());
        objects.push(obj);
    }
    let lib = out.join("libae_mpm.a");
    let status = Command::new("ar").arg("crs").arg(&lib).args(&objects).status().expect("ar");
    assert!(status.success());
    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=static=ae_mpm");
    let cuda = env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rustc-link-search=native={}/lib64", cuda);
    println!("cargo:rustc-link-lib=static=cudart_static");
    println!("cargo:rustc-link-lib=dylib=stdc++");
    println!("cargo:rustc-link-lib=dylib=dl");
    println!("cargo:rustc-link-lib=dylib=rt");
    println!("cargo:rustc-link-lib=dylib=gomp");
    println!("cargo:rustc-link-lib=dylib=pthread");
    println!("cargo:rerun-if-changed=../../include/ae_mpm.h");
}
