// Build script of hdc-sys: link libhdc, the sm_100a build of this repository's
// CUDA sources.
//
// Two ways, chosen by the environment:
//
// * HDC_LIB_DIR=<dir holding libhdc.so>: link that library (e.g. the one
//   `python -m mwa_hyperdrive_b200.build` leaves in mwa_hyperdrive_b200/).
// * otherwise: compile every mwa_hyperdrive_b200/csrc/*.cu with nvcc for
//   sm_100a into a static archive in OUT_DIR and link it with the CUDA
//   runtime.  Every .cu, .cuh and .h that the build reads is listed with
//   rerun-if-changed (the same scan mwa_hyperdrive's build.rs does over
//   src/gpu), so editing a kernel rebuilds the crate.
//
// NVCC (default: nvcc on PATH) and CUDA_LIB_DIR (default:
// /usr/local/cuda/lib64) locate the toolkit.

use std::env;
use std::path::{Path, PathBuf};
use std::process::Command;

fn scan(dir: &Path, sources: &mut Vec<PathBuf>) {
    let entries = match std::fs::read_dir(dir) {
        Ok(e) => e,
        Err(_) => return,
    };
    for entry in entries.flatten() {
        let path = entry.path();
        if path.is_dir() {
            scan(&path, sources);
            continue;
        }
        match path.extension().and_then(|e| e.to_str()) {
            Some("cu") => {
                println!("cargo:rerun-if-changed={}", path.display());
                sources.push(path);
            }
            Some("cuh") | Some("h") => println!("cargo:rerun-if-changed={}", path.display()),
            _ => {}
        }
    }
}

fn main() {
    println!("cargo:rerun-if-changed=build.rs");
    println!("cargo:rerun-if-env-changed=HDC_LIB_DIR");
    println!("cargo:rerun-if-env-changed=NVCC");
    println!("cargo:rerun-if-env-changed=CUDA_LIB_DIR");

    if let Ok(dir) = env::var("HDC_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
        println!("cargo:rustc-link-lib=dylib=hdc");
        return;
    }

    let root = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..");
    let csrc = root.join("mwa_hyperdrive_b200").join("csrc");
    let include = root.join("include");
    let mut sources = vec![];
    scan(&csrc, &mut sources);
    let mut headers = vec![];
    scan(&include, &mut headers);
    sources.sort();

    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = env::var("NVCC").unwrap_or_else(|_| "nvcc".to_string());
    let mut objects = vec![];
    for src in &sources {
        let obj = out.join(src.file_stem().unwrap()).with_extension("o");
        let status = Command::new(&nvcc)
            .args(["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo"])
            .args(["--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-rdc=false", "-c"])
            .arg(src)
            .arg("-o")
            .arg(&obj)
            .status()
            .expect("could not run nvcc (set NVCC, or HDC_LIB_DIR to link a prebuilt libhdc.so)");
        assert!(status.success(), "nvcc failed on {}", src.display());
        objects.push(obj);
    }
    let lib = out.join("libhdc.a");
    let status = Command::new("ar").arg("crs").arg(&lib).args(&objects).status().expect("could not run ar");
    assert!(status.success(), "ar failed");

    let cuda_lib = env::var("CUDA_LIB_DIR").unwrap_or_else(|_| "/usr/local/cuda/lib64".to_string());
    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=static=hdc");
    println!("cargo:rustc-link-search=native={cuda_lib}");
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rustc-link-lib=dylib=stdc++");
}
