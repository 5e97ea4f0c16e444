// Builds libphysgpu.so from the CUDA sources of this repository (nvcc for
// sm_100a, through phys-rs_b200/physgpu/build.py) and links it, or links a
// prebuilt library from PHYSGPU_LIB_DIR.
use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("CARGO_MANIFEST_DIR"));
    // phys-rs_b200/rust/phys-gpu -> phys-rs_b200
    let pkg = manifest.join("..").join("..");
    let lib_dir = match env::var("PHYSGPU_LIB_DIR") {
        Ok(dir) => PathBuf::from(dir),
        Err(_) => {
            let status = Command::new(env::var("PYTHON").unwrap_or_else(|_| "python3".into()))
                .arg(pkg.join("physgpu").join("build.py"))
                .status()
                .expect("python3 and nvcc are needed to build libphysgpu.so");
            assert!(status.success(), "building libphysgpu.so failed");
            pkg.join("lib")
        }
    };
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-lib=dylib=physgpu");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
    println!("cargo:rerun-if-env-changed=PHYSGPU_LIB_DIR");
    println!("cargo:rerun-if-changed={}", pkg.join("csrc").display());
    println!("cargo:rerun-if-changed={}", pkg.join("..").join("include").join("physgpu.h").display());
}
