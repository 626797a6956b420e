//! Builds libxk.so, the sm_100a Kirchhoff engine, with nvcc and links it.
//!
//! XK_CSRC_DIR names the directory of the engine's `.cu` sources
//! (`xrt-rs_b200/csrc` of the engine's repository) and XK_INCLUDE_DIR the
//! directory of `xk.h`; NVCC overrides the compiler (default: `nvcc` on PATH,
//! else /usr/local/cuda/bin/nvcc). Set XK_LIB_DIR instead to link a prebuilt
//! libxk.so without compiling. The CUDA runtime is linked statically into
//! libxk.so, so the binary needs only the driver at run time.

use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    println!("cargo:rerun-if-env-changed=XK_LIB_DIR");
    println!("cargo:rerun-if-env-changed=XK_CSRC_DIR");
    println!("cargo:rerun-if-env-changed=XK_INCLUDE_DIR");
    println!("cargo:rerun-if-env-changed=NVCC");

    let lib_dir = match env::var_os("XK_LIB_DIR") {
        Some(dir) => PathBuf::from(dir),
        None => build_with_nvcc(),
    };
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-lib=dylib=xk");
    // Let test and bench binaries find the library without LD_LIBRARY_PATH.
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
}

fn build_with_nvcc() -> PathBuf {
    let csrc = PathBuf::from(env::var("XK_CSRC_DIR").expect(
        "set XK_CSRC_DIR to the engine's csrc directory (or XK_LIB_DIR to a prebuilt libxk.so)",
    ));
    let include = PathBuf::from(
        env::var("XK_INCLUDE_DIR").unwrap_or_else(|_| csrc.join("../../include").display().to_string()),
    );
    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = env::var("NVCC").unwrap_or_else(|_| {
        if Command::new("nvcc").arg("--version").output().is_ok() {
            "nvcc".into()
        } else {
            "/usr/local/cuda/bin/nvcc".into()
        }
    });
    let mut sources: Vec<PathBuf> = std::fs::read_dir(&csrc)
        .expect("read XK_CSRC_DIR")
        .filter_map(|e| e.ok().map(|e| e.path()))
        .filter(|p| p.extension().is_some_and(|x| x == "cu"))
        .collect();
    sources.sort();
    assert!(!sources.is_empty(), "no .cu sources in {}", csrc.display());
    for entry in std::fs::read_dir(&csrc).unwrap().flatten() {
        println!("cargo:rerun-if-changed={}", entry.path().display());
    }

    let flags = [
        "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
        "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
    ];
    let mut objects = Vec::new();
    for src in &sources {
        let obj = out.join(src.file_stem().unwrap()).with_extension("o");
        run(Command::new(&nvcc).args(flags).arg("-I").arg(&include).arg("-c").arg(src)
            .arg("-o").arg(&obj));
        objects.push(obj);
    }
    let lib = out.join("libxk.so");
    run(Command::new(&nvcc)
        .args(["-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static"])
        .arg("-o").arg(&lib).args(&objects));
    out
}

fn run(cmd: &mut Command) {
    let status = cmd.status().unwrap_or_else(|e| panic!("failed to start {cmd:?}: {e}"));
    assert!(status.success(), "{cmd:?} failed with {status}");
}

