//! Compiles libhl (every `.cu` file under `hit-leiden_b200/csrc/`) with nvcc
//! for sm_100a into `$OUT_DIR/libhl.so` and links the crate against it.
//!
//! The flags are those of `hit-leiden_b200/build.py`: `-fmad=false` keeps
//! every FP64 expression rounding step by step (the bit-exact gains and sums
//! depend on it), the CUDA runtime is linked statically, and only the `HL_API`
//! symbols are exported.  `NVCC` (or `CUDA_HOME/bin/nvcc`, or `nvcc` on
//! `PATH`) selects the compiler.
use std::env;
use std::fs;
use std::path::{Path, PathBuf};
use std::process::Command;

fn nvcc() -> PathBuf {
    if let Ok(p) = env::var("NVCC") {
        return PathBuf::from(p);
    }
    if let Ok(home) = env::var("CUDA_HOME") {
        let p = Path::new(&home).join("bin").join("nvcc");
        if p.exists() {
            return p;
        }
    }
    let p = Path::new("/usr/local/cuda/bin/nvcc");
    if p.exists() {
        return p.to_path_buf();
    }
    PathBuf::from("nvcc")
}

fn run(cmd: &mut Command) {
    let status = cmd.status().unwrap_or_else(|e| panic!("failed to start {:?}: {}", cmd, e));
    if !status.success() {
        panic!("{:?} exited with {}", cmd, status);
    }
}

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
    let root = manifest.join("..").join("..");
    let csrc = root.join("hit-leiden_b200").join("csrc");
    let include = root.join("include");
    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = nvcc();

    let mut sources: Vec<PathBuf> = fs::read_dir(&csrc)
        .expect("hit-leiden_b200/csrc not found")
        .filter_map(|e| e.ok().map(|e| e.path()))
        .filter(|p| p.extension().map(|x| x == "cu").unwrap_or(false))
        .collect();
    sources.sort();

    let mut objects = Vec::new();
    for src in &sources {
        println!("cargo:rerun-if-changed={}", src.display());
        let obj = out.join(format!("{}.o", src.file_name().unwrap().to_string_lossy()));
        run(Command::new(&nvcc)
            .args(["-gencode", "arch=compute_100a,code=sm_100a"])
            .args(["-O3", "-lineinfo", "-std=c++17", "-fmad=false"])
            .args(["-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"])
            .arg("--expt-relaxed-constexpr")
            .arg("-I").arg(&include)
            .arg("-I").arg(&csrc)
            .arg("-c").arg(src)
            .arg("-o").arg(&obj));
        objects.push(obj);
    }
    for h in ["hl.h", "hl_debug.h"] {
        println!("cargo:rerun-if-changed={}", include.join(h).display());
    }
    for h in ["hl_engine.cuh", "hl_internal.cuh"] {
        println!("cargo:rerun-if-changed={}", csrc.join(h).display());
    }

    let lib = out.join("libhl.so");
    run(Command::new(&nvcc)
        .args(["-gencode", "arch=compute_100a,code=sm_100a"])
        .args(["-shared", "-cudart", "static"])
        .arg("-o").arg(&lib)
        .args(&objects));

    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=dylib=hl");
    // find libhl.so next to the build output at run time
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", out.display());
    println!("cargo:rerun-if-env-changed=NVCC");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
}
