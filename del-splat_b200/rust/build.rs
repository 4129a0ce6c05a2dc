// Links libdsplat.so (del-splat_b200/lib, built by del-splat_b200/build.py);
// DSPLAT_LIB_DIR overrides the directory.
fn main() {
    let dir = std::env::var("DSPLAT_LIB_DIR").unwrap_or_else(|_| {
        let manifest = std::env::var("CARGO_MANIFEST_DIR").unwrap();
        format!("{}/../lib", manifest)
    });
    println!("cargo:rustc-link-search=native={}", dir);
    println!("cargo:rustc-link-lib=dylib=dsplat");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir);
    println!("cargo:rerun-if-env-changed=DSPLAT_LIB_DIR");
}
