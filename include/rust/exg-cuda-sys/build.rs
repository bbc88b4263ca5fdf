// Links libexg.so: EXG_LIB_DIR names the directory that holds it (the in-tree build puts it in
// exgame_b200/, three levels above this crate), and the library is found there at run time too.
fn main() {
    let dir = std::env::var("EXG_LIB_DIR").unwrap_or_else(|_| {
        let here = std::env::var("CARGO_MANIFEST_DIR").expect("cargo sets CARGO_MANIFEST_DIR");
        format!("{}/../../../exgame_b200", here)
    });
    println!("cargo:rerun-if-env-changed=EXG_LIB_DIR");
    println!("cargo:rustc-link-search=native={}", dir);
    println!("cargo:rustc-link-lib=dylib=exg");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir);
}
