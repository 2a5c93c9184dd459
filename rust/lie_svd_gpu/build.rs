// Links liblsvd_b200.so; LSVD_LIB_DIR points at lie_cliffalg_analog_svd_b200/_lib.
fn main() {
    if let Ok(dir) = std::env::var("LSVD_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
    }
    println!("cargo:rustc-link-lib=dylib=lsvd_b200");
    println!("cargo:rerun-if-env-changed=LSVD_LIB_DIR");
}
