"""The Rust drop-in's FFI module (rust/src/gpu/xk_ffi.rs) against the C ABI
(include/xk.h): every entry point declared in the header is declared in
Rust, and every #[repr(C)] struct lists the C struct's fields in the same
order (a Rust caller's layout then matches the library's). No compiler is
involved: the image has no cargo, so this is a source-level check."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "xk.h")
RUST = os.path.join(ROOT, "rust", "src", "gpu", "xk_ffi.rs")


def _strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def c_functions():
    src = _strip_c_comments(open(HEADER).read())
    return set(re.findall(r"^\s*(?:int|void|const char\s*\*)\s*(xk_\w+)\s*\(", src, flags=re.M))


def c_structs():
    src = _strip_c_comments(open(HEADER).read())
    out = {}
    for name, body, alias in re.findall(r"typedef struct (xk_\w+)\s*\{(.*?)\}\s*(\w+);", src,
                                        flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for i, part in enumerate(decl.split(",")):
                part = re.sub(r"\[.*?\]", "", part).replace("*", " ").split()
                fields.append(part[-1])
        out[alias] = fields
    return out


def rust_functions():
    return set(re.findall(r"pub fn (xk_\w+)\s*\(", open(RUST).read()))


def rust_structs():
    src = re.sub(r"//[^\n]*", " ", open(RUST).read())
    out = {}
    for name, body in re.findall(r"pub struct (xk_\w+)\s*\{(.*?)\}", src, flags=re.S):
        out[name] = re.findall(r"pub (\w+)\s*:", body)
    return out


def test_every_entry_point_is_declared_in_rust():
    missing = c_functions() - rust_functions()
    assert not missing, f"xk_ffi.rs lacks {sorted(missing)}"
    assert len(c_functions()) >= 30


def test_struct_fields_match_in_order():
    cs, rs = c_structs(), rust_structs()
    # GpuRay / GpuPixel are the reference's own record types on the Rust side.
    for name, fields in cs.items():
        if name in ("xk_gpu_ray", "xk_gpu_pixel"):
            continue
        assert name in rs, f"xk_ffi.rs lacks struct {name}"
        assert rs[name] == fields, (name, rs[name], fields)
