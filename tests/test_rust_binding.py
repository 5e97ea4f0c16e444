"""The Rust crate (phys-rs_b200/rust/phys-gpu) agrees with include/physgpu.h.

No Rust toolchain exists here, so the crate is checked as text: its
`extern "C"` block declares every entry point of the header with the same
argument count, and each argument and result has the header's width and
pointer-ness (int/int32_t -> i32, int64_t -> i64, uint64_t -> u64, double ->
f64, size_t -> usize, const T* -> *const, T* -> *mut); its #[repr(C)]
structs have the header's fields in the header's order and types; its
constants have the header's values; the safe API exposes the reverse-mode
gradient over phys_adjoint_direct; and the drop-in ECS system keeps the
reference's signature (barnes_hut_gravity_system, gravity_tree.rs:260-263)."""
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CRATE = os.path.join(REPO, "phys-rs_b200", "rust", "phys-gpu")

C_SCALAR = {"int": "i32", "int32_t": "i32", "int64_t": "i64", "uint64_t": "u64",
            "double": "f64", "size_t": "usize", "char": "c_char", "void": "void",
            "phys_ctx": "phys_ctx", "phys_params": "phys_params",
            "phys_timings": "phys_timings", "phys_nfw_halo": "phys_nfw_halo"}
RS_SCALAR = {"c_int": "i32", "i32": "i32", "i64": "i64", "u64": "u64", "f64": "f64",
             "usize": "usize", "c_char": "c_char", "c_void": "void",
             "phys_ctx": "phys_ctx", "phys_params": "phys_params",
             "phys_timings": "phys_timings", "phys_nfw_halo": "phys_nfw_halo"}


def _strip_c(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def c_type(t):
    """'const double*' -> ('ptr-const', 'f64'); 'int64_t' -> ('val', 'i64')."""
    t = t.strip()
    ptrs = t.count("*")
    base = t.replace("*", " ").split()
    const = "const" in base
    base = [b for b in base if b not in ("const", "struct")]
    assert len(base) == 1, t
    s = C_SCALAR[base[0]]
    if ptrs == 0:
        return ("val", s)
    if ptrs == 2:
        return ("ptr-mut", ("ptr-mut", s))
    return ("ptr-const" if const else "ptr-mut", s)


def rs_type(t):
    t = t.strip()
    if t.startswith("*const "):
        return ("ptr-const", rs_type(t[len("*const "):])[1])
    if t.startswith("*mut "):
        inner = rs_type(t[len("*mut "):])
        return ("ptr-mut", inner if inner[0] != "val" else inner[1])
    return ("val", RS_SCALAR[t])


def header_functions():
    src = _strip_c(open(os.path.join(REPO, "include", "physgpu.h")).read())
    src = re.sub(r"#[^\n]*", "", src)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(phys_\w+)\s*\(([^)]*)\)\s*;", src):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        ret = ret.replace("extern", "").strip()
        params = []
        for a in [x.strip() for x in args.split(",") if x.strip()]:
            a = re.sub(r"\b\w+$", "", a) if not a.endswith("*") else a  # drop the name
            params.append(c_type(a))
        out[name] = (c_type(ret), params)
    return out


def rust_functions():
    src = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    src = re.sub(r"//[^\n]*", "", src)
    block = src[src.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (phys_\w+)\s*\(([^)]*)\)\s*(?:->\s*([^;]+))?;", block, re.S):
        name, args, ret = m.group(1), m.group(2), m.group(3)
        params = []
        for a in [x.strip() for x in args.split(",") if x.strip()]:
            params.append(rs_type(a.split(":", 1)[1]))
        out[name] = (rs_type(ret) if ret else ("val", "void"), params)
    return out


def test_every_header_function_is_declared_with_the_same_types():
    h, r = header_functions(), rust_functions()
    assert sorted(h) == sorted(r)
    for name in h:
        assert h[name][0] == r[name][0], (name, "result", h[name][0], r[name][0])
        assert len(h[name][1]) == len(r[name][1]), (name, "argument count")
        for k, (a, b) in enumerate(zip(h[name][1], r[name][1])):
            assert a == b, (name, k, a, b)


def _c_struct(name):
    src = _strip_c(open(os.path.join(REPO, "include", "physgpu.h")).read())
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, re.S).group(1)
    fields = []
    for decl in [d.strip() for d in body.split(";") if d.strip()]:
        m = re.match(r"(.+?)\s+(\w+)(\[(\d+)\])?$", decl)
        fields.append((m.group(2), C_SCALAR[m.group(1).strip()], m.group(4)))
    return fields


def _rs_struct(name):
    src = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    body = re.search(r"pub struct %s \{(.*?)\}" % name, src, re.S).group(1)
    fields = []
    for m in re.finditer(r"pub (\w+):\s*(\[(\w+);\s*(\d+)\]|\w+)", body):
        if m.group(3):
            fields.append((m.group(1), RS_SCALAR[m.group(3)], m.group(4)))
        else:
            fields.append((m.group(1), RS_SCALAR[m.group(2)], None))
    return fields


def test_repr_c_structs_match():
    for name in ("phys_params", "phys_timings", "phys_nfw_halo"):
        assert _c_struct(name) == _rs_struct(name), name


def test_constants_match():
    hdr = open(os.path.join(REPO, "include", "physgpu.h")).read()
    cdefs = dict(re.findall(r"#define (PHYS_\w+) (\d+)", hdr))
    rs = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    rdefs = dict(re.findall(r"pub const (PHYS_\w+): \w+ = (\d+);", rs))
    assert cdefs == rdefs


def test_reverse_mode_api_and_drop_in_signature():
    lib = open(os.path.join(CRATE, "src", "lib.rs")).read()
    assert re.search(r"pub fn trajectory_gradient\(.*?\) -> Result<Grad>", lib, re.S)
    assert "ffi::phys_adjoint_direct(" in lib
    drop = re.sub(r"\s+", " ", open(os.path.join(CRATE, "drop_in", "gpu_gravity.rs")).read())
    assert ("pub fn gpu_gravity_system( mut query: Query<(Entity, &mut Force, &Mass, &Sector, "
            "&LocalPosition)>, config: Res<UniverseConfig>, )") in drop
    build = open(os.path.join(CRATE, "build.rs")).read()
    assert "rustc-link-lib=dylib=physgpu" in build
