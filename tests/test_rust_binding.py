"""The Rust drop-in crate (rust/morphogen-gpu-dpf-b200) binds the C ABI that
include/morphogen_gpu.h declares: the same entry points with the same
argument counts and C types, the same struct layouts and the same constants.
cargo is not available here, so the check is made on the sources: both
declarations are parsed and every function, parameter and field compared."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "morphogen_gpu.h"
CRATE = ROOT / "rust" / "morphogen-gpu-dpf-b200"
FFI = CRATE / "src" / "ffi.rs"

RUST_BASE = {"c_int": "int", "c_char": "char", "c_void": "void", "u8": "uint8_t", "u32": "uint32_t",
             "u64": "uint64_t", "usize": "size_t", "f64": "double"}


def strip_c_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def c_type(decl: str) -> tuple[str, str]:
    """'const mg_table* const* tables' -> ('const mg_table**', 'tables').
    Qualifiers of the pointers themselves are dropped (they do not change the
    ABI and Rust cannot spell them); an array parameter decays to a pointer."""
    decl = decl.strip()
    arr = 0
    m = re.match(r"^(.*?)(\w+)\s*((?:\[\w*\])*)$", decl)
    body, name, dims = m.group(1), m.group(2), m.group(3)
    arr = dims.count("[")
    toks = re.findall(r"[A-Za-z_]\w*|\*", body)
    base_const = False
    base = []
    stars = 0
    for t in toks:
        if t == "*":
            stars += 1
        elif t == "const":
            if stars == 0:
                base_const = True
        else:
            base.append(t)
    return ("const " if base_const else "") + " ".join(base) + "*" * (stars + arr), name


def rust_type(t: str) -> str:
    t = t.strip()
    if t.startswith("*const "):
        inner = t[len("*const "):].strip()
        ci = rust_type(inner)
        return ci + "*" if inner.startswith("*") else "const " + ci + "*"
    if t.startswith("*mut "):
        return rust_type(t[len("*mut "):]) + "*"
    return RUST_BASE.get(t, t)


def header_functions() -> dict:
    src = strip_c_comments(HEADER.read_text())
    src = "\n".join(ln for ln in src.splitlines() if not ln.lstrip().startswith("#"))
    out = {}
    for m in re.finditer(r"^[ \t]*([A-Za-z_][\w \t\*]*?)\b(mg_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.M):
        ret = c_type(m.group(1).strip() + " _ret")[0]
        params = m.group(3).strip()
        args = [] if params in ("", "void") else [c_type(p)[0] for p in params.split(",")]
        out[m.group(2)] = (ret, args)
    return out


def rust_functions() -> dict:
    src = FFI.read_text()
    block = src[src.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (mg_\w+)\s*\(([^)]*)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        params = [p.strip() for p in m.group(2).split(",") if p.strip()]
        args = [rust_type(p.split(":", 1)[1]) for p in params]
        ret = rust_type(m.group(3)) if m.group(3) else "void"
        out[m.group(1)] = (ret, args)
    return out


def header_structs() -> dict:
    src = strip_c_comments(HEADER.read_text())
    out = {}
    for m in re.finditer(r"typedef struct \{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
        fields = []
        for stmt in m.group(1).split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            typ, names = re.match(r"^([\w\s\*]+?)\s+(\w+(?:\s*,\s*\w+)*)$", stmt).groups()
            for n in names.split(","):
                fields.append((n.strip(), c_type(typ + " " + n.strip())[0]))
        out[m.group(2)] = fields
    return out


def rust_structs() -> dict:
    src = FFI.read_text()
    out = {}
    for m in re.finditer(r"#\[repr\(C\)\]\s*(?:#\[derive\([^)]*\)\]\s*)?pub struct (\w+) \{(.*?)\}", src, flags=re.S):
        fields = re.findall(r"pub (\w+):\s*([^,]+),", m.group(2))
        if fields:
            out[m.group(1)] = [(n, rust_type(t)) for n, t in fields]
    return out


def test_crate_files_exist():
    for f in ("Cargo.toml", "build.rs", "src/lib.rs", "src/ffi.rs", "src/kernel.rs", "src/storage.rs", "src/dpf.rs"):
        assert (CRATE / f).exists(), f
    toml = (CRATE / "Cargo.toml").read_text()
    assert 'name = "morphogen-gpu-dpf"' in toml and 'name = "morphogen_gpu_dpf"' in toml


def test_every_header_function_is_bound_with_the_same_c_types():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 50
    assert sorted(h) == sorted(r), (sorted(set(h) ^ set(r)))
    for name, (ret, args) in h.items():
        rret, rargs = r[name]
        assert rret == ret, (name, ret, rret)
        assert len(rargs) == len(args), (name, args, rargs)
        assert rargs == args, (name, args, rargs)


def test_every_header_struct_has_the_same_fields():
    h, r = header_structs(), rust_structs()
    assert set(h) == {"mg_timing", "mg_plan_info", "mg_server_config", "mg_server_stats"}
    for name, fields in h.items():
        assert r[name] == fields, (name, fields, r.get(name))


def test_status_codes_and_limits_match():
    src = strip_c_comments(HEADER.read_text())
    enum = dict(re.findall(r"(MG_E?\w+)\s*=\s*(\d+)", src))
    defines = {n: str(int(v) << int(s)) if s else v
               for n, v, s in re.findall(r"#define (MG_\w+) \(?(\d+)u?(?: << (\d+))?\)?", src)}
    assert {"MG_MAX_DOMAIN_BITS", "MG_NOALLOC_SCRATCH_BYTES", "MG_NOALLOC_MAX_KEYS"} <= set(defines)
    rs = FFI.read_text()
    rconst = {n: v for n, v in re.findall(r"pub const (MG_\w+): \w+ = ([\d <]+);", rs)}

    def ev(v):
        v = v.strip()
        if "<<" in v:
            a, b = v.split("<<")
            return int(a) << int(b)
        return int(v)
    for n, v in {**enum, **defines}.items():
        assert n in rconst, n
        assert ev(rconst[n]) == int(v), (n, v, rconst[n])


def test_python_binding_lists_the_same_entry_points():
    # The ctypes binding and the Rust binding cover the same header.
    from morphogen_b200 import _native as N
    assert sorted(N.EXPORTED) == sorted(header_functions())


@pytest.mark.parametrize("decl,want", [
    ("const mg_table* const* tables", "const mg_table**"),
    ("const uint8_t root_seed0[16]", "const uint8_t*"),
    ("const void** dptr", "const void**"),
    ("void* stream", "void*"),
])
def test_c_type_normaliser(decl, want):
    assert c_type(decl)[0] == want
