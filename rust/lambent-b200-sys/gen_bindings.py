#!/usr/bin/env python
"""Generates src/lib.rs of the lambent-b200-sys crate from include/lambent.h: the enums and #defines
as constants, the plain-data structs as #[repr(C)] structs, the opaque handles as zero-sized enums,
the callback typedefs as Option<extern "C" fn> types and every entry point in one extern "C" block.

  python rust/lambent-b200-sys/gen_bindings.py            rewrites src/lib.rs
  python rust/lambent-b200-sys/gen_bindings.py --check    exits 1 when src/lib.rs is out of date

The header is plain C in a regular style (one declaration per statement, no macros in signatures),
which this parser relies on; it fails loudly on anything it does not understand."""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HEADER = os.path.join(ROOT, "include", "lambent.h")
OUT = os.path.join(HERE, "src", "lib.rs")

SCALARS = {
    "uint8_t": "u8", "uint16_t": "u16", "uint32_t": "u32", "uint64_t": "u64", "int32_t": "i32", "int": "c_int",
    "size_t": "usize", "float": "f32", "double": "f64", "char": "c_char", "void": "c_void",
    "unsigned int": "c_uint",
}


def strip_comments(src):
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    return re.sub(r"//[^\n]*", " ", src)


def rust_type(ctype, known):
    """A C type (without the declarator name) as a Rust type: [const] base [const] (* [const])*.
    Each pointer is *const when what it points to is const."""
    tokens = re.findall(r"const|\*|unsigned int|[A-Za-z_][A-Za-z0-9_]*", " ".join(ctype.split()))
    base, base_const, ptr_const = None, False, []  # ptr_const[k]: pointer k itself is const
    for tok in tokens:
        if tok == "const":
            if ptr_const:
                ptr_const[-1] = True
            else:
                base_const = True
        elif tok == "*":
            ptr_const.append(False)
        elif base is None:
            base = tok
        else:
            raise SystemExit(f"cannot parse type {ctype!r}")
    if base is None:
        raise SystemExit(f"cannot parse type {ctype!r}")
    if base in SCALARS:
        r = SCALARS[base]
    elif base in known:
        r = base
    else:
        raise SystemExit(f"unknown type {base!r} in {ctype!r}")
    pointee_const = base_const
    for k in range(len(ptr_const)):
        r = ("*const " if pointee_const else "*mut ") + r
        pointee_const = ptr_const[k]
    return r


def split_decl(decl):
    """'const float* tex_pos[2]' -> ('const float*', 'tex_pos', '2')."""
    decl = " ".join(decl.split())
    m = re.match(r"^(.*?)([A-Za-z_][A-Za-z0-9_]*)\s*(\[\s*([A-Za-z0-9_]+)\s*\])?$", decl)
    if not m:
        raise SystemExit(f"cannot parse declaration {decl!r}")
    return m.group(1).strip(), m.group(2), m.group(4)


def main():
    src = strip_comments(open(HEADER).read())
    out = []
    consts = []
    for body in re.findall(r"\benum\s*\{(.*?)\}\s*;", src, flags=re.S):
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            name, value = [x.strip() for x in item.split("=")]
            value = value.replace("u", "") if re.match(r"^[0-9xXa-fA-F]+u$", value) else value
            value = re.sub(r"(\d)u\b", r"\1", value)
            consts.append((name, "c_int", value))
    for name, value in re.findall(r"#define\s+(LAM_[A-Z0-9_]+)\s+([0-9xXa-fA-FuU]+)\b", src):
        consts.append((name, "u32", value.rstrip("uU")))
    opaque = re.findall(r"typedef\s+struct\s+(lam_[a-z0-9_]+)\s+\1\s*;", src)
    structs = {}
    order = []
    for name, body in re.findall(r"typedef\s+struct\s+(lam_[a-z0-9_]+)\s*\{(.*?)\}\s*\1\s*;", src, flags=re.S):
        fields = []
        for stmt in body.split(";"):
            stmt = " ".join(stmt.split())
            if not stmt:
                continue
            # "float pos[3], normal[3], wo[3]" -> three fields of the first declarator's base type
            parts = [p.strip() for p in stmt.split(",")]
            base, fname, dim = split_decl(parts[0])
            fields.append((fname, base, dim))
            for p in parts[1:]:
                _, fname2, dim2 = split_decl(base + " " + p)
                fields.append((fname2, base, dim2))
        structs[name] = fields
        order.append(name)
    callbacks = re.findall(r"typedef\s+(\w+)\s*\(\s*\*\s*(lam_[a-z0-9_]+)\s*\)\s*\((.*?)\)\s*;", src, flags=re.S)
    funcs = re.findall(r"^\s*((?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**)\s*(lam_[a-z0-9_]+)\s*\(([^)]*)\)\s*;",
                       src, flags=re.M)

    def params(plist):
        plist = " ".join(plist.split())
        if plist in ("", "void"):
            return []
        res = []
        for p in plist.split(","):
            base, pname, dim = split_decl(p.strip())
            if dim is not None:
                base = base + "*"  # an array parameter is a pointer
            if pname == "type":
                pname = "type_"
            res.append((pname, rust_type(base, known)))
        return res

    known = set(structs) | set(opaque) | {c[1] for c in callbacks}
    out.append("// @generated by gen_bindings.py from include/lambent.h - do not edit by hand.")
    out.append("#![allow(non_camel_case_types, non_upper_case_globals, clippy::all)]")
    out.append("#![no_std]")
    out.append("")
    out.append("pub use core::ffi::{c_char, c_int, c_uint, c_void};")
    out.append("")
    for name, ty, value in consts:
        out.append(f"pub const {name}: {ty} = {value};")
    out.append("")
    for name in opaque:
        out.append(f"#[repr(C)]\npub struct {name} {{\n    _private: [u8; 0],\n}}")
    out.append("")
    for ret, name, plist in callbacks:
        ps = ", ".join(f"{n}: {t}" for n, t in params(plist))
        r = rust_type(ret, known)
        out.append(f"pub type {name} = Option<unsafe extern \"C\" fn({ps}) -> {r}>;")
    out.append("")
    for name in order:
        out.append("#[repr(C)]\n#[derive(Clone, Copy, Debug)]")
        out.append(f"pub struct {name} {{")
        for fname, base, dim in structs[name]:
            t = rust_type(base, known)
            if dim is not None:
                t = f"[{t}; {dim}]"
            out.append(f"    pub {fname}: {t},")
        out.append("}")
        out.append("")
    out.append('extern "C" {')
    for ret, name, plist in funcs:
        r = rust_type(ret, known)
        ps = ", ".join(f"{n}: {t}" for n, t in params(plist))
        tail = "" if r == "c_void" else f" -> {r}"
        out.append(f"    pub fn {name}({ps}){tail};")
    out.append("}")
    text = "\n".join(out) + "\n"
    if "--check" in sys.argv:
        cur = open(OUT).read() if os.path.exists(OUT) else ""
        if cur != text:
            print("src/lib.rs is out of date: run gen_bindings.py", file=sys.stderr)
            sys.exit(1)
        return
    with open(OUT, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
