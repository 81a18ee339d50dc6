"""The Rust binding crates (rust/lambent-b200-sys, rust/lambent-b200) against the C-ABI.  No Rust
toolchain is needed: the -sys crate's generated declarations must match include/lambent.h, and every
call the safe crate makes into it must name a declared entry point with the declared arity."""
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SYS = os.path.join(ROOT, "rust", "lambent-b200-sys")
SAFE = os.path.join(ROOT, "rust", "lambent-b200", "src", "lib.rs")


def header_entry_points():
    src = open(os.path.join(ROOT, "include", "lambent.h")).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(lam_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
        params = " ".join(params.split())
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def sys_entry_points():
    src = open(os.path.join(SYS, "src", "lib.rs")).read()
    out = {}
    for name, params in re.findall(r"pub fn (lam_[a-z0-9_]+)\(([^)]*)\)", src):
        out[name] = 0 if not params.strip() else params.count(",") + 1
    return out


def test_sys_bindings_are_generated_from_the_header():
    r = subprocess.run([sys.executable, os.path.join(SYS, "gen_bindings.py"), "--check"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr


def test_sys_declares_every_entry_point_with_its_arity():
    assert sys_entry_points() == header_entry_points()


def _calls(src):
    """(name, argument count) of every sys::lam_* call, counting top-level commas."""
    for m in re.finditer(r"sys::(lam_[a-z0-9_]+)\(", src):
        depth, i, args, cur = 1, m.end(), 0, ""
        while depth:
            c = src[i]
            if c in "([{":
                depth += 1
            elif c in ")]}":
                depth -= 1
            elif c == "," and depth == 1:
                args += 1
            if depth:
                cur += c
            i += 1
        yield m.group(1), (0 if not cur.strip() else args + (0 if cur.rstrip().endswith(",") else 1))


def test_safe_crate_calls_match_the_declarations():
    decl = sys_entry_points()
    src = open(SAFE).read()
    calls = list(_calls(src))
    assert len(calls) >= 25
    for name, n in calls:
        assert name in decl, name
        assert n == decl[name], (name, n, decl[name])
    # the reference's API names are all there
    for item in ("pub struct Material", "pub fn new(", "pub struct Camera", "pub fn from_proj_view",
                 "pub fn update_from_proj_view", "pub struct TextureLoader", "pub fn load_from_bytes", "pub fn raw",
                 "pub struct RayTracer", "pub fn set_intersection_handler", "pub fn create_pipeline",
                 "pub struct Low", "pub struct Medium", "pub struct High", "pub struct PathTracerOpts",
                 "pub enum RestirTemporalMode", "pub struct DataBuffers", "pub fn advance_frame", "pub fn dispatch_size"):
        assert item in src, item
