"""CPU checks of the Julia binding against the C ABI (Julia is not installed
here, so the binding itself never runs in these tests).

Every `ccall((:cgd_..., libcgd), R, (T1, ..., Tn), ...)` in
cgdycore.jl_b200/julia/*.jl must name a function that include/cgd_b200.h
declares and the library exports, with as many argument types as the C
prototype has parameters, each of a compatible kind (pointer, 32- or 64-bit
integer, double), and a compatible return type.  A mismatch here would make
the drop-in pass garbage to the library without any error at the call.
"""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL_DIR = os.path.join(ROOT, "cgdycore.jl_b200", "julia")


def _split_top(s):
    """Split s at commas outside (), {} and []."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur).strip())
    return out


def _ccalls():
    """(file, symbol, return type, [argument types]) of every ccall."""
    calls = []
    for path in sorted(glob.glob(os.path.join(JL_DIR, "*.jl"))):
        src = open(path).read()
        for m in re.finditer(r"ccall\(\(:(cgd_[a-z0-9_]+)\s*,", src):
            # the balanced argument list of this ccall
            i = src.index("(", m.start())
            depth = 0
            for j in range(i, len(src)):
                if src[j] == "(":
                    depth += 1
                elif src[j] == ")":
                    depth -= 1
                    if depth == 0:
                        break
            parts = _split_top(src[i + 1:j])
            ret = parts[1]
            tup = parts[2]
            assert tup.startswith("(") and tup.endswith(")"), (path, m.group(1), tup)
            args = [a for a in _split_top(tup[1:-1]) if a]
            calls.append((os.path.basename(path), m.group(1), ret, args))
    return calls


def _prototypes():
    """name -> (return type, [parameter types]) from include/cgd_b200.h."""
    txt = open(os.path.join(ROOT, "include", "cgd_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"//[^\n]*", "", txt)
    txt = re.sub(r"^\s*#[^\n]*", "", txt, flags=re.M)   # preprocessor lines
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(cgd_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", txt):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        ps = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        types = []
        for p in ps:
            if "*" in p:
                types.append("ptr")
            else:
                words = p.replace("const", " ").split()
                types.append(" ".join(words[:-1]) if len(words) > 1 else words[0])
        protos[name] = ("ptr" if "*" in ret else ret.replace("const", "").strip(), types)
    return protos


# Julia type -> kind, C type -> kind
def _jl_kind(t):
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{")) or t in ("Cstring", "Ptr"):
        return "ptr"
    return {"Cint": "i32", "Int32": "i32", "Cuint": "u32", "UInt32": "u32", "Int64": "i64", "Clonglong": "i64",
            "Csize_t": "u64", "UInt64": "u64", "Cdouble": "f64", "Float64": "f64", "Cfloat": "f32",
            "Float32": "f32", "Cvoid": "void"}.get(t, "?" + t)


def _c_kind(t):
    return {"ptr": "ptr", "int": "i32", "int32_t": "i32", "unsigned": "u32", "uint32_t": "u32",
            "int64_t": "i64", "long long": "i64", "size_t": "u64", "uint64_t": "u64", "double": "f64",
            "float": "f32", "void": "void"}.get(t, "?" + t)


CALLS = _ccalls()


def test_binding_has_calls():
    assert len(CALLS) >= 20, len(CALLS)


def _mismatches(call, protos):
    """What is wrong with one ccall against the prototypes (empty if nothing)."""
    fname, name, ret, args = call
    if name not in protos:
        return [f"{fname}: {name} is not declared in include/cgd_b200.h"]
    cret, cparams = protos[name]
    if len(args) != len(cparams):
        return [f"{fname}: {name} passes {len(args)} arguments, the C prototype takes {len(cparams)}"]
    bad = [f"{fname}: {name} argument {k + 1}: Julia {ja} against C {ca}"
           for k, (ja, ca) in enumerate(zip(args, cparams)) if _jl_kind(ja) != _c_kind(ca)]
    if _jl_kind(ret) != _c_kind(cret):
        bad.append(f"{fname}: {name} returns C {cret}, Julia expects {ret}")
    return bad


@pytest.mark.parametrize("call", CALLS, ids=[f"{c[1]}@{c[0]}:{k}" for k, c in enumerate(CALLS)])
def test_ccall_matches_header(call):
    assert _mismatches(call, _prototypes()) == []


def test_checker_flags_mismatches():
    protos = _prototypes()
    ok = ("x.jl", "cgd_ros_step", "Cint", ["Ptr{Cvoid}", "Ptr{Float64}", "Cdouble", "Int32"])
    assert _mismatches(ok, protos) == []
    assert _mismatches(("x.jl", "cgd_ros_step", "Cint", ok[3][:3]), protos)          # an argument missing
    assert _mismatches(("x.jl", "cgd_ros_step", "Cint", ["Ptr{Cvoid}", "Ptr{Float64}", "Int32", "Int32"]),
                       protos)                                                       # double passed as Int32
    assert _mismatches(("x.jl", "cgd_ros_step", "Cdouble", ok[3]), protos)          # wrong return type
    assert _mismatches(("x.jl", "cgd_no_such_call", "Cint", []), protos)             # undeclared


def test_ccall_symbols_are_exported(built_lib):
    from cgd_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    for fname, name, _, _ in CALLS:
        assert hasattr(L, name), f"{fname}: {name} is not exported by {os.path.basename(_lib.LIB_PATH)}"
