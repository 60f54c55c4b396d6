"""The Julia bindings written in INTEGRATION.md agree with the C ABI: every
`ccall((:oxi_..., liboxi), Ret, (Args...), ...)` names an entry point that
include/oxiblas_b200.h declares, with the same number of arguments and the
same kind of each argument and of the result (CPU only: the text is parsed)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C type -> kind; Julia type -> kind
C_KINDS = {"int64_t": "i64", "int": "i32", "int32_t": "i32", "char": "u8", "double": "f64",
           "float": "f32", "void": "void"}
JL_KINDS = {"Int64": "i64", "Cint": "i32", "Int32": "i32", "UInt8": "u8", "Cchar": "u8",
            "Float64": "f64", "Float32": "f32", "Cvoid": "void", "Cstring": "ptr"}


def c_kind(decl: str) -> str:
    decl = decl.replace("const", " ").strip()
    if "*" in decl or decl.startswith("oxi_handle_t"):
        return "ptr"
    base = decl.split()[0]
    if base.startswith("oxi_refine_report"):
        return "ptr"
    return C_KINDS[base]


def jl_kind(t: str) -> str:
    t = t.strip()
    if t.startswith(("Ptr{", "CuPtr{", "Ref{")) or t == "Cstring":
        return "ptr"
    return JL_KINDS[t]


def header_decls():
    txt = open(os.path.join(ROOT, "include", "oxiblas_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(int|const char\s*\*)\s*(oxi_\w+)\s*\(([^)]*)\)\s*;", txt, flags=re.S):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        params = [p.strip() for p in params.split(",") if p.strip()]
        out[name] = ("ptr" if "*" in ret else "i32", [c_kind(p) for p in params])
    return out


def split_top(s: str):
    """Split at commas outside braces/parentheses."""
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return [p.strip() for p in parts]


def doc_ccalls():
    txt = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    calls = []
    for m in re.finditer(r"ccall\(\(\s*(:oxi_\w+|_\w+sym\(T\))\s*,\s*\w+\)\s*,", txt):
        i = m.end()
        rest = txt[i:]
        # return type, then the argument tuple in parentheses
        ret = re.match(r"\s*([\w{}]+)\s*,\s*", rest)
        j = ret.end()
        assert rest[j] == "(", rest[j:j + 40]
        depth, k = 0, j
        while True:
            if rest[k] == "(":
                depth += 1
            elif rest[k] == ")":
                depth -= 1
                if depth == 0:
                    break
            k += 1
        args = split_top(rest[j + 1:k])
        calls.append((m.group(1), ret.group(1), args))
    return calls


SYM_FAMILIES = {"_getrf_sym(T)": ["oxi_dgetrf", "oxi_sgetrf"], "_getrs_sym(T)": ["oxi_dgetrs", "oxi_sgetrs"]}


def test_every_ccall_matches_the_header():
    decls = header_decls()
    calls = doc_ccalls()
    assert len(calls) >= 15
    seen = set()
    for sym, ret, args in calls:
        names = SYM_FAMILIES.get(sym, [sym.lstrip(":")])
        for name in names:
            assert name in decls, f"{name} is not declared in include/oxiblas_b200.h"
            cret, cargs = decls[name]
            assert jl_kind(ret) == cret, (name, ret, cret)
            kinds = [jl_kind(a) for a in args]
            assert kinds == cargs, (name, kinds, cargs)
            seen.add(name)
    # the drop-in path's entry points are all bound
    for must in ("oxi_create", "oxi_destroy", "oxi_set_stream", "oxi_dgetrf", "oxi_sgetrf", "oxi_dgetrs",
                 "oxi_sgetrs", "oxi_dgesv_mixed", "oxi_dequilibrate", "oxi_dlu_adjoint", "oxi_set_option",
                 "oxi_last_error", "oxi_status_string", "oxi_dgemm_update"):
        assert must in seen, must


def test_precision_table_has_the_benchmarked_default():
    txt = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"const PREC = Dict\(([^)]*)\)", txt)
    assert m, "PREC table missing"
    table = dict((k.strip(), int(v)) for k, v in (e.split("=>") for e in m.group(1).split(",")))
    assert table[":fp16x3"] == 5 and table["Float32"] == 0 and table[":bf16x3"] == 4
    assert "lowtype=:fp16x3" in txt
