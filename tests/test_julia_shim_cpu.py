"""The Julia binding cannot run here (no Julia), so its `ccall`s are checked statically against
the C ABI: every symbol it calls is declared in include/ptstokes.h and exported by
libptstokes.so, and each call passes as many arguments as the C prototype takes. The
`Desc` struct lists the fields of pts_desc in order."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JULIA = os.path.join(ROOT, "pseudotransientstokes.jl_b200", "julia")
HEADER = os.path.join(ROOT, "include", "ptstokes.h")


def split_top(s):
    """Split a comma list at depth 0 of {} and () nesting."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "{(":
            depth += 1
        elif ch in "})":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def tuple_after(text, start):
    """The parenthesised tuple that starts at text[start] == '(' (balanced)."""
    assert text[start] == "("
    depth = 0
    for k in range(start, len(text)):
        depth += text[k] == "("
        depth -= text[k] == ")"
        if depth == 0:
            return text[start + 1:k]
    raise AssertionError("unbalanced")


def header_prototypes():
    h = open(HEADER).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    protos = {}
    for m in re.finditer(r"PTS_API\s+[\w\s\*]+?\b(pts_\w+)\s*\(([^;]*?)\)\s*;", h, flags=re.S):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else len(split_top(args))
    return protos


def julia_calls():
    calls = []
    for f in sorted(os.listdir(JULIA)):
        if not f.endswith(".jl"):
            continue
        text = open(os.path.join(JULIA, f)).read()
        for m in re.finditer(r"ccall\(\((.*?),\s*libpts\),\s*(\w+),\s*", text):
            lit = re.fullmatch(r":(pts_\w+)", m.group(1).strip())
            name = lit.group(1) if lit else None  # None: a symbol interpolated by @eval
            types = tuple_after(text, m.end())
            calls.append((f, name, len(split_top(types))))
    return calls


def test_every_ccall_matches_the_header():
    protos = header_prototypes()
    assert len(protos) > 40
    calls = julia_calls()
    assert len(calls) >= 30
    checked = 0
    for f, name, nargs in calls:
        if name is None:  # the role loop interpolates its symbol: checked below
            continue
        assert name in protos, (f, name)
        assert nargs == protos[name], (f, name, nargs, protos[name])
        checked += 1
    assert checked >= 25
    # the role entry points the @eval loop binds take the context only
    text = open(os.path.join(JULIA, "PTStokesB200.jl")).read()
    for sym in re.findall(r"\(:\w+!?, :(pts_\w+)\)", text):
        assert sym in protos, sym
        assert protos[sym] in (1, 5), sym  # (ctx) roles; init_inclusion! takes ctx + 4 numbers


def test_every_ccall_symbol_is_exported():
    lib = pytest.importorskip("ctypes").CDLL(os.path.join(ROOT, "pseudotransientstokes.jl_b200", "lib",
                                                         "libptstokes.so"))
    text = "".join(open(os.path.join(JULIA, f)).read() for f in os.listdir(JULIA) if f.endswith(".jl"))
    for sym in sorted(set(re.findall(r":(pts_\w+)", text))):
        assert hasattr(lib, sym), sym


def test_desc_struct_field_order():
    h = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct pts_desc \{(.*?)\} pts_desc;", h, flags=re.S).group(1)
    cfields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        names = decl.split(None, 1)[1]
        cfields += [n.strip() for n in names.split(",")]
    jl = open(os.path.join(JULIA, "PTStokesB200.jl")).read()
    jbody = re.search(r"struct Desc\n(.*?)\nend", jl, flags=re.S).group(1)
    jfields = [m.group(1) for m in re.finditer(r"(\w+)::", jbody)]
    assert jfields == cfields
