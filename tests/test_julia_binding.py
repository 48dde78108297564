"""CPU: the Julia module's ccall signatures and struct layouts against
include/dfft.h.  Julia is not installed here, so the binding is checked
mechanically: every `ccall((:dfft_..., libdfft), Ret, (Args...), ...)` names
a declared entry point with the same number of arguments and compatible
types, and every Julia struct mirroring a C struct has the C field offsets
and size (C side measured with offsetof in a probe compiled by the host
compiler)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "daggerfft.jl_b200", "julia", "DaggerFFTB200.jl")
HDR = os.path.join(ROOT, "include", "dfft.h")


def _balanced(s, i):
    """Index just past the bracket group that opens at s[i]."""
    pairs = {"(": ")", "{": "}", "[": "]"}
    stack = [pairs[s[i]]]
    j = i + 1
    while stack:
        ch = s[j]
        if ch in pairs:
            stack.append(pairs[ch])
        elif ch == stack[-1]:
            stack.pop()
        j += 1
    return j


def _split_top(s):
    """Split at commas that are not inside brackets."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def julia_ccalls():
    src = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(\(:(dfft_\w+),\s*libdfft\)", src):
        start = m.start() + len("ccall")
        end = _balanced(src, start)
        parts = _split_top(src[start + 1:end - 1])
        ret = parts[1]
        tup = parts[2]
        assert tup.startswith("(") and tup.endswith(")"), (m.group(1), tup)
        args = _split_top(tup[1:-1])
        calls.append((m.group(1), ret, args))
    return calls


def c_prototypes():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    protos = {}
    for m in re.finditer(r"DFFT_API\s+([\w\s\*]+?)\b(dfft_\w+)\s*\(([^)]*)\)\s*;", txt):
        ret = " ".join(m.group(1).split())
        params = [" ".join(p.split()) for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
        ptypes = []
        for p in params:
            t = re.sub(r"\b\w+$", "", p).strip()  # drop the parameter name
            ptypes.append(t.replace(" *", "*").replace("* ", "*"))
        protos[m.group(2)] = (ret, ptypes)
    return protos


OPAQUE = {"dfft_plan", "dfft_batch", "dfft_server", "dfft_copy_plan"}
STRUCTS = {"dfft_request": "DfftRequest", "dfft_server_stats": "DfftServerStats",
           "dfft_block_copy": "DfftBlockCopy"}
SCALAR = {"int": {"Cint"}, "unsigned": {"Cuint"}, "int64_t": {"Int64"}, "size_t": {"Csize_t"},
          "uint64_t": {"UInt64"}, "int32_t": {"Int32"}}
PTR_OF = {"int64_t": {"Int64"}, "int32_t": {"Int32"}, "int": {"Cint"}, "uint64_t": {"UInt64"},
          "size_t": {"Csize_t"}, "char": {"UInt8", "Cchar"}}


def compatible(ctype, jtype):
    c = ctype.replace("const ", "").strip()
    j = jtype.strip()
    if c in SCALAR:
        return j in SCALAR[c]
    if c in OPAQUE:
        return j == "Ptr{Cvoid}"
    if c == "void*":
        return j in ("Ptr{Cvoid}", "CuPtr{Cvoid}")
    if c == "char*":
        return j in ("Ptr{UInt8}", "Cstring", "Ptr{Cchar}")
    if c.endswith("*const*") or c == "void*const*":
        return j in ("Ptr{Ptr{Cvoid}}", "Ptr{CuPtr{Cvoid}}")
    if c.endswith("*"):
        base = c[:-1].strip()
        inner = re.match(r"^(?:Ptr|Ref)\{(.+)\}$", j)
        if not inner:
            return False
        jin = inner.group(1)
        if base in OPAQUE:
            return jin == "Ptr{Cvoid}"
        if base in STRUCTS:
            return jin == STRUCTS[base]
        if base in PTR_OF:
            return jin in PTR_OF[base]
        if base == "void":
            return jin in ("Cvoid",)
    return False


def test_every_ccall_matches_the_header():
    protos = c_prototypes()
    calls = julia_ccalls()
    assert len(calls) >= 25, len(calls)
    bad = []
    for name, ret, args in calls:
        if name not in protos:
            bad.append(f"{name}: not declared in dfft.h")
            continue
        cret, cargs = protos[name]
        if len(args) != len(cargs):
            bad.append(f"{name}: {len(args)} arguments, header has {len(cargs)}")
            continue
        if cret == "int" and ret != "Cint":
            bad.append(f"{name}: returns {ret}, header int")
        if cret == "const char*" and ret != "Cstring":
            bad.append(f"{name}: returns {ret}, header const char*")
        for i, (jt, ct) in enumerate(zip(args, cargs)):
            if not compatible(ct, jt):
                bad.append(f"{name} arg {i + 1}: Julia {jt} vs C {ct}")
    assert not bad, "\n".join(bad)


def test_binding_covers_the_entry_points_a_julia_user_needs():
    names = {n for n, _, _ in julia_ccalls()}
    need = {"dfft_plan_create", "dfft_execute", "dfft_plan_destroy", "dfft_plan_output_shape",
            "dfft_plan_describe", "dfft_wisdom_export", "dfft_wisdom_import", "dfft_batch_create_ex",
            "dfft_batch_execute", "dfft_server_create", "dfft_server_submit", "dfft_server_wait",
            "dfft_server_poll", "dfft_server_get_stats", "dfft_server_release", "dfft_copy_plan_create",
            "dfft_copy_plan_execute", "dfft_last_error"}
    assert need <= names, need - names


JULIA_SIZES = {"Cint": 4, "Cuint": 4, "Int32": 4, "Int64": 8, "UInt64": 8, "Csize_t": 8, "Cdouble": 8,
               "Ptr{Cvoid}": 8}


def julia_struct(name):
    src = open(JL).read()
    m = re.search(r"^struct " + name + r"\n(.*?)^end", src, flags=re.S | re.M)
    assert m, name
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("#")[0].strip()
        if not line:
            continue
        fname, ftype = [x.strip() for x in line.split("::")]
        tm = re.match(r"NTuple\{(\d+),(\w+)\}", ftype)
        if tm:
            n, el = int(tm.group(1)), tm.group(2)
            fields.append((fname, JULIA_SIZES[el], n * JULIA_SIZES[el]))
        else:
            fields.append((fname, JULIA_SIZES[ftype], JULIA_SIZES[ftype]))
    # C layout rules (what Julia uses for isbits structs): align each field
    off, offs, maxal = 0, {}, 1
    for fname, al, sz in fields:
        off = (off + al - 1) // al * al
        offs[fname] = off
        off += sz
        maxal = max(maxal, al)
    return offs, (off + maxal - 1) // maxal * maxal


@pytest.mark.parametrize("cname,jname", sorted(STRUCTS.items()))
def test_struct_layouts_match_c(cname, jname, tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    offs, size = julia_struct(jname)
    src = tmp_path / "probe.c"
    body = "".join(f'  printf("{f} %zu\\n", offsetof({cname}, {f}));\n' for f in offs)
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"dfft.h\"\nint main(void) {\n"
                   + body + f'  printf("sizeof %zu\\n", sizeof({cname}));\n  return 0;\n}}\n')
    exe = tmp_path / "probe"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                         text=True).stdout.splitlines())
    for f, o in offs.items():
        assert int(got[f]) == o, (cname, f, got[f], o)
    assert int(got["sizeof"]) == size, (cname, got["sizeof"], size)
