"""The Fortran iso_c_binding layer (ls-sph-benchmarks_b200/fortran/lssph_cuda_mod.f90)
checked against the C ABI it binds, without a Fortran compiler.

A Fortran host that keeps the reference's driver (source/main.f90) calls the engine through
this module, so a slip in its hand-written mirror of lssph_params or in one interface would
corrupt every call from the reference's own language.  The module text is parsed here and
compared with include/lssph.h and the compiled library:
  * the bind(c) type lssph_params has the fields of the C struct, in order, with the same
    kinds; its natural-alignment layout gives the library's offsets and sizeof;
  * every bind(c, name=...) interface names a function the library exports and the header
    declares, with as many arguments, each passed the way the prototype takes it (VALUE for
    a C scalar, by reference or a type(c_ptr) value for a C pointer).
"""
import ctypes as C
import os
import re

import pytest

import lssph
from lssph import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "ls-sph-benchmarks_b200", "fortran", "lssph_cuda_mod.f90")
HDR = os.path.join(ROOT, "include", "lssph.h")

# Fortran kind -> (bytes, class); class c = character array of the stated length
KINDS = {"integer(c_int32_t)": (4, "i"), "integer(c_int64_t)": (8, "i"), "integer(c_int)": (4, "i"),
         "real(c_double)": (8, "f")}


def _strip(line: str) -> str:
    return line.split("!", 1)[0].rstrip()


def fortran_type_fields():
    text = open(MOD).read()
    body = re.search(r"type, bind\(c\) :: lssph_params\n(.*?)\n\s*end type lssph_params", text, re.S).group(1)
    fields = []
    for raw in body.splitlines():
        line = _strip(raw).strip()
        if not line:
            continue
        kind, names = (s.strip() for s in line.split("::"))
        for name in (n.strip() for n in names.split(",")):
            m = re.fullmatch(r"(\w+)\((\d+)\)", name)
            if kind == "character(kind=c_char)":
                assert m, line
                fields.append((m.group(1), int(m.group(2)), "c"))
            else:
                assert not m and kind in KINDS, line
                fields.append((name, *KINDS[kind]))
    return fields


def ctypes_class(t):
    if issubclass(t, C.Array):
        return t._length_, "c"
    if t in (C.c_double,):
        return 8, "f"
    return C.sizeof(t), "i"


def test_fortran_params_type_matches_the_c_struct():
    f = fortran_type_fields()
    c = [(name, *ctypes_class(t)) for name, t in _abi.Params._fields_]
    assert [x[0].lower() for x in f] == [x[0].lower() for x in c]
    assert [x[1:] for x in f] == [x[1:] for x in c]
    # natural-alignment layout of the Fortran type = the library's offsets and size
    off = 0
    for name, size, cls in f:
        align = 1 if cls == "c" else size
        off = (off + align - 1) // align * align
        assert off == getattr(_abi.Params, name).offset, name
        off += size
    off = (off + 7) // 8 * 8
    assert off == C.sizeof(_abi.Params) == lssph.load().lssph_params_sizeof()


def fortran_interfaces():
    text = open(MOD).read()
    block = re.search(r"\n\s*interface\n(.*?)\n\s*end interface", text, re.S).group(1)
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\(([^)]*)\)\s*(?:&\s*\n\s*)?bind\(c,\s*name=\"(\w+)\"\)"
                         r"(.*?)\n\s*end (?:function|subroutine)", block, re.S):
        _, args, cname, decls = m.groups()
        dummies = [a.strip() for a in args.split(",") if a.strip()]
        how = {}
        for raw in decls.splitlines():
            line = _strip(raw).strip()
            if "::" not in line or line.startswith("import"):
                continue
            spec, names = (s.strip() for s in line.split("::"))
            value = "value" in [s.strip() for s in spec.split(",")]
            is_cptr = spec.startswith("type(c_ptr)")
            for n in names.split(","):
                n = re.sub(r"\(.*\)", "", n).strip()
                how[n] = "pointer" if (not value or is_cptr) else "scalar"
        out[cname] = [how[d] for d in dummies]
    return out


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"^\s*[\w\s\*]*?\b(lssph_\w+)\s*\(([^;{]*?)\)\s*;", text, re.S | re.M):
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        protos[m.group(1)] = ["pointer" if "*" in p else "scalar" for p in params]
    return protos


def test_every_fortran_interface_binds_an_exported_function_with_matching_arguments():
    lib = lssph.load()
    ifaces = fortran_interfaces()
    protos = c_prototypes()
    assert len(ifaces) >= 20
    for name, args in ifaces.items():
        assert hasattr(lib, name), f"{name} is not exported by liblssph.so"
        assert name in protos, f"{name} is not declared in include/lssph.h"
        assert args == protos[name], f"{name}: Fortran passes {args}, the prototype takes {protos[name]}"


@pytest.mark.parametrize("name", ["lssph_create", "lssph_step", "lssph_download", "lssph_destroy"])
def test_the_time_loop_entry_points_are_bound(name):
    # the calls main_gpu.f90 makes in place of source/main.f90:119-166
    assert name in fortran_interfaces()
