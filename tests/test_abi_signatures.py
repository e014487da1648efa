"""The Python bindings agree with include/gfn1_b200.h (CPU only, no compute
calls): every prototype the bindings declare has the header's parameter count,
pointer/scalar kinds and scalar widths, and the option and output structs have
the header's fields in the header's order.  A mismatch here would pass wrong
arguments or shift struct fields silently."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gfn1_b200.h")

# C scalar types of the header and their ctypes counterparts
_SCALARS = {
    "int": ctypes.c_int, "int32_t": ctypes.c_int32, "int64_t": ctypes.c_int64, "uint64_t": ctypes.c_uint64,
    "double": ctypes.c_double, "float": ctypes.c_float,
}


def _strip_comments(text: str) -> str:
    return re.sub(r"/\*.*?\*/", " ", text, flags=re.S)


def _kind(ctype: str):
    """'ptr' for pointers, else the ctypes scalar type of a C declaration."""
    ctype = ctype.replace("const", " ").strip()
    if "*" in ctype:
        return "ptr"
    base = ctype.split()[0]
    return _SCALARS[base]


def _ctypes_kind(t):
    if t in (ctypes.c_void_p, ctypes.c_char_p) or issubclass(t, ctypes._Pointer):
        return "ptr"
    return t


def _same_scalar(a, b) -> bool:
    """Same width, both floating or both integer, and the same signedness
    (ctypes codes: lower case signed, upper case unsigned)."""
    fa, fb = a._type_ in "fd", b._type_ in "fd"
    return ctypes.sizeof(a) == ctypes.sizeof(b) and fa == fb and (fa or a._type_.islower() == b._type_.islower())


def _prototypes():
    text = _strip_comments(open(HEADER).read())
    protos = {}
    for m in re.finditer(r"([\w\s\*]+?)\b(gfn1_\w+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        ret, name, params = m.group(1).strip().split("\n")[-1].strip(), m.group(2), m.group(3).strip()
        args = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        # every parameter is named: drop the name (the last identifier)
        kinds = [_kind(re.sub(r"\b\w+\s*$", "", a)) for a in args]
        protos[name] = (ret, kinds)
    return protos


def _struct_fields(name: str):
    text = _strip_comments(open(HEADER).read())
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(.*?)(\w+)$", decl, flags=re.S)
        fields.append((m.group(2), _kind(m.group(1))))
    return fields


def test_header_prototypes_parse():
    protos = _prototypes()
    assert len(protos) >= 30
    assert protos["gfn1_run"][1][:3] == ["ptr", ctypes.c_int, "ptr"]
    assert protos["gfn1_guess_param_count"] == ("int64_t", [])


def test_bound_functions_match_header():
    from gfn1_rs import _build, _lib

    _build.build()
    L = _lib.load()
    protos = _prototypes()
    checked = 0
    for name, (ret, kinds) in sorted(protos.items()):
        fn = getattr(L, name)
        if fn.argtypes is None:
            continue  # not bound from Python
        got = [_ctypes_kind(t) for t in fn.argtypes]
        assert len(got) == len(kinds), (name, len(got), len(kinds))
        for i, (g, h) in enumerate(zip(got, kinds)):
            if h == "ptr" or g == "ptr":
                assert g == h, (name, i, g, h)
            else:
                assert _same_scalar(g, h), (name, i, g, h)
        if ret == "int64_t":
            assert fn.restype is not None and ctypes.sizeof(fn.restype) == 8, name
        elif ret == "void":
            assert fn.restype is None, name
        elif "char" in ret and "*" in ret:
            assert fn.restype is ctypes.c_char_p, name
        else:
            assert fn.restype in (ctypes.c_int, ctypes.c_int32), (name, fn.restype)
        checked += 1
    assert checked >= 30


@pytest.mark.parametrize("cname,pyname", [("gfn1_options", "Options"), ("gfn1_outputs", "Outputs")])
def test_structs_match_header(cname, pyname):
    from gfn1_rs import _lib

    header = _struct_fields(cname)
    py = [(n, _ctypes_kind(t)) for n, t in getattr(_lib, pyname)._fields_]
    assert [n for n, _ in py] == [n for n, _ in header]
    for (n, g), (_, h) in zip(py, header):
        if h == "ptr" or g == "ptr":
            assert g == h, n
        else:
            assert _same_scalar(g, h), n
