"""The Fortran binding (ocotillo_b200/fortran/oco_b200.f90, ISO_C_BINDING) against include/oco.h:
no Fortran compiler is available here, so the check is textual -- the bind(C) derived type
oco_params has the C struct's members in order with matching kinds, and every bind(C) procedure
names a function oco.h declares, with the same number of arguments and by-value/pointer
agreement for each."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "ocotillo_b200", "fortran", "oco_b200.f90")
HDR = os.path.join(ROOT, "include", "oco.h")

KIND = {"int32_t": "integer(c_int32_t)", "double": "real(c_double)"}


def _c_struct(text, name):
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S)
    fields = []
    for line in re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S).split(";"):
        line = line.strip()
        if not line:
            continue
        typ, rest = line.split(None, 1)
        fields += [(n.strip(), typ) for n in rest.split(",")]
    return fields


def _f_type(text, name):
    m = re.search(r"type, bind\(C\) :: %s\n(.*?)end type %s" % (name, name), text, re.S)
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        kind, names = line.split("::")
        fields += [(n.strip(), kind.strip()) for n in names.split(",")]
    return fields


def _c_protos(text):
    body = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|void|int64_t|const char \*)\s*\*?\s*(oco_\w+)\((.*?)\);", body, re.S):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = args
    return out


def _f_procs(text):
    out = {}
    for m in re.finditer(r"(?:function|subroutine) (\w+)\(([^)]*)\)\s*(?:&\s*)?bind\(C, name=\"(\w+)\"\)(.*?)end (?:function|subroutine)",
                         text, re.S):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        decls = m.group(4)
        byval = {}
        for line in decls.splitlines():
            line = line.split("!")[0]
            if "::" not in line:
                continue
            attrs, names = line.split("::")
            for n in names.split(","):
                n = re.sub(r"\(.*", "", n).strip()
                byval[n] = ("value" in attrs)
        out[m.group(3)] = (args, byval)
    return out


def test_params_struct_matches_header():
    c = _c_struct(open(HDR).read(), "oco_params")
    f = _f_type(open(F90).read(), "oco_params")
    assert [n for n, _ in f] == [n for n, _ in c]
    assert [k for _, k in f] == [KIND[t] for _, t in c]


def test_procedures_match_header():
    protos = _c_protos(open(HDR).read())
    procs = _f_procs(open(F90).read())
    assert len(procs) >= 10
    for name, (args, byval) in procs.items():
        assert name in protos, name
        cargs = protos[name]
        assert len(args) == len(cargs), name
        for a, ca in zip(args, cargs):
            c_pointer = "*" in ca
            # a C pointer is a Fortran array/derived-type/intent(out) dummy or a c_ptr by value;
            # a C scalar is a Fortran dummy passed by value
            if not c_pointer:
                assert byval.get(a, False), (name, a, ca)
