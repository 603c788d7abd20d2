"""The Fortran iso_c_binding module (interfaces/chidg_gpu_mod.f90) against
include/chidg_gpu.h, checked as text (no Fortran compiler is needed): every
entry point of the header has exactly one bind(c) interface under its own
name, with the same number of arguments, and every argument is passed the
way the C prototype takes it -- C scalars by value with the matching
iso_c_binding kind, C pointers by reference or as type(c_ptr), value."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

C_KIND = {"int": "c_int", "int32_t": "c_int32_t", "int64_t": "c_int64_t", "double": "c_double",
          "size_t": "c_size_t"}
FUNPTR_TYPES = {"chidg_gpu_fill_fn"}     # C function pointer typedefs: type(c_funptr), value


def header_prototypes():
    text = open(os.path.join(ROOT, "include", "chidg_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\bint\s+(chidg_gpu_\w+)\s*\(([^)]*)\)\s*;", text):
        args = [" ".join(a.split()) for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = args
    return out


def fortran_interfaces():
    text = open(os.path.join(ROOT, "interfaces", "chidg_gpu_mod.f90")).read()
    text = "\n".join(line.split("!")[0] for line in text.splitlines())
    text = re.sub(r"&\s*\n\s*&?", " ", text)
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(c,\s*name='(\w+)'\)(.*?)end function", text, re.S):
        names = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        decls = {}
        for line in m.group(4).splitlines():
            if "::" not in line or line.strip().startswith("import"):
                continue
            attrs, vars_ = line.split("::", 1)
            for v in re.sub(r"\([^)]*\)", "", vars_).split(","):
                if v.strip():
                    decls[v.strip().lower()] = attrs.strip().lower()
        assert m.group(3) not in out, f"two interfaces bind {m.group(3)}"
        out[m.group(3)] = [(n, decls.get(n)) for n in names]
    return out


def test_every_header_entry_point_has_a_fortran_interface():
    hdr, ftn = header_prototypes(), fortran_interfaces()
    assert len(hdr) >= 60
    assert sorted(set(hdr) - set(ftn)) == []
    assert sorted(set(ftn) - set(hdr)) == []


def test_fortran_arguments_match_the_prototypes():
    hdr, ftn = header_prototypes(), fortran_interfaces()
    for name, cargs in hdr.items():
        fargs = ftn[name]
        assert len(fargs) == len(cargs), (name, cargs, fargs)
        for carg, (fname, decl) in zip(cargs, fargs):
            assert decl is not None, (name, fname, "undeclared")
            is_ptr = "*" in carg
            by_value = "value" in decl
            if is_ptr:
                assert (not by_value) or decl.startswith("type(c_ptr)"), (name, carg, decl)
            else:
                ctype = carg.replace("const ", "").split()[0]
                assert by_value, (name, carg, decl)
                if ctype in FUNPTR_TYPES:
                    assert decl.startswith("type(c_funptr)"), (name, carg, decl)
                else:
                    assert f"({C_KIND[ctype]})" in decl, (name, carg, decl)
