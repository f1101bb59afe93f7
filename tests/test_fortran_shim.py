"""The Fortran drop-in (volcano-ash3d_b200/fortran/ash3d_b200_shim.f90) binds
the C-ABI as include/ash3d_b200.h declares it.  There is no Fortran compiler
here, so its ISO_C_BINDING interface blocks are read as text: every bound
name exists in the header, with the same number of arguments, and each
argument's passing (a pointer, or a value of int32 / int / double) matches
the C prototype."""
import pathlib
import re

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _header():
    txt = (ROOT / "include" / "ash3d_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b[\w\s\*]+?\b(a3g_\w+)\s*\(([^)]*)\)\s*;", txt):
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        kinds = []
        for p in params:
            if "*" in p:
                kinds.append("ptr")
            elif re.search(r"\bint32_t\b", p):
                kinds.append("int32")
            elif re.search(r"\bdouble\b", p):
                kinds.append("double")
            elif re.search(r"\bint\b", p):
                kinds.append("int")
            else:
                kinds.append("?" + p)
        out[m.group(1)] = kinds
    return out


def _shim():
    txt = (ROOT / "volcano-ash3d_b200" / "fortran" / "ash3d_b200_shim.f90").read_text()
    txt = re.sub(r"&\s*\n\s*", " ", txt)  # join continuation lines
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(a3g_\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(a3g_\w+)\"\)"
                         r"(.*?)end (?:function|subroutine)", txt, flags=re.S):
        fname, args, cname, body = m.group(1), m.group(2), m.group(3), m.group(4)
        assert fname == cname, (fname, cname)
        names = [a.strip().lower() for a in args.split(",") if a.strip()]
        decl = {}
        for line in body.splitlines():
            d = re.match(r"\s*(type\(\w+\)|integer\(c_int32_t\)|integer\(c_int\)|real\(c_double\))"
                         r"((?:\s*,\s*[\w()]+)*)\s*::\s*(.*)", line)
            if not d:
                continue
            by_value = "value" in d.group(2)
            for v in d.group(3).split(","):
                v = v.strip().lower()
                if not v:
                    continue
                if not by_value or d.group(1) == "type(c_ptr)":
                    decl[v] = "ptr"
                else:
                    decl[v] = {"integer(c_int32_t)": "int32", "integer(c_int)": "int",
                               "real(c_double)": "double"}[d.group(1)]
        out[cname] = [decl.get(n, "undeclared " + n) for n in names]
    return out


def test_shim_interfaces_match_header():
    hdr, shim = _header(), _shim()
    txt = (ROOT / "volcano-ash3d_b200" / "fortran" / "ash3d_b200_shim.f90").read_text()
    assert len(shim) == len(re.findall(r"bind\(C,\s*name=", txt))  # every interface block parsed
    for name, kinds in shim.items():
        assert name in hdr, f"{name} is bound by the shim but not declared"
        want = ["int" if k == "int32" else k for k in hdr[name]]
        got = ["int" if k == "int32" else k for k in kinds]
        assert got == want, f"{name}: shim {kinds} against header {hdr[name]}"


def test_new_restart_entry_points_are_bound():
    shim = _shim()
    for name in ("a3g_output_ashcon", "a3g_restart_load", "a3g_set_topo", "a3g_add_source_umbrella"):
        assert name in shim, name
