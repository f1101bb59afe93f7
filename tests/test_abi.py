"""The C-ABI library loads, exports every symbol include/ash3d_b200.h
declares, and reports errors instead of falling back to a CPU path (these
tests make no compute calls, so they run without a GPU)."""
import ctypes as C
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _declared():
    txt = (ROOT / "include" / "ash3d_b200.h").read_text()
    return sorted(set(re.findall(r"\b(a3g_[a-z_0-9]+)\s*\(", txt)))


def test_header_and_binding_agree(pkg):
    from volcano_ash3d_b200 import _lib
    assert sorted(_lib.EXPORTED) == _declared()


def test_library_exports_every_symbol(pkg):
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.a3g_abi_version() == 1


def test_default_params_are_reference_defaults(pkg):
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    p = _lib.Params()
    lib.a3g_default_params(C.byref(p))
    assert p.limiter == _lib.LIMITERS["superbee"]
    assert (p.cfl, p.dt_min, p.dt_max) == (0.8, 1.0e-5, 1.0)       # Ash3d_VariableModules.f90:367-371
    assert (p.imp_fac, p.imp_dt_fac) == (0.5, 4.0)                # Diffusion.F90:53-54
    assert p.eps_thresh == 1.0e-10 and p.cloudcon_grid_thresh == 1.0e-7
    assert p.magma_density == 2500.0


def test_create_rejects_bad_arguments(pkg):
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    g = _lib.GridDesc(nx=0, ny=4, nz=4, ns=1)
    p = _lib.Params()
    lib.a3g_default_params(C.byref(p))
    ctx = C.c_void_p()
    rc = lib.a3g_create(C.byref(g), C.byref(p), 0, C.byref(ctx))
    assert rc == 1 and not ctx
    g = _lib.GridDesc(nx=4, ny=4, nz=4, ns=1)
    p.zscaling_id = 3  # ZScaling_ID is 0, 1 or 2 (src/AdvectionVert_DCU.f90:71-80)
    rc = lib.a3g_create(C.byref(g), C.byref(p), 0, C.byref(ctx))
    assert rc == 1 and b"ZScaling_ID" in lib.a3g_last_error()


def test_no_cpu_fallback_without_gpu(pkg):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    g = _lib.GridDesc(nx=4, ny=4, nz=4, ns=1)
    p = _lib.Params()
    lib.a3g_default_params(C.byref(p))
    ctx = C.c_void_p()
    rc = lib.a3g_create(C.byref(g), C.byref(p), 0, C.byref(ctx))
    assert rc != 0 and not ctx


def _header_kinds():
    """Parameter kinds of every a3g_ prototype: 'int32', 'int64', 'uint64',
    'double', or 'p:<element>' for pointers."""
    txt = (ROOT / "include" / "ash3d_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(a3g_\w+)\s*\(([^)]*)\)\s*;", txt):
        kinds = []
        for p in (q.strip() for q in m.group(2).split(",")):
            if not p or p == "void":
                continue
            base = ("double" if re.search(r"\bdouble\b", p) else "float" if re.search(r"\bfloat\b", p)
                    else "int32" if re.search(r"\bint32_t\b|\bint\b", p) else "int64" if "int64_t" in p
                    and "uint" not in p else "uint64" if re.search(r"\buint64_t\b|\bsize_t\b", p)
                    else "other")
            stars = p.count("*")
            if re.search(r"\ba3g_met_provider\b", p):  # the met-step callback (a function pointer)
                kinds.append("fn")
                continue
            kinds.append("p:p" if stars >= 2 else "p:" + base if stars else base)
        out[m.group(1)] = kinds
    return out


def _ctypes_kind(t):
    if isinstance(t, type) and issubclass(t, C._CFuncPtr):
        return "fn"
    if t is C.c_void_p:
        return "p:void"
    if hasattr(t, "_type_") and isinstance(t, type) and issubclass(t, C._Pointer):
        inner = _ctypes_kind(t._type_)
        if inner.startswith("p:"):
            return "p:p"
        return "p:" + (inner if not inner.startswith("?") else "other")
    return {C.c_int32: "int32", C.c_int64: "int64", C.c_uint64: "uint64", C.c_double: "double",
            C.c_float: "float"}.get(t, "?" + getattr(t, "__name__", str(t)))


def test_ctypes_signatures_match_header(pkg):
    """Every argtypes list the binding sets has the prototype's arity, scalar
    types and pointer element types (c_void_p stands for any pointer)."""
    from volcano_ash3d_b200 import _lib
    lib = _lib.load()
    hdr = _header_kinds()
    for name in _lib.EXPORTED:
        got = [_ctypes_kind(t) for t in (getattr(lib, name).argtypes or [])]
        want = hdr[name]
        assert len(got) == len(want), f"{name}: {got} against {want}"
        for g, w in zip(got, want):
            assert g == w or (g == "p:void" and w.startswith("p:")) or (g == "p:other" and w == "p:other"), \
                f"{name}: {got} against {want}"
