"""The C-ABI library loads and exports every entry point include/*.h
declares, with the status-code constants of the reference enum. CPU only:
no compute call is made."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cupcfd_gpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cupcfd_gpu_gradient_phi_gauss_dolfyn" in names
    assert "cupcfd_gpu_flux_mass_dolfyn_face_loop" in names
    assert len(names) >= 20


def test_library_loads_and_exports_every_symbol(cg):
    L = cg.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers exactly the declared surface
    assert set(cg.SIGNATURES) == set(declared_functions())


def test_exported_symbols_are_c_linkage(cg):
    cg.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", cg.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (cupcfd_gpu_\w+)$", out, re.M))
    assert set(declared_functions()) <= exported


def test_status_constants_match_reference_enum(cg):
    text = open(os.path.join(ROOT, "include", "cupcfd_gpu.h")).read()
    consts = dict((k, int(v)) for k, v in re.findall(r"#define CUPCFD_(E_\w+)\s+(\d+)", text))
    # values of cupcfd::error::eCodes (include/error/Error.h:32-144, enum from 0)
    assert consts == {"E_ARRAY_SIZE_MISMATCH": 25, "E_INVALID_INDEX": 68, "E_CONFIG_INVALID_VALUE": 90,
                      "E_SUCCESS": 95, "E_ERROR": 98, "E_NULL_PTR": 99, "E_NOT_IMPLEMENTED": 109,
                      "E_FILE_MISSING": 10, "E_INVALID_FILE_FORMAT": 105, "E_CONFIG_OPT_NOT_FOUND": 92}
    assert (cg.E_SUCCESS, cg.E_INVALID_INDEX, cg.E_ERROR) == (95, 68, 98)


def test_version_and_error_string_without_gpu(cg):
    L = cg.lib()
    assert b"sm_100a" in L.cupcfd_gpu_version()
    assert isinstance(cg.last_error(), str)


def test_null_arguments_rejected_without_touching_the_gpu(cg):
    import ctypes as C
    L = cg.lib()
    assert L.cupcfd_gpu_mesh_create(None, None, None) == cg.E_NULL_PTR
    assert L.cupcfd_gpu_mesh_destroy(None) == cg.E_NULL_PTR
    assert L.cupcfd_gpu_mesh_get_info(None, None) == cg.E_NULL_PTR
    assert L.cupcfd_gpu_gradient_phi_gauss_dolfyn(None, 1, None, 0, None, 0, None, 0, 32, 8, None, 0, 32, 8, 8, 0, 0) == cg.E_NULL_PTR
    h = C.c_void_p()
    assert L.cupcfd_gpu_mesh_create_structgen(0, 4, 4, None, None, C.byref(h)) == cg.E_CONFIG_INVALID_VALUE
    assert L.cupcfd_gpu_mesh_create_jittered(4, 4, 4, 0.7, 1, 1, None, C.byref(h)) == cg.E_CONFIG_INVALID_VALUE
    assert L.cupcfd_gpu_mesh_create_structgen(2048, 2048, 2048, None, None, C.byref(h)) == cg.E_NOT_IMPLEMENTED


def declared_arity():
    """Parameter count of every function declared in include/*.h."""
    out = {}
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"\b(cupcfd_gpu_\w+)\s*\(([^)]*)\)\s*;", text):
            params = [p for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
            out[m.group(1)] = len(params)
    return out


def test_binding_arity_matches_header(cg):
    ar = declared_arity()
    assert set(ar) == set(cg.SIGNATURES)
    bad = {n: (len(cg.SIGNATURES[n][0]), k) for n, k in ar.items() if len(cg.SIGNATURES[n][0]) != k}
    assert not bad, bad


def test_device_timers_without_gpu(cg):
    """Timers off by default; enabling and reading with nothing recorded
    needs no GPU and reports no kernels."""
    import ctypes as C
    L = cg.lib()
    assert L.cupcfd_gpu_timing_read(0, None, None, None, None) == cg.E_NULL_PTR
    cg.timing_enable(True)
    assert cg.timing_read() == {}
    cg.timing_enable(False)
    n = C.c_int32(-1)
    assert L.cupcfd_gpu_timing_read(0, None, None, None, C.byref(n)) == cg.E_SUCCESS and n.value == 0
