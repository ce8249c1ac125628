"""cupcfd_b200 -- Python front end of libcupcfd_gpu (the C-ABI CUDA library).

The library implements CUP-CFD's finite-volume face-loop path on B200:
``GradientPhiGaussDolfyn`` (include/fvm/implementation/component/GradientKernels.ipp)
and ``FluxMassDolfynFaceLoop`` (include/fvm/implementation/component/MassKernels.ipp)
over the MiniSoA mesh. This module is a thin ctypes layer over
``include/cupcfd_gpu.h``: host calls take numpy arrays in the reference's
numbering and layout and return the reference's eCodes integers; device calls
take torch CUDA tensors in the mesh's internal numbering. torch is used only
for device memory and streams.

There is no CPU fallback: every call runs the CUDA library, and importing
fails loudly when the library cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# CUPCFD_GPU_LIB selects another build of the same library (e.g. a variant
# built with different CUPCFD_* tuning macros); default: the in-tree build.
LIB_PATH = os.environ.get("CUPCFD_GPU_LIB") or os.path.join(HERE, "libcupcfd_gpu.so")

# eCodes values (include/error/Error.h)
E_ARRAY_SIZE_MISMATCH = 25
E_INVALID_INDEX = 68
E_CONFIG_INVALID_VALUE = 90
E_SUCCESS = 95
E_ERROR = 98
E_NULL_PTR = 99
E_NOT_IMPLEMENTED = 109
E_FILE_MISSING = 10
E_INVALID_FILE_FORMAT = 105

RTYPE_DEFAULT, RTYPE_INLET, RTYPE_OUTLET, RTYPE_SYMP, RTYPE_WALL = range(5)
PREC_F64, PREC_F32C, PREC_F32REF = 0, 1, 2
ORDER_NATIVE, ORDER_MORTON, ORDER_OWNER, ORDER_RCM = 0, 1, 2, 3
SIGN_REFERENCE, SIGN_SIGNED = 0, 1

_lock = threading.Lock()
_lib = None


class CupcfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cupcfd_gpu error {code}: {msg}")
        self.code = code


class Vec3View(C.Structure):
    _fields_ = [("base", C.c_void_p), ("stride", C.c_int32), ("offset", C.c_int32)]


class MeshView(C.Structure):
    _fields_ = [("nCells", C.c_int32), ("nFaces", C.c_int32), ("nBoundaries", C.c_int32), ("real_size", C.c_int32),
                ("faceCell1", C.c_void_p), ("faceCell2", C.c_void_p), ("faceBnd", C.c_void_p),
                ("faceLambda", C.c_void_p), ("faceArea", C.c_void_p),
                ("faceNorm", Vec3View), ("faceCenter", Vec3View), ("faceXpac", Vec3View), ("faceXnac", Vec3View),
                ("cellCenter", Vec3View), ("cellVolume", C.c_void_p)]


class HaloField(C.Structure):
    _fields_ = [("field", C.c_void_p), ("elemSize", C.c_int32), ("ncomp", C.c_int32), ("ld", C.c_int64),
                ("buffer", C.c_void_p)]


class MeshOptions(C.Structure):
    _fields_ = [("order", C.c_int32), ("precisions", C.c_int32), ("device", C.c_int32)]


class MeshInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("nCells", "nFaces", "nInteriorFaces", "nBoundaries", "nRegions",
                                         "nIncidences", "maxCellFaces", "order", "precisions", "bandwidth")] + [
        ("deviceBytes", C.c_int64), ("tiles", C.c_int32), ("fullWidth", C.c_int32)]


# exported symbols of include/cupcfd_gpu.h with their ctypes signatures
_VP, _I, _I64, _D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
SIGNATURES = {
    "cupcfd_gpu_last_error": ([], C.c_char_p),
    "cupcfd_gpu_version": ([], C.c_char_p),
    "cupcfd_gpu_launch_count": ([], C.c_int64),
    "cupcfd_gpu_timing_enable": ([_I], _I),
    "cupcfd_gpu_timing_read": ([_I, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_mesh_create": ([_VP, _VP, _VP], _I),
    "cupcfd_gpu_mesh_create_structgen": ([_I, _I, _I, _VP, _VP, _VP], _I),
    "cupcfd_gpu_mesh_create_jittered": ([_I, _I, _I, _D, C.c_uint64, _I, _VP, _VP], _I),
    "cupcfd_gpu_mesh_destroy": ([_VP], _I),
    "cupcfd_gpu_mesh_save": ([_VP, C.c_char_p], _I),
    "cupcfd_gpu_mesh_load": ([C.c_char_p, _VP, _VP], _I),
    "cupcfd_gpu_hdf5_mesh_counts": ([C.c_char_p, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_hdf5_mesh_read": ([C.c_char_p, _I, _I, _I] + [_VP] * 11, _I),
    "cupcfd_gpu_mesh_load_hdf5": ([C.c_char_p, _VP, _VP], _I),
    "cupcfd_gpu_hdf5_mesh_write": ([C.c_char_p, _I, _I, _I, _I] + [_VP] * 11, _I),
    "cupcfd_gpu_mesh_save_hdf5": ([_VP, C.c_char_p], _I),
    "cupcfd_gpu_hdf5_dataset_shape": ([C.c_char_p, C.c_char_p, _VP, _VP, _VP], _I),
    "cupcfd_gpu_hdf5_dataset_read": ([C.c_char_p, C.c_char_p, _VP, C.c_int64], _I),
    "cupcfd_gpu_mesh_get_info": ([_VP, _VP], _I),
    "cupcfd_gpu_mesh_set_regions": ([_VP, _I, _VP, _VP, _VP, _VP, _I], _I),
    "cupcfd_gpu_mesh_set_region_split": ([_VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop1": ([_VP, _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop2": ([_VP, _VP, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop3": ([_VP, _D, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop4": ([_VP, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _D, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop5": ([_VP, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _D, _I, _I, _I,
                                                    _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_region_loop": ([_VP, _VP, _I, _VP, _I, _D], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop1_f32": ([_VP, _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop2_f32": ([_VP, _VP, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop3_f32": ([_VP, C.c_float, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop4_f32": ([_VP, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _VP, _I, C.c_float,
                                                        _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_boundary_loop5_f32": ([_VP, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _VP, _I, C.c_float,
                                                        _I, _I, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_flux_mass_dolfyn_region_loop_f32": ([_VP, _VP, _I, _VP, _I, C.c_float], _I),
    "cupcfd_gpu_dev_boundary_loop1": ([_VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_boundary_loop2": ([_VP, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_boundary_loop3": ([_VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_boundary_loop4": ([_VP] * 9, _I),
    "cupcfd_gpu_dev_boundary_loop5": ([_VP] * 6 + [_D, _I, _I, _I, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_region_loop": ([_VP] * 5, _I),
    "cupcfd_gpu_mesh_set_face_rlencos": ([_VP, _VP, _I], _I),
    "cupcfd_gpu_mesh_set_boundary_distance": ([_VP, _VP, _I], _I),
    "cupcfd_gpu_mesh_boundary_shear": ([_VP, _VP, _VP, _I], _I),
    "cupcfd_gpu_mesh_region_force_tangent": ([_VP, _VP, _VP, _I], _I),
    "cupcfd_gpu_flux_uvw_dolfyn_face_loop1": ([_VP, _D, _D] + [_VP, _I] * 9 + [Vec3View, _I] * 3 + [_VP, _I] * 7, _I),
    "cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32": ([_VP, C.c_float, C.c_float] + [_VP, _I] * 9 + [Vec3View, _I] * 3 + [_VP, _I] * 7, _I),
    "cupcfd_gpu_flux_uvw_dolfyn_region_loop1": ([_VP], _I),
    "cupcfd_gpu_flux_uvw_dolfyn_bnds_loop1": ([_VP], _I),
    "cupcfd_gpu_dev_uvw_face_loop1": ([_VP, _D, _D] + [_VP] * 10 + [_I64] + [_VP] * 8, _I),
    "cupcfd_gpu_dev_uvw_region_loop1": ([_VP, _VP], _I),
    "cupcfd_gpu_dev_halo_pack": ([_VP, _I, _I, _I64, _VP, _I, _VP, _VP], _I),
    "cupcfd_gpu_dev_halo_unpack": ([_VP, _I, _I, _I, _VP, _VP, _I64, _VP], _I),
    "cupcfd_gpu_dev_halo_pack_fields": ([_VP, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_dev_halo_unpack_fields": ([_VP, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_dev_uvw_bnds_loop1": ([_VP, _VP], _I),
    "cupcfd_gpu_mesh_check_status": ([_VP, _VP], _I),
    "cupcfd_gpu_mesh_get_cell_face_csr": ([_VP, _VP, _I, _VP, _I], _I),
    "cupcfd_gpu_mesh_get_incidences": ([_VP, _VP, _I, _VP, _VP, _I], _I),
    "cupcfd_gpu_mesh_get_geometry": ([_VP] * 10, _I),
    "cupcfd_gpu_mesh_get_numbering": ([_VP, _VP, _VP], _I),
    "cupcfd_gpu_gradient_phi_gauss_dolfyn": ([_VP, _I, _VP, _I, _VP, _I, _VP, _I, _I, _I, _VP, _I, _I, _I, _I, _I, _I], _I),
    "cupcfd_gpu_flux_mass_dolfyn_face_loop": ([_VP, Vec3View, _I, Vec3View, _I, Vec3View, _I, Vec3View, _I]
                                              + [_VP, _I] * 10 + [_D] + [_VP] * 4 + [_I] * 4 + [_VP, _I] * 8, _I),
    "cupcfd_gpu_flux_mass_dolfyn_face_loop_f32": ([_VP, Vec3View, _I, Vec3View, _I, Vec3View, _I, Vec3View, _I]
                                                  + [_VP, _I] * 10 + [C.c_float] + [_VP] * 4 + [_I] * 4
                                                  + [_VP, _I] * 8, _I),
    "cupcfd_gpu_forward_adjoint": ([_VP, _I] + [_VP] * 16, _I),
    "cupcfd_gpu_forward_adjoint_f32": ([_VP, _I] + [_VP] * 16, _I),
    "cupcfd_gpu_dev_permute_cells": ([_VP, _I, _I, _VP, _I, _I64, _VP, _I, _I64, _VP], _I),
    "cupcfd_gpu_dev_permute_faces": ([_VP, _I, _VP, _I, _VP, _I, _VP], _I),
    "cupcfd_gpu_dev_gradient": ([_VP, _I, _I, _I, _VP, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_mass_plain": ([_VP, _I, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_gradient_adjoint": ([_VP, _I, _I, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_mass_plain_adjoint": ([_VP, _I, _VP, _VP, _VP, _VP], _I),
    "cupcfd_gpu_dev_forward": ([_VP, _I] + [_VP] * 8, _I),
    "cupcfd_gpu_dev_adjoint": ([_VP, _I] + [_VP] * 7, _I),
    "cupcfd_gpu_dev_forward_noalloc": ([_VP, _I] + [_VP] * 8, _I),
    "cupcfd_gpu_dev_forward_adjoint": ([_VP, _I] + [_VP] * 11, _I),
    "cupcfd_gpu_dev_error_norms": ([_VP, _I, _VP, _I, _I64, _D, _VP, _VP], _I),
}


def lib():
    """The loaded library (built from csrc/ with nvcc if the .so is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                import importlib.util
                spec = importlib.util.spec_from_file_location("_cupcfd_build", os.path.join(HERE, "build.py"))
                b = importlib.util.module_from_spec(spec)
                spec.loader.exec_module(b)
                b.build()
            L = C.CDLL(LIB_PATH)
            for name, (args, res) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _lib = L
        return _lib


def last_error() -> str:
    return lib().cupcfd_gpu_last_error().decode()


def launch_count() -> int:
    return int(lib().cupcfd_gpu_launch_count())


def timing_enable(on: bool = True):
    """Bracket this library's forward/adjoint kernel launches with CUDA events."""
    check(lib().cupcfd_gpu_timing_enable(1 if on else 0))


def timing_read(capacity: int = 32) -> dict:
    """{kernel name: (launches, device ms)} since the previous read (waits for the events)."""
    names = C.create_string_buffer(64 * capacity)
    launches = (C.c_int64 * capacity)()
    ms = (C.c_double * capacity)()
    count = C.c_int32()
    check(lib().cupcfd_gpu_timing_read(capacity, names, launches, ms, C.byref(count)))
    out = {}
    for i in range(min(count.value, capacity)):
        nm = names.raw[64 * i:64 * (i + 1)].split(b"\0", 1)[0].decode()
        out[nm] = (int(launches[i]), float(ms[i]))
    return out


def check(rc):
    if rc != E_SUCCESS:
        raise CupcfdError(rc, last_error())
    return rc


def _p(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    assert a.flags["C_CONTIGUOUS"], "host arrays must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


def _vec(a, real_size=8):
    """Vec3View of a host array: (n,3) packed, or an (n, k) array whose
    components sit at columns 1..3 (emulating the vptr-carrying
    EuclideanVector layout: k = 4 for double gives a 32-byte stride)."""
    if a is None:
        return Vec3View(None, 3 * real_size, 0)
    assert a.flags["C_CONTIGUOUS"]
    if a.ndim == 2 and a.shape[1] == 3:
        return Vec3View(a.ctypes.data, 3 * real_size, 0)
    if a.ndim == 2 and a.shape[1] == 4:
        return Vec3View(a.ctypes.data, 4 * real_size, real_size)
    raise ValueError("vector arrays must be (n,3) packed or (n,4) with a leading pad slot")


def _stream(s):
    if s is None:
        return None
    if hasattr(s, "cuda_stream"):
        return C.c_void_p(s.cuda_stream)
    return C.c_void_p(int(s))


# ---------------------------------------------------------------------------
# mesh
# ---------------------------------------------------------------------------
class Mesh:
    """A device mesh (cupcfd_gpu_mesh). Build with ``structgen``, ``jittered``
    or ``from_arrays``; free with ``close`` (or garbage collection)."""

    def __init__(self, handle):
        self.h = handle
        info = MeshInfo()
        check(lib().cupcfd_gpu_mesh_get_info(self.h, C.byref(info)))
        self.nCells, self.nFaces, self.nInteriorFaces = info.nCells, info.nFaces, info.nInteriorFaces
        self.nBoundaries, self.nIncidences, self.maxCellFaces = info.nBoundaries, info.nIncidences, info.maxCellFaces
        self.order, self.precisions, self.deviceBytes = info.order, info.precisions, info.deviceBytes
        self.bandwidth = info.bandwidth
        self.tiles = bool(info.tiles)
        self.full_width = info.fullWidth

    @staticmethod
    def _opts(order, precisions, device):
        return MeshOptions(order, precisions, device)

    @classmethod
    def structgen(cls, nx, ny, nz, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), order=ORDER_MORTON,
                  precisions=(1 << PREC_F64) | (1 << PREC_F32C), device=-1):
        h = C.c_void_p()
        b = (C.c_double * 6)(*bounds)
        o = cls._opts(order, precisions, device)
        check(lib().cupcfd_gpu_mesh_create_structgen(nx, ny, nz, b, C.byref(o), C.byref(h)))
        return cls(h)

    @classmethod
    def jittered(cls, nx, ny, nz, jitter=0.25, seed=1, permute=True, order=ORDER_MORTON,
                 precisions=(1 << PREC_F64) | (1 << PREC_F32C), device=-1):
        h = C.c_void_p()
        o = cls._opts(order, precisions, device)
        check(lib().cupcfd_gpu_mesh_create_jittered(nx, ny, nz, float(jitter), int(seed), int(bool(permute)),
                                                     C.byref(o), C.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, m, order=ORDER_MORTON, precisions=(1 << PREC_F64) | (1 << PREC_F32C), device=-1,
                    return_code=False):
        """Upload a host mesh given as a dict of numpy arrays (keys of a
        one-rank CupCfdSoAMesh: faceCell1/2, faceBnd, faceLambda, faceArea,
        faceNorm, faceCenter, faceXpac, faceXnac, cellCenter, cellVolume)."""
        rs = m["faceLambda"].dtype.itemsize
        keep = {k: np.ascontiguousarray(v) for k, v in m.items() if isinstance(v, np.ndarray)}
        v = MeshView()
        v.nCells, v.nFaces, v.nBoundaries, v.real_size = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"]), rs
        v.faceCell1, v.faceCell2, v.faceBnd = _p(keep["faceCell1"]), _p(keep["faceCell2"]), _p(keep["faceBnd"])
        v.faceLambda, v.faceArea, v.cellVolume = _p(keep["faceLambda"]), _p(keep["faceArea"]), _p(keep["cellVolume"])
        v.faceNorm, v.faceCenter, v.cellCenter = _vec(keep["faceNorm"], rs), _vec(keep["faceCenter"], rs), _vec(keep["cellCenter"], rs)
        v.faceXpac = _vec(keep.get("faceXpac"), rs)
        v.faceXnac = _vec(keep.get("faceXnac"), rs)
        h = C.c_void_p()
        o = cls._opts(order, precisions, device)
        rc = lib().cupcfd_gpu_mesh_create(C.byref(v), C.byref(o), C.byref(h))
        if return_code:
            return rc, (cls(h) if rc == E_SUCCESS else None)
        check(rc)
        return cls(h)

    @classmethod
    def load(cls, path, order=ORDER_MORTON, precisions=(1 << PREC_F64) | (1 << PREC_F32C), device=-1,
             return_code=False):
        """Rebuild a mesh saved by ``save`` (geometry, regions, split levels)
        with the given layout options."""
        h = C.c_void_p()
        o = cls._opts(order, precisions, device)
        rc = lib().cupcfd_gpu_mesh_load(os.fsencode(path), C.byref(o), C.byref(h))
        if return_code:
            return rc, (cls(h) if rc == E_SUCCESS else None)
        check(rc)
        return cls(h)

    @classmethod
    def load_hdf5(cls, path, order=ORDER_MORTON, precisions=(1 << PREC_F64) | (1 << PREC_F32C), device=-1):
        """A mesh from one of the reference's HDF5 mesh files (MeshHDF5Source)."""
        h = C.c_void_p()
        o = cls._opts(order, precisions, device)
        check(lib().cupcfd_gpu_mesh_load_hdf5(os.fsencode(path), C.byref(o), C.byref(h)))
        return cls(h)

    def save(self, path):
        """Write the mesh's source arrays, regions and split levels to a
        raw-binary mesh file (format in include/cupcfd_gpu.h)."""
        return lib().cupcfd_gpu_mesh_save(self.h, os.fsencode(path))

    def save_hdf5(self, path):
        """Write the mesh in the reference's HDF5 mesh layout (regions as
        boundary region ids; their types are not part of that format)."""
        check(lib().cupcfd_gpu_mesh_save_hdf5(self.h, os.fsencode(path)))

    def close(self):
        if getattr(self, "h", None):
            lib().cupcfd_gpu_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_regions(self, region_type, region_uvw, region_den, bnd_region):
        rt = np.ascontiguousarray(region_type, np.int32)
        uvw = np.ascontiguousarray(region_uvw, np.float64)
        den = np.ascontiguousarray(region_den, np.float64)
        br = np.ascontiguousarray(bnd_region, np.int32)
        return lib().cupcfd_gpu_mesh_set_regions(self.h, len(rt), _p(rt), _p(uvw), _p(den), _p(br), len(br))

    def set_region_split(self, splvl):
        sp = np.ascontiguousarray(splvl, np.float64)
        return lib().cupcfd_gpu_mesh_set_region_split(self.h, len(sp), _p(sp))

    def set_face_rlencos(self, rlencos):
        """getFaceRLencos per face (reference order); None resets to zero."""
        a = None if rlencos is None else np.ascontiguousarray(rlencos, np.float64)
        return lib().cupcfd_gpu_mesh_set_face_rlencos(self.h, _p(a), 0 if a is None else len(a))

    def set_boundary_distance(self, distance):
        """getBoundaryDistance per boundary; None resets to zero."""
        a = None if distance is None else np.ascontiguousarray(distance, np.float64)
        return lib().cupcfd_gpu_mesh_set_boundary_distance(self.h, _p(a), 0 if a is None else len(a))

    def boundary_shear(self, value=None):
        """The boundary shear [nBoundaries, 3] (set first when given)."""
        out = np.empty((self.nBoundaries, 3))
        a = None if value is None else np.ascontiguousarray(value, np.float64)
        check(lib().cupcfd_gpu_mesh_boundary_shear(self.h, _p(a), _p(out), self.nBoundaries))
        return out

    def region_force_tangent(self, n_regions, value=None):
        """The region force tangents [nRegions, 3] (set first when given)."""
        out = np.empty((n_regions, 3))
        a = None if value is None else np.ascontiguousarray(value, np.float64)
        check(lib().cupcfd_gpu_mesh_region_force_tangent(self.h, _p(a), _p(out), n_regions))
        return out

    def check_status(self, stream=None):
        return lib().cupcfd_gpu_mesh_check_status(self.h, _stream(stream))

    def cell_face_csr(self):
        xadj = np.empty(self.nCells + 1, np.int32)
        adj = np.empty(self.nIncidences, np.int32)
        check(lib().cupcfd_gpu_mesh_get_cell_face_csr(self.h, _p(xadj), len(xadj), _p(adj), len(adj)))
        return xadj, adj

    def incidences(self):
        """The kernels' incidence lists per internal cell: (xadj, face << 1 | role, other)."""
        xadj = np.empty(self.nCells + 1, np.int32)
        face = np.empty(self.nIncidences, np.int32)
        other = np.empty(self.nIncidences, np.int32)
        check(lib().cupcfd_gpu_mesh_get_incidences(self.h, _p(xadj), len(xadj), _p(face), _p(other), len(face)))
        return xadj, face, other

    def geometry(self):
        nF, nC = self.nFaces, self.nCells
        g = dict(faceCell1=np.empty(nF, np.int32), faceCell2=np.empty(nF, np.int32), faceBnd=np.empty(nF, np.int32),
                 faceLambda=np.empty(nF), faceArea=np.empty(nF), faceNorm=np.empty((nF, 3)),
                 faceCenter=np.empty((nF, 3)), cellCenter=np.empty((nC, 3)), cellVolume=np.empty(nC))
        check(lib().cupcfd_gpu_mesh_get_geometry(self.h, *[_p(g[k]) for k in (
            "faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
            "cellVolume")]))
        return g

    def numbering(self):
        c = np.empty(self.nCells, np.int32)
        f = np.empty(self.nFaces, np.int32)
        check(lib().cupcfd_gpu_mesh_get_numbering(self.h, _p(c), _p(f)))
        return c, f


# ---------------------------------------------------------------------------
# reference-facing calls (host numpy arrays, reference numbering)
# ---------------------------------------------------------------------------
def GradientPhiGaussDolfyn(mesh, nGradient, phiCell, phiBoundary, dPhidxCell, dPhidxoCell,
                           precision=PREC_F64, sign_mode=SIGN_REFERENCE):
    """Mirror of cupcfd::fvm::GradientPhiGaussDolfyn (GradientKernels.h:48-54).
    dPhidxCell / dPhidxoCell are (n,3) or (n,4) (leading pad slot, the
    EuclideanVector layout) arrays written in place. Returns an eCodes value."""
    rs = phiCell.dtype.itemsize
    v, vo = _vec(dPhidxCell, rs), _vec(dPhidxoCell, rs)
    return lib().cupcfd_gpu_gradient_phi_gauss_dolfyn(
        mesh.h, int(nGradient), _p(phiCell), len(phiCell), _p(phiBoundary), len(phiBoundary),
        v.base, len(dPhidxCell), v.stride, v.offset, vo.base, len(dPhidxoCell), vo.stride, vo.offset,
        rs, precision, sign_mode)


def FluxMassDolfynFaceLoop(mesh, dudx, dvdx, dwdx, dpdx, denCell, denBoundary, uCell, vCell, wCell, massFlux, p, ar,
                           su, rface, small, counters, solveTurbEnergy, solveTurbDiss, solveVisc, solveEnthalpy,
                           teCell, teBoundary, edCell, edBoundary, viseffCell, viseffBoundary, tCell, tBoundary):
    """Mirror of cupcfd::fvm::FluxMassDolfynFaceLoop (MassKernels.h:48-81).
    ``counters`` is an int32 array [icinl, icout, icsym, icwal] updated in
    place; in/out arrays are updated in place. Returns an eCodes value.
    float32 arrays run the reference's T = float instantiation
    (cupcfd_gpu_flux_mass_dolfyn_face_loop_f32), float64 arrays T = double."""
    cnt = counters
    ptrs = [C.c_void_p(cnt.ctypes.data + 4 * k) for k in range(4)]
    f32 = np.asarray(denCell).dtype == np.float32

    def a(x):
        return (_p(x), 0 if x is None else len(x))

    args = [mesh.h]
    for vv in (dudx, dvdx, dwdx, dpdx):
        args += [_vec(vv, 4 if f32 else 8), len(vv)]
    for x in (denCell, denBoundary, uCell, vCell, wCell, massFlux, p, ar, su):
        args += list(a(x))
    args += [_p(rface), len(rface), float(small)] + ptrs
    args += [int(bool(solveTurbEnergy)), int(bool(solveTurbDiss)), int(bool(solveVisc)), int(bool(solveEnthalpy))]
    for x in (teCell, teBoundary, edCell, edBoundary, viseffCell, viseffBoundary, tCell, tBoundary):
        args += list(a(x))
    if f32:
        return lib().cupcfd_gpu_flux_mass_dolfyn_face_loop_f32(*args)
    return lib().cupcfd_gpu_flux_mass_dolfyn_face_loop(*args)


def forward_adjoint(mesh, precision, phi, phiB, den, u, v, w, gface, out=None):
    """Forward + adjoint of the benchmark loss through host buffers.
    Returns a dict of host arrays (grad (n,3), massFlux, phiBar, phiBBar,
    denBar, uBar, vBar, wBar; FP64, or float32 when phi is float32 -- the
    float-array call, cupcfd_gpu_forward_adjoint_f32) and loss (FP64)."""
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    f32 = np.asarray(phi).dtype == np.float32
    dt = np.float32 if f32 else np.float64
    if out is None:
        out = dict(grad=np.empty((nC, 3), dt), massFlux=np.empty(nF, dt), phiBar=np.empty(nC, dt),
                   phiBBar=np.empty(nB, dt), denBar=np.empty(nC, dt), uBar=np.empty(nC, dt), vBar=np.empty(nC, dt),
                   wBar=np.empty(nC, dt), loss=np.empty(1))
    fn = lib().cupcfd_gpu_forward_adjoint_f32 if f32 else lib().cupcfd_gpu_forward_adjoint
    check(fn(mesh.h, precision, _p(phi), _p(phiB), _p(den), _p(u), _p(v), _p(w), _p(gface),
             *[_p(out[k]) for k in ("grad", "massFlux", "phiBar", "phiBBar", "denBar", "uBar", "vBar", "wBar", "loss")]))
    return out


# ---------------------------------------------------------------------------
# device-resident calls (torch CUDA tensors, internal numbering)
# ---------------------------------------------------------------------------
def _es(prec):
    return 8 if prec == PREC_F64 else 4


def permute_cells(mesh, to_internal, src, dst, ncomp=1, stream=None):
    check(lib().cupcfd_gpu_dev_permute_cells(mesh.h, int(bool(to_internal)), ncomp, _p(src), src.element_size(), 0,
                                             _p(dst), dst.element_size(), 0, _stream(stream)))


def permute_faces(mesh, to_internal, src, dst, stream=None):
    check(lib().cupcfd_gpu_dev_permute_faces(mesh.h, int(bool(to_internal)), _p(src), src.element_size(), _p(dst),
                                             dst.element_size(), _stream(stream)))


def dev_gradient(mesh, precision, phi, phiB, grad, grad_o=None, nGradient=1, sign_mode=SIGN_REFERENCE, stream=None):
    check(lib().cupcfd_gpu_dev_gradient(mesh.h, precision, nGradient, sign_mode, _p(phi), _p(phiB), _p(grad),
                                        _p(grad_o), _stream(stream)))


def dev_mass_plain(mesh, precision, state, mflux, stream=None):
    check(lib().cupcfd_gpu_dev_mass_plain(mesh.h, precision, _p(state), _p(mflux), _stream(stream)))


def dev_gradient_adjoint(mesh, precision, gbar, phiBar, phiBBar, sign_mode=SIGN_REFERENCE, stream=None):
    check(lib().cupcfd_gpu_dev_gradient_adjoint(mesh.h, precision, sign_mode, _p(gbar), _p(phiBar), _p(phiBBar),
                                                _stream(stream)))


def dev_mass_plain_adjoint(mesh, precision, state, mbar, stateBar, stream=None):
    check(lib().cupcfd_gpu_dev_mass_plain_adjoint(mesh.h, precision, _p(state), _p(mbar), _p(stateBar), _stream(stream)))


def dev_forward(mesh, precision, phi, phiB, state, grad, mflux, gface=None, loss=None, stream=None):
    check(lib().cupcfd_gpu_dev_forward(mesh.h, precision, _p(phi), _p(phiB), _p(state), _p(gface), _p(grad), _p(mflux),
                                       _p(loss), _stream(stream)))


def dev_forward_noalloc(mesh, precision, phi, phiB, state, grad, mflux, gface=None, loss=None, stream=None):
    """cupcfd_gpu_dev_forward without allocation; returns the status code."""
    return lib().cupcfd_gpu_dev_forward_noalloc(mesh.h, precision, _p(phi), _p(phiB), _p(state), _p(gface), _p(grad),
                                                _p(mflux), _p(loss), _stream(stream))


def dev_adjoint(mesh, precision, grad, state, gface, phiBar, phiBBar, stateBar, stream=None):
    check(lib().cupcfd_gpu_dev_adjoint(mesh.h, precision, _p(grad), _p(state), _p(gface), _p(phiBar), _p(phiBBar),
                                       _p(stateBar), _stream(stream)))


def dev_forward_adjoint(mesh, precision, phi, phiB, state, gface, grad, mflux, phiBar, phiBBar, stateBar, loss=None,
                        stream=None):
    check(lib().cupcfd_gpu_dev_forward_adjoint(mesh.h, precision, _p(phi), _p(phiB), _p(state), _p(gface), _p(grad),
                                               _p(mflux), _p(phiBar), _p(phiBBar), _p(stateBar), _p(loss),
                                               _stream(stream)))


def error_norms(a, b, floor=0.0, stream=None):
    """FP64 norms of device tensors a vs b: dict(max_abs, max_ref, rms_rel, max_rel_floor)."""
    out = (C.c_double * 5)()
    check(lib().cupcfd_gpu_dev_error_norms(_p(a), a.element_size(), _p(b), b.element_size(), a.numel(), float(floor),
                                           out, _stream(stream)))
    mx, mb, s2, b2, mr = list(out)
    return dict(max_abs=mx, max_ref=mb, max_rel_norm=mx / mb if mb else 0.0,
                rms_rel=(s2 / b2) ** 0.5 if b2 else 0.0, max_rel_floor=mr)


# ---------------------------------------------------------------------------
# boundary / region loops of the mass-flux step (MassKernels.ipp:311-554).
# Host arrays in the reference's numbering; in/out arrays are updated in
# place, scalar outputs returned. Each returns (status, outputs...). float64
# arrays run the reference's T = double instantiation, float32 arrays its
# T = float one (the _f32 calls); all arrays of a call share one type.
# ---------------------------------------------------------------------------
def _bnd_kind(first, *rest):
    dt = np.asarray(first).dtype
    assert dt in (np.float64, np.float32), dt
    for a in (first,) + rest:
        assert a.dtype == dt and a.flags["C_CONTIGUOUS"], "arrays must share one real type and be contiguous"
    f32 = dt == np.float32
    return f32, (C.c_float if f32 else C.c_double), ("_f32" if f32 else "")


def _bnd_fn(name, suffix):
    return getattr(lib(), "cupcfd_gpu_flux_mass_dolfyn_" + name + suffix)


def FluxMassDolfynBoundaryLoop1(mesh, massFlux):
    f32, S, sfx = _bnd_kind(massFlux)
    out = S(np.nan)
    rc = _bnd_fn("boundary_loop1", sfx)(mesh.h, _p(massFlux), len(massFlux), C.byref(out))
    return rc, out.value


def FluxMassDolfynBoundaryLoop2(mesh, massFlux, flowRegion):
    f32, S, sfx = _bnd_kind(massFlux, flowRegion)
    out = S(np.nan)
    rc = _bnd_fn("boundary_loop2", sfx)(mesh.h, _p(massFlux), len(massFlux), _p(flowRegion), len(flowRegion),
                                        C.byref(out))
    return rc, out.value


def FluxMassDolfynBoundaryLoop3(mesh, flowin, f32=False):
    """f32: the T = float instantiation (flowin rounded to float)."""
    S, sfx = (C.c_float, "_f32") if f32 else (C.c_double, "")
    out = S(np.nan)
    rc = _bnd_fn("boundary_loop3", sfx)(mesh.h, float(flowin), C.byref(out))
    return rc, out.value


def FluxMassDolfynBoundaryLoop4(mesh, massFlux, uB, vB, wB, denB, ratearea):
    f32, S, sfx = _bnd_kind(massFlux, uB, vB, wB, denB)
    out = S(np.nan)
    rc = _bnd_fn("boundary_loop4", sfx)(
        mesh.h, _p(massFlux), len(massFlux), _p(uB), len(uB), _p(vB), len(vB), _p(wB), len(wB),
        _p(denB), len(denB), float(ratearea), C.byref(out))
    return rc, out.value


def FluxMassDolfynBoundaryLoop5(mesh, massFlux, su, uB, vB, wB, fact, solve, flowFact, flowout2):
    f32, S, sfx = _bnd_kind(massFlux, su, uB, vB, wB, flowFact)
    out = S(flowout2)
    rc = _bnd_fn("boundary_loop5", sfx)(
        mesh.h, _p(massFlux), len(massFlux), _p(su), len(su), _p(uB), len(uB), _p(vB), len(vB),
        _p(wB), len(wB), float(fact), *[int(bool(x)) for x in solve], _p(flowFact), len(flowFact),
        C.byref(out))
    return rc, out.value


def FluxMassDolfynRegionLoop(mesh, flowFact, flowRegion, flowIn):
    f32, S, sfx = _bnd_kind(flowFact, flowRegion)
    return _bnd_fn("region_loop", sfx)(mesh.h, _p(flowFact), len(flowFact), _p(flowRegion), len(flowRegion),
                                       float(flowIn))


def dev_boundary_loop1(mesh, massFlux, flowin, stream=None):
    check(lib().cupcfd_gpu_dev_boundary_loop1(mesh.h, _p(massFlux), _p(flowin), _stream(stream)))


def dev_boundary_loop2(mesh, massFlux, flowRegion, flowout, stream=None):
    check(lib().cupcfd_gpu_dev_boundary_loop2(mesh.h, _p(massFlux), _p(flowRegion), _p(flowout), _stream(stream)))


def dev_boundary_loop3(mesh, flowin, ratearea, stream=None):
    check(lib().cupcfd_gpu_dev_boundary_loop3(mesh.h, _p(flowin), _p(ratearea), _stream(stream)))


def dev_boundary_loop4(mesh, massFlux, uB, vB, wB, denB, ratearea, flowout, stream=None):
    check(lib().cupcfd_gpu_dev_boundary_loop4(mesh.h, _p(massFlux), _p(uB), _p(vB), _p(wB), _p(denB), _p(ratearea),
                                              _p(flowout), _stream(stream)))


def dev_boundary_loop5(mesh, massFlux, su, uB, vB, wB, fact, solve, flowFact, flowout2, stream=None):
    check(lib().cupcfd_gpu_dev_boundary_loop5(mesh.h, _p(massFlux), _p(su), _p(uB), _p(vB), _p(wB), float(fact),
                                              *[int(bool(x)) for x in solve], _p(flowFact), _p(flowout2),
                                              _stream(stream)))


def dev_region_loop(mesh, flowFact, flowRegion, flowIn, stream=None):
    check(lib().cupcfd_gpu_dev_region_loop(mesh.h, _p(flowFact), _p(flowRegion), _p(flowIn), _stream(stream)))


# ---------------------------------------------------------------------------
# momentum face loop (UVWKernels.h:45-92)
# ---------------------------------------------------------------------------
def FluxUVWDolfynFaceLoop1(mesh, gammaBlend, small, uCell, vCell, wCell, uBoundary, vBoundary, wBoundary, visEffCell,
                           visEffBoundary, massFlux, dudx, dvdx, dwdx, rFace, su, sv, sw, au, av, aw):
    """Mirror of cupcfd::fvm::FluxUVWDolfynFaceLoop1 (UVWKernels.h:45-67) on
    host arrays in the reference's numbering; in/out arrays (boundary
    velocities, massFlux, rFace, su..aw) are updated in place; dudx/dvdx/dwdx
    are (n,3) or (n,4) (leading pad slot). float32 arrays run the reference's
    T = float instantiation, float64 arrays T = double. Returns an eCodes
    value."""
    f32 = np.asarray(uCell).dtype == np.float32

    def a(x):
        return [_p(x), 0 if x is None else len(x)]
    args = [mesh.h, float(gammaBlend), float(small)]
    for x in (uCell, vCell, wCell, uBoundary, vBoundary, wBoundary, visEffCell, visEffBoundary, massFlux):
        args += a(x)
    for vv in (dudx, dvdx, dwdx):
        args += [_vec(vv, 4 if f32 else 8), len(vv)]
    args += a(rFace)
    for x in (su, sv, sw, au, av, aw):
        args += a(x)
    if f32:
        return lib().cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32(*args)
    return lib().cupcfd_gpu_flux_uvw_dolfyn_face_loop1(*args)


def FluxUVWDolfynRegionLoop1(mesh):
    return lib().cupcfd_gpu_flux_uvw_dolfyn_region_loop1(mesh.h)


def FluxUVWDolfynBndsLoop1(mesh):
    return lib().cupcfd_gpu_flux_uvw_dolfyn_bnds_loop1(mesh.h)


def dev_uvw_face_loop1(mesh, gammaBlend, small, u, v, w, uB, vB, wB, visC, visB, massFlux, grads, rFace, su, sv, sw,
                       au, av, aw, stream=None):
    """Device-resident momentum face loop: torch CUDA FP64 tensors in the
    mesh's internal numbering; grads is (9, ldg) (dudx x,y,z, dvdx, dwdx)."""
    check(lib().cupcfd_gpu_dev_uvw_face_loop1(
        mesh.h, float(gammaBlend), float(small), _p(u), _p(v), _p(w), _p(uB), _p(vB), _p(wB), _p(visC), _p(visB),
        _p(massFlux), _p(grads), int(grads.stride(0)), _p(rFace), _p(su), _p(sv), _p(sw), _p(au), _p(av), _p(aw),
        _stream(stream)))


def dev_uvw_region_loop1(mesh, stream=None):
    check(lib().cupcfd_gpu_dev_uvw_region_loop1(mesh.h, _stream(stream)))


def dev_uvw_bnds_loop1(mesh, stream=None):
    check(lib().cupcfd_gpu_dev_uvw_bnds_loop1(mesh.h, _stream(stream)))


# ---------------------------------------------------------------------------
# the reference's HDF5 mesh files (MeshHDF5Source)
# ---------------------------------------------------------------------------
def hdf5_mesh_read(path):
    """Host arrays of an HDF5 mesh file in the reference's numbering, as a
    dict in the oracle's mesh format (plus bndDistance), or raises
    CupcfdError with the library's code."""
    n = [C.c_int32() for _ in range(4)]
    check(lib().cupcfd_gpu_hdf5_mesh_counts(os.fsencode(path), *[C.byref(x) for x in n]))
    nC, nF, nB, nR = (x.value for x in n)
    m = dict(nCells=nC, nFaces=nF, nBnd=nB, nRegions=max(nR, 1),
             faceCell1=np.empty(nF, np.int32), faceCell2=np.empty(nF, np.int32), faceBnd=np.empty(nF, np.int32),
             faceLambda=np.empty(nF), faceArea=np.empty(nF), faceNorm=np.empty((nF, 3)), faceCenter=np.empty((nF, 3)),
             cellCenter=np.empty((nC, 3)), cellVolume=np.empty(nC), bndRegion=np.empty(nB, np.int32),
             bndDistance=np.empty(nB))
    check(lib().cupcfd_gpu_hdf5_mesh_read(os.fsencode(path), nC, nF, nB, *[_p(m[k]) for k in (
        "faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
        "cellVolume", "bndRegion", "bndDistance")]))
    return m


def hdf5_mesh_write(path, m, bnd_distance=None):
    """Write mesh dict ``m`` (the oracle's format: 0-based ids, faceCell2 -1
    and faceBnd the boundary id on boundary faces; bndRegion optional) as an
    HDF5 mesh file in the reference's layout."""
    nC, nF, nB = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"])
    a = dict(c1=np.ascontiguousarray(m["faceCell1"], np.int32), c2=np.ascontiguousarray(m["faceCell2"], np.int32),
             fb=np.ascontiguousarray(m["faceBnd"], np.int32), lam=np.ascontiguousarray(m["faceLambda"], np.float64),
             area=np.ascontiguousarray(m["faceArea"], np.float64),
             S=np.ascontiguousarray(m["faceNorm"], np.float64).reshape(-1),
             X=np.ascontiguousarray(m["faceCenter"], np.float64).reshape(-1),
             cc=np.ascontiguousarray(m["cellCenter"], np.float64).reshape(-1),
             vol=np.ascontiguousarray(m["cellVolume"], np.float64))
    breg = None if m.get("bndRegion") is None else np.ascontiguousarray(m["bndRegion"], np.int32)
    dist = None if bnd_distance is None else np.ascontiguousarray(bnd_distance, np.float64)
    check(lib().cupcfd_gpu_hdf5_mesh_write(os.fsencode(path), nC, nF, nB, int(m.get("nRegions", 1)),
                                           *[_p(a[k]) for k in ("c1", "c2", "fb", "lam", "area", "S", "X", "cc", "vol")],
                                           _p(breg), _p(dist)))


def hdf5_dataset(path, name):
    """Any numeric dataset of an HDF5 mesh file, as float64 with its shape
    (integers exact)."""
    nd, isr = C.c_int32(), C.c_int32()
    dims = (C.c_int64 * 4)()
    check(lib().cupcfd_gpu_hdf5_dataset_shape(os.fsencode(path), name.encode(), C.byref(nd), dims, C.byref(isr)))
    shape = tuple(int(dims[i]) for i in range(nd.value))
    out = np.empty(shape, np.float64)
    check(lib().cupcfd_gpu_hdf5_dataset_read(os.fsencode(path), name.encode(), _p(out), out.size))
    return out
