"""ctypes wrapper of the CPU oracle and of the reference harness libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline / reference legs as the checker, never by the library.

``liboracle.so`` is the C restatement of the reference's serial algorithm
(oracle.c). ``_ref/libref_*.so`` are the reference's own sources compiled by the
oracle Makefile (host pattern builders, the Q4 serial host assembly and, on a
GPU, the reference's device element-stiffness functions).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def build() -> None:
    """Compile liboracle.so (and the reference harness if the sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.oracle_ke_q4.argtypes = [vp, vp, f64, f64, f64, vp]
        L.oracle_ke_t3.argtypes = [vp, vp, f64, f64, f64, vp]
        L.oracle_ke_hex20.argtypes = [vp, vp, vp, f64, f64, vp]
        L.oracle_pattern.argtypes = [C.c_int, i32, i32, i32, vp, vp, vp, vp, i64]
        L.oracle_pattern.restype = i64
        L.oracle_assemble.argtypes = [C.c_int, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp,
                                      f64, f64, f64, vp, vp, vp]
        L.oracle_assemble.restype = i64
        L.oracle_assemble_rows.argtypes = [C.c_int, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp,
                                           f64, f64, f64, vp, vp, vp, vp]
        L.oracle_assemble_rows.restype = i64
        L.oracle_precision.argtypes = [i64, vp, vp, vp]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------
# oracle
# ---------------------------------------------------------------------------

def ke_q4(x, y, E=1.0, nu=0.3, t=1.0) -> np.ndarray:
    x, y = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
    ke = np.zeros(64)
    lib().oracle_ke_q4(_ptr(x), _ptr(y), E, nu, t, _ptr(ke))
    return ke.reshape(8, 8)


def ke_t3(x, y, E=1.0, nu=0.3, t=1.0) -> np.ndarray:
    x, y = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
    ke = np.zeros(36)
    lib().oracle_ke_t3(_ptr(x), _ptr(y), E, nu, t, _ptr(ke))
    return ke.reshape(6, 6)


def ke_hex20(x, y, z, E=1.0, nu=0.3) -> np.ndarray:
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    ke = np.zeros(3600)
    lib().oracle_ke_hex20(_ptr(x), _ptr(y), _ptr(z), E, nu, _ptr(ke))
    return ke.reshape(60, 60)


def pattern(mesh):
    """Sorted-unique CSR pattern (row_ptr, col_idx) of a meshgen.Mesh."""
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    types = None if mesh.types is None else np.ascontiguousarray(mesh.types, np.uint8)
    row_ptr = np.zeros(mesh.num_dofs + 1, np.int32)
    nnz = lib().oracle_pattern(mesh.kind, mesh.num_nodes, mesh.num_elems, mesh.stride,
                               _ptr(conn), _ptr(types), _ptr(row_ptr), None, 0)
    if nnz < 0:
        raise ValueError(f"oracle_pattern failed ({nnz})")
    col = np.zeros(nnz, np.int32)
    nnz2 = lib().oracle_pattern(mesh.kind, mesh.num_nodes, mesh.num_elems, mesh.stride,
                                _ptr(conn), _ptr(types), _ptr(row_ptr), _ptr(col), nnz)
    assert nnz2 == nnz
    return row_ptr, col


def assemble(mesh, row_ptr=None, col_idx=None, E0=None, nu0=None, thickness=None,
             uniform_material=False):
    """Serial FP64 assembly; returns (row_ptr, col_idx, values)."""
    if row_ptr is None:
        row_ptr, col_idx = pattern(mesh)
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    types = None if mesh.types is None else np.ascontiguousarray(mesh.types, np.uint8)
    z = None if mesh.z is None else np.ascontiguousarray(mesh.z, np.float64)
    E = None if (uniform_material or mesh.E is None) else np.ascontiguousarray(mesh.E, np.float64)
    nu = None if (uniform_material or mesh.nu is None) else np.ascontiguousarray(mesh.nu, np.float64)
    vals = np.zeros(col_idx.shape[0], np.float64)
    r = lib().oracle_assemble(mesh.kind, mesh.num_nodes, mesh.num_elems, mesh.stride,
                              _ptr(conn), _ptr(types), _ptr(np.ascontiguousarray(mesh.x)),
                              _ptr(np.ascontiguousarray(mesh.y)), _ptr(z), _ptr(E), _ptr(nu),
                              mesh.E0 if E0 is None else E0, mesh.nu0 if nu0 is None else nu0,
                              mesh.thickness if thickness is None else thickness,
                              _ptr(row_ptr), _ptr(col_idx), _ptr(vals))
    if r < 0:
        raise ValueError("oracle_assemble: entry missing from pattern")
    return row_ptr, col_idx, vals


def assemble_rows(mesh, row_ptr, col_idx, row_nodes):
    """Serial FP64 assembly of the dof rows of `row_nodes` only, into the given
    pattern; returns a values array whose other rows are zero."""
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    types = None if mesh.types is None else np.ascontiguousarray(mesh.types, np.uint8)
    z = None if mesh.z is None else np.ascontiguousarray(mesh.z, np.float64)
    E = None if mesh.E is None else np.ascontiguousarray(mesh.E, np.float64)
    nu = None if mesh.nu is None else np.ascontiguousarray(mesh.nu, np.float64)
    mask = np.zeros(mesh.num_nodes, np.uint8)
    mask[np.asarray(row_nodes, np.int64)] = 1
    row_ptr = np.ascontiguousarray(row_ptr, np.int32)
    col_idx = np.ascontiguousarray(col_idx, np.int32)
    vals = np.zeros(col_idx.shape[0], np.float64)
    r = lib().oracle_assemble_rows(mesh.kind, mesh.num_nodes, mesh.num_elems, mesh.stride,
                                   _ptr(conn), _ptr(types), _ptr(np.ascontiguousarray(mesh.x)),
                                   _ptr(np.ascontiguousarray(mesh.y)), _ptr(z), _ptr(E), _ptr(nu),
                                   mesh.E0, mesh.nu0, mesh.thickness, _ptr(row_ptr), _ptr(col_idx),
                                   _ptr(mask), _ptr(vals))
    if r < 0:
        raise ValueError("oracle_assemble_rows: entry missing from pattern")
    return vals


def precision(ref: np.ndarray, test: np.ndarray) -> dict:
    out = np.zeros(6)
    ref = np.ascontiguousarray(ref, np.float64)
    test = np.ascontiguousarray(test, np.float64)
    lib().oracle_precision(ref.shape[0], _ptr(ref), _ptr(test), _ptr(out))
    keys = ["max_abs", "max_rel", "mean_abs", "mean_rel", "frobenius_rel", "count_gt_1e-10"]
    return dict(zip(keys, out.tolist()))


# ---------------------------------------------------------------------------
# reference harness (built from the reference sources)
# ---------------------------------------------------------------------------

_ref = {}


def ref_available(name: str = "q4a") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{name}.so"))


def ref_lib(name: str):
    if name not in _ref:
        L = C.CDLL(os.path.join(REF_DIR, f"libref_{name}.so"))
        vp, i64, f64 = C.c_void_p, C.c_int64, C.c_double
        if name == "q4a":
            L.ref_q4a_material.argtypes = [vp, vp, vp]
            L.ref_q4a_generate_mesh.argtypes = [C.c_int, C.c_int, f64, f64, vp, vp, vp]
            L.ref_q4a_build_csr.argtypes = [C.c_int, C.c_int, vp, vp, vp, i64]
            L.ref_q4a_build_csr.restype = i64
            L.ref_q4a_host_assemble.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
        elif name in ("t3", "mix"):
            f = getattr(L, f"ref_{name}_build_csr")
            f.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, i64]
            f.restype = i64
            g = getattr(L, f"ref_{name}_gpu_element_ke")
            g.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, f64, f64, f64, vp]
            g.restype = C.c_int
        elif name == "h20":
            L.ref_h20_generate_mesh.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]
            L.ref_h20_build_csr.argtypes = [C.c_int, C.c_int, vp, vp, vp, i64]
            L.ref_h20_build_csr.restype = i64
            L.ref_h20_gpu_element_ke.argtypes = [C.c_int, vp, vp, vp, vp, f64, f64, vp]
            L.ref_h20_gpu_element_ke.restype = C.c_int
        _ref[name] = L
    return _ref[name]


def ref_q4a_material():
    E, nu, t = C.c_double(), C.c_double(), C.c_double()
    ref_lib("q4a").ref_q4a_material(C.byref(E), C.byref(nu), C.byref(t))
    return E.value, nu.value, t.value


def ref_pattern(mesh):
    """CSR pattern from the reference's own host builder for this mesh kind."""
    from meshgen import Q4, T3, MIXED_2D, HEX20  # noqa: F401  (kind constants)
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    types = None if mesh.types is None else np.ascontiguousarray(mesh.types, np.uint8)
    rp = np.zeros(mesh.num_dofs + 1, np.int32)

    def call(col, cap):
        if mesh.kind == 0:
            return ref_lib("q4a").ref_q4a_build_csr(mesh.num_nodes, mesh.num_elems, _ptr(conn),
                                                    _ptr(rp), _ptr(col), cap)
        if mesh.kind == 1:
            return ref_lib("t3").ref_t3_build_csr(mesh.num_nodes, mesh.num_elems, mesh.stride,
                                                  _ptr(conn), None, _ptr(rp), _ptr(col), cap)
        if mesh.kind == 3:
            return ref_lib("mix").ref_mix_build_csr(mesh.num_nodes, mesh.num_elems, mesh.stride,
                                                    _ptr(conn), _ptr(types), _ptr(rp), _ptr(col), cap)
        return ref_lib("h20").ref_h20_build_csr(mesh.num_nodes, mesh.num_elems, _ptr(conn),
                                                _ptr(rp), _ptr(col), cap)

    nnz = call(None, 0)
    col = np.zeros(nnz, np.int32)
    call(col, nnz)
    return rp, col


def ref_q4a_host_assemble(mesh, row_ptr, col_idx) -> np.ndarray:
    """The reference's serial host assembly (reference material constants)."""
    vals = np.zeros(col_idx.shape[0])
    ref_lib("q4a").ref_q4a_host_assemble(
        mesh.num_nodes, mesh.num_elems, _ptr(np.ascontiguousarray(mesh.conn, np.int32)),
        _ptr(np.ascontiguousarray(mesh.x)), _ptr(np.ascontiguousarray(mesh.y)),
        _ptr(np.ascontiguousarray(row_ptr)), _ptr(np.ascontiguousarray(col_idx)), _ptr(vals))
    return vals


def ref_q4a_generate_mesh(nx: int, ny: int, lx: float = 1.0, ly: float = 1.0):
    conn = np.zeros(nx * ny * 4, np.int32)
    x = np.zeros((nx + 1) * (ny + 1))
    y = np.zeros_like(x)
    ref_lib("q4a").ref_q4a_generate_mesh(nx, ny, lx, ly, _ptr(conn), _ptr(x), _ptr(y))
    return conn.reshape(-1, 4), x, y


def ref_gpu_element_ke(mesh, E: float, nu: float, t: float = 1.0) -> np.ndarray:
    """Per-element Ke from the reference's device functions (needs a GPU).
    2-D: [num_elems, 8, 8] (T3 in the top-left 6x6). Hex20: [num_elems, 60, 60] float32."""
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    if mesh.kind == 2:
        out = np.zeros(mesh.num_elems * 3600, np.float32)
        rc = ref_lib("h20").ref_h20_gpu_element_ke(
            mesh.num_elems, _ptr(conn), _ptr(np.ascontiguousarray(mesh.x)),
            _ptr(np.ascontiguousarray(mesh.y)), _ptr(np.ascontiguousarray(mesh.z)), E, nu, _ptr(out))
        if rc:
            raise RuntimeError(f"reference Hex20 Ke harness failed: CUDA error {rc}")
        return out.reshape(-1, 60, 60)
    name = "mix" if mesh.kind == 3 else "t3"
    types = None if mesh.types is None else np.ascontiguousarray(mesh.types, np.uint8)
    out = np.zeros(mesh.num_elems * 64)
    rc = getattr(ref_lib(name), f"ref_{name}_gpu_element_ke")(
        mesh.num_elems, mesh.stride, _ptr(conn), _ptr(types), _ptr(np.ascontiguousarray(mesh.x)),
        _ptr(np.ascontiguousarray(mesh.y)), E, nu, t, _ptr(out))
    if rc:
        raise RuntimeError(f"reference {name} Ke harness failed: CUDA error {rc}")
    return out.reshape(-1, 8, 8)
