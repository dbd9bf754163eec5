"""Python binding of the assembler's C ABI (include/fem_alls.h) over ctypes.

The library is ``lib/libfem_alls.so`` (built by build.py from csrc/); this
module only marshals arguments. Device memory for meshes and CSR outputs comes
from torch tensors on a CUDA device (torch is used as an allocator and stream
provider, nothing else). Every call goes through the C ABI; there is no Python
or CPU fallback: if the library or a GPU is missing the calls raise.

Names mirror the reference's host-side assembly steps:
``alls_scatter`` ~ assembleGlobalStiffnessKernelALLS
(ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:394-468), ``alls_consolidate`` ~
buildCSRStructure + convertALLStoCSRKernel (Q4A:605-645, Q4A:471-501), and
``assemble`` the whole sequence of the reference driver (Q4A:794-827).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# FEM_ALLS_LIB selects another build of the library (same C ABI).
LIB_PATH = os.environ.get("FEM_ALLS_LIB") or os.path.join(HERE, "lib", "libfem_alls.so")

FEM_OK = 0
STATUS_NAMES = {0: "FEM_OK", 1: "FEM_ERR_BAD_ARG", 2: "FEM_ERR_BAD_MESH", 3: "FEM_ERR_POOL_OVERFLOW",
                4: "FEM_ERR_DETJ", 5: "FEM_ERR_CUDA", 6: "FEM_ERR_CAPACITY", 7: "FEM_ERR_WORKSPACE",
                8: "FEM_ERR_TIMEOUT", 9: "FEM_ERR_RANGE", 10: "FEM_ERR_INTERNAL"}
globals().update({v: k for k, v in STATUS_NAMES.items()})

# C ABI exports (kept in sync with include/fem_alls.h by tests/test_abi.py).
EXPORTS = ["fem_alls_workspace_size", "fem_alls_scatter", "fem_alls_consolidate", "fem_alls_read_info",
           "fem_assemble", "fem_assemble_async", "fem_context_create", "fem_context_destroy",
           "fem_assemble_host", "fem_status_string", "fem_last_cuda_error", "fem_abi_version",
           "fem_assemble_static", "fem_colour_workspace_size", "fem_colour_prepare", "fem_colour_assemble",
           "fem_colour_read_info", "fem_element_stiffness_size", "fem_element_stiffness",
           "fem_scatter_map_size", "fem_scatter_map_build", "fem_reassemble_values", "fem_scatter_map_read_info",
           "fem_batched_workspace_size", "fem_assemble_batched", "fem_alls_consolidate_bsr",
           "fem_autotune_workspace_size", "fem_autotune", "fem_autotune_batched", "fem_alls_consolidate_upper",
           "fem_assemble_body_force", "fem_apply_dirichlet"]
STATIC_WORKSPACE_BYTES = 32 << 20  # FEM_STATIC_WORKSPACE_BYTES


class FemMesh(C.Structure):
    _fields_ = [("kind", C.c_int32), ("num_nodes", C.c_int32), ("num_elems", C.c_int32),
                ("conn_stride", C.c_int32), ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("conn", C.c_void_p), ("elem_type", C.c_void_p), ("E", C.c_void_p), ("nu", C.c_void_p),
                ("E0", C.c_double), ("nu0", C.c_double), ("thickness", C.c_double)]


class FemOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("first_slots", C.c_int32), ("chunk_slots", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("pool_factor", C.c_double), ("wait_limit_us", C.c_int32),
                ("reserved", C.c_int32)]


class FemCsr(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("pad", C.c_int32), ("nnz", C.c_int64), ("capacity", C.c_int64),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("values", C.c_void_p)]


class FemInfo(C.Structure):
    _fields_ = [("nnz", C.c_int64), ("list_entries", C.c_int64), ("status_bits", C.c_int32),
                ("overflow_chunks", C.c_int32), ("pool_chunks", C.c_int32), ("max_row_entries", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FemError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        extra = ""
        if status == 5:
            extra = f" (cudaError {load().fem_last_cuda_error()})"
        super().__init__(f"{what}: {name}{extra}")


_lib = None


def load() -> C.CDLL:
    """Load lib/libfem_alls.so (building it first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import build as _b  # noqa: WPS433 (local build script)
            _b.build()
        L = C.CDLL(LIB_PATH)
        vp, p = C.c_void_p, C.POINTER
        L.fem_alls_workspace_size.argtypes = [p(FemMesh), p(FemOpts), p(C.c_size_t)]
        L.fem_alls_scatter.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, vp]
        L.fem_alls_consolidate.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, vp, vp, vp, C.c_int64, vp]
        L.fem_alls_read_info.argtypes = [vp, p(FemInfo), vp]
        L.fem_assemble.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, p(FemCsr), vp]
        L.fem_assemble_async.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, p(FemCsr), vp]
        L.fem_context_create.argtypes = [p(vp)]
        L.fem_context_destroy.argtypes = [vp]
        L.fem_context_destroy.restype = None
        L.fem_assemble_host.argtypes = [vp, p(FemMesh), p(FemOpts), p(FemCsr), vp]
        L.fem_colour_workspace_size.argtypes = [p(FemMesh), p(C.c_size_t)]
        L.fem_colour_prepare.argtypes = [p(FemMesh), vp, C.c_size_t, p(C.c_int32), vp, vp]
        L.fem_colour_assemble.argtypes = [p(FemMesh), vp, C.c_size_t, C.c_int32, vp, vp, vp, C.c_int64, vp]
        L.fem_colour_read_info.argtypes = [vp, p(C.c_int32), vp]
        L.fem_element_stiffness_size.argtypes = [p(FemMesh), p(C.c_int64)]
        L.fem_element_stiffness.argtypes = [p(FemMesh), p(FemOpts), vp, vp, vp]
        L.fem_scatter_map_size.argtypes = [p(FemMesh), p(C.c_size_t)]
        L.fem_scatter_map_build.argtypes = [p(FemMesh), vp, vp, vp, C.c_size_t, vp]
        L.fem_reassemble_values.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, vp, vp, C.c_int64, vp]
        L.fem_scatter_map_read_info.argtypes = [vp, vp]
        L.fem_batched_workspace_size.argtypes = [p(FemMesh), C.c_int32, p(FemOpts), C.c_int32, p(C.c_size_t)]
        L.fem_assemble_batched.argtypes = [p(FemMesh), C.c_int32, p(FemOpts), C.c_int32, vp, C.c_size_t, p(FemCsr),
                                           vp, vp, vp]
        L.fem_alls_consolidate_bsr.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, vp, vp, vp, C.c_int64, vp]
        L.fem_alls_consolidate_upper.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, vp, vp, vp, C.c_int64, vp]
        L.fem_assemble_body_force.argtypes = [p(FemMesh), vp, vp, vp, vp, vp]
        L.fem_apply_dirichlet.argtypes = [C.c_int32, vp, vp, vp, vp, vp, vp, vp]
        L.fem_autotune_workspace_size.argtypes = [p(FemMesh), p(FemOpts), p(C.c_size_t)]
        L.fem_autotune.argtypes = [p(FemMesh), p(FemOpts), vp, C.c_size_t, p(FemCsr), C.c_int32, p(FemOpts),
                                   p(C.c_float), vp]
        L.fem_autotune_batched.argtypes = [p(FemMesh), C.c_int32, p(FemOpts), vp, C.c_size_t, p(FemCsr), vp,
                                           C.c_int32, p(C.c_int32), p(C.c_float), vp]
        L.fem_status_string.argtypes = [C.c_int32]
        L.fem_status_string.restype = C.c_char_p
        for f in EXPORTS:
            if f not in ("fem_context_destroy", "fem_status_string"):
                getattr(L, f).restype = C.c_int32
        _lib = L
    return _lib


FEM_PREC_FP64, FEM_PREC_TC_F16X3, FEM_PREC_FP64_SIMT, FEM_PREC_FP32 = 0, 1, 2, 3


def opts(first_slots: int = 0, chunk_slots: int = 0, pool_factor: float = 0.0, precision: int = 0,
         ctas_per_sm: int = 0, wait_limit_us: int = 0) -> FemOpts:
    return FemOpts(precision, first_slots, chunk_slots, ctas_per_sm, pool_factor, wait_limit_us, 0)


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def fem_mesh_struct(mesh, arrays: dict) -> FemMesh:
    """FemMesh over the buffers in `arrays` (device tensors or host numpy arrays)."""
    return FemMesh(mesh.kind, mesh.num_nodes, mesh.num_elems, mesh.stride, _ptr(arrays["x"]), _ptr(arrays["y"]),
                   _ptr(arrays.get("z")), _ptr(arrays["conn"]), _ptr(arrays.get("types")), _ptr(arrays.get("E")),
                   _ptr(arrays.get("nu")), float(mesh.E0), float(mesh.nu0), float(mesh.thickness))


def host_arrays(mesh) -> dict:
    a = {"x": np.ascontiguousarray(mesh.x, np.float64), "y": np.ascontiguousarray(mesh.y, np.float64),
         "conn": np.ascontiguousarray(mesh.conn, np.int32)}
    if mesh.z is not None:
        a["z"] = np.ascontiguousarray(mesh.z, np.float64)
    if mesh.types is not None:
        a["types"] = np.ascontiguousarray(mesh.types, np.uint8)
    if mesh.E is not None:
        a["E"] = np.ascontiguousarray(mesh.E, np.float64)
    if mesh.nu is not None:
        a["nu"] = np.ascontiguousarray(mesh.nu, np.float64)
    return a


def device_arrays(mesh, device="cuda"):
    import torch
    return {k: torch.from_numpy(v).to(device) for k, v in host_arrays(mesh).items()}


def check(status: int, what: str, allow=(FEM_OK,)):
    if status not in allow:
        raise FemError(status, what)
    return status


def workspace_size(mesh, o: Optional[FemOpts] = None) -> int:
    """Bytes of workspace (pure host computation; works without a GPU)."""
    m = fem_mesh_struct(mesh, host_arrays(mesh))
    n = C.c_size_t(0)
    check(load().fem_alls_workspace_size(C.byref(m), C.byref(o) if o else None, C.byref(n)), "workspace_size")
    return n.value


class Assembler:
    """Device-resident assembly of one mesh through the C ABI.

    Holds the mesh arrays, workspace and CSR outputs as torch CUDA tensors so
    repeated assemblies (benchmarks) allocate nothing."""

    def __init__(self, mesh, o: Optional[FemOpts] = None, device="cuda", capacity: Optional[int] = None):
        import torch
        self.torch = torch
        self.mesh = mesh
        self.opts = o if o is not None else opts()
        self.dev = device_arrays(mesh, device)
        self.cm = fem_mesh_struct(mesh, self.dev)
        self.ws_bytes = workspace_size(mesh, self.opts)
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=device)
        base = self.ws.data_ptr()
        self.ws_ptr = (base + 255) // 256 * 256
        self.n_rows = mesh.num_dofs
        self.row_ptr = torch.empty(self.n_rows + 1, dtype=torch.int32, device=device)
        self.capacity = 0
        self.col_idx = None
        self.values = None
        if capacity:
            self.reserve(capacity)
        self.lib = load()

    def reserve(self, capacity: int):
        if capacity > self.capacity:
            self.col_idx = self.torch.empty(capacity, dtype=self.torch.int32, device=self.row_ptr.device)
            self.values = self.torch.empty(capacity, dtype=self.torch.float64, device=self.row_ptr.device)
            self.capacity = capacity

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def scatter(self):
        check(self.lib.fem_alls_scatter(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                        self._stream()), "fem_alls_scatter")

    def consolidate(self, capacity: Optional[int] = None):
        cap = self.capacity if capacity is None else capacity
        check(self.lib.fem_alls_consolidate(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                            _ptr(self.row_ptr), _ptr(self.col_idx) if cap else None,
                                            _ptr(self.values) if cap else None, cap, self._stream()),
              "fem_alls_consolidate")

    def consolidate_bsr(self):
        """Node-block (BSR) form of the last scatter: (block_row_ptr, block_col_idx, block_values) tensors."""
        torch = self.torch
        st, info = self.read_info()
        nb = int(info.nnz) // (self.mesh.dpn ** 2) if info.nnz else 0
        brp = torch.empty(self.mesh.num_nodes + 1, dtype=torch.int32, device=self.row_ptr.device)
        bci = torch.empty(max(nb, 1), dtype=torch.int32, device=self.row_ptr.device)
        bv = torch.empty(max(nb, 1) * self.mesh.dpn ** 2, dtype=torch.float64, device=self.row_ptr.device)
        check(self.lib.fem_alls_consolidate_bsr(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                                _ptr(brp), _ptr(bci), _ptr(bv), nb, self._stream()),
              "fem_alls_consolidate_bsr")
        check(self.read_info()[0], "bsr consolidation")
        return brp, bci[:nb], bv[: nb * self.mesh.dpn ** 2]

    def consolidate_upper(self, capacity: Optional[int] = None):
        """Upper-triangle CSR of the last scatter (fem_alls_consolidate_upper):
        (row_ptr, col_idx, values) tensors. Sizes its outputs with a counting
        pass when capacity is None."""
        torch = self.torch
        dev = self.row_ptr.device
        rp = torch.empty(self.n_rows + 1, dtype=torch.int32, device=dev)
        if capacity is None:
            check(self.lib.fem_alls_consolidate_upper(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                                      _ptr(rp), None, None, 0, self._stream()),
                  "fem_alls_consolidate_upper")
            st, info = self.read_info()
            capacity = int(info.nnz)
        ci = torch.empty(max(capacity, 1), dtype=torch.int32, device=dev)
        v = torch.empty(max(capacity, 1), dtype=torch.float64, device=dev)
        check(self.lib.fem_alls_consolidate_upper(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                                  _ptr(rp), _ptr(ci), _ptr(v), capacity, self._stream()),
              "fem_alls_consolidate_upper")
        return rp, ci, v

    def read_info(self) -> tuple:
        info = FemInfo()
        st = self.lib.fem_alls_read_info(self.ws_ptr, C.byref(info), self._stream())
        return st, info

    def autotune(self, repeats: int = 3) -> tuple:
        """fem_autotune on this mesh: picks the fastest scatter grid / list shape,
        adopts it (self.opts, a workspace that fits it) and leaves its assembly in
        the outputs. Returns (opts, mean ms per assembly)."""
        torch = self.torch
        if self.capacity == 0:
            self.assemble()                      # sizes the outputs
        n = C.c_size_t(0)
        check(self.lib.fem_autotune_workspace_size(C.byref(self.cm), C.byref(self.opts), C.byref(n)),
              "fem_autotune_workspace_size")
        if n.value > self.ws_bytes:
            self.ws = torch.empty(n.value + 256, dtype=torch.uint8, device=self.row_ptr.device)
            self.ws_ptr = (self.ws.data_ptr() + 255) // 256 * 256
            self.ws_bytes = n.value
        out = FemCsr(self.n_rows, 0, 0, self.capacity, _ptr(self.row_ptr), _ptr(self.col_idx), _ptr(self.values))
        best = FemOpts()
        ms = C.c_float(0.0)
        st = self.lib.fem_autotune(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes, C.byref(out),
                                   repeats, C.byref(best), C.byref(ms), self._stream())
        check(st if st != FEM_ERR_DETJ else FEM_OK, "fem_autotune")
        self.opts = best
        return best, ms.value

    def assemble_async(self):
        """scatter + consolidate into the reserved capacity, no host sync."""
        out = FemCsr(self.n_rows, 0, 0, self.capacity, _ptr(self.row_ptr), _ptr(self.col_idx),
                     _ptr(self.values))
        check(self.lib.fem_assemble_async(C.byref(self.cm), C.byref(self.opts), self.ws_ptr, self.ws_bytes,
                                          C.byref(out), self._stream()), "fem_assemble_async")

    def assemble(self, allow=(FEM_OK,)):
        """Full assembly; sizes the outputs on first use. Returns (row_ptr, col_idx, values, info) tensors."""
        self.scatter()
        self.consolidate()
        st, info = self.read_info()
        if st == FEM_ERR_CAPACITY:
            self.reserve(int(info.nnz))
            self.consolidate()
            st, info = self.read_info()
        check(st, "assemble", allow)
        nnz = int(info.nnz)
        if self.col_idx is None:
            self.reserve(max(nnz, 1))
        return self.row_ptr, self.col_idx[:nnz], self.values[:nnz], info


def assemble(mesh, o: Optional[FemOpts] = None, allow=(FEM_OK,)):
    """Assemble on the GPU; returns numpy (row_ptr, col_idx, values, info dict)."""
    a = Assembler(mesh, o)
    rp, ci, v, info = a.assemble(allow)
    return rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy(), info.as_dict()


class HostContext:
    """fem_assemble_host: host arrays in, host CSR out (copies inside the call)."""

    def __init__(self):
        self.lib = load()
        self.ctx = C.c_void_p()
        check(self.lib.fem_context_create(C.byref(self.ctx)), "fem_context_create")

    def close(self):
        if self.ctx:
            self.lib.fem_context_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def assemble(self, mesh, arrays: dict, row_ptr: np.ndarray, col_idx: Optional[np.ndarray],
                 values: Optional[np.ndarray], o: Optional[FemOpts] = None, stream=None) -> tuple:
        m = fem_mesh_struct(mesh, arrays)
        cap = 0 if col_idx is None else int(min(col_idx.shape[0], values.shape[0]))
        out = FemCsr(mesh.num_dofs, 0, 0, cap, _ptr(row_ptr), _ptr(col_idx), _ptr(values))
        st = self.lib.fem_assemble_host(self.ctx, C.byref(m), C.byref(o) if o else None, C.byref(out), stream)
        return st, int(out.nnz)


class Colouring:
    """The element-colouring baseline through the C ABI (fem_colour_*): device
    colouring of the elements, then one launch per colour adding element blocks
    into a given CSR pattern without atomics (the reference's coloured path,
    ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:504-572,648-747, rebuilt)."""

    def __init__(self, mesh, device="cuda", dev_arrays=None):
        import torch
        self.torch = torch
        self.mesh = mesh
        self.dev = dev_arrays if dev_arrays is not None else device_arrays(mesh, device)
        self.cm = fem_mesh_struct(mesh, self.dev)
        self.lib = load()
        n = C.c_size_t(0)
        check(self.lib.fem_colour_workspace_size(C.byref(self.cm), C.byref(n)), "fem_colour_workspace_size")
        self.ws_bytes = n.value
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=device)
        self.ws_ptr = (self.ws.data_ptr() + 255) // 256 * 256
        self.colours = torch.empty(max(mesh.num_elems, 1), dtype=torch.int32, device=device)
        self.num_colours = 0

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def prepare(self, allow=(FEM_OK,)) -> int:
        nc = C.c_int32(0)
        st = self.lib.fem_colour_prepare(C.byref(self.cm), self.ws_ptr, self.ws_bytes, C.byref(nc),
                                         _ptr(self.colours), self._stream())
        check(st, "fem_colour_prepare", allow)
        self.num_colours = nc.value
        return self.num_colours

    def assemble(self, row_ptr, col_idx, values, nnz: int, allow=(FEM_OK,)):
        check(self.lib.fem_colour_assemble(C.byref(self.cm), self.ws_ptr, self.ws_bytes, self.num_colours,
                                           _ptr(row_ptr), _ptr(col_idx), _ptr(values), nnz, self._stream()),
              "fem_colour_assemble", allow)

    def read_info(self) -> tuple:
        nc = C.c_int32(0)
        st = self.lib.fem_colour_read_info(self.ws_ptr, C.byref(nc), self._stream())
        return st, nc.value


def element_stiffness(mesh, o: Optional[FemOpts] = None, device="cuda", dev_arrays=None, out=None):
    """Packed symmetric element stiffness of every element (fem_element_stiffness):
    returns (ke [num_elems, doubles_per_element] tensor, status bits)."""
    import torch
    dev = dev_arrays if dev_arrays is not None else device_arrays(mesh, device)
    cm = fem_mesh_struct(mesh, dev)
    lib = load()
    n = C.c_int64(0)
    check(lib.fem_element_stiffness_size(C.byref(cm), C.byref(n)), "fem_element_stiffness_size")
    if out is None:
        out = torch.empty((max(mesh.num_elems, 1), n.value), dtype=torch.float64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    check(lib.fem_element_stiffness(C.byref(cm), C.byref(o) if o else None, _ptr(out), _ptr(status),
                                    torch.cuda.current_stream().cuda_stream), "fem_element_stiffness")
    return out[: mesh.num_elems], int(status.item())


def unpack_element_stiffness(packed: np.ndarray, npe: int, dpn: int) -> np.ndarray:
    """Full ndof x ndof Ke of one element from its packed upper node blocks."""
    nd = npe * dpn
    ke = np.zeros((nd, nd))
    k = 0
    for a in range(npe):
        for b in range(a, npe):
            blk = packed[k * dpn * dpn:(k + 1) * dpn * dpn].reshape(dpn, dpn)
            ke[a * dpn:(a + 1) * dpn, b * dpn:(b + 1) * dpn] = blk
            ke[b * dpn:(b + 1) * dpn, a * dpn:(a + 1) * dpn] = blk.T
            k += 1
    return ke


class Reassembler:
    """Value-only re-assembly (fem_scatter_map_* / fem_reassemble_values) into
    the CSR pattern of an Assembler's last assembly."""

    def __init__(self, asm: "Assembler"):
        import torch
        self.torch = torch
        self.asm = asm
        self.lib = load()
        n = C.c_size_t(0)
        check(self.lib.fem_scatter_map_size(C.byref(asm.cm), C.byref(n)), "fem_scatter_map_size")
        self.map_bytes = n.value
        self.buf = torch.empty(self.map_bytes + 256, dtype=torch.uint8, device=asm.row_ptr.device)
        self.map_ptr = (self.buf.data_ptr() + 255) // 256 * 256

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def build(self, nnz: int):
        self.nnz = nnz
        check(self.lib.fem_scatter_map_build(C.byref(self.asm.cm), _ptr(self.asm.row_ptr), _ptr(self.asm.col_idx),
                                             self.map_ptr, self.map_bytes, self._stream()), "fem_scatter_map_build")
        check(self.lib.fem_scatter_map_read_info(self.map_ptr, self._stream()), "scatter map")

    def reassemble(self, values, o: Optional[FemOpts] = None):
        """values: device float64 tensor of nnz entries (overwritten)."""
        check(self.lib.fem_reassemble_values(C.byref(self.asm.cm), C.byref(o) if o else None, self.map_ptr,
                                             self.map_bytes, _ptr(self.asm.row_ptr), _ptr(values), self.nnz,
                                             self._stream()), "fem_reassemble_values")

    def read_info(self) -> int:
        return self.lib.fem_scatter_map_read_info(self.map_ptr, self._stream())


class Batch:
    """Batched assembly of many meshes (fem_assemble_batched) with device-resident
    inputs, workspace and outputs. sizes() runs a counting pass (capacity 0) to
    size the CSR outputs; run() assembles; results(i) returns mesh i's CSR."""

    def __init__(self, meshes, o: Optional[FemOpts] = None, concurrency: int = 4, device="cuda"):
        import torch
        self.torch = torch
        self.meshes = meshes
        self.opts = o
        self.concurrency = concurrency
        self.device = device
        self.lib = load()
        self.dev = [device_arrays(m, device) for m in meshes]
        n = len(meshes)
        self.cm = (FemMesh * n)(*[fem_mesh_struct(m, d) for m, d in zip(meshes, self.dev)])
        need = 0
        for k in sorted({1, concurrency}):   # the workspace serves every concurrency up to this one
            b = C.c_size_t(0)
            check(self.lib.fem_batched_workspace_size(self.cm, n, C.byref(o) if o else None, k, C.byref(b)),
                  "fem_batched_workspace_size")
            need = max(need, b.value)
        self.ws_bytes = need
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=device)
        self.ws_ptr = (self.ws.data_ptr() + 255) // 256 * 256
        self.row_ptr = [torch.empty(m.num_dofs + 1, dtype=torch.int32, device=device) for m in meshes]
        self.col_idx = [None] * n
        self.values = [None] * n
        self.infos = torch.zeros((n, C.sizeof(FemInfo) // 8), dtype=torch.int64, device=device)
        self.stamps = torch.zeros(n + 1, dtype=torch.int64, device=device)
        self.outs = (FemCsr * n)()
        self._set_outs(capacity=False)

    def _set_outs(self, capacity: bool):
        for i, m in enumerate(self.meshes):
            cap = int(self.col_idx[i].numel()) if capacity and self.col_idx[i] is not None else 0
            self.outs[i] = FemCsr(m.num_dofs, 0, 0, cap, _ptr(self.row_ptr[i]),
                                  _ptr(self.col_idx[i]) if cap else None, _ptr(self.values[i]) if cap else None)

    def workspace_bytes(self, concurrency: int) -> int:
        b = C.c_size_t(0)
        check(self.lib.fem_batched_workspace_size(self.cm, len(self.meshes), C.byref(self.opts) if self.opts else None,
                                                  concurrency, C.byref(b)), "fem_batched_workspace_size")
        return b.value

    def _launch(self, concurrency: Optional[int] = None):
        k = self.concurrency if concurrency is None else concurrency
        check(self.lib.fem_assemble_batched(self.cm, len(self.meshes), C.byref(self.opts) if self.opts else None,
                                            k, self.ws_ptr, self.ws_bytes, self.outs,
                                            _ptr(self.infos), _ptr(self.stamps),
                                            self.torch.cuda.current_stream().cuda_stream), "fem_assemble_batched")

    def info(self, i: int) -> dict:
        raw = self.infos[i].cpu().numpy().tobytes()
        return FemInfo.from_buffer_copy(raw).as_dict()

    def sizes(self):
        """Counting pass: nnz of every mesh; allocates the CSR outputs."""
        self._set_outs(capacity=False)
        self._launch()
        self.torch.cuda.synchronize()
        nnz = []
        for i in range(len(self.meshes)):
            inf = self.info(i)
            nz = int(inf["nnz"])
            nnz.append(nz)
            self.col_idx[i] = self.torch.empty(max(nz, 1), dtype=self.torch.int32, device=self.device)
            self.values[i] = self.torch.empty(max(nz, 1), dtype=self.torch.float64, device=self.device)
        self._set_outs(capacity=True)
        return nnz

    def run(self, concurrency: Optional[int] = None):
        self._launch(concurrency)

    def autotune(self, repeats: int = 2) -> tuple:
        """fem_autotune_batched: the fastest concurrency that fits this batch's
        workspace (sized for concurrency at construction); adopts it. Returns
        (concurrency, mean ms per batch)."""
        best = C.c_int32(0)
        ms = C.c_float(0.0)
        check(self.lib.fem_autotune_batched(self.cm, len(self.meshes), C.byref(self.opts) if self.opts else None,
                                            self.ws_ptr, self.ws_bytes, self.outs, _ptr(self.infos), repeats,
                                            C.byref(best), C.byref(ms), self.torch.cuda.current_stream().cuda_stream),
              "fem_autotune_batched")
        self.concurrency = best.value
        return best.value, ms.value

    def statuses(self) -> list:
        raw = self.infos.cpu().numpy()
        return [int(FemInfo.from_buffer_copy(r.tobytes()).status_bits) for r in raw]

    def latencies_ms(self):
        """Per-mesh completion time after the batch start (GPU global timer), ms."""
        st = self.stamps.cpu().numpy()
        return (st[1:] - st[0]) / 1e6

    def result(self, i: int):
        nz = int(self.info(i)["nnz"])
        return (self.row_ptr[i].cpu().numpy(), self.col_idx[i][:nz].cpu().numpy(),
                self.values[i][:nz].cpu().numpy())


def body_force(mesh, b, dev_arrays=None, device="cuda"):
    """Load vector of a body force (fem_assemble_body_force). b: a per-element
    [num_elems, dim] numpy array, or a uniform length-dim sequence. Returns
    (f tensor [ndof], status bits)."""
    import torch
    dev = dev_arrays if dev_arrays is not None else device_arrays(mesh, device)
    cm = fem_mesh_struct(mesh, dev)
    f = torch.zeros(mesh.num_dofs, dtype=torch.float64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    b = np.asarray(b, np.float64)
    if b.ndim == 2:
        bd = torch.from_numpy(np.ascontiguousarray(b)).to(device)
        args = (_ptr(bd), None)
    else:
        b0 = np.ascontiguousarray(b)
        args = (None, b0.ctypes.data)
    check(load().fem_assemble_body_force(C.byref(cm), args[0], args[1], _ptr(f), _ptr(status),
                                         torch.cuda.current_stream().cuda_stream), "fem_assemble_body_force")
    return f, int(status.item())


def apply_dirichlet(row_ptr, col_idx, values, f, fixed, u):
    """Symmetric elimination of the fixed dofs in place (fem_apply_dirichlet); all device tensors."""
    import torch
    check(load().fem_apply_dirichlet(int(row_ptr.numel() - 1), _ptr(row_ptr), _ptr(col_idx), _ptr(values),
                                     _ptr(f) if f is not None else None, _ptr(fixed), _ptr(u),
                                     torch.cuda.current_stream().cuda_stream), "fem_apply_dirichlet")
