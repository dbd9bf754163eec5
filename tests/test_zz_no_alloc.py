"""fem_assemble_static (workspace in the library's static device array) against
fem_assemble (caller workspace), through the C ABI, on consecutive calls.

The static array keeps the previous call's contents, so the meshes alternate in
size and kind: each call must clear what it needs and give fem_assemble's result.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import diag_scale

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _csr(fem, torch, mesh, capacity, device):
    rp = torch.empty(mesh.num_dofs + 1, dtype=torch.int32, device=device)
    ci = torch.empty(capacity, dtype=torch.int32, device=device)
    v = torch.empty(capacity, dtype=torch.float64, device=device)
    out = fem.FemCsr(mesh.num_dofs, 0, 0, capacity, rp.data_ptr(), ci.data_ptr(), v.data_ptr())
    return out, rp, ci, v


def _with_workspace(fem, torch, lib, cm, mesh, capacity, device, stream):
    nbytes = fem.workspace_size(mesh)
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
    ptr = (ws.data_ptr() + 255) // 256 * 256
    out, rp, ci, v = _csr(fem, torch, mesh, capacity, device)
    st = lib.fem_assemble(C.byref(cm), None, C.c_void_p(ptr), C.c_size_t(nbytes), C.byref(out), C.c_void_p(stream))
    assert st == fem.FEM_OK, fem.load().fem_status_string(st)
    n = int(out.nnz)
    return rp.cpu().numpy(), ci[:n].cpu().numpy(), v[:n].cpu().numpy()


def _static(fem, torch, lib, cm, mesh, capacity, device, stream):
    out, rp, ci, v = _csr(fem, torch, mesh, capacity, device)
    st = lib.fem_assemble_static(C.byref(cm), None, C.byref(out), C.c_void_p(stream))
    assert st == fem.FEM_OK, fem.load().fem_status_string(st)
    n = int(out.nnz)
    return rp.cpu().numpy(), ci[:n].cpu().numpy(), v[:n].cpu().numpy()


def test_static_workspace_matches_fem_assemble(fem, cuda_device):
    import torch
    import meshgen as mg
    lib = fem.load()
    lib.fem_assemble_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    meshes = [mg.q4_grid(60, 50, seed=31), mg.hex20_grid(4, 3, 3, seed=32), mg.by_name("mixed_small"),
              mg.q4_grid(60, 50, seed=31)]
    for m in meshes:
        assert fem.workspace_size(m) <= fem.STATIC_WORKSPACE_BYTES
        dev = fem.device_arrays(m, cuda_device)
        cm = fem.fem_mesh_struct(m, dev)
        cap = m.contributions()  # upper bound of nnz
        rp0, ci0, v0 = _with_workspace(fem, torch, lib, cm, m, cap, cuda_device, stream)
        rp1, ci1, v1 = _static(fem, torch, lib, cm, m, cap, cuda_device, stream)
        np.testing.assert_array_equal(rp1, rp0)
        np.testing.assert_array_equal(ci1, ci0)
        # values differ only by the order of the FP64 atomic adds
        scale = np.maximum(np.abs(v0), diag_scale(rp0, ci0, v0))
        assert np.all(np.abs(v1 - v0) <= RTOL * scale), m.name


def test_static_workspace_refuses_large_meshes(fem, cuda_device):
    import torch
    import meshgen as mg
    lib = fem.load()
    lib.fem_assemble_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    m = mg.hex20_grid(12)
    assert fem.workspace_size(m) > fem.STATIC_WORKSPACE_BYTES
    dev = fem.device_arrays(m, cuda_device)
    cm = fem.fem_mesh_struct(m, dev)
    out, *_ = _csr(fem, torch, m, 16, cuda_device)
    st = lib.fem_assemble_static(C.byref(cm), None, C.byref(out),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == fem.FEM_ERR_WORKSPACE


def test_static_second_call_allocates_nothing(fem, cuda_device):
    # After a first call (which may load the module), a second call of the
    # same mesh leaves the device's free memory exactly as it was: nothing is
    # allocated or freed by the library.
    import torch
    import meshgen as mg
    lib = fem.load()
    lib.fem_assemble_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    m = mg.hex20_grid(4, 3, 3, seed=33)
    dev = fem.device_arrays(m, cuda_device)
    cm = fem.fem_mesh_struct(m, dev)
    out, rp, ci, v = _csr(fem, torch, m, m.contributions(), cuda_device)
    assert lib.fem_assemble_static(C.byref(cm), None, C.byref(out), C.c_void_p(stream)) == fem.FEM_OK
    torch.cuda.synchronize()
    free0, total0 = torch.cuda.mem_get_info()
    assert lib.fem_assemble_static(C.byref(cm), None, C.byref(out), C.c_void_p(stream)) == fem.FEM_OK
    torch.cuda.synchronize()
    free1, total1 = torch.cuda.mem_get_info()
    assert (free1, total1) == (free0, total0)
