"""The C ABI library: it loads, exports every symbol include/*.h declares, and its
host-side argument checking and workspace sizing behave (CPU, no kernel launches)."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*FEM_API\s+[^(;]*?\b(fem_[A-Za-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(fem):
    lib = fem.load()
    decl = declared_functions()
    assert len(decl) >= 12
    for name in decl:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", fem.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (fem_\w+)", out))
    assert exported == set(decl), (exported ^ set(decl))
    assert set(fem.EXPORTS) == set(decl)


def test_abi_version_and_status_strings(fem):
    lib = fem.load()
    assert lib.fem_abi_version() == 2
    assert lib.fem_status_string(0) == b"ok"
    assert b"pool" in lib.fem_status_string(3)


def test_workspace_size_host_only(fem):
    import meshgen as mg
    m = mg.by_name("q4_small")
    n = fem.workspace_size(m)
    assert n > 0 and n % 256 == 0
    # grows with the pool factor
    assert fem.workspace_size(m, fem.opts(pool_factor=2.0)) > n
    h = mg.by_name("hex20_small")
    nh = fem.workspace_size(h)
    nh2 = fem.workspace_size(h, fem.opts(first_slots=94, chunk_slots=62))
    assert nh2 > nh


def test_bad_arguments_are_rejected_before_any_launch(fem):
    import meshgen as mg
    lib = fem.load()
    m = mg.by_name("q4_small")
    arrays = fem.host_arrays(m)
    cm = fem.fem_mesh_struct(m, arrays)
    n = C.c_size_t()
    assert lib.fem_alls_workspace_size(None, None, C.byref(n)) == fem.FEM_ERR_BAD_ARG
    bad = fem.fem_mesh_struct(m, arrays)
    bad.conn_stride = 3
    assert lib.fem_alls_workspace_size(C.byref(bad), None, C.byref(n)) == fem.FEM_ERR_BAD_ARG
    bad = fem.fem_mesh_struct(m, arrays)
    bad.kind = 7
    assert lib.fem_alls_workspace_size(C.byref(bad), None, C.byref(n)) == fem.FEM_ERR_BAD_ARG
    # 2-D chunk rows are fixed
    o = fem.opts(first_slots=30)
    assert lib.fem_alls_workspace_size(C.byref(cm), C.byref(o), C.byref(n)) == fem.FEM_ERR_BAD_ARG
    # Hex20 chunk rows must be a multiple of 16 bytes
    h = mg.by_name("hex20_small")
    ch = fem.fem_mesh_struct(h, fem.host_arrays(h))
    o = fem.opts(first_slots=31)
    assert lib.fem_alls_workspace_size(C.byref(ch), C.byref(o), C.byref(n)) == fem.FEM_ERR_BAD_ARG
    # a workspace that is too small is refused before touching the device
    assert lib.fem_alls_scatter(C.byref(cm), None, C.c_void_p(256), 16, None) == fem.FEM_ERR_WORKSPACE
    # misaligned workspace
    size = fem.workspace_size(m)
    assert lib.fem_alls_scatter(C.byref(cm), None, C.c_void_p(257), size, None) == fem.FEM_ERR_WORKSPACE
    # consolidate: capacity without buffers
    assert lib.fem_alls_consolidate(C.byref(cm), None, C.c_void_p(256), size, C.c_void_p(512), None, None, 10,
                                    None) == fem.FEM_ERR_BAD_ARG
    assert lib.fem_alls_read_info(None, None, None) == fem.FEM_ERR_BAD_ARG


def test_host_entry_point_checks_arguments(fem):
    import meshgen as mg
    ctx = fem.HostContext()
    m = mg.by_name("q4_small")
    arrays = fem.host_arrays(m)
    bad = fem.fem_mesh_struct(m, arrays)
    bad.num_nodes = 0
    out = fem.FemCsr()
    assert fem.load().fem_assemble_host(ctx.ctx, C.byref(bad), None, C.byref(out), None) == fem.FEM_ERR_BAD_ARG
    ctx.close()


def _host_workspace(fem, m, o=None):
    """A host buffer standing in for the workspace: the calls below must return
    before the first device access, so it is never dereferenced."""
    n = fem.workspace_size(m, o)
    buf = np.zeros(n + 256, np.uint8)
    ptr = (buf.ctypes.data + 255) // 256 * 256
    return buf, C.c_void_p(ptr), n


def test_precision_and_grid_options_are_checked(fem):
    import meshgen as mg
    lib = fem.load()
    for name, bad_prec in (("t3_small", fem.FEM_PREC_TC_F16X3), ("t3_small", fem.FEM_PREC_FP64_SIMT),
                           ("hex20_small", fem.FEM_PREC_FP32), ("q4_small", 9)):
        m = mg.by_name(name)
        cm = fem.fem_mesh_struct(m, fem.host_arrays(m))
        keep, ws, n = _host_workspace(fem, m)
        o = fem.opts(precision=bad_prec)
        assert lib.fem_alls_scatter(C.byref(cm), C.byref(o), ws, n, None) == fem.FEM_ERR_BAD_ARG, (name, bad_prec)
        st = C.c_int32(0)
        if bad_prec != fem.FEM_PREC_FP64_SIMT or m.kind != mg.HEX20:
            assert lib.fem_element_stiffness(C.byref(cm), C.byref(o), C.c_void_p(256), C.byref(st), None) \
                == fem.FEM_ERR_BAD_ARG, (name, bad_prec)
    m = mg.by_name("t3_small")
    cm = fem.fem_mesh_struct(m, fem.host_arrays(m))
    keep, ws, n = _host_workspace(fem, m)
    o = fem.opts(ctas_per_sm=-1)
    assert lib.fem_alls_scatter(C.byref(cm), C.byref(o), ws, n, None) == fem.FEM_ERR_BAD_ARG


def test_upper_output_and_autotuner_arguments(fem):
    import meshgen as mg
    lib = fem.load()
    m = mg.by_name("t3_small")
    cm = fem.fem_mesh_struct(m, fem.host_arrays(m))
    keep, ws, n = _host_workspace(fem, m)
    # no row pointer / no col_idx with a capacity
    assert lib.fem_alls_consolidate_upper(C.byref(cm), None, ws, n, None, None, None, 0, None) == fem.FEM_ERR_BAD_ARG
    assert lib.fem_alls_consolidate_upper(C.byref(cm), None, ws, n, C.c_void_p(256), None, None, 5, None) \
        == fem.FEM_ERR_BAD_ARG
    # the autotuner's workspace covers every candidate, so at least the default one
    for name in ("t3_small", "hex20_small"):
        mm = mg.by_name(name)
        cmm = fem.fem_mesh_struct(mm, fem.host_arrays(mm))
        t = C.c_size_t(0)
        assert lib.fem_autotune_workspace_size(C.byref(cmm), None, C.byref(t)) == fem.FEM_OK
        assert t.value >= fem.workspace_size(mm) and t.value % 256 == 0
    out = fem.FemCsr(m.num_dofs, 0, 0, 0, None, None, None)
    best = fem.FemOpts()
    assert lib.fem_autotune(C.byref(cm), None, ws, n, C.byref(out), 0, C.byref(best), None, None) \
        == fem.FEM_ERR_BAD_ARG          # repeats < 1
    assert lib.fem_autotune(C.byref(cm), None, ws, n, None, 2, C.byref(best), None, None) == fem.FEM_ERR_BAD_ARG
    k = C.c_int32(0)
    assert lib.fem_autotune_batched(C.byref(cm), 1, None, ws, n, C.byref(out), C.c_void_p(256), 0, C.byref(k),
                                    None, None) == fem.FEM_ERR_BAD_ARG
    assert lib.fem_autotune_batched(C.byref(cm), 0, None, ws, n, C.byref(out), C.c_void_p(256), 1, C.byref(k),
                                    None, None) == fem.FEM_ERR_BAD_ARG


def test_batched_workspace_sizing_host_only(fem):
    # Slots are dealt the meshes largest first, one slot per mesh until every
    # slot has one, so a slot's size is that of its first (largest) mesh (a
    # Hex20 mesh's slot also holds a second wave's group records, 5220 words
    # per group of 8 elements): the workspace
    # grows with the slot count and is capped by the mesh count. A control
    # block (descriptors, schedule, counters) comes first.
    import meshgen as mg
    lib = fem.load()
    meshes = mg.batch_meshes(6, seed=3, emin=20, emax=400)
    arrs = [fem.host_arrays(m) for m in meshes]
    cm = (fem.FemMesh * len(meshes))(*[fem.fem_mesh_struct(m, a) for m, a in zip(meshes, arrs)])
    single = max(fem.workspace_size(m) for m in meshes)
    sizes = []
    for k in (1, 2, 4, 6, 8, 16):
        b = C.c_size_t(0)
        assert lib.fem_batched_workspace_size(cm, len(meshes), None, k, C.byref(b)) == fem.FEM_OK
        sizes.append(b.value)
    assert sizes[0] >= single and sizes[0] % 256 == 0
    assert all(a <= b for a, b in zip(sizes, sizes[1:]))
    assert sizes[3] == sizes[4] == sizes[5]          # at most one slot per mesh
    up = lambda v: -(-v // 256) * 256  # noqa: E731
    total = sum(up(fem.workspace_size(m)) + (up(-(-min(m.num_elems, 4096) // 8) * 5220 * 4) if m.kind == 2 else 0)
                for m in meshes)
    assert total < sizes[3] <= total + 64 * 1024
    b = C.c_size_t(0)
    assert lib.fem_batched_workspace_size(cm, 0, None, 4, C.byref(b)) == fem.FEM_ERR_BAD_ARG
