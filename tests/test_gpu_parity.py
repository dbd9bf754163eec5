"""Parity of the CUDA library (called through its C ABI) with the oracle.

Pattern (row_ptr, col_idx): bit-exact. Values: the plain FP64 path must agree
with the serial FP64 oracle within 1e-12, measured per entry relative to
max(|K_ij|, sqrt(|K_ii K_jj|)) (entries that cancel to near zero between
elements are compared on the scale of their row and column); the plain
per-entry relative error is reported too.
"""
import numpy as np
import pytest

from conftest import value_errors

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _check(fem, oracle_mod, m, o=None, allow=(0,)):
    rp, ci, v, info = fem.assemble(m, o, allow=allow)
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    rel, scaled = value_errors(orp, oci, ov, v)
    scale = np.maximum(np.abs(ov), __import__("conftest").diag_scale(orp, oci, ov))
    bad = np.abs(v - ov) > RTOL * scale
    assert not bad.any(), f"{bad.sum()} entries off; max rel {rel:.3e}, max scaled {scaled:.3e}"
    assert info["nnz"] == oci.shape[0]
    # every column is inserted once per row: the lists hold no duplicates
    assert info["list_entries"] == oci.shape[0] // (m.dpn * m.dpn)
    return rel, scaled, info


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small"])
def test_small_meshes(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    rel, scaled, info = _check(fem, oracle_mod, mg.by_name(name))
    print(f"{name}: max rel {rel:.2e}, max scaled {scaled:.2e}, info {info}")


@pytest.mark.parametrize("name", ["q4", "t3", "mixed"])
def test_benchmark_meshes_2d(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    rel, scaled, info = _check(fem, oracle_mod, mg.by_name(name))
    print(f"{name}: max rel {rel:.2e}, max scaled {scaled:.2e}, info {info}")


def test_reference_material_q4_values(fem, oracle_mod, cuda_device):
    # The reference's own accuracy-test mesh and material (Q4A:968-969, E=2.1e11,
    # nu=0.3, t=0.01); the reference's pass threshold is |diff| <= 1e-10 absolute
    # on values of order 1e9 (Q4A:1157).
    import meshgen as mg
    conn, x, y = oracle_mod.ref_q4a_generate_mesh(10, 100) if oracle_mod.ref_available() else (None, None, None)
    if conn is None:
        g = np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "reference_host.npz"))
        conn, x, y = g["q4_ref10x100/conn"], g["q4_ref10x100/x"], g["q4_ref10x100/y"]
    m = mg.Mesh(mg.Q4, x, y, None, conn, None, None, None, E0=2.1e11, nu0=0.3, thickness=0.01)
    rel, scaled, _ = _check(fem, oracle_mod, m)
    # On this unperturbed mesh many off-diagonal entries cancel exactly between
    # elements, so the per-entry relative error is meaningless there; the
    # error relative to the row/column scale is what is bounded.
    assert scaled < 1e-13


def test_hex20_reference_lattice_with_orphan_nodes(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.hex20_grid(3, 2, 2, seed=21, compact=False)   # keeps face/body-centre points: empty rows
    _check(fem, oracle_mod, m)


def test_hex20_chained_chunks(fem, oracle_mod, cuda_device):
    # Tiny chunks force every Hex20 row through several overflow chunks.
    import meshgen as mg
    m = mg.hex20_grid(3, 3, 2, seed=22)
    rel, scaled, info = _check(fem, oracle_mod, m, fem.opts(first_slots=6, chunk_slots=2, pool_factor=60.0))
    assert info["overflow_chunks"] > 0


def _fan_mesh(k=40):
    """T3 fan: k triangles around node 0, so node 0's row has k+1 entries and the
    2-D list must chain overflow chunks."""
    import meshgen as mg
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    x = np.concatenate([[0.0], np.cos(ang)])
    y = np.concatenate([[0.0], np.sin(ang)])
    conn = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int32)
    return mg.Mesh(mg.T3, x, y, None, conn, None, None, None, E0=1.0, nu0=0.3, thickness=1.0, name="fan")


def test_t3_fan_high_degree_node(fem, oracle_mod, cuda_device):
    rel, scaled, info = _check(fem, oracle_mod, _fan_mesh(40))
    assert info["overflow_chunks"] >= 2 and info["max_row_entries"] >= 41


def test_single_element_each_kind(fem, oracle_mod, cuda_device):
    import meshgen as mg
    for m in (mg.q4_grid(1, 1), mg.t3_grid(1, 1, shuffle=False), mg.hex20_grid(1)):
        _check(fem, oracle_mod, m)


def test_empty_mesh(fem, cuda_device):
    import meshgen as mg
    m = mg.q4_grid(2, 2)
    m.conn = m.conn[:0]
    rp, ci, v, info = fem.assemble(m)
    assert info["nnz"] == 0 and np.all(rp == 0)


def test_bad_node_id_reports_bad_mesh(fem, cuda_device):
    import meshgen as mg
    m = mg.t3_grid(4, 4, seed=3)
    m.conn = m.conn.copy()
    m.conn[5, 1] = m.num_nodes + 7
    a = fem.Assembler(m)
    a.scatter()
    a.consolidate(0)
    st, info = a.read_info()
    assert st == fem.FEM_ERR_BAD_MESH
    m.conn[5, 1] = -1
    a = fem.Assembler(m)
    a.scatter()
    a.consolidate(0)
    assert a.read_info()[0] == fem.FEM_ERR_BAD_MESH


def test_inverted_element_reports_detj_but_assembles(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.q4_grid(3, 3, jitter=0.0)
    m.conn = m.conn.copy()
    m.conn[4] = m.conn[4][[1, 0, 3, 2]]   # clockwise element
    rp, ci, v, info = fem.assemble(m, allow=(fem.FEM_ERR_DETJ,))
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(ci, oci)
    np.testing.assert_allclose(v, ov, rtol=1e-12, atol=1e-12 * np.abs(ov).max())


def test_pool_overflow_then_retry(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.hex20_grid(2, seed=5)
    small = fem.opts(first_slots=6, chunk_slots=2, pool_factor=1e-9)   # 64 overflow chunks only
    a = fem.Assembler(m, small)
    a.scatter()
    a.consolidate(0)
    st, info = a.read_info()
    assert st == fem.FEM_ERR_POOL_OVERFLOW
    assert info.overflow_chunks > info.pool_chunks
    _check(fem, oracle_mod, m, fem.opts(first_slots=6, chunk_slots=2, pool_factor=80.0))


def test_capacity_too_small_then_rerun(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.by_name("q4_small")
    a = fem.Assembler(m, capacity=100)
    a.scatter()
    a.consolidate()
    st, info = a.read_info()
    assert st == fem.FEM_ERR_CAPACITY and info.nnz > 100
    a.reserve(int(info.nnz))
    a.consolidate()   # the lists are intact: consolidation alone is re-run
    st, info = a.read_info()
    assert st == fem.FEM_OK
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(a.col_idx[:info.nnz].cpu().numpy(), oci)


def test_repeatable(fem, cuda_device):
    import meshgen as mg
    m = mg.by_name("t3_small")
    a = fem.Assembler(m)
    r1 = [t.cpu().numpy().copy() for t in a.assemble()[:3]]
    for _ in range(3):
        r2 = [t.cpu().numpy() for t in a.assemble()[:3]]
        np.testing.assert_array_equal(r1[0], r2[0])
        np.testing.assert_array_equal(r1[1], r2[1])
        np.testing.assert_allclose(r1[2], r2[2], rtol=1e-14, atol=1e-15 * np.abs(r1[2]).max())


def test_host_entry_point(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.by_name("mixed_small")
    orp, oci, ov = oracle_mod.assemble(m)
    ctx = fem.HostContext()
    arrays = fem.host_arrays(m)
    rp = np.zeros(m.num_dofs + 1, np.int32)
    st, nnz = ctx.assemble(m, arrays, rp, None, None)
    assert st == fem.FEM_ERR_CAPACITY and nnz == oci.shape[0]
    ci = np.zeros(nnz, np.int32)
    v = np.zeros(nnz)
    st, nnz = ctx.assemble(m, arrays, rp, ci, v)
    assert st == fem.FEM_OK
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    np.testing.assert_allclose(v, ov, rtol=1e-12, atol=1e-12 * np.abs(ov).max())
    ctx.close()


# Full assembly with the tensor-core Ke form (FEM_PREC_TC_F16X3): the pattern
# is the same bit for bit; values (FP64 global accumulation of the per-element
# FP16-split contraction) agree with the FP64 oracle within TC_RTOL on the
# row/column scale max(|K_ij|, sqrt(|K_ii K_jj|)), bounded at the north star's
# 1e-6 (measured: about 4e-7).
TC_RTOL = 1e-6


@pytest.mark.parametrize("name", ["hex20_small"])
def test_tensor_core_form_assembly(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    rp, ci, v, info = fem.assemble(m, fem.opts(precision=1))
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    rel, scaled = value_errors(orp, oci, ov, v)
    print(f"{name} tensor-core form: max scaled error {scaled:.3e}, max per-entry relative {rel:.3e}")
    assert scaled <= TC_RTOL


# Full assembly with the FP32 Ke form of the 2-D kinds (FEM_PREC_FP32): the
# pattern is the same bit for bit; the FP32 blocks accumulated in FP64 agree
# with the FP64 oracle within FP32_RTOL on the row/column scale.
FP32_RTOL = 1e-5


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "t3"])
def test_fp32_form_assembly(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    rp, ci, v, info = fem.assemble(m, fem.opts(precision=fem.FEM_PREC_FP32))
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    rel, scaled = value_errors(orp, oci, ov, v)
    print(f"{name} FP32 form: max scaled error {scaled:.3e}, max per-entry relative {rel:.3e}")
    assert scaled <= FP32_RTOL
    assert info["list_entries"] == oci.shape[0] // 4


def test_fp32_form_rejected_for_hex20(fem, cuda_device):
    import meshgen as mg
    with pytest.raises(fem.FemError):
        fem.assemble(mg.by_name("hex20_small"), fem.opts(precision=fem.FEM_PREC_FP32))
