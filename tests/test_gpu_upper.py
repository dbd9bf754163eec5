"""Upper-triangle CSR output (fem_alls_consolidate_upper) through the C ABI:
for the same lists it must hold exactly the entries of the full CSR with
column >= row (pattern and values bit for bit), for every element kind, for
chained overflow chunks, for a row longer than the in-register sort, and at
the full T3 1000^2 size; it must also match the upper triangle of the
oracle's assembly directly (pattern bit for bit, values within 1e-12 of the
row/column scale); a too-small capacity raises FEM_ERR_CAPACITY."""
import numpy as np
import pytest

from conftest import diag_scale

pytestmark = pytest.mark.gpu


def _upper_of(rp, ci, v):
    n = rp.shape[0] - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    keep = ci >= rows
    urp = np.zeros(n + 1, np.int64)
    np.add.at(urp, rows[keep] + 1, 1)
    return np.cumsum(urp).astype(np.int32), ci[keep], v[keep]


def _check(fem, m, o=None, oracle_mod=None):
    asm = fem.Assembler(m, o)
    rp, ci, v, info = asm.assemble()
    full = int(info.nnz)
    rp, ci, v = rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy()
    urp, uci, uv = asm.consolidate_upper()
    st, uinfo = asm.read_info()
    assert st == 0
    erp, eci, ev = _upper_of(rp, ci, v)
    nz = int(uinfo.nnz)
    assert nz == eci.shape[0]
    np.testing.assert_array_equal(urp.cpu().numpy(), erp)
    np.testing.assert_array_equal(uci[:nz].cpu().numpy(), eci)
    np.testing.assert_array_equal(uv[:nz].cpu().numpy(), ev)   # the same list values: bit for bit
    if oracle_mod is not None:
        orp, oci, ov = oracle_mod.assemble(m)
        scale = np.maximum(np.abs(ov), diag_scale(orp, oci, ov))
        _, _, usc = _upper_of(orp, oci, scale)
        orp, oci, ov = _upper_of(orp, oci, ov)
        np.testing.assert_array_equal(urp.cpu().numpy(), orp)
        np.testing.assert_array_equal(uci[:nz].cpu().numpy(), oci)
        assert np.all(np.abs(uv[:nz].cpu().numpy() - ov) <= 1e-12 * usc)
    return asm, nz, full


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small", "t3"])
def test_upper_equals_upper_part_of_full(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    asm, nz, full = _check(fem, m, oracle_mod=oracle_mod)
    # symmetric storage: the diagonal once, each off-diagonal pair once
    assert 2 * nz - m.num_dofs == full
    print(f"{name}: upper {nz} of {full} entries")


def test_upper_chained_chunks_and_long_row(fem, oracle_mod, cuda_device):
    import meshgen as mg
    from test_gpu_parity import _fan_mesh
    _check(fem, mg.hex20_grid(3, 3, 2, seed=22), fem.opts(first_slots=6, chunk_slots=2, pool_factor=60.0),
           oracle_mod=oracle_mod)
    _check(fem, _fan_mesh(40), oracle_mod=oracle_mod)   # node 0: 41 column nodes, past the 2-D sort capacity


def test_upper_capacity_too_small(fem, cuda_device):
    import meshgen as mg
    m = mg.by_name("t3_small")
    asm = fem.Assembler(m)
    asm.assemble()
    rp, ci, v = asm.consolidate_upper()
    nz = int(asm.read_info()[1].nnz)
    with pytest.raises(fem.FemError):
        asm.consolidate_upper(capacity=nz - 1)
        st, _ = asm.read_info()
        fem.check(st, "upper")
    assert asm.read_info()[0] == fem.FEM_ERR_CAPACITY
