"""Node-block (BSR) output of the consolidation (fem_alls_consolidate_bsr),
through the C ABI: expanded to scalar CSR it must equal the CSR output of the
same lists exactly (same entries, same values bit for bit), for 2x2 and 3x3
blocks, including the long-row path (a high-degree node); and, expanded, it
must match the oracle directly: the pattern of the reference's host builder
bit for bit, the values within 1e-12 of the row/column scale."""
import numpy as np
import pytest

from conftest import diag_scale

pytestmark = pytest.mark.gpu


def _bsr_to_csr(brp, bci, bv, dpn):
    n = brp.shape[0] - 1
    rows, cols, vals = [], [], []
    for node in range(n):
        for k in range(brp[node], brp[node + 1]):
            blk = bv[k * dpn * dpn:(k + 1) * dpn * dpn].reshape(dpn, dpn)
            for i in range(dpn):
                for j in range(dpn):
                    rows.append(node * dpn + i)
                    cols.append(bci[k] * dpn + j)
                    vals.append(blk[i, j])
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    order = np.lexsort((cols, rows))
    rp = np.zeros(n * dpn + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp), cols[order], vals[order]


def _fan():
    from test_gpu_parity import _fan_mesh
    return _fan_mesh(40)


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small", "fan"])
def test_bsr_equals_csr(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = _fan() if name == "fan" else mg.by_name(name)
    asm = fem.Assembler(m)
    rp, ci, v, info = asm.assemble()
    rp, ci, v = rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy()
    brp, bci, bv = asm.consolidate_bsr()
    brp, bci, bv = brp.cpu().numpy(), bci.cpu().numpy(), bv.cpu().numpy()
    d = m.dpn
    assert brp[-1] * d * d == ci.shape[0]
    # block columns sorted within each block row
    for node in range(m.num_nodes):
        assert np.all(np.diff(bci[brp[node]:brp[node + 1]]) > 0)
    erp, eci, ev = _bsr_to_csr(brp, bci, bv, d)
    np.testing.assert_array_equal(erp, rp)
    np.testing.assert_array_equal(eci, ci)
    np.testing.assert_array_equal(ev, v)
    # pinned to the oracle itself, not only to the library's own CSR
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(erp, orp)
    np.testing.assert_array_equal(eci, oci)
    scale = np.maximum(np.abs(ov), diag_scale(orp, oci, ov))
    assert np.all(np.abs(ev - ov) <= 1e-12 * scale)
