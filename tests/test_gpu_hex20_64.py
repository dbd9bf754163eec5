"""Parity on the full Hex20 64^3 configuration (1,085,825 nodes, 262,144
elements, 557,286,921 CSR nonzeros), through the C ABI.

* pattern: the device row_ptr / col_idx equal the oracle's sorted-unique
  pattern (restating buildCSRStructureHex20,
  ALLS_Hex20_3D_Assembly_Performance.cu:364-392) bit for bit, all of it;
* values: a seeded sample of 2,048 row nodes (6,144 dof rows) is assembled by
  the serial FP64 oracle from only the elements that touch those nodes
  (oracle_assemble_rows, the same element loop and addition order as the
  reference's serial host assembly, ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:
  329-380) and compared entry by entry;
* the tensor-core Ke form (FEM_PREC_TC_F16X3) on the same sample, at the
  north-star bound of 1e-6.

Error measures (printed, and bounded below):
  scaled    |K - K_oracle| / max(|K_ij|, sqrt(|K_ii K_jj|))  (K_ii from the
            device's assembled diagonal)
  per-entry |K - K_oracle| / |K_oracle|, over the entries that do not cancel
            between elements: |K_oracle,ij| >= 1e-8 sqrt(|K_ii K_jj|)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 64
SAMPLE_NODES = 2048
RTOL_FP64 = 1e-12          # scaled, plain FP64 path
REL_FP64 = 1e-6            # per entry, entries >= 1e-8 of their row/column scale
RTOL_TC = 1e-6             # scaled, tensor-core Ke form
SIGNIFICANT = 1e-8


@pytest.fixture(scope="module")
def h20(oracle_mod):
    import meshgen as mg
    m = mg.hex20_grid(N)
    orp, oci = oracle_mod.pattern(m)
    rng = np.random.default_rng(64)
    nodes = np.sort(rng.choice(m.num_nodes, SAMPLE_NODES, replace=False))
    return m, orp, oci, nodes


def _diag_at(rp, ci, v, dofs):
    """K_jj for the dofs j (vectorised binary search of column j in row j)."""
    lo, hi = rp[dofs].astype(np.int64), rp[dofs + 1].astype(np.int64) - 1
    for _ in range(40):
        mid = (lo + hi) // 2
        less = ci[np.clip(mid, 0, ci.shape[0] - 1)] < dofs
        lo = np.where(less & (lo <= hi), mid + 1, lo)
        hi = np.where(~less & (lo <= hi), mid - 1, hi)
    assert np.all(ci[lo] == dofs), "diagonal entry missing"
    return v[lo]


def _sampled_errors(orp, oci, ov, v_dev, nodes):
    """Errors of the sampled rows: device values v_dev (numpy, full CSR) against
    the oracle's ov (same pattern), on the scales described above."""
    rows = (3 * nodes[:, None] + np.arange(3)[None, :]).ravel()
    lo, hi = orp[rows], orp[rows + 1]
    idx = np.concatenate([np.arange(a, b) for a, b in zip(lo, hi)])
    r = np.repeat(rows, hi - lo)
    c = oci[idx].astype(np.int64)
    ref, test = ov[idx], v_dev[idx]
    d = np.abs(test - ref)
    dofs = np.unique(np.concatenate([rows, c]))
    dv = np.zeros(orp.shape[0] - 1)
    dv[dofs] = _diag_at(orp, oci, v_dev, dofs)
    sc_diag = np.sqrt(np.abs(dv[r] * dv[c]))
    scaled = float(np.max(d / np.maximum(np.abs(ref), np.where(sc_diag > 0, sc_diag, 1.0))))
    sig = np.abs(ref) >= SIGNIFICANT * sc_diag
    rel_sig = float(np.max(d[sig] / np.abs(ref[sig]))) if sig.any() else 0.0
    nz = ref != 0
    rel_all = float(np.max(d[nz] / np.abs(ref[nz]))) if nz.any() else 0.0
    return {"entries": int(idx.size), "scaled": scaled, "rel_significant": rel_sig, "rel_all_nonzero": rel_all,
            "significant_fraction": float(sig.mean())}


def _assemble(fem, m, o=None):
    a = fem.Assembler(m, o)
    rp, ci, v, info = a.assemble()
    return a, rp, ci, v, info


def test_hex20_64_pattern_and_sampled_values(fem, oracle_mod, cuda_device, h20):
    m, orp, oci, nodes = h20
    a, rp, ci, v, info = _assemble(fem, m)
    assert int(info.nnz) == oci.shape[0] == 557_286_921
    np.testing.assert_array_equal(rp.cpu().numpy(), orp)
    np.testing.assert_array_equal(ci.cpu().numpy(), oci)
    assert int(info.list_entries) == oci.shape[0] // 9   # no duplicate list entries
    vh = v.cpu().numpy()
    ov = oracle_mod.assemble_rows(m, orp, oci, nodes)
    err = _sampled_errors(orp, oci, ov, vh, nodes)
    print(f"hex20 64^3 FP64 sampled rows: {err}")
    assert err["scaled"] <= RTOL_FP64
    assert err["rel_significant"] <= REL_FP64


def test_hex20_64_tensor_core_form(fem, oracle_mod, cuda_device, h20):
    m, orp, oci, nodes = h20
    a, rp, ci, v, info = _assemble(fem, m, fem.opts(precision=fem.FEM_PREC_TC_F16X3))
    np.testing.assert_array_equal(rp.cpu().numpy(), orp)
    np.testing.assert_array_equal(ci.cpu().numpy(), oci)
    vh = v.cpu().numpy()
    ov = oracle_mod.assemble_rows(m, orp, oci, nodes)
    err = _sampled_errors(orp, oci, ov, vh, nodes)
    print(f"hex20 64^3 tensor-core form sampled rows: {err}")
    assert err["scaled"] <= RTOL_TC
