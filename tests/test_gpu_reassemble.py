"""Value-only re-assembly through a scatter map (fem_scatter_map_build /
fem_reassemble_values), through the C ABI: the map is built from a full
A-LLS assembly; re-assembly after moving the nodes and changing the materials
must match the oracle's assembly of the new mesh within 1e-12 on the
row/column scale, in the same pattern."""
import numpy as np
import pytest

from conftest import value_errors

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _perturbed(m, seed):
    rng = np.random.default_rng(seed)
    m2 = __import__("copy").copy(m)
    # a small fraction of the element size, so that no element inverts
    size = (np.max(m.x) - np.min(m.x)) / (np.cbrt(m.num_elems) if m.z is not None else np.sqrt(m.num_elems))
    h = 1e-2 * size
    m2.x = m.x + rng.uniform(-h, h, m.x.shape)
    m2.y = m.y + rng.uniform(-h, h, m.y.shape)
    if m.z is not None:
        m2.z = m.z + rng.uniform(-h, h, m.z.shape)
    if m.E is not None:  # per-element materials change too
        m2.E = m.E * rng.uniform(0.5, 2.0, m.num_elems)
    return m2


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small", "t3"])
def test_reassembly_after_moving_nodes(fem, oracle_mod, cuda_device, name):
    import torch
    import meshgen as mg
    m = mg.by_name(name)
    asm = fem.Assembler(m)
    rp, ci, v, info = asm.assemble()
    nnz = int(info.nnz)
    re = fem.Reassembler(asm)
    re.build(nnz)
    vals = torch.empty(nnz, dtype=torch.float64, device=rp.device)
    # same coordinates: the values of the full assembly
    re.reassemble(vals)
    assert re.read_info() == 0
    orp, oci, ov = oracle_mod.assemble(m)
    rel, scaled = value_errors(orp, oci, ov, vals.cpu().numpy())
    assert scaled <= RTOL, scaled
    # moved nodes, new materials: swap the device arrays in place and re-assemble
    m2 = _perturbed(m, 5)
    for k, arr in fem.host_arrays(m2).items():
        asm.dev[k].copy_(torch.from_numpy(arr))
    re.reassemble(vals)
    assert re.read_info() == 0
    orp2, oci2, ov2 = oracle_mod.assemble(m2)
    np.testing.assert_array_equal(orp2, orp)
    rel, scaled = value_errors(orp2, oci2, ov2, vals.cpu().numpy())
    print(f"{name}: re-assembly max scaled error {scaled:.2e}")
    assert scaled <= RTOL, scaled


@pytest.mark.parametrize("name", ["t3_small", "mixed_small"])
def test_fp32_reassembly(fem, oracle_mod, cuda_device, name):
    # value-only re-assembly with the FP32 blocks of the 2-D kinds
    import torch
    import meshgen as mg
    m = mg.by_name(name)
    asm = fem.Assembler(m)
    rp, ci, v, info = asm.assemble()
    nnz = int(info.nnz)
    re = fem.Reassembler(asm)
    re.build(nnz)
    vals = torch.empty(nnz, dtype=torch.float64, device=rp.device)
    re.reassemble(vals, fem.opts(precision=fem.FEM_PREC_FP32))
    assert re.read_info() == 0
    orp, oci, ov = oracle_mod.assemble(m)
    rel, scaled = value_errors(orp, oci, ov, vals.cpu().numpy())
    print(f"{name}: FP32 re-assembly max scaled error {scaled:.2e}")
    assert scaled <= 1e-5, scaled
