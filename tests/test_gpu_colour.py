"""The element-colouring baseline (fem_colour_*), through the C ABI.

The colouring must be valid (no two elements of one colour share a node) and
the coloured assembly must give the same FP64 values as the oracle (1e-12 on
the row/column scale, as the A-LLS path) in the pattern the A-LLS path built.
The reference's coloured kernels run all colours at once and race
(ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:504-572); this one is correct.
"""
import numpy as np
import pytest

from conftest import diag_scale

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _valid_colouring(mesh, colours):
    npe = mesh.nodes_per_elem()
    for k in range(mesh.stride):
        has = npe > k
        nodes = mesh.conn[has, k].astype(np.int64)
        pairs = nodes * 64 + colours[has]
        if k == 0:
            allp = pairs
        else:
            allp = np.concatenate([allp, pairs])
    # each (node, colour) pair may occur once: elements sharing a node differ in colour
    assert np.unique(allp).shape[0] == allp.shape[0], "two elements of one colour share a node"


def _run(fem, oracle_mod, mesh):
    import torch
    asm = fem.Assembler(mesh)
    rp, ci, v, info = asm.assemble()
    nnz = int(info.nnz)
    col = fem.Colouring(mesh, dev_arrays=asm.dev)
    nc = col.prepare()
    colours = col.colours.cpu().numpy()[: mesh.num_elems]
    assert 0 < nc <= 64 and colours.max() == nc - 1 and colours.min() >= 0
    _valid_colouring(mesh, colours)
    vals = torch.empty(nnz, dtype=torch.float64, device=rp.device)
    col.assemble(rp, ci, vals, nnz)
    st, nc2 = col.read_info()
    assert st == 0 and nc2 == nc
    orp, oci, ov = oracle_mod.assemble(mesh)
    np.testing.assert_array_equal(rp.cpu().numpy(), orp)
    vc = vals.cpu().numpy()
    scale = np.maximum(np.abs(ov), diag_scale(orp, oci, ov))
    bad = np.abs(vc - ov) > RTOL * scale
    assert not bad.any(), f"{bad.sum()} coloured values off"
    return nc


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "q4"])
def test_coloured_assembly_matches_oracle(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    nc = _run(fem, oracle_mod, mg.by_name(name))
    print(f"{name}: {nc} colours")


def test_fan_needs_one_colour_per_triangle(fem, oracle_mod, cuda_device):
    from test_gpu_parity import _fan_mesh
    m = _fan_mesh(40)
    assert _run(fem, oracle_mod, m) >= 40


def test_too_many_colours_is_range_error(fem, cuda_device):
    from test_gpu_parity import _fan_mesh
    m = _fan_mesh(70)   # 70 triangles share node 0: 70 colours > 64
    col = fem.Colouring(m)
    with pytest.raises(fem.FemError) as e:
        col.prepare()
    assert "RANGE" in str(e.value)


def test_hex20_coloured_assembly_matches_oracle(fem, oracle_mod, cuda_device):
    import meshgen as mg
    nc = _run(fem, oracle_mod, mg.by_name("hex20_small"))
    assert nc >= 8  # a structured hex grid needs at least 8 colours (2x2x2 parity)
