"""The autotuner (fem_autotune, fem_autotune_batched) through the C ABI: it
must return one of its candidate shapes, and the assembly it leaves behind
(with the chosen options) must match the oracle like any other: pattern
bit-exact, values within 1e-12 on the row/column scale. The scatter-grid
option it tunes (fem_opts.ctas_per_sm) must not change the result."""
import numpy as np
import pytest

from conftest import value_errors

pytestmark = pytest.mark.gpu


def _check(fem, oracle_mod, m, rp, ci, v):
    orp, oci, ov = oracle_mod.assemble(m)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    rel, scaled = value_errors(orp, oci, ov, v)
    assert scaled <= 1e-12, scaled


@pytest.mark.parametrize("name", ["t3_small", "mixed_small", "hex20_small"])
def test_autotune_single_mesh(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    asm = fem.Assembler(m)
    asm.assemble()
    best, ms = asm.autotune(repeats=2)
    assert ms > 0.0
    assert best.ctas_per_sm in (0, 1, 2, 3)
    if m.kind == mg.HEX20:
        assert best.first_slots in (94, 62, 46) and best.chunk_slots == 30
    print(f"{name}: first_slots {best.first_slots}, ctas_per_sm {best.ctas_per_sm}, {ms:.3f} ms")
    st, info = asm.read_info()
    assert st == 0
    nz = int(info.nnz)
    _check(fem, oracle_mod, m, asm.row_ptr.cpu().numpy(), asm.col_idx[:nz].cpu().numpy(),
           asm.values[:nz].cpu().numpy())
    # the adopted options keep working for later assemblies
    rp, ci, v, info = asm.assemble()
    _check(fem, oracle_mod, m, rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy())


@pytest.mark.parametrize("ctas", [1, 2])
def test_scatter_grid_option(fem, oracle_mod, cuda_device, ctas):
    import meshgen as mg
    for name in ("t3_small", "hex20_small"):
        m = mg.by_name(name)
        rp, ci, v, info = fem.assemble(m, fem.opts(ctas_per_sm=ctas))
        _check(fem, oracle_mod, m, rp, ci, v)
    with pytest.raises(fem.FemError):
        fem.assemble(mg.by_name("t3_small"), fem.opts(ctas_per_sm=-1))


def test_autotune_batched(fem, oracle_mod, cuda_device):
    import torch
    import meshgen as mg
    meshes = mg.batch_meshes(10, seed=9, emin=20, emax=500)
    b = fem.Batch(meshes, concurrency=16)
    b.sizes()
    k, ms = b.autotune(repeats=1)
    assert k in (1, 2, 4, 8, 16) and k <= len(meshes) and ms > 0.0
    torch.cuda.synchronize()
    assert all(s == 0 for s in b.statuses())
    for i, m in enumerate(meshes):
        rp, ci, v = b.result(i)
        _check(fem, oracle_mod, m, rp, ci, v)
