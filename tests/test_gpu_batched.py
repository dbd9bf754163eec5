"""Batched assembly (fem_assemble_batched) through the C ABI: every mesh of a
batch of all element kinds and uneven sizes must come out as if assembled
alone (pattern bit-exact and values within 1e-12 of the oracle), with the
per-mesh info words and completion stamps filled in; also captured in a CUDA
graph and replayed."""
import numpy as np
import pytest

from conftest import value_errors

pytestmark = pytest.mark.gpu


def _small_batch():
    import meshgen as mg
    return mg.batch_meshes(12, seed=7, emin=20, emax=600)


@pytest.mark.parametrize("concurrency", [1, 3])
def test_batch_matches_oracle(fem, oracle_mod, cuda_device, concurrency):
    import torch
    meshes = _small_batch()
    assert len({m.kind for m in meshes}) >= 3
    b = fem.Batch(meshes, concurrency=concurrency)
    nnz = b.sizes()
    b.run()
    torch.cuda.synchronize()
    assert all(s == 0 for s in b.statuses())
    for i, m in enumerate(meshes):
        rp, ci, v = b.result(i)
        orp, oci, ov = oracle_mod.assemble(m)
        np.testing.assert_array_equal(rp, orp)
        np.testing.assert_array_equal(ci, oci)
        assert nnz[i] == oci.shape[0]
        rel, scaled = value_errors(orp, oci, ov, v)
        assert scaled <= 1e-12, (m.name, scaled)
    lat = b.latencies_ms()
    assert np.all(lat > 0) and np.all(lat < 1e4)


def test_batch_in_cuda_graph(fem, oracle_mod, cuda_device):
    import torch
    meshes = _small_batch()
    b = fem.Batch(meshes, concurrency=4)
    b.sizes()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.run()  # warm-up outside the capture (first use sets up the library streams)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    for v in b.values:
        v.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b.run()
    g.replay()
    torch.cuda.synchronize()
    assert all(st == 0 for st in b.statuses())
    for i, m in enumerate(meshes):
        rp, ci, v = b.result(i)
        orp, oci, ov = oracle_mod.assemble(m)
        np.testing.assert_array_equal(ci, oci)
        rel, scaled = value_errors(orp, oci, ov, v)
        assert scaled <= 1e-12
