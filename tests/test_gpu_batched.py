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
        b.run()  # warm-up outside the capture
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


def _sampled_rows_ok(oracle_mod, m, rp, ci, v, rows=256, seed=0):
    """Hex20 mesh of a batch, checked on a sample of row nodes: each sampled
    row's columns against the sorted dofs of every node sharing an element with
    it (built here in numpy), and its values against the serial oracle's
    assembly of those rows alone. Returns the worst value error scaled by the
    largest sampled entry."""
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0) and rp[-1] == ci.shape[0]
    nodes = np.random.default_rng(seed).choice(m.num_nodes, min(rows, m.num_nodes), replace=False)
    conn = np.asarray(m.conn, np.int64)
    flat = conn.ravel()
    order = np.argsort(flat, kind="stable")
    first = np.searchsorted(flat[order], nodes)
    last = np.searchsorted(flat[order], nodes, side="right")
    for n, a, b in zip(nodes, first, last):
        elems = order[a:b] // conn.shape[1]
        nbr = np.unique(conn[elems])
        want = (3 * nbr[:, None] + np.arange(3)[None, :]).ravel()
        for d in range(3):
            r = 3 * n + d
            np.testing.assert_array_equal(ci[rp[r]:rp[r + 1]], want)
    ov = oracle_mod.assemble_rows(m, rp, ci, nodes)
    sel = np.zeros(m.num_dofs, bool)
    for d in range(3):
        sel[3 * nodes + d] = True
    ent = np.repeat(sel, np.diff(rp))
    scale = np.abs(ov[ent]).max()
    return float(np.max(np.abs(v[ent] - ov[ent])) / scale)


def test_batch_256_configuration(fem, oracle_mod, cuda_device):
    # The batched configuration itself: 256 meshes of every kind, 1k-200k
    # elements each, 16 workspace slots (16 rounds). 2-D meshes are checked in
    # full, Hex20 meshes by pattern and sampled rows.
    import torch
    import meshgen as mg
    meshes = mg.batch_meshes(256, seed=5)
    b = fem.Batch(meshes, concurrency=16)
    b.sizes()
    b.run()
    torch.cuda.synchronize()
    st = b.statuses()
    assert all(s == 0 for s in st), [i for i, s in enumerate(st) if s]
    worst = 0.0
    for i, m in enumerate(meshes):
        rp, ci, v = b.result(i)
        if m.kind == mg.HEX20:
            worst = max(worst, _sampled_rows_ok(oracle_mod, m, rp, ci, v, seed=i))
        else:
            orp, oci, ov = oracle_mod.assemble(m)
            np.testing.assert_array_equal(rp, orp)
            np.testing.assert_array_equal(ci, oci)
            rel, scaled = value_errors(orp, oci, ov, v)
            worst = max(worst, scaled)
    print(f"256-mesh batch: worst error {worst:.3e}")
    assert worst <= 1e-12
    lat = b.latencies_ms()
    assert np.all(lat > 0)


def test_batch_calls_on_two_threads(fem, oracle_mod, cuda_device):
    # Two batched calls at once from two host threads: one captured into a
    # CUDA graph on its stream, one running on another stream; each uses only
    # its own workspace, so both come out right.
    import threading
    import torch
    meshes = _small_batch()
    b1 = fem.Batch(meshes, concurrency=4)
    b2 = fem.Batch(meshes, concurrency=2)
    b1.sizes()
    b2.sizes()
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    errors = []

    def captured():
        try:
            with torch.cuda.stream(s1):
                with torch.cuda.graph(g, stream=s1, capture_error_mode="thread_local"):
                    b1.run()
        except Exception as e:  # reported below
            errors.append(e)

    def plain():
        try:
            with torch.cuda.stream(s2):
                for _ in range(3):
                    b2.run()
        except Exception as e:
            errors.append(e)

    t1, t2 = threading.Thread(target=captured), threading.Thread(target=plain)
    t1.start()
    t2.start()
    t1.join()
    t2.join()
    assert not errors, errors
    g.replay()
    torch.cuda.synchronize()
    for b in (b1, b2):
        assert all(s == 0 for s in b.statuses())
        for i, m in enumerate(meshes):
            rp, ci, v = b.result(i)
            orp, oci, ov = oracle_mod.assemble(m)
            np.testing.assert_array_equal(ci, oci)
            assert value_errors(orp, oci, ov, v)[1] <= 1e-12
