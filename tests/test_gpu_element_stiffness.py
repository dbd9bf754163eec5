"""fem_element_stiffness: every element's Ke on its own, through the C ABI,
against the oracle's element functions (restated from the reference's
computeElementStiffness / computeElementStiffnessHex20), within 1e-12 of the
element's largest diagonal entry."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_ke(oracle_mod, m, e):
    import meshgen as mg
    nodes = m.conn[e]
    E = m.E[e] if m.E is not None else m.E0
    nu = m.nu[e] if m.nu is not None else m.nu0
    if m.kind == mg.HEX20:
        return oracle_mod.ke_hex20(m.x[nodes], m.y[nodes], m.z[nodes], E, nu), 20, 3
    q4 = m.types[e] == mg.Q4 if m.types is not None else m.kind == mg.Q4
    if q4:
        return oracle_mod.ke_q4(m.x[nodes[:4]], m.y[nodes[:4]], E, nu, m.thickness), 4, 2
    return oracle_mod.ke_t3(m.x[nodes[:3]], m.y[nodes[:3]], E, nu, m.thickness), 3, 2


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small"])
def test_element_stiffness_matches_oracle(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    ke, status = fem.element_stiffness(m)
    assert status == 0
    ke = ke.cpu().numpy()
    rng = np.random.default_rng(0)
    for e in rng.choice(m.num_elems, size=min(m.num_elems, 40), replace=False):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        scale = np.max(np.abs(np.diag(ref)))
        err = np.max(np.abs(got - ref)) / scale
        assert err <= 1e-12, f"element {e}: {err:.3e}"
        if m.types is not None and npe == 3:
            assert np.all(ke[e, 24:] == 0.0)


def test_element_stiffness_reports_bad_node(fem, cuda_device):
    import meshgen as mg
    m = mg.by_name("hex20_small")
    m.conn = m.conn.copy()
    m.conn[1, 5] = m.num_nodes + 7
    ke, status = fem.element_stiffness(m)
    assert status & (1 << 2)
    assert np.all(ke[1].cpu().numpy() == 0.0)


# The tensor-core form (FEM_PREC_TC_F16X3): FP16 split operands, FP32
# accumulation of the node-pair contraction, FP64 everywhere else. Its error is
# measured against the FP64 oracle on the element's scale and bounded at the
# north star's 1e-6 (measured: about 5e-7).
TC_ELEMENT_TOL = 1e-6


def test_tensor_core_element_stiffness_error(fem, oracle_mod, cuda_device):
    import meshgen as mg
    m = mg.by_name("hex20_small")
    ke, status = fem.element_stiffness(m, fem.opts(precision=1))
    assert status == 0
    ke = ke.cpu().numpy()
    worst = 0.0
    for e in range(m.num_elems):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        err = np.max(np.abs(got - ref)) / np.max(np.abs(np.diag(ref)))
        worst = max(worst, err)
    print(f"tensor-core Ke: max error {worst:.3e} of the element's largest diagonal entry")
    assert worst <= TC_ELEMENT_TOL


def test_tensor_core_form_rejected_for_2d(fem, cuda_device):
    import meshgen as mg
    with pytest.raises(fem.FemError):
        fem.element_stiffness(mg.by_name("t3_small"), fem.opts(precision=1))


def test_plain_fp64_simt_form_matches_oracle(fem, oracle_mod, cuda_device):
    # FEM_PREC_FP64_SIMT: the same Ke with the contraction as plain FP64 dot
    # products (no tensor cores), the comparison point of the tensor-core forms
    import meshgen as mg
    m = mg.by_name("hex20_small")
    ke, status = fem.element_stiffness(m, fem.opts(precision=2))
    assert status == 0
    ke = ke.cpu().numpy()
    for e in range(m.num_elems):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(np.diag(ref)))
    with pytest.raises(fem.FemError):   # not an assembly precision
        fem.assemble(m, fem.opts(precision=2))


# The FP32 form of the 2-D kinds (FEM_PREC_FP32): each block in FP32 from
# node coordinates relative to the element's first node.
FP32_ELEMENT_TOL = 1e-5


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small"])
def test_fp32_element_stiffness_error(fem, oracle_mod, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    ke, status = fem.element_stiffness(m, fem.opts(precision=fem.FEM_PREC_FP32))
    assert status == 0
    ke = ke.cpu().numpy()
    worst = 0.0
    for e in range(min(m.num_elems, 200)):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        worst = max(worst, np.max(np.abs(got - ref)) / np.max(np.abs(np.diag(ref))))
    print(f"{name} FP32 Ke: max error {worst:.3e} of the element's largest diagonal entry")
    assert worst <= FP32_ELEMENT_TOL
    with pytest.raises(fem.FemError):
        fem.element_stiffness(mg.by_name("hex20_small"), fem.opts(precision=fem.FEM_PREC_FP32))


def _tc_error(fem, oracle_mod, m, ke):
    worst = 0.0
    for e in range(m.num_elems):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        worst = max(worst, np.max(np.abs(got - ref)) / np.max(np.abs(np.diag(ref))))
    return worst


def test_tensor_core_odd_count_and_unaligned_output(fem, oracle_mod, cuda_device):
    # The tensor-core kernel takes elements in pairs: an odd count leaves the
    # last pair half empty. An output that is not 16-byte aligned is written
    # with plain stores instead of the bulk copy; the neighbouring doubles
    # must stay untouched.
    import torch
    import meshgen as mg
    m = mg.by_name("hex20_small")
    k = m.num_elems - 1 if m.num_elems % 2 == 0 else m.num_elems
    m.conn = m.conn[:k].copy()
    if m.E is not None:
        m.E = m.E[:k]
    if m.nu is not None:
        m.nu = m.nu[:k]
    assert k % 2 == 1
    ke, status = fem.element_stiffness(m, fem.opts(precision=1))
    assert status == 0
    assert _tc_error(fem, oracle_mod, m, ke.cpu().numpy()) <= TC_ELEMENT_TOL
    n = ke.shape[1]
    buf = torch.full((k * n + 2,), 7.0, dtype=torch.float64, device=ke.device)
    out = buf[1:1 + k * n].view(k, n)                     # 8 bytes past a 16-byte boundary
    ke2, status = fem.element_stiffness(m, fem.opts(precision=1), out=out)
    assert status == 0
    assert torch.equal(ke2, ke)
    assert buf[0].item() == 7.0 and buf[-1].item() == 7.0


def test_tensor_core_inverted_element(fem, oracle_mod, cuda_device):
    # An element with negative Gauss-point weights (detJ < 0): FEM_ERR_DETJ is
    # raised and its Ke still follows the signed weights (B = A diag(sgn w)).
    import meshgen as mg
    m = mg.hex20_grid(2, seed=3)
    m.conn = m.conn.copy()
    c = m.conn[1]
    # mirror the element in zeta: swap its bottom and top faces (and the edge nodes)
    m.conn[1] = c[[4, 5, 6, 7, 0, 1, 2, 3, 12, 13, 14, 15, 8, 9, 10, 11, 16, 17, 18, 19]]
    ke, status = fem.element_stiffness(m, fem.opts(precision=1))
    assert status & (1 << fem.FEM_ERR_DETJ)
    ke64, status64 = fem.element_stiffness(m)
    assert status64 & (1 << fem.FEM_ERR_DETJ)
    ke, ke64 = ke.cpu().numpy(), ke64.cpu().numpy()
    for e in range(m.num_elems):
        ref, npe, dpn = _oracle_ke(oracle_mod, m, e)
        got = fem.unpack_element_stiffness(ke[e], npe, dpn)
        assert np.max(np.abs(got - ref)) <= TC_ELEMENT_TOL * np.max(np.abs(np.diag(ref))), e
        got64 = fem.unpack_element_stiffness(ke64[e], npe, dpn)
        assert np.max(np.abs(got64 - ref)) <= 1e-12 * np.max(np.abs(np.diag(ref))), e


def test_tensor_core_wait_timeout_is_reported(fem, oracle_mod, cuda_device):
    # The bounded wait of the tensor-core kernels for their own products: with
    # fem_opts.wait_limit_us < 0 the first wait of every CTA counts as run out
    # while its six 128x128x16 products are in flight. The kernel must raise
    # FEM_ERR_TIMEOUT, wait for the products in flight with the default bound
    # (no FEM_ERR_INTERNAL), release its tensor memory and return; the context
    # stays usable and the next call with the default bound is exact.
    import meshgen as mg
    m = mg.by_name("hex20_small")
    ke, status = fem.element_stiffness(m, fem.opts(precision=1, wait_limit_us=-1))
    assert status & (1 << fem.FEM_ERR_TIMEOUT)
    assert not status & (1 << fem.FEM_ERR_INTERNAL)
    ke, status = fem.element_stiffness(m, fem.opts(precision=1))
    assert status == 0
    assert _tc_error(fem, oracle_mod, m, ke.cpu().numpy()) <= TC_ELEMENT_TOL
    # the assembly's tensor-core value pass reports it through the info word
    a = fem.Assembler(m, fem.opts(precision=1, wait_limit_us=-1))
    a.scatter()
    a.consolidate(0)
    st, info = a.read_info()
    assert st == fem.FEM_ERR_TIMEOUT
    assert not info.status_bits & (1 << fem.FEM_ERR_INTERNAL)
    rp, ci, v, info = fem.Assembler(m, fem.opts(precision=1)).assemble()
    assert int(info.status_bits) == 0
