"""The oracle pinned against the reference's own code (CPU).

Golden vectors come from tests/golden/reference_host.npz (outputs of the
reference's host functions built from its sources, see make_golden.py) and,
where the reference harness is built in this checkout, from calling it
directly. Known-answer tests are derived from the mathematics.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

HOST_NPZ = os.path.join(GOLDEN, "reference_host.npz")


def _mesh(npz, name):
    import meshgen as mg
    kind = int(npz[f"{name}/kind"])
    z = npz[f"{name}/z"] if f"{name}/z" in npz else None
    types = npz[f"{name}/types"] if f"{name}/types" in npz else None
    return mg.Mesh(kind, npz[f"{name}/x"], npz[f"{name}/y"], z, npz[f"{name}/conn"], types, None, None)


@pytest.fixture(scope="module")
def golden():
    return np.load(HOST_NPZ)


NAMES = ["q4_small", "t3_small", "mixed_small", "hex20_small", "q4_ref10x100", "hex20_ref_lattice2"]


@pytest.mark.parametrize("name", NAMES)
def test_pattern_matches_reference_golden(oracle_mod, golden, name):
    m = _mesh(golden, name)
    rp, ci = oracle_mod.pattern(m)
    np.testing.assert_array_equal(rp, golden[f"{name}/row_ptr"])
    np.testing.assert_array_equal(ci, golden[f"{name}/col_idx"])


@pytest.mark.parametrize("name", ["q4_small", "q4_ref10x100"])
def test_q4_values_bitwise_equal_reference_host_assembly(oracle_mod, golden, name):
    E, nu, t = golden["material"]
    m = _mesh(golden, name)
    _, _, v = oracle_mod.assemble(m, golden[f"{name}/row_ptr"], golden[f"{name}/col_idx"], E0=E, nu0=nu, thickness=t)
    np.testing.assert_array_equal(v, golden[f"{name}/values_ref_material"])
    prec = oracle_mod.precision(golden[f"{name}/values_ref_material"], v)
    assert prec["count_gt_1e-10"] == 0 and prec["max_abs"] == 0.0


DEVICE_NPZ = os.path.join(GOLDEN, "reference_device_ke.npz")


@pytest.mark.parametrize("name,bound", [("t3_small", 1e-14), ("mixed_small", 1e-14), ("hex20_small", 5e-6)])
def test_element_stiffness_matches_reference_device_functions(oracle_mod, name, bound):
    # Per-element Ke of the reference's own device functions (computeElementStiffness
    # T3:136 and MIX:145 in FP64, computeElementStiffnessHex20 H20:130 in FP32) on
    # jittered meshes, generated on a B200 by make_golden.py --gpu. The error is
    # measured against sqrt(|K_ii K_jj|); the Hex20 bound is the reference's FP32.
    g = np.load(DEVICE_NPZ)
    E, nu, t = g[f"{name}/material"]
    conn, x, y = g[f"{name}/conn"], g[f"{name}/x"], g[f"{name}/y"]
    worst = 0.0
    for e in range(conn.shape[0]):
        c = conn[e]
        if name == "hex20_small":
            k = oracle_mod.ke_hex20(x[c], y[c], g[f"{name}/z"][c], E, nu)
            r = g[f"{name}/ke"][e].astype(np.float64)
        elif name == "mixed_small" and g[f"{name}/types"][e] == 0:
            k = oracle_mod.ke_q4(x[c], y[c], E, nu, t)
            r = g[f"{name}/ke"][e]
        else:
            k = oracle_mod.ke_t3(x[c[:3]], y[c[:3]], E, nu, t)
            r = g[f"{name}/ke"][e][:6, :6]
        d = np.sqrt(np.abs(np.diag(k)))
        worst = max(worst, float(np.max(np.abs(k - r) / np.outer(d, d))))
    assert worst <= bound, worst


def test_hex20_reference_lattice_has_orphan_rows(golden):
    rp = golden["hex20_ref_lattice2/row_ptr"]
    empty = int(np.sum(np.diff(rp) == 0))
    # 5^3 lattice: face- and body-centre points (odd count >= 2) own no element.
    assert empty == 3 * (125 - 81)


def test_q4_unit_square_known_answer(oracle_mod):
    # Plane-stress unit-square Q4, corner diagonal entry: E t (3 - nu) / (6 (1 - nu^2)).
    E, nu, t = 2.1e11, 0.3, 0.01
    ke = oracle_mod.ke_q4([0, 1, 1, 0], [0, 0, 1, 1], E, nu, t)
    assert ke[0, 0] == pytest.approx(E * t * (3 - nu) / (6 * (1 - nu * nu)), rel=1e-14)
    np.testing.assert_allclose(ke, ke.T, rtol=0, atol=1e-12 * np.abs(ke).max())


def test_t3_right_triangle_known_answer(oracle_mod):
    # CST on (0,0),(1,0),(0,1), t=1: K = A * B^T D B with A = 1/2.
    E, nu = 1.0, 0.25
    ke = oracle_mod.ke_t3([0, 1, 0], [0, 0, 1], E, nu, 1.0)
    f = E / (1 - nu * nu)
    D = f * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
    B = np.array([[-1, 0, 1, 0, 0, 0], [0, -1, 0, 0, 0, 1], [-1, -1, 0, 1, 1, 0]], float)
    np.testing.assert_allclose(ke, 0.5 * B.T @ D @ B, rtol=1e-14, atol=1e-15)


def _rigid_modes_2d(x, y):
    n = len(x)
    tx = np.tile([1.0, 0.0], n)
    ty = np.tile([0.0, 1.0], n)
    rz = np.ravel(np.column_stack([-np.asarray(y), np.asarray(x)]))
    return [tx, ty, rz]


def _rigid_modes_3d(x, y, z):
    n = len(x)
    X = np.column_stack([x, y, z])
    modes = []
    for d in range(3):
        u = np.zeros((n, 3))
        u[:, d] = 1
        modes.append(u.ravel())
    for a, b in ((0, 1), (1, 2), (2, 0)):
        u = np.zeros((n, 3))
        u[:, a] = -X[:, b]
        u[:, b] = X[:, a]
        modes.append(u.ravel())
    return modes


def test_element_rigid_body_null_space_and_symmetry(oracle_mod):
    rng = np.random.default_rng(7)
    xq = np.array([0, 1, 1, 0]) + rng.uniform(-0.1, 0.1, 4)
    yq = np.array([0, 0, 1, 1]) + rng.uniform(-0.1, 0.1, 4)
    kq = oracle_mod.ke_q4(xq, yq, 3.0, 0.3, 0.7)
    xt, yt = np.array([0, 1.1, 0.2]), np.array([0.1, 0, 0.9])
    kt = oracle_mod.ke_t3(xt, yt, 3.0, 0.3, 0.7)
    for ke, x, y in ((kq, xq, yq), (kt, xt, yt)):
        np.testing.assert_allclose(ke, ke.T, rtol=0, atol=1e-13 * np.abs(ke).max())
        for u in _rigid_modes_2d(x, y):
            assert np.abs(ke @ u).max() < 1e-12 * np.abs(ke).max() * np.abs(u).max()
        assert np.all(np.linalg.eigvalsh(ke)[3:] > 0)   # exactly 3 zero-energy modes
    import meshgen as mg
    m = mg.hex20_grid(1, seed=3, jitter=0.3)   # a single distorted element; all nodes on the boundary
    rng = np.random.default_rng(8)
    x = m.x + rng.uniform(-0.04, 0.04, m.num_nodes)
    y = m.y + rng.uniform(-0.04, 0.04, m.num_nodes)
    z = m.z + rng.uniform(-0.04, 0.04, m.num_nodes)
    c = m.conn[0]
    kh = oracle_mod.ke_hex20(x[c], y[c], z[c], 2.0, 0.3)
    np.testing.assert_allclose(kh, kh.T, rtol=0, atol=1e-13 * np.abs(kh).max())
    for u in _rigid_modes_3d(x[c], y[c], z[c]):
        assert np.abs(kh @ u).max() < 1e-12 * np.abs(kh).max() * max(1.0, np.abs(u).max())


def test_hex20_patch_uniform_strain(oracle_mod):
    # A linear displacement field u = A x gives constant stress; on an undistorted
    # cube the nodal forces K u sum to zero per direction (self-equilibrated).
    import meshgen as mg
    m = mg.hex20_grid(1, jitter=0.0)
    c = m.conn[0]
    kh = oracle_mod.ke_hex20(m.x[c], m.y[c], m.z[c], 1.0, 0.3)
    A = np.array([[0.01, 0.002, 0], [0.002, -0.003, 0.001], [0, 0.001, 0.004]])
    X = np.column_stack([m.x[c], m.y[c], m.z[c]])
    f = (kh @ (X @ A.T).ravel()).reshape(20, 3)
    np.testing.assert_allclose(f.sum(axis=0), 0, atol=1e-14)
    # E x (uniaxial strain energy) check: u^T K u = volume * eps : C : eps
    lam, mu = 1.0 * 0.3 / (1.3 * 0.4), 1.0 / 2.6
    eps = 0.5 * (A + A.T)
    energy = lam * np.trace(eps) ** 2 + 2 * mu * np.sum(eps * eps)
    u = (X @ A.T).ravel()
    assert u @ kh @ u == pytest.approx(energy, rel=1e-12)


def test_precision_statistics(oracle_mod):
    ref = np.array([1.0, -2.0, 0.0, 4.0])
    test = np.array([1.0, -2.002, 1e-3, 4.0])
    p = oracle_mod.precision(ref, test)
    assert p["max_abs"] == pytest.approx(0.002)
    assert p["max_rel"] == pytest.approx(0.001)
    assert p["count_gt_1e-10"] == 2


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libref_t3.so")),
                    reason="reference harness not built in this checkout")
@pytest.mark.parametrize("name", ["q4", "t3_small", "mixed_small", "hex20_small"])
def test_pattern_matches_reference_live(oracle_mod, name):
    import meshgen as mg
    m = mg.by_name(name)
    rp, ci = oracle_mod.pattern(m)
    rrp, rci = oracle_mod.ref_pattern(m)
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(ci, rci)
