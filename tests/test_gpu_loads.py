"""Load vector and Dirichlet conditions (fem_assemble_body_force,
fem_apply_dirichlet) through the C ABI, against numpy restatements of the
same integrals and of symmetric elimination."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G2 = 0.577350269189626
G3 = (-0.774596669241483, 0.0, 0.774596669241483)
W3 = (0.555555555555556, 0.888888888888889, 0.555555555555556)


def _hex20_N(xi, eta, zeta):
    import meshgen as mg
    off = mg.HEX20_OFFSETS  # lattice offsets (0..2) of the 20 nodes in reference order
    a, b, c = off[:, 0] - 1, off[:, 1] - 1, off[:, 2] - 1
    N = np.empty(20)
    for n in range(20):
        if n < 8:
            N[n] = 0.125 * (1 + a[n] * xi) * (1 + b[n] * eta) * (1 + c[n] * zeta) * (a[n] * xi + b[n] * eta + c[n] * zeta - 2)
        elif a[n] == 0:
            N[n] = 0.25 * (1 - xi * xi) * (1 + b[n] * eta) * (1 + c[n] * zeta)
        elif b[n] == 0:
            N[n] = 0.25 * (1 + a[n] * xi) * (1 - eta * eta) * (1 + c[n] * zeta)
        else:
            N[n] = 0.25 * (1 + a[n] * xi) * (1 + b[n] * eta) * (1 - zeta * zeta)
    return N


def _ref_body_force(m, b):
    import meshgen as mg
    dim = 3 if m.kind == mg.HEX20 else 2
    f = np.zeros(m.num_dofs)
    for e in range(m.num_elems):
        be = b[e] if b.ndim == 2 else b
        nodes = m.conn[e]
        if m.kind == mg.HEX20:
            X = np.stack([m.x[nodes], m.y[nodes], m.z[nodes]], 1)
            w = np.zeros(20)
            for i, xi in enumerate(G3):
                for j, eta in enumerate(G3):
                    for k, zeta in enumerate(G3):
                        dN = mg.hex20_shape_derivs(xi, eta, zeta)  # [3, 20]
                        J = dN @ X
                        w += _hex20_N(xi, eta, zeta) * np.linalg.det(J) * W3[i] * W3[j] * W3[k]
            for a in range(20):
                f[3 * nodes[a]:3 * nodes[a] + 3] += w[a] * be
            continue
        q4 = (m.types[e] == mg.Q4) if m.types is not None else m.kind == mg.Q4
        if not q4:
            n3 = nodes[:3]
            x, y = m.x[n3], m.y[n3]
            A = 0.5 * ((x[1] - x[0]) * (y[2] - y[0]) - (y[1] - y[0]) * (x[2] - x[0]))
            for a in range(3):
                f[2 * n3[a]:2 * n3[a] + 2] += A / 3 * be * m.thickness
            continue
        x, y = m.x[nodes[:4]], m.y[nodes[:4]]
        w = np.zeros(4)
        for xi in (-G2, G2):
            for eta in (-G2, G2):
                N = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
                dxi = 0.25 * np.array([-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)])
                deta = 0.25 * np.array([-(1 - xi), -(1 + xi), 1 + xi, 1 - xi])
                J = np.array([[dxi @ x, dxi @ y], [deta @ x, deta @ y]])
                w += N * np.linalg.det(J)
        for a in range(4):
            f[2 * nodes[a]:2 * nodes[a] + 2] += w[a] * be * m.thickness
    return f


@pytest.mark.parametrize("name", ["q4_small", "t3_small", "mixed_small", "hex20_small"])
def test_body_force(fem, cuda_device, name):
    import meshgen as mg
    m = mg.by_name(name)
    dim = 3 if m.kind == mg.HEX20 else 2
    b_uni = np.array([0.3, -1.0, 0.5][:dim])
    f, st = fem.body_force(m, b_uni)
    assert st == 0
    ref = _ref_body_force(m, b_uni)
    np.testing.assert_allclose(f.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    # total force = b * volume (partition of unity)
    vol_ref = ref.reshape(-1, dim).sum(0)
    assert np.allclose(f.cpu().numpy().reshape(-1, dim).sum(0), vol_ref, rtol=1e-12)
    rng = np.random.default_rng(3)
    b_el = rng.normal(size=(m.num_elems, dim))
    f, st = fem.body_force(m, b_el)
    ref = _ref_body_force(m, b_el)
    np.testing.assert_allclose(f.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", ["q4_small", "hex20_small"])
def test_dirichlet_symmetric_elimination(fem, cuda_device, name):
    import torch
    import meshgen as mg
    m = mg.by_name(name)
    asm = fem.Assembler(m)
    rp, ci, v, info = asm.assemble()
    rp_h, ci_h, v_h = rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy().copy()
    n = m.num_dofs
    rng = np.random.default_rng(1)
    fixed = (rng.random(n) < 0.2).astype(np.uint8)
    u = rng.normal(size=n)
    f0 = rng.normal(size=n)
    f = torch.from_numpy(f0.copy()).cuda()
    vals = v.clone()
    fem.apply_dirichlet(rp, ci, vals, f, torch.from_numpy(fixed).cuda(), torch.from_numpy(u).cuda())
    # reference: dense symmetric elimination
    K = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp_h))
    K[rows, ci_h] = v_h
    fx = fixed.astype(bool)
    f_ref = f0 - K[:, fx] @ u[fx]
    f_ref[fx] = u[fx]
    K[fx, :] = 0.0
    K[:, fx] = 0.0
    K[np.where(fx)[0], np.where(fx)[0]] = 1.0
    got = vals.cpu().numpy()
    np.testing.assert_array_equal(got, K[rows, ci_h])
    np.testing.assert_allclose(f.cpu().numpy(), f_ref, rtol=1e-12, atol=1e-12 * np.abs(f_ref).max())
    # symmetric up to the last bits of the assembled input (FP64 atomics add a
    # block's contributions in arrival order, so K_ij and K_ji can differ there)
    Kg = np.zeros((n, n))
    Kg[rows, ci_h] = got
    np.testing.assert_allclose(Kg, Kg.T, rtol=0, atol=1e-14 * np.abs(Kg).max())
    assert np.array_equal(Kg == 0, Kg.T == 0)
