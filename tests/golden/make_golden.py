"""Generates the golden fixtures that pin the oracle to the reference.

The reference ships no fixtures or tests; its only check compares its GPU
values with its serial host assembly (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu
:1061-1186). These fixtures are outputs of the reference's OWN code, built from
its sources by oracle/Makefile into oracle/_ref/:

* ``reference_host.npz`` (run here, CPU): for small meshes of every element kind
  the CSR pattern of the reference's host builders (buildCSRStructure, Q4A:605;
  T3:458; MIX:488; buildCSRStructureHex20, H20:364), including the reference's
  own Hex20 lattice with orphan nodes (generateMeshHex20, H20:324) and the
  reference's accuracy-test mesh (generateMesh 10x100, Q4A:968-969); for Q4 also
  the values of its serial host assembly (assembleGlobalStiffnessHost,
  Q4A:329-380) with the reference's material constants.
* ``reference_device_ke.npz`` (``--gpu``, needs a B200): per-element stiffness of
  the reference's device functions (computeElementStiffness T3:136, MIX:145;
  computeElementStiffnessHex20 H20:130) on small jittered meshes.

    python tests/golden/make_golden.py            # CPU fixtures
    python tests/golden/make_golden.py --gpu OUT  # device fixtures into OUT
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "a-lls-matrix-parallel-assembly_b200"), os.path.join(ROOT, "oracle")]

import meshgen as mg  # noqa: E402
import oracle as O  # noqa: E402


def mesh_dict(prefix, m):
    d = {f"{prefix}/kind": np.int32(m.kind), f"{prefix}/x": m.x, f"{prefix}/y": m.y,
         f"{prefix}/conn": m.conn.astype(np.int32)}
    if m.z is not None:
        d[f"{prefix}/z"] = m.z
    if m.types is not None:
        d[f"{prefix}/types"] = m.types
    return d


def host_fixtures(path):
    E, nu, t = O.ref_q4a_material()
    out = {"material": np.array([E, nu, t])}
    meshes = {name: mg.by_name(name) for name in ("q4_small", "t3_small", "mixed_small", "hex20_small")}
    conn, x, y = O.ref_q4a_generate_mesh(10, 100)
    meshes["q4_ref10x100"] = mg.Mesh(mg.Q4, x, y, None, conn, None, None, None, E0=E, nu0=nu, thickness=t)
    n = 2
    L = 2 * n + 1
    conn = np.zeros(n ** 3 * 20, np.int32)
    xs, ys, zs = (np.zeros(L ** 3) for _ in range(3))
    O.ref_lib("h20").ref_h20_generate_mesh(n, n, n, O._ptr(conn), O._ptr(xs), O._ptr(ys), O._ptr(zs))
    meshes["hex20_ref_lattice2"] = mg.Mesh(mg.HEX20, xs, ys, zs, conn.reshape(-1, 20), None, None, None)
    for name, m in meshes.items():
        rp, ci = O.ref_pattern(m)
        out.update(mesh_dict(name, m))
        out[f"{name}/row_ptr"] = rp
        out[f"{name}/col_idx"] = ci
        if m.kind == mg.Q4:
            out[f"{name}/values_ref_material"] = O.ref_q4a_host_assemble(m, rp, ci)
        print(name, "nodes", m.num_nodes, "elems", m.num_elems, "nnz", ci.shape[0])
    np.savez_compressed(path, **out)


def device_fixtures(path):
    out = {}
    for name, E, nu, t in (("t3_small", 1.0, 0.3, 1.0), ("mixed_small", 2.0, 0.25, 0.5), ("hex20_small", 1.0, 0.3, 1.0)):
        m = mg.by_name(name)
        out.update(mesh_dict(name, m))
        out[f"{name}/material"] = np.array([E, nu, t])
        out[f"{name}/ke"] = O.ref_gpu_element_ke(m, E, nu, t)
        print(name, out[f"{name}/ke"].shape)
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    if "--gpu" in sys.argv:
        dst = sys.argv[sys.argv.index("--gpu") + 1]
        device_fixtures(os.path.join(dst, "reference_device_ke.npz"))
    else:
        host_fixtures(os.path.join(HERE, "reference_host.npz"))
