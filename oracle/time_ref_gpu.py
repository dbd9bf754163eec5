"""Times the reference's own GPU A-LLS assembly of the T3 benchmark mesh on
this GPU, beside this library's assembly of the same mesh (TEST INFRASTRUCTURE:
a comparison measurement, not part of the product path).

    python oracle/time_ref_gpu.py [--size 1000] [--iters 10] [--warmup 3]

The reference side (oracle/_ref/libref_t3.so, built from the reference's source
by oracle/Makefile) runs assembleGlobalStiffnessKernelALLS and
convertALLStoCSRKernel (ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:
227-315) timed as its driver times them (T3:586-640: resets outside the window,
CUDA events, values only, the CSR pattern built on the host beforehand by its
buildCSRStructure, T3:458-482, which is timed separately). The reference's
material is global, so both sides assemble the mesh with uniform E = 1,
nu = 0.3, t = 1 here. Prints one JSON line.
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "a-lls-matrix-parallel-assembly_b200"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=1000)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    import torch
    import fem_alls as fem
    import meshgen as mg
    import oracle

    m = mg.t3_grid(args.size, args.size)
    m.E, m.nu, m.E0, m.nu0, m.thickness = None, None, 1.0, 0.3, 1.0
    conn = np.ascontiguousarray(m.conn, np.int32)
    x, y = np.ascontiguousarray(m.x), np.ascontiguousarray(m.y)

    # the reference's host pattern (its own builder), timed
    L = oracle.ref_lib("t3")
    rp = np.zeros(m.num_dofs + 1, np.int32)
    t0 = time.perf_counter()
    nnz = L.ref_t3_build_csr(m.num_nodes, m.num_elems, 3, conn.ctypes.data, None, None, None, 0)
    ci = np.zeros(nnz, np.int32)
    L.ref_t3_build_csr(m.num_nodes, m.num_elems, 3, conn.ctypes.data, None, rp.ctypes.data, ci.ctypes.data, nnz)
    pattern_s = time.perf_counter() - t0

    f = L.ref_t3_gpu_alls_time
    vp = C.c_void_p
    f.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp,
                  C.c_int64, C.c_int, C.c_int, vp, C.POINTER(C.c_float)]
    f.restype = C.c_int
    ref_vals = np.zeros(nnz, np.float64)
    ms = C.c_float(0.0)
    rc = f(m.num_nodes, m.num_elems, 3, conn.ctypes.data, None, x.ctypes.data, y.ctypes.data, 1.0, 0.3, 1.0,
           rp.ctypes.data, ci.ctypes.data, nnz, args.warmup, args.iters, ref_vals.ctypes.data, C.byref(ms))
    if rc:
        raise RuntimeError(f"reference GPU A-LLS: CUDA error {rc}")

    # this library on the same mesh and material, timed the same way (pattern included)
    asm = fem.Assembler(m)
    orp, oci, ov, info = asm.assemble()
    stream = torch.cuda.current_stream()
    ts = []
    for i in range(args.warmup + args.iters):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        asm.assemble_async()
        b.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            ts.append(a.elapsed_time(b))
    fem.check(asm.read_info()[0], "assembly")
    orp, oci, ov = orp.cpu().numpy(), oci[:nnz].cpu().numpy(), ov[:nnz].cpu().numpy()
    same_pattern = bool(np.array_equal(orp, rp) and np.array_equal(oci, ci))
    # the reference's racy list inserts can drop or duplicate contributions:
    # compare on the row/column scale
    rows = np.repeat(np.arange(m.num_dofs), np.diff(rp))
    d = np.zeros(m.num_dofs)
    on = rows == ci
    d[rows[on]] = np.abs(ov[on])
    scale = np.maximum(np.abs(ov), np.sqrt(d[rows] * d[ci]))
    scale[scale == 0] = 1.0
    diff = float(np.max(np.abs(ref_vals - ov) / scale))
    ours = float(np.mean(ts))
    print(json.dumps({
        "workload": m.name, "elements": m.num_elems, "nnz": int(nnz),
        "reference_gpu_alls_ms": ms.value,
        "reference_host_pattern_s": pattern_s,
        "reference_total_ms": ms.value + 1e3 * pattern_s,
        "ours_ms": ours, "speedup_vs_reference_kernels": ms.value / ours,
        "speedup_vs_reference_total": (ms.value + 1e3 * pattern_s) / ours,
        "same_pattern": same_pattern, "max_scaled_diff_reference_vs_ours": diff,
        "what": "reference: assembleGlobalStiffnessKernelALLS + convertALLStoCSRKernel, values only, pattern "
                "prebuilt on the host (its timing window); ours: full device assembly with the pattern; "
                "uniform material on both sides",
    }))


if __name__ == "__main__":
    main()
