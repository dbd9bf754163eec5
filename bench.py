"""Benchmark of the FEM global-stiffness assembly (A-LLS path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload hex20|t3|q4|mixed|batched]
                    [--impl ours|reference]

A step is one full device assembly of a seeded synthetic mesh: list reset,
element order, element stiffness + A-LLS list scatter, and list -> CSR
consolidation (pattern and FP64 values), inputs resident in HBM. The default
workload is the Hex20 64^3 configuration (1,085,825 nodes, 262,144 elements,
557,286,921 CSR nonzeros). ``value`` is elements/s over the whole job; nnz/s,
the rooflines, the accuracy of every CSR value against the serial FP64 oracle,
the end-to-end figure through the host-buffer C ABI entry point (host<->device
copies inside the timed region), the tensor-core Ke form, the colouring
baseline, the value-only re-assembly, the T3 1000^2 and 256-mesh batched
configurations and a CPU baseline are added to the same JSON line. With
--gpus N > 1 (one process per GPU under torchrun) every rank assembles its own
replica (the path has no exchange step): weak scaling, headline fields only.

``--impl reference`` runs the reference's own code for the same workload on
the full configuration: its host CSR pattern builder (buildCSRStructureHex20,
ALLS_Hex20_3D_Assembly_Performance.cu:364-392, compiled from the reference
sources into oracle/_ref) plus the serial FP64 value scatter of
assembleGlobalStiffnessHost (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:329-380,
the reference's own function for Q4, the oracle's restatement of it for the
other element kinds, which the reference has no host assembly for), one core,
pattern and values timed separately; and, in a `reference_gpu` field, the
reference's GPU kernels on the same mesh and GPU, timed by the reference's own
compareAssemblyMethods (H20:421-543).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "a-lls-matrix-parallel-assembly_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

WORKLOADS = {
    "q4": ("q4_100x100", "Q4 plane stress 100x100 unit square, jitter 0.1h, E=1, nu=0.3, t=1, natural order"),
    "t3": ("t3_1000x1000", "T3 1000x1000 grid, random diagonals, jitter 0.2h, shuffled, E~LogNormal(0,0.5), nu=0.3"),
    "mixed": ("mixed_1500x1500", "Q4+T3 1500x1500 grid (p_Q4=0.5), jitter 0.15h, shuffled, E~LogNormal(0,0.5), nu~U[0.2,0.4]"),
    "hex20": ("hex20_64x64x64", "Hex20 64^3 compact serendipity mesh, jitter 0.05h, E=1, nu=0.3, 3x3x3 Gauss"),
    "batched": ("batched_256", "256 independent meshes, kind uniform over {Q4, T3, mixed, Hex20}, elements "
                "log-uniform over 1k-200k, each kind's jitter and material distributions"),
}
DEFAULT_WORKLOAD = "hex20"
L2_BYTES = 126 * 2 ** 20
L2_NOTE = ("a buffer of 2x L2 (252 MB) is zeroed between timed steps, outside the step events; the Hex20 64^3 "
           "step also moves 24.6 GB of algorithmic traffic, far above L2")
METRIC = "elements/s (device FP64 A-LLS assembly: element stiffness, list scatter, CSR pattern + values)"
SCATTER_KERNEL = {"q4": "k_scatter_2d<4>", "t3": "k_scatter_2d<3>", "mixed": "k_scatter_2d<4> + k_scatter_2d<3>",
                  "hex20": "k_claim_hex20 + k_values_group (two-pass list scatter by element groups, in waves)"}


def make_mesh(workload: str, size: int = 0, **kw):
    import meshgen as mg
    if size:
        kw = {"nx": size} if workload == "hex20" else {"nx": size, "ny": size}
    if workload == "q4":
        return mg.q4_grid(**kw) if kw else mg.q4_grid(100, 100)
    if workload == "t3":
        return mg.t3_grid(**kw) if kw else mg.t3_grid(1000, 1000)
    if workload == "mixed":
        return mg.mixed_grid(**kw) if kw else mg.mixed_grid(1500, 1500)
    if workload == "hex20":
        return mg.hex20_grid(**kw) if kw else mg.hex20_grid(64)
    raise ValueError(workload)


def workload_config(workload: str, mesh, nnz: int, world: int, sized: bool = False) -> dict:
    """The configuration both arms report (identical keys and values); `sized`:
    a smaller instance of the generator (--size), named by its mesh."""
    name, desc = WORKLOADS[workload]
    return {"workload": mesh.name if sized else name, "description": desc, "elements": mesh.num_elems,
            "nodes": mesh.num_nodes, "dofs": mesh.num_dofs, "nnz": int(nnz), "l2": L2_NOTE,
            "parallelism": f"replicas{world}"}


def algorithmic_bytes(mesh, nnz: int) -> dict:
    """Algorithmic bytes of one assembly: inputs, CSR output and the A-LLS list
    entries written once and read once (16 B each way per nnz)."""
    dim = 3 if mesh.z is not None else 2
    conn = int(np.sum(mesh.nodes_per_elem())) * 4
    b_in = mesh.num_nodes * dim * 8 + conn + mesh.num_elems * 16 + (mesh.num_elems if mesh.types is not None else 0)
    b_out = 4 * (mesh.num_dofs + 1) + 12 * nnz
    b_list = 32 * nnz
    return {"in": b_in, "out": b_out, "list": b_list, "total": b_in + b_out + b_list}


def job_ms(local_ms: float, world: int, device) -> float:
    """Time of the whole job: the maximum over the ranks of each rank's device
    time (weak scaling: every rank did the same amount of work)."""
    if world <= 1:
        return float(local_ms)
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def measured_peaks() -> dict:
    """Denominators of the rooflines: MEASURED_PEAKS.json when present, else the
    profiling recipe's fallback figures."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d.get("bf16_tflops", 1590.0)),
                "kind": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "kind": "fallback"}


def host_info() -> dict:
    model = platform.processor() or ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def library_identity(path: str) -> dict:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return {"path": os.path.relpath(path, ROOT), "sha256": h.hexdigest()}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# The serial FP64 oracle (CPU baseline and accuracy reference)
# ---------------------------------------------------------------------------

def oracle_full(mesh) -> dict:
    """The serial FP64 host assembly of the whole mesh by the oracle (pattern,
    then values), each phase timed; one core."""
    import oracle as O
    t0 = time.perf_counter()
    rp, ci = O.pattern(mesh)
    t1 = time.perf_counter()
    _, _, v = O.assemble(mesh, rp, ci)
    t2 = time.perf_counter()
    return {"row_ptr": rp, "col_idx": ci, "values": v, "pattern_s": t1 - t0, "values_s": t2 - t1}


def cpu_baseline_line(mesh, orc: dict) -> dict:
    total = orc["pattern_s"] + orc["values_s"]
    return {"value": mesh.num_elems / total, "unit": "elements/s", "cores": 1, "kind": "port",
            "sample": f"the full configuration ({mesh.num_elems} elements): the oracle's serial restatement of "
                      f"the reference's host pattern build and assembleGlobalStiffnessHost, one thread; pattern "
                      f"{orc['pattern_s']:.2f} s, values {orc['values_s']:.2f} s",
            "pattern_s": orc["pattern_s"], "values_s": orc["values_s"], **host_info()}


def _diag_positions(rp: np.ndarray, ci: np.ndarray) -> np.ndarray:
    """Position of the diagonal entry of every row (vectorised binary search)."""
    n = rp.shape[0] - 1
    dofs = np.arange(n, dtype=np.int64)
    lo, hi = rp[:-1].astype(np.int64), rp[1:].astype(np.int64) - 1
    for _ in range(40):
        act = lo <= hi
        if not act.any():
            break
        mid = (lo + hi) // 2
        less = ci[np.clip(mid, 0, max(ci.shape[0] - 1, 0))] < dofs
        lo = np.where(act & less, mid + 1, lo)
        hi = np.where(act & ~less, mid - 1, hi)
    return lo


def accuracy(rp: np.ndarray, ci: np.ndarray, ref: np.ndarray, test: np.ndarray, chunk: int = 1 << 26) -> dict:
    """Error of every CSR value `test` against the FP64 oracle `ref` (same
    pattern), as the reference's analyzePrecision states it
    (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:896-960: max / mean absolute and
    relative error over the nonzero reference entries, Frobenius-relative error,
    count of |diff| > 1e-10), plus the error on the row/column scale
    max(|K_ij|, sqrt(|K_ii K_jj|)) and the per-entry relative error of the
    entries that do not cancel between elements (|K_ij| >= 1e-8 sqrt(|K_ii K_jj|))."""
    dpos = _diag_positions(rp, ci)
    diag = np.abs(ref[np.clip(dpos, 0, max(ref.shape[0] - 1, 0))]) if ref.shape[0] else np.zeros(0)
    nnz = ref.shape[0]
    out = {"max_abs": 0.0, "max_rel": 0.0, "sum_abs": 0.0, "sum_rel": 0.0, "fro_d": 0.0, "fro_ref": 0.0,
           "count_gt_1e-10": 0, "max_scaled": 0.0, "max_rel_significant": 0.0, "significant": 0}
    for s in range(0, nnz, chunk):
        e = min(nnz, s + chunk)
        idx = np.arange(s, e, dtype=np.int64)
        rows = np.searchsorted(rp, idx, side="right") - 1
        r, t = ref[s:e], test[s:e]
        d = np.abs(t - r)
        nz = r != 0
        rel = d[nz] / np.abs(r[nz])
        out["max_abs"] = max(out["max_abs"], float(d[nz].max()) if nz.any() else 0.0)
        out["max_rel"] = max(out["max_rel"], float(rel.max()) if rel.size else 0.0)
        out["sum_abs"] += float(d[nz].sum())
        out["sum_rel"] += float(rel.sum())
        out["fro_d"] += float(np.sum((t[nz] - r[nz]) ** 2))
        out["fro_ref"] += float(np.sum(r * r))
        out["count_gt_1e-10"] += int(np.count_nonzero(d > 1e-10))
        sc = np.sqrt(diag[rows] * diag[ci[s:e]])
        out["max_scaled"] = max(out["max_scaled"], float(np.max(d / np.maximum(np.abs(r), np.where(sc > 0, sc, 1.0)))))
        sig = np.abs(r) >= 1e-8 * sc
        if sig.any():
            out["max_rel_significant"] = max(out["max_rel_significant"], float(np.max(d[sig] / np.abs(r[sig]))))
        out["significant"] += int(np.count_nonzero(sig))
    return {"max_rel": out["max_rel"], "mean_rel": out["sum_rel"] / max(nnz, 1), "max_abs": out["max_abs"],
            "mean_abs": out["sum_abs"] / max(nnz, 1),
            "frobenius_rel": (out["fro_d"] ** 0.5) / (out["fro_ref"] ** 0.5) if out["fro_ref"] > 0 else 0.0,
            "count_gt_1e-10": out["count_gt_1e-10"], "max_scaled": out["max_scaled"],
            "max_rel_significant": out["max_rel_significant"], "significant_entries": out["significant"],
            "entries": int(nnz),
            "what": "every CSR value against the serial FP64 oracle: analyzePrecision's statistics (max_rel over "
                    "nonzero entries, mean_rel, frobenius_rel, count_gt_1e-10), max_scaled = max |d| / "
                    "max(|K_ij|, sqrt(|K_ii K_jj|)), max_rel_significant = max |d| / |K_ij| over entries with "
                    "|K_ij| >= 1e-8 sqrt(|K_ii K_jj|)"}


# ---------------------------------------------------------------------------
# GPU legs
# ---------------------------------------------------------------------------

def timed_steps(torch, stream, flush, fn, steps: int, warmup: int = 0):
    """Mean device milliseconds of fn over `steps` calls (CUDA events on the
    launching stream, L2 flushed before each, outside the events)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.mean(ts)


def run_batched(args, rank: int, world: int, local_rank: int, compact: bool = False):
    """The batched configuration: 256 meshes assembled by fem_assemble_batched
    (one call per step, graph-captured), concurrency picked by the library's
    autotuner (fem_autotune_batched: 1/2/4/8/16 slots timed on this batch);
    concurrency 1 is the sequential baseline (the same per-mesh launches one
    after another on one stream). value = elements/s of the whole batch.
    compact: return the fields as a dict (the default line's batched field)."""
    import torch
    import fem_alls as fem
    import meshgen as mg
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    name, desc = WORKLOADS["batched"]
    t0 = time.perf_counter()
    meshes = mg.batch_meshes(256, seed=5 + rank)
    gen_s = time.perf_counter() - t0
    elems = sum(m.num_elems for m in meshes)
    b = fem.Batch(meshes, concurrency=16, device=dev)
    nnz = b.sizes()
    t0 = time.perf_counter()
    best, tune_ms = b.autotune(repeats=1)
    tune_s = time.perf_counter() - t0
    slots = (1, best) if best != 1 else (1,)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        ts = []
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            z = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            z.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(z))
        return ts

    per_k = {}
    for k in slots:
        for _ in range(args.warmup):
            b.run(k)
        torch.cuda.synchronize()
        ts = timed(lambda: b.run(k), args.steps)
        lat = b.latencies_ms()
        per_k[k] = {"ms": statistics.mean(ts), "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99))}
    # the chosen concurrency captured in a CUDA graph and replayed
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        b.run(best)
    stream.wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b.run(best)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local_rank) as clk:
        ts = timed(g.replay, args.steps)
    st = b.statuses()
    bad = [i for i, v in enumerate(st) if v & ~(1 << 4)]
    if bad:
        raise RuntimeError(f"batched assembly: status bits {st[bad[0]]} on mesh {bad[0]}")
    lat = b.latencies_ms()
    ms = job_ms(sum(ts), world, dev) / args.steps
    del g
    if rank != 0:
        return None
    seq = per_k[1]
    fields = {
        "value": world * elems / (ms / 1e3), "unit": "elements/s", "ms_per_step": ms,
        "meshes_per_s": world * len(meshes) / (ms / 1e3),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "what": "per-mesh completion after the batch start (GPU global timer), graph replay"},
        "concurrency": {"chosen": best, "timed": {str(k): v for k, v in per_k.items()},
                        "autotune": {"api": "fem_autotune_batched (1, 2, 4, 8, 16 slots)", "best_ms": tune_ms,
                                     "tuning_s": tune_s}},
        "sequential": {"ms": seq["ms"], "meshes_per_s": len(meshes) / (seq["ms"] / 1e3),
                       "p50_ms": seq["p50_ms"], "p99_ms": seq["p99_ms"],
                       "what": "the 256 meshes' launches one after another on one stream (concurrency 1)"},
        "speedup_vs_sequential": seq["ms"] / ms,
        "meshes": len(meshes), "elements": elems, "nnz": int(sum(nnz)),
        "kinds": {k: sum(1 for m in meshes if m.kind == k) for k in range(4)}, "mesh_generation_s": gen_s,
        "clocks": clk.summary(), "gpu_launches": args.steps * batch_launches(meshes),
        "api": "fem_assemble_batched, captured in one CUDA graph",
    }
    if compact:
        return fields
    line = {"metric": METRIC, "value": fields["value"], "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh generator)",
            "config": {"workload": name, "description": desc, "meshes": len(meshes), "elements": elems,
                       "nnz": int(sum(nnz)), "l2": L2_NOTE, "parallelism": f"replicas{world}"}}
    line.update({k: v for k, v in fields.items() if k not in line})
    print(json.dumps(line), flush=True)
    return None


def assembly_leg(torch, fem, mesh, dev, stream, flush, steps: int, warmup: int, o=None, clocks: bool = False,
                 world: int = 1, local_rank: int = 0):
    """Timed full assemblies (scatter phase and consolidation split by events);
    returns (assembler, info, dict of times)."""
    asm = fem.Assembler(mesh, o, device=dev)
    _, _, _, info = asm.assemble()          # sizes the outputs
    for _ in range(warmup):
        asm.assemble_async()
    torch.cuda.synchronize()
    st, info = asm.read_info()
    fem.check(st, "warmup assembly")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    mids = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank) if clocks else None
    if clk:
        clk.__enter__()
    try:
        for i in range(steps):
            flush.zero_()                      # evict L2 between steps (outside the step events)
            starts[i].record(stream)
            asm.scatter()                      # = fem_assemble_async, split to time the scatter phase
            mids[i].record(stream)
            asm.consolidate()
            stops[i].record(stream)
        torch.cuda.synchronize()
    finally:
        if clk:
            clk.__exit__()
    if world > 1:
        torch.distributed.barrier()
    times = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    st, info = asm.read_info()
    fem.check(st, "timed assembly")
    t = {"total_ms_sum": sum(times), "ms": statistics.mean(times),
         "scatter_ms": statistics.mean(s.elapsed_time(e) for s, e in zip(starts, mids)),
         "consolidate_ms": statistics.mean(s.elapsed_time(e) for s, e in zip(mids, stops)),
         "clocks": clk.summary() if clk else None}
    return asm, info, t


def rooflines(mesh, nnz: int, t: dict, peak: dict, workload: str) -> dict:
    ab = algorithmic_bytes(mesh, nnz)
    hbm = peak["hbm_gbs"]
    # scatter phase: reads the inputs, writes every list entry once (16 B per
    # CSR nonzero); consolidation reads the entries back and writes the CSR
    scatter_bytes = ab["in"] + ab["list"] // 2
    consolidate_bytes = ab["list"] // 2 + ab["out"]
    sg = scatter_bytes / (t["scatter_ms"] / 1e3) / 1e9
    cg = consolidate_bytes / (t["consolidate_ms"] / 1e3) / 1e9
    step = ab["total"] / (t["ms"] / 1e3) / 1e9
    return {
        "roofline": {"bound": "hbm", "achieved": sg, "peak": hbm, "unit": "GB/s", "frac": sg / hbm,
                     "traffic": read_profile_traffic(workload), "peak_kind": peak["kind"],
                     "kernel": SCATTER_KERNEL.get(workload, "") + " (scatter phase: list reset, element order, scatter)",
                     "algorithmic_bytes_per_launch": scatter_bytes,
                     "algorithmic_bytes_per_element": scatter_bytes / max(mesh.num_elems, 1),
                     "ms_per_launch": t["scatter_ms"]},
        "consolidate_roofline": {"bound": "hbm", "achieved": cg, "peak": hbm, "unit": "GB/s", "frac": cg / hbm,
                                 "kernel": "k_write (consolidation phase: count, scan, sorted write)",
                                 "algorithmic_bytes_per_launch": consolidate_bytes, "ms_per_launch": t["consolidate_ms"]},
        "step_roofline": {"achieved": step, "frac": step / hbm, "algorithmic_bytes": ab,
                          "frac_nominal_8tbs": step / 8000.0,
                          "compulsory_frac": (ab["in"] + ab["out"]) / (t["ms"] / 1e3) / 1e9 / hbm},
    }


def e2e_leg(torch, fem, mesh, nnz, stream, flush, steps: int, warmup: int, world: int, dev):
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in fem.host_arrays(mesh).items()}
    harr = {k: v.numpy() for k, v in pinned.items()}
    rp = torch.empty(mesh.num_dofs + 1, dtype=torch.int32).pin_memory().numpy()
    ci = torch.empty(nnz, dtype=torch.int32).pin_memory().numpy()
    vv = torch.empty(nnz, dtype=torch.float64).pin_memory().numpy()
    ctx = fem.HostContext()
    s = stream.cuda_stream
    for _ in range(max(1, warmup)):
        fem.check(ctx.assemble(mesh, harr, rp, ci, vv, stream=s)[0], "fem_assemble_host")
    torch.cuda.synchronize()
    e_times = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fem.check(ctx.assemble(mesh, harr, rp, ci, vv, stream=s)[0], "fem_assemble_host")
        b.record(stream)
        b.synchronize()
        e_times.append(a.elapsed_time(b))
    ctx.close()
    e_ms = job_ms(sum(e_times), world, dev) / steps
    h2d = sum(v.nbytes for v in harr.values())
    d2h = rp.nbytes + ci.nbytes + vv.nbytes
    return {"value": world * mesh.num_elems / (e_ms / 1e3), "unit": "elements/s", "ms_per_step": e_ms,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "api": "fem_assemble_host (pinned host buffers, copies inside the call)"}


def ke_form(fem, torch, mesh, dev_arrays, args, flush, stream, peak: dict) -> dict:
    """The Hex20 element stiffness on its own (fem_element_stiffness) in its
    three forms (FP64 tensor cores, FP16-split tensor cores, plain FP64 on the
    CUDA cores), timed alike; the tensor-core values are compared with the FP64
    ones per element, on the scale of the element's largest diagonal entry."""
    out = {}
    kes = {}
    for prec, name in ((0, "fp64"), (1, "tc_f16x3"), (2, "fp64_simt")):
        o = fem.opts(precision=prec)
        ke, st = fem.element_stiffness(mesh, o, dev_arrays=dev_arrays)
        fem.check(0 if st == 0 else 1, f"element stiffness {name}")
        out[name + "_ms"] = timed_steps(torch, stream, flush,
                                        lambda: fem.element_stiffness(mesh, o, dev_arrays=dev_arrays, out=ke),
                                        args.steps, args.warmup)
        kes[name] = ke
    # diagonal entries of the packed upper blocks: block (I, I) entries 0, 4, 8
    diag_idx = [9 * (i * 20 - i * (i - 1) // 2) + v for i in range(20) for v in (0, 4, 8)]
    d = kes["fp64"][:, diag_idx].abs().max(dim=1).values
    err = ((kes["tc_f16x3"] - kes["fp64"]).abs().max(dim=1).values / d).max()
    flops = 2 * 60 * 60 * 27 * mesh.num_elems  # the node-pair contraction (dense, one pass)
    # three FP16 products per split contraction, 64 x 64 x 32 padded tiles of the tensor pipe
    tc_flops = 3 * 2 * 64 * 64 * 32 * mesh.num_elems
    out.update({"speedup_tc_vs_fp64": out["fp64_ms"] / out["tc_f16x3_ms"],
                "speedup_tc_vs_fp64_simt": out["fp64_simt_ms"] / out["tc_f16x3_ms"],
                "forms": "fp64: contraction on the FP64 tensor cores (the library's default); tc_f16x3: FP16 split "
                         "operands on the FP16 tensor cores (tcgen05); fp64_simt: plain FP64 dot products on the "
                         "CUDA cores",
                "max_err_tc_vs_fp64": float(err),
                "err_scale": "per element, max |difference| / the element's largest diagonal entry",
                "contraction_gflop": flops / 1e9,
                "tensor_pipe": {"issued_tflop_per_s": tc_flops / (out["tc_f16x3_ms"] / 1e3) / 1e12,
                                "peak_tflops": peak["bf16_tflops"], "peak_kind": peak["kind"],
                                "utilisation": tc_flops / (out["tc_f16x3_ms"] / 1e3) / 1e12 / peak["bf16_tflops"],
                                "what": "3 split products x 2 x 64 x 64 x 32 (padded) flops per element / Ke time / "
                                        "dense 16-bit tensor peak"},
                "bytes_written": int(kes["fp64"].numel() * 8),
                "write_floor_ms": kes["fp64"].numel() * 8 / (peak["hbm_gbs"] * 1e6),
                "what": "fem_element_stiffness: packed symmetric Ke (210 3x3 blocks, 15.1 KB) of every element"})
    return out


def fp32_form(fem, torch, asm, mesh, nnz, args, flush, stream, ref_values) -> dict:
    """The whole A-LLS assembly with the FP32 Ke blocks of the 2-D kinds
    (FEM_PREC_FP32), timed like the FP64 step; its values are compared with
    the FP64 oracle."""
    o64 = asm.opts
    asm.opts = fem.opts(precision=fem.FEM_PREC_FP32)
    try:
        ms = timed_steps(torch, stream, flush, lambda: (asm.scatter(), asm.consolidate()), args.steps, args.warmup)
        st, _ = asm.read_info()
        fem.check(st, "FP32-form assembly")
        rp = asm.row_ptr.cpu().numpy()
        acc = accuracy(rp, asm.col_idx[:nnz].cpu().numpy(), ref_values, asm.values[:nnz].cpu().numpy())
    finally:
        asm.opts = o64
        asm.assemble()                         # leave the FP64 values in place
    return {"value": mesh.num_elems / (ms / 1e3), "unit": "elements/s", "ms_per_step": ms, "accuracy": acc,
            "what": "fem_alls_scatter + fem_alls_consolidate with FEM_PREC_FP32 (Ke blocks in FP32 from "
                    "coordinates relative to the element's first node, FP64 accumulation)"}


def tc_assembly(fem, torch, mesh, dev, args, flush, stream, fp64_ms, ref_values) -> dict:
    """The whole Hex20 A-LLS assembly with the tensor-core Ke form
    (FEM_PREC_TC_F16X3), timed like the FP64 step, every value compared with
    the FP64 oracle."""
    o = fem.opts(precision=fem.FEM_PREC_TC_F16X3)
    asm, info, t = assembly_leg(torch, fem, mesh, dev, stream, flush, args.steps, args.warmup, o)
    nnz = int(info.nnz)
    acc = accuracy(asm.row_ptr.cpu().numpy(), asm.col_idx[:nnz].cpu().numpy(), ref_values,
                   asm.values[:nnz].cpu().numpy()) if ref_values is not None else None
    del asm
    torch.cuda.empty_cache()
    return {"value": mesh.num_elems / (t["ms"] / 1e3), "unit": "elements/s", "ms_per_step": t["ms"],
            "scatter_ms": t["scatter_ms"], "consolidate_ms": t["consolidate_ms"],
            "speedup_vs_fp64_assembly": fp64_ms / t["ms"], "accuracy": acc,
            "what": "fem_alls_scatter + fem_alls_consolidate with FEM_PREC_TC_F16X3 (the Ke contraction on the "
                    "FP16 tensor cores from split operands, FP32 accumulation; Jacobians and the global "
                    "accumulation in FP64)"}


def upper_output(fem, torch, asm, mesh, nnz, args, flush, stream) -> dict:
    """The consolidation into the upper triangle (fem_alls_consolidate_upper)
    of the same lists, timed like the full consolidation phase."""
    asm.scatter()
    rp, ci, v = asm.consolidate_upper()
    cap = int(ci.numel())
    ms = timed_steps(torch, stream, flush, lambda: fem.check(asm.lib.fem_alls_consolidate_upper(
        fem.C.byref(asm.cm), fem.C.byref(asm.opts), asm.ws_ptr, asm.ws_bytes, fem._ptr(rp), fem._ptr(ci),
        fem._ptr(v), cap, stream.cuda_stream), "fem_alls_consolidate_upper"), args.steps, args.warmup)
    st, info = asm.read_info()
    fem.check(st, "upper-triangle consolidation")
    unz = int(info.nnz)
    del rp, ci, v
    asm.assemble()                             # leave the full form in place
    return {"ms": ms, "nnz_upper": unz, "nnz_full": nnz, "bytes_out": 4 * (mesh.num_dofs + 1) + 12 * unz,
            "what": "fem_alls_consolidate_upper: count of columns >= row per node, scan, upper part of each "
                    "sorted row (symmetric storage)"}


def reassembly(fem, torch, asm, mesh, nnz, args, flush, stream) -> dict:
    """Value-only re-assembly of the same mesh into the pattern of the A-LLS
    assembly through a scatter map (built once, timed apart): per step the
    values are zeroed and every element block is added at its mapped position."""
    re = fem.Reassembler(asm)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    re.build(nnz)
    b.record(stream)
    torch.cuda.synchronize()
    build_ms = a.elapsed_time(b)
    vals = torch.empty(nnz, dtype=torch.float64, device=asm.row_ptr.device)
    ms = timed_steps(torch, stream, flush, lambda: re.reassemble(vals), args.steps, args.warmup)
    fem.check(re.read_info(), "re-assembly")
    v_alls = asm.values[:nnz]
    diff = 0.0
    for s in range(0, nnz, 1 << 26):
        e = min(nnz, s + (1 << 26))
        diff = max(diff, float(((vals[s:e] - v_alls[s:e]).abs() / v_alls[s:e].abs().clamp_min(1e-300)).max()))
    del vals, re
    torch.cuda.empty_cache()
    return {"value": mesh.num_elems / (ms / 1e3), "unit": "elements/s", "ms_per_step": ms, "map_build_ms": build_ms,
            "max_rel_diff_vs_alls_nonzero": diff,
            "what": "fem_reassemble_values: values zeroed, element blocks added at scatter-map positions (FP64 "
                    "atomics); no lists, no pattern build"}


def colour_baseline(fem, torch, asm, mesh, nnz, args, flush, stream) -> dict:
    """The rebuilt element-colouring path on the same mesh and GPU: device
    colouring (timed once, it syncs the host every round), then K assemblies of
    the values into the A-LLS pattern, one launch per colour, no atomics."""
    col = fem.Colouring(mesh, dev_arrays=asm.dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nc = col.prepare()
    prep_ms = (time.perf_counter() - t0) * 1e3
    rp, ci = asm.row_ptr, asm.col_idx
    vals = torch.empty(nnz, dtype=torch.float64, device=rp.device)
    ms = timed_steps(torch, stream, flush, lambda: col.assemble(rp, ci, vals, nnz), args.steps, args.warmup)
    st, _ = col.read_info()
    fem.check(st, "colour assembly")
    # agreement with the A-LLS values of the same pattern, relative to the largest entry
    v_alls = asm.values[:nnz]
    vmax = float(v_alls.abs().max())
    diff = 0.0
    for s in range(0, nnz, 1 << 26):
        e = min(nnz, s + (1 << 26))
        diff = max(diff, float((vals[s:e] - v_alls[s:e]).abs().max()) / vmax)
    del vals, col
    torch.cuda.empty_cache()
    return {"num_colours": nc, "prepare_ms": prep_ms, "assemble_ms": ms,
            "value": mesh.num_elems / (ms / 1e3), "unit": "elements/s (values into the A-LLS pattern; colouring "
            "and pattern excluded, as the reference times its coloured kernel)",
            "max_diff_vs_alls_of_max_entry": diff,
            "kernels": ("k_values_hex20<kToCsrColour>" if mesh.kind == 2 else "k_colour_assemble_2d") +
                       ", one launch per colour and element type"}


def autotune_leg(asm, ms) -> dict:
    t0 = time.perf_counter()
    best, best_ms = asm.autotune(repeats=3)
    return {"api": "fem_autotune (scatter grid CTAs/SM; Hex20 also first/overflow chunk slots)",
            "best": {"ctas_per_sm": best.ctas_per_sm, "first_slots": best.first_slots,
                     "chunk_slots": best.chunk_slots, "pool_factor": best.pool_factor},
            "best_ms": best_ms, "default_ms": ms, "tuning_s": time.perf_counter() - t0,
            "note": "timed back to back without the L2 flush; the headline uses the default options"}


def secondary_workload(torch, fem, workload: str, dev, stream, flush, args, peak) -> dict:
    """A compact record of another configuration (same step, same timing)."""
    mesh = make_mesh(workload)
    asm, info, t = assembly_leg(torch, fem, mesh, dev, stream, flush, args.steps, args.warmup)
    nnz = int(info.nnz)
    r = rooflines(mesh, nnz, t, peak, workload)
    del asm
    torch.cuda.empty_cache()
    return {"workload": WORKLOADS[workload][0], "value": mesh.num_elems / (t["ms"] / 1e3), "unit": "elements/s",
            "ms_per_step": t["ms"], "nnz": nnz, "nnz_per_s": nnz / (t["ms"] / 1e3),
            "scatter_ms": t["scatter_ms"], "consolidate_ms": t["consolidate_ms"],
            "roofline_frac": r["roofline"]["frac"], "consolidate_frac": r["consolidate_roofline"]["frac"],
            "step_frac": r["step_roofline"]["frac"]}


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import fem_alls as fem
    import build
    if os.environ.get("FEM_ALLS_LIB"):
        raise SystemExit("bench.py times the library built from this tree only: unset FEM_ALLS_LIB")
    lib_path = build.build()
    if args.workload == "batched":
        run_batched(args, rank, world, local_rank)
        return
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    peak = measured_peaks()
    if args.ke_only:
        mesh = make_mesh("hex20", args.size)
        flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
        line = {"workload": mesh.name, "elements": mesh.num_elems,
                "ke_form": ke_form(fem, torch, mesh, fem.device_arrays(mesh, dev), args, flush,
                                   torch.cuda.current_stream(), peak)}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    mesh = make_mesh(args.workload, args.size)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    asm, info, t = assembly_leg(torch, fem, mesh, dev, stream, flush, args.steps, args.warmup, clocks=True,
                                world=world, local_rank=local_rank)
    nnz = int(info.nnz)
    ms = job_ms(t["total_ms_sum"], world, dev) / args.steps
    t["ms"] = ms
    extras = world == 1 and not args.headline_only
    e2e = None if args.no_e2e else e2e_leg(torch, fem, mesh, nnz, stream, flush, args.steps, args.warmup, world, dev)
    line_extra = {}
    orc = None
    if extras:
        if not args.no_colour:
            line_extra["colour_baseline"] = colour_baseline(fem, torch, asm, mesh, nnz, args, flush, stream)
        if not args.no_reassembly:
            line_extra["reassembly"] = reassembly(fem, torch, asm, mesh, nnz, args, flush, stream)
            line_extra["upper_output"] = upper_output(fem, torch, asm, mesh, nnz, args, flush, stream)
        if not args.no_cpu:
            orc = oracle_full(mesh)            # the CPU baseline and the accuracy reference at once
            rp_h = asm.row_ptr.cpu().numpy()
            ci_h = asm.col_idx[:nnz].cpu().numpy()
            if not (np.array_equal(rp_h, orc["row_ptr"]) and np.array_equal(ci_h, orc["col_idx"])):
                raise RuntimeError("CSR pattern differs from the oracle's")
            del ci_h
            line_extra["accuracy"] = accuracy(orc["row_ptr"], orc["col_idx"], orc["values"],
                                              asm.values[:nnz].cpu().numpy())
            line_extra["accuracy"]["pattern"] = "bit-exact (row_ptr and col_idx equal to the oracle's)"
        if mesh.kind == 2 and not args.no_ke:
            line_extra["ke_form"] = ke_form(fem, torch, mesh, asm.dev, args, flush, stream, peak)
            line_extra["tc_assembly"] = tc_assembly(fem, torch, mesh, dev, args, flush, stream, ms,
                                                    orc["values"] if orc else None)
        if mesh.kind != 2 and not args.no_ke and orc:
            line_extra["fp32_form"] = fp32_form(fem, torch, asm, mesh, nnz, args, flush, stream, orc["values"])
        if not args.no_autotune:
            line_extra["autotune"] = autotune_leg(asm, ms)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": world * mesh.num_elems / (ms / 1e3), "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator)",
        "config": workload_config(args.workload, mesh, nnz, world, bool(args.size)),
        "nnz_per_s": world * nnz / (ms / 1e3),
    }
    line.update(rooflines(mesh, nnz, t, peak, args.workload))
    line["kernels_ms"] = {"scatter": t["scatter_ms"], "consolidate": t["consolidate_ms"]}
    line["list"] = {"entries": int(info.list_entries), "unique": nnz // mesh.dpn ** 2,
                    "max_row_entries": int(info.max_row_entries), "overflow_chunks": int(info.overflow_chunks)}
    line["clocks"] = t["clocks"]
    line["gpu_launches"] = kernels_per_step(args.workload, mesh) * args.steps
    line["library"] = library_identity(lib_path)
    if e2e:
        line["e2e"] = e2e
    line.update(line_extra)
    if orc:
        line["cpu_baseline"] = cpu_baseline_line(mesh, orc)
    del asm
    torch.cuda.empty_cache()
    if extras and args.workload == DEFAULT_WORKLOAD and not args.no_secondary and not args.size:
        line["t3_1000x1000"] = secondary_workload(torch, fem, "t3", dev, stream, flush, args, peak)
        line["batched_256"] = run_batched(args, rank, world, local_rank, compact=True)
    print(json.dumps(line), flush=True)


def kernels_per_step(workload: str, mesh) -> int:
    """Library kernels launched by one assembly step."""
    if workload == "hex20":
        waves = (mesh.num_elems + 32767) // 32768
        # k_info_init, k_bbox_init, k_bbox, Morton key count / bucket scan / scatter;
        # node -> element incidence (count, tile sums, tile scan, tile apply, fill);
        # claim + value pass per wave; k_consolidate_reset, k_scan_reduce,
        # k_scan_tiles, k_row_ptr, k_write (the launch list of one step)
        return 6 + 5 + 2 * waves + 5
    return {"q4": 10, "t3": 10, "mixed": 11}[workload]


def batch_launches(meshes) -> int:
    """Library kernels of one fem_assemble_batched call: the copies of the mesh
    descriptors (96 a launch) and of the schedule (700 segments a launch; a
    mesh's segments: reset, 2-D scatter or a claim and a value segment per
    4,096-element Hex20 wave, scan tiles, top scan, row pointers, write,
    finish), the start kernel (counters, ticket, start stamp) and the
    persistent kernel."""
    segs = sum(6 + 2 * ((m.num_elems + 4095) // 4096) if m.kind == 2 else 7 for m in meshes)
    return -(-len(meshes) // 96) + -(-segs // 700) + 2


def read_profile_traffic(workload: str):
    """DRAM bytes (read + write) of one scatter-phase launch on this workload,
    from the committed ncu summary, if there is one."""
    p = os.path.join(ROOT, "profiles", f"traffic_{workload}.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get("dram_bytes_per_launch")
        except (ValueError, OSError):
            return None
    return None


# ---------------------------------------------------------------------------
# The reference arm
# ---------------------------------------------------------------------------

def reference_gpu(workload: str, mesh, rp, ci, ref_values) -> dict:
    """The reference's own GPU kernels on the same mesh, on this GPU, through
    the harness built from its sources (oracle/_ref), timed as its driver times
    them; their values compared with the FP64 oracle on the row/column scale."""
    import ctypes as C
    import oracle as O
    vp = C.c_void_p
    if workload == "hex20":
        L = O.ref_lib("h20")
        f = L.ref_h20_gpu_compare
        f.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, vp, vp, vp, C.c_int64]
        f.restype = C.c_int
        out = np.zeros(8)
        nnz = ci.shape[0]
        va = np.zeros(nnz, np.float32)
        vc = np.zeros(nnz, np.float32)
        conn = np.ascontiguousarray(mesh.conn, np.int32)
        xs = [np.ascontiguousarray(a) for a in (mesh.x, mesh.y, mesh.z)]
        rc = f(mesh.num_nodes, mesh.num_elems, conn.ctypes.data, xs[0].ctypes.data, xs[1].ctypes.data,
               xs[2].ctypes.data, float(mesh.E0), float(mesh.nu0), out.ctypes.data, va.ctypes.data, vc.ctypes.data,
               nnz)
        if rc:
            return {"unavailable": f"reference harness CUDA error {rc}"}
        acc_a = accuracy(rp, ci, ref_values, va.astype(np.float64))
        acc_c = accuracy(rp, ci, ref_values, vc.astype(np.float64))
        return {"alls_ms": out[0], "coloured_ms": out[1], "host_pattern_ms": out[2], "host_colouring_ms": out[3],
                "colours": int(out[4]), "nnz": int(out[5]), "alls_row_array_bytes": int(out[7]),
                "alls_value": mesh.num_elems / (out[0] / 1e3), "coloured_value": mesh.num_elems / (out[1] / 1e3),
                "alls_total_ms_with_host_pattern": out[0] + out[2],
                "coloured_total_ms_with_host_pattern_and_colouring": out[1] + out[2] + out[3],
                "alls_max_scaled_err_vs_fp64": acc_a["max_scaled"],
                "coloured_max_scaled_err_vs_fp64": acc_c["max_scaled"],
                "what": "assembleGlobalStiffnessKernelALLSFixedArray + convertALLStoCSRKernelFixedArray and "
                        "assembleGlobalStiffnessKernelColoredNoAtomic (ALLS_Hex20_3D_Assembly_Performance.cu:"
                        "208-321), timed by the reference's compareAssemblyMethods (3 warm-up, 10 measured, CUDA "
                        "events, values only: the CSR pattern is built on the host beforehand and timed apart); "
                        "FP32 values, as the reference computes them"}
    if workload == "t3":
        L = O.ref_lib("t3")
        f = L.ref_t3_gpu_alls_time
        f.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp,
                      C.c_int64, C.c_int, C.c_int, vp, C.POINTER(C.c_float)]
        f.restype = C.c_int
        vals = np.zeros(ci.shape[0])
        ms = C.c_float(0.0)
        conn = np.ascontiguousarray(mesh.conn, np.int32)
        x, y = np.ascontiguousarray(mesh.x), np.ascontiguousarray(mesh.y)
        # the reference's material is global: uniform-material copy of the mesh
        rc = f(mesh.num_nodes, mesh.num_elems, 3, conn.ctypes.data, None, x.ctypes.data, y.ctypes.data, 1.0, 0.3,
               1.0, rp.ctypes.data, ci.ctypes.data, ci.shape[0], 3, 10, vals.ctypes.data, C.byref(ms))
        if rc:
            return {"unavailable": f"reference harness CUDA error {rc}"}
        return {"alls_ms": ms.value, "alls_value": mesh.num_elems / (ms.value / 1e3),
                "what": "assembleGlobalStiffnessKernelALLS + convertALLStoCSRKernel "
                        "(ALLS_T3_Unstructed_Elements_Assemble_Performance.cu:227-315), timed as its driver times "
                        "them (T3:586-640), values only, uniform material E=1, nu=0.3"}
    return {"unavailable": f"no reference GPU timing harness for {workload}"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    import oracle as O
    workload = args.workload
    if workload == "batched":
        print(json.dumps({"impl": "reference", "unavailable": "the reference assembles one mesh per program run; "
                          "it has no batched path"}), flush=True)
        return
    mesh = make_mesh(workload, args.size)
    use_ref = O.ref_available("h20" if workload == "hex20" else "t3")
    t0 = time.perf_counter()
    if use_ref:
        rp, ci = O.ref_pattern(mesh)           # the reference's own host pattern builder
        kind = "reference"
    else:
        rp, ci = O.pattern(mesh)
        kind = "port"
    t1 = time.perf_counter()
    if mesh.kind == 0 and use_ref:
        vals = O.ref_q4a_host_assemble(mesh, rp, ci)
    else:
        _, _, vals = O.assemble(mesh, rp, ci)   # the serial value scatter of assembleGlobalStiffnessHost
    t2 = time.perf_counter()
    total = t2 - t0
    v = mesh.num_elems / total
    nnz = int(ci.shape[0])
    cb = {"value": v, "unit": "elements/s", "cores": 1, "kind": kind,
          "sample": f"the full configuration ({mesh.num_elems} elements), one pass: the reference's host pattern "
                    f"builder ({'compiled from its source' if use_ref else 'oracle port'}, {t1 - t0:.2f} s) and the "
                    f"serial FP64 value scatter of assembleGlobalStiffnessHost ({t2 - t1:.2f} s); the reference's "
                    f"host path is single-threaded",
          "pattern_s": t1 - t0, "values_s": t2 - t1, **host_info()}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "elements/s", "n_gpus": world,
            "steps": 1, "warmup": 0, "requested_steps": args.steps, "ms_per_step": total * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh generator)",
            "config": workload_config(workload, mesh, nnz, world, bool(args.size)),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        try:
            import torch
            gpu = torch.cuda.is_available()
        except Exception:
            gpu = False
        if gpu and use_ref:
            line["reference_gpu"] = reference_gpu(workload, mesh, rp, ci, vals)
        else:
            line["reference_gpu"] = {"unavailable": "no GPU or no reference harness build in this run"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=0,
                    help="grid cells per side instead of the configuration's (profiling a smaller case)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the oracle leg (CPU baseline and accuracy)")
    ap.add_argument("--no-colour", action="store_true", help="skip the element-colouring baseline leg")
    ap.add_argument("--no-reassembly", action="store_true", help="skip the value-only re-assembly and upper legs")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner leg")
    ap.add_argument("--no-ke", action="store_true", help="skip the precision-form legs")
    ap.add_argument("--no-secondary", action="store_true", help="skip the T3 and batched fields of the default line")
    ap.add_argument("--no-reference-gpu", action="store_true", help="reference arm: skip its GPU kernels")
    ap.add_argument("--headline-only", action="store_true", help="only the timed assembly and e2e")
    ap.add_argument("--ke-only", action="store_true",
                    help="Hex20: time only the element-stiffness kernels (FP64 and tensor-core forms)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
