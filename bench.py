"""Benchmark of the FEM global-stiffness assembly (A-LLS path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload t3|q4|mixed|hex20]
                    [--impl ours|reference]

A step is one full device assembly of a seeded synthetic mesh: list reset,
fused element stiffness + A-LLS scatter, and list -> CSR consolidation (pattern
and FP64 values), inputs resident in HBM. The default workload is the T3
unstructured configuration (1000x1000 grid, random diagonals, shuffled
elements, lognormal E). ``value`` is elements/s over the whole job; nnz/s,
the roofline, the end-to-end figure through the host-buffer C ABI entry point
(host<->device copies inside the timed region) and a CPU baseline are added to
the same JSON line. With --gpus N > 1 (one process per GPU under torchrun) every
rank assembles its own replica (the path has no exchange step): weak scaling.

``--impl reference`` times the reference's own CPU path for the same workload:
its host CSR pattern builder (buildCSRStructure, compiled from the reference
sources into oracle/_ref) plus the serial FP64 value scatter of
assembleGlobalStiffnessHost (ALLS_Quad2D_Assembly_Accuracy_Analysis.cu:329-380;
the reference's own function for Q4, the oracle's restatement of it for the
other element kinds), on a bounded sample, in parallel on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
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
# A smaller instance of each workload's generator, for the CPU legs.
CPU_SAMPLES = {"q4": ("q4", {}), "t3": ("t3", {"nx": 400, "ny": 400}),
               "mixed": ("mixed", {"nx": 450, "ny": 450}), "hex20": ("hex20", {"nx": 20})}
L2_BYTES = 126 * 2 ** 20


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


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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
# CPU legs (oracle / reference code)
# ---------------------------------------------------------------------------

def _cpu_sample_worker(args):
    workload, use_reference = args
    name, kw = CPU_SAMPLES[workload]
    mesh = make_mesh(name, **kw)
    import oracle as O
    t0 = time.perf_counter()
    if use_reference and O.ref_available("t3"):
        rp, ci = O.ref_pattern(mesh)
        if mesh.kind == 0:
            vals = O.ref_q4a_host_assemble(mesh, rp, ci)  # noqa: F841 (reference material)
        else:
            O.assemble(mesh, rp, ci)
        kind = "reference" if mesh.kind == 0 else "reference pattern + ported value scatter"
    else:
        O.assemble(mesh)
        kind = "port"
    dt = time.perf_counter() - t0
    return mesh.num_elems, dt, kind, mesh.name


def cpu_baseline(workload: str, use_reference: bool, workers: int) -> dict:
    """Serial assembly on a bounded sample; `workers` independent copies in parallel."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    if workers <= 1:
        res = [_cpu_sample_worker((workload, use_reference))]
    else:
        with ctx.Pool(workers) as pool:
            res = pool.map(_cpu_sample_worker, [(workload, use_reference)] * workers)
    wall = time.perf_counter() - t0
    elems = sum(r[0] for r in res)
    per = [r[0] / r[1] for r in res]
    kind = res[0][2]
    return {"value": float(sum(per)), "unit": "elements/s", "cores": workers,
            "kind": "reference" if kind == "reference" else "port",
            "sample": f"{len(res)} x {res[0][3]} ({res[0][0]} elements each), {kind}; serial pattern build + FP64 "
                      f"values per copy, copies in parallel processes; wall {wall:.1f}s",
            "elements": elems}


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------

def run_batched(args, rank: int, world: int, local_rank: int):
    """The batched configuration: 256 meshes assembled by fem_assemble_batched
    (one call per step, graph-captured), concurrency picked by the library's
    autotuner (fem_autotune_batched: 1/2/4/8/16 slots timed on this batch);
    concurrency 1 is the sequential baseline (the same per-mesh launches one
    after another on one stream). value = elements/s of the whole batch."""
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
    if rank != 0:
        return
    seq = per_k[1]
    line = {
        "metric": "elements/s (device FP64 A-LLS assembly: element stiffness, list scatter, CSR pattern + values)",
        "value": world * elems / (ms / 1e3), "unit": "elements/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded mesh generator)",
        "config": {"workload": name, "description": desc, "meshes": len(meshes), "elements": elems,
                   "nnz": int(sum(nnz)), "kinds": {k: sum(1 for m in meshes if m.kind == k) for k in range(4)},
                   "l2": "2x L2 buffer zeroed between steps, outside the per-step events",
                   "parallelism": f"replicas{world}", "mesh_generation_s": gen_s},
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
        "clocks": clk.summary(),
        "gpu_launches": args.steps * batch_launches(meshes),
        "api": "fem_assemble_batched, captured in one CUDA graph",
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import fem_alls as fem
    import build
    build.build()
    if args.workload == "batched":
        run_batched(args, rank, world, local_rank)
        return
    if args.ke_only:
        torch.cuda.set_device(local_rank)
        dev = torch.device("cuda", local_rank)
        mesh = make_mesh("hex20", args.size)
        flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
        line = {"workload": mesh.name, "elements": mesh.num_elems,
                "ke_form": ke_form(fem, torch, mesh, fem.device_arrays(mesh, dev), args, flush,
                                   torch.cuda.current_stream())}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    name, desc = WORKLOADS[args.workload]
    mesh = make_mesh(args.workload, args.size)
    if args.size:
        name = mesh.name
    asm = fem.Assembler(mesh, device=dev)
    _, _, _, info = asm.assemble()          # sizes the outputs
    nnz = int(info.nnz)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        asm.assemble_async()
    torch.cuda.synchronize()
    st, info = asm.read_info()
    fem.check(st, "warmup assembly")

    # per-kernel breakdown (untimed pass)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    asm.scatter()
    ev[1].record(stream)
    asm.consolidate()
    ev[2].record(stream)
    torch.cuda.synchronize()
    t_scatter, t_cons = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    mids = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.zero_()                      # evict L2 between steps (outside the step events)
            starts[i].record(stream)
            asm.scatter()                      # = fem_assemble_async, split to time the scatter phase
            mids[i].record(stream)
            asm.consolidate()
            stops[i].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    times = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    scatter_ms = statistics.mean(s.elapsed_time(e) for s, e in zip(starts, mids))
    consolidate_ms = statistics.mean(s.elapsed_time(e) for s, e in zip(mids, stops))
    st, info = asm.read_info()
    fem.check(st, "timed assembly")
    ms = job_ms(sum(times), world, dev) / args.steps
    clocks = clk.summary()

    # end to end through the host-buffer entry point
    e2e = None
    if not args.no_e2e:
        pinned = {k: torch.from_numpy(v).pin_memory() for k, v in fem.host_arrays(mesh).items()}
        harr = {k: v.numpy() for k, v in pinned.items()}
        rp = torch.empty(mesh.num_dofs + 1, dtype=torch.int32).pin_memory().numpy()
        ci = torch.empty(nnz, dtype=torch.int32).pin_memory().numpy()
        vv = torch.empty(nnz, dtype=torch.float64).pin_memory().numpy()
        ctx = fem.HostContext()
        s = stream.cuda_stream
        for _ in range(max(1, args.warmup)):
            fem.check(ctx.assemble(mesh, harr, rp, ci, vv, stream=s)[0], "fem_assemble_host")
        torch.cuda.synchronize()
        e_times = []
        for _ in range(args.steps):
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
        e_ms = job_ms(sum(e_times), world, dev) / args.steps
        h2d = sum(v.nbytes for v in harr.values())
        d2h = rp.nbytes + ci.nbytes + vv.nbytes
        e2e = {"value": world * mesh.num_elems / (e_ms / 1e3), "unit": "elements/s", "ms_per_step": e_ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "fem_assemble_host (pinned host buffers, copies inside the call)"}

    colour = None
    if not args.no_colour:
        colour = colour_baseline(fem, torch, asm, mesh, nnz, args, flush, stream)
    reasm = None if args.no_reassembly else reassembly(fem, torch, asm, mesh, nnz, args, flush, stream)
    upper = None if args.no_reassembly else upper_output(fem, torch, asm, mesh, nnz, args, flush, stream)
    kef = ke_form(fem, torch, mesh, asm.dev, args, flush, stream) if mesh.kind == 2 and not args.no_ke else None
    f32 = fp32_form(fem, torch, asm, mesh, nnz, args, flush, stream) if mesh.kind != 2 and not args.no_ke else None
    tuned = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        best, best_ms = asm.autotune(repeats=3)
        tuned = {"api": "fem_autotune (scatter grid CTAs/SM; Hex20 also first/overflow chunk slots)",
                 "best": {"ctas_per_sm": best.ctas_per_sm, "first_slots": best.first_slots,
                          "chunk_slots": best.chunk_slots, "pool_factor": best.pool_factor},
                 "best_ms": best_ms, "default_ms": ms, "tuning_s": time.perf_counter() - t0,
                 "note": "timed back to back without the L2 flush; the headline uses the default options"}

    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    ab = algorithmic_bytes(mesh, nnz)
    achieved = ab["total"] / (ms / 1e3) / 1e9
    # The dominant kernel is the scatter: it reads the inputs and writes every
    # list entry once (16 B per CSR nonzero); consolidation reads the entries
    # back and writes the CSR.
    scatter_bytes = ab["in"] + ab["list"] // 2
    consolidate_bytes = ab["list"] // 2 + ab["out"]
    scatter_gbs = scatter_bytes / (scatter_ms / 1e3) / 1e9
    consolidate_gbs = consolidate_bytes / (consolidate_ms / 1e3) / 1e9
    traffic = read_profile_traffic(args.workload)
    line = {
        "metric": "elements/s (device FP64 A-LLS assembly: element stiffness, list scatter, CSR pattern + values)",
        "value": world * mesh.num_elems / (ms / 1e3),
        "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator)",
        "config": {"workload": name, "description": desc, "elements": mesh.num_elems, "nodes": mesh.num_nodes,
                   "dofs": mesh.num_dofs, "nnz": nnz, "contributions": mesh.contributions(),
                   "l2": "2x L2 buffer zeroed between steps, outside the per-step events",
                   "parallelism": f"replicas{world}"},
        "nnz_per_s": world * nnz / (ms / 1e3),
        "roofline": {"bound": "hbm", "achieved": scatter_gbs, "peak": peak, "unit": "GB/s",
                     "frac": scatter_gbs / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": SCATTER_KERNEL[args.workload] + " (scatter phase: list reset, element order, scatter)",
                     "algorithmic_bytes_per_launch": scatter_bytes,
                     "algorithmic_bytes_per_element": scatter_bytes / max(mesh.num_elems, 1),
                     "ms_per_launch": scatter_ms},
        "consolidate_roofline": {"bound": "hbm", "achieved": consolidate_gbs, "peak": peak, "unit": "GB/s",
                                 "frac": consolidate_gbs / peak, "kernel": "k_write (consolidation phase: count, "
                                 "scan, sorted write)", "algorithmic_bytes_per_launch": consolidate_bytes,
                                 "ms_per_launch": consolidate_ms},
        "step_roofline": {"achieved": achieved, "frac": achieved / peak, "algorithmic_bytes": ab,
                          "frac_nominal_8tbs": achieved / 8000.0,
                          "compulsory_frac": (ab["in"] + ab["out"]) / (ms / 1e3) / 1e9 / peak},
        "kernels_ms": {"scatter": scatter_ms, "consolidate": consolidate_ms,
                       "scatter_untimed_pass": t_scatter, "consolidate_untimed_pass": t_cons},
        "list": {"entries": int(info.list_entries), "unique": nnz // mesh.dpn ** 2,
                 "max_row_entries": int(info.max_row_entries), "overflow_chunks": int(info.overflow_chunks)},
        "clocks": clocks,
        "gpu_launches": KERNELS_PER_STEP[args.workload] * args.steps,
    }
    if e2e:
        line["e2e"] = e2e
    if colour:
        line["colour_baseline"] = colour
    if reasm:
        line["reassembly"] = reasm
    if upper:
        line["upper_output"] = upper
    if kef:
        line["ke_form"] = kef
    if f32:
        line["fp32_form"] = f32
    if tuned:
        line["autotune"] = tuned
    if not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.workload, use_reference=False, workers=1)
    print(json.dumps(line), flush=True)


def ke_form(fem, torch, mesh, dev_arrays, args, flush, stream) -> dict:
    """The Hex20 element stiffness on its own (fem_element_stiffness) in its
    three forms (FP64 tensor cores, FP16-split tensor cores, plain FP64 on the
    CUDA cores), timed alike;
    the tensor-core values are compared with the FP64 ones per element, on the
    scale of the element's largest diagonal entry."""
    out = {}
    kes = {}
    for prec, name in ((0, "fp64"), (1, "tc_f16x3"), (2, "fp64_simt")):
        o = fem.opts(precision=prec)
        ke, st = fem.element_stiffness(mesh, o, dev_arrays=dev_arrays)
        fem.check(0 if st == 0 else 1, f"element stiffness {name}")
        for _ in range(args.warmup):
            fem.element_stiffness(mesh, o, dev_arrays=dev_arrays, out=ke)
        ts = []
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fem.element_stiffness(mesh, o, dev_arrays=dev_arrays, out=ke)
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        out[name + "_ms"] = statistics.mean(ts)
        kes[name] = ke
    # diagonal entries of the packed upper blocks: block (I, I) entries 0, 4, 8
    diag_idx = [9 * (i * 20 - i * (i - 1) // 2) + v for i in range(20) for v in (0, 4, 8)]
    d = kes["fp64"][:, diag_idx].abs().max(dim=1).values
    err = ((kes["tc_f16x3"] - kes["fp64"]).abs().max(dim=1).values / d).max()
    flops = 2 * 60 * 60 * 27 * mesh.num_elems  # the node-pair contraction
    out.update({"speedup_tc_vs_fp64": out["fp64_ms"] / out["tc_f16x3_ms"],
                "speedup_tc_vs_fp64_simt": out["fp64_simt_ms"] / out["tc_f16x3_ms"],
                "forms": "fp64: contraction on the FP64 tensor cores (the library's default); tc_f16x3: FP16 split "
                         "operands on the FP16 tensor cores; fp64_simt: plain FP64 dot products on the CUDA cores",
                "max_err_tc_vs_fp64": float(err),
                "err_scale": "per element, max |difference| / the element's largest diagonal entry",
                "contraction_gflop": flops / 1e9, "bytes_written": int(kes["fp64"].numel() * 8),
                "what": "fem_element_stiffness: packed symmetric Ke (210 3x3 blocks, 15.1 KB) of every element"})
    return out


def row_col_scale(torch, rp, ci, v, n):
    """max(|K_ij|, sqrt(|K_ii K_jj|)) of every entry of a CSR matrix."""
    rows = torch.repeat_interleave(torch.arange(n, device=rp.device), (rp[1:] - rp[:-1]).long())
    diag = torch.zeros(n, dtype=torch.float64, device=rp.device)
    on = rows == ci.long()
    diag[rows[on]] = v[on].abs()
    scale = torch.maximum(v.abs(), torch.sqrt(diag[rows] * diag[ci.long()]))
    return torch.where(scale > 0, scale, torch.ones_like(scale))


def fp32_form(fem, torch, asm, mesh, nnz, args, flush, stream) -> dict:
    """The whole A-LLS assembly with the FP32 Ke blocks of the 2-D kinds
    (FEM_PREC_FP32), timed like the FP64 step; its values are compared with
    the FP64 assembly's on the row/column scale."""
    v64 = asm.values[:nnz].clone()
    o64 = asm.opts
    asm.opts = fem.opts(precision=fem.FEM_PREC_FP32)
    try:
        for _ in range(args.warmup):
            asm.assemble_async()
        ts = []
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            asm.scatter()
            asm.consolidate()
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        st, _ = asm.read_info()
        fem.check(st, "FP32-form assembly")
        scale = row_col_scale(torch, asm.row_ptr, asm.col_idx[:nnz], v64, mesh.num_dofs)
        err = float(((asm.values[:nnz] - v64).abs() / scale).max()) if nnz else 0.0
    finally:
        asm.opts = o64
        asm.assemble()                         # leave the FP64 values in place
    ms = statistics.mean(ts)
    return {"value": mesh.num_elems / (ms / 1e3), "unit": "elements/s", "ms_per_step": ms,
            "max_scaled_err_vs_fp64": err,
            "err_scale": "max |difference| / max(|K_ij|, sqrt(|K_ii K_jj|)) over the CSR entries",
            "what": "fem_alls_scatter + fem_alls_consolidate with FEM_PREC_FP32 (Ke blocks in FP32 from "
                    "coordinates relative to the element's first node, FP64 accumulation)"}


def upper_output(fem, torch, asm, mesh, nnz, args, flush, stream) -> dict:
    """The consolidation into the upper triangle (fem_alls_consolidate_upper)
    of the same lists, timed like the full consolidation phase."""
    asm.scatter()
    rp, ci, v = asm.consolidate_upper()
    cap = int(ci.numel())
    ts = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fem.check(asm.lib.fem_alls_consolidate_upper(fem.C.byref(asm.cm), fem.C.byref(asm.opts), asm.ws_ptr,
                                                     asm.ws_bytes, fem._ptr(rp), fem._ptr(ci), fem._ptr(v), cap,
                                                     stream.cuda_stream), "fem_alls_consolidate_upper")
        b.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            ts.append(a.elapsed_time(b))
    st, info = asm.read_info()
    fem.check(st, "upper-triangle consolidation")
    unz = int(info.nnz)
    asm.assemble()                             # leave the full form in place
    ms = statistics.mean(ts)
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
    for _ in range(args.warmup):
        re.reassemble(vals)
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        re.reassemble(vals)
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    fem.check(re.read_info(), "re-assembly")
    ms = statistics.mean(ts)
    v_alls = asm.values[:nnz]
    diff = float(((vals - v_alls).abs() / v_alls.abs().clamp_min(1e-300)).max()) if nnz else 0.0
    return {"value": mesh.num_elems / (ms / 1e3), "unit": "elements/s", "ms_per_step": ms, "map_build_ms": build_ms,
            "map_bytes": re.map_bytes, "max_rel_diff_vs_alls_nonzero": diff,
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
    for _ in range(args.warmup):
        col.assemble(rp, ci, vals, nnz)
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        col.assemble(rp, ci, vals, nnz)
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    st, _ = col.read_info()
    fem.check(st, "colour assembly")
    ms = statistics.mean(ts)
    # agreement with the A-LLS values of the same pattern, on the row/column scale
    v_alls = asm.values[:nnz]
    scale = row_col_scale(torch, rp, ci[:nnz], v_alls, mesh.num_dofs)
    diff = float(((vals - v_alls).abs() / scale).max())
    return {"num_colours": nc, "prepare_ms": prep_ms, "assemble_ms": ms,
            "value": mesh.num_elems / (ms / 1e3), "unit": "elements/s (values into the A-LLS pattern; colouring "
            "and pattern excluded, as the reference times its coloured kernel)",
            "max_scaled_diff_vs_alls": diff,
            "kernels": ("k_scatter_hex20 (colour form)" if mesh.kind == 2 else "k_colour_assemble_2d") +
                       ", one launch per colour and element type"}


# k_info_init; element order (2-D: key count, k_bucket_scan, key scatter; Hex20 also
# k_bbox_init, k_bbox); scatter kernel(s) (mixed: Q4 and T3); k_consolidate_reset,
# k_scan_reduce, k_scan_tiles, k_row_ptr, k_write
KERNELS_PER_STEP = {"q4": 10, "t3": 10, "mixed": 11, "hex20": 12}


def batch_launches(meshes) -> int:
    """Library kernels of one fem_assemble_batched call: each mesh's assembly
    (as KERNELS_PER_STEP) and its completion kernel (k_finish), plus the start
    stamp (k_stamp)."""
    per_kind = {0: KERNELS_PER_STEP["q4"], 1: KERNELS_PER_STEP["t3"], 2: KERNELS_PER_STEP["hex20"],
                3: KERNELS_PER_STEP["mixed"]}
    return 1 + sum(per_kind[m.kind] + 1 for m in meshes)


SCATTER_KERNEL = {"q4": "k_scatter_2d<4>", "t3": "k_scatter_2d<3>", "mixed": "k_scatter_2d<4> + k_scatter_2d<3>",
                  "hex20": "k_scatter_hex20"}


def read_profile_traffic(workload: str):
    """DRAM bytes (read + write) of one scatter-kernel launch on this workload,
    from the committed ncu summary, if there is one."""
    p = os.path.join(ROOT, "profiles", f"traffic_{workload}.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get("dram_bytes_per_launch")
        except (ValueError, OSError):
            return None
    return None


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    import multiprocessing as mp
    workers = max(1, min(mp.cpu_count(), 16))
    name, desc = WORKLOADS[args.workload]
    vals = []
    for _ in range(max(1, args.steps)):
        cb = cpu_baseline(args.workload, use_reference=True, workers=workers)
        vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    line = {"impl": "reference", "metric": "elements/s (device FP64 A-LLS assembly: element stiffness, list scatter, "
            "CSR pattern + values)", "value": v, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh generator)", "config": {"workload": name, "description": desc},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="t3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=0,
                    help="grid cells per side instead of the configuration's (profiling a smaller case)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-colour", action="store_true", help="skip the element-colouring baseline leg")
    ap.add_argument("--no-reassembly", action="store_true", help="skip the value-only re-assembly leg")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner leg")
    ap.add_argument("--no-ke", action="store_true", help="skip the precision-form leg (Hex20: element-stiffness forms; 2-D: the FP32-form assembly)")
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
