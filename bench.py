"""Throughput of the NEXD-3D time-stepping hot path on B200.

Default workload: the two-layer anelastic model with NPML (4 x 4 x 2 km,
40x40x20 hexahedra x 6 = 192,000 tets, N=4, 3 Zener mechanisms, 3-cell NPML on
the sides and bottom, free top, seeded double-couple source, 100 surface
receivers, LSERK4), synthetic and seeded.  A step is one LSERK4 time step
(5 stages) over the whole mesh.  Metric: DOF-stage updates per second,
9 * Np * K * stages * steps * wavefields / time (only the 9 velocity-stress
fields count).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload twolayer|cube|batch64|multimodel|learned|partitions]
                  [--contraction fp32|bf16x3|auto|fp32_pairs]
                  [--kernels npml=KIND,rest=KIND]   (pinned per-class kernels)

Other workloads (measurements beside the headline, not the headline):
  cube     homogeneous elastic 2 km cube, 6,000 tets, N=3, absorbing sides,
           free top, vertical force, 9 receivers (the CPU-sized case)
  batch64  the two-layer model with 64 independent moment-tensor sources in
           one launch (64 wavefields, ~115 GB of state)
  multimodel  16 seeded models (8k-300k tets, N=2..5, elastic or anelastic)
           stepped together as one CUDA graph: one persistent launch per stage
           for all models or one branch per model, whichever the autotune
           measures faster
  partitions  the two-layer model split into --parts partitions (coordinate
           bisection) on one GPU with the per-stage halo exchange of a
           domain-decomposed run (the reference's SendRecVar)
  learned  the two-layer model with its NPML replaced by the learned
           absorbing boundary: the network is trained first (wide-NPML runs
           at 1,536 tets, scored on held-out sources against the wide run,
           reported under "learned_boundary"), then the 192k-tet model is
           timed with it

value: device time (CUDA events on the library's stream) of K steps with the
state resident in HBM, the steps replayed as captured CUDA graphs (the ~4 GB
of wavefield, residual, memory-variable and NPML arrays exceed the 126 MB L2 on
every step).  roofline: a second pass over K further steps with a CUDA event
pair around every launch (steps launched one kernel at a time), which gives the
per-kernel durations.  e2e: K steps through the C-ABI streaming call
nexd_step_io, each step copying its source samples in from the host and its
receiver samples out, wall clock.  Under torchrun each rank runs an independent
replica (its own seeded source); the time is the maximum over ranks.
--impl reference times the CPU restatement of the reference's solver (the
oracle, FP32 like the reference) on the host cores.
"""
import argparse
import ctypes as C
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nexd-3d_b200")
sys.path.insert(0, PKG)

from nexd_b200 import Mesh, synth, _abi, replicas  # noqa: E402

WORKLOADS = {
    "twolayer": dict(name="twolayer_anelastic_npml_192k_tets_N4_lserk4", cells=(40, 40, 20), N=4, nt=3000),
    "cube": dict(name="cube_elastic_absorbing_6k_tets_N3_lserk4", cells=(10, 10, 10), N=3, nt=1000),
    "batch64": dict(name="twolayer_anelastic_npml_192k_tets_N4_lserk4_64_sources", cells=(40, 40, 20), N=4,
                    nt=2000, nsrc=64),
    "multimodel": dict(name="16_models_8k_to_300k_tets_N2_to_5_one_graph", cells=None, N=None, nt=1500),
    "learned": dict(name="twolayer_anelastic_learned_boundary_192k_tets_N4_lserk4", cells=(40, 40, 20), N=4, nt=3000),
    "partitions": dict(name="twolayer_anelastic_npml_192k_tets_N4_lserk4_partitions", cells=(40, 40, 20), N=4,
                       nt=3000),
}


def train_learned_boundary(tmp, n_train=16, n_eval=4, seed=11, max_reflection=0.5, epochs=30):
    """Learned boundary at training scale: 2 x 2 x 1 km two-layer models (1,536
    tets) with seeded random layers (vp 2500-5500 m/s, vp/vs 1.6-1.9, rho
    2200-2900 kg/m^3) inside an 8-element NPML; train the boundary MLP on
    n_train source/material pairs, score plain and learned boundaries against
    the wide run on n_eval held-out sources and materials.  Returns
    (parameters, summary)."""
    from nexd_b200 import boundary
    from nexd_b200.solver import Solver
    cells, h, P, dur = (8, 8, 4), 250.0, 8, 1.2
    srcs = boundary.random_sources(n_train + n_eval, cells, h, seed=seed)
    mats = boundary.random_layers(n_train + n_eval, cells, h, seed=seed + 12)
    t0 = time.perf_counter()
    # held-out pairs also carry the small model inside a 3-element NPML (the layer
    # the learned boundary replaces), scored against the same wide-NPML reference
    pairs = [boundary.ModelPair(tmp, f"lb{i}", src, cells=cells, h=h, pml_cells=P, duration=dur, layers=mats[i],
                                npml_cells=3 if i >= n_train else 0)
             for i, src in enumerate(srcs)]
    xs, ys = zip(*(p.training_pairs(Solver, every=2) for p in pairs[:n_train]))
    x, y = np.concatenate(xs), np.concatenate(ys)
    t_data = time.perf_counter() - t0
    tr = boundary.Trainer(9 * 15, batch=2048, lr=1e-3, seed=0)
    hist = tr.fit(x, y, epochs=epochs)
    t_train = time.perf_counter() - t0 - t_data
    params = tr.parameters()
    scores = []
    for ev in pairs[n_train:]:
        res = ev.evaluate(Solver, params, [int(ev.nt * 0.6), int(ev.nt * 0.8), ev.nt], max_reflection=max_reflection)
        scores.append(res)
    mean = lambda k, f: float(np.mean([np.mean(r[k][f]) for r in scores]))
    kinds = ("plain", "learned", "npml")
    summary = {"train_sources": n_train, "heldout_sources": n_eval, "materials": "seeded random two-layer",
               "samples": int(len(x)), "epochs": epochs,
               "loss_first_last": [hist[0], hist[-1]], "data_s": round(t_data, 1), "train_s": round(t_train, 1),
               "max_reflection": max_reflection,
               "boundaries": {"plain": "absorbing faces (exterior state zero)",
                              "learned": "absorbing faces with the trained network (no extra elements)",
                              "npml": "3-element NPML around the same model"},
               "field_err_vs_wide_npml": {k: mean(k, "field_err") for k in kinds},
               "trace_err_vs_wide_npml": {k: mean(k, "trace_err") for k in kinds},
               "reflection_energy": {k: mean(k, "reflection_energy") for k in kinds},
               "reflection_energy_note": "kinetic energy of the difference from the wide-NPML run inside the model, "
                                         "as a fraction of the reference's peak kinetic energy there; mean over "
                                         "60/80/100 % of the run and the held-out cases",
               "reference_solution": "8-element NPML around the model (the method itself)"}
    return params, summary


def run_partitions(args, grp, tmp, steps, warmup, cells, workload):
    """The headline model split into --parts partitions (recursive coordinate
    bisection) on this GPU, stepped together with the per-stage halo exchange
    (nexd_halo_run).  Reports the whole-mesh rate and the halo kernels' share;
    on one GPU the halo writes go to this GPU's memory, on several they would
    cross NVLink (bytes per stage reported for that)."""
    import torch
    from nexd_b200.halo import Partitions, PartitionedSolver, element_centroids
    torch.cuda.set_device(0)
    wl = WORKLOADS["partitions"]
    d = os.path.join(tmp, "model")
    synth.write_twolayer(d, cells=cells, nt=wl["nt"], nrec=100, nsrc=1, src_seed=replicas.replica_seed(2, 0))
    mesh = Mesh(d, N=wl["N"], stf_stage_time=True)
    ps = Partitions(mesh.desc_ptr, args.parts, centroids=element_centroids(mesh))
    p = PartitionedSolver(ps, nrec_total=mesh.nrec)
    p0 = p.solvers[0]
    for x in p.solvers:  # each partition's kernels chosen like the whole mesh's (autotune by default)
        x.set_contraction(args.contraction if (mesh.N == 4 or args.contraction != "bf16x3") else "fp32")
    p.run(1, warmup)
    torch.cuda.synchronize()
    clk_file = os.path.join(tmp, "clocks.csv")
    clk = sample_clocks(None, clk_file)
    time.sleep(0.3)
    l0 = sum(x.launch_count() for x in p.solvers)
    p0.profile("span")
    p.run(warmup + 1, warmup + steps)
    span = p0.profile()["span_ms"]
    launches = sum(x.launch_count() for x in p.solvers) - l0
    for x in p.solvers:
        x.profile(True)
    p.run(warmup + steps + 1, warmup + 2 * steps)
    profs = [x.profile() for x in p.solvers]
    for x in p.solvers:
        x.profile(False)
    clk.terminate()
    clk.wait()
    hbytes = p.halo_bytes()
    kinds = {k: {"launches": sum(q[k]["launches"] for q in profs), "ms": round(sum(q[k]["ms"] for q in profs), 3)}
             for k in ("record", "stage_pml", "stage_main", "halo")}
    units = 9 * mesh.Np * mesh.K * 5 * steps
    halo_ms_stage = kinds["halo"]["ms"] / (5 * steps)
    line = {
        "metric": "DOF-stage updates/s", "value": units / (span * 1e-3), "unit": "DOF-stage/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": span / steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded two-layer model, seeded source)",
        "config": {"workload": workload, "tets": mesh.K, "N": mesh.N, "partitions": args.parts,
                   "partition_tets": [x.K for x in p.solvers], "integrator": "LSERK4 (5 stages)",
                   "kernels_per_class": [x.contraction()[0] for x in p.solvers],
                   "timed": "partitions interleaved stage by stage in one stream, launched kernel by kernel"},
        "halo": {"bytes_per_stage": hbytes, "ms_per_stage": halo_ms_stage,
                 "share_of_step": kinds["halo"]["ms"] / max(1e-9, sum(v["ms"] for v in kinds.values())),
                 "nvlink_us_per_stage_at_770GBps": hbytes / 770e9 * 1e6},
        "kernels": kinds, "gpu_launches": int(launches),
        "clocks": summarize_clocks(clk_file, 0),
    }
    p.close()
    ps.close()
    print(json.dumps(line), flush=True)


def multimodel_specs(seed=4, n=16):
    """16 seeded models: sizes 8,000-300,000 tets (log-uniform), orders 2-5,
    elastic or 3-mechanism anelastic, homogeneous or two-layer, absorbing
    sides and bottom, one double-couple source and 25 surface receivers each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = float(np.exp(rng.uniform(np.log(8000.0), np.log(300000.0))))
        nz = max(2, int(round((k / 24.0) ** (1.0 / 3.0))))
        out.append(dict(cells=(2 * nz, 2 * nz, nz), N=int(rng.choice([2, 3, 4, 5])), att=bool(rng.random() < 0.5),
                        homogeneous=bool(rng.random() < 0.5), src_seed=int(rng.integers(1 << 30))))
    return out


def run_multimodel(args, grp, tmp, steps, warmup):
    """16 models of 8,000-300,000 tets stepped together as one CUDA graph, grids autotuned."""
    from nexd_b200.solver import Solver, Group
    import torch
    torch.cuda.set_device(0 if grp.dist is None else grp.local)
    meshes, solvers = [], []
    for i, sp in enumerate(multimodel_specs(seed=replicas.replica_seed(4, grp.rank))):
        d = os.path.join(tmp, f"model{i}")
        synth.write_twolayer(d, cells=sp["cells"], nt=WORKLOADS["multimodel"]["nt"], nrec=25, nsrc=1,
                             attenuation=sp["att"], pml=False, src_depth=(500.0, 500.0), src_seed=sp["src_seed"],
                             homogeneous=sp["homogeneous"])
        m = Mesh(d, N=sp["N"], stf_stage_time=True)
        s = Solver(m.desc_ptr)
        s.set_contraction(args.contraction if (m.N == 4 or args.contraction != "bf16x3") else "fp32")
        meshes.append(m)
        solvers.append(s)
    g = Group(solvers)
    div = g.autotune()
    gmode, gblocks, gms = g.mode()
    g.run(1, warmup)
    grp.barrier()
    torch.cuda.synchronize()
    clk_file = os.path.join(tmp, "clocks.csv")
    clk = sample_clocks(None, clk_file) if grp.rank == 0 else None
    time.sleep(0.3 if clk else 0)
    l0 = sum(s.launch_count() for s in solvers)
    g.run(warmup + 1, warmup + steps)
    span_ms = g.span_ms()
    launches = sum(s.launch_count() for s in solvers) - l0
    # end to end: K more steps from the host call to the traces of every model in host memory
    t0 = time.perf_counter()
    g.run(warmup + steps + 1, warmup + 2 * steps)
    trace_bytes = 0
    for s in solvers:
        trace_bytes += s.traces().nbytes
    e2e_s = grp.max(time.perf_counter() - t0)
    if clk:
        clk.terminate()
        clk.wait()
    units = sum(9 * m.Np * m.K * 5 * steps for m in meshes)
    total = grp.sum(units)
    dev_ms = grp.max(span_ms)
    value = total / (dev_ms * 1e-3)
    abytes = sum(algorithmic_bytes(m, "stage_main", m.K) for m in meshes) * 5 * steps
    achieved = grp.sum(abytes) / (dev_ms * 1e-3) / 1e9
    peak, peak_kind = load_peaks()
    if grp.rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline and grp.world == 1:
        v, cores, sample, _ = oracle_baseline(tmp, "twolayer")
        cpu = {"value": v, "unit": "DOF-stage/s", "cores": cores, "kind": "port", "sample": sample}
    line = {
        "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": grp.world, "steps": steps,
        "warmup": warmup, "ms_per_step": dev_ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (16 seeded models per rank)",
        "config": {"workload": WORKLOADS["multimodel"]["name"],
                   "models": [dict(tets=m.K, N=m.N, anelastic=bool(m.desc.attenuation),
                                   kernel=s.contraction()[0]["rest"]) for m, s in zip(meshes, solvers)],
                   "total_tets": int(sum(m.K for m in meshes)), "integrator": "LSERK4 (5 stages)",
                   "timed": "one CUDA graph per two steps; autotuned between one branch per model "
                            "(grid divisor) and one persistent launch per stage for all models",
                   "group_mode": "one persistent launch per stage" if gmode == 1 else "one graph branch per model",
                   "autotune_ms_three_probe_stages": gms, "persistent_blocks_per_model": gblocks,
                   "grid_divisor": div, "l2": "inputs larger than L2",
                   "parallelism": f"replicas x{grp.world}"},
        "roofline": {"bound": "hbm", "kernel": "all stage kernels of the group (step average)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "peak_source": peak_kind},
        "e2e": {"value": total / e2e_s, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(trace_bytes / steps)},
        "gpu_launches": int(launches),
        "cpu_baseline": cpu,
        "clocks": summarize_clocks(clk_file, grp.local) if clk else None,
    }
    print(json.dumps(line), flush=True)
    g.close()
    for s in solvers:
        s.close()
N_ORDER = 4
# CPU baseline: a bounded number of steps of the timed model itself (the same
# mesh), the time of the oracle's step loop only (set-up excluded)
CPU_STEPS = 2


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(mesh, kind, elements):
    """Compulsory DRAM bytes of one stage launch: every stored field-node is
    read and written twice per LSERK stage (wavefield in/out, residual in/out:
    16 B in FP32), plus per-element constants (~40 words) and, for NPML
    elements, the 9 damping profiles per node (read once)."""
    Np = mesh.Np
    fields = 9 + (6 * mesh.desc.nMB if mesh.desc.attenuation else 0)
    per = Np * fields * 16 + 160
    if kind == "stage_pml":
        per += Np * 27 * 16 + Np * 9 * 4
    return per * elements


def sample_clocks(stop_file, out_file):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        return subprocess.Popen(cmd, stdout=open(out_file, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def summarize_clocks(path, device):
    try:
        rows = [l.split(",") for l in open(path).read().splitlines() if l.strip()]
    except Exception:
        return None
    rows = [[x.strip() for x in r] for r in rows if len(r) >= 9 and r[0].strip() == str(device)]
    if not rows:
        return None
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    reasons = set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for r in rows:
        for i, n in enumerate(names):
            if r[5 + i].lower().startswith("active"):
                reasons.add(n)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]) if rows else None,
            "reasons": sorted(reasons), "samples": len(rows)}


def oracle_baseline(tmp, workload="twolayer", mesh=None, steps=CPU_STEPS, seed=None, warmup=0):
    """The CPU restatement of the reference solver (the oracle, FP32 like the
    reference's default CUSTOM_REAL) on the host cores, all OpenMP threads,
    over `steps` steps of the same workload (the mesh given, or one built
    with the same generator, sizes and seed), after `warmup` untimed steps;
    the rate counts the timed step loop only.  Returns (DOF-stage/s, threads,
    sample description, ms per step)."""
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.oracle_run.argtypes = [C.POINTER(_abi.NexdDesc), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_void_p, C.c_int]
    lib.oracle_loop_seconds.restype = C.c_double
    if WORKLOADS[workload]["cells"] is None:  # the multi-model group: its largest member family
        workload = "twolayer"
    if mesh is None:
        d = os.path.join(tmp, "cpu_model")
        wl = WORKLOADS[workload]
        seed = replicas.replica_seed(1 if workload == "cube" else 2, 0) if seed is None else seed
        if workload == "cube":
            synth.write_cube(d, cells=wl["cells"][0], nt=wl["nt"], seed=seed)
        else:
            nsrc = wl.get("nsrc", 1)
            kw = dict(src_depth=(500.0, 1800.0), f0_range=(2.0, 4.0)) if nsrc > 1 else {}
            synth.write_twolayer(d, cells=wl["cells"], nt=wl["nt"], nrec=100, nsrc=nsrc, src_seed=seed,
                                 pml=(workload != "learned"), **kw)
        mesh = Mesh(d, N=wl["N"], stf_stage_time=True, nbatch=wl.get("nsrc", 1))
    m = mesh
    if workload == "cube":
        steps = max(steps, 20)
    tr = np.zeros((m.nrec, m.nt, 9, m.nbatch), dtype=np.float32, order="F")
    if warmup > 0:
        if lib.oracle_run(m.desc_ptr, 32, warmup, tr.ctypes.data_as(C.POINTER(C.c_float)), None, 0) != 0:
            raise RuntimeError("oracle failed in the warm-up steps")
    t0 = time.perf_counter()
    st = lib.oracle_run(m.desc_ptr, 32, steps, tr.ctypes.data_as(C.POINTER(C.c_float)), None, 0)
    wall = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(f"oracle failed: {st}")
    el = lib.oracle_loop_seconds()
    units = 9 * m.Np * m.K * 5 * steps * m.nbatch
    cores = os.cpu_count() or 1
    sample = (f"{steps} LSERK4 steps of the timed workload itself ({m.K} tets, N={m.N}, {m.nbatch} wavefield(s)), "
              f"FP32, {cores} OpenMP threads; step loop {el:.1f} s (set-up excluded, {wall:.1f} s wall in total)")
    return units / el, cores, sample, 1e3 * el / steps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--contraction", default="auto", choices=["fp32", "bf16x3", "auto", "fp32_pairs"],
                    help="element contraction: FP32 CUDA cores, split-BF16 tcgen05 tensor cores, or the faster "
                         "per element class (timed before the run)")
    ap.add_argument("--kernels", default=None,
                    help="pin the kernel per element class instead of --contraction, e.g. npml=bf16x3,rest=fp32 "
                         "(the choice an auto run reports in kernels_per_class; profiled runs use it, since "
                         "timing under a profiler would change the auto choice)")
    ap.add_argument("--workload", default="twolayer", choices=sorted(WORKLOADS))
    ap.add_argument("--lb-train", type=int, default=16, help="learned workload: training source/material pairs")
    ap.add_argument("--lb-eval", type=int, default=4, help="learned workload: held-out pairs scored")
    ap.add_argument("--lb-epochs", type=int, default=30, help="learned workload: training epochs")
    ap.add_argument("--parts", type=int, default=2, help="partitions workload: number of partitions")
    ap.add_argument("--cells", default=None, help="hexahedra per axis of the two-layer box (profiling runs use 20,20,10)")
    args = ap.parse_args()
    grp = replicas.init()
    rank, world, local = grp.rank, grp.world, grp.local
    wl = WORKLOADS[args.workload]
    cells = wl["cells"] if args.cells is None else tuple(int(x) for x in args.cells.split(","))
    workload = wl["name"] if cells == wl["cells"] else \
        wl["name"].replace("192k_tets", f"{6 * cells[0] * cells[1] * cells[2]}_tets")
    if args.workload == "multimodel" and args.impl == "ours":
        steps, warmup = args.steps, max(3, args.warmup)
        tmp = tempfile.mkdtemp(prefix=f"nexd_bench_{rank}_")
        try:
            run_multimodel(args, grp, tmp, steps, warmup)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
            grp.close()
        return
    if args.workload == "partitions" and args.impl == "ours":
        tmp = tempfile.mkdtemp(prefix=f"nexd_bench_{rank}_")
        try:
            if rank == 0:
                run_partitions(args, grp, tmp, args.steps, max(3, args.warmup), cells, workload)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
            grp.close()
        return
    steps, warmup = args.steps, max(3, args.warmup)
    tmp = tempfile.mkdtemp(prefix=f"nexd_bench_{rank}_")
    metric = "DOF-stage updates/s"
    try:
        if args.impl == "reference":
            if rank == 0:
                # each step of this arm is one LSERK4 step of the whole workload on the host cores
                v, cores, sample, ms = oracle_baseline(tmp, args.workload, steps=steps, warmup=warmup)
                line = {"metric": metric, "value": v, "unit": "DOF-stage/s", "n_gpus": args.gpus, "steps": steps,
                        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                        "config": {"workload": workload, "tets": wl["cells"][0] * wl["cells"][1] * wl["cells"][2] * 6
                                   if wl["cells"] else None, "N": wl["N"], "integrator": "LSERK4 (5 stages)",
                                   "sample": f"{steps} steps of this workload after {warmup} untimed (see cpu_baseline)"},
                        "impl": "reference",
                        "cpu_baseline": {"value": v, "unit": "DOF-stage/s", "cores": cores, "kind": "port",
                                         "sample": sample},
                        "e2e": {"value": v, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
                print(json.dumps(line), flush=True)
            return
        from nexd_b200.solver import Solver
        import torch
        if grp.dist is None:
            torch.cuda.set_device(0)
        learned = None
        if args.workload == "learned":
            lb_params, learned = train_learned_boundary(tmp, n_train=args.lb_train, n_eval=args.lb_eval,
                                                        epochs=args.lb_epochs)
        d = os.path.join(tmp, "model")
        if args.workload == "cube":
            synth.write_cube(d, cells=cells[0], nt=wl["nt"], seed=replicas.replica_seed(1, rank))
            mesh = Mesh(d, N=wl["N"], stf_stage_time=True)
        else:
            nsrc = wl.get("nsrc", 1)
            kw = dict(src_depth=(500.0, 1800.0), f0_range=(2.0, 4.0)) if nsrc > 1 else {}
            synth.write_twolayer(d, cells=cells, nt=wl["nt"], nrec=100, nsrc=nsrc,
                                 src_seed=replicas.replica_seed(2, rank), pml=(args.workload != "learned"), **kw)
            mesh = Mesh(d, N=wl["N"], stf_stage_time=True, nbatch=nsrc)
        s = Solver(mesh.desc_ptr)
        contraction = args.contraction if (mesh.N == 4 or args.contraction != "bf16x3") else "fp32"
        if args.kernels:
            pinned = dict(kv.split("=") for kv in args.kernels.split(","))
            s.set_contraction_kinds(pinned["npml"], pinned["rest"])
            contraction = "pinned " + args.kernels
        else:
            s.set_contraction(contraction)  # the tensor-core kernels cover N=4
        if learned is not None:
            s.set_boundary_mlp(lb_params, learned["max_reflection"])
        nstage = 5
        need = warmup + 3 * steps + 1
        if need > mesh.nt:
            raise SystemExit(f"--warmup + 3*--steps + 1 must be <= {mesh.nt}")
        s.run(1, warmup)
        grp.barrier()
        torch.cuda.synchronize()
        clk_file = os.path.join(tmp, "clocks.csv")
        clk = sample_clocks(None, clk_file) if rank == 0 else None
        time.sleep(0.3 if clk else 0)
        # timed region: K steps, CUDA graphs, run-span events only
        l0 = s.launch_count()
        s.profile("span")
        grp.barrier()
        torch.cuda.synchronize()
        s.run(warmup + 1, warmup + steps)
        torch.cuda.synchronize()
        span = s.profile()
        launches = s.launch_count() - l0
        # roofline pass: K further steps, an event pair around every launch
        s.profile(True)
        s.run(warmup + steps + 1, warmup + 2 * steps)
        torch.cuda.synchronize()
        prof = s.profile()
        s.profile(False)
        if clk:
            clk.terminate()
            clk.wait()
        dev_ms = grp.max(span["span_ms"])
        units = 9 * mesh.Np * mesh.K * nstage * steps * mesh.nbatch
        total_units = grp.sum(units)
        value = total_units / (dev_ms * 1e-3)
        # end to end through the streaming C-ABI call, host buffers in and out
        nspt, nsrc, nrec = mesh.desc.stf_per_step, mesh.nsrc, mesh.nrec
        stf_all = mesh.array("stf")  # (nspt, nt, nsrc)
        stf_in = np.zeros((nspt, nsrc), dtype=np.float32, order="F")
        tr_out = np.zeros((nrec, 9, mesh.nbatch), dtype=np.float32, order="F")
        # one untimed streaming step first: it captures the one-step graphs
        it_first = warmup + 2 * steps + 1
        stf_in[:, :] = stf_all[:, it_first - 1, :]
        s.step_io(it_first, stf_in, tr_out)
        grp.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for it in range(it_first + 1, it_first + steps + 1):
            stf_in[:, :] = stf_all[:, it - 1, :]
            s.step_io(it, stf_in, tr_out)
        e2e_s = grp.max(time.perf_counter() - t0)
        e2e = total_units / e2e_s
        # end of run: every replica's receiver traces on rank 0 (outside the timed regions)
        gathered = replicas.gather_traces(grp, s.traces())
        if rank != 0:
            return
        peak, peak_kind = load_peaks()
        kinds = [k for k in ("stage_main", "stage_pml") if prof[k]["launches"] > 0]
        nb = mesh.nbatch
        dom = max(kinds, key=lambda k: prof[k]["ms"])
        ckinds = s.contraction()[0]
        tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")

        def kernel_roofline(k):
            # algorithmic bytes per launch / mean launch time; DRAM traffic per launch from the ncu capture
            ms = prof[k]["ms"] / prof[k]["launches"]
            ab = algorithmic_bytes(mesh, k, prof[k]["elements"]) * nb
            tr = None
            if os.path.exists(tp):
                try:
                    t = json.load(open(tp)).get(workload, {}).get(f"{k}/{ckinds['npml' if k == 'stage_pml' else 'rest']}")
                    tr = None if t is None else float(t)
                except Exception:
                    tr = None
            return ms, ab, ab / (ms * 1e-3) / 1e9, tr

        per_launch_ms, abytes, achieved, traffic = kernel_roofline(dom)
        step_bytes = sum(algorithmic_bytes(mesh, k, prof[k]["elements"]) * nb for k in kinds) * nstage
        per_kernel = {}
        for k in kinds:
            ms_k, ab_k, ach_k, tr_k = kernel_roofline(k)
            per_kernel[k] = {"kernel_kind": ckinds["npml" if k == "stage_pml" else "rest"], "achieved": ach_k,
                             "frac": ach_k / peak, "traffic": tr_k, "algorithmic_bytes_per_launch": ab_k,
                             "avg_launch_ms": ms_k, "share_of_stage_time": prof[k]["ms"] /
                             sum(prof[j]["ms"] for j in kinds)}
        s.close()  # frees the device state before the CPU leg
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            v, cores, sample, _ = oracle_baseline(tmp, args.workload, mesh=mesh)
            cpu = {"value": v, "unit": "DOF-stage/s", "cores": cores, "kind": "port", "sample": sample}
        clocks = summarize_clocks(clk_file, local) if clk else None
        state_gb = (2 * 9 + 9 + 2 * 6 * mesh.desc.nMB) * mesh.K * mesh.Np * 4 * nb / 1e9
        line = {
            "metric": metric, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": dev_ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if "bf16x3" not in ckinds.values() else
                     "f32 state and update; contraction as three-way split bf16 on tcgen05 with f32 accumulation",
            "data": "synthetic (seeded two-layer model, per-rank seeded source)",
            "config": {"workload": workload, "tets": mesh.K, "N": mesh.N, "Np": mesh.Np, "nt": mesh.nt,
                       "integrator": "LSERK4 (5 stages)",
                       "contraction": contraction,
                       "kernels_per_class": ckinds, "pml_tets": int(prof["stage_pml"]["elements"]),
                       "receivers": nrec, "sources_per_rank": nsrc, "wavefields_per_rank": nb,
                       "timed": "CUDA graphs of two steps; roofline from a per-launch-event pass of K more steps",
                       "l2": f"inputs larger than L2: {state_gb:.1f} GB of state streamed per stage",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": abytes, "avg_launch_ms": per_launch_ms,
                         "per_kernel": per_kernel,
                         # the whole step: all stage launches' algorithmic bytes over the device-timed step
                         "step_achieved": step_bytes / (dev_ms / steps * 1e-3) / 1e9,
                         "step_frac": step_bytes / (dev_ms / steps * 1e-3) / 1e9 / peak},
            "kernels": {k: {"launches": prof[k]["launches"], "ms": round(prof[k]["ms"], 3)}
                        for k in ("record", "stage_pml", "stage_main")},
            "per_launch_pass_ms_per_step": prof["span_ms"] / steps,
            "e2e": {"value": e2e, "unit": "DOF-stage/s", "h2d_bytes_per_step": int(nspt * nsrc * 4),
                    "d2h_bytes_per_step": int(nrec * 9 * mesh.nbatch * 4)},
            "gpu_launches": int(launches),
            "cpu_baseline": cpu,
            "clocks": clocks,
            "traces_gathered_on_rank0": list(gathered.shape),
        }
        if learned is not None:
            line["learned_boundary"] = learned
            line["kernels"]["boundary"] = {"launches": prof["boundary"]["launches"], "ms": round(prof["boundary"]["ms"], 3)}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        grp.close()


if __name__ == "__main__":
    main()
