#!/usr/bin/env python
"""Throughput of the 2G HDNNP energy + force path on B200.

Workload (default): the batched benchmark configuration -- 2048 periodic water
boxes of 32..512 molecules (log-uniform, seeded; ~1.06 M atoms), 40 symmetry
functions per element (G2 + narrow G3, poly2 cutoff, rc = 12 bohr),
40-25-25-1 softplus networks, plain FP64, all structures evaluated per step
(neighbour lists, symmetry functions, networks, energies, forces) from one
CUDA-graph launch.  Inputs are synthetic (seeded recipe), not a dataset.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0.  `value` = atoms/s over all ranks (weak scaling:
every rank evaluates its own batch of the same size, no collective on the
data path; the time is the max over ranks).  `e2e` = the same metric through
the C-ABI call with host buffers (positions H2D and energies + forces D2H
inside the timed region).  `mixed` = the FP32-descriptor form on the same
batch with its error against the FP64 reference.  `roofline` = the
symmetry-function stage against the measured FP64 FMA throughput.
`cpu_baseline` = the reference library on the host cores (bounded sample).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MODEL = os.path.join(ROOT, "tests", "golden", "models", "water40")
TEACHER = os.path.join(ROOT, "tests", "golden", "models", "water56")
STUDENT = os.path.join(ROOT, "tests", "golden", "models", "student_water56")
# the same recipe with the descriptor chosen by force span (angular cutoff 12 bohr): slower, closer to the teacher
STUDENT_SPAN = os.path.join(ROOT, "tests", "golden", "models", "student_water56_span")
METRIC = "atoms/s (E+F) on 1×B200: mixed/student vs plain FP64 at ≤1 meV/atom, 30 meV/Å"
HA_TO_MEV = 27211.386
HA_BOHR_TO_MEV_A = 27211.386 / 0.529177
BOHR_TO_A = 0.529177210903
HA_TO_EV = 27.211386245988

# DRAM bytes (read + write) of the two symmetry-function passes per neighbour
# entry, from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum)
# of the 256-box case (FP64, acceptance masks present, first tier 128 x 4),
# all three tiers: G pass 571.3 + 118.0 MB, force pass 817.8 + 301.5 MB over
# 13,792,482 entries; scaled to a batch by its entry count.
SF_DRAM_BYTES_PER_ENTRY = (571.3 + 118.0 + 817.8 + 301.5) * 1e6 / 13792482

# Algorithmic FLOPs per unit of the reference's symmetry-function algorithm
# with derivatives (add/mul/div/sqrt = 1, exp counted separately):
# G2 23 per pair-member + 14 per pair (cutoff function), narrow G3 60 per
# triplet + 57 per triplet-member, wide G9 45 per pair + 50 per pair-member.
FLOPS_PER = {"radial_terms": 23, "radial_pairs": 14, "narrow_triplets": 60, "narrow_terms": 57,
             "wide_pairs": 45, "wide_terms": 50}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--boxes", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-student", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-lammps", action="store_true")
    ap.add_argument("--no-scaling", action="store_true")
    ap.add_argument("--no-compact", action="store_true")
    ap.add_argument("--no-training", action="store_true")
    ap.add_argument("--student-boxes", type=int, default=2048)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(boxes, seed):
    from n2p2_b200 import water
    return water.water_batch(boxes, seed=seed)


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    def __init__(self, index):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            w = [x.strip() for x in line.split(",")]
            if len(w) < 9:
                continue
            try:
                sm.append(float(w[1]))
                smax.append(float(w[2]))
            except ValueError:
                continue
            for n, v in zip(names, w[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(texts, threads):
    from oracle import ref
    sec, energies = ref.time_batch(MODEL, texts, threads, fast=True)
    return sec, energies


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(structs, threads, target_atoms=None):
    """A bounded sample of the workload for the CPU reference: whole
    structures, round-robin over the batch, about 12 s of work on `threads`."""
    if target_atoms is None:
        target_atoms = int(1700 * 12 * max(1, threads) * 0.7)
    out, n = [], 0
    stride = max(1, len(structs) // 256)
    for k in range(0, len(structs), stride):
        out.append(structs[k])
        n += structs[k].numAtoms
        if n >= target_atoms:
            break
    return out, n


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    structs = workload(args.boxes, args.seed)
    threads = host_threads()
    sample, natoms = cpu_sample(structs, threads)
    texts = [s.to_text() for s in sample]
    for _ in range(args.warmup):
        cpu_reference(texts[: max(1, len(texts) // 8)], threads)
    secs = []
    for _ in range(args.steps):
        sec, _ = cpu_reference(texts, threads)
        secs.append(sec)
    t = float(np.mean(secs))
    v = natoms / t
    total_atoms = sum(s.numAtoms for s in structs)
    # a step is the timed sample (a bounded part of the workload): ms_per_step is its measured time, the
    # atoms/s value is the throughput on it
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "atoms/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded water boxes)",
            "config": {"workload": "%d water boxes, 32-512 molecules log-uniform (%d atoms), water40 model, FP64"
                       % (args.boxes, total_atoms), "boxes": args.boxes, "atoms": total_atoms,
                       "timed_sample": "%d of the %d structures (%d atoms) per step" % (len(sample), len(structs), natoms),
                       "full_workload_ms_estimate": 1000.0 * total_atoms / v},
            "cpu_baseline": {"value": v, "unit": "atoms/s", "cores": threads, "kind": "reference",
                             "sample": "%d of %d structures (%d atoms) per step, structure-parallel, "
                                       "reference libnnp (-O3 -march=x86-64-v3)" % (len(sample), len(structs), natoms)},
            "e2e": {"value": v, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    from n2p2_b200 import Mode
    from n2p2_b200 import ranks
    rank, world, local = ranks.rank_env()
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    structs = workload(args.boxes, ranks.rank_seed(args.seed, rank))
    natoms = sum(s.numAtoms for s in structs)
    pos = np.ascontiguousarray(np.concatenate([s.positions for s in structs]))

    mode = Mode(local)
    mode.setupFromDirectory(MODEL)
    mode.setPrecision("fp64")
    batch = mode.batch(structs)
    batch.setPositions(pos)
    batch.evaluate(forces=True)     # establishes neighbour capacity (direct launches)
    batch.synchronize()
    tune = batch.autotune(useCache=False)   # kernel shapes measured on this batch (outside the timed steps)
    stream = torch.cuda.ExternalStream(batch.stream(), device=torch.device("cuda", local))

    def timed(steps, warmup):
        for _ in range(warmup):
            batch.evaluate(forces=True)
        batch.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            batch.evaluate(forces=True)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return ranks.max_over_ranks(ms, device="cuda")

    clocks = ClockSampler(local)
    clocks.start()
    ms = timed(args.steps, args.warmup)
    clk = clocks.stop()
    E64 = batch.energies()
    F64 = batch.forces()
    launches = batch.launchCount() * args.steps

    # end to end through the C ABI with pinned host buffers
    nbytes_pos = pos.nbytes
    hp = ctypes_pinned(nbytes_pos)
    he = ctypes_pinned(8 * len(structs))
    hf = ctypes_pinned(nbytes_pos)
    np.frombuffer(hp[1], dtype=np.float64)[:] = pos.ravel()
    for _ in range(2):
        batch.evaluateHost(np.frombuffer(hp[1], dtype=np.float64), np.frombuffer(he[1], dtype=np.float64),
                           np.frombuffer(hf[1], dtype=np.float64))
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        batch.evaluateHost(np.frombuffer(hp[1], dtype=np.float64), np.frombuffer(he[1], dtype=np.float64),
                           np.frombuffer(hf[1], dtype=np.float64))
    e2e_ms = ranks.max_over_ranks((time.perf_counter() - t0) * 1000.0 / args.steps, device="cuda")

    # stage profile and algorithmic work (rank-local, one direct evaluation)
    stages = batch.profileStages(forces=True)
    work = batch.countWork()
    fp64_peak = fp32_peak = None
    d64, d32 = ctypes_double(), ctypes_double()
    if mode._lib.n2p2_device_fma_peak(local, d64.ref, d32.ref) == 0:
        fp64_peak, fp32_peak = d64.value, d32.value

    # mixed-precision form on the same batch
    mixed = None
    if not args.no_mixed:
        mode.setPrecision("mixed")
        batch.evaluate(forces=True)
        batch.synchronize()
        tune_mixed = batch.autotune(useCache=False)
        ms_mixed = timed(args.steps, args.warmup)
        Em, Fm = batch.energies(), batch.forces()
        stages_mixed = batch.profileStages(forces=True)
        mode.setPrecision("fp64")
        atoms_per = np.array([s.numAtoms for s in structs])
        de = np.abs(Em - E64) / atoms_per * HA_TO_MEV
        df = np.abs(Fm - F64) * HA_BOHR_TO_MEV_A
        mixed = {"value": world * natoms / (ms_mixed / 1000.0), "unit": "atoms/s", "ms_per_step": ms_mixed,
                 "speedup_vs_fp64": ms / ms_mixed, "autotune": _shape_names(tune_mixed),
                 "stages_ms": {n: round(t, 4) for n, t in stages_mixed},
                 "err_vs_fp64_gpu": {"energy_meV_per_atom_max": float(de.max()),
                                     "force_meV_per_A_max": float(df.max()),
                                     "force_meV_per_A_rms": float(np.sqrt((df ** 2).mean()))}}

    # the large single-system configuration (FP64 and mixed)
    large = None
    if rank == 0 and world == 1 and not args.no_large:
        large = bench_large(args.steps, args.warmup, local)

    # MD steps through the LAMMPS interface (local + ghost atoms, host arrays)
    lammps = None
    if rank == 0 and world == 1 and not args.no_lammps:
        lammps = bench_lammps(args.steps, args.warmup, local, cpu=not args.no_cpu)

    # compact symmetry functions (the reference's SCAN example model)
    compact = None
    if rank == 0 and world == 1 and not args.no_compact:
        compact = bench_compact(args.steps, args.warmup, local, cpu=not args.no_cpu)

    # training updates (Kalman filter over the water40 networks)
    training = None
    if rank == 0 and world == 1 and not args.no_training:
        training = bench_training(args.steps, args.warmup, local, cpu=not args.no_cpu)

    # nnp-scaling (input.data read + symmetry-function statistics) on the batched workload
    scal = None
    if rank == 0 and world == 1 and not args.no_scaling:
        scal = bench_scaling(structs, local, cpu=not args.no_cpu)

    # distilled student (with teacher fallback) against the plain FP64 teacher
    stud = None
    if rank == 0 and world == 1 and not args.no_student and os.path.isdir(STUDENT):
        from n2p2_b200 import student as student_mod
        stud = student_mod.benchmark(STUDENT, TEACHER, num=args.student_boxes, steps=args.steps,
                                     warmup=args.warmup)
        stud["descriptor"] = "teacher functions of largest energy sensitivity, angular cutoff 8 bohr"
        if os.path.isdir(STUDENT_SPAN):
            span = student_mod.benchmark(STUDENT_SPAN, TEACHER, num=args.student_boxes, steps=args.steps,
                                         warmup=args.warmup)
            stud["span_descriptor"] = {k: span[k] for k in (
                "value", "unit", "ms_per_step", "speedup_vs_fp64", "fallback_rate", "err_vs_teacher_fp64_gpu",
                "err_vs_teacher_fp64_gpu_teacher_in_range", "held_out_monitor", "_predictions")}
            stud["span_descriptor"]["descriptor"] = ("chosen by force span from a candidate grid within the groups the "
                                                     "specialised kernels run, angular cutoff 12 bohr")

    sf_ms = sum(t for n, t in stages if n in ("sf_values", "sf_forces"))
    sf_flops = sum(work[k] * f for k, f in FLOPS_PER.items())
    roofline = None
    if fp64_peak and sf_ms > 0:
        achieved = sf_flops / (sf_ms * 1e-3) / 1e12
        roofline = {"bound": "fp64", "kernel": "kSFValues + kSFForces (symmetry functions, values + derivatives)",
                    "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                    "peak_source": "measured FP64 FMA throughput of this GPU (n2p2_device_fma_peak)",
                    "algorithmic_flops_per_step": sf_flops,
                    "traffic": SF_DRAM_BYTES_PER_ENTRY * work["entries"],
                    "traffic_source": "ncu DRAM bytes of a 256-box capture, scaled by neighbour entries",
                    "traffic_GBps": SF_DRAM_BYTES_PER_ENTRY * work["entries"] / (sf_ms * 1e-3) / 1e9}

    if mixed is not None and fp32_peak:
        # the FP32 symmetry-function passes of the mixed form against the measured FP32 FMA throughput
        ms32 = sum(t for n, t in mixed["stages_ms"].items() if n in ("sf_values", "sf_forces"))
        if ms32 > 0:
            a32 = sf_flops / (ms32 * 1e-3) / 1e12
            mixed["roofline"] = {"bound": "fp32", "kernel": "kSFValues + kSFForces, FP32 instances",
                                 "achieved": a32, "peak": fp32_peak, "unit": "TFLOP/s", "frac": a32 / fp32_peak,
                                 "peak_source": "measured FP32 FMA throughput of this GPU (n2p2_device_fma_peak)",
                                 "algorithmic_flops_per_step": sf_flops}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            threads = host_threads()
            sample, nsample = cpu_sample(structs, threads)
            sec, e_ref = cpu_reference([s.to_text() for s in sample], threads)
            idx = [structs.index(s) for s in sample]
            rel = float(np.max(np.abs(E64[idx] - e_ref) / np.abs(e_ref)))
            cpu = {"value": nsample / sec, "unit": "atoms/s", "cores": threads, "kind": "reference",
                   "sample": "%d of %d structures (%d atoms), structure-parallel on %d host threads, reference "
                             "libnnp (-O3 -march=x86-64-v3)" % (len(sample), len(structs), nsample, threads),
                   "fp64_energy_max_rel_err_vs_gpu": rel}
        except Exception as exc:  # the timed GPU numbers stand without it
            cpu = {"value": None, "unit": "atoms/s", "cores": host_threads(), "kind": "reference",
                   "sample": "failed: %s" % exc}
        if stud is not None:
            stud["err_vs_fp64_oracle"] = student_vs_oracle(stud["_predictions"])
            if "span_descriptor" in stud:
                stud["span_descriptor"]["err_vs_fp64_oracle"] = \
                    student_vs_oracle(stud["span_descriptor"]["_predictions"])
    if stud is not None:
        stud.pop("_predictions", None)
        if "span_descriptor" in stud:
            stud["span_descriptor"].pop("_predictions", None)

    value = world * natoms / (ms / 1000.0)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water boxes)",
                "config": {"workload": "%d water boxes, 32-512 molecules log-uniform (%d atoms per GPU), "
                                       "water40 model (40 SFs/element, 40-25-25-1 softplus), plain FP64, "
                                       "one CUDA-graph launch per step" % (args.boxes, natoms),
                           "boxes": args.boxes, "atoms_per_gpu": natoms,
                           "neighbor_entries_per_gpu": work["entries"],
                           "l2": "inputs larger than L2 (neighbour data %.1f GB per step)" % (
                               work["entries"] * 40 / 1e9),
                           "parallelism": "dp%d (independent structures per GPU)" % world},
                "e2e": {"value": world * natoms / (e2e_ms / 1000.0), "unit": "atoms/s", "ms_per_step": e2e_ms,
                        "h2d_bytes_per_step": nbytes_pos, "d2h_bytes_per_step": nbytes_pos + 8 * len(structs)},
                "gpu_launches": launches, "autotune": _shape_names(tune), "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
                "mixed": mixed, "student": stud, "large_system": large, "lammps_interface": lammps, "nnp_scaling": scal, "compact_functions": compact, "training": training, "stages_ms": {n: round(t, 4) for n, t in stages}, "work": work,
                "fp32_fma_peak_tflops": fp32_peak}
        print(json.dumps(line), flush=True)
    mode.close()
    for h in (hp, he, hf):
        mode._lib.n2p2_host_free(h[0])
    if dist is not None:
        dist.destroy_process_group()


# Algorithmic HBM bytes of the symmetry-function passes: per neighbour entry
# j, d, dx, dy, dz (36) + f_c, df_c (16) read by each pass, h_x,y,z (24)
# written by the force pass; per atom G written (values) and dE/dG read
# (forces), 8 bytes per function.
SF_BYTES_PER_ENTRY = {"sf_values": 52, "sf_forces": 52 + 24}


def bench_large(steps, warmup, device):
    """36,864-molecule water box, water56 model, FP64 and mixed."""
    import torch
    from n2p2_b200 import Mode, water
    s = water.water_box(36864, seed=2024, sigma=0.15)
    out = {"workload": "36864-molecule water box (%d atoms, edge %.2f bohr, 1.0 g/cm^3, 0.15 bohr displacements), "
                       "water56 model (G2 + G3 + wide G9, 56-64-64-1 softplus)" % (s.numAtoms, s.box[0, 0])}
    mode = Mode(device)
    mode.setupFromDirectory(TEACHER)
    res = {}
    for prec in ("fp64", "mixed"):
        mode.setPrecision(prec)
        b = mode.batch([s])
        b.setPositions(s.positions)
        b.evaluate(forces=True)
        b.synchronize()
        stream = torch.cuda.ExternalStream(b.stream(), device=torch.device("cuda", device))
        for _ in range(warmup):
            b.evaluate(forces=True)
        b.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.evaluate(forces=True)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        stages = dict(b.profileStages(forces=True))
        work = b.countWork()
        nsf = 56
        gbs = {}
        for k, per in SF_BYTES_PER_ENTRY.items():
            if stages.get(k):
                nbytes = work["entries"] * per + s.numAtoms * 8 * nsf
                gbs[k] = nbytes / (stages[k] * 1e-3) / 1e9
        res[prec] = {"value": s.numAtoms / (ms / 1000.0), "unit": "atoms/s", "ms_per_step": ms,
                     "stages_ms": {k: round(v, 4) for k, v in stages.items()},
                     "sf_hbm_GBps_algorithmic": gbs,
                     "E": b.energies()[0], "F": b.forces()}
        b.close()
    de = abs(res["mixed"]["E"] - res["fp64"]["E"]) / s.numAtoms * HA_TO_MEV
    df = np.abs(res["mixed"]["F"] - res["fp64"]["F"]) * HA_BOHR_TO_MEV_A
    for prec in res:
        res[prec].pop("E")
        res[prec].pop("F")
    res["mixed"]["speedup_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
    res["mixed"]["err_vs_fp64_gpu"] = {"energy_meV_per_atom": float(de), "force_meV_per_A_max": float(df.max()),
                                       "force_meV_per_A_rms": float(np.sqrt((df ** 2).mean()))}
    out.update(res)
    out["network"] = ("FP64 form: CUDA-core kernel over 16-atom tiles (the 56-64-64-1 stage does not fit 32-atom "
                      "tiles); mixed form: tcgen05 tensor-core products with split-bfloat16 operands and FP32 "
                      "accumulators (tensor-pipe activity is an ncu counter: profiles/ncu_network_tc_water110k_mixed.md)")
    mode.close()
    return out


def bench_scaling(structs, device, cpu=True):
    """nnp-scaling on the GPU for the batched workload: the input.data file
    read by the library's reader, then the symmetry-function statistics
    written as scaling.data (n2p2_b200.scaling), wall clock per phase; beside
    it the reference's per-structure nnp-scaling work (neighbour list +
    symmetry functions without derivatives) on the host threads."""
    import shutil
    from n2p2_b200 import read_structures, scaling, write_structures
    natoms = sum(s.numAtoms for s in structs)
    out = {"workload": "%d water boxes (%d atoms), water40 descriptors, input.data -> scaling.data"
                       % (len(structs), natoms), "unit": "atoms/s"}
    with tempfile.TemporaryDirectory() as d:
        shutil.copy(os.path.join(MODEL, "input.nn"), d)
        path = os.path.join(d, "input.data")
        write_structures(path, structs)
        t0 = time.perf_counter()
        ss = read_structures(path)
        t_read = time.perf_counter() - t0
        scaling.nnp_scaling(d, structures=ss[:64], device=device)   # CUDA context and kernels warm
        t0 = time.perf_counter()
        scaling.nnp_scaling(d, structures=ss, device=device)
        t_stats = time.perf_counter() - t0
        out["read_input_data"] = {"value": natoms / t_read, "seconds": t_read,
                                  "file_bytes": os.path.getsize(path)}
        out["statistics"] = {"value": natoms / t_stats, "seconds": t_stats}
        out["value"] = natoms / (t_read + t_stats)
    if cpu:
        try:
            from oracle import ref
            threads = host_threads()
            sample, nsample = cpu_sample(structs, threads)
            sec = ref.time_sf_batch(MODEL, [x.to_text() for x in sample], threads, fast=True)
            out["cpu_reference"] = {"value": nsample / sec, "unit": "atoms/s", "cores": threads, "kind": "reference",
                                    "sample": "%d structures (%d atoms): neighbour list + calculateSymmetryFunction"
                                              "Groups (no derivatives), reference libnnp -O3, structure-parallel"
                                              % (len(sample), nsample)}
        except Exception as exc:   # the GPU numbers stand without it
            out["cpu_reference"] = {"value": None, "sample": "failed: %s" % exc}
    return out


def _compact_run(d, structs, steps, warmup, device, cpu, cpu_sample=None):
    """FP64 energies and forces of `structs` under the model in `d`, CUDA
    events on the batch stream; beside it the reference library on a bounded
    sample, all host threads."""
    import torch
    from n2p2_b200 import Mode
    natoms = sum(x.numAtoms for x in structs)
    mode = Mode(device)
    mode.setupFromDirectory(d)
    b = mode.batch(structs)
    b.setPositions(np.concatenate([x.positions for x in structs]))
    b.evaluate(forces=True)
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream(), device=torch.device("cuda", device))
    for _ in range(warmup):
        b.evaluate(forces=True)
    b.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        b.evaluate(forces=True)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    stages = dict(b.profileStages(forces=True))
    out = {"value": natoms / (ms / 1e3), "unit": "atoms/s", "ms_per_step": ms,
           "stages_ms": {k: round(v, 3) for k, v in stages.items()}}
    b.close()
    mode.close()
    if cpu:
        try:
            from oracle import ref
            threads = host_threads()
            sample = structs[:max(1, min(len(structs), cpu_sample or threads))]
            sec, _ = ref.time_batch(d, [x.to_text() for x in sample], threads, fast=True)
            n = sum(x.numAtoms for x in sample)
            out["cpu_reference"] = {"value": n / sec, "unit": "atoms/s", "cores": threads, "kind": "reference",
                                    "sample": "%d structures (%d atoms), reference libnnp -O3 evaluateNNP, "
                                              "structure-parallel" % (len(sample), n)}
        except Exception as exc:   # the GPU numbers stand without it
            out["cpu_reference"] = {"value": None, "sample": "failed: %s" % exc}
    return natoms, out


def _compact_wide_work(d, structs, nbr):
    """Pairs and FP64 operations per E+F evaluation of the wide angular
    groups (types 22, 25) of the model in `d`, counted for the factored
    algorithm of the staged kernels: per pair of a group with nR radial and
    nA angular parts, G pass 8 (geometry) + 8 nA (angular parts) + nR
    (radial products) + 2 nR nA (grid sums); force pass 11 (geometry,
    dtheta/dcos) + 12 nA (parts and derivatives) + 4 nR nA (U_r, V_r) +
    9 nR (radial sums) + 34 (coefficients, both neighbours' forces).  The
    radial parts of the neighbours (per neighbour, not per pair) and acos
    are not counted."""
    import collections
    groups = collections.defaultdict(lambda: (set(), set()))
    for line in open(os.path.join(d, "input.nn")):
        t = line.split()
        if t[:1] != ["symfunction_short"] or t[2] not in ("22", "25"):
            continue
        if t[2] == "22":
            key = (t[1], "22") + tuple(sorted((t[3], t[4])))
            rl, rc, al, ar, sub = t[5], t[6], t[7], t[8], t[9]
        else:
            key = (t[1], "25")
            rl, rc, al, ar, sub = t[3], t[4], t[5], t[6], t[7]
        groups[key][0].add((float(rl), float(rc), sub))
        groups[key][1].add((float(al), float(ar), sub.rstrip("a")))
    elem = np.concatenate([np.array(x.elements) for x in structs])
    off, idx = nbr["offset"], nbr["index"]
    pairs = flops = 0
    for i in range(len(elem)):
        ne = collections.Counter(elem[idx[off[i]:off[i + 1]]])
        n = off[i + 1] - off[i]
        for key, (rad, ang) in groups.items():
            if key[0] != elem[i]:
                continue
            if key[1] == "25":
                p = n * (n - 1) // 2
            elif key[2] == key[3]:
                p = ne[key[2]] * (ne[key[2]] - 1) // 2
            else:
                p = ne[key[2]] * ne[key[3]]
            nR, nA = len(rad), len(ang)
            pairs += p
            flops += p * ((8 + 8 * nA + nR + 2 * nR * nA) + (11 + 12 * nA + 4 * nR * nA + 9 * nR + 34))
    return pairs, flops


def _perturbed(s0, count, seed, sigma):
    from n2p2_b200 import Structure
    rng = np.random.default_rng(seed)
    return [Structure(s0.positions + rng.normal(scale=sigma, size=s0.positions.shape), s0.elements, box=s0.box)
            for _ in range(count)]


def bench_compact(steps, warmup, device, cpu=True):
    """Compact symmetry functions, FP64 energies and forces.  Headline: the
    reference's Anisole SCAN model (331-354 functions per element, compact
    radial 20 + wide angular 22) on 64 copies of its 256-atom periodic box
    with seeded 0.02 displacements.  Beside it the other compact types: the
    SCAN functions made narrow (type 21) on 16 copies of the Ethylbenzene
    288-atom box, and the reference's QM9 settings (weighted types 23-25,
    five elements) on 4096 molecules (its 19 fixture molecules, seeded 0.02
    displacements)."""
    from n2p2_b200 import read_structures
    golden = os.path.join(ROOT, "tests", "golden")
    d = os.path.join(golden, "examples", "Anisole_SCAN")
    anisole = _perturbed(read_structures(os.path.join(d, "input.data"))[0], 64, 5, 0.02)
    natoms, out = _compact_run(d, anisole, steps, warmup, device, cpu)
    out = {"workload": "Anisole_SCAN model (reference example; compact types 20 + 22), 64 x 256-atom periodic boxes "
                       "(%d atoms)" % natoms, **out}
    # roofline of the staged angular passes (the stage times include the radial type-20 launches)
    from n2p2_b200 import Mode
    m = Mode(device)
    m.setupFromDirectory(d)
    b = m.batch(anisole)
    b.setPositions(np.concatenate([x.positions for x in anisole]))
    b.evaluate(forces=False)
    pairs, flops = _compact_wide_work(d, anisole, b.neighbors())
    d64, d32 = ctypes_double(), ctypes_double()
    peak = d64.value if m._lib.n2p2_device_fma_peak(device, d64.ref, d32.ref) == 0 else None   # TFLOP/s
    b.close()
    m.close()
    sec = (out["stages_ms"]["sf_values"] + out["stages_ms"]["sf_forces"]) / 1e3
    out["roofline"] = {"bound": "fp64", "kernel": "kCompactWideValues + kCompactWideForces (with the type-20 launches)",
                       "achieved": flops / sec / 1e12, "peak": peak, "unit": "TFLOP/s",
                       "frac": (flops / sec / 1e12 / peak) if peak else None,
                       "peak_source": "measured FP64 FMA throughput of this GPU (n2p2_device_fma_peak)",
                       "pairs_per_step": pairs, "flops_per_step": flops,
                       "flops_model": "factored staged algorithm per pair (bench.py _compact_wide_work)"}
    d = os.path.join(golden, "models", "scan_narrow")
    natoms, o = _compact_run(d, _perturbed(read_structures(os.path.join(d, "input.data"))[0], 16, 6, 0.02),
                             steps, warmup, device, cpu)
    out["narrow"] = {"workload": "SCAN functions made narrow (types 20 + 21), 16 x 288-atom Ethylbenzene boxes "
                                 "(%d atoms)" % natoms, **o}
    d = os.path.join(golden, "models", "qm9_weighted")
    mols = read_structures(os.path.join(d, "input.data"))
    rng = np.random.default_rng(7)
    picks = [mols[k] for k in rng.integers(0, len(mols), size=4096)]
    from n2p2_b200 import Structure
    structs = [Structure(m.positions + rng.normal(scale=0.02, size=m.positions.shape), m.elements) for m in picks]
    natoms, o = _compact_run(d, structs, steps, warmup, device, cpu, cpu_sample=512)
    out["weighted"] = {"workload": "QM9 settings (reference training example; weighted types 23 + 24 + 25, five "
                                   "elements), 4096 molecules (%d atoms)" % natoms, **o}
    return out


def bench_training(steps, warmup, device, cpu=True):
    """Training updates (Training::update with KalmanFilter::update, standard
    filter, force weight 10): the water40 networks (3402 weights, covariance
    3402 x 3402 FP64 = 92.6 MB), 256 water boxes of 32-128 molecules labelled
    by the model's own weights, training from weights perturbed by N(0, 0.02).
    Energy and force updates are timed separately (CUDA events on the set's
    stream), 256 updates per timed step.  Each filter update reads and writes
    the covariance's lower half once (the previous update's rank-one change
    fused with this update's X = P H): 8 n^2 bytes, the HBM roofline of the
    filter's share of an update.  Beside it the numpy restatement of the
    same updates on a bounded sample (the reference's training program needs
    MPI and GSL, which this image lacks)."""
    import time
    import torch
    from n2p2_b200 import Mode, water
    from n2p2_b200.training import ENERGY, FORCE, Training
    wdir = os.path.join(ROOT, "tests", "golden", "models", "water40")
    m = Mode(device)
    m.setupFromDirectory(wdir)
    ss = water.water_batch(256, seed=31, n_min=32, n_max=128)
    b = m.batch(ss)
    b.setPositions(np.concatenate([x.positions for x in ss]))
    b.evaluate(forces=True)
    E, F = b.energies(), b.forces()
    b.close()
    tr = Training(m, ss, E, F)
    w0 = tr.weights() + np.random.default_rng(5).normal(0.0, 0.02, tr.numWeights)
    tr.setWeights(w0)
    tr.setupUpdaterKalman(0)
    tr.setForceWeight(10.0)
    n = tr.numWeights
    ec, (fs, fa, fc) = tr.updateCandidates()
    rng = np.random.default_rng(2)
    per = 256
    eo = rng.permutation(ec.size)
    fo = rng.permutation(fs.size)[:per * (steps + warmup)]
    stream = torch.cuda.ExternalStream(tr.batch.stream(), device=torch.device("cuda", device))
    out = {"workload": "water40 networks (%d weights, covariance %.1f MB FP64), 256 water boxes of 32-128 molecules "
                       "(%d atoms), standard Kalman filter, force weight 10"
                       % (n, 8.0 * n * n / 1e6, sum(x.numAtoms for x in ss)),
           "unit": "updates/s"}
    for name, prop in (("energy", ENERGY), ("force", FORCE)):
        def run(k):
            idx = np.arange(k * per, (k + 1) * per)
            if prop == ENERGY:
                tr.update(ENERGY, ec[eo[idx % ec.size]])
            else:
                tr.update(FORCE, fs[fo[idx]], fa[fo[idx]], fc[fo[idx]])
        for k in range(warmup):
            run(k)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(warmup, warmup + steps):
            run(k)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / (steps * per)
        out[name] = {"value": 1e3 / ms, "ms_per_update": ms,
                     "kalman_hbm_GBps_lower_bound": 8.0 * n * n / (ms * 1e-3) / 1e9}
    out["errors_after"] = tr.errors()
    out["kalman_status"] = tr.kalmanStatus()
    tr.close()
    m.close()
    if cpu:
        try:
            from oracle import training_ref as T
            sample = ss[:2]
            up = T.KalmanFilter(n, 0, 1e-2, 0.01, 2.302, 1e-6, 0.01, 2.302, 1.0)
            ref = T.Training(wdir, sample, E[:2], F[:sum(x.numAtoms for x in sample)], up, force_weight=10.0)
            ref.nets.weights = w0.copy()
            t0 = time.perf_counter()
            for k in range(3):
                ref.update(0, k % 2)
            sec = (time.perf_counter() - t0) / 3
            out["cpu_reference"] = {"value": 1.0 / sec, "unit": "updates/s", "cores": 1, "kind": "port",
                                    "sample": "3 energy updates (numpy restatement: network Jacobian over a "
                                              "box's atoms + Kalman update of the full covariance)"}
        except Exception as exc:
            out["cpu_reference"] = {"value": None, "sample": "failed: %s" % exc}
    return out


def lammps_rank(s, list_cut_bohr, type_of):
    """One LAMMPS rank holding a whole cubic periodic box (Angstrom units):
    local atoms wrapped into the cell, ghost images within the list cutoff
    (pair cutoff + skin) outside it, full neighbour lists of the local atoms
    (ascending j, self excluded).  Returns x [nall,3], type [nall], nlocal,
    numneigh, firstneigh (flat), ilist."""
    import itertools
    from scipy.spatial import cKDTree
    L = np.diag(np.asarray(s.box, dtype=np.float64))
    n = s.numAtoms
    frac = s.positions / L
    frac -= np.floor(frac)
    xs, owners = [frac * L], [np.arange(n)]
    for sh in itertools.product((-1, 0, 1), repeat=3):
        if sh != (0, 0, 0):
            f = frac + np.array(sh, dtype=np.float64)
            keep = np.all((f >= -list_cut_bohr / L) & (f < 1.0 + list_cut_bohr / L), axis=1)
            xs.append(f[keep] * L)
            owners.append(np.nonzero(keep)[0])
    x = np.concatenate(xs)
    owner = np.concatenate(owners)
    m = cKDTree(x[:n]).sparse_distance_matrix(cKDTree(x), list_cut_bohr, output_type="coo_matrix")
    keep = m.row != m.col
    r, c = m.row[keep], m.col[keep]
    o = np.lexsort((c, r))
    r, c = r[o], c[o]
    types = np.array([type_of[e] for e in s.elements], dtype=np.int32)[owner]
    return {"x": x * BOHR_TO_A, "type": types, "nlocal": n,
            "numneigh": np.bincount(r, minlength=n).astype(np.int32), "firstneigh": c.astype(np.int32),
            "ilist": np.arange(n, dtype=np.int32)}


def bench_lammps(steps, warmup, device, cpu=True):
    """MD steps through the LAMMPS interface (n2p2_lammps_*), as pair_style
    hdnnp drives it on one rank: 12,288-molecule water box (36,864 local
    atoms) in Angstrom/eV with its ghost atoms and full neighbour lists
    (6.5 A pair cutoff + 1 A skin), water56 model.  Each step: setLocalAtoms,
    neighbour transfer, process, energy, forces on local and ghost atoms; host
    arrays in and out, wall clock (the interface is synchronous)."""
    from n2p2_b200 import water
    from n2p2_b200.lammps import InterfaceLammps
    pair_cut, skin = 6.5, 1.0
    cfl, cfe = 1.0 / BOHR_TO_A, 1.0 / HA_TO_EV
    s = water.water_box(12288, seed=77, sigma=0.1)
    dom = lammps_rank(s, (pair_cut + skin) / BOHR_TO_A, {"H": 1, "O": 2})
    n, nall = dom["nlocal"], len(dom["x"])
    out = {"workload": "LAMMPS-style rank: 12288-molecule water box (%d local + %d ghost atoms, %d list entries), "
                       "water56, Angstrom/eV, pair cutoff 6.5 A + 1 A skin" % (n, nall - n, len(dom["firstneigh"])),
           "unit": "atoms/s"}
    F = np.zeros((nall, 3))
    for prec in ("fp64", "mixed"):
        lmp = InterfaceLammps(device).initialize(TEACHER, "1:H,2:O", False, False, 0, -1, cfl, cfe, pair_cut, 2, 0)
        lmp.setPrecision(prec)
        t_tr = t_pr = t_f = 0.0
        for k in range(warmup + steps):
            t0 = time.perf_counter()
            lmp.setLocalAtoms(n, dom["type"][:n])
            lmp.transferNeighborList(dom["ilist"], dom["numneigh"], dom["firstneigh"], dom["x"], dom["type"], pair_cut)
            t1 = time.perf_counter()
            lmp.process()
            lmp.getEnergy()
            t2 = time.perf_counter()
            F[:] = 0.0
            lmp.getForces(F)
            t3 = time.perf_counter()
            if k >= warmup:
                t_tr += t1 - t0
                t_pr += t2 - t1
                t_f += t3 - t2
        ms = 1e3 * (t_tr + t_pr + t_f) / steps
        out[prec] = {"value": n / (ms / 1e3), "ms_per_step": ms,
                     "host_ms": {"transfer_neighbor_list": 1e3 * t_tr / steps,
                                 "process_and_energy": 1e3 * t_pr / steps, "get_forces": 1e3 * t_f / steps}}
        lmp.close()
    if cpu:
        # the reference's own InterfaceLammps (timed build, one host thread) on
        # a 1,536-atom rank of the same recipe
        try:
            from oracle import lammps_ref
            small = water.water_box(512, seed=78, sigma=0.1)
            d2 = lammps_rank(small, (pair_cut + skin) / BOHR_TO_A, {"H": 1, "O": 2})
            ref = lammps_ref.RefInterfaceLammps(TEACHER, "1:H,2:O", cfl, cfe, pair_cut, 2, fast=True)
            x = d2["x"]
            offs, js, drs, d2s = [0], [], [], []
            start = 0
            for i in range(d2["nlocal"]):
                nb = d2["firstneigh"][start:start + d2["numneigh"][i]]
                start += d2["numneigh"][i]
                dr = x[i] - x[nb]
                q = dr[:, 0] * dr[:, 0] + dr[:, 1] * dr[:, 1] + dr[:, 2] * dr[:, 2]
                sel = q <= pair_cut * pair_cut
                js.append(nb[sel])
                drs.append(dr[sel])
                d2s.append(q[sel])
                offs.append(offs[-1] + int(sel.sum()))
            js = np.concatenate(js)
            args = (d2["type"][:d2["nlocal"]], np.array(offs), js, d2["type"][js], np.concatenate(drs),
                    np.concatenate(d2s), len(x))
            ref.evaluate(*args, num_centres=0)
            t0 = time.perf_counter()
            ref.evaluate(*args, num_centres=0)
            sec = time.perf_counter() - t0
            ref.close()
            out["cpu_reference"] = {"value": d2["nlocal"] / sec, "unit": "atoms/s", "cores": 1, "kind": "reference",
                                    "sample": "reference InterfaceLammps (libnnp -O3, x86-64-v3), setLocalAtoms + "
                                              "addNeighbor + process + getForces on a %d-atom rank, one thread"
                                              % d2["nlocal"]}
        except Exception as exc:   # the GPU numbers stand without it
            out["cpu_reference"] = {"value": None, "sample": "failed: %s" % exc}
    return out


def _oracle_teacher(args):
    """Teacher energy and forces of one structure by the FP64 CPU oracle (a
    worker of student_vs_oracle's process pool); args = (model directory,
    input.data text)."""
    from oracle.port import PortModel
    from n2p2_b200.structure import read_structures
    teacher, text = args
    s = read_structures(text, is_text=True)[0]
    r = PortModel(teacher).evaluate(s)
    return r["energy"], np.asarray(r["forces"])


def student_vs_oracle(pred, count=64, teacher=TEACHER):
    """Student (with fallback) against the FP64 CPU oracle of the teacher on
    the first `count` held-out structures (the oracle restates the reference
    on the host; it is the checker here, not a timed path), evaluated by a
    pool of host processes."""
    import multiprocessing as mp
    from n2p2_b200 import student as student_mod
    structs, Es, Fs = pred
    count = min(count, len(structs))
    texts = [s.to_text() for s in structs[:count]]
    with mp.get_context("spawn").Pool(max(1, min(16, host_threads()))) as pool:
        res = pool.map(_oracle_teacher, [(teacher, t) for t in texts])
    E_o = [r[0] for r in res]
    F_o = [r[1] for r in res]
    na = [s.numAtoms for s in structs[:count]]
    out = student_mod.errors(Es[:count], Fs[:sum(na)], E_o, np.concatenate(F_o), na)
    out["structures"] = count
    return out


def _shape_names(t):
    from n2p2_b200.mode import Batch
    name = lambda v: "%d x %d" % Batch.SHAPES[v]
    return {"values": name(t["values"]), "forces": name(t["forces"]),
            "values_ms": {name(v): round(x, 3) for v, x in enumerate(t["values_ms"])},
            "forces_ms": {name(v): round(x, 3) for v, x in enumerate(t["forces_ms"])},
            "shape": "first-tier stage capacity x warps per block"}


class ctypes_double:
    def __init__(self):
        import ctypes
        self._v = ctypes.c_double()
        self.ref = ctypes.byref(self._v)

    @property
    def value(self):
        return self._v.value


def ctypes_pinned(nbytes):
    import ctypes
    from n2p2_b200 import _lib
    lib = _lib.load()
    p = ctypes.c_void_p()
    _lib.check(lib.n2p2_host_alloc(ctypes.byref(p), nbytes))
    buf = (ctypes.c_char * nbytes).from_address(p.value)
    return p, buf


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
