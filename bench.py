#!/usr/bin/env python3
"""Benchmark: mixed-precision batched CG solves/s on one B200 at 1e-10.

Workload (the uneven batch): 64 independent D D^dag solves drawn with seed 7
from lattices {8^4, 12^4, 16^4, 16^3x32}, masses {0.05, 0.1, 0.2}, gauge
roughness eps {0.3, 1.0} and 1-8 Gaussian right-hand sides each, solved
together as one batch (CUDA graphs of 16 CG iterations per replay) to an FP64
true relative residual of 1e-10.  A "solve"
is one full-lattice solve of D D^dag X = phi (both parity blocks), the unit of
the reference's solve_CG_DDdagger.  Inputs are synthetic: gauge links
U = exp(i eps H) and N(0,1) sources from the library's seeded generators.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision f32|f16]
    python bench.py --impl reference ...     (reference CPU arm)

Prints one JSON line on rank 0.  Multi-GPU runs are replicas (weak scaling,
no collective on the data path): every rank solves its own copy of the batch.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LATTICES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32)]
MASSES = [0.05, 0.1, 0.2]
EPSES = [0.3, 1.0]
TOL = 1e-10
MAXIT = 20000
METRIC = "mixed-prec batched CG solves/s vs FP64 CG on 1 B200 @1e-10 resid; Dslash HBM GB/s"


def batch_spec(seed=7, nsys=64):
    rng = np.random.default_rng(seed)
    spec = []
    for k in range(nsys):
        dims = LATTICES[int(rng.integers(len(LATTICES)))]
        mass = MASSES[int(rng.integers(len(MASSES)))]
        eps = EPSES[int(rng.integers(len(EPSES)))]
        nrhs = int(rng.integers(1, 9))
        spec.append({"dims": dims, "mass": mass, "eps": eps, "nrhs": nrhs,
                     "gauge_seed": 1000 + k, "rhs_seed": 100000 + 100 * k})
    return spec


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes of one batched solve, per iteration kernel
#
# Per lane (one parity system of one RHS) and CG iteration, per site of the
# lane's parity (s = spinor bytes, sx = bytes of the solution increment):
#   cg_hop1   reads p, writes t                       2 s
#   cg_hop2   reads t, r, p, writes v                 4 s
#   cg_update reads p, r, v, x, writes x, r, p        5 s + 2 sx
# Links: each hop kernel reads the 8 links of every output site once per
# (system, parity, iteration), shared by all RHS of the system.  A reliable
# update (mixed precision) adds an FP64 hop in each hop kernel (8 FP64 links,
# the FP64 solution or temporary) and the FP64 residual in cg_hop2.
# ---------------------------------------------------------------------------
# the arithmetic each solver precision computes in (dtype of the bench line)
DTYPE = {"f16": "f16", "bf16": "f32", "f32": "f32", "f32_18": "f32", "f64": "f64"}
ARITHMETIC = {
    "f16": "f16 storage with a per-site scale; hop products in packed f16 (half2), each neighbour's product "
           "accumulated in f32; f64 reliable updates",
    "bf16": "bf16 storage with a per-site scale; f32 products and accumulation; f64 reliable updates",
    "f32": "f32 storage (12-real links); f32 products and accumulation; f64 reliable updates",
    "f32_18": "f32 storage (18-real links); f32 products and accumulation; f64 reliable updates",
    "f64": "f64 storage and arithmetic (plain CG)",
}
SPINOR_BYTES = {"f64": 48, "f32": 24, "f16": 16, "f32_18": 24, "bf16": 16}
LINK_BYTES = {"f64": 144, "f32": 48, "f16": 24, "f32_18": 72, "bf16": 24}
# the solution increment x_lo between reliable updates: FP32 for every mixed
# precision (the FP64 solve updates x_hi directly)
X_BYTES = {"f64": 48, "f32": 24, "f16": 24, "f32_18": 24, "bf16": 24}
KERNELS = ("cg_hop1", "cg_hop2", "cg_update")


def kernel_bytes(spec, infos, precision, ru_separate=False):
    """{kernel: algorithmic bytes over one solve} from the lanes' iteration
    and reliable-update counts.  ru_separate: the reliable-update hops run in
    kernels of their own (cg_ru1, cg_ru2; the system-blocked schedule)."""
    s = SPINOR_BYTES[precision]
    sx = X_BYTES[precision]
    lb = LINK_BYTES[precision]
    out = dict.fromkeys(KERNELS + (("cg_ru1", "cg_ru2") if ru_separate else ()), 0.0)
    ru1, ru2 = ("cg_ru1", "cg_ru2") if ru_separate else ("cg_hop1", "cg_hop2")
    for k, sys_ in enumerate(spec):
        Vh = int(np.prod(sys_["dims"])) // 2
        group_iters = [0, 0]
        for j in range(sys_["nrhs"]):
            inf = infos[k][j]
            for par in (0, 1):
                it = inf["iters_parity"][par]
                nru = inf["reliable_updates"] / 2.0
                out["cg_hop1"] += it * Vh * 2 * s
                out["cg_hop2"] += it * Vh * 4 * s
                out["cg_update"] += it * Vh * (5 * s + 2 * sx)
                if precision != "f64":
                    # FP64 hop of x (links, x_hi + x_lo in, t_hi out); FP64
                    # hop of t_hi, x_hi, x_lo, b in, x_hi, x_lo, r out, and
                    # the search direction rebuilt (r, p in, p out)
                    out[ru1] += nru * Vh * (8 * 144 + 48 + sx + 48)
                    out[ru2] += nru * Vh * (8 * 144 + 48 + 2 * 48 + 2 * sx + 48 + s + 3 * s)
                group_iters[par] = max(group_iters[par], it)
        for par in (0, 1):
            out["cg_hop1"] += group_iters[par] * 8 * lb * Vh
            out["cg_hop2"] += group_iters[par] * 8 * lb * Vh
    return out


def solve_bytes(spec, infos, precision):
    return sum(kernel_bytes(spec, infos, precision).values())  # the same whichever kernels do the hops


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per
# algorithmic byte of cg_hop2 for one launch of the first 8 systems of the
# batch with every lane active, RHS groups of 2, 4 tiles per work item, links
# read directly, reliable updates in the lane-list kernels (the headline
# schedule): f16 283.4 MB for 291.9 MB (an ncu capture of the hop kernels,
# summarised under profiles/); f32 553.2 MB for 491.0 MB (the FP32 capture
# summarised there, of the same work items with the updates inside the hop
# kernels).  The bench scales it to its own launches by their algorithmic
# bytes.
HOP2_TRAFFIC_PER_ALG_BYTE = {"f32": 553.2 / 491.0, "f16": 283.4 / 291.9}


def build_batch(sfh, spec, precision, device):
    B = sfh.Batch([(s["dims"], s["mass"], s["nrhs"]) for s in spec], precision=precision, device=device)
    for k, s in enumerate(spec):
        B.random_gauge(k, s["eps"], s["gauge_seed"])
        for j in range(s["nrhs"]):
            B.random_rhs(k, j, s["rhs_seed"] + j)
    return B


def time_steps(torch, stream_ptr, fn, steps, warmup):
    stream = torch.cuda.ExternalStream(stream_ptr)
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = []
    with torch.cuda.stream(stream):
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            ev.append((a, b))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def e2e_pipelined(torch, pair, upload, download, steps):
    """ms per step of `steps` end-to-end steps through the public API, the
    two batches of `pair` taking turns: step n uploads its inputs, solves and
    downloads its solutions on batch n % 2, and its uploads and downloads run
    (from a second host thread; the library's calls release the GIL) while
    the other batch solves.  CUDA events on the first batch's stream bracket
    every step's copies and solve, the first upload and the last download
    included."""
    import threading
    for X in pair:  # warm-up: builds each batch's graph
        upload(X)
        X.solve(tol=TOL, max_iter=MAXIT)
        download(X)
    torch.cuda.synchronize()
    s0 = torch.cuda.ExternalStream(pair[0].stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s0)
    upload(pair[0])
    for n in range(steps):
        jobs = []
        if n >= 1:
            jobs.append((download, pair[(n - 1) % 2]))
        if n + 1 < steps:
            jobs.append((upload, pair[(n + 1) % 2]))
        errors = []

        def side():
            try:
                for fn, X in jobs:
                    fn(X)
            except Exception as e:  # re-raised on the main thread
                errors.append(e)

        t = threading.Thread(target=side)
        t.start()
        try:
            pair[n % 2].solve(tol=TOL, max_iter=MAXIT)
        finally:
            t.join()
        if errors:
            raise errors[0]
    download(pair[(steps - 1) % 2])
    torch.cuda.synchronize()
    e1.record(s0)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


# ---------------------------------------------------------------------------
# CPU baselines: the reference's own CG on a sample stratified over the
# batch's (lattice, mass, eps) classes
#
# The batch's 296 solves fall into at most 24 classes (4 lattices x 3 masses x
# 2 gauge roughnesses).  A sample times one reference solve of a class's first
# system (its first right-hand side), classes taken in a fixed rotation that
# continues from step to step.  The batch's CPU time is estimated as
# sum_c n_c t_c (n_c the class's number of solves, t_c its mean timed solve),
# and the CPU solves/s as total_solves / that time, so every class counts
# with its share of the batch.  Inputs come from the oracle's restatement of
# the library's seeded generators (identical fields to the GPU arm's, without
# loading the library).
# ---------------------------------------------------------------------------
def batch_classes(spec):
    """[(key, first system index, number of solves)] in batch order of first
    appearance; key = (dims, mass, eps)."""
    order, info = [], {}
    for k, s in enumerate(spec):
        key = (tuple(s["dims"]), s["mass"], s["eps"])
        if key not in info:
            info[key] = [k, 0]
            order.append(key)
        info[key][1] += s["nrhs"]
    return [(key, info[key][0], info[key][1]) for key in order]


def class_name(key):
    dims, mass, eps = key
    return f"{'x'.join(map(str, dims))}/m{mass}/eps{eps}"


class CpuSampler:
    """Times reference solves class by class, in rotation.  kind per sample:
    'reference' (oracle/_ref, the reference's own sources) or 'port' (the C
    restatement in-process, where no reference binary exists)."""

    def __init__(self, spec, workdir):
        import oracle
        oracle.lib()
        self.oracle = oracle
        self.spec = spec
        self.classes = batch_classes(spec)
        self.cursor = 0
        self.workdir = workdir
        self.inputs = {}

    def _exe(self, key):
        from oracle import build_ref
        dims, mass, _ = key
        if not (dims[0] == dims[1] == dims[2]):
            return None
        exe = build_ref.exe_path(dims[0], dims[3], mass, TOL)
        return exe if os.path.exists(exe) else None

    def _input_dir(self, ci):
        """U.bin / phi.bin of class ci's representative solve, written once."""
        if ci not in self.inputs:
            key, k, _ = self.classes[ci]
            s = self.spec[k]
            d = os.path.join(self.workdir, f"class{ci}")
            os.makedirs(d, exist_ok=True)
            U = self.oracle.philox_gauge(s["dims"], s["eps"], s["gauge_seed"])
            b = self.oracle.philox_spinor(s["dims"], s["rhs_seed"])
            U.astype("<f8").tofile(os.path.join(d, "U.bin"))
            b.astype("<f8").tofile(os.path.join(d, "phi.bin"))
            self.inputs[ci] = d
        return self.inputs[ci]

    def time_class(self, ci):
        key, k, _ = self.classes[ci]
        d = self._input_dir(ci)
        exe = self._exe(key)
        if exe:
            out = subprocess.run([exe, "time", d, "1"], check=True, capture_output=True, text=True,
                                 env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count())))
            return float(json.loads(out.stdout.strip().splitlines()[-1])["solve_s"]), "reference"
        dims, mass, _ = key
        U = np.fromfile(os.path.join(d, "U.bin"))
        b = np.fromfile(os.path.join(d, "phi.bin"))
        t0 = time.perf_counter()
        self.oracle.cg(dims, mass, U, b, TOL, MAXIT)
        return time.perf_counter() - t0, "port"

    def step(self, budget_s, max_classes=None):
        """Time classes in rotation until budget_s of wall time is spent (at
        least one); returns [(class index, solve seconds, kind)]."""
        out, t0 = [], time.perf_counter()
        while not out or (time.perf_counter() - t0 < budget_s
                          and (max_classes is None or len(out) < max_classes)):
            ci = self.cursor
            self.cursor = (self.cursor + 1) % len(self.classes)
            t, kind = self.time_class(ci)
            out.append((ci, t, kind))
        return out

    def estimate(self, samples):
        """Class-weighted CPU solves/s over the classes that have samples."""
        per = {}
        for ci, t, _ in samples:
            per.setdefault(ci, []).append(t)
        covered = sorted(per)
        n = sum(self.classes[ci][2] for ci in covered)
        secs = sum(self.classes[ci][2] * float(np.mean(per[ci])) for ci in covered)
        kinds = sorted({kind for _, _, kind in samples})
        kind = kinds[0] if len(kinds) == 1 else "mixed"
        total = sum(c[2] for c in self.classes)
        return {
            "value": n / secs, "kind": kind,
            "classes_timed": len(covered), "classes": len(self.classes),
            "solves_timed": len(samples),
            "reference_solves": sum(1 for x in samples if x[2] == "reference"),
            "port_solves": sum(1 for x in samples if x[2] == "port"),
            "batch_cpu_seconds_estimate": secs * total / n,
            "per_class_seconds": {class_name(self.classes[ci][0]): float(np.mean(per[ci])) for ci in covered},
        }


def cpu_sample_desc(est):
    return (f"{est['solves_timed']} reference CG solves (solve_CG_DDdagger) stratified over "
            f"{est['classes_timed']} of the batch's {est['classes']} (lattice, mass, eps) classes, "
            f"one solve of each class's first system, weighted by the class's share of the batch's "
            f"solves; inputs from the oracle's Philox generators (the GPU arm's fields)")


# ---------------------------------------------------------------------------
def max_over_ranks(x, world, device="cuda"):
    """The step time of a replica run: the slowest rank's (all ranks call it
    in the same order)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, solves_per_rank, ms):
    """Whole-job solves/s: every rank solves its own copy of the batch."""
    return world * solves_per_rank / (ms / 1000.0)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_config(spec, world):
    """The workload both arms report (the same dict in both lines)."""
    return {"workload": "uneven batch: 64 systems from {8^4,12^4,16^4,16^3x32} x m{0.05,0.1,0.2}"
                        " x eps{0.3,1.0}, 1-8 RHS, seed 7",
            "total_solves": sum(s["nrhs"] for s in spec), "tol": TOL,
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (gauge+vectors of the batch >> 126 MB)"}


def run_reference_arm(args, spec):
    """The reference's own CG (oracle/_ref, all host threads) on the batch's
    classes in rotation, each step a bounded sample (--ref-budget seconds of
    solves).  The value is the class-weighted CPU solves/s over the timed
    steps' samples; ms_per_step is the measured wall time of a step."""
    import tempfile
    world, rank, local = dist_setup()
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as td:
        sampler = CpuSampler(spec, td)
        warm, timed, step_ms = [], [], []
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            got = sampler.step(args.ref_budget)
            ms = 1000.0 * (time.perf_counter() - t0)
            if step < args.warmup:
                warm += got
            else:
                timed += got
                step_ms.append(ms)
        # classes no timed step reached keep their warm-up samples
        seen = {ci for ci, _, _ in timed}
        est = sampler.estimate(timed + [x for x in warm if x[0] not in seen])
    v = est["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(step_ms), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded exp(i eps H) links, N(0,1) sources)",
            "config": workload_config(spec, world),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": os.cpu_count(), "kind": est["kind"],
                             "sample": cpu_sample_desc(est)},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_sample": {k: est[k] for k in ("classes_timed", "classes", "solves_timed", "reference_solves",
                                                     "port_solves", "batch_cpu_seconds_estimate")},
            "per_class_seconds": est["per_class_seconds"]}
    print(json.dumps(line), flush=True)


def c4_oracle_check(B, spec):
    """The batch's solutions against the oracle on the host: for the first
    system of every (lattice, mass, eps) class, the FP64 true residual of its
    first solution by the oracle's D D^dag (apply_DDdagger,
    Fermions.cpp:530-547); for the first system of each lattice also the
    distance to the oracle's FP64 CG solution (Fermions.cpp:553-617) and the
    oracle's iteration count beside the lane's."""
    import oracle
    oracle.lib()
    out, worst = {}, 0.0
    seen_dims = set()
    for key, k, _ in batch_classes(spec):
        s = spec[k]
        dims = s["dims"]
        U, b, X = B.gauge(k), B.rhs(k, 0), B.solution(k, 0)
        r = float(np.linalg.norm(b - oracle.ddag(dims, s["mass"], U, X)) / np.linalg.norm(b))
        worst = max(worst, r)
        row = {"true_resid": r, "iters": B.info(k, 0)["iters_parity"]}
        if dims not in seen_dims:
            seen_dims.add(dims)
            Xo, it, _, _ = oracle.cg(dims, s["mass"], U, b, TOL, MAXIT)
            row["err_vs_oracle_fp64"] = float(np.linalg.norm(X - Xo) / np.linalg.norm(Xo))
            row["oracle_iters_full_lattice"] = it
        out[class_name(key)] = row
    return {"worst_true_resid_oracle": worst, "per_class": out}


# algorithmic bytes per output site of one hop: its 8 links (144 / 48 / 24 /
# 72 / 24 / 96 B), one input vector (each is the neighbour of 8 sites but
# leaves DRAM once) and one output vector (48 / 24 / 16 / 24 / 16 / 48 B)
# (6 and 7: the storages of 2 and 4, time and z neighbours staged in shared
# memory by one bulk asynchronous copy per block)
DSLASH_BYTES = {0: 1248, 1: 432, 2: 224, 3: 624, 4: 224, 5: 864, 6: 224, 7: 224}
DSLASH_NAMES = {0: "f64_18", 1: "f32_12", 2: "f16_12", 3: "f32_18", 4: "bf16_12", 5: "f64_12",
                6: "f16_12_tstaged", 7: "bf16_12_tstaged"}


def run_extras(sfh, hbm, quick=False):
    """Secondary measurements on the other configurations of the workload
    family: Dslash GB/s at 32^3x64, the ill-conditioned 32^3x64 solve, the
    16^4 precision grid and the 4^4 trajectory (the 24^4 HMC configuration
    is its own run: --workload c5)."""
    import oracle
    ex = {}
    # Dslash at 32^3x64 (eps = 1.0 links), one parity per hop, inputs >> L2
    dims = (32, 32, 32, 64)
    lat = sfh.Lattice(dims, 0.01, 4.2)
    lat.random_gauge(1.0, 3)
    Vh = int(np.prod(dims)) // 2
    ds = {}
    for st in (0, 5, 3, 1, 2, 6, 4, 7):
        ms = lat.dslash_timing(st, nrep=20)
        gbs = DSLASH_BYTES[st] * Vh / (ms * 1e-3) / 1e9
        ds[DSLASH_NAMES[st]] = {"ms_per_hop": ms, "GB/s": gbs, "frac": gbs / hbm,
                                "frac_of_spec": gbs / HBM_SPEC_GBS, "bytes_per_site": DSLASH_BYTES[st]}
    ex["dslash_32x32x32x64"] = ds
    # ill-conditioned single solve: 32^3x64, eps = 1.0, m = 0.01; each
    # solution's true residual by the oracle's D D^dag on the host
    phi = lat.gaussian_spinor(11)
    U = lat.download_gauge()

    def oracle_resid(X):
        return float(np.linalg.norm(phi - oracle.ddag(dims, 0.01, U, X)) / np.linalg.norm(phi))

    sol = {}
    for prec in ("f64", "f16", "bf16", "f32"):  # the first solve of each builds its workspace
        lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec)
    t0 = time.perf_counter()
    X64, i64 = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision="f64", info=True)
    t64 = time.perf_counter() - t0
    sol["f64"] = {"iters": i64["iters"], "seconds": t64, "true_resid_oracle": oracle_resid(X64)}
    for prec in ("f16", "bf16", "f32"):
        t0 = time.perf_counter()
        try:
            Xm, im = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec, info=True)
        except sfh.SfhError as e:
            sol[prec] = {"error": str(e)}
            continue
        tm = time.perf_counter() - t0
        sol[prec] = {"iters": im["iters"], "reliable_updates": im["reliable_updates"], "seconds": tm,
                     "true_resid_oracle": oracle_resid(Xm),
                     "dist_to_f64_solution": float(np.linalg.norm(Xm - X64) / np.linalg.norm(X64)),
                     "speedup_vs_f64": t64 / tm, "arithmetic": ARITHMETIC[prec]}
    sol["note"] = ("bf16 and f32 are the configuration's 'FP32 math' (f32 products); f16 multiplies in "
                   "packed half2 and accumulates in f32")
    ex["c3_32x32x32x64_m0.01"] = sol
    del U
    lat.close()
    if quick:
        return ex
    # 16^4 grid: eps {0.3, 1.0} x m {0.1, 0.02} x storage
    grid = {}
    lat = sfh.Lattice((16, 16, 16, 16), 0.1, 4.2)
    for geps in (0.3, 1.0):
        lat.random_gauge(geps, 21)
        U = lat.download_gauge()
        phi = lat.gaussian_spinor(22)
        for m in (0.1, 0.02):
            lat.set_mass(m)
            Xo, it_o, _, _ = oracle.cg(lat.dims, m, U, phi, TOL, 40000)
            row = {"oracle_fp64_iters": it_o}
            for prec in ("f64", "f32_18", "f32", "f16", "bf16", "f16_persistent", "f32_persistent"):
                sched = (1, 1, 3) if prec.endswith("_persistent") else (0, 0, 0)
                lat.set_schedule(*sched)
                t0 = time.perf_counter()
                X, inf = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec.split("_p")[0],
                                               info=True)
                row[prec] = {"iters": inf["iters"], "ms": 1e3 * (time.perf_counter() - t0),
                             "true_resid_oracle": float(np.linalg.norm(phi - oracle.ddag(lat.dims, m, U, X))
                                                        / np.linalg.norm(phi)),
                             "err_vs_oracle_fp64": float(np.linalg.norm(X - Xo) / np.linalg.norm(Xo))}
            lat.set_schedule(0, 0, 0)
            grid[f"eps{geps}_m{m}"] = row
    ex["c2_16^4"] = grid
    lat.close()
    # 4^4 trajectory (beta 4.2, m 0.1, eps_md 0.1, N 10) and its CPU time
    dims = (4, 4, 4, 4)
    U = oracle.random_gauge(dims, 0.3, 1)
    P = oracle.random_momenta(dims, 2)
    phi = oracle.random_spinor(dims, 3) / np.sqrt(2.0)
    lat = sfh.Lattice(dims, 0.1, 4.2)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    t0 = time.perf_counter()
    X, its = lat.leapfrog(phi, 0.1, 10, tol=TOL)
    tg = time.perf_counter() - t0
    t0 = time.perf_counter()
    P2, U2, X2, its2 = oracle.leapfrog(dims, 0.1, 4.2, 0.1, 10, phi, P, U, tol=TOL)
    tc = time.perf_counter() - t0
    ex["c1_4^4_trajectory"] = {"gpu_seconds": tg, "cpu_seconds_port": tc, "cg_iters": its,
                               "max_abs_diff_U_vs_cpu": float(np.abs(lat.download_gauge() - U2).max()),
                               "plaquette": lat.compute_avg_plaq()}
    info = lat.hmc_trajectory(0.1, 10, seed=1, tol=TOL)
    ex["c1_4^4_trajectory"]["hmc"] = {"dH": info["dH"], "accepted": info["accepted"],
                                      "plaquette": info["plaquette"], "seconds": info["seconds"]}
    lat.close()
    return ex


# ---------------------------------------------------------------------------
# C5: full HMC on 24^4 (bench.py --workload c5)
# ---------------------------------------------------------------------------
# algorithmic bytes and flops per link of the HMC kernels (FP64 links 144 B,
# momenta 144 B, spinors 48 B per site = 24 B per link of the site):
#   gauge force + kick   U in, P in and out; 84 staple matmuls + U V, 198 flop each
#   fermion force + kick U, X, Y in, P in and out; two outer products and matmuls
#   staples              U in, A1 and A2 out; 84 matmuls
#   link update          U in and out, P in; exp(iQ) and one matmul
#   stout level          U in, U' out; 12 plaquette-staple matmuls, exp, one matmul
#   action, plaquette    U in; 84 / 12 staple matmuls and the traces
HMC_KERNEL_COST = {  # (bytes, flops) per link
    "gauge_force": (3 * 144, 85 * 198),
    "fermion_force": (3 * 144 + 2 * 24, 4 * 198),
    "staples": (3 * 144, 84 * 198),
    "link_update": (3 * 144, 3 * 198 + 200),
    "stout_level": (2 * 144, 14 * 198 + 200),
    "action": (144, 85 * 198),
    "plaquette": (144, 13 * 198),
}
FP64_TFLOPS_NOMINAL = 40.0  # B200 datasheet FP64 (no measured FP64 peak on this pool)
HBM_SPEC_GBS = 8000.0  # B200 datasheet HBM3e bandwidth; fractions of it are reported beside the measured ones


def hmc_kernel_table(lat, hbm):
    """ms per launch and roofline fractions of the HMC kernels on the
    lattice's current fields."""
    nlinks = 4 * lat.V
    out = {}
    for name in lat.HMC_KERNELS:
        ms = lat.kernel_timing(name, nrep=10)
        row = {"ms": ms}
        if name in HMC_KERNEL_COST:
            b, f = HMC_KERNEL_COST[name]
            gbs = b * nlinks / (ms * 1e-3) / 1e9
            tfs = f * nlinks / (ms * 1e-3) / 1e12
            row.update({"GB/s": gbs, "frac_hbm": gbs / hbm, "TFLOP/s_fp64": tfs,
                        "frac_fp64_nominal": tfs / FP64_TFLOPS_NOMINAL,
                        "bound": "fp64" if f / b > FP64_TFLOPS_NOMINAL * 1e3 / hbm else "hbm"})
        out[name] = row
    return out


def run_c5(args):
    """24^4, beta 4.2, Hasenbusch pair m 0.02 / 0.2 on fermion links with 4
    stout levels (rho 0.125), leapfrog tau = 1 with N = 20 steps, --c5-traj
    trajectories from an eps = 0.3 start; the same chain with FP64 solves from
    the same start and seeds beside it; a step-size scan of dH; the HMC
    kernels' device times."""
    import staggered_fermions_hmc_b200 as sfh
    sfh.load_library()
    hbm, peak_kind = peaks()
    dims, N, ntraj = (24, 24, 24, 24), args.c5_steps, args.c5_traj

    def new_lattice():
        lat = sfh.Lattice(dims, 0.02, 4.2)
        if args.c5_schedule:
            lat.set_schedule(*[int(x) for x in args.c5_schedule.split(",")])
        lat.random_gauge(0.3, 5)
        lat.set_fermion_smearing(0.125, 4)
        lat.set_hasenbusch(0.2)
        return lat

    def chain(precision):
        lat = new_lattice()
        rows, poly = [], []
        for k in range(ntraj):
            inf = lat.hmc_trajectory(1.0 / N, N, seed=1000 + k, tol=TOL, precision=precision)
            g = lat.precompute_polyakov_grid()
            parts = [f - i for f, i in zip(inf["H_final"], inf["H_initial"])]
            rows.append({"dH": inf["dH"], "dH_kinetic": parts[0], "dH_gauge": parts[1], "dH_fermion": parts[2],
                         "accepted": inf["accepted"], "plaquette": inf["plaquette"], "seconds": inf["seconds"],
                         "cg_iters": inf["cg_iters"], "solves": inf["solves"]})
            poly.append(complex(g.mean()))
        return lat, rows, poly

    def summary(rows, poly):
        acc = [r["accepted"] for r in rows]
        return {"trajectories": len(rows), "acceptance": float(np.mean(acc)),
                "plaquette_mean": float(np.mean([r["plaquette"] for r in rows])),
                "plaquette_conventional_mean": float(np.mean([r["plaquette"] for r in rows])) / 6.0,
                "polyakov_mean": [float(np.mean([p.real for p in poly])), float(np.mean([p.imag for p in poly]))],
                "dH_mean": float(np.mean([r["dH"] for r in rows])),
                "dH_parts_mean": {k: float(np.mean([r[k] for r in rows]))
                                  for k in ("dH_kinetic", "dH_gauge", "dH_fermion")},
                "seconds_per_trajectory": float(np.mean([r["seconds"] for r in rows])),
                "trajectories_per_hour": 3600.0 / float(np.mean([r["seconds"] for r in rows])),
                "cg_iters_per_trajectory": float(np.mean([r["cg_iters"] for r in rows]))}

    lat, mixed, pmix = chain(args.c5_precision)
    kernels = hmc_kernel_table(lat, hbm)
    lat.close()
    lat, f64, p64 = chain("f64")
    lat.close()
    same = [a["accepted"] == b["accepted"] for a, b in zip(mixed, f64)]
    # step-size scan from the start configuration, same momenta and
    # pseudofermions: dH ~ eps^2 for a second-order integrator
    scan = {}
    for n in (N, 2 * N, 4 * N):
        lat = new_lattice()
        inf = lat.hmc_trajectory(1.0 / n, n, seed=1000, tol=TOL, precision=args.c5_precision)
        scan[str(n)] = {"eps": 1.0 / n, "dH": inf["dH"]}
        lat.close()
    ns = sorted(int(n) for n in scan)
    ratios = [scan[str(a)]["dH"] / scan[str(b)]["dH"] for a, b in zip(ns, ns[1:])]
    line = {
        "metric": "C5 full HMC on 24^4: trajectories/hour, acceptance, plaquette, Polyakov loop vs the FP64 path",
        "workload": "24^4, Symanzik beta 4.2, Hasenbusch pair m 0.02 / 0.2 on 4-level stout (rho 0.125) fermion "
                    f"links, leapfrog tau = 1 with {N} steps, {ntraj} trajectories from an eps = 0.3 start "
                    "(seed 5), no heatbath",
        "precision": {"mixed": args.c5_precision, "arithmetic": ARITHMETIC[args.c5_precision],
                      "schedule": args.c5_schedule or "default"},
        "mixed": summary(mixed, pmix), "fp64": summary(f64, p64),
        "accept_decisions_equal": float(np.mean(same)),
        "dH_mixed_minus_fp64_max": float(max(abs(a["dH"] - b["dH"]) for a, b in zip(mixed, f64))),
        "step_size_scan": {"dH": scan, "ratios_per_halving": ratios},
        "hmc_kernels_24^4": kernels, "peak_hbm": hbm, "peak_kind": peak_kind,
        "per_trajectory_mixed": mixed,
    }
    print(json.dumps(line), flush=True)


def run_profile_hmc(args):
    """A short launch of every HMC kernel on an L^4 lattice (eps = 0.3 links,
    random momenta, one launch each after the untimed ones of
    sfh_kernel_timing): the case for kernel profiling; prints one line."""
    import staggered_fermions_hmc_b200 as sfh
    sfh.load_library()
    L = args.profile_hmc
    lat = sfh.Lattice((L, L, L, L), 0.02, 4.2)
    lat.random_gauge(0.3, 5)
    lat.generate_conjugate_field_configuration(6)
    ms = {name: lat.kernel_timing(name, nrep=1) for name in lat.HMC_KERNELS}
    lat.close()
    print(json.dumps({"profile_hmc": True, "dims": [L] * 4, "ms": ms}), flush=True)


def run_profile_case(args, spec):
    import staggered_fermions_hmc_b200 as sfh
    sfh.load_library()
    B = build_batch(sfh, spec, args.precision, 0)
    B.set_schedule(args.rhs_block or 2, args.tiles, args.stage)
    for _ in range(args.warmup):
        B.solve(tol=TOL, max_iter=MAXIT)
    st = B.solve(tol=TOL, max_iter=args.maxit, check=False)
    print(json.dumps({"profile_case": True, "nsys": len(spec), "precision": args.precision,
                      "maxit": args.maxit, "status": st}), flush=True)
    B.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sfh", choices=["sfh", "reference"])
    ap.add_argument("--precision", default="f16", choices=["f32", "f16", "f32_18", "bf16"],
                    help="storage of the iterated vectors and links: f16 (half precision with a per-site "
                         "scale; packed-half products, f32 accumulation), bf16 (per-site scale; f32 products), "
                         "f32 (12-real links) or f32_18; reliable updates f64")
    ap.add_argument("--nsys", type=int, default=64)
    ap.add_argument("--ref-budget", type=float, default=6.0,
                    help="seconds of reference CPU solves per step of the reference arm")
    ap.add_argument("--cpu-budget", type=float, default=30.0,
                    help="seconds of reference CPU solves for the cpu_baseline of the GPU arm")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-serial", action="store_true",
                    help="end-to-end steps one after another only (no second batch alternating)")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--rhs-block", type=int, default=0,
                    help="RHS-block width of the hop kernels (0: time the schedules and keep the fastest)")
    ap.add_argument("--hop2-width", type=int, default=0,
                    help="with --rhs-block: the second hop's RHS-block width (the first hop takes --rhs-block)")
    ap.add_argument("--tiles", type=int, default=2, help="tiles per block with --rhs-block")
    ap.add_argument("--stage", type=int, default=0, help="stage links in shared memory with --rhs-block (0/1)")
    ap.add_argument("--profile-case", action="store_true",
                    help="build the batch, run --warmup solves, then one solve capped at --maxit "
                         "iterations (a short launch for kernel profiling); prints one line")
    ap.add_argument("--maxit", type=int, default=MAXIT)
    ap.add_argument("--profile-hmc", type=int, default=0, metavar="L",
                    help="launch every HMC kernel once on an L^4 lattice (a case for kernel profiling)")
    ap.add_argument("--workload", default="batch", choices=["batch", "c5"],
                    help="batch: the headline uneven-batch CG (default); c5: full HMC on 24^4, its own JSON line")
    ap.add_argument("--c5-traj", type=int, default=50)
    ap.add_argument("--c5-steps", type=int, default=20)
    ap.add_argument("--c5-precision", default="f32", choices=["f32", "f16", "bf16", "f32_18"])
    ap.add_argument("--c5-schedule", default="",
                    help="W,T,S: schedule of the trajectory's mixed-precision solves (sfh_set_schedule)")
    args = ap.parse_args()
    spec = batch_spec(nsys=args.nsys)
    if args.workload == "c5":
        run_c5(args)
        return
    if args.profile_hmc:
        run_profile_hmc(args)
        return
    if args.profile_case:
        run_profile_case(args, spec)
        return

    if args.impl == "reference":
        run_reference_arm(args, spec)
        return

    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import staggered_fermions_hmc_b200 as sfh
    sfh.load_library()
    total_rhs = sum(s["nrhs"] for s in spec)

    B = build_batch(sfh, spec, args.precision, local)
    if args.rhs_block:
        B.set_schedule(args.rhs_block, args.tiles, args.stage)
        if args.hop2_width:
            B.set_hop_widths(args.rhs_block, args.hop2_width)
    else:
        B.autotune()
    schedule = B.schedule()
    hop_widths = B.hop_widths()

    def solve():
        B.solve(tol=TOL, max_iter=MAXIT)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # warm-up (also establishes the iteration counts)
    for _ in range(args.warmup):
        solve()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    times = time_steps(torch, B.stream, solve, args.steps, 0)
    barrier()
    clk = clocks.stop()
    infos = [[B.info(k, j) for j in range(s["nrhs"])] for k, s in enumerate(spec)]
    launches_per_solve = B.kernel_launches()
    worst = max(B.true_residual(k, j) for k, s in enumerate(spec) for j in range(s["nrhs"]))
    ms = max_over_ranks(statistics.mean(times), world)
    value = replica_value(world, total_rhs, ms)

    hbm, peak_kind = peaks()
    alg_bytes = solve_bytes(spec, infos, args.precision)
    achieved = alg_bytes / (ms / 1000.0) / 1e9
    # per-kernel device time: one more solve with the kernels launched one by
    # one between CUDA events on the batch's stream (same kernels and results)
    per_kernel = B.solve_timed(tol=TOL, max_iter=MAXIT)
    kbytes = kernel_bytes(spec, infos, args.precision, ru_separate="cg_ru1" in per_kernel)
    if "cg_persistent" in per_kernel:  # the whole solve in one launch
        kbytes = {"cg_persistent": sum(kbytes.values())}
    ktot = sum(v[0] for v in per_kernel.values())
    kernels = {}
    for name, (kms, kn) in per_kernel.items():
        kernels[name] = {"launches": kn, "ms_total": kms, "share": kms / ktot if ktot else None,
                         "alg_bytes_total": kbytes[name],
                         "GB/s": kbytes[name] / (kms / 1000.0) / 1e9 if kms else None}
    top = max(kernels, key=lambda n: kernels[n]["ms_total"])
    top_n = max(1, kernels[top]["launches"])
    top_gbs = kernels[top]["GB/s"]
    ratio = HOP2_TRAFFIC_PER_ALG_BYTE.get(args.precision)
    top_traffic = ratio * kbytes[top] / top_n if (ratio and top == "cg_hop2") else None

    # FP64 batched CG on the same batch, same kernel family (the comparison)
    B64 = build_batch(sfh, spec, "f64", local)
    if args.rhs_block:
        B64.set_schedule(min(args.rhs_block, 2), args.tiles, False)
    else:
        B64.autotune()
    B64.solve(tol=TOL, max_iter=MAXIT)
    t64 = time_steps(torch, B64.stream, lambda: B64.solve(tol=TOL, max_iter=MAXIT), max(2, args.steps // 2), 1)
    ms64 = statistics.mean(t64)
    fp64_value = total_rhs / (ms64 / 1000.0)
    B64.close()

    # the other mixed precisions on the same batch, autotuned (secondary)
    other = {}
    if not args.no_extras:
        for prec in [p for p in ("f32", "f16", "bf16") if p != args.precision]:
            try:
                Bo = build_batch(sfh, spec, prec, local)
                Bo.autotune()
                Bo.solve(tol=TOL, max_iter=MAXIT)
                to = time_steps(torch, Bo.stream, lambda: Bo.solve(tol=TOL, max_iter=MAXIT),
                                max(2, args.steps // 2), 1)
                mso = statistics.mean(to)
                other[prec] = {"value": total_rhs / (mso / 1000.0), "unit": "solves/s", "ms_per_step": mso,
                               "schedule": list(Bo.schedule())}
                Bo.close()
            except Exception as e:  # a secondary measurement never hides the headline
                other[prec] = {"error": str(e)[:200]}

    # end to end through the public API: host (pinned) buffers in and out
    e2e = None
    if not args.no_e2e:
        host_U = []
        host_b = []
        for k, s in enumerate(spec):
            V = int(np.prod(s["dims"]))
            u = torch.empty(72 * V, dtype=torch.float64, pin_memory=True).numpy()
            u[:] = B.gauge(k)
            host_U.append(u)
            bs = []
            for j in range(s["nrhs"]):
                x = torch.empty(6 * V, dtype=torch.float64, pin_memory=True).numpy()
                x[:] = B.rhs(k, j)
                bs.append(x)
            host_b.append(bs)
        host_x = [[torch.empty(6 * int(np.prod(s["dims"])), dtype=torch.float64, pin_memory=True).numpy()
                   for _ in range(s["nrhs"])] for s in spec]
        h2d = sum(u.nbytes for u in host_U) + sum(x.nbytes for bs in host_b for x in bs)
        d2h = sum(x.nbytes for xs in host_x for x in xs)

        def upload(X):
            for k, s in enumerate(spec):
                X.set_gauge(k, host_U[k])
                for j in range(s["nrhs"]):
                    X.set_rhs(k, j, host_b[k][j])

        def download(X):
            for k, s in enumerate(spec):
                for j in range(s["nrhs"]):
                    X.solution(k, j, out=host_x[k][j])

        def e2e_step():
            upload(B)
            B.solve(tol=TOL, max_iter=MAXIT)
            download(B)

        te = time_steps(torch, B.stream, e2e_step, max(2, args.steps // 2), 1)
        mse_serial = max_over_ranks(statistics.mean(te), world)
        e2e = {"value": replica_value(world, total_rhs, mse_serial), "unit": "solves/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "mode": "serial"}
        if not args.e2e_serial:
            # two batches alternate: while one solves, a second host thread
            # downloads the other's solutions and uploads its next inputs
            B2 = sfh.Batch([(s["dims"], s["mass"], s["nrhs"]) for s in spec], precision=args.precision,
                           device=local)
            B2.set_schedule(*schedule)
            B2.set_hop_widths(*hop_widths)
            mse = max_over_ranks(e2e_pipelined(torch, (B, B2), upload, download, max(4, args.steps)), world)
            B2.close()
            e2e = {"value": replica_value(world, total_rhs, mse), "unit": "solves/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "mode": ("pipelined: two batches on two streams alternate; each step uploads its gauge fields "
                            "and sources from pinned host memory, solves and downloads every solution, its copies "
                            "overlapping the other batch's solve (CUDA events around all steps)"),
                   "serial": {"value": replica_value(world, total_rhs, mse_serial), "unit": "solves/s",
                              "ms_per_step": mse_serial}, "ms_per_step": mse}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # one pass over the batch's classes (bounded by --cpu-budget seconds)
        import tempfile
        with tempfile.TemporaryDirectory() as td:
            sampler = CpuSampler(spec, td)
            est = sampler.estimate(sampler.step(args.cpu_budget, max_classes=len(sampler.classes)))
        cpu = {"value": est["value"], "unit": "solves/s", "cores": os.cpu_count(), "kind": est["kind"],
               "sample": cpu_sample_desc(est), "classes_timed": est["classes_timed"],
               "batch_cpu_seconds_estimate": est["batch_cpu_seconds_estimate"]}

    c4_check = None
    if rank == 0 and not args.no_cpu:
        try:
            c4_check = c4_oracle_check(B, spec)
        except Exception as e:  # a secondary check never hides the headline
            c4_check = {"error": f"{type(e).__name__}: {e}"}

    extras = None
    if rank == 0 and not args.no_extras:
        B.close()
        try:
            extras = run_extras(sfh, hbm)
        except Exception as e:  # secondary measurements never hide the headline
            extras = {"error": f"{type(e).__name__}: {e}"}

    iters = [inf["iters"] for row in infos for inf in row]
    nru = [inf["reliable_updates"] for row in infos for inf in row]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE[args.precision],
        "data": "synthetic (seeded exp(i eps H) links, N(0,1) sources)",
        "config": workload_config(spec, world),
        "roofline": {"bound": "hbm", "achieved": top_gbs, "peak": hbm, "unit": "GB/s",
                     "frac": top_gbs / hbm, "frac_of_spec": top_gbs / HBM_SPEC_GBS, "spec_gbs": HBM_SPEC_GBS,
                     "traffic": top_traffic, "peak_kind": peak_kind,
                     "kernel": top, "alg_bytes_per_launch": kbytes[top] / top_n,
                     "ms_per_launch": kernels[top]["ms_total"] / top_n},
        "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": args.steps * launches_per_solve,
        "extras": extras,
        "kernels": kernels,
        "solve_roofline": {"achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                           "frac_of_spec": achieved / HBM_SPEC_GBS,
                           "alg_bytes_per_step": alg_bytes,
                           "what": "every iteration kernel, graph replay, per timed step"},
        "other_mixed_precisions": other,
        "solver_config": {"precision": args.precision, "arithmetic": ARITHMETIC[args.precision],
                          "schedule": {"rhs_block": schedule[0], "tiles_per_block": schedule[1],
                                       "staged_links": schedule[2], "hop_widths": list(hop_widths)}},
        "c4_oracle_check": c4_check,
        "solver": {"iters_mean": float(np.mean(iters)), "iters_max": int(max(iters)),
                   "reliable_updates_mean": float(np.mean(nru)), "worst_true_resid": worst},
        "fp64_batched": {"value": fp64_value, "unit": "solves/s", "ms_per_step": ms64,
                         "mixed_over_fp64": value / world / fp64_value},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    B.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
