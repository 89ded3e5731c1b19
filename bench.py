#!/usr/bin/env python
"""Benchmark of the direct J+K Fock build (libdgfock) on B200.

Workload (default): (H2O)32 water cluster, cc-pVDZ, 768 spherical basis
functions, closed-shell RHF density after a 12-iteration SCF.  A step is one
J+K build (IFCTYP 13, Schwarz 1e-12) of that density.  Both the all-FP64
drop-in and the mixed form (quartets with Q_AB Q_CD |D| < 1e-6 contracted in
FP32) are timed; the headline value is the mixed form when its energy error
against the FP64 build is within 1e-6 Eh, else the FP64 form.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) each rank evaluates 1/N of every class's quartet
queue and the partial Fock matrices are summed with an NCCL all-reduce inside
the timed step (strong scaling: the molecule is fixed).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "J+K build ms & ERI quartets/s, mixed vs FP64 at <=1e-6 Eh; HF gradient ms"
MIXED_CUTOFF = 1e-6
THRS = 1e-12
# dgf_class_time.kernel: 0 thread-per-quartet, 1 cooperative team, 2 warp teams, 4 warp-per-quartet
KERNEL_KIND = {0: "thread", 1: "team", 2: "team", 4: "warp", 6: "warp"}


def kernel_name(kind, la, lb, lc, ld, precision):
    """Template name of a profiled class kernel (kind as dgf_class_time.kernel;
    the warp kernel's last argument says whether its transforms run on the
    FP64 tensor cores)."""
    t = "double" if precision == 64 else "float"
    mma = {4: ",false", 6: ",true"}.get(kind, "")
    return f"jk_{KERNEL_KIND[kind]}_kernel<{la},{lb},{lc},{ld},{t}{mma}>"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dgfock", choices=["dgfock", "reference"])
    ap.add_argument("--workload", default="h2o32_ccpvdz")
    ap.add_argument("--scf-iters", type=int, default=12)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gradient", action="store_true")
    ap.add_argument("--no-extra-configs", action="store_true",
                    help="skip the (H2O)4, C20H42 and batch legs")
    ap.add_argument("--profile-run", action="store_true",
                    help="only run warmup+steps builds of a core-guess density (for ncu captures)")
    ap.add_argument("--mixed", action="store_true", help="with --profile-run: mixed form")
    ap.add_argument("--grad", action="store_true", help="with --profile-run: the two-electron gradient kernels")
    ap.add_argument("--pin", action="append", default=[],
                    help="with --profile-run: la,lb,lc,ld:variant pins one class's kernel (e.g. 2,1,2,1:-4 for the "
                         "warp kernel with tensor-core transforms); repeatable")
    return ap.parse_args()


def profile_run(args):
    """Minimal driver for profiler captures: W+K J+K builds, no SCF, no timing."""
    import torch

    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder

    mol, basis = molecules.config(args.workload)
    bs = build_basis(mol, basis)
    fb = FockBuilder(bs)
    for pin in args.pin:
        cls, variant = pin.split(":")
        fb.set_class_kernel(tuple(int(x) for x in cls.split(",")), int(variant))
    S, T, V = fb.oneint()
    Hm = torch.tensor(T + V, device="cuda")
    Sm = torch.tensor(S, device="cuda")
    s, U = torch.linalg.eigh(Sm)
    X = U / torch.sqrt(s)
    e, C = torch.linalg.eigh(X.T @ Hm @ X)
    C = X @ C
    nocc = mol.nelectrons() // 2
    D = (2.0 * C[:, :nocc] @ C[:, :nocc].T).contiguous()
    if args.grad:
        from dalton_b200.grad import grad2e_bilinear

        for _ in range(args.warmup + args.steps):
            grad2e_bilinear(fb, D, D, 1.0, THRS)
    else:
        for _ in range(args.warmup + args.steps):
            fb.herfck_device(D, ifctyp=13, thrs=THRS, mixed_cutoff=MIXED_CUTOFF if args.mixed else 0.0)
    torch.cuda.synchronize()
    print(json.dumps({"profile_run": args.workload, "builds": args.warmup + args.steps, "stats": fb.last_stats}))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline_sample(bs, dmat, target_s, threads=0, k=None):
    """Oracle (CPU restatement of Dalton's HERMIT J+K) on a fixed
    pseudo-random subset of the workload's significant quartets (hash-selected,
    so the class mix is the workload's), all host cores; the sampling
    fraction 2^-k is chosen from a short calibration run so that the sample
    takes target_s to 2 target_s seconds, unless k is given."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc

    orc.build()
    if threads:
        orc.set_threads(threads)
    cores = orc.threads()
    if k is None:
        k0 = 16
        n, sec, tot = orc.fock_hash_sample(bs, dmat, k0, THRS)
        est_full = tot * sec / max(n, 1)
        k = max(0, min(30, int(np.floor(np.log2(max(est_full / max(target_s, 1e-3), 1.0))))))
    n, sec, tot = orc.fock_hash_sample(bs, dmat, k, THRS)
    rate = n / sec
    return {"value": rate, "unit": "quartets/s", "cores": cores, "kind": "port",
            "sample": f"oracle J+K (C++ restatement of Dalton's HERMIT McMurchie-Davidson build and FCKCON "
                      f"digestion; Dalton itself needs gfortran, absent here) on a fixed hash-selected 2^-{k} "
                      f"subset of the workload's {tot} significant quartets ({n} quartets, all classes in the "
                      f"workload's proportions) in {sec:.2f} s on {cores} threads, i.e. a full build of "
                      f"{tot / rate:.0f} s; unlike HERMIT it evaluates general contractions (cc-pVDZ O 1s/2s, "
                      f"H 1s) as separate segmented shells, so it repeats their primitive integrals",
            "k": k, "est_full_build_s": tot / rate, "quartets": tot, "seconds": sec}


def workload_config(name, bs, mol, basis):
    """The `config` both arms print for a workload (same dict, same string)."""
    return {"workload": f"{name}: (H2O)32 cluster (seeded), {basis}, {bs.nbf} spherical basis functions, "
                        f"J+K IFCTYP 13, Schwarz {THRS}, RHF density after 12 SCF iterations"}


def bench_density(bs):
    """The timed density: RHF after 12 SCF iterations, read from the stored
    occupied orbitals (tests/golden/make_bench_density.py writes them)."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_bench_density

    return make_bench_density.load_density(bs)


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from dalton_b200.basis import build_basis
    from dalton_b200 import molecules

    mol, basis = molecules.config(args.workload)
    bs = build_basis(mol, basis)
    d = bench_density(bs)
    if d is None:
        print(json.dumps({"impl": "reference", "unavailable": "the stored benchmark density "
                          "(tests/golden/h2o32_ccpvdz_scf12_cocc.npz) is missing"}), flush=True)
        return
    per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
    vals = []
    info = None
    k = None  # sampling fraction fixed by the first step's calibration
    for step in range(args.warmup + args.steps):
        info = cpu_baseline_sample(bs, d, per_step, k=k)
        k = info["k"]
        if step >= args.warmup:
            vals.append(info["value"])
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.workload, bs, mol, basis),
            "cpu_sample_per_step_s": per_step,
            "step_values": vals,
            "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": info["cores"], "kind": "port",
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def scf_summary(ref, inc, mix, seconds):
    """Whole-SCF comparison (converged to |FDS - SDF| < 1e-6): full FP64 builds
    against incremental builds under the IFTHRS schedule, FP64 and mixed."""
    if ref is None:
        return None
    leg = lambda r: {"energy": r["energy"], "iterations": r["niter"], "fock_ms_total": r["fock_ms"],
                     "ifthrs": r["ifthrs"]}
    return {"fp64_full_builds": leg(ref), "fp64_incremental_screened": leg(inc),
            "mixed_incremental_screened": leg(mix),
            "energy_diff_mixed_vs_fp64_full_Eh": abs(mix["energy"] - ref["energy"]),
            "energy_diff_incremental_vs_fp64_full_Eh": abs(inc["energy"] - ref["energy"]),
            "fock_speedup_mixed_incremental_vs_fp64_full": ref["fock_ms"] / mix["fock_ms"],
            "fock_speedup_fp64_incremental_vs_fp64_full": ref["fock_ms"] / inc["fock_ms"],
            "note": "fock_ms_total: synchronised host time of the Fock builds summed over the SCF iterations",
            "seconds_all": seconds}


def ncu_traffic(kernel, workload):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of
    `kernel` on `workload`, as recorded from an ncu capture of the same
    command in profiles/traffic.txt (lines: kernel workload bytes), or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == kernel and f[1] == workload:
            return float(f[2])
    return None


def best_choices(tuning):
    """Fastest candidate per class and precision from an autotune report:
    {"la lb lc ld/precision": [variant (-1 = team kernel), ms, chunks]} and the
    mixed-form split decisions {"la lb lc ld/split": [0|1, ms FP64, ms split]}."""
    best = {}
    for r in tuning:
        if "split" in r:  # mixed-form decision: [split?, ms FP64 only, ms FP64+FP32]
            best[" ".join(str(x) for x in r["class"]) + "/split"] = [r["split"], round(r["ms_fp64"], 3),
                                                                     round(r["ms_split"], 3)]
            continue
        key = " ".join(str(x) for x in r["class"]) + f"/{r['precision']}"
        if key not in best or r["ms"] < best[key][1]:
            best[key] = [r["variant"], round(r["ms"], 3), r["chunks"]]
    return best


def run_batch(args):
    print(json.dumps(batch_leg(args.workload, args.steps, args.warmup)), flush=True)


def batch_leg(workload, steps, warmup):
    """Batched J+K of many molecules: one graph-replayed launch sequence vs a
    per-molecule launch loop (same contexts, same densities)."""
    import torch

    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.batch import BatchBuilder
    from dalton_b200.fock import FockBuilder

    mols, basis = molecules.config(workload)
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    fbs = [FockBuilder(build_basis(m, basis)) for m in mols]
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    ds = []
    for fb in fbs:  # a guess-like symmetric density (the Schwarz-screened quartet set does not depend on D)
        d = rng.normal(size=(fb.nbf, fb.nbf)) * 1e-2
        ds.append(torch.tensor(d + d.T + np.eye(fb.nbf) * 0.5, device=dev))
    outs = [torch.empty_like(d) for d in ds]
    # tune the kernel choices on the largest molecule and share them (loop and batch alike)
    big = max(range(len(fbs)), key=lambda k: fbs[k].nbf)
    t0 = time.perf_counter()
    fbs[big].autotune(ds[big], thrs=THRS, mixed_cutoff=MIXED_CUTOFF)
    tune_s = time.perf_counter() - t0
    for fb in fbs:
        fb.copy_tuning_from(fbs[big])
    bb = BatchBuilder(fbs)
    dp = bb.pack(ds)
    fp = torch.empty_like(dp)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def loop():
        for fb, d, o in zip(fbs, ds, outs):
            fb.herfck_device(d, fmat=o, stats=False)

    loop_ms = timed(loop)
    graph_ms = timed(lambda: bb.herfck_batch(dp, fp, use_graph=True, stats=False))
    nograph_ms = timed(lambda: bb.herfck_batch(dp, fp, use_graph=False, stats=False))
    bb.herfck_batch(dp, fp, use_graph=True)
    st = bb.last_stats
    loop()
    torch.cuda.synchronize(dev)
    err = max(float(torch.max(torch.abs(a - b))) for a, b in zip(bb.unpack(fp), outs))
    # mixed form of the batch (the split classes of the tuned context)
    fpm = torch.empty_like(dp)
    mixed_ms = timed(lambda: bb.herfck_batch(dp, fpm, use_graph=True, stats=False, mixed_cutoff=MIXED_CUTOFF))
    bb.herfck_batch(dp, fpm, use_graph=True, mixed_cutoff=MIXED_CUTOFF)
    stm = bb.last_stats
    err_m = max(float(torch.max(torch.abs(a - b))) for a, b in zip(bb.unpack(fpm), outs))
    de_m = max(abs(0.5 * float(torch.sum(d * (a - b)))) for d, a, b in zip(ds, bb.unpack(fpm), outs))
    for fb in fbs:
        fb.close()
    return {"workload": f"{workload}: {len(mols)} water clusters of 1-16 molecules (seeded), {basis}, "
                        f"{sum(fb.nbf for fb in fbs)} basis functions in all, J+K IFCTYP 13, Schwarz {THRS}",
            "quartets": st["quartets_total"], "steps": steps, "warmup": warmup,
            "per_molecule_loop_ms": loop_ms, "batched_graph_ms": graph_ms, "batched_no_graph_ms": nograph_ms,
            "speedup_graph_vs_loop": loop_ms / graph_ms, "quartets_per_s_graph": st["quartets_total"] / (graph_ms * 1e-3),
            "launches_batched": st["kernel_launches"], "max_abs_diff_vs_loop": err,
            "batched_graph_mixed_ms": mixed_ms, "mixed_fp32_quartets": stm["quartets_fp32"],
            "mixed_max_abs_dF_vs_fp64": err_m, "mixed_max_energy_error_Eh": de_m,
            "streams": 4, "context_setup_s": setup_s,
            "autotune_s_largest_molecule": tune_s,
            "data": "synthetic (seeded clusters, guess-like densities)"}


def stored_leg(fb, D, Fref, args, flush, dev, max_bytes=150 * 10**9):
    """Conventional form on the headline workload: store size, the time of
    the one integral pass that fills it, and FP64 Fock builds from it (L2
    flushed before every step), against the direct FP64 build Fref."""
    import torch

    from dalton_b200 import _lib

    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    try:
        nbytes = fb.store_integrals(THRS, max_bytes=max_bytes)
    except _lib.DgfError as e:
        return {"skipped": str(e)}
    torch.cuda.synchronize(dev)
    store_ms = (time.perf_counter() - t0) * 1e3
    stream = torch.cuda.current_stream(dev)
    out = torch.empty_like(D)
    for _ in range(args.warmup):
        fb.herfck_stored(D, fmat=out, thrs=THRS, stats=False)
    total = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fb.herfck_stored(D, fmat=out, thrs=THRS, stats=False)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    ms = total / args.steps
    err = float(torch.max(torch.abs(out - Fref)))
    fb.release_store()
    return {"form": "conventional: integral blocks stored in HBM once, Fock builds digest them",
            "store_bytes": nbytes, "store_fill_ms": store_ms, "fock_ms": ms,
            "store_read_gbs": nbytes / (ms * 1e-3) / 1e9, "max_abs_dF_vs_direct_fp64": err}


def core_guess_density(fb, mol):
    """Closed-shell density of the core-Hamiltonian orbitals (a guess-like density)."""
    import torch

    S, T, V = fb.oneint()
    Hm = torch.tensor(T + V, device="cuda")
    Sm = torch.tensor(S, device="cuda")
    s, U = torch.linalg.eigh(Sm)
    X = U / torch.sqrt(s)
    _, C = torch.linalg.eigh(X.T @ Hm @ X)
    C = X @ C
    nocc = mol.nelectrons() // 2
    return (2.0 * C[:, :nocc] @ C[:, :nocc].T).contiguous(), torch.tensor(T + V, device="cuda")


def timed_builds(fb, D, steps, warmup, flush, mixed_cutoff=0.0):
    """Mean device ms of one J+K build (CUDA events on the launching stream,
    L2 flushed before every step)."""
    import torch

    stream = torch.cuda.current_stream()
    out = torch.empty_like(D)
    for _ in range(warmup):
        fb.herfck_device(D, fmat=out, mixed_cutoff=mixed_cutoff, stats=False)
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fb.herfck_device(D, fmat=out, mixed_cutoff=mixed_cutoff, stats=False)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / steps, out


def top_kernel(fb, D, mixed_cutoff, fp64_peak, fp32_peak):
    """Per-launch profile of one build: the dominant class kernel with its
    model FLOP rate and fraction of the measured FMA peak."""
    from dalton_b200.perfmodel import class_flops

    fb.set_profiling(True)
    fb.herfck_device(D, mixed_cutoff=mixed_cutoff)
    prof = fb.profile()
    fb.set_profiling(False)
    agg = {}
    for r in prof:
        k = (r["la"], r["lb"], r["lc"], r["ld"], r["precision"], r["kernel"])
        a = agg.setdefault(k, {"ms": 0.0, "evaluated": 0, "prim_quartets": 0})
        a["ms"] += r["ms"]
        a["evaluated"] += r["evaluated"]
        a["prim_quartets"] += r["prim_quartets"]
    k, a = max(agg.items(), key=lambda kv: kv[1]["ms"])
    flops = class_flops(k[0], k[1], k[2], k[3], a["prim_quartets"], a["evaluated"])
    peak = fp64_peak if k[4] == 64 else fp32_peak
    ach = flops / (a["ms"] * 1e-3) / 1e12
    tot = sum(v["ms"] for v in agg.values())
    return {"kernel": kernel_name(k[5], k[0], k[1], k[2], k[3], k[4]), "ms": a["ms"], "quartets": a["evaluated"],
            "achieved_tflops": ach, "peak_tflops": peak, "frac": ach / peak, "share_of_build": a["ms"] / tot}


def small_leg(args, flush, fp64_peak, fp32_peak):
    """C1: (H2O)4 / cc-pVDZ, FP64 J+K at the converged RHF density and the
    full SCF energy; the oracle's full build of the same density on the host
    cores beside it."""
    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.scf import rhf

    mol, basis = molecules.config("h2o4_ccpvdz")
    bs = build_basis(mol, basis)
    res = rhf(bs, conv=1e-9, incremental=False, thrs=THRS)
    fb = res["builder"]
    D = res["dmat"].contiguous()
    ms, _ = timed_builds(fb, D, args.steps, args.warmup, flush)
    quartets = fb.ao_quartets(THRS)
    out = {"workload": f"h2o4_ccpvdz: (H2O)4 cluster (seeded), {basis}, {bs.nbf} spherical basis functions, "
                       f"J+K IFCTYP 13, Schwarz {THRS}, converged RHF density",
           "fp64_ms": ms, "quartets": quartets, "quartets_per_s": quartets / (ms * 1e-3),
           "scf_energy": res["energy"], "scf_iterations": res["niter"],
           "top_kernel": top_kernel(fb, D, 0.0, fp64_peak, fp32_peak)}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import orc

        orc.build()
        d = D.cpu().numpy()
        t0 = time.perf_counter()
        orc.fock(bs, d, 13, 1.0, THRS)
        out["oracle_full_build_s"] = time.perf_counter() - t0
        out["oracle_threads"] = orc.threads()
    fb.close()
    return out


def alkane_leg(args, flush, fp64_peak, fp32_peak):
    """C3: C20H42 / cc-pVTZ (f shells), per-class autotuned kernels, FP64 and
    mixed J+K at the core-Hamiltonian guess density."""
    import torch

    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder

    mol, basis = molecules.config("c20h42_ccpvtz")
    bs = build_basis(mol, basis)
    t0 = time.perf_counter()
    fb = FockBuilder(bs)
    setup_s = time.perf_counter() - t0
    D, H = core_guess_density(fb, mol)
    steps, warmup = max(2, min(args.steps, 3)), 1
    ms_untuned, Fdef = timed_builds(fb, D, steps, warmup, flush)
    Fdef = Fdef.clone()
    t0 = time.perf_counter()
    fb.autotune(D, thrs=THRS, mixed_cutoff=MIXED_CUTOFF)
    tune_s = time.perf_counter() - t0
    ms64, F64 = timed_builds(fb, D, steps, warmup, flush)
    F64 = F64.clone()
    tuned_dF = float(torch.max(torch.abs(F64 - Fdef)))  # the tuned kernels against the default ones
    msmx, Fmx = timed_builds(fb, D, steps, warmup, flush, MIXED_CUTOFF)
    dE = abs(0.5 * float(torch.sum(D * (Fmx - F64))))
    quartets = fb.ao_quartets(THRS)
    out = {"workload": f"c20h42_ccpvtz: all-trans C20H42 (seeded jitter), {basis}, {bs.nbf} spherical basis "
                       f"functions (up to f), J+K IFCTYP 13, Schwarz {THRS}, core-Hamiltonian guess density",
           "fp64_ms_default_kernels": ms_untuned, "autotune_s": tune_s, "context_s": setup_s,
           "fp64_ms": ms64, "mixed_ms": msmx, "speedup_mixed_vs_fp64": ms64 / msmx,
           "mixed_energy_error_Eh": dE, "mixed_max_abs_dF": float(torch.max(torch.abs(Fmx - F64))),
           "tuned_vs_default_kernels_max_abs_dF": tuned_dF,
           "quartets": quartets, "quartets_per_s_fp64": quartets / (ms64 * 1e-3),
           "quartets_per_s_mixed": quartets / (msmx * 1e-3),
           "top_kernel_fp64": top_kernel(fb, D, 0.0, fp64_peak, fp32_peak)}
    fb.close()
    return out


def main():
    args = parse()
    if args.workload.startswith("batch") and args.impl != "reference":
        run_batch(args)
        return
    if args.profile_run:
        profile_run(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    world, rank, local = dist_setup(args)
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (libdgfock has no CPU path)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.fock import FockBuilder
    from dalton_b200.perfmodel import class_flops
    from dalton_b200.scf import rhf
    from dalton_b200 import _lib

    mol, basis = molecules.config(args.workload)
    bs = build_basis(mol, basis)
    fb = FockBuilder(bs, device=local)
    shard = (rank, world)

    def build(D, mixed, out=None):
        F = fb.herfck_device(D, fmat=out, ifctyp=13, thrs=THRS, mixed_cutoff=MIXED_CUTOFF if mixed else 0.0,
                             shard=shard)
        if pg is not None:
            pg.all_reduce(F)
        return F

    # Density of the timed builds: RHF after 12 SCF iterations with FP64
    # builds, read from the stored orbitals that the CPU reference arm reads
    # too (recomputed when they are missing).
    D_np = bench_density(bs) if args.scf_iters == 12 else None
    density_source = "stored (tests/golden/h2o32_ccpvdz_scf12_cocc.npz)"
    if D_np is None:
        scf64 = rhf(bs, fb, maxiter=args.scf_iters, fixed_iterations=args.scf_iters, thrs=THRS)
        D = scf64["dmat"].contiguous()
        density_source = f"computed ({args.scf_iters} SCF iterations in this run)"
    else:
        D = torch.tensor(D_np, device=dev)
    S_np, T_np, V_np = fb.oneint()
    H = torch.tensor(T_np + V_np, device=dev)
    enuc = mol.nuclear_repulsion()
    # Per-class kernel choice on this density (FP64 and FP32 candidates, mixed split).
    Fdef = build(D, False).clone()  # default kernels, to check the tuned choice against
    t0 = time.perf_counter()
    tuning = fb.autotune(D, thrs=THRS, mixed_cutoff=MIXED_CUTOFF)
    tune_s = time.perf_counter() - t0
    # Whole SCF to |FDS - SDF| < 1e-6 three ways: full FP64 builds (the drop-in), and
    # incremental difference-density builds under Dalton's IFTHRS schedule, FP64 and mixed.
    t0 = time.perf_counter()
    scf_ref = scf_inc = scf_mix = None
    if world == 1:
        scf_ref = rhf(bs, fb, conv=1e-6, maxiter=60, thrs=THRS, incremental=False)
        scf_inc = rhf(bs, fb, conv=1e-6, maxiter=60, thrs=THRS, ifthrs_schedule=True)
        scf_mix = rhf(bs, fb, conv=1e-6, maxiter=60, thrs=THRS, mixed_cutoff=MIXED_CUTOFF, ifthrs_schedule=True)
    scf_s = time.perf_counter() - t0
    # Accuracy of the mixed build at the converged density.
    F64 = build(D, False).clone()
    Fmx = build(D, True).clone()
    e64 = float(0.5 * torch.sum(D * (2 * H + F64))) + enuc
    emx = float(0.5 * torch.sum(D * (2 * H + Fmx))) + enuc
    dE = abs(emx - e64)
    dF = float(torch.max(torch.abs(Fmx - F64)))
    tuned_dF = float(torch.max(torch.abs(F64 - Fdef)))
    mixed_ok = dE <= 1e-6

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    Fout = torch.empty_like(D)

    def timed(mixed, steps, warmup):
        for _ in range(warmup):
            build(D, mixed, Fout)
        torch.cuda.synchronize(dev)
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)
        total = 0.0
        launches = 0
        quartets = 0
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            build(D, mixed, Fout)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            launches += int(fb.last_stats.get("kernel_launches", 0))
            quartets += int(fb.last_stats.get("quartets_total", 0))
        torch.cuda.synchronize(dev)
        ms = total / steps
        if pg is not None:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            q = torch.tensor([quartets], device=dev, dtype=torch.float64)
            pg.all_reduce(q)
            ms, quartets = float(t), int(q)
        return ms, quartets / steps, launches

    clocks = ClockSampler(local)
    clocks.start()
    ms64, q64, l64 = timed(False, args.steps, args.warmup)
    msmx, qmx, lmx = timed(True, args.steps, args.warmup)
    clk = clocks.stop()
    headline_mixed = mixed_ok
    ms = msmx if headline_mixed else ms64
    # The unit is the workload's AO-basis contracted shell quartets (the same
    # count the CPU arms use); the kernels' own working-basis quartets (general
    # contractions resolved into primitives) are reported beside it.
    quartets = fb.ao_quartets(THRS)
    value = quartets / (ms * 1e-3)

    # End to end through the host-pointer C ABI (pinned host D in, host F out).
    Dh = torch.empty(D.shape, dtype=torch.float64, pin_memory=True)
    Dh.copy_(D)
    Fh = torch.empty(D.shape, dtype=torch.float64, pin_memory=True)
    d_np, f_np = Dh.numpy(), Fh.numpy()
    for _ in range(args.warmup):
        f_np[...] = fb.herfck(d_np, 13, thrs=THRS, mixed_cutoff=MIXED_CUTOFF if headline_mixed else 0.0, shard=shard)
    e2e_total = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        if pg is not None:
            pg.barrier()
        t0 = time.perf_counter()
        f_np[...] = fb.herfck(d_np, 13, thrs=THRS, mixed_cutoff=MIXED_CUTOFF if headline_mixed else 0.0,
                              shard=shard)
        if pg is not None:
            Fdev = torch.from_numpy(f_np).to(dev)
            pg.all_reduce(Fdev)
            Fh.copy_(Fdev)
        e2e_total += time.perf_counter() - t0
    e2e_ms = e2e_total / args.steps * 1e3
    if pg is not None:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t)
    nbytes = D.numel() * 8

    # Roofline of the dominant class kernel (profiled build, same stream).
    fb.set_profiling(True)
    build(D, headline_mixed, Fout)
    prof = fb.profile()
    fb.set_profiling(False)
    fp64_peak, fp32_peak = _lib.measure_fma_peak(local)
    by_time = sorted(prof, key=lambda r: -r["ms"])
    top = by_time[0]
    top_flops = class_flops(top["la"], top["lb"], top["lc"], top["ld"], top["prim_quartets"], top["evaluated"])
    achieved = top_flops / (top["ms"] * 1e-3) / 1e12
    peak = fp64_peak if top["precision"] == 64 else fp32_peak
    tot_ms = sum(r["ms"] for r in prof)
    kname = lambda r: kernel_name(r["kernel"], r["la"], r["lb"], r["lc"], r["ld"], r["precision"])
    roofline = {"bound": "fp64" if top["precision"] == 64 else "fp32",
                "kernel": kname(top),
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "measured FMA-loop peak on this GPU (MEASURED_PEAKS.json has no FP64 figure)",
                "traffic": ncu_traffic(kname(top), args.workload),
                "share_of_build": top["ms"] / tot_ms if tot_ms else None,
                "flops_model": "dalton_b200/perfmodel.py (per primitive and per contracted quartet)"}
    all_flops = sum(class_flops(r["la"], r["lb"], r["lc"], r["ld"], r["prim_quartets"], r["evaluated"]) for r in prof)
    build_tflops = all_flops / (tot_ms * 1e-3) / 1e12 if tot_ms else None

    # Conventional form (Dalton's SIRFCK2 over the AOTWOINT file, the file in
    # HBM): one evaluation of every quartet's integral block, then Fock
    # builds that read the blocks and digest them.
    stored_info = None
    if world == 1 and not args.no_extra_configs:
        stored_info = stored_leg(fb, D, Fdef, args, flush, dev)

    # HF nuclear gradient of (H2O)16 / cc-pVDZ (384 bf): backward kernel and full gradient.
    grad_info = None
    if not args.no_gradient and world == 1:
        from dalton_b200.grad import grad2e_bilinear, rhf_gradient

        gmol, gbas = molecules.config("h2o16_ccpvdz")
        gbs = build_basis(gmol, gbas)
        gfb = FockBuilder(gbs, device=local)
        gscf = rhf(gbs, gfb, conv=1e-8, thrs=THRS)
        Dg = gscf["dmat"].contiguous()
        for _ in range(2):
            grad2e_bilinear(gfb, Dg, Dg, 1.0, THRS)
        torch.cuda.synchronize(dev)
        gsteps = max(2, min(args.steps, 5))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(gsteps):
            grad2e_bilinear(gfb, Dg, Dg, 1.0, THRS)
        e1.record(stream)
        e1.synchronize()
        g2_ms = e0.elapsed_time(e1) / gsteps
        t0 = time.perf_counter()
        gfull = rhf_gradient(gfb, Dg, gscf["wmat"], thrs=THRS)
        torch.cuda.synchronize(dev)
        full_ms = (time.perf_counter() - t0) * 1e3
        # roofline of the backward kernels: one profiled call, per-class device times
        from dalton_b200.perfmodel import grad_class_flops

        gfb.set_profiling(True)
        grad2e_bilinear(gfb, Dg, Dg, 1.0, THRS)
        gprof = gfb.profile()
        gfb.set_profiling(False)
        gtop = max(gprof, key=lambda r: r["ms"])
        gflops = grad_class_flops(gtop["la"], gtop["lb"], gtop["lc"], gtop["ld"], gtop["prim_quartets"],
                                  gtop["evaluated"])
        gall = sum(grad_class_flops(r["la"], r["lb"], r["lc"], r["ld"], r["prim_quartets"], r["evaluated"])
                   for r in gprof)
        gms = sum(r["ms"] for r in gprof)
        g_roof = {"kernel": f"grad_thread_kernel<{gtop['la']},{gtop['lb']},{gtop['lc']},{gtop['ld']}>",
                  "ms": gtop["ms"], "share": gtop["ms"] / gms if gms else None,
                  "achieved_tflops": gflops / (gtop["ms"] * 1e-3) / 1e12,
                  "frac": gflops / (gtop["ms"] * 1e-3) / 1e12 / fp64_peak,
                  "all_kernels_tflops": gall / (gms * 1e-3) / 1e12 if gms else None,
                  "flops_model": "dalton_b200/perfmodel.py grad_class_flops"}
        grad_info = {"workload": f"h2o16_ccpvdz: (H2O)16 cluster, {gbas}, {gbs.nbf} basis functions, RHF "
                                 f"converged to 1e-8 ({gscf['niter']} iterations)",
                     "grad2e_ms": g2_ms, "full_gradient_ms": full_ms, "energy": gscf["energy"],
                     "roofline": g_roof,
                     "max_abs_gradient": float(np.abs(gfull).max()),
                     "translational_sum": float(np.abs(gfull.sum(0)).max())}
        gfb.close()

    legs = {}
    if world == 1 and not args.no_extra_configs:
        legs["c1"] = small_leg(args, flush, fp64_peak, fp32_peak)
        legs["c3"] = alkane_leg(args, flush, fp64_peak, fp32_peak)
        legs["c4"] = batch_leg("batch256_631gs", max(2, min(args.steps, 3)), 2)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(bs, D.cpu().numpy(), args.cpu_seconds)
        for key in ("seconds", "quartets", "k"):
            cpu.pop(key, None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64+f32 (mixed)" if headline_mixed else "f64", "data": "synthetic",
            "config": workload_config(args.workload, bs, mol, basis),
            "run": {"mixed_cutoff": MIXED_CUTOFF, "parallelism": f"cost-weighted quartet-queue shards x{world}",
                    "l2": "flushed (256 MB write) before every timed step", "density": density_source},
            "fp64": {"ms": ms64, "quartets_per_s": quartets / (ms64 * 1e-3), "quartets": quartets,
                     "working_basis_quartets": q64, "tuned_vs_default_kernels_max_abs_dF": tuned_dF},
            "mixed": {"ms": msmx, "quartets_per_s": quartets / (msmx * 1e-3), "quartets": quartets,
                      "working_basis_quartets": qmx,
                      "energy_error_Eh": dE, "max_abs_dF": dF, "speedup_vs_fp64": ms64 / msmx},
            "scf": scf_summary(scf_ref, scf_inc, scf_mix, scf_s),
            "stored": stored_info,
            "e2e": {"value": quartets / (e2e_ms * 1e-3), "unit": "quartets/s", "ms": e2e_ms,
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "roofline": roofline, "build_tflops_model": build_tflops,
            "autotune": {"seconds": tune_s, "candidates_timed": len(tuning), "best": best_choices(tuning)},
            "peaks_measured": {"fp64_tflops": fp64_peak, "fp32_tflops": fp32_peak},
            "gpu_launches": int((lmx if headline_mixed else l64)),
            "hf_gradient": grad_info,
            "c1": legs.get("c1"), "c3": legs.get("c3"), "c4": legs.get("c4"),
            "clocks": clk, "cpu_baseline": cpu,
            "profile_top": [{k: r[k] for k in ("la", "lb", "lc", "ld", "precision", "kernel", "evaluated",
                                               "prim_quartets", "ms")} for r in by_time[:8]],
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    fb.close()


if __name__ == "__main__":
    main()
