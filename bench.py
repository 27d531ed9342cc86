"""Benchmark of the polar Fourier correlation search on B200.

One step = one pass of the hot path over the workload's particle batch: Kaiser-
Bessel gridding of the particles' half-plane FTs to polar, their |CTF| matrices,
and the exhaustive search over all references x the shift grid x all in-plane
rotations (best (ref, rot, shift) per particle, the top-8 re-scored in FP32).

Workload (default): 128^3 Gaussian-blob volume, 500 references, 20,000 particles,
81 shifts (9x9 grid, 0.5 px), 360 rotations, shells 2..40, i.e.
500 x 20,000 x 81 x 360 = 2.916e11 correlation evaluations per step.  Inputs are
seeded synthetic data with those shapes and distributions (no dataset exists for
this path); the particle inputs (1.33 GB) exceed L2, so no flush is needed.

Arms:
  default           libpftcc_b200 through its C ABI (value: inputs resident in HBM;
                    e2e: host buffers, host<->device copies inside the timed region)
  --impl reference  the reference algorithm on the host cores (the FP32 FFT path of
                    polarft_corrcalc restated in C with OpenMP), bounded sample
Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

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
import __graft_entry__ as entry  # noqa: E402

METRIC = "ref x ptcl x rot corr evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp32", "exact"])
    ap.add_argument("--workload", default="config1", choices=["config1", "config0"])
    ap.add_argument("--nptcls", type=int, default=0, help="override the particle count (testing)")
    ap.add_argument("--nrefs", type=int, default=0, help="override the reference count (testing)")
    ap.add_argument("--ntop", type=int, default=8)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-arms", action="store_true", help="skip the FP32 / exact / reference-frame arms")
    ap.add_argument("--no-autotune", action="store_true", help="the automatic wave sizes, no autotuner")
    ap.add_argument("--wisdom", default=os.path.join(ROOT, "simple3.0_b200", "wisdom.txt"),
                    help="the autotuner's wisdom file (read, and appended when a shape is tuned)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--chunks", type=int, default=64, help="chunks of the batching report")
    ap.add_argument("--repeats", type=int, default=3, help="timed runs per worker count in the batching report")
    ap.add_argument("--report", default="", choices=["", "precision", "refine", "batching", "project", "euclid", "ingest", "hbm"],
                    help="precision: error of the FP32 and BF16-split paths against the FP64-accumulated direct "
                         "kernel over a particle sample; refine: the continuous shift/defocus refinement of every "
                         "particle at +-5 rotations around its pose against the exhaustive GPU shift grid (each "
                         "prints a report line instead of the bench line); batching: a queue of chunks of the "
                         "three batching geometries, U[50,300] references x U[500,5000] particles each; project: "
                         "the polar projector on the config-1 geometry; hbm: write-only, read-only and copy "
                         "rates of this GPU's memory (the denominators of the stage-1 / stage-2 fractions)")
    ap.add_argument("--grid-ptcls", type=int, default=200, help="particles whose problems also run the exhaustive grid")
    ap.add_argument("--report-ptcls", type=int, default=256, help="particles in the precision sample")
    return ap.parse_args()


def workload(pkg, args):
    w = getattr(pkg.synth, args.workload)()
    if args.nptcls:
        w.nptcls = args.nptcls
    if args.nrefs:
        w.nrefs = args.nrefs
    return w


def shifts_of(w):
    g = w.shift_grid if w.shift_grid else ((0.0, 0.0),)
    return np.asarray(g, np.float32)


def evals_per_step(w, nshifts):
    return float(w.nrefs) * w.nptcls * nshifts * w.nrots


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region"""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline
def cpu_sample(pkg, O, w, shifts, seconds: float):
    """time the oracle's OpenMP FFT-path search (reference loop structure) on a bounded
    sample: all host threads, nthreads particles x R references x all shifts"""
    nthreads = os.cpu_count() or 1
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    refs, R = pkg.synth.make_refs(w)
    refs = refs.numpy()
    npart = nthreads
    parts = pkg.synth.make_particles(w, R, count=npart)
    ptcls = np.stack([O.polarize(g, t, parts.cmat[i].numpy()) for i in range(npart)]).astype(np.complex64)
    ctfs = np.stack([O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]),
                                               float(parts.dfy[i]), float(parts.angast[i])))
                     for i in range(npart)]).astype(np.float32)
    # calibrate: one particle, one reference, all shifts, single thread
    t0 = time.perf_counter()
    O.cpu_search(g, refs[:1], ptcls[:1], ctfs[:1], shifts, nthreads=1)
    per_call = (time.perf_counter() - t0) / len(shifts)
    nr = int(max(1, min(w.nrefs, seconds / (per_call * len(shifts)))))
    t0 = time.perf_counter()
    _, _, _, _, used = O.cpu_search(g, refs[:nr], ptcls, ctfs, shifts, nthreads=nthreads)
    dt = time.perf_counter() - t0
    evals = float(nr) * npart * len(shifts) * w.nrots
    return {"value": evals / dt, "unit": "evals/s", "cores": int(used), "kind": "port",
            "sample": f"{npart} particles x {nr} refs x {len(shifts)} shifts x {w.nrots} rots "
                      f"({evals:.3g} evals, FP32 FFT path in the reference's loop structure, "
                      f"project-written mixed-radix FFT in place of FFTW, {dt:.1f} s)"}


def run_reference(args):
    pkg = entry.load_package()
    O = entry.load_oracle()
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(pkg, args)
    shifts = shifts_of(w)
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_sample(pkg, O, w, shifts, args.cpu_seconds / 2 if i < args.warmup else args.cpu_seconds)
        if i >= args.warmup:
            vals.append(r["value"])
            base = r
    v = float(statistics.median(vals))
    base["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": evals_per_step(w, len(shifts)) / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded Gaussian-blob volume, analytic sections, CTF, SNR 0.1)",
            "config": {"workload": w.name, "nrefs": w.nrefs, "nptcls": w.nptcls, "nshifts": len(shifts),
                       "nrots": w.nrots, "kfromto": [w.kfrom, w.kto], "box": w.box},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def algorithmic_costs(w, nshifts, kernel):
    """algorithmic work per step for each kernel class: (flops, bytes)"""
    P, N = w.pftsz, w.nrots
    Ks = w.K
    trip = float(w.nrefs) * nshifts * w.nptcls
    F = 8.0 * Ks * (P + 1)                      # complex MACs of the m-domain contraction per triple
    if kernel == "stage1":
        return 3.0 * F * trip, 0.0               # BF16 hi+lo: three issued products
    if kernel == "stage2":
        return 0.0, trip * P * 8.0               # stage 1's packed spectrum Z (P planes) read back once
    if kernel == "polarize":
        return 0.0, w.nptcls * (w.box * (w.box // 2 + 1) * 8.0 + Ks * P * 8.0)
    return 0.0, 0.0


# DRAM bytes (read + write) per (reference, shift, particle) triple measured by ncu on one
# launch of the same kernel (box 128 / nrots 360: 4096 rows x 512 columns, 3.0601 GB read +
# 0.0043 GB written = 1461.2 B per triple against 1440 B algorithmic); the stage-2 traffic grows
# with the triples processed, so the bench scales it to its own launches
DRAM_BYTES_PER_TRIPLE = {("stage2", 180): (3.060076e9 + 0.004345e9) / (4096 * 512)}


def run_ours(args):
    import torch
    import torch.distributed as dist

    pkg = entry.load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workload(pkg, args)
    # weak scaling: every rank searches its own particle batch (distinct seeds)
    w.seed_base += 100000 * rank
    shifts = shifts_of(w)
    ns = len(shifts)
    refs, R = pkg.synth.make_refs(w, device=dev)
    parts = pkg.synth.make_particles(w, R, device=dev)
    cmats = parts.cmat.contiguous()                               # resident in HBM
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True,
           ctf_frame="ptcl", device=local)
    stream = torch.cuda.current_stream(dev)
    pc.set_stream(stream.cuda_stream)
    r_host = refs.cpu().numpy()
    pc.set_refs(1, r_host, True)
    pc.set_refs(1, r_host, False)
    ctfp = pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca, dfx=parts.dfx,
                               dfy=parts.dfy, angast=parts.angast)
    best = torch.empty((w.nptcls, 4), dtype=torch.int32, device=dev)     # 16-byte pftcc_best records
    gathered = torch.empty((world, w.nptcls, 4), dtype=torch.int32, device=dev) if world > 1 else None

    def step():
        pc.polarize_ptcls_dev(0, w.nptcls, cmats.data_ptr())
        pc.create_polar_absctfmats(ctfp)
        pc.search_best_dev(shifts, args.precision, args.ntop if args.precision != "exact" else 0, best.data_ptr())
        if world > 1:
            dist.all_gather_into_tensor(gathered, best)

    # wave / tile sizes from the autotuner (untimed; a wisdom line for this shape skips the timing)
    tuning = None
    if args.precision in ("bf16x3", "fp32") and not args.no_autotune:
        step()      # the particles' polar FTs and CTFs for the tuning searches
        tuning = pc.autotune(shifts, args.precision, args.ntop, wisdom=args.wisdom)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    pc.prof_reset()
    pc.prof_enable(True)
    launches0 = pc.kernel_launches()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    launches = pc.kernel_launches() - launches0
    prof = pc.prof_read()
    pc.prof_enable(False)
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    evals = evals_per_step(w, ns)
    value = evals * world / (ms / 1e3)

    # dominant kernel and its roofline
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    tc_peak = peaks.get("bf16_tflops_sustained", 1400.0)
    peak_src = "measured" if peaks else "fallback"
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    shares = {k: round(v[0] / max(1e-9, sum(x[0] for x in prof.values())), 4) for k, v in prof.items() if v[1]}
    flops, byts = algorithmic_costs(w, ns, dom)
    per_launch_s = dom_ms / 1e3 / max(1, dom_n)
    n_launch_per_step = dom_n / args.steps
    if dom == "stage1" and args.precision == "bf16x3":
        ach = flops / n_launch_per_step / per_launch_s / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": tc_peak, "unit": "TFLOP/s", "frac": ach / tc_peak,
                "traffic": None, "kernel": "k_umma_stage1", "peak_source": f"{peak_src} bf16 sustained"}
    else:
        flops_b, byts_b = algorithmic_costs(w, ns, dom)
        ach = byts_b / n_launch_per_step / per_launch_s / 1e9 if byts_b else 0.0
        per_trip = DRAM_BYTES_PER_TRIPLE.get((dom, w.pftsz))
        trip_launch = float(w.nrefs) * ns * w.nptcls / n_launch_per_step
        roof = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                "traffic": per_trip * trip_launch if per_trip else None,
                "algorithmic_bytes": byts_b / n_launch_per_step,
                "kernel": f"k_{dom}", "peak_source": f"{peak_src} hbm copy"}
    roof["kernel_ms_per_step"] = {k: round(v[0] / args.steps, 3) for k, v in prof.items() if v[1]}
    roof["kernel_share"] = shares

    # e2e: host inputs through the public API, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        host_cm = torch.empty(cmats.shape, dtype=cmats.dtype, pin_memory=True)
        host_cm.copy_(cmats)
        host_np = host_cm.numpy()
        pc.set_stream(stream.cuda_stream)
        ntop_e = args.ntop if args.precision != "exact" else 0

        def max_ranks(x):
            if world > 1:
                t = torch.tensor([x], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                x = float(t.item())
            return x

        # serial: every step's calls with host buffers (polarize_ptcls copies the particles'
        # FTs, search_best returns the results to the host)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(args.steps):
            pc.polarize_ptcls(0, host_np)
            pc.create_polar_absctfmats(ctfp)
            out = pc.search_best(shifts, args.precision, ntop_e)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ems_serial = max_ranks(e0.elapsed_time(e1) / args.steps)
        # pipelined, as a streaming caller would run it: step k + 1's particle FTs cross from pinned
        # host memory into one of two device buffers on a copy stream while step k searches; each
        # step grids from its buffer (polarize_ptcls_dev), uploads its CTF records, searches
        # (search_best_dev) and reads its results back into pinned host memory
        copy_stream = torch.cuda.Stream(dev)
        dbuf = [torch.empty_like(cmats), torch.empty_like(cmats)]
        hbest = torch.empty((w.nptcls, 4), dtype=torch.int32, pin_memory=True)
        landed = [torch.cuda.Event(), torch.cuda.Event()]     # the copy into dbuf[i] has finished
        read = [torch.cuda.Event(), torch.cuda.Event()]       # the gridding from dbuf[i] has finished

        def issue_copy(i):
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(read[i])
                dbuf[i].copy_(host_cm, non_blocking=True)
                landed[i].record(copy_stream)

        torch.cuda.synchronize(dev)
        e0.record(stream)
        copy_stream.wait_stream(stream)       # the first copy starts inside the timed region
        issue_copy(0)
        for k in range(args.steps):
            i = k & 1
            if k + 1 < args.steps:
                issue_copy(1 - i)
            stream.wait_event(landed[i])
            pc.polarize_ptcls_dev(0, w.nptcls, dbuf[i].data_ptr())
            read[i].record(stream)
            pc.create_polar_absctfmats(ctfp)
            pc.search_best_dev(shifts, args.precision, ntop_e, best.data_ptr())
            hbest.copy_(best, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ems = max_ranks(e0.elapsed_time(e1) / args.steps)
        assert np.array_equal(hbest.numpy().view(np.int32).reshape(-1, 4), out.view(np.int32).reshape(-1, 4))
        e2e = {"value": evals * world / (ems / 1e3), "unit": "evals/s",
               "h2d_bytes_per_step": int(host_cm.numel() * host_cm.element_size() + w.nptcls * 36),
               "d2h_bytes_per_step": int(hbest.numel() * hbest.element_size()), "ms_per_step": ems,
               "mode": "pipelined: each step's particle FTs copied from pinned host memory on a copy stream "
                       "while the previous step searches (two device buffers), CTF records uploaded and "
                       "results read back every step; public calls polarize_ptcls_dev, "
                       "create_polar_absctfmats, search_best_dev",
               "serial": {"value": evals * world / (ems_serial / 1e3), "ms_per_step": ems_serial,
                          "mode": "polarize_ptcls (host FTs) + create_polar_absctfmats + search_best (host "
                                  "results), one after another"}}

    # the other arms on the same workload, after the timed region: the plain FP32 m-domain
    # search (the BF16 split's comparison), the exact drop-in kernel on a bounded sample, and the
    # search in the reference CTF frame (the drop-in semantics: top 8 re-scored by the exact
    # kernel).  Device time over steps with CUDA events on the launching stream.
    arms = None
    if not args.no_arms and args.precision == "bf16x3":
        arms = other_arms(pkg, pc, w, shifts, parts, r_host, ctfp, cmats, best, stream, dev, args, world)
    if arms is not None:
        arms["bf16x3_over_fp32"] = value / arms["fp32_mdomain"]["value"]
    if args.precision == "bf16x3":
        # the contraction's tensor work (3 issued BF16 products per complex MAC) over the whole step
        fl3, _ = algorithmic_costs(w, ns, "stage1")
        st1 = prof.get("stage1", (0.0, 0))
        roof["tensor"] = {"kernel": "k_umma_stage1", "issued_flops_per_step": fl3,
                          "achieved_stage1": fl3 / (st1[0] / args.steps / 1e3) / 1e12 if st1[0] else None,
                          "achieved_whole_step": fl3 / (ms / 1e3) / 1e12, "peak": tc_peak, "unit": "TFLOP/s",
                          "peak_source": f"{peak_src} bf16 sustained"}
        if st1[0]:
            roof["tensor"]["frac_stage1"] = roof["tensor"]["achieved_stage1"] / tc_peak
        roof["tensor"]["frac_whole_step"] = roof["tensor"]["achieved_whole_step"] / tc_peak

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_sample(pkg, entry.load_oracle(), w, shifts, args.cpu_seconds)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": {"bf16x3": "bf16x3 (bf16 hi+lo products, fp32 accumulate)",
                                               "fp32": "fp32", "exact": "fp32"}[args.precision],
                "data": "synthetic (seeded Gaussian-blob volume, analytic sections, CTF, SNR 0.1)",
                "config": {"workload": w.name, "nrefs": w.nrefs, "nptcls": w.nptcls, "nshifts": ns,
                           "nrots": w.nrots, "kfromto": [w.kfrom, w.kto], "box": w.box,
                           "precision": args.precision, "ntop_rescore": args.ntop, "ctf_frame": "ptcl",
                           "l2": "inputs larger than L2 (1.33 GB particle FTs)", "parallelism": f"dp{world}",
                           "tuning": tuning},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clocks}
        if arms is not None:
            line["value_fp32"] = arms["fp32_mdomain"]["value"]
            line["bf16_over_fp32"] = arms["bf16x3_over_fp32"]
            line["arms"] = arms
        print(json.dumps(line), flush=True)
    pc.kill()
    if world > 1:
        dist.destroy_process_group()


def other_arms(pkg, pc, w, shifts, parts, r_host, ctfp, cmats, best, stream, dev, args, world):
    """rates of the other search paths on the same workload (evals/s, device time)"""
    import torch
    ns = len(shifts)

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    def handle(nrefs, nptcls, frame, cp):
        h = pkg.polarft_corrcalc()
        h.new(nrefs, (1, nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame=frame,
              device=dev.index)
        h.set_stream(stream.cuda_stream)
        h.set_refs(1, r_host[:nrefs], True)
        h.set_refs(1, r_host[:nrefs], False)
        h.polarize_ptcls_dev(0, nptcls, cmats.data_ptr())
        h.create_polar_absctfmats(cp)
        return h

    out = {}
    k = max(1, min(args.steps, 3))
    # plain FP32: the m-domain contraction on the CUDA cores, FP32 end to end, with its own tuning
    bf16_tuning = pc.get_tuning()
    t32 = None if args.no_autotune else pc.autotune(shifts, "fp32", args.ntop, wisdom=args.wisdom)
    ms32 = timed(lambda: pc.search_best_dev(shifts, "fp32", args.ntop, best.data_ptr()), k, 1)
    pc.set_tuning(bf16_tuning["w_rows"], bf16_tuning["w_cols"], bf16_tuning["s1_stages"])
    out["fp32_mdomain"] = {"value": evals_per_step(w, ns) * world / (ms32 / 1e3), "ms_per_step": ms32, "steps": k,
                           "tuning": t32,
                           "what": "search_best PFTCC_PREC_FP32 (particle frame, the same top-8 re-score), "
                                   "inputs resident"}
    # the exact drop-in kernel (direct sums, FP32 products, FP64 accumulation) on a bounded
    # sample: 2 particles per SM x 50 references x every shift x every rotation
    ne, nre = min(w.nptcls, 296), min(w.nrefs, 50)
    pe = handle(nre, ne, "ref", pkg.ctfparams_array(ne, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                    dfx=parts.dfx[:ne], dfy=parts.dfy[:ne], angast=parts.angast[:ne]))
    bdev = torch.empty((ne, 4), dtype=torch.int32, device=dev)
    msx = timed(lambda: pe.search_best_dev(shifts, "exact", 0, bdev.data_ptr()), 1, 1)
    out["exact_ref_frame"] = {"value": float(ne) * nre * ns * w.nrots * world / (msx / 1e3), "ms_per_step": msx,
                              "sample": f"{ne} particles x {nre} refs x {ns} shifts x {w.nrots} rots",
                              "what": "search_best PFTCC_PREC_EXACT (the drop-in gencorrs kernel), inputs resident"}
    pe.kill()
    # the m-domain search in the reference frame: particle-frame screening with BF16 products,
    # the top 8 re-scored by the exact kernel in the reference frame
    pr = handle(w.nrefs, w.nptcls, "ref", ctfp)
    kr = max(1, min(args.steps, 2))
    msr = timed(lambda: pr.search_best_dev(shifts, "bf16x3", 8, best.data_ptr()), kr, 1)
    out["bf16x3_ref_frame"] = {"value": evals_per_step(w, ns) * world / (msr / 1e3), "ms_per_step": msr, "steps": kr,
                               "what": "search_best PFTCC_PREC_BF16X3 on a reference-frame handle: top 8 re-scored "
                                       "by the exact kernel in the reference frame, inputs resident"}
    pr.kill()
    return out


# ------------------------------------------------------------------ precision report
def run_precision_report(args):
    """Every correlation of a particle sample of the workload (all references x all
    shifts x all rotations) through the FP32 and BF16-split m-domain paths, against
    the direct kernel with FP64 accumulation (the same objective, particle-frame CTF):
    max / mean |dcc|, max / mean relative error with |cc| floored at 1e-3, the
    agreement of the best (ref, shift, rot) per particle, and of the BF16-split search
    with its FP32 re-score of the top 8.  A disagreement is excused where the exact
    scores of the two poses differ by less than the path's tolerance."""
    pkg = entry.load_package()
    w = workload(pkg, args)
    shifts = shifts_of(w)
    ns = len(shifts)
    refs, R = pkg.synth.make_refs(w)
    r_host = refs.numpy()
    chunk = 16
    nsub = min(args.report_ptcls, w.nptcls)
    tol = {"fp32": 1e-5, "bf16x3": 1e-4}
    acc = {p: {"max_abs": 0.0, "sum_abs": 0.0, "max_rel": 0.0, "sum_rel": 0.0, "agree": 0, "excused": 0}
           for p in ("fp32", "bf16x3")}
    srch = {"agree": 0, "excused": 0}
    count = 0
    t0 = time.time()
    for first in range(0, nsub, chunk):
        n = min(chunk, nsub - first)
        parts = pkg.synth.make_particles(w, R, first=first, count=n)
        pc = pkg.polarft_corrcalc()
        pc.new(w.nrefs, (1, n), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ptcl")
        pc.set_refs(1, r_host, True)
        pc.set_refs(1, r_host, False)
        pc.polarize_ptcls(0, parts.cmat.numpy())
        pc.create_polar_absctfmats(pkg.ctfparams_array(n, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                       dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
        ex = pc.corr_all_prec(shifts, "exact").reshape(n, -1).astype(np.float64)
        best_ex = ex.argmax(1)
        count += ex.size
        for prec in ("fp32", "bf16x3"):
            cc = pc.corr_all_prec(shifts, prec).reshape(n, -1).astype(np.float64)
            d = np.abs(cc - ex)
            rel = d / np.maximum(np.abs(ex), 1e-3)
            a = acc[prec]
            a["max_abs"] = max(a["max_abs"], float(d.max()))
            a["sum_abs"] += float(d.sum())
            a["max_rel"] = max(a["max_rel"], float(rel.max()))
            a["sum_rel"] += float(rel.sum())
            bi = cc.argmax(1)
            same = bi == best_ex
            a["agree"] += int(same.sum())
            gap = ex[np.arange(n), best_ex] - ex[np.arange(n), bi]
            a["excused"] += int(((~same) & (gap < tol[prec])).sum())
        sb = pc.search_best(shifts, "bf16x3", ntop=8)
        pose = (sb["iref"].astype(np.int64) - 1) * ns * w.nrots + sb["ishift"].astype(np.int64) * w.nrots + \
            sb["irot"].astype(np.int64) - 1
        same = pose == best_ex
        srch["agree"] += int(same.sum())
        gap = ex[np.arange(n), best_ex] - ex[np.arange(n), pose]
        srch["excused"] += int(((~same) & (gap < tol["bf16x3"])).sum())
        pc.kill()
    out = {"report": "precision", "workload": w.name, "oracle": "direct kernel, FP64 accumulation, particle-frame CTF",
           "sample": f"{nsub} particles x {w.nrefs} refs x {ns} shifts x {w.nrots} rots", "correlations": count,
           "seconds": round(time.time() - t0, 1)}
    for prec, a in acc.items():
        out[prec] = {"max_abs_dcc": a["max_abs"], "mean_abs_dcc": a["sum_abs"] / count,
                     "max_rel_err_floor1e-3": a["max_rel"], "mean_rel_err_floor1e-3": a["sum_rel"] / count,
                     "best_pose_agreement": a["agree"] / nsub,
                     "best_pose_agreement_with_excused": (a["agree"] + a["excused"]) / nsub, "tolerance": tol[prec]}
    out["search_bf16x3_fp32_rescore_top8"] = {"best_pose_agreement": srch["agree"] / nsub,
                                              "best_pose_agreement_with_excused":
                                                  (srch["agree"] + srch["excused"]) / nsub}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ refinement report
def refine_problems(pkg, w, seed=3):
    """Continuous-refinement problems of the workload: every particle against its own
    reference at the 11 in-plane indices around its pose, the shift started U[-2,2] px
    away from the one that undoes the particle's shift, the CTF handed to the search
    off by U[-0.1,0.1] microns of defocus.  Returns (handle, iref, iptcl, irot, x0)."""
    import math
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R, device="cuda")
    rng = np.random.default_rng(seed)
    delta = rng.uniform(-0.1, 0.1, w.nptcls)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True)
    r_host = refs.numpy()
    pc.set_refs(1, r_host, True)
    pc.set_refs(1, r_host, False)
    pc.polarize_ptcls_dev(0, w.nptcls, parts.cmat.contiguous().data_ptr())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx + delta, dfy=parts.dfy + delta,
                                                   angast=parts.angast))
    iref, iptcl, irot, x0, truth = [], [], [], [], []
    for i in range(w.nptcls):
        psi = math.radians(parts.psi[i])
        tx, ty = parts.shift[i]
        r0 = int(round(parts.psi[i] * w.nrots / 360.0))
        sh = (-(math.cos(psi) * tx + math.sin(psi) * ty), -(-math.sin(psi) * tx + math.cos(psi) * ty))
        start = (sh[0] + rng.uniform(-2, 2), sh[1] + rng.uniform(-2, 2))
        for d in range(-5, 6):
            iref.append(parts.ref[i] + 1)
            iptcl.append(i + 1)
            irot.append((r0 + d) % w.nrots + 1)
            x0.append((start[0], start[1], 0.0))
            truth.append((sh[0], sh[1], -delta[i]))
    return (pc, np.array(iref), np.array(iptcl), np.array(irot), np.array(x0, np.float64),
            np.array(truth, np.float64))


def run_refine_report(args):
    """Config-3 style measurement: all problems refined in shift and defocus together; on
    the problems of the first --grid-ptcls particles, the shift-only refinement against the
    exhaustive shift grid (0.1 px over the same +-2 px box, defocus held) evaluated by the
    same adjoint kernel, both timed as wall time of the library calls."""
    pkg = entry.load_package()
    w = workload(pkg, args)
    pc, iref, iptcl, irot, x0, truth = refine_problems(pkg, w)
    n = iref.size
    half = np.array([2.0, 2.0, 0.2])
    lb, ub = x0 - half, x0 + half
    t0 = time.perf_counter()
    x, f, nev, nit, conv = pc.refine_batch(iref, iptcl, irot, x0, lb, ub, maxits=100)
    t_all = time.perf_counter() - t0
    centre = np.arange(n) % 11 == 5                    # the problems at the particle's own pose index
    dsh = np.hypot(*(x[centre, :2] - truth[centre, :2]).T)
    ns = min(args.grid_ptcls, w.nptcls) * 11
    lb0, ub0 = lb[:ns].copy(), ub[:ns].copy()
    lb0[:, 2] = ub0[:, 2] = 0.0
    t0 = time.perf_counter()
    xs, fs, nevs, _, _ = pc.refine_batch(iref[:ns], iptcl[:ns], irot[:ns], x0[:ns], lb0, ub0, maxits=100)
    t_ref = time.perf_counter() - t0
    g = np.arange(-20, 21) * 0.1
    GX, GY = (a.ravel() for a in np.meshgrid(g, g, indexing="ij"))
    npts = GX.size
    best = np.full(ns, -np.inf)
    chunk = max(1, 250000 // npts)
    t0 = time.perf_counter()
    for p0 in range(0, ns, chunk):
        p1 = min(ns, p0 + chunk)
        k = p1 - p0
        fg, _ = pc.grad_batch(np.repeat(iref[p0:p1], npts), np.repeat(iptcl[p0:p1], npts), np.repeat(irot[p0:p1], npts),
                              (x0[p0:p1, 0][:, None] + GX[None, :]).ravel(), (x0[p0:p1, 1][:, None] + GY[None, :]).ravel(),
                              np.zeros(k * npts))
        best[p0:p1] = fg.reshape(k, npts).max(1)
    t_grid = time.perf_counter() - t0
    out = {"report": "refine", "workload": w.name,
           "problems": int(n), "problem": "one particle vs its own reference at one of 11 in-plane indices around "
                                          "its pose; start U[-2,2] px off, CTF defocus off by U[-0.1,0.1] um",
           "all_shift_defocus": {"seconds": round(t_all, 3), "problems_per_s": n / t_all,
                                 "median_evaluations": float(np.median(nev)), "converged": float(conv.mean()),
                                 "median_shift_error_px_at_pose": float(np.median(dsh))},
           "sample": {"problems": int(ns), "grid_points_per_problem": int(npts), "grid_seconds": round(t_grid, 3),
                      "refine_shift_seconds": round(t_ref, 3), "refine_over_grid_time": t_ref / t_grid,
                      "median_refine_evaluations": float(np.median(nevs)),
                      "reaching_grid_best_within_1e-4": float(np.mean(fs >= best - 1e-4))}}
    print(json.dumps(out), flush=True)
    pc.kill()


# ------------------------------------------------------------------ batching report
def run_batching_report(args):
    """The batching workload: --chunks chunks, each of a geometry drawn from box 64 /
    nrots 128 / k 2..20, box 128 / nrots 360 / k 2..40 and box 200 / nrots 600 / k 2..60
    with U[50,300] references and U[500,5000] particles, searched (BF16 split, FP32 re-score
    of the top 8) through the chunk queue with one and with two worker streams; inputs are
    resident on the device; every chunk's result must be the same in both runs.  One untimed
    pass over the queue comes first, so both timed runs start with the memory pool grown; each
    worker count is timed --repeats times (wall clock, host work included) and the best kept."""
    import torch
    pkg = entry.load_package()
    b = pkg.batching
    rng = np.random.default_rng(2024)
    spec = [(str(rng.choice(list("ABC"))), int(rng.integers(50, 301)), int(rng.integers(500, 5001)))
            for _ in range(args.chunks)]
    cache = {}
    t0 = time.perf_counter()
    chunks = [b.synthetic_chunk(g, nr, npt, seed=i, ref_cache=cache) for i, (g, nr, npt) in enumerate(spec)]
    t_gen = time.perf_counter() - t0
    evals = sum(ch.evals() for ch in chunks)
    b.SearchQueue(workers=1).run(chunks)              # warm-up: the whole queue once (pool grown, kernels loaded)
    out = {"report": "batching", "chunks": len(chunks),
           "geometry_chunks": {g: sum(1 for s_ in spec if s_[0] == g) for g in "ABC"},
           "particles": sum(s_[2] for s_ in spec), "evals": evals, "data_seconds": round(t_gen, 1)}
    results = {}
    for workers in (1, 2, 4):
        times = []
        for _ in range(args.repeats):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            results[workers] = b.SearchQueue(workers=workers).run(chunks)
            times.append(time.perf_counter() - t0)
        t = min(times)
        out[f"workers_{workers}"] = {"seconds": round(t, 3), "seconds_all": [round(x, 3) for x in times],
                                     "evals_per_s": evals / t, "chunks_per_s": len(chunks) / t}
    out["identical_results"] = all(np.array_equal(a.view(np.int32).reshape(len(a), -1), c.view(np.int32).reshape(len(c), -1))
                                   for w_ in (2, 4) for a, c in zip(results[1], results[w_]))
    # the grouped search: one handle and one pftcc_search_groups call per geometry (one persistent
    # stage-1 launch and one stage-2 launch over all its chunks), after an untimed pass
    b.search_grouped(chunks)
    times = []
    for _ in range(args.repeats):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        grouped = b.search_grouped(chunks)
        times.append(time.perf_counter() - t0)
    t = min(times)
    out["grouped"] = {"seconds": round(t, 3), "seconds_all": [round(x, 3) for x in times], "evals_per_s": evals / t,
                      "chunks_per_s": len(chunks) / t,
                      "identical_to_queue": all(np.array_equal(a.view(np.int32).reshape(len(a), -1),
                                                               c.view(np.int32).reshape(len(c), -1))
                                                for a, c in zip(results[1], grouped))}
    # the grouped searches captured as CUDA graphs (one per geometry, after an uncaptured call) and
    # replayed: the queue's whole search as three graph launches, with the handles' references and
    # particles already resident; device time by CUDA events, results against the queue's
    keys = {}
    for i, ch in enumerate(chunks):
        keys.setdefault((ch.box, ch.nrots, ch.kfrom, ch.kto), []).append(i)
    side = torch.cuda.Stream()
    graphs, handles, outs = [], [], []
    try:
        for k, idx in keys.items():
            pc, groups = b.grouped_handle([chunks[i] for i in idx], stream=side.cuda_stream)
            handles.append((pc, groups, idx))
            o = torch.zeros((sum(chunks[i].nptcls for i in idx), 4), dtype=torch.int32, device="cuda")
            with torch.cuda.stream(side):
                pc.search_groups_dev(groups, None, "bf16x3", 8, o.data_ptr())
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                pc.search_groups_dev(groups, None, "bf16x3", 8, o.data_ptr())
            graphs.append(g)
            outs.append(o)
        torch.cuda.synchronize()
        times = []
        for _ in range(max(3, args.repeats)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(side):
                e0.record(side)
                for g in graphs:
                    g.replay()
                e1.record(side)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        same = True
        for (pc, groups, idx), o in zip(handles, outs):
            pc.search_check()
            res = o.cpu().numpy().view(np.int32).reshape(-1, 4)
            for (r0, _, s0, n), i in zip(groups, idx):
                x = res[s0 - 1:s0 - 1 + n].copy()
                x[:, 0] -= (r0 - 1) * (x[:, 0] > 0)
                same &= np.array_equal(x, results[1][i].view(np.int32).reshape(-1, 4))
        t = min(times)
        out["graph_replay"] = {"seconds": round(t, 4), "seconds_all": [round(x, 4) for x in times],
                               "evals_per_s": evals / t, "graphs": len(graphs), "identical_to_queue": bool(same),
                               "what": "the grouped searches of the three geometries captured as CUDA graphs and "
                                       "replayed; handles, references and particles resident (search only)"}
    finally:
        graphs.clear()
        torch.cuda.synchronize()
        for pc, _, _ in handles:
            pc.kill()
    print(json.dumps(out), flush=True)


def run_project_report(args):
    """The polar projector (pftcc_set_volume_ft = expand_cmat, pftcc_fproject_polar =
    fproject_polar) on the config-1 geometry: a seeded box-128 volume FT, 500 orientations
    (K = 39 shells x 180 rotations each); GPU wall time per call (synchronous, the host's
    rotation matrices and uploads included), parity of three references against the
    oracle, and the oracle's single-thread time per reference beside it."""
    pkg = entry.load_package()
    O = entry.load_oracle()
    w = pkg.synth.config1()
    box = w.box
    rng = np.random.default_rng(5)
    shape = (box, box, box // 2 + 1)
    vol = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    n = w.nrefs
    euls = np.stack([rng.uniform(0, 360, n), rng.uniform(0, 180, n), rng.uniform(0, 360, n)], 1).astype(np.float32)
    pc = pkg.polarft_corrcalc()
    pc.new(n, (1, 1), box=box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    pc.set_volume_ft(vol)
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        pc.set_volume_ft(vol)
    t_expand = (time.perf_counter() - t0) / reps
    for _ in range(3):
        pc.fproject_polar(1, euls)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        pc.fproject_polar(1, euls)
    t_proj = (time.perf_counter() - t0) / reps
    g = O.geom(w.nrots, w.kfrom, w.kto, box)
    t = O.tables(g)
    ex = O.expand_cmat3d(vol, box)
    worst = 0.0
    t0 = time.perf_counter()
    for r in range(3):
        want = O.fproject_polar(g, t, ex, box, euls[r].astype(np.float64))
        got = pc.get_ref_pft(r + 1, True)
        worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
    t_cpu = (time.perf_counter() - t0) / 3
    # the orientation-gradient inputs: sections and their three angle derivatives
    e64 = euls.astype(np.float64)
    pc.fdf_project_polar(1, e64)
    reps = 10
    t0 = time.perf_counter()
    for _ in range(reps):
        pc.fdf_project_polar(1, e64)
    t_fdf = (time.perf_counter() - t0) / reps
    want, dwant = O.fdf_project_polar(g, t, ex, box, e64[0])
    fdf_err = max(float(np.max(np.abs(pc.get_ref_pft(1, True) - want)) / np.max(np.abs(want))),
                  float(np.max(np.abs(pc.get_dref_pft(1, True) - dwant)) / np.max(np.abs(dwant))))
    t0 = time.perf_counter()
    O.fdf_project_polar(g, t, ex, box, e64[1])
    t_fdf_cpu = time.perf_counter() - t0
    pc.kill()
    samples = n * (w.kto - w.kfrom + 1) * w.pftsz
    print(json.dumps({"report": "project", "box": box, "refs": n, "samples_per_call": samples,
                      "gpu_seconds_per_call": t_proj, "refs_per_s": n / t_proj, "samples_per_s": samples / t_proj,
                      "expand_cmat_seconds": t_expand, "parity_max_rel_err_vs_oracle": worst,
                      "oracle_seconds_per_ref_1_thread": t_cpu, "fdf_gpu_seconds_per_call": t_fdf,
                      "fdf_refs_per_s": n / t_fdf, "fdf_parity_max_rel_err_vs_oracle": fdf_err,
                      "fdf_oracle_seconds_per_ref_1_thread": t_fdf_cpu}), flush=True)


def run_euclid_report(args):
    """The Euclidean objective (cc_objfun = OBJFUN_EUCLID) on the config-1 geometry: the exact
    batched search (search_best, PFTCC_PREC_EXACT) of 1,000 particles over 100 references x 9
    shifts x 360 rotations under OBJFUN_CC and under OBJFUN_EUCLID (GPU wall time per call,
    synchronous), 1,000 batched sigma_contrib requests, parity of gencorrs_euclid for three
    pairs against the oracle and the oracle's single-thread time per pair."""
    pkg = entry.load_package()
    O = entry.load_oracle()
    w = pkg.synth.config1(nrefs=100, nptcls=1000)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ref")
    pc.set_refs(1, refs, True)
    pc.set_refs(1, refs, False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    K = w.kto - w.kfrom + 1
    sig = (np.random.default_rng(6).uniform(0.5, 2.0, (w.nptcls, K)) * np.linspace(4.0, 0.5, K)).astype(np.float32)
    pc.assign_sigma2_noise(sig)
    shifts = np.array([[x, y] for x in (-1.0, 0.0, 1.0) for y in (-1.0, 0.0, 1.0)], np.float32)
    out = {"report": "euclid", "box": w.box, "nrefs": w.nrefs, "nptcls": w.nptcls, "nshifts": len(shifts),
           "nrots": w.nrots, "shells": w.kto - w.kfrom + 1}
    evals = w.nptcls * w.nrefs * len(shifts) * w.nrots
    for name, obj in (("cc", pkg._lib.OBJFUN_CC), ("euclid", pkg._lib.OBJFUN_EUCLID)):
        pc.set_objfun(obj)
        pc.search_best(shifts, "exact")
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            pc.search_best(shifts, "exact")
        dt = (time.perf_counter() - t0) / reps
        out[f"exact_search_{name}_seconds"] = dt
        out[f"exact_search_{name}_evals_per_s"] = evals / dt
    n = 1000
    rng = np.random.default_rng(7)
    ir = rng.integers(1, w.nrefs + 1, n)
    ip = rng.integers(1, w.nptcls + 1, n)
    ro = rng.integers(1, w.nrots + 1, n)
    sh = rng.uniform(-2, 2, (n, 2)).astype(np.float32)
    pc.sigma_contrib_batch(ir, ip, ro, sh)
    t0 = time.perf_counter()
    pc.sigma_contrib_batch(ir, ip, ro, sh)
    out["sigma_contrib_batch_1000_seconds"] = time.perf_counter() - t0
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    worst = 0.0
    t0 = time.perf_counter()
    for i in range(3):
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
        want = O.gencorrs_euclid(g, t, refs[i], pc.get_ptcl_pft(i + 1), sig[i].astype(np.float64), c, [0.5, -0.5])
        got = pc.gencorrs_euclid(i + 1, i + 1, [0.5, -0.5])
        worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
    out["oracle_seconds_per_pair_1_thread"] = (time.perf_counter() - t0) / 3
    out["parity_max_scaled_err_vs_oracle"] = worst
    pc.kill()
    # the m-domain search (particle CTF frame, BF16 hi+lo products, FP32 re-score of the top 8)
    # over a 9 x 9 shift grid under both objectives
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ptcl")
    pc.set_refs(1, refs, True)
    pc.set_refs(1, refs, False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    pc.assign_sigma2_noise(sig)
    grid = np.array(w.shift_grid, np.float32).reshape(-1, 2)
    evals_md = w.nptcls * w.nrefs * len(grid) * w.nrots
    out["mdomain_nshifts"] = len(grid)
    for name, obj in (("cc", pkg._lib.OBJFUN_CC), ("euclid", pkg._lib.OBJFUN_EUCLID)):
        pc.set_objfun(obj)
        pc.search_best(grid, "bf16x3", ntop=8)
        t0 = time.perf_counter()
        reps = 5
        for _ in range(reps):
            pc.search_best(grid, "bf16x3", ntop=8)
        dt = (time.perf_counter() - t0) / reps
        out[f"mdomain_search_{name}_seconds"] = dt
        out[f"mdomain_search_{name}_evals_per_s"] = evals_md / dt
    pc.kill()
    print(json.dumps(out), flush=True)


def run_ingest_report(args):
    """Particle ingestion (pftcc_prep_ptcls: prepimg4align + polarize) on the config-1 geometry:
    4,096 seeded box-128 particle images (shifted Gaussian blobs in noise, random shifts within
    +-5 px, CTFFLAG_YES with astigmatic defocus), GPU wall time per call with the images copied
    from host memory inside it, parity of three particles against the oracle's prepimg4align +
    polarize, and the oracle's single-thread time per particle."""
    pkg = entry.load_package()
    O = entry.load_oracle()
    w = pkg.synth.config1()
    B, n, msk = w.box, 4096, w.box / 2 - 10.0
    rng = np.random.default_rng(8)
    yy, xx = np.mgrid[0:B, 0:B]
    base = np.exp(-((xx - B / 2) ** 2 + (yy - B / 2) ** 2) / (2 * 12.0 ** 2)).astype(np.float32)
    imgs = (2.0 + 4.0 * base[None] + 0.8 * rng.standard_normal((n, B, B))).astype(np.float32)
    xy = rng.uniform(-5, 5, (n, 2)).astype(np.float32)
    flags = np.ones(n, np.int32)
    dfx = rng.uniform(1.0, 3.0, n)
    ctfp = pkg.ctfparams_array(n, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca, dfx=dfx, dfy=dfx - 0.2,
                               angast=rng.uniform(0, 180, n))
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, n), box=B, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    pc.prep_ptcls(0, imgs, xy, flags, ctfp, msk)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        pc.prep_ptcls(0, imgs, xy, flags, ctfp, msk)
    dt = (time.perf_counter() - t0) / reps
    g = O.geom(w.nrots, w.kfrom, w.kto, B)
    t = O.tables(g)
    worst = 0.0
    t0 = time.perf_counter()
    for i in range(3):
        c = O.make_ctf(smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca, dfx=float(np.float32(dfx[i])),
                       dfy=float(np.float32(dfx[i] - 0.2)), angast=float(ctfp[i].angast))
        want = O.polarize(g, t, O.prepimg4align(imgs[i], B, msk, float(xy[i, 0]), float(xy[i, 1]), c))
        worst = max(worst, float(np.max(np.abs(pc.get_ptcl_pft(i + 1) - want)) / np.max(np.abs(want))))
    t_cpu = (time.perf_counter() - t0) / 3
    pc.kill()
    print(json.dumps({"report": "ingest", "box": B, "particles": n, "gpu_seconds_per_call": dt,
                      "particles_per_s": n / dt, "h2d_bytes_per_call": int(imgs.nbytes),
                      "parity_max_rel_err_vs_oracle": worst, "oracle_seconds_per_particle_1_thread": t_cpu}),
          flush=True)


def run_hbm_report(args):
    """DRAM rates of this GPU on 8 GiB buffers (far above L2), CUDA events, best of 10 after 3
    warm-ups: write-only (a memset), read-only (a max-reduction over FP32, whose output is one
    value) and copy (read + write bytes).  Stage 1 of the search writes its spectra and reads
    little, stage 2 reads them and writes little, so these are the rates their fractions use."""
    import torch
    dev = torch.device("cuda", 0)
    n = (8 << 30) // 4
    a = torch.ones(n, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)

    def timed(fn):
        for _ in range(3):
            fn()
        best = float("inf")
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return best

    nb = n * 4
    t_w = timed(lambda: b.zero_())
    t_r = timed(lambda: torch.amax(a))
    t_c = timed(lambda: b.copy_(a))
    print(json.dumps({"report": "hbm", "bytes": nb, "write_only_gbs": nb / t_w / 1e9, "read_only_gbs": nb / t_r / 1e9,
                      "copy_gbs": 2 * nb / t_c / 1e9, "how": "8 GiB FP32: zero_ (write), amax (read), copy_ "
                      "(read + write bytes); best of 10 after 3 warm-ups, CUDA events"}), flush=True)


def main():
    args = parse()
    if args.report == "hbm":
        run_hbm_report(args)
        return
    if args.report == "ingest":
        run_ingest_report(args)
        return
    if args.report == "euclid":
        run_euclid_report(args)
        return
    if args.report == "batching":
        run_batching_report(args)
        return
    if args.report == "precision":
        run_precision_report(args)
        return
    if args.report == "refine":
        run_refine_report(args)
        return
    if args.report == "project":
        run_project_report(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
