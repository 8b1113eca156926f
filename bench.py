#!/usr/bin/env python
"""(T) energy+VJP throughput on B200: triples/s and TFLOP/s, mixed vs FP64.

Workload: the nocc=48, nvir=500, naux=1500, seed-3 system (the large
single-system configuration), inputs generated directly in HBM.  One step is
the energy + VJP of one reference slab block (a0,a1,b0,b1) = (v-da, v, v-da, v)
— the first block pyscfad's driver processes (pyscfad/cc/ccsd_t.py:145, reversed
prange_tril) — through the device C-ABI ``ct_energy_vjp_block``.

  triples/s  = ordered (i,j,k,a,b,c) amplitudes covered per step / step time
               (a sorted job a>=b>=c covers nocc^3 x {6,3,1} orderings)
  TFLOP/s    = 3 F_E per job / step time, F_E = 12 nocc^3 (nvir+nocc) (the
               reference's dgemm count for the energy; energy+VJP = 3 F_E)

Multi-GPU runs (torchrun) are independent replicas ("weak" scaling): the (T)
kernel has no exchange step on one system.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

O, V, NAUX, SEED = 48, 500, 1500, 3
KEYS = ("mo_energy", "t1T", "t2T", "vooo", "fvo", "vvop")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="auto", choices=["auto", "fp64", "tf32", "bf16x3"])
    ap.add_argument("--da", type=int, default=0, help="slab width of the timed block (0 = by mode)")
    ap.add_argument("--fp64-da", type=int, default=0, help="slab width of the FP64 block (0 = the timed block)")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--no-fp64-e2e", action="store_true")
    ap.add_argument("--whole-system", type=int, default=0,
                    help="time one whole system of this configuration (3: nocc=32 nvir=300) through "
                         "ct_energy_vjp in every mode instead of the block benchmark")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--nocc", type=int, default=0, help="override nocc (small profiling cases)")
    ap.add_argument("--nvir", type=int, default=0, help="override nvir (small profiling cases)")
    ap.add_argument("--naux", type=int, default=0, help="override naux (small profiling cases)")
    return ap.parse_args()


# ---------------------------------------------------------------- job algebra
def block_jobs(v, a0, a1, b0, b1):
    """(njobs, ordered amplitude multiplicity sum) of a reference slab block
    (_ccsd_t_gen_jobs, ccsd_t.c:16-69)."""
    nj = 0
    mult = 0
    for a in range(a0, a1):
        bs = range(b0, b1) if b1 <= a0 else range(a0, a + 1)
        for b in bs:
            if b > a:
                continue
            for c in range(0, b + 1):
                nj += 1
                mult += 1 if a == c else (3 if (a == b or b == c) else 6)
    return nj, mult


def flops_per_job(o, v):
    return 12.0 * o ** 3 * (v + o)


# profiled kernel kinds (ct_profile_read ids) of the tensor-core contractions
GEMM_OV = {0, 4, 5, 10, 11, 12}      # 12 o^3 v flops per job (F1, VB, TB)
GEMM_OO = {1, 6, 7, 13, 14, 15}      # 12 o^4 flops per job (F2, OB1, OB2)


def roofline_units(kind, mode, o, v):
    """(bound, algorithmic units per job, unit) of one kernel kind: flops for
    the contractions (bf16x3 issues three bf16 products per product, counted
    as issued tensor flops), bytes for the orbit epilogue (reads the six
    G slots and the V-term tiles, writes the six W-bar slots and ybar) and
    the V-term kernel (reads ybar once per axis)."""
    es = 8 if mode == "fp64" else 4
    if kind in GEMM_OV or kind in GEMM_OO:
        f = 12.0 * o ** 3 * (v if kind in GEMM_OV else o)
        return ("tensor", f * (3.0 if mode == "bf16x3" else 1.0), "TFLOP/s")
    if kind == 2:
        return ("hbm", 13.0 * o ** 3 * es + 12.0 * o * o * es, "GB/s")
    if kind == 3:
        return ("hbm", 3.0 * o ** 3 * es + 12.0 * o * o * 8, "GB/s")
    return ("hbm", 8.0, "GB/s")


# ---------------------------------------------------------------- ranks
def max_over_ranks(x: float, dist, device=None) -> float:
    """The largest value of x over all ranks (every rank gets it); x itself
    when not distributed.  Replicas time their own steps; the job's time is
    the slowest replica's."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(amps_per_step: float, sec_per_step: float, world: int) -> float:
    """Weak-scaling throughput: every replica processes the same step, so the
    job covers world x amps_per_step amplitudes per (slowest) step time."""
    return world * amps_per_step / sec_per_step


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mem = float(parts[9]) if len(parts) > 9 else float("nan")
                rows.append((float(parts[1]), float(parts[2]), parts[5:9], float(parts[3]), mem))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, flag in enumerate(r[2]) if flag.lower() == "active"})
        load = [r for r in rows if r[3] > 300.0] or rows
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": max(r[1] for r in rows),
                "mem_mhz": statistics.median(r[4] for r in load), "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, dist):
    import torch
    from pyscfad_b200 import native, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    L = native.lib()
    mode = args.mode
    if mode == "auto":
        mode = os.environ.get("CTB_BENCH_MODE", "tf32")
    st = torch.cuda.current_stream(dev)
    stream = ctypes.c_void_p(st.cuda_stream)

    t0 = time.time()
    Ld = synth.device_layouts(O, V, NAUX, SEED, device=dev)
    gen_s = time.time() - t0
    G = {k: torch.zeros_like(Ld[k]) for k in KEYS}
    prob = native.CtProblem(O, V, *[ctypes.c_void_p(Ld[k].data_ptr()) for k in KEYS])
    grads = native.CtGrads(*[ctypes.c_void_p(G[k].data_ptr()) for k in KEYS])
    e_dev = torch.zeros((), dtype=torch.float64, device=dev)

    def step(m, a0, a1):
        s = L.ct_energy_vjp_block(ctypes.byref(prob), native.mode_id(m), 2.0, ctypes.byref(grads),
                                  a0, a1, a0, a1, ctypes.c_void_p(e_dev.data_ptr()), stream)
        native.check(s, "ct_energy_vjp_block")

    # probe: fall back to FP64 if the mixed path is unavailable in this build
    da = args.da or (24 if mode != "fp64" else 2)
    try:
        step(mode, V - 1, V)
    except native.CtError:
        if mode == "fp64":
            raise
        mode, da = "fp64", (args.da or 2)
    a0, a1 = V - da, V
    njobs, mult = block_jobs(V, a0, a1, a0, a1)
    amps = mult * O ** 3
    flops = 3.0 * flops_per_job(O, V) * njobs

    for _ in range(args.warmup):
        step(mode, a0, a1)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    L.ct_profile_enable(1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev0.record(st)
        evs[0].record(st)
        for i in range(args.steps):
            step(mode, a0, a1)
            evs[i + 1].record(st)
        ev1.record(st)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
    ms = ev0.elapsed_time(ev1)
    step_ms = [round(evs[i].elapsed_time(evs[i + 1]), 1) for i in range(args.steps)]
    prof = {}
    for kind in range(16):
        tot = ctypes.c_double(0)
        n = ctypes.c_int(0)
        native.check(L.ct_profile_read(kind, ctypes.byref(tot), ctypes.byref(n)))
        if n.value:
            prof[kind] = (tot.value, n.value)
    L.ct_profile_enable(0)
    clocks = clk.summary()
    ms = max_over_ranks(ms, dist, dev)
    sec = ms / 1e3
    res = dict(mode=mode, da=da, njobs=njobs, amps=amps, flops=flops, ms=ms, sec=sec, prof=prof, step_ms=step_ms,
               clocks=clocks, gen_s=gen_s, energy_block=float(e_dev.item()))

    # roofline of the dominant kernel
    kind_names = {0: "W-build GEMM (F1)", 1: "vooo W term (F2)", 2: "orbit epilogue", 3: "V-term bars",
                  4: "vvop-bar GEMM (VB)", 5: "t2-bar GEMM (TB)", 6: "vooo-bar GEMM (OB1)",
                  7: "t2 vooo-bar GEMM (OB2)", 8: "energy reduction", 9: "mixed operand prep",
                  10: "tcgen05 W-build GEMM", 11: "tcgen05 vvop-bar GEMM", 12: "tcgen05 t2-bar GEMM",
                  13: "tcgen05 vooo W term (F2)", 14: "tcgen05 vooo-bar GEMM (OB1)", 15: "tcgen05 t2 vooo-bar GEMM (OB2)"}
    dom = max(prof, key=lambda k: prof[k][0]) if prof else None
    res["dominant"] = dom
    if dom is not None:
        tot_ms, launches = prof[dom]
        res["roofline_kind"] = roofline_units(dom, mode, O, V)
        bound, per_job, _ = res["roofline_kind"]
        res["roofline_achieved"] = per_job * njobs * args.steps / (tot_ms / 1e3) / (1e12 if bound == "tensor" else 1e9)
        res["dominant_name"] = kind_names.get(dom, str(dom))
        res["dominant_launches"] = launches
        res["dominant_ms_per_launch"] = tot_ms / launches
    res["prof_share"] = {kind_names.get(k, str(k)): round(v[0] / sum(x[0] for x in prof.values()), 4)
                         for k, v in prof.items()}

    # FP64 on the same block: the like-for-like denominator of the speed-up,
    # and the float64 block energy each mode's error is measured against
    if mode != "fp64" and not args.no_fp64:
        fa0 = V - (args.fp64_da or da)
        fj, fm = block_jobs(V, fa0, V, fa0, V)
        step("fp64", V - 1, V)      # warm-up on a one-a block: float64 scratch, caches
        torch.cuda.synchronize(dev)
        nf = max(1, args.fp64_steps)
        fev = [torch.cuda.Event(enable_timing=True) for _ in range(nf + 1)]
        fev[0].record(st)
        for i in range(nf):
            step("fp64", fa0, V)
            fev[i + 1].record(st)
        torch.cuda.synchronize(dev)
        f_step = [fev[i].elapsed_time(fev[i + 1]) for i in range(nf)]
        fms = max_over_ranks(statistics.mean(f_step), dist, dev)
        res["fp64"] = dict(njobs=fj, ms=fms, step_ms=[round(x, 1) for x in f_step], steps=nf,
                           block=[fa0, V, fa0, V], triples_per_s=fm * O ** 3 / (fms / 1e3),
                           tflops=3.0 * flops_per_job(O, V) * fj / (fms / 1e3) / 1e12)
        if fa0 == a0:
            e64 = float(e_dev.item())
            em = res["energy_block"]
            s_phys = synth.PHYSICAL_ERI_SCALE.get(4) if (O, V) == (48, 500) else None
            acc = {"block_energy_fp64_Eh": e64, "block_energy_mode_Eh": em, "abs_err_Eh": abs(em - e64),
                   "rel_err": abs(em - e64) / abs(e64)}
            if s_phys:
                acc["physical_scale"] = {"eri_scale": s_phys, "block_energy_Eh": s_phys ** 2 * e64,
                                         "abs_err_Eh": s_phys ** 2 * abs(em - e64),
                                         "gate_Eh": 1e-6, "note": "ERIs x 2^-16 (|E(T)| of the whole system "
                                         "about 1e-2 Eh); a power-of-two scale changes no rounding, so the "
                                         "error is s^2 times the one measured at the generator scale"}
            res["accuracy"] = acc
    # peaks for the roofline denominators
    pk = ctypes.c_double(0)
    if L.ct_peak_probe(0, ctypes.byref(pk)) == 0:
        res["fp64_dmma_peak"] = pk.value
    if L.ct_peak_probe(1, ctypes.byref(pk)) == 0:
        res["fp64_dfma_peak"] = pk.value

    # CPU baseline (rank 0 at N=1): the reference's compiled kernel on a bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        host = host_inputs(Ld)
        cpu = cpu_reference_sample(host, target_s=12.0)
        del host

    # e2e through the host-pointer C-ABI (pinned buffers, copies inside the timed region)
    if not args.no_e2e:
        hb = {k: torch.empty(Ld[k].shape, dtype=torch.float64, pin_memory=True) for k in KEYS if k != "vvop"}
        for k in hb:
            hb[k].copy_(Ld[k])
        row = torch.empty((da, a1) + tuple(Ld["vvop"].shape[2:]), dtype=torch.float64, pin_memory=True)
        row.copy_(Ld["vvop"][a0:a1, :a1])
        col = torch.empty((a0, da) + tuple(Ld["vvop"].shape[2:]), dtype=torch.float64, pin_memory=True)
        col.copy_(Ld["vvop"][:a0, a0:a1])
        del Ld, G
        torch.cuda.empty_cache()
        hbar = {k: torch.zeros_like(hb[k]) for k in hb}
        rowb, colb = torch.zeros_like(row), torch.zeros_like(col)
        p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

        def host_step():
            s = L.ctb_ccsd_t_energy_vjp_mode(
                p(hb["mo_energy"]), p(hb["t1T"]), p(hb["t2T"]), p(hb["vooo"]), p(hb["fvo"]), 2.0,
                O, V, a0, a1, a0, a1, p(row), p(col), p(row), p(col),
                p(hbar["mo_energy"]), p(hbar["t1T"]), p(hbar["t2T"]), p(hbar["vooo"]), p(hbar["fvo"]),
                p(rowb), p(colb), p(rowb), p(colb), native.mode_id(mode))
            native.check(s, "ctb_ccsd_t_energy_vjp_mode")

        host_step()
        if dist is not None:
            dist.barrier()
        w0 = time.perf_counter()
        ne = max(1, min(args.steps, 2))
        for _ in range(ne):
            host_step()
        w1 = time.perf_counter()
        esec = (w1 - w0) / ne
        esec = max_over_ranks(esec, dist, dev)
        h2d = sum(hb[k].numel() for k in hb) * 8 + (row.numel() + col.numel()) * 8
        d2h = sum(hbar[k].numel() for k in hbar) * 8 + (rowb.numel() + colb.numel()) * 8
        res["e2e"] = dict(sec=esec, h2d=h2d, d2h=d2h)
        if mode != "fp64" and not args.no_fp64 and not args.no_fp64_e2e:
            # the float64 path through the reference's own 25-argument entry
            def host_step64():
                s = L.ctb_ccsd_t_energy_vjp(
                    p(hb["mo_energy"]), p(hb["t1T"]), p(hb["t2T"]), p(hb["vooo"]), p(hb["fvo"]), 2.0,
                    O, V, a0, a1, a0, a1, p(row), p(col), p(row), p(col),
                    p(hbar["mo_energy"]), p(hbar["t1T"]), p(hbar["t2T"]), p(hbar["vooo"]), p(hbar["fvo"]),
                    p(rowb), p(colb), p(rowb), p(colb))
                native.check(s, "ctb_ccsd_t_energy_vjp")
            w0 = time.perf_counter()
            host_step64()
            e64sec = max_over_ranks(time.perf_counter() - w0, dist, dev)
            res["e2e_fp64"] = dict(sec=e64sec, h2d=h2d, d2h=d2h)
        del hb, hbar, row, col, rowb, colb
    return res, cpu


# ---------------------------------------------------------------- CPU (reference C kernel)
def host_inputs(Ld):
    """Host copies the reference CPU kernel needs for one-a blocks (a0,a1)=(v-1,v)."""
    h = {k: np.ascontiguousarray(Ld[k].cpu().numpy()) for k in ("mo_energy", "t1T", "t2T", "vooo", "fvo")}
    h["row_a"] = np.ascontiguousarray(Ld["vvop"][V - 1:V, :V].cpu().numpy())
    h["col_a"] = np.ascontiguousarray(Ld["vvop"][:V - 1, V - 1:V].cpu().numpy())
    vv = Ld["vvop"]
    h["get_b"] = lambda b: (np.ascontiguousarray(vv[b:b + 1, :b + 1].cpu().numpy()),
                            np.ascontiguousarray(vv[:b, b:b + 1].cpu().numpy()) if b > 0 else None)
    return h


def cpu_reference_sample(host, target_s=15.0, steps=1, warmup=0):
    """Times the reference's ccsd_t_energy_vjp (oracle/_ref) on one-a slab
    blocks of the same system: (a0,a1)=(v-1,v) with one b (off-diagonal block,
    b+1 jobs) sized to ~target_s of CPU work.  Returns (amplitudes/s, info)."""
    import psutil
    from oracle import ref
    cores = os.cpu_count() or 1
    per_thread = (V * V * O * O + V * O ** 3) * 8 + (1 * V + V) * O * (O + V) * 8
    avail = psutil.virtual_memory().available
    threads = int(max(1, min(cores, 128, (0.6 * avail) // per_thread)))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    lib = ref.lib()
    bufs = {k: np.ascontiguousarray(host[k]) for k in ("mo_energy", "t1T", "t2T", "vooo", "fvo")}
    bars = {k: np.zeros_like(bufs[k]) for k in bufs}

    def run(b):
        # off-diagonal block a in [v-1, v), b in [b, b+1), c in [0, b]
        a0, a1, b0, b1 = V - 1, V, b, b + 1
        row_a = host["row_a"]                      # vvop[v-1:v, :v]
        col_a = host["col_a"]                      # vvop[:v-1, v-1:v]
        row_b, col_b = host["get_b"](b)
        if col_b is None:
            col_b = row_b
        rab, cab = np.zeros_like(row_a), np.zeros_like(col_a)
        rbb, cbb = np.zeros_like(row_b), np.zeros_like(col_b)
        t = time.perf_counter()
        ref.ref_call(bufs["mo_energy"], bufs["t1T"], bufs["t2T"], bufs["vooo"], bufs["fvo"], 2.0,
                     O, V, a0, a1, b0, b1, row_a, col_a, row_b, col_b,
                     bars["mo_energy"], bars["t1T"], bars["t2T"], bars["vooo"], bars["fvo"],
                     rab, cab, rbb, cbb)
        return time.perf_counter() - t

    # size: first a 10-job block, then scale b
    t_small = run(9)
    per_job = t_small / 10.0
    b = int(min(V - 2, max(9, target_s / max(per_job, 1e-6) - 1)))
    for _ in range(warmup):
        run(b)
    times = [run(b) for _ in range(max(1, steps))]
    sec = statistics.mean(times)
    njobs = b + 1
    mult = sum(1 if (V - 1) == c else (3 if (V - 1 == b or b == c) else 6) for c in range(b + 1))
    info = dict(cores=threads, sample=f"ccsd_t_energy_vjp block (a0,a1,b0,b1)=({V-1},{V},{b},{b+1}): "
                f"{njobs} jobs of nocc={O} nvir={V}; OMP_NUM_THREADS={threads} (of {cores} cores, "
                f"capped by the kernel's per-thread t2T_bar copies), scipy OpenBLAS 1 thread",
                sec=sec, njobs=njobs, steps=len(times))
    return mult * O ** 3 / sec, info


# ---------------------------------------------------------------- whole system
def whole_system(args):
    """One whole system (every sorted job a>=b>=c) through the one-call device
    entry ct_energy_vjp in FP64, TF32 and BF16x3: device time per call, and
    each mixed mode's energy and gradient errors against FP64; then the
    energy-only per-job contributions of every mode (ct_energy with job
    energies out), whose relative errors show how a mode's error is spread
    over the jobs (mean = systematic part)."""
    import torch
    from pyscfad_b200 import native, synth
    o, v, naux, seed = synth.CONFIGS[args.whole_system]
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = native.lib()
    st = torch.cuda.current_stream(dev)
    stream = ctypes.c_void_p(st.cuda_stream)
    Ld = synth.device_layouts(o, v, naux, seed, device=dev)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    prob = native.CtProblem(o, v, *[vp(Ld[k]) for k in KEYS])
    nj = v * (v + 1) * (v + 2) // 6
    amps = float(o) ** 3 * float(v) ** 3
    flops = 3.0 * flops_per_job(o, v) * nj
    G64 = {k: torch.zeros_like(Ld[k]) for k in KEYS}
    Gm = {k: torch.zeros_like(Ld[k]) for k in KEYS}
    e_out = torch.zeros((), dtype=torch.float64, device=dev)
    out = {"config": {"nocc": o, "nvir": v, "naux": naux, "seed": seed, "jobs": nj, "amplitudes": amps,
                      "flops_3FE": flops}, "modes": {}}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for m in ("fp64", "tf32", "bf16x3"):
        G = G64 if m == "fp64" else Gm
        for k in KEYS:
            G[k].zero_()
        gr = native.CtGrads(*[vp(G[k]) for k in KEYS])
        # workspace, operand copies and the full plan are set up by a first small call
        native.check(L.ct_energy_vjp_block(ctypes.byref(prob), native.mode_id(m), 0.0, ctypes.byref(gr),
                                           v - 1, v, v - 1, v, vp(e_out), stream))
        calls = 1 if m == "fp64" else 2
        times = []
        for c in range(calls):
            if c:
                for k in KEYS:
                    G[k].zero_()
            torch.cuda.synchronize(dev)
            ev0.record(st)
            native.check(L.ct_energy_vjp(ctypes.byref(prob), native.mode_id(m), 2.0, ctypes.byref(gr), vp(e_out),
                                         stream), "ct_energy_vjp")
            ev1.record(st)
            torch.cuda.synchronize(dev)
            times.append(ev0.elapsed_time(ev1))
        ms = min(times)
        rec = {"ms_per_call": [round(t, 1) for t in times], "triples_per_s": amps / (ms / 1e3),
               "tflops_3FE": flops / (ms / 1e3) / 1e12, "energy_Eh": float(e_out.item())}
        if m != "fp64":
            e64 = out["modes"]["fp64"]["energy_Eh"]
            rec["abs_err_Eh"] = abs(rec["energy_Eh"] - e64)
            rec["rel_err"] = rec["abs_err_Eh"] / abs(e64)
            rec["grad_rel_err"] = {k: float(torch.linalg.norm(Gm[k] - G64[k]) / torch.linalg.norm(G64[k]))
                                   for k in KEYS if float(torch.linalg.norm(G64[k])) > 0}
            s_phys = synth.PHYSICAL_ERI_SCALE.get(args.whole_system)
            if s_phys:
                rec["physical_scale"] = {"eri_scale": s_phys, "energy_Eh": s_phys ** 2 * e64,
                                         "abs_err_Eh": s_phys ** 2 * rec["abs_err_Eh"]}
            rec["speedup_vs_fp64"] = out["modes"]["fp64"]["ms_per_call"][0] / ms
        out["modes"][m] = rec
    del G64, Gm
    # per-job energies, energy only
    je = {}
    for m in ("fp64", "tf32", "bf16x3"):
        je[m] = torch.zeros(nj, dtype=torch.float64, device=dev)
        native.check(L.ct_energy(ctypes.byref(prob), native.mode_id(m), None, vp(je[m]), stream), "ct_energy")
    torch.cuda.synchronize(dev)
    ref = je["fp64"]
    mask = ref.abs() > 1e-12 * ref.abs().max()
    for m in ("tf32", "bf16x3"):
        rel = ((je[m] - ref) / ref.abs())[mask]
        out["modes"][m]["job_rel_err"] = {"mean": float(rel.mean()), "std": float(rel.std()),
                                          "median_abs": float(rel.abs().median()),
                                          "frac_magnitude_low": float(((je[m] - ref) * ref.sign() < 0)[mask]
                                                                      .double().mean()),
                                          "energy_only_sum_rel_err": float((je[m].sum() - ref.sum()).abs()
                                                                           / ref.sum().abs())}
    print(json.dumps(out), flush=True)



def main():
    global O, V, NAUX
    args = parse()
    if args.whole_system:
        whole_system(args)
        return
    O, V, NAUX = args.nocc or O, args.nvir or V, args.naux or NAUX
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    cfg = {"workload": f"ccsd(t) energy+vjp, nocc={O} nvir={V} naux={NAUX} seed={SEED}, "
                       f"one reference slab block per step",
           "nocc": O, "nvir": V, "naux": NAUX, "seed": SEED,
           "l2": "inputs larger than L2 (vvop 52.6 GB float64)",
           "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return
        import torch
        from pyscfad_b200 import synth
        Ld = synth.device_layouts(O, V, NAUX, SEED, device="cuda")
        host = host_inputs(Ld)
        val, info = cpu_reference_sample(host, steps=args.steps, warmup=min(args.warmup, 1))
        cfg["workload"] += f"; reference CPU sample: {info['sample']}"
        line = {"impl": "reference", "metric": "(T) energy+VJP triples/s", "value": val, "unit": "triples/s",
                "n_gpus": 1, "steps": info["steps"], "warmup": min(args.warmup, 1),
                "ms_per_step": info["sec"] * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": val, "unit": "triples/s", "cores": info["cores"],
                                 "kind": "reference", "sample": info["sample"]},
                "e2e": {"value": val, "unit": "triples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    res, cpu = gpu_arm(args, rank, world, dist)
    value = whole_job_value(res["amps"], res["sec"] / args.steps, world)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    mode = res["mode"]
    bound, per_job, unit = res.get("roofline_kind", ("tensor", None, "TFLOP/s"))

    def peak_of(key, fallback, what):
        if key in peaks:
            return float(peaks[key]), f"of measured: {what} (MEASURED_PEAKS.json {key})"
        return fallback, f"of fallback: {what} = {fallback:g} (MEASURED_PEAKS.json absent)"

    if bound == "hbm":
        peak, peak_src = peak_of("hbm_gbs", 6650.0, "HBM copy GB/s")
    elif mode == "fp64":
        peak, peak_src = res.get("fp64_dmma_peak"), "of measured: fp64 DMMA pipe, ct_peak_probe on this GPU"
    elif mode == "tf32":
        bf, src = peak_of("bf16_tflops_sustained", 1400.0, "bf16 sustained TFLOP/s")
        peak, peak_src = 0.5 * bf, "tf32 dense = 1/2 of " + src
    else:
        peak, peak_src = peak_of("bf16_tflops_sustained", 1400.0, "bf16 sustained TFLOP/s")
        peak_src += "; achieved counts the 3 issued bf16 products"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath) and res.get("dominant_launches"):
        try:
            tj = json.load(open(tpath))
            ent = tj.get(mode, {}).get(str(res.get("dominant")))
            if ent and ent.get("nocc") == O:
                traffic = ent["dram_bytes_per_job"] * res["njobs"] * args.steps / res["dominant_launches"]
        except Exception:
            traffic = None
    achieved = res.get("roofline_achieved")
    roofline = {"bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                "kernel": res.get("dominant_name"), "peak_source": peak_src,
                "algorithmic_per_job": per_job,
                "ms_per_launch": res.get("dominant_ms_per_launch"), "launches": res.get("dominant_launches"),
                "time_share": res.get("prof_share")}
    cfg.update({"mode": mode, "block": [V - res["da"], V, V - res["da"], V], "jobs_per_step": res["njobs"],
                "amplitudes_per_step": res["amps"], "flops_per_step": res["flops"],
                "tflops": world * res["flops"] / (res["sec"] / args.steps) / 1e12,
                "energy_block_Eh": res["energy_block"], "input_gen_s": round(res["gen_s"], 1),
                "step_ms": res["step_ms"]})
    if "fp64" in res:
        cfg["fp64"] = res["fp64"]
        cfg["speedup_vs_fp64"] = (res["amps"] / (res["sec"] / args.steps)) / res["fp64"]["triples_per_s"]
        cfg["speedup_vs_fp64_basis"] = ("same block, mean step times" if res["fp64"]["block"][0] == V - res["da"]
                                        else "FP64 rate on a smaller block of the same system")
    if "accuracy" in res:
        cfg["accuracy_vs_fp64"] = res["accuracy"]
    if "e2e_fp64" in res and "e2e" in res:
        cfg["e2e_fp64"] = {"value": whole_job_value(res["amps"], res["e2e_fp64"]["sec"], world), "unit": "triples/s",
                           "ms_per_step": res["e2e_fp64"]["sec"] * 1e3, "api": "ctb_ccsd_t_energy_vjp (25 arguments)",
                           "h2d_bytes_per_step": res["e2e_fp64"]["h2d"], "d2h_bytes_per_step": res["e2e_fp64"]["d2h"]}
        cfg["e2e_speedup_vs_fp64"] = res["e2e_fp64"]["sec"] / res["e2e"]["sec"]
    if "fp64_dmma_peak" in res:
        cfg["fp64_peaks_tflops"] = {"dmma": res["fp64_dmma_peak"], "dfma": res.get("fp64_dfma_peak")}
    line = {"metric": "(T) energy+VJP triples/s", "value": value, "unit": "triples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "tf32": "tf32/f32-acc/f64-reduce",
                      "bf16x3": "bf16x3/f32-acc/f64-reduce"}[mode],
            "data": "synthetic (seeded generator: DF ERIs, random t1/t2)", "config": cfg,
            "roofline": roofline, "clocks": res["clocks"],
            "gpu_launches": sum(v[1] for v in res["prof"].values())}
    if "e2e" in res:
        e = res["e2e"]
        line["e2e"] = {"value": whole_job_value(res["amps"], e["sec"], world), "unit": "triples/s",
                       "h2d_bytes_per_step": e["h2d"], "d2h_bytes_per_step": e["d2h"],
                       "ms_per_step": e["sec"] * 1e3,
                       "api": "ctb_ccsd_t_energy_vjp_mode (host pointers, pinned)"}
    if cpu is not None:
        cval, info = cpu
        line["cpu_baseline"] = {"value": cval, "unit": "triples/s", "cores": info["cores"],
                                "kind": "reference", "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
