#!/usr/bin/env python
"""Benchmark of the RI-JK Fock build (REST src/scf_io vj/vk) on B200.

One step = one FP64 Fock build on the synthetic kernel-sweep workload
(n = 1200 basis functions, N = 4800 auxiliary functions, nocc = 200):
J (vj_upper_with_rimatr_v) + K in the occupied-orbital form
(vk_upper_with_ri_v), with the fitted tensor resident in HBM (28 GB packed,
29 GB tile-packed, larger than the 126 MB L2 so no flush is needed).

  value  = (J + K algorithmic FLOPs) / device time of the step, TFLOP/s
           (CUDA events on the launching stream, max over ranks)
  e2e    = the same build through the host C ABI (host density / orbitals
           in, host J / K out, pinned buffers, copies inside the timed region)

--impl reference times REST's CPU algorithm restated in C (oracle/cpu_rijk.c,
OpenMP over the aux index, single-threaded OpenBLAS per P as REST does) on a
bounded sample of the same workload with all host threads.

With --gpus N (launched under torchrun) every rank runs an independent
replica on its own molecule: the kernel sweep has no exchange step.
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
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def workload(n: int, nocc: int = 0) -> dict:
    naux, nocc = 4 * n, (nocc or n // 6)
    npair = n * (n + 1) // 2
    return {
        "n": n,
        "naux": naux,
        "nocc": nocc,
        "npair": npair,
        "j_flops": 4.0 * naux * npair,
        "k_flops": 4.0 * naux * n * n * nocc,
        "half_flops": 2.0 * naux * n * n * nocc,  # X_P = B_P C, per build
        "rank_flops": 2.0 * naux * n * n * nocc,  # K += X_P X_P^T, per build
        "j_pass_bytes": 8.0 * naux * npair,  # one pass over packed B
    }


def config_of(w: dict, ngpu: int) -> dict:
    return {
        "workload": f"synthetic RI-JK sweep, FP64 plain form: n={w['n']}, N={w['naux']}, nocc={w['nocc']}; "
        "one Fock build (J of D = C C^T + occupied-orbital K) per step",
        "num_basis": w["n"],
        "num_auxbas": w["naux"],
        "nocc": w["nocc"],
        "tensor": "packed upper B[P, mu<=nu], FP64, resident in HBM",
        "l2": "inputs larger than L2 (28 GB tensor vs 126 MB L2); no flush needed",
        "parallelism": f"replicas x{ngpu}" if ngpu > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self, busy_mhz_floor: float = 600.0) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    rows.append((float(p[1]), float(p[2]), p[5:9]))
                except ValueError:
                    continue
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        busy = [r for r in rows if r[0] >= busy_mhz_floor] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in busy for i in range(4) if r[2][i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in busy),
                "reasons": reasons, "samples": len(busy)}


# ---------------------------------------------------------------------------
# CPU leg (REST's algorithm restated in C)
# ---------------------------------------------------------------------------
def cpu_sample_run(w: dict, target_s: float, seed: int = 2024):
    """Time one bounded-sample Fock build on the host; returns (TFLOP/s, threads, sample text)."""
    import numpy as np

    from oracle import rijk_oracle as O
    from oracle.cpu_baseline import CpuRijk
    from rest_b200.synth import host_case

    cpu = CpuRijk()
    n, nocc = w["n"], w["nocc"]
    probe = max(1, min(w["naux"], cpu.nthreads))
    case = host_case(n, w["naux"], nocc, seed=seed, rows=(0, probe))
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    occ = np.ones(nocc)
    t0 = time.perf_counter()
    cpu.vk_upper_with_ri_v(ri3, case.c_occ, nocc - 1, occ, -1.0)
    per_row = (time.perf_counter() - t0) / probe
    rows = int(max(probe, min(w["naux"], target_s / max(per_row, 1e-6))))
    rows = max(cpu.nthreads, (rows // cpu.nthreads) * cpu.nthreads) if rows >= cpu.nthreads else rows
    case = host_case(n, w["naux"], nocc, seed=seed, rows=(0, rows))
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)

    def step():
        t = time.perf_counter()
        cpu.vj_upper_with_rimatr(case.rimatr, n, case.dm, 1.0)
        cpu.vk_upper_with_ri_v(ri3, case.c_occ, nocc - 1, occ, -1.0)
        return time.perf_counter() - t

    flops = 4.0 * rows * w["npair"] + 4.0 * rows * n * n * nocc
    sample = (f"{rows} of {w['naux']} aux rows of the n={n} workload (J a2 + K a3 on those rows), "
              f"REST algorithm restated in C with OpenMP + OpenBLAS; REST binary unavailable on this box")
    return step, flops, cpu.nthreads, sample


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    step, flops, threads, sample = cpu_sample_run(w, target_s=4.0)
    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    t = sum(times) / len(times)
    v = flops / t / 1e12
    line = {
        "impl": "reference",
        "metric": "RI-JK TFLOP/s",
        "value": v,
        "unit": "TFLOP/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded NumPy draw of the kernel-sweep workload)",
        "config": config_of(w, 1),
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def measure_dgemm_peak(torch) -> float:
    """FP64 dense peak of this GPU, measured now: cuBLAS DGEMM 8192^3 (best of 5)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    a @ b
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / best / 1e12


def run_ours(args, w):
    import ctypes as C

    import numpy as np
    import torch

    from rest_b200 import RIJK, lib, replicas
    from rest_b200.synth import device_case

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rk = replicas.init("nccl", timeout_s=600)
    world, rank, local = rk.world, rk.rank, rk.local

    fp64_peak = measure_dgemm_peak(torch)
    ctx = RIJK(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.set_stream(stream)
    c_cm, dm = device_case(ctx, w["n"], w["naux"], w["nocc"], seed=1000 + rank)
    n, nocc, npair = w["n"], w["nocc"], w["npair"]
    occ = torch.ones(nocc, dtype=torch.float64, device="cuda")
    vj = torch.empty(npair, dtype=torch.float64, device="cuda")
    vk = torch.empty(npair, dtype=torch.float64, device="cuda")
    st = ctx.stream

    def step_separate():
        ctx.vj_upper_dev(dm.data_ptr(), 1, 1.0, 1, vj.data_ptr(), st)
        ctx.vk_upper_occ_dev(c_cm.data_ptr(), nocc, [nocc - 1], occ.data_ptr(), 1, -1.0, vk.data_ptr(), st)

    def step_fused():
        # J of D = C C^T and K in one build: J's aux-row scalars come out of the K half-transform
        ctx.vjk_upper_occ_dev(c_cm.data_ptr(), nocc, [nocc - 1], occ.data_ptr(), 1, 1.0, -1.0, vj.data_ptr(),
                              vk.data_ptr(), st)

    step = step_fused if args.jk == "fused" else step_separate

    def barrier():
        torch.cuda.synchronize()
        replicas.barrier(rk)

    for _ in range(max(3, args.warmup)):
        step()
    ctx.synchronize(st)
    ctx.profile(True)
    ctx.profile_read()
    barrier()
    launches0 = RIJK.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = (RIJK.kernel_launches() - launches0) // args.steps
    ctx.synchronize(st)
    prof = ctx.profile_read()
    ctx.profile(False)
    dt = replicas.max_over_ranks(rk, e0.elapsed_time(e1) / 1e3)  # the slowest rank's device time
    t_step = dt / args.steps
    flops = w["j_flops"] + w["k_flops"]
    value = world * flops / t_step / 1e12

    # roofline of the dominant kernel class (live events over the timed region)
    cls_time = {k: v[0] / 1e3 / args.steps for k, v in prof.items()}
    dom = max(cls_time, key=cls_time.get)
    algo = {"k_half": (w["half_flops"], "tensor"), "k_rank": (w["rank_flops"], "tensor"),
            "j_pass1": (w["j_pass_bytes"], "hbm"), "j_pass2": (w["j_pass_bytes"], "hbm")}
    peaks = json.load(open(MEASURED_PEAKS)) if os.path.exists(MEASURED_PEAKS) else {}
    work, bound = algo.get(dom, (w["half_flops"], "tensor"))
    dom_launches = max(1, prof[dom][1] // args.steps)
    if bound == "tensor":
        achieved = work / cls_time[dom] / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak,
                "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 via torch.matmul (FP64 has no "
                               "entry in MEASURED_PEAKS.json; tcgen05 has no FP64 kind, DMMA is the FP64 tensor path)"}
    else:
        achieved = work / cls_time[dom] / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6.65 TB/s"}
    roof["kernel"] = dom
    roof["launches_per_step"] = dom_launches
    roof["traffic"] = traffic_per_launch(dom, w, dom_launches)
    if roof["traffic"] is not None:
        roof["traffic_source"] = TRAFFIC_SOURCE
    # J kernels' own HBM roofline, reported beside the dominant one
    j_rates = {}
    for k in ("j_pass1", "j_pass2"):
        if cls_time.get(k):
            j_rates[k] = w["j_pass_bytes"] / cls_time[k] / 1e9

    # the other J/K form on the same workload, timed the same way (for the record)
    other = None
    if not args.no_split:
        alt = step_separate if args.jk == "fused" else step_fused
        for _ in range(2):
            alt()
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            alt()
        a1.record(stream)
        torch.cuda.synchronize()
        t_alt = a0.elapsed_time(a1) / 1e3 / args.steps
        other = {"jk": "separate" if args.jk == "fused" else "fused", "ms_per_step": t_alt * 1e3,
                 "value": world * flops / t_alt / 1e12,
                 "what": "J by two passes over the tensor (rijk_vj_upper_dev) + K (rijk_vk_upper_occ_dev)"
                 if args.jk == "fused" else "rijk_vjk_upper_occ_dev"}

    # split-precision exchange (3 x BF16 on tcgen05) on the same workload: the
    # first call builds the BF16 copies of the tensor (once per geometry)
    split = None
    if not args.no_split:
        vk_split = torch.empty(npair, dtype=torch.float64, device="cuda")

        def k_split():
            ctx.vk_upper_occ_split_dev(c_cm.data_ptr(), nocc, [nocc - 1], occ.data_ptr(), 1, -1.0,
                                       vk_split.data_ptr(), st)

        t_prep0 = time.perf_counter()
        k_split()
        ctx.synchronize(st)
        t_prep = time.perf_counter() - t_prep0
        for _ in range(2):
            k_split()
        ctx.synchronize(st)
        ctx.profile(True)
        ctx.profile_read()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            ctx.vj_upper_dev(dm.data_ptr(), 1, 1.0, 1, vj.data_ptr(), st)
            k_split()
        s1.record(stream)
        torch.cuda.synchronize()
        sp = ctx.profile_read()
        ctx.profile(False)
        t_mixed = s0.elapsed_time(s1) / 1e3 / args.steps
        rel = float((vk_split - vk).abs().max() / vk.abs().max())
        half_ms = sp["k_half"][0] / args.steps
        rank_ms = sp["k_rank"][0] / args.steps
        bf16_peak = peaks.get("bf16_tflops", 1590.0)
        half_tc = 3 * w["half_flops"] / (half_ms / 1e3) / 1e12  # BF16 tensor flops actually issued (3 products)
        split = {
            "what": "J in FP64 + K as 3 x BF16 split products on tcgen05 (FP32 accumulation in TMEM)",
            "fock_build_ms": t_mixed * 1e3,
            "value_tflops_alg": world * flops / t_mixed / 1e12,
            "speedup_vs_fp64_build": t_step / t_mixed,
            "k_rel_err_vs_fp64": rel,
            "k_half_ms": half_ms,
            "k_rank_ms": rank_ms,
            "half_roofline": {"bound": "tensor", "achieved": half_tc, "peak": bf16_peak, "unit": "TFLOP/s",
                              "frac": half_tc / bf16_peak,
                              "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if "bf16_tflops" in peaks
                              else "fallback 1.59 PFLOP/s"},
            "split_tensor_build_s": t_prep,
        }
        # the form a split step of the mixed SCF runs (rijk_vjk_upper_lowrank_split_dev):
        # J's scalars w_P = <C, B_P C> from the split half-transform's epilogue, so
        # J reads the FP64 tensor once (pass 2) instead of twice
        vj_f = torch.empty(npair, dtype=torch.float64, device="cuda")
        vk_f = torch.empty(npair, dtype=torch.float64, device="cuda")

        def jk_split_fused():
            ctx.vjk_upper_lowrank_split_dev(c_cm.data_ptr(), n, nocc, nocc, 1.0, -1.0, False, vj_f.data_ptr(),
                                            vk_f.data_ptr(), st)

        for _ in range(2):
            jk_split_fused()
        ctx.synchronize(st)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            jk_split_fused()
        f1.record(stream)
        torch.cuda.synchronize()
        t_fused = f0.elapsed_time(f1) / 1e3 / args.steps
        split["fused_split_jk"] = {
            "what": "J and K of D = C C^T from one split build (rijk_vjk_upper_lowrank_split_dev): J's scalars "
                    "from the split half-transform, J pass 2 over the FP64 tensor",
            "fock_build_ms": t_fused * 1e3,
            "speedup_vs_fp64_build": t_step / t_fused,
            "j_rel_err_vs_fp64": float((vj_f - vj).abs().max() / vj.abs().max()),
            "k_rel_err_vs_fp64": float((vk_f - vk).abs().max() / vk.abs().max()),
        }

    # e2e through the host C ABI, pinned host buffers
    e2e = None
    if not args.no_e2e:
        L = lib()
        h_dm = torch.empty(n * n, dtype=torch.float64).pin_memory()
        h_dm.copy_(dm.reshape(-1).cpu())
        h_c = torch.empty(n * nocc, dtype=torch.float64).pin_memory()
        h_c.copy_(c_cm.reshape(-1).cpu())
        h_occ = torch.ones(nocc, dtype=torch.float64).pin_memory()
        h_vj = torch.empty(npair, dtype=torch.float64).pin_memory()
        h_vk = torch.empty(npair, dtype=torch.float64).pin_memory()
        homo = (C.c_int64 * 2)(nocc - 1, 0)

        def e2e_step():
            if args.jk == "fused":
                r1 = L.rijk_vjk_upper_with_ri_v(ctx.handle, C.c_void_p(h_c.data_ptr()), nocc, homo,
                                                C.c_void_p(h_occ.data_ptr()), 1, 1.0, -1.0,
                                                C.c_void_p(h_vj.data_ptr()), C.c_void_p(h_vk.data_ptr()))
                r2 = 0
            else:
                r1 = L.rijk_vj_upper_with_rimatr_v(ctx.handle, C.c_void_p(h_dm.data_ptr()), 1, 1.0,
                                                   C.c_void_p(h_vj.data_ptr()))
                r2 = L.rijk_vk_upper_with_ri_v(ctx.handle, C.c_void_p(h_c.data_ptr()), nocc, homo,
                                               C.c_void_p(h_occ.data_ptr()), 1, -1.0, C.c_void_p(h_vk.data_ptr()))
            if r1 or r2:
                raise RuntimeError(f"e2e call failed: {r1} {r2}")

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        te = replicas.max_over_ranks(rk, time.perf_counter() - t0)
        h2d = ((n * n if args.jk == "separate" else 0) + n * nocc + nocc) * 8
        d2h = 2 * npair * 8
        e2e = {"value": world * flops / (te / args.steps) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": te / args.steps * 1e3,
               "how": ("rijk_vjk_upper_with_ri_v (orbitals and occupations in, J and K out)" if args.jk == "fused"
                       else "rijk_vj_upper_with_rimatr_v + rijk_vk_upper_with_ri_v")
               + " on pinned host buffers, wall clock"}

    # RI-HF SCF on the water molecule of the plain config (def2-SVP / def2-SVP-JKFIT):
    # FP64 GPU path and mixed-precision path, same converged energy
    scf = None
    if rank == 0 and not args.no_scf:
        from rest_b200.basis import Molecule
        from rest_b200.scf import SCF, ScfOptions

        water = Molecule.from_angstrom(["O", "H", "H"], [[0.0, 0.0, 0.0], [0.757, 0.587, 0.0], [-0.757, 0.587, 0.0]])
        tight = dict(scf_acc_etot=1e-8, scf_acc_rho=1e-6, scf_acc_eev=1e-6, max_scf_cycle=100)
        res = {}
        sctx = RIJK(local)
        for prec in ("fp64", "mixed"):
            t0 = time.perf_counter()
            runner = SCF(water, "def2-SVP", "def2-SVP-JKFIT", ScfOptions(precision=prec, **tight), ctx=sctx)
            r = runner.run()
            res[prec] = {"wall_s": time.perf_counter() - t0, "iterations": r.iterations, "energy": r.energy,
                         "converged": r.converged, "scf_s": r.timings["scf_s"],
                         "setup_s": r.timings["one_electron_s"] + r.timings["ri_integrals_s"] + r.timings["fit_s"],
                         "split_k_builds": r.timings["split_k_builds"]}
        sctx.close()
        scf = {"molecule": "H2O def2-SVP/def2-SVP-JKFIT (24 AO, 113 aux), RHF, 1e-8 Eh",
               "fp64": res["fp64"], "mixed": res["mixed"],
               "mixed_minus_fp64_energy": res["mixed"]["energy"] - res["fp64"]["energy"],
               "molecules_per_s_fp64": 1.0 / res["fp64"]["wall_s"],
               "molecules_per_s_mixed": 1.0 / res["mixed"]["wall_s"]}

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        stepf, cflops, threads, sample = cpu_sample_run(w, target_s=6.0)
        stepf()
        times = [stepf() for _ in range(2)]
        cpu_base = {"value": cflops / min(times) / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                    "sample": sample}

    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream())  # the context's stream ends with it
    ctx.close()
    torch.cuda.empty_cache()
    apps = {}
    if rank == 0 and world == 1 and not args.no_apps:
        apps["ri_tensor_build"] = measure_tensor_build(local)
        apps["precision_alkanes"] = measure_alkanes(local)
        apps["molecule_set"] = molecule_set_in_child(local, args.set_size)

    if rank == 0:
        line = {
            "metric": "RI-JK TFLOP/s",
            "value": value,
            "unit": "TFLOP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(3, args.warmup),
            "ms_per_step": t_step * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded torch CUDA draw of the kernel-sweep workload)",
            "config": config_of(w, world),
            "roofline": roof,
            "j_hbm_gbs": j_rates,
            "kernel_ms_per_step": {k: v * 1e3 for k, v in cls_time.items() if v},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu_base,
            "jk_form": args.jk,
            "other_jk_form": other,
            "split_precision": split,
            "scf_water": scf,
            **apps,
        }
        print(json.dumps(line), flush=True)
    replicas.finalize(rk)
    return 0


# ---------------------------------------------------------------------------
# application configs: device tensor build, alkane precision runs, molecule sets
# ---------------------------------------------------------------------------
def _shell_prefix(sh, nshell):
    """The first nshell shells of a ShellSet (a bounded CPU sample)."""
    from rest_b200.basis import ShellSet

    return ShellSet(sh.l[:nshell].copy(), sh.nprim[:nshell].copy(), sh.prim_off[:nshell].copy(), sh.exps, sh.coefs,
                    sh.centers[:nshell].copy(), sh.atom[:nshell].copy())


def measure_tensor_build(device: int, k: int = 50) -> dict:
    """All-device fitted tensor for (H2O)_k (def2-SVP / def2-SVP-JKFIT): device
    integrals + Cholesky metric + fit, against the host integral engine timed
    on the first water's auxiliary shells and scaled by the function count."""
    import numpy as np
    import torch

    from rest_b200 import RIJK
    from rest_b200.basis import int3c2e
    from rest_b200.geometry import water_cluster

    mol = water_cluster(k, seed=11)
    bas, aux = mol.shells("def2-SVP"), mol.shells("def2-SVP-JKFIT")
    n, naux = bas.nfun, aux.nfun
    npair = n * (n + 1) // 2
    ctx = RIJK(device)
    try:
        small = water_cluster(2, seed=5)
        ctx.build_rimatr_from_shells(small.shells("def2-SVP"), small.shells("def2-SVP-JKFIT"))  # load kernels
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.build_rimatr_from_shells(bas, aux)
        torch.cuda.synchronize()
        t_build = time.perf_counter() - t0
    finally:
        ctx.close()
    torch.cuda.empty_cache()
    nsh = int(np.sum(aux.atom < 3))  # the first water's auxiliary shells
    sub = _shell_prefix(aux, nsh)
    t0 = time.perf_counter()
    int3c2e(bas, sub)
    t_cpu = time.perf_counter() - t0
    cpu_full = t_cpu * naux / sub.nfun
    return {
        "molecule": f"(H2O)_{k} def2-SVP / def2-SVP-JKFIT, {n} AO, {naux} aux",
        "device_build_s": t_build,
        "integrals_per_s": npair * naux / t_build,
        "host_int3c2e_sample": f"{sub.nfun} of {naux} auxiliary functions, {os.cpu_count()} threads",
        "host_int3c2e_s_scaled": cpu_full,
        "device_vs_host_int3c2e_only": cpu_full / t_build,
    }


def measure_alkanes(device: int, sizes=(10, 20, 40)) -> list:
    """Precision config: FP64 vs mixed-precision batched driver on C_nH_{2n+2}."""
    from rest_b200.geometry import alkane
    from rest_b200.scf_batch import BatchedRHF

    crit = dict(acc_etot=1e-8, acc_rho=1e-6, acc_eev=1e-6, max_cycle=100)
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_energies.json")))
    oracle = {a["carbons"]: a["energy"] for a in golden["alkanes"]}
    out = []
    for nc in sizes:
        mol = alkane(nc)
        rec = {"molecule": f"C{nc}H{2 * nc + 2}", "num_basis": mol.shells("def2-SVP").nfun,
               "num_auxbas": mol.shells("def2-SVP-JKFIT").nfun, "nocc": mol.nelec // 2}
        for prec in ("fp64", "mixed"):
            # split_min_basis=0: the split path on every alkane (BatchedRHF's default
            # keeps molecules below 512 basis functions in FP64)
            b = BatchedRHF([mol], "def2-SVP", "def2-SVP-JKFIT", device=device, precision=prec, metric="cholesky",
                           split_min_basis=0)
            try:
                r = b.run(**crit)
            finally:
                b.close()
            rec[prec] = {"energy": r.energies[0], "converged": r.converged[0], "iterations": r.iterations[0],
                         "scf_s": r.scf_s, "setup_s": r.setup_s, "fp64_k_builds": r.timings["fp64_k_builds"][0],
                         "split_k_builds": r.timings["split_k_builds"][0]}
        rec["mixed_minus_fp64_energy"] = rec["mixed"]["energy"] - rec["fp64"]["energy"]
        if nc in oracle:  # FP64 CPU oracle energy (1e-10 Eh, committed fixture)
            rec["fp64_minus_oracle_energy"] = rec["fp64"]["energy"] - oracle[nc]
            rec["mixed_minus_oracle_energy"] = rec["mixed"]["energy"] - oracle[nc]
        rec["scf_speedup_mixed_vs_fp64"] = rec["fp64"]["scf_s"] / rec["mixed"]["scf_s"]
        out.append(rec)
    return out


def measure_molecule_set(device: int, nmol: int, plain_subset: int = 16, group: int = 32) -> dict:
    """Batched config: water clusters k uniform in 1..16 converged together
    (FP64; mixed precision; mixed precision from the learned guess) against the
    plain per-molecule FP64 GPU path on a subset."""
    import numpy as np
    import torch

    from rest_b200 import RIJK
    from rest_b200.basis import int1e
    from rest_b200.geometry import water_cluster, water_cluster_set_spec
    from rest_b200.guess import LearnedGuess
    from rest_b200.sad import sad_density
    from rest_b200.scf import SCF, ScfOptions
    from rest_b200.scf_batch import run_molecule_set

    crit = dict(acc_etot=1e-8, acc_rho=1e-6, acc_eev=1e-6, max_cycle=100)
    spec = water_cluster_set_spec(nmol, seed=2024)
    mols = [water_cluster(k, s) for k, s in spec]
    # FP64 oracle energies of a fixed subset of the set (converged on the CPU
    # oracle to 1e-10 Eh once, committed as a fixture; nothing runs the oracle here)
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_energies.json")))
    oracle_sub = {e["index"]: e["energy"] for e in golden["water_set"]["entries"]
                  if e["index"] < nmol and tuple(spec[e["index"]]) == (e["k"], e["seed"])}
    run_molecule_set(mols[:4], "def2-SVP", "def2-SVP-JKFIT", group_size=4, precision="mixed", device=device, **crit)
    # the guess model is loaded (weights read and uploaded, kernels loaded) once,
    # outside the timed runs, as a model is before serving; its time is reported
    t0 = time.perf_counter()
    guess = LearnedGuess.load(device=device)
    guess.density(mols[0], ovlp=int1e(mols[0], mols[0].shells("def2-SVP"), "ovlp"))
    guess_load_s = time.perf_counter() - t0
    res = {}

    def timed(tag, **kw):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if kw.pop("learned", False):
            kw["guess"] = guess  # predicted on the device, checked against the driver's S
        if kw.pop("sad", False):
            # REST's SAD guess: atomic densities (cached after the first call) on the block diagonal
            kw["initial_densities"] = [sad_density(m, "def2-SVP", "def2-SVP-JKFIT")[0] for m in mols]
        r = run_molecule_set(mols, "def2-SVP", "def2-SVP-JKFIT", group_size=group, device=device, **kw, **crit)
        wall = time.perf_counter() - t0
        extra = r.timings["setup_parts"].get("guess", 0.0)
        res[tag] = {"molecules_per_s": nmol / wall, "wall_s": wall, "setup_s": r.setup_s, "scf_s": r.scf_s,
                    "iterations_mean": float(np.mean(r.iterations)), "converged": int(sum(r.converged)),
                    "guess_s": extra, "eigensolves": r.timings["eigensolves"],
                    "fp64_k_builds": int(sum(r.timings["fp64_k_builds"])),
                    "split_k_builds": int(sum(r.timings["split_k_builds"])),
                    "max_abs_energy_error_vs_oracle": float(max(abs(r.energies[i] - e) for i, e in oracle_sub.items()))
                    if oracle_sub else None,
                    "setup_parts_s": r.timings["setup_parts"]}
        return r

    sad_density(mols[0], "def2-SVP", "def2-SVP-JKFIT")  # the atomic SCFs, once, untimed like the model load
    ref = timed("batched_fp64", precision="fp64")
    mix = timed("batched_mixed", precision="mixed")
    # the two guesses, each run twice in the order A B B A so that a drift over
    # the run (cached allocations, host load) falls on both alike; each arm
    # reports the mean of its two runs
    timed("batched_mixed_sad", precision="mixed", sad=True)
    lrn = timed("batched_mixed_learned_guess", precision="mixed", learned=True)
    timed("batched_mixed_learned_guess#2", precision="mixed", learned=True)
    timed("batched_mixed_sad#2", precision="mixed", sad=True)
    for tag in ("batched_mixed_sad", "batched_mixed_learned_guess"):
        a, b = res[tag], res.pop(tag + "#2")
        a["order"] = "sad, learned, learned, sad"
        for key in ("wall_s", "setup_s", "scf_s", "guess_s"):
            a["runs_" + key] = [a[key], b[key]]
            a[key] = 0.5 * (a[key] + b[key])
        a["molecules_per_s"] = nmol / a["wall_s"]
        # the shared hosts slow a whole run now and then (setup and SCF alike);
        # the faster of the two runs is reported beside the mean
        a["molecules_per_s_best_run"] = nmol / min(a["runs_wall_s"])
    e_ref = np.array(ref.energies)
    res["batched_mixed"]["max_abs_energy_error_vs_fp64"] = float(np.max(np.abs(np.array(mix.energies) - e_ref)))
    res["batched_mixed_learned_guess"]["model_load_s_untimed"] = guess_load_s
    res["batched_mixed_learned_guess"]["max_abs_energy_error_vs_fp64"] = float(
        np.max(np.abs(np.array(lrn.energies) - e_ref)))
    from threadpoolctl import threadpool_limits

    sctx = RIJK(device)
    popts = ScfOptions(scf_acc_etot=1e-8, scf_acc_rho=1e-6, scf_acc_eev=1e-6)
    # The plain path's host work (REST's LAPACK generalised eigensolve and DIIS
    # products) is timed at the host BLAS thread count that runs it fastest on
    # this box, chosen on a three-molecule calibration: numpy and scipy each
    # bring an OpenBLAS pool, and at their defaults the pools compete.
    cores = len(os.sched_getaffinity(0))
    cal = {}
    for th in sorted({1, 2, 4, 8, cores}):
        with threadpool_limits(limits=th, user_api="blas"):
            t0 = time.perf_counter()
            for m in mols[:3]:
                SCF(m, "def2-SVP", "def2-SVP-JKFIT", popts, ctx=sctx).run()
            cal[th] = time.perf_counter() - t0
    blas = min(cal, key=cal.get)
    e_plain = []
    with threadpool_limits(limits=blas, user_api="blas"):
        t0 = time.perf_counter()
        for m in mols[:plain_subset]:
            e_plain.append(SCF(m, "def2-SVP", "def2-SVP-JKFIT", popts, ctx=sctx).run().energy)
        wall = time.perf_counter() - t0
        # the same path from REST's SAD guess (atomic densities already cached)
        sopts = ScfOptions(scf_acc_etot=1e-8, scf_acc_rho=1e-6, scf_acc_eev=1e-6, initial_guess="sad")
        t0 = time.perf_counter()
        for m in mols[:plain_subset]:
            SCF(m, "def2-SVP", "def2-SVP-JKFIT", sopts, ctx=sctx).run()
        wall_sad = time.perf_counter() - t0
    sctx.close()
    plain = plain_subset / wall
    plain_sad = plain_subset / wall_sad
    res["plain_fp64_per_molecule"] = {"molecules_per_s": plain, "molecules_timed": plain_subset,
                                      "molecules_per_s_from_sad": plain_sad,
                                      "host_cores": cores, "host_blas_threads": blas,
                                      "blas_calibration_s": {str(k): round(v, 3) for k, v in cal.items()},
                                      "max_abs_energy_error_vs_batched_fp64": float(
                                          np.max(np.abs(np.array(e_plain) - e_ref[:plain_subset])))}
    for tag in ("batched_fp64", "batched_mixed", "batched_mixed_sad", "batched_mixed_learned_guess"):
        res[tag]["speedup_vs_plain_fp64"] = res[tag]["molecules_per_s"] / plain
        res[tag]["speedup_vs_plain_fp64_from_sad"] = res[tag]["molecules_per_s"] / plain_sad
    res["set"] = f"{nmol} water clusters (H2O)_k, k uniform in 1..16 (seeded), def2-SVP / def2-SVP-JKFIT, " \
                 f"RHF to 1e-8 Eh, groups of {group}, device Cholesky metric"
    res["oracle_subset"] = (f"clusters {sorted(oracle_sub)} (k = {[spec[i][0] for i in sorted(oracle_sub)]}): "
                            "FP64 CPU oracle energies converged to 1e-10 Eh, tests/golden/oracle_energies.json")
    res["split_k_builds_note"] = ("the mixed arms run split-precision K only for molecules of at least "
                                  "split_min_basis basis functions; clusters below it take FP64 builds")
    return res


# DRAM traffic of the half-transform per launch.  ncu at n=600, nocc=72 (N=2400,
# one launch over all aux rows, the fused form with remainder columns) measured
# dram read 3.8403 GB +
# write 0.9461 GB = 4.7865 GB, which is 1.036 of the bytes the launch must move:
# the tile-packed tensor rows it reads plus the X rows it writes (ldx x nocc per
# aux row).  The n=1200 tensor (29 GB) is too large to capture under a
# multi-pass ncu run, so its traffic is that ratio times the same byte count for
# the rows of one n=1200 launch.
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_half_transform at n=600, nocc=72 "
                  "(1.036 of tensor rows read + X rows written), scaled to this launch's rows and sizes")


def half_transform_bytes(n: int, nocc: int, rows: float) -> float:
    """Bytes one half-transform launch must move: the tile-packed tensor rows it
    reads and the X rows it writes (ldx x nocc per aux row, no column padding)."""
    nt = -(-n // 32)
    ldb = nt * (nt + 1) // 2 * 1024
    ldx = -(-n // 128) * 128
    return rows * 8.0 * (ldb + ldx * nocc)


TRAFFIC_RATIO_K_HALF = 4.7865e9 / half_transform_bytes(600, 72, 2400)


def traffic_per_launch(kernel: str, w: dict, launches: int):
    if kernel != "k_half":
        return None
    return TRAFFIC_RATIO_K_HALF * half_transform_bytes(w["n"], w["nocc"], w["naux"] / max(1, launches))


def molecule_set_in_child(device: int, nmol: int) -> dict:
    """The molecule-set config (both its batched runs and the plain per-molecule
    comparator) measured in a fresh process, as a job of its own: the stages
    before it in this process leave tens of GB of device allocations and their
    frees behind, which slowed the set's per-context allocations and teardown
    about twofold when it ran here."""
    import subprocess

    import torch

    torch.cuda.empty_cache()  # this process's cached blocks go back to the device for the child
    try:
        out = subprocess.run([sys.executable, os.path.abspath(__file__), "--molecule-set-only", str(nmol),
                              "--device", str(device)], capture_output=True, text=True, timeout=1800)
    except subprocess.TimeoutExpired:
        return {"error": "molecule-set child process timed out after 1800 s"}
    if out.returncode != 0:
        # the headline line still prints; this config reports why it has no numbers
        print(out.stderr[-4000:], file=sys.stderr)
        return {"error": "molecule-set child process failed: " + (out.stderr.strip().splitlines() or ["?"])[-1]}
    res = json.loads(out.stdout.strip().splitlines()[-1])
    res["process"] = "measured in a fresh child process"
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1200, help="num_basis of the sweep workload")
    ap.add_argument("--nocc", type=int, default=0, help="occupied orbitals (default n // 6; for profiling cases)")
    ap.add_argument("--jk", choices=["fused", "separate"], default="fused",
                    help="fused: J and K from one build (rijk_vjk_upper_occ_dev); separate: J by its own two passes")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-split", action="store_true",
                    help="skip the split-precision (tcgen05) measurement and the timing of the other J/K form")
    ap.add_argument("--no-scf", action="store_true", help="skip the water SCF timing")
    ap.add_argument("--no-apps", action="store_true",
                    help="skip the application configs (device tensor build, alkanes, molecule set)")
    ap.add_argument("--set-size", type=int, default=512, help="molecules in the batched water-cluster set")
    ap.add_argument("--molecule-set-only", type=int, default=0, metavar="NMOL",
                    help="measure only the molecule-set config with NMOL molecules and print its JSON")
    ap.add_argument("--device", type=int, default=0, help="device of --molecule-set-only")
    args = ap.parse_args()
    if args.molecule_set_only:
        import torch

        torch.cuda.set_device(args.device)
        print(json.dumps(measure_molecule_set(args.device, args.molecule_set_only)))
        return 0
    w = workload(args.n, args.nocc)
    if args.impl == "reference":
        return run_reference(args, w)
    return run_ours(args, w)


if __name__ == "__main__":
    sys.exit(main())
