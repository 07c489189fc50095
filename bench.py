"""Benchmark: g(k,q,nu) elements/s of the full-band e-ph pass on the config-2 workload.

Workload (synthetic, seeded): nw = 16 electrons on a 9^3 Re grid (729), natom = 4 (12 modes) on a
5^3 Rp grid (125), g(Re,Rp) ~ CN(0,1) exp(-|Re|/2 - |Rp|/1.5), H(R) ~ CN(0,1) exp(-|R|/1.5),
spring-model force constants; 2048 random k x 8192 random q; all bands (no energy window), i.e.
2048 * 8192 * 16 * 16 * 12 = 5.15e10 g elements per pass. One step = one whole pass (both
electron eigensolves, phonons, both Fourier stages, rotations, g2 and its in-place reduction).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--prec mixed|fp64] [--impl epb|reference]

`--workload filter` measures the learned energy-window filter instead (config 4: nw = 32, R grid
11^3, 96^3 k grid, 8192 random q, window E_F -/+ 0.3 eV with E_F the median of band 16): (k, k+q)
pair tests per second over the kept k, with the surrogate pre-filter and without it (the plain
window), whose kept sets must be identical.

`--workload bands` measures config 1 (nw = 8, R grid 7^3, 4096 random k): H(k) by the Fourier sum and
all eigenvalues + eigenvectors, FP64 and mixed (eigenvalue deviation of the mixed path reported).

`--workload bte` measures the SERTA consumer (config 5: the config-2 model on 64^3 k = q grids,
window E_F -/+ 0.3 eV around the median of band 8, T = 300 K, Gaussian 10 meV, method 5):
in-window (k, k+q) pairs per second and the conductivity tensor.

`--workload outerq` measures the batched outer-q loop (run_eph_over_q_and_k) on the config-2 model:
8192 random k x 64 random q, all bands, eigenmode basis, the per-q gauge-invariant record as the only
consumer: g(k,q,nu) elements per second (nk nq nw^2 nm per step), mixed and FP64.

`--workload epw` measures the EPW e-ph matrix reader: a config-2-size `<prefix>.epmatwp` (4.48 GB, EPW
order, shuffled R lists, per-orbital Wigner-Seitz degeneracies) streamed from the page cache into HBM in
the "el" layout: file bytes per second.

`--workload eigh` measures the uneven batched eigensolve (config 3: 1,000,000 Hermitian matrices,
n uniform in {4, 8, ..., 96}, 5 % with planted 2-4-fold clusters spaced 1e-10, eigenvalues and
eigenvectors, FP32 solve + FP64 refinement): matrices per second.

Multi-GPU: one process per GPU (torchrun); every rank runs its own full pass on its own k set
(weak scaling, no data-path collective); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "electronphonon.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "g(k,q,ν) elems/s, nw=16: mixed-prec+filter vs FP64 plain, |g|² rel err≤1e-5"
UNIT = "elements/s"
NW, NATOM, N_EL, N_PH = 16, 4, 4, 2
NK, NQ = 2048, 8192
SEED = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="epb", choices=["epb", "reference"])
    ap.add_argument("--prec", default="auto", choices=["auto", "mixed", "fp64"])
    ap.add_argument("--nk", type=int, default=NK)
    ap.add_argument("--nq", type=int, default=NQ)
    ap.add_argument("--k-batch", type=int, default=0, help="inner k batch of the pass; 0 = autotuned")
    ap.add_argument("--tune-table", default=None,
                    help="pass workload: load the autotuner's choices from this text table (skips the timing trials)")
    ap.add_argument("--save-tune", default=None, help="pass workload: write the autotuner's choices to this file")
    ap.add_argument("--sample-stride", type=int, default=4096)
    ap.add_argument("--err-stride", type=int, default=512,
                    help="pass workload: q stride of the blocks compared against the FP64 pass (untimed runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="pass workload: skip the FP64 plain-pass denominator")
    ap.add_argument("--fp64-steps", type=int, default=1, help="pass workload: timed FP64 plain passes")
    ap.add_argument("--cpu-nk", type=int, default=16)
    ap.add_argument("--cpu-nq", type=int, default=1024)
    ap.add_argument("--workload", default="pass", choices=["pass", "filter", "eigh", "bands", "bte", "outerq", "epw"])
    ap.add_argument("--count", type=int, default=1_000_000, help="eigh workload: matrices per batch")
    ap.add_argument("--grid", type=int, default=96, help="filter workload: k grid per axis")
    ap.add_argument("--decay", type=float, default=1.5, help="filter workload: H(R) decay length")
    ap.add_argument("--epochs", type=int, default=200, help="filter workload: surrogate training epochs")
    ap.add_argument("--small", action="store_true",
                    help="profiling case: Re grid 5^3, 32 k x 2048 q (a few GB on the device)")
    a = ap.parse_args()
    if a.small:
        global N_EL
        N_EL = 2
        a.nk, a.nq = 32, 2048
    return a


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def build_model_host_small():
    """Host model without epmat (H and D only); the 4.5 GB epmat is generated on the device."""
    from epb200 import synth

    return synth.config2_model(seed=SEED, with_epmat=False, n_el=N_EL)


def config_dict(args, prec_name):
    return {"workload": f"config2 full-band e-ph pass: nw={NW}, natom={NATOM} (nm={3 * NATOM}), "
                        f"Re {2 * N_EL + 1}^3, Rp {2 * N_PH + 1}^3, {args.nk} random k x {args.nq} random q",
            "nk": args.nk, "nq": args.nq, "nw": NW, "nmodes": 3 * NATOM, "nr_el": (2 * N_EL + 1) ** 3,
            "nr_ep": (2 * N_PH + 1) ** 3, "window": "all bands", "filter": "none in the timed step: config 2 states no energy window, so both paths "
            "keep every (k, q) pair and band (identical kept sets); the learned window filter is timed by "
            "--workload filter on config 4", "precision": prec_name,
            "k_batch": args.k_batch if args.k_batch > 0 else "autotuned",
            "l2": "inputs larger than L2 (g(Re,Rp) is 4.48 GB and is re-read every pass)",
            "parallelism": f"dp{args.gpus} (k sharded per rank, weak)"}


# ---------------------------------------------------------------------------------------------
def clocks_start():
    try:
        # raw samples go to the file named by EPB_CLOCKS_CSV (if set); the JSON line carries the summary
        f = open(os.environ.get("EPB_CLOCKS_CSV") or os.devnull, "w")
        p = subprocess.Popen(["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                              "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        return (p, f)
    except Exception:
        return None


def clocks_stop(h, device_index):
    if h is None:
        return None
    p, f = h
    p.terminate()
    try:
        out, _ = p.communicate(timeout=5)
    except Exception:
        p.kill()
        out = ""
    f.write(out)
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9 or parts[0] != str(device_index):
            continue
        try:
            sm.append(float(parts[1]))
            mx = float(parts[2])
        except ValueError:
            continue
        for n, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d, "measured (MEASURED_PEAKS.json)"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def measure_fp64_peak(torch):
    """cuBLAS DGEMM 8192^3 throughput (TFLOP/s), the FP64 denominator (no FP64 figure is provided)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e9
    for _ in range(3):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def measure_fp32_simt_peak(torch):
    """FP32 CUDA-core throughput (TFLOP/s): cuBLAS SGEMM 8192^3 with TF32 disabled (FFMA path)."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
        b = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
        for _ in range(2):
            a @ b
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e9
        for _ in range(3):
            e0.record()
            a @ b
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


# Algorithmic HBM bytes and flops per launch of the families of the mixed pass (one launch covers one
# inner batch of nkb k x nq q, i.e. nkb * nq matrices / pairs):
#   eigh (FP32 Jacobi): packed FP32 H (nw^2 floats) in, FP32 eigenvectors (nw^2 complex64) out;
#       40 n^3 real flops per Hermitian eigensolve with vectors (the algorithmic count of the e-ph
#       pass's work table; a Jacobi solve executes several times that);
#   eigh_refine: H (nw^2 floats) + FP32 vectors in, FP32 vectors out; FP64 work;
#   rotation: g(k,q) block (2 nw^2 nm floats) + U (nw^2 complex64) in; 8 (nw^3 nm + nw^2 nm^2) flops.
def family_bytes_flops(name, args, nkb):
    nw2, nm = NW * NW, 3 * NATOM
    units = nkb * args.nq
    if name == "eigh":
        return units * (4 * nw2 + 8 * nw2), units * 40.0 * NW ** 3
    if name == "eigh_refine":
        return units * (4 * nw2 + 8 * nw2 + 8 * nw2), None
    if name == "rotation":
        return units * (8 * nw2 * nm + 8 * nw2), units * 8.0 * (NW ** 3 * nm + nw2 * nm * nm)
    return None, None


# Algorithmic flops per launch of each kernel family (8 real flops per complex MAC).
def family_flops(name, args, nkb):
    nw2, nm, nr_el, nr_ep = NW * NW, 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3
    if name == "zgemm":      # kR->kq for one k: (nw^2 nm) x nr_ep x nq
        return 8.0 * nw2 * nm * nr_ep * args.nq
    if name == "umma_kq":    # kR->kq for a k batch
        return 8.0 * nw2 * nm * nr_ep * args.nq * nkb
    if name == "umma_rr":    # RR->kR for 256 k: (nw^2 nm nr_ep) x nr_el x 256
        return 8.0 * nw2 * nm * nr_ep * nr_el * min(256, args.nk)
    if name in ("fourier_f64", "umma_h"):  # dominated by H(k+q): nw^2 x nr_el per k+q point
        return 8.0 * nw2 * nr_el * args.nq * nkb
    return None


def run_epb(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    from epb200 import pipeline, synth
    from epb200 import _lib

    prec = {"auto": None, "mixed": pipeline.PREC_MIXED, "fp64": pipeline.PREC_FP64}[args.prec]
    m = build_model_host_small()
    ep_dev = synth.epmat_el_device(SEED, NW, 3 * NATOM, m.el_ham.irvec, synth.irvec_box(N_PH))
    m.epmat = synth.device_epmat_object(ep_dev, m.el_ham.irvec, synth.irvec_box(N_PH))
    want_mixed = prec in (None, pipeline.PREC_MIXED)
    try:
        dm = pipeline.DeviceModel(m, mixed=want_mixed)
    except _lib.EpbError:
        if prec == pipeline.PREC_MIXED:
            raise
        dm = pipeline.DeviceModel(m, mixed=False)
        want_mixed = False
    if prec is None:
        prec = pipeline.PREC_MIXED if want_mixed else pipeline.PREC_FP64
    prec_name = ("mixed (tcgen05: FP16x2 kR->kq, split-BF16x3 RR->kR and H(k+q); rotation on the warp tensor cores "
                 "(FP16x2, FP32 accumulate) or in FP32, autotuned; FP32 Jacobi + FP64 refinement)") if prec == pipeline.PREC_MIXED else "fp64"
    xks = synth.random_kpoints(args.nk, 1000 + rank)
    xqs = synth.random_kpoints(args.nq, 2000)
    from epb200.batched import jl

    xk_d, xq_d = jl(xks), jl(xqs)
    ctx = dm.ctx
    if args.tune_table:
        with open(args.tune_table) as f:
            _lib.TuneTable(f.read()).import_into(ctx)
    ctx.set_graph_mode(True)  # repeated passes on the same buffers replay one captured CUDA graph
    run = lambda: pipeline.run_eph_over_k_and_q(dm, xk_d, xq_d, prec=prec, k_batch=args.k_batch,
                                                sample_stride=args.sample_stride, out=out_holder[0])
    out_holder = [None]
    out_holder[0] = run()
    for _ in range(max(args.warmup - 1, 0)):
        run()
    torch.cuda.synchronize()
    # ---- device-timed region ----
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = clocks_start()
    launches0 = ctx.launch_count()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        run()
    e1.record(s)
    torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    clocks = clocks_stop(clk, local)
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    n_el = out_holder[0].n_elements
    value = ws * n_el / (ms * 1e-3)

    # ---- per-kernel profile of one extra pass (not part of the timed region) ----
    ctx.profile(True)
    run()
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    peaks, peak_src = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_cnt) = dom
    kb_used = out_holder[0].k_batch or args.k_batch
    flops = family_flops(dom_name, args, kb_used)
    tot_ms = sum(v[0] for v in prof.values())
    profile = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / tot_ms, 4)}
               for k, v in prof.items() if v[1]}
    roof = None
    roof_compute = None
    if flops is None and dom_cnt > 0:
        # a CUDA-core family dominates: HBM roofline from its algorithmic bytes (the schema's bounds are
        # HBM or tensor), plus its FP32 compute roofline against a live FFMA (SGEMM) measurement
        nbytes, nflops = family_bytes_flops(dom_name, args, kb_used)
        if nbytes is not None:
            avg_s = dom_ms / dom_cnt * 1e-3
            ach = nbytes / avg_s / 1e9
            traffic = None
            tp = os.path.join(ROOT, "profiles", "traffic.json")
            if os.path.exists(tp):
                with open(tp) as fh:
                    tr = json.load(fh).get(dom_name)
                if isinstance(tr, dict):  # measured bytes per unit x the units of one launch
                    traffic = int(tr["bytes_per_unit"] * kb_used * args.nq)
            roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 2), "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": round(ach / peaks["hbm_gbs"], 5), "traffic": traffic,
                    "peak_source": f"{peak_src} hbm copy", "launch_ms": round(dom_ms / dom_cnt, 4),
                    "launches_per_pass": dom_cnt, "algorithmic_bytes_per_launch": nbytes,
                    "note": "the family is FP32 CUDA-core compute bound; see roofline_compute",
                    "share_of_pass": {k: round(v[0] / tot_ms, 4) for k, v in prof.items() if v[1]}}
            if nflops is not None:
                p32 = measure_fp32_simt_peak(torch)
                a32 = nflops / avg_s / 1e12
                roof_compute = {"bound": "fp32 cuda cores", "kernel": dom_name, "achieved": round(a32, 2),
                                "peak": round(p32, 2), "unit": "TFLOP/s", "frac": round(a32 / p32, 4),
                                "peak_source": "measured live: cuBLAS SGEMM 8192^3, TF32 off",
                                "algorithmic_flops_per_launch": nflops}
    if flops is not None and dom_cnt > 0:
        avg_s = dom_ms / dom_cnt * 1e-3
        if dom_name.startswith("umma"):
            # split BF16x3: six products per real MAC; the pass's kR->kq runs FP16x2 (three products)
            nprod = 3 if dom_name == "umma_kq" else 6
            peak = peaks["bf16_tflops_sustained"] / nprod
            psrc = f"{peak_src} bf16 (= fp16) sustained / {nprod} split products"
        else:
            peak = measure_fp64_peak(torch)
            psrc = "measured live: cuBLAS DGEMM 8192^3 (no FP64 figure in MEASURED_PEAKS.json)"
        ach = flops / avg_s / 1e12
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            with open(tp) as fh:
                tr = json.load(fh).get(dom_name)
            if isinstance(tr, dict):  # measured bytes per unit x the units of one launch
                traffic = int(tr["bytes_per_unit"] * kb_used * args.nq)
        roof = {"bound": "tensor", "kernel": dom_name, "achieved": round(ach, 3), "peak": round(peak, 2),
                "unit": "TFLOP/s", "frac": round(ach / peak, 4), "traffic": traffic, "peak_source": psrc,
                "launch_ms": round(dom_ms / dom_cnt, 4), "launches_per_pass": dom_cnt,
                "algorithmic_flops_per_launch": flops,
                "share_of_pass": {k: round(v[0] / sum(x[0] for x in prof.values()), 4) for k, v in prof.items() if v[1]}}

    # ---- whole-pass roofline: the pass's algorithmic work (8 real flops per complex MAC, per (k, q) pair:
    # kR->kq 8 nw^2 nm nr_ep, H(k+q) 8 nw^2 nr_el, rotations 8 (nw^3 nm + nw^2 nm^2), RR->kR amortised over
    # the q list 8 nw^2 nm nr_ep nr_el / nq, eigensolve 40 nw^3) against the tensor cores' split-product rate
    nw2, nm_, nr_el, nr_ep = NW * NW, 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3
    per_pair = 8.0 * (nw2 * nm_ * nr_ep + nw2 * nr_el + NW ** 3 * nm_ + nw2 * nm_ * nm_ +
                      nw2 * nm_ * nr_ep * nr_el / args.nq) + 40.0 * NW ** 3
    pass_flops = per_pair * args.nk * args.nq
    pass_tf = pass_flops / (ms * 1e-3) / 1e12
    roof_pass = {"bound": "tensor", "achieved": round(pass_tf, 2), "unit": "TFLOP/s",
                 "peak": round(peaks["bf16_tflops_sustained"] / 3, 2),
                 "frac": round(pass_tf / (peaks["bf16_tflops_sustained"] / 3), 4),
                 "algorithmic_flops_per_pass": pass_flops, "per_pair": per_pair,
                 "peak_source": f"{peak_src} bf16 (= fp16) sustained / 3 split products",
                 "note": "whole pass (both eigensolves, phonons, both Fourier stages, rotations) at the device-timed step"}

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        xk_h = torch.from_numpy(np.ascontiguousarray(xks.T)).pin_memory()
        xq_h = torch.from_numpy(np.ascontiguousarray(xqs.T)).pin_memory()
        r0 = out_holder[0]
        outs = [r0.ek, r0.omega, r0.g2sum] + ([r0.g2_sample] if r0.g2_sample is not None else [])
        host_outs = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in outs]
        bi = xk_h.numel() * 8 + xq_h.numel() * 8
        bo = sum(o.numel() * o.element_size() for o in outs)
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(args.steps):
            # host k / q lists into the pass's device buffers (the graph replays on the same buffers)
            xk_d.copy_(xk_h, non_blocking=True)
            xq_d.copy_(xq_h, non_blocking=True)
            r = pipeline.run_eph_over_k_and_q(dm, xk_d, xq_d, prec=prec, k_batch=args.k_batch,
                                              sample_stride=args.sample_stride, out=r0)
            for ho, o in zip(host_outs, outs):
                ho.copy_(o, non_blocking=True)
        e1.record(s)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1) / args.steps
        if ws > 1:
            t = torch.tensor([ms_e2e], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms_e2e = float(t.item())
        e2e = {"value": ws * n_el / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": bi,
               "d2h_bytes_per_step": bo, "ms_per_step": round(ms_e2e, 3)}

    # ---- the metric's denominator: this project's plain FP64 GPU pass on the same k, q (and the error) ----
    fp64 = None
    if prec == pipeline.PREC_MIXED and not args.no_fp64:
        fp64 = fp64_denominator(args, torch, pipeline, dm, xk_d, xq_d, out_holder[0], ws, n_el, value)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, m_host_for_cpu(m, ep_dev), xks, xqs)

    mixed = prec == pipeline.PREC_MIXED
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": fp64["ratio"] if fp64 else None,
            "vs_baseline_note": ("value / this project's plain FP64 GPU pass on the same k and q lists, measured "
                                 "in this run (the metric's own denominator; no published number exists)")
            if fp64 else None,
            "fp64_plain": fp64,
            "dtype": ("fp16x2 (kR->kq, 3 products) + bf16x3 (RR->kR, H(k+q), 6 products) on tcgen05, f32 "
                      "accumulate; fp16x2 rotation on mma.sync (f32 accumulate); f32 Jacobi, f64 refinement and "
                      "k, q sides") if mixed else "f64",
            "data": "synthetic (seeded generator; random-init Wannier model of the config-2 shape)",
            "config": dict(config_dict(args, prec_name), k_batch_used=kb_used,
                           autotuned={"k_batch": kb_used, "rotation": {0: "warp tensor cores (mma.sync)",
                                                                      1: "FP32 CUDA cores"}.get(out_holder[0].rot_variant, "fp64"),
                                      "kq_gemm": {1: "A-resident tcgen05", 0: "streamed tcgen05"}.get(
                                          out_holder[0].kq_form, "fp64"),
                                      "table": dm.ctx.tune_text(),
                                      "source": "loaded table" if args.tune_table else "timed in the first warm-up pass"}),
            "roofline": roof,
            "roofline_compute": roof_compute, "roofline_pass": roof_pass,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "impl": "epb", "profile_one_pass": profile}
    if rank == 0:
        print(json.dumps(line), flush=True)
        if args.save_tune:
            with open(args.save_tune, "w") as f:
                f.write(dm.ctx.tune_text())
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def fp64_denominator(args, torch, pipeline, dm, xk_d, xq_d, r_mixed, ws, n_el, value):
    """Time the plain FP64 GPU pass (FP64 Fourier sums, FP64 Jacobi, FP64 rotations) on the same k and q
    lists and compare the results of both passes on a denser sample (every err_stride-th q, untimed runs):
    the sampled |g|^2 blocks (normwise per (k, q) block with its tail, and elementwise above floors of the
    block maximum), the mode sums g2sum[nu, k] and the energies."""
    ctx = dm.ctx
    ctx.set_graph_mode(False)
    s = torch.cuda.current_stream()
    run64 = lambda o: pipeline.run_eph_over_k_and_q(dm, xk_d, xq_d, prec=pipeline.PREC_FP64, k_batch=16,
                                                    sample_stride=args.sample_stride, out=o)
    ctx.profile(True)
    # untimed: sizes the FP64 workspace, gives the per-family profile of the line and the FP64 side of the
    # accuracy comparison, sampled every err_stride-th q (denser than the timed runs' samples)
    r64e = pipeline.run_eph_over_k_and_q(dm, xk_d, xq_d, prec=pipeline.PREC_FP64, k_batch=16,
                                         sample_stride=args.err_stride)
    torch.cuda.synchronize()
    prof64 = {k: round(v[0], 1) for k, v in ctx.profile_read(reset=True).items() if v[1]}
    ctx.profile(False)
    rme = pipeline.run_eph_over_k_and_q(dm, xk_d, xq_d, prec=pipeline.PREC_MIXED, k_batch=r_mixed.k_batch,
                                        sample_stride=args.err_stride)
    r64 = run64(None)
    if ws > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.fp64_steps):
        run64(r64)
    e1.record(s)
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1) / args.fp64_steps
    if ws > 1:
        t = torch.tensor([ms64], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms64 = float(t.item())
    v64 = ws * n_el / (ms64 * 1e-3)
    err = {}
    if rme.g2_sample is not None:
        # Julia (nw, nw, nm, nsamp, nk) arrays are torch tensors of shape (nk, nsamp, nm, nw, nw): one (k, q)
        # block per row after flattening the first two axes
        a, b = rme.g2_sample, r64e.g2_sample
        nblk = a.shape[0] * a.shape[1]
        d = (a - b).reshape(nblk, -1)
        bb = b.reshape(nblk, -1)
        blk = torch.linalg.vector_norm(d, dim=1) / torch.linalg.vector_norm(bb, dim=1)
        bmax = bb.abs().amax(dim=1, keepdim=True)
        srt = torch.sort(blk).values
        worst = int(blk.argmax())
        err = {"g2_block_normwise_max": float(blk.max()), "g2_block_normwise_median": float(blk.median()),
               "g2_block_normwise_p99": float(srt[int(0.99 * (srt.numel() - 1))]),
               "g2_block_normwise_p999": float(srt[int(0.999 * (srt.numel() - 1))]),
               "blocks_above_1e-5": int((blk > 1e-5).sum()), "blocks_compared": int(blk.numel()),
               "sample_q_stride": args.err_stride,
               "worst_block_k_q": [worst // a.shape[1], (worst % a.shape[1]) * args.err_stride]}
        # elementwise relative error of the entries above a floor (fraction of their block's largest entry);
        # an entry at the floor f carries the block's absolute error / f, so the figure grows as f falls
        for f in (1e-6, 1e-4, 1e-2):
            big = bb.abs() > f * bmax
            elem = torch.where(big, d.abs() / torch.where(big, bb.abs(), torch.ones_like(bb)), torch.zeros_like(bb))
            err[f"g2_elementwise_max_above_{f:g}_floor"] = float(elem.max())
        err["g2_abs_err_max_over_block_max"] = float((d.abs().amax(dim=1, keepdim=True) / bmax).max())
    err["g2sum_rel_max"] = float(((rme.g2sum - r64e.g2sum).abs() / r64e.g2sum.abs()).max())
    err["ek_abs_max_ry"] = float((rme.ek - r64e.ek).abs().max())
    err["omega_abs_max_ry"] = float((rme.omega - r64e.omega).abs().max())
    del rme, r64e
    ctx.set_graph_mode(True)
    # the denominator's own roofline: the pass's algorithmic flops (same count as the mixed pass) against a
    # live cuBLAS DGEMM; its GEMMs are cuBLAS ZGEMMs (csrc/epb_f64blas.cu), as in the reference's GPU path
    nw2, nm_, nr_el, nr_ep = NW * NW, 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3
    per_pair = 8.0 * (nw2 * nm_ * nr_ep + nw2 * nr_el + NW ** 3 * nm_ + nw2 * nm_ * nm_ +
                      nw2 * nm_ * nr_ep * nr_el / args.nq) + 40.0 * NW ** 3
    tf64 = per_pair * args.nk * args.nq / (ms64 * 1e-3) / 1e12
    p64 = measure_fp64_peak(torch)
    return {"value": v64, "unit": UNIT, "ms_per_step": round(ms64, 1), "steps": args.fp64_steps,
            "ratio": value / v64, "target_ratio": 3.0, "error_vs_fp64": err, "error_bar": 1e-5,
            "kept_set": "identical by construction (all bands, every (k, q) pair in both paths)",
            "roofline": {"bound": "fp64", "achieved": round(tf64, 2), "peak": round(p64, 2), "unit": "TFLOP/s",
                         "frac": round(tf64 / p64, 4), "peak_source": "measured live: cuBLAS DGEMM 8192^3",
                         "note": "whole FP64 pass: H(k+q) Fourier, kR->kq and both rotations as cuBLAS ZGEMMs (the "
                                 "reference's GPU path), FP64 Jacobi eigensolves of this project"},
            "profile_ms": prof64}


def m_host_for_cpu(m, ep_dev):
    """Host copy of the model (the device-generated epmat copied back) for the CPU port."""
    from epb200 import synth
    from epb200.wannier import WannierObject

    op = ep_dev.cpu().numpy().T  # Fortran-ordered (ndata, nr_el)
    mm = synth.SynthModel(m.nw, m.nmodes, m.mass, m.el_ham, m.ph_dyn,
                          WannierObject(m.el_ham.irvec, op, irvec_next=synth.irvec_box(N_PH)), m.seed)
    return mm


def cpu_baseline(args, model, xks, xqs):
    """CPU port of the reference's batched path (oracle/cpu_pass.py) on a bounded sample."""
    from oracle import cpu_pass

    nk, nq = min(args.cpu_nk, xks.shape[1]), min(args.cpu_nq, xqs.shape[1])
    xk, xq = np.asfortranarray(xks[:, :nk]), np.asfortranarray(xqs[:, :nq])
    t0 = time.perf_counter()
    r = cpu_pass.eph_pass_cpu(model, xk, xq)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
    return {"value": r["n_elements"] / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{nk} k x {nq} q of the same model (all bands), {dt:.1f} s; numpy/scipy OpenBLAS "
                      f"ZGEMM + LAPACK ZHEEV per matrix"}


def run_reference(args):
    """Reference arm: the reference's CPU batched path restated (the Julia reference cannot run here)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from epb200 import synth
    from oracle import cpu_pass

    m = synth.config2_model(seed=SEED)
    xks = synth.random_kpoints(args.nk, 1000)
    xqs = synth.random_kpoints(args.nq, 2000)
    nk, nq = min(args.cpu_nk, args.nk), min(args.cpu_nq, args.nq)
    xk, xq = np.asfortranarray(xks[:, :nk]), np.asfortranarray(xqs[:, :nq])
    for _ in range(args.warmup):
        cpu_pass.eph_pass_cpu(m, xk[:, :1], xq[:, :64])
    t0 = time.perf_counter()
    n = 0
    for _ in range(args.steps):
        r = cpu_pass.eph_pass_cpu(m, xk, xq)
        n += r["n_elements"]
    dt = time.perf_counter() - t0
    v = n / dt
    cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": config_dict(args, "fp64 (CPU)"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{nk} k x {nq} q per step of the config-2 model, all bands"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
FILTER_METRIC = "(k, k+q) pair window tests/s, nw=32 learned filter (kept set identical to the plain filter)"
FILTER_UNIT = "pairs/s"


def filter_setup(args, torch):
    """Config-4 model, E_F, kept k, trained + calibrated surrogate (untimed setup)."""
    from epb200 import learned, synth
    from epb200.wannier import WannierObject

    rng = np.random.default_rng(4)
    irvec = synth.irvec_box(5)
    ham = WannierObject(irvec, synth.hermitian_op_r(rng, 32, irvec, args.decay))
    bm = learned.BandModel(ham)
    xk_grid = synth.grid_kpoints((args.grid,) * 3)
    xqs = synth.random_kpoints(args.nq, 4000)
    t0 = time.perf_counter()
    ef = float(torch.median(bm.band_energy(xk_grid, 16)).item())
    half = 0.3 * synth.UNIT_EV
    wmin, wmax = ef - half, ef + half
    _, _, kkeep, kst = bm.window(xk_grid, wmin, wmax, prec=learned.PREC_MIXED)
    from epb200.batched import jl

    xk_kept = jl(xk_grid).index_select(0, kkeep.long()).contiguous()
    t_grid = time.perf_counter() - t0
    t0 = time.perf_counter()
    r2 = np.random.default_rng(44)
    xt, xh = r2.random((3, 1 << 15)), r2.random((3, 1 << 16))
    Et, Eh = bm.eigvals(xt), bm.eigvals(xh)
    mlp = learned.Surrogate(nf=128, hidden=256, nhidden=3, nout=32, seed=45)
    loss = mlp.train(xt, Et, epochs=args.epochs, batch=2048, lr=2e-3, lr_final=2e-5)
    margin = mlp.calibrate(xh, Eh)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    info = {"e_fermi_ry": ef, "window_ry": [wmin, wmax], "k_grid": args.grid ** 3, "k_kept": int(kkeep.numel()),
            "k_window_stats": kst, "train_points": 1 << 15, "train_energies": 32 << 15, "holdout_points": 1 << 16,
            "margin_safety": 1.5,
            "train_loss_first_last": [float(loss[0]), float(loss[-1])], "margin_ry_max": float(margin.max()),
            "margin_ry_mean": float(margin.mean()), "setup_s": {"grid": round(t_grid, 2), "surrogate": round(t_train, 2)}}
    return bm, mlp, xk_kept, xqs, wmin, wmax, info


def run_filter(args):
    import torch

    from epb200 import learned
    from epb200.batched import jl

    torch.cuda.set_device(0)
    bm, mlp, xk_kept, xqs, wmin, wmax, info = filter_setup(args, torch)
    xq_d = jl(xqs)
    ctx = bm.ctx
    nk = xk_kept.shape[0]
    npairs = nk * args.nq
    cap = max(npairs // 4, 1 << 20)

    def step(use_mlp):
        return learned.pair_window(bm, xk_kept, xq_d, wmin, wmax, mlp=mlp if use_mlp else None,
                                   prec=learned.PREC_MIXED, capacity=cap)

    res = {}
    for use_mlp in (True, False):
        for _ in range(args.warmup):
            out = step(use_mlp)
        torch.cuda.synchronize()
        clk = clocks_start() if use_mlp else None
        l0 = ctx.launch_count()
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            out = step(use_mlp)
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res[use_mlp] = {"ms": ms, "out": out, "launches": ctx.launch_count() - l0,
                        "clocks": clocks_stop(clk, 0) if use_mlp else None}
    a, b = res[True]["out"], res[False]["out"]
    identical = bool(torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and torch.equal(a[2], b[2]))
    # per-family profile of one learned step
    ctx.profile(True)
    step(True)
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    tot = sum(v[0] for v in prof.values())
    profile = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / tot, 4)} for k, v in prof.items() if v[1]}
    st = a[3]
    peaks, psrc = measured_peaks()
    roof = None
    dom_name, (dom_ms, dom_cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    if dom_name == "umma_h" and dom_cnt:
        # H(x) of every plainly evaluated point: 1024 x 1331 complex MACs, 8 flops each
        flops = 8.0 * 1024 * 1331 * st["evaluated"]
        ach = flops / (dom_ms * 1e-3) / 1e12
        peak = peaks["bf16_tflops_sustained"] / 6
        roof = {"bound": "tensor", "kernel": dom_name, "achieved": round(ach, 3), "peak": round(peak, 2),
                "unit": "TFLOP/s", "frac": round(ach / peak, 4), "traffic": None,
                "peak_source": f"{psrc} bf16 sustained / 6 split products"}
    # end to end: host k / q lists in, kept pairs out
    xk_h = xk_kept.cpu().pin_memory()
    xq_h = xq_d.cpu().pin_memory()
    kept = a[0].numel()
    ho = [torch.empty(kept, dtype=torch.int64).pin_memory(), torch.empty(kept, dtype=torch.int32).pin_memory(),
          torch.empty(kept, dtype=torch.int32).pin_memory()]
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        xk_dd = xk_h.to("cuda", non_blocking=True)
        xq_dd = xq_h.to("cuda", non_blocking=True)
        o = learned.pair_window(bm, xk_dd, xq_dd, wmin, wmax, mlp=mlp, prec=learned.PREC_MIXED, capacity=cap)
        for h, d in zip(ho, o[:3]):
            h.copy_(d, non_blocking=True)
    e1.record(s)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / args.steps
    cpu = None
    if not args.no_cpu:
        from oracle import mlp_oracle as M

        xk_s = xk_kept[:2].cpu().numpy().T.copy(order="F")
        xq_s = xqs[:, :256]
        t0 = time.perf_counter()
        M.pair_window(bm.ham_host_op, 32, bm.ham.irvec, xk_s, xq_s, wmin, wmax)
        dt = time.perf_counter() - t0
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": 2 * 256 / dt, "unit": FILTER_UNIT, "cores": cores, "kind": "port",
               "sample": f"2 kept k x 256 q: FP64 Fourier (GEMM) + LAPACK ZHEEV + searchsorted, {dt:.1f} s"}
    ms = res[True]["ms"]
    line = {"metric": FILTER_METRIC, "value": npairs / (ms * 1e-3), "unit": FILTER_UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3/f32/f64 (window), f32 (surrogate)",
            "data": f"synthetic (seeded; H(R) ~ CN(0,1) exp(-|R|/{args.decay}))",
            "config": {"workload": f"config4 learned window filter: nw=32, R 11^3, {args.grid}^3 k grid, {args.nq} random q, "
                                   "window E_F -/+ 0.3 eV, E_F = median of band 16",
                       "pairs_per_step": npairs, "l2": "inputs larger than L2 (phase planes and H planes per chunk)",
                       **info},
            "plain_ms_per_step": round(res[False]["ms"], 3), "plain_value": npairs / (res[False]["ms"] * 1e-3),
            "learned_speedup_vs_plain": round(res[False]["ms"] / ms, 3), "kept_sets_identical": identical,
            "window_stats": st, "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": npairs / (ms_e2e * 1e-3), "unit": FILTER_UNIT,
                    "h2d_bytes_per_step": xk_h.numel() * 8 + xq_h.numel() * 8,
                    "d2h_bytes_per_step": kept * 16, "ms_per_step": round(ms_e2e, 3)},
            "gpu_launches": res[True]["launches"] // args.steps * args.steps, "clocks": res[True]["clocks"],
            "impl": "epb", "profile_one_step": profile}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
BTE_METRIC = "SERTA in-window (k, k+q) pairs/s, config-2 model on 64^3 k = q grids (sigma vs FP64)"


def run_bte(args):
    import torch

    from epb200 import bte, pipeline, synth
    from oracle import bte_oracle as BO
    from oracle import epb_oracle as O

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:  # one process per GPU: each rank takes a contiguous share of the kept k (weak in the grid)
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    ng = args.grid if args.grid != 96 else 64
    m = build_model_host_small()
    ep_dev = synth.epmat_el_device(SEED, NW, 3 * NATOM, m.el_ham.irvec, synth.irvec_box(N_PH))
    m.epmat = synth.device_epmat_object(ep_dev, m.el_ham.irvec, synth.irvec_box(N_PH))
    dm = pipeline.DeviceModel(m, mixed=True)
    # E_F = median of band 8 over the grid (host, from the grid energies of a coarse sample of the grid)
    xs, _ = BO.grid_points(16)
    hk = O.fourier_batched(m.el_ham.op_r, NW * NW, m.el_ham.irvec, xs)
    Es = O.eigvals_batched(np.asfortranarray(hk.reshape(NW, NW, -1, order="F")))
    ef = float(np.median(Es[NW // 2 - 1]))
    half = 0.3 * synth.UNIT_EV
    T, eta = 300 * O.UNIT_K, 0.01 * synth.UNIT_EV
    kw = dict(method=5, k_batch=args.k_batch if args.k_batch > 0 else 128,
              prec=pipeline.PREC_MIXED if args.prec != "fp64" else pipeline.PREC_FP64,
              shard=(rank, ws) if ws > 1 else None)
    for _ in range(args.warmup):
        sig, st, _ = bte.serta(dm, ng, ef - half, ef + half, ef, T, eta, **kw)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clk = clocks_start()
    l0 = dm.ctx.launch_count()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        sig, st, _ = bte.serta(dm, ng, ef - half, ef + half, ef, T, eta, **kw)
    e1.record(s)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = clocks_stop(clk, local)
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        from epb200 import shard

        ms = shard.max_over_ranks(ms, device="cuda")
    launches = dm.ctx.launch_count() - l0
    st_rank = dict(st)  # this rank's shard: the per-launch roofline below is per GPU
    sig, st = bte.reduce_shards(sig, st)
    dm.ctx.profile(True)
    bte.serta(dm, ng, ef - half, ef + half, ef, T, eta, **kw)
    torch.cuda.synchronize()
    prof = dm.ctx.profile_read(reset=True)
    dm.ctx.profile(False)
    profile = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in prof.items() if v[1]}
    # the FP64 plain path on the same inputs: time and conductivity for the comparison
    kw64 = dict(kw, prec=pipeline.PREC_FP64)
    e0.record(s)
    sig64, st64, _ = bte.serta(dm, ng, ef - half, ef + half, ef, T, eta, **kw64)
    e1.record(s)
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1)
    if ws > 1:
        ms64 = shard.max_over_ranks(ms64, device="cuda")
    sig64, st64 = bte.reduce_shards(sig64, st64)
    rel = float(np.max(np.abs(sig - sig64)) / np.abs(sig64).max())
    # roofline of the dominant family (total algorithmic flops of one step / its total device time)
    peaks, peak_src = measured_peaks()
    tot = sum(v[0] for v in prof.values())
    for k in profile:
        profile[k]["share"] = round(profile[k]["ms"] / tot, 4)
    dom_name, (dom_ms, dom_cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    nm, nr_el, nr_ep = 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3
    W = max(int(st["width"]), 1)
    roof = None
    if dom_name == "umma_kq":   # grouped kR->kq of the kept k's pairs, split BF16x3
        flops = 8.0 * NW * W * nm * nr_ep * st_rank["pairs"]
        peak, psrc = peaks["bf16_tflops_sustained"] / 6, f"{peak_src} bf16 sustained / 6 split products"
    elif dom_name == "rotation":  # fused rotation + accumulation: HBM-bound on its per-pair operands
        flops = None
        nb = st_rank["pairs"] * (8 * NW * W * nm + 16 * nm * nm + 16 * NW * W + 8 * nm + 12)
        ach = nb / (dom_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 2), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(ach / peaks["hbm_gbs"], 4), "traffic": None,
                "peak_source": f"{peak_src} hbm copy", "launch_ms": round(dom_ms / dom_cnt, 4),
                "launches_per_step": dom_cnt, "algorithmic_bytes_per_step": nb,
                "note": "per pair: g(k,q) complex64 block, u_ph, u_{k+q} slice, omega, column map"}
    elif dom_name == "zgemm":   # kR->kq per kept k: (nw W nm) x nr_ep x pairs of that k, FP64
        flops = 8.0 * NW * W * nm * nr_ep * st_rank["pairs"]
        peak, psrc = measure_fp64_peak(torch), "measured live: cuBLAS DGEMM 8192^3"
    elif dom_name == "umma_rr":  # RR->kR over Re for the kept k (all nw^2 nm nr_ep rows), split BF16x3
        from epb200 import shard as _sh

        a_k, b_k = _sh.shard_range(int(st_rank["kept_k"]), ws, rank)
        flops = 8.0 * NW * NW * nm * nr_ep * nr_el * (b_k - a_k)
        peak, psrc = peaks["bf16_tflops_sustained"] / 6, f"{peak_src} bf16 sustained / 6 split products"
    else:
        flops = None
    if flops is not None and dom_cnt:
        ach = flops / (dom_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "kernel": dom_name, "achieved": round(ach, 3), "peak": round(peak, 2),
                "unit": "TFLOP/s", "frac": round(ach / peak, 4), "traffic": None, "peak_source": psrc,
                "launch_ms": round(dom_ms / dom_cnt, 4), "launches_per_step": dom_cnt,
                "algorithmic_flops_per_step": flops}
    cpu = None
    if not args.no_cpu and ws == 1:
        mh = m_host_for_cpu(m, ep_dev)
        cng = 16
        t0 = time.perf_counter()
        _, _, info = BO.serta(mh, cng, ef - half, ef + half, ef, T, eta, method=5)
        dt = time.perf_counter() - t0
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": info["npairs"] / dt, "unit": "pairs/s", "cores": cores, "kind": "port",
               "sample": f"the same model and window on a {cng}^3 k = q grid ({len(info['kept'])} kept k, "
                         f"{info['npairs']} pairs), {dt:.1f} s; numpy/scipy per-pair chain"}
        del mh
    line = {"metric": BTE_METRIC, "value": st["pairs"] / (ms * 1e-3), "unit": "pairs/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3/f64" if kw["prec"] == 1 else "f64",
            "data": "synthetic (seeded config-2 model; g(Re,Rp) generated on the device)",
            "config": {"workload": f"config5 SERTA: nw=16, nm=12, Re 9^3, Rp 5^3, {ng}^3 k = q grids, window E_F -/+ 0.3 eV, "
                                   "T = 300 K, Gaussian 10 meV, method 5", "e_fermi_ry": ef, "k_batch": kw["k_batch"], **st},
            "sigma": sig.tolist(), "sigma_fp64": sig64.tolist(), "sigma_max_rel_dev_vs_fp64": rel,
            "fp64_ms_per_step": round(ms64, 3), "speedup_vs_fp64": round(ms64 / ms, 3), "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": st["pairs"] / (ms * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 72,
                    "note": "the public call takes the grid size and returns sigma (9 doubles) to the host"},
            "gpu_launches": launches,
            "clocks": clocks, "impl": "epb", "profile_one_step": profile}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


OUTERQ_METRIC = "g(k,q,ν) elems/s of the batched outer-q loop, nw=16 config-2 model, all bands"


def outerq_family_work(name, nk, nq, kb, nd, nr_el, nr_ep):
    """Algorithmic (flops, bytes) of one outer-q step for a profiler family (8 real flops per complex MAC).

    umma_kq / umma_h / umma_rr (mixed): g(k, q) over Re (nd x nr_el x nk per q), H(k+q) (nw^2 x nr_el x nk
    per q), RR->Rq (nd nr_el x nr_ep x nq); fourier_f64 (FP64 mode): H(k+q) + RR->Rq + the k / q states;
    rotation: g(k, q) block (16 nd bytes) + two nw^2 eigenvector blocks in, 16 nw^3 nm flops per k and q."""
    nw2 = NW * NW
    nm = 3 * NATOM
    if name == "umma_kq":   # g(k, q) of the mixed mode
        return 8.0 * nd * nr_el * nk * nq, None
    if name == "umma_h":    # H(k+q) of the mixed mode
        return 8.0 * nw2 * nr_el * nk * nq, None
    if name == "umma_rr":   # RR->Rq of the mixed mode
        return 8.0 * nd * nr_el * nr_ep * nq, None
    if name == "fourier_f64":
        return 8.0 * (nw2 * nr_el * nk * nq + nd * nr_el * nr_ep * nq + nw2 * nr_el * nk), None
    if name == "rotation":
        return 16.0 * NW ** 3 * nm * nk * nq, (16.0 * nd + 32.0 * nw2) * nk * nq
    return None, None


def run_outerq(args):
    import torch

    from epb200 import outer_q, pipeline, synth
    from oracle import epb_oracle as O

    torch.cuda.set_device(0)
    nk = args.nk if args.nk != NK else 8192
    nq = args.nq if args.nq != NQ else 64
    if args.small:  # profiling case: Re 5^3, 4096 k x 8 q (a few GB on the device)
        nk, nq = 4096, 8
    m = build_model_host_small()
    ep_dev = synth.epmat_el_device(SEED, NW, 3 * NATOM, m.el_ham.irvec, synth.irvec_box(N_PH))
    m.epmat = synth.device_epmat_object(ep_dev, m.el_ham.irvec, synth.irvec_box(N_PH))
    dm = pipeline.DeviceModel(m)
    xks = synth.random_kpoints(nk, 3000)
    xqs = synth.random_kpoints(nq, 4000)
    nm, nr_el, nr_ep = 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3
    nd = NW * NW * nm
    n_el = nk * nq * NW * NW * nm
    prec = pipeline.PREC_FP64 if args.prec == "fp64" else pipeline.PREC_MIXED
    kw = dict(prec=prec, nk_batch_max=args.k_batch if args.k_batch > 0 else 0)

    def step(p=prec):
        return outer_q.run_eph_over_q_and_k(dm, xks, xqs, **dict(kw, prec=p))

    for _ in range(args.warmup):
        A, st = step()
    torch.cuda.synchronize()
    clk = clocks_start()
    l0 = dm.ctx.launch_count()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        A, st = step()
    e1.record(s)
    torch.cuda.synchronize()
    clocks = clocks_stop(clk, 0)
    ms = e0.elapsed_time(e1) / args.steps
    launches = dm.ctx.launch_count() - l0
    dm.ctx.profile(True)
    step()
    torch.cuda.synchronize()
    prof = dm.ctx.profile_read(reset=True)
    dm.ctx.profile(False)
    tot = sum(v[0] for v in prof.values())
    profile = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / tot, 4)} for k, v in prof.items() if v[1]}
    # FP64 on the same inputs: time and the record deviation of the mixed path
    e0.record(s)
    A64, _ = step(pipeline.PREC_FP64)
    e1.record(s)
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1)
    rel = float(np.max(np.abs(A - A64) / np.abs(A64)))

    peaks, peak_src = measured_peaks()
    dom_name, (dom_ms, dom_cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    flops, nbytes = outerq_family_work(dom_name, nk, nq, st["k_batch"], nd, nr_el, nr_ep)
    roof = None
    if flops is not None and dom_cnt:
        t = dom_ms * 1e-3
        if dom_name.startswith("umma"):
            peak, psrc, bound = peaks["bf16_tflops_sustained"] / 6, f"{peak_src} bf16 sustained / 6 split products", "tensor"
        elif dom_name == "rotation":
            peak, psrc, bound = None, None, "hbm"
        else:
            peak, psrc, bound = measure_fp64_peak(torch), "measured live: cuBLAS DGEMM 8192^3", "tensor"
        if bound == "hbm":
            ach = nbytes / t / 1e9
            roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 2), "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": round(ach / peaks["hbm_gbs"], 5), "traffic": None,
                    "peak_source": f"{peak_src} hbm copy"}
        else:
            ach = flops / t / 1e12
            roof = {"bound": bound, "kernel": dom_name, "achieved": round(ach, 3), "peak": round(peak, 2),
                    "unit": "TFLOP/s", "frac": round(ach / peak, 4), "traffic": None, "peak_source": psrc}
        roof.update({"launch_ms": round(dom_ms / dom_cnt, 4), "launches_per_step": dom_cnt,
                     "algorithmic_work_per_step": flops if bound != "hbm" else nbytes})

    cpu = None
    if not args.no_cpu:
        # the oracle's per-point outer-q chain on a bounded sample of the same workload
        mh = m_host_for_cpu(m, ep_dev)
        cnk, cnq = min(256, nk), 2
        t0 = time.perf_counter()
        Ac = O.outer_q_record(mh, xks[:, :cnk], xqs[:, :cnq])
        dt = time.perf_counter() - t0
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": cnk * cnq * NW * NW * nm / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cnk} k x {cnq} q of the same model (all bands), {dt:.1f} s; numpy/scipy per-point "
                         "outer-q chain (RR->Rq per q, Rq->kq per k, ZHEEV)"}
        del mh
    line = {"metric": OUTERQ_METRIC, "value": n_el / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3/f32/f64" if prec == pipeline.PREC_MIXED else "f64",
            "data": "synthetic (seeded config-2 model; g(Re,Rp) generated on the device)",
            "config": {"workload": f"outer-q loop: nw=16, nm=12, Re {2 * N_EL + 1}^3, Rp 5^3, {nk} random k x {nq} random q, "
                                   "all bands, eigenmode basis, record consumer", **st,
                       "l2": "inputs larger than L2 (g(Re,Rp) 4.48 GB re-read per q chunk)"},
            "record_max_rel_dev_vs_fp64": rel, "fp64_ms_per_step": round(ms64, 3),
            "speedup_vs_fp64": round(ms64 / ms, 3), "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": n_el / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 24 * (nk + nq),
                    "d2h_bytes_per_step": 8 * nq, "note": "the public call takes host k / q lists and returns "
                                                          "the host record; the timed step is that call"},
            "gpu_launches": launches, "clocks": clocks, "impl": "epb", "profile_one_step": profile}
    print(json.dumps(line), flush=True)


EPW_METRIC = "EPW epmatwp bytes/s into HBM (\"el\" layout, R sort + Wigner-Seitz divisions), config-2 size"


def run_epw(args):
    import ctypes as C

    import torch

    from epb200 import _lib
    from oracle import epw_oracle as EO

    torch.cuda.set_device(0)
    nw, nm, nr_el, nr_ep, nat = NW, 3 * NATOM, (2 * N_EL + 1) ** 3, (2 * N_PH + 1) ** 3, NATOM
    ctx = _lib.default_context()
    rng = np.random.default_rng(9)
    path = os.path.join("/tmp", f"epb_bench_{os.getpid()}.epmatwp")
    slab = nw * nw * nr_el * nm  # complex values per Rp
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    with open(path, "wb") as fh:  # random file content, one Rp at a time
        for _ in range(nr_ep):
            fh.write(torch.randn(slab, dtype=torch.complex128, device="cuda", generator=g).cpu().numpy().tobytes())
    nbytes = 16 * slab * nr_ep
    ind_el = (rng.permutation(nr_el) + 1).astype(np.int64)
    ind_ep = (rng.permutation(nr_ep) + 1).astype(np.int64)
    nd_el = np.asfortranarray(rng.integers(1, 4, (nw, nw, nr_el)).astype(np.int32))
    nd_ep = np.asfortranarray(rng.integers(1, 4, (nw, nat, nr_ep)).astype(np.int32))
    out = torch.empty(nbytes // 16, dtype=torch.complex128, device="cuda")

    def read(fn=path, nr=nr_ep, ip=ind_ep, nde=nd_ep, dst=out):
        _lib.check(_lib.lib().epb_read_epmat(ctx.h, fn.encode(), nw, nm, nr_el, nr, ind_el.ctypes.data, ip.ctypes.data,
                                             nd_el.ctypes.data, nw, nde.ctypes.data, nw, nat, 0, 0, 0, dst.data_ptr()))

    try:
        for _ in range(args.warmup):
            read()
        torch.cuda.synchronize()
        clk = clocks_start()
        l0 = ctx.launch_count()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            read()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.steps
        clocks = clocks_stop(clk, 0)
        launches = ctx.launch_count() - l0
        # live pinned host -> device bandwidth (the pipeline's bound) and the scatter kernel's HBM roofline
        hb = torch.empty(1 << 28, dtype=torch.uint8).pin_memory()
        db = torch.empty(1 << 28, dtype=torch.uint8, device="cuda")
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        db.copy_(hb, non_blocking=True)
        e0.record(s)
        for _ in range(4):
            db.copy_(hb, non_blocking=True)
        e1.record(s)
        torch.cuda.synchronize()
        h2d = 4 * (1 << 28) / (e0.elapsed_time(e1) * 1e-3) / 1e9
        peaks, peak_src = measured_peaks()
        # CPU port on a bounded sample: the same slabs for the first 8 Rp
        cnr = 8
        cpath = path + ".sample"
        with open(path, "rb") as fi, open(cpath, "wb") as fo:
            fo.write(fi.read(16 * slab * cnr))
        ip8 = np.argsort(rng.permutation(cnr)).astype(np.int64)
        t1 = time.perf_counter()
        EO.read_epmat(cpath, nw, nm, nr_el, cnr, ind_el - 1, ip8, nd_el, nd_ep[:, :, :cnr])
        cdt = time.perf_counter() - t1
        os.remove(cpath)
    finally:
        os.remove(path)
    cores = 1
    line = {"metric": EPW_METRIC, "value": nbytes / dt, "unit": "bytes/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (random file content, seeded permutations and "
                                                           "degeneracies)",
            "config": {"workload": f"epmatwp reader: nw={nw}, nm={nm}, nr_el={nr_el}, nr_ep={nr_ep}, {nbytes / 1e9:.2f} GB, "
                                   "page-cache resident file, per-orbital ndegen, layout el",
                       "l2": "inputs larger than L2", "timing": "host wall clock around the synchronous call"},
            "roofline": {"bound": "hbm", "kernel": "pipeline (pinned host -> HBM copy)", "achieved": round(nbytes / dt / 1e9, 2),
                         "peak": round(h2d, 2), "unit": "GB/s", "frac": round(nbytes / dt / 1e9 / h2d, 4), "traffic": None,
                         "peak_source": "measured live: pinned 256 MiB host-to-device copies",
                         "note": "the file streams through PCIe; the scatter kernel moves 2 x the file bytes in HBM "
                                 f"against a {peaks['hbm_gbs']} GB/s copy peak ({peak_src})"},
            "cpu_baseline": {"value": 16 * slab * cnr / cdt, "unit": "bytes/s", "cores": cores, "kind": "port",
                             "sample": f"numpy read_epmat of the first {cnr} Rp slabs ({16 * slab * cnr / 1e6:.0f} MB), {cdt:.1f} s"},
            "e2e": {"value": nbytes / dt, "unit": "bytes/s", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": 0,
                    "note": "file on the host to the final layout in HBM; the timed call is the public entry point"},
            "gpu_launches": launches, "clocks": clocks, "impl": "epb"}
    print(json.dumps(line), flush=True)


BANDS_METRIC = "k-points/s: H(k) Fourier + eigenvalues and eigenvectors, nw=8 tight-binding (config 1)"


def run_bands(args):
    import torch

    from epb200 import batched as B
    from epb200 import synth
    from epb200.wannier import to_device

    from epb200 import _lib

    torch.cuda.set_device(0)
    ham, xks = synth.config1(seed=1)
    nk = xks.shape[1]
    itp = B.get_interpolator(to_device(ham))
    xk_d = B.jl(xks)
    ctx = _lib.default_context()
    res = {}
    clocks, launches = None, 0
    for prec, name in ((B.PREC_FP64, "fp64"), (B.PREC_MIXED, "mixed")):
        for _ in range(args.warmup):
            E, U = B.get_el_eigen_batched(itp, xk_d, prec=prec)
        torch.cuda.synchronize()
        clk = clocks_start() if name == "fp64" else None
        l0 = ctx.launch_count()
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            E, U = B.get_el_eigen_batched(itp, xk_d, prec=prec)
        e1.record(s)
        torch.cuda.synchronize()
        if name == "fp64":
            clocks = clocks_stop(clk, 0)
            launches = ctx.launch_count() - l0
        res[name] = (e0.elapsed_time(e1) / args.steps, B.host(E))
    dev = float(np.max(np.abs(res["mixed"][1] - res["fp64"][1])))
    # profile one FP64 step: the dominant family and its HBM roofline (the step is launch-bound)
    ctx.profile(True)
    B.get_el_eigen_batched(itp, xk_d, prec=B.PREC_FP64)
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    profile = {k: {"ms": round(v[0], 4), "launches": v[1]} for k, v in prof.items() if v[1]}
    dom_name, (dom_ms, dom_cnt) = max(prof.items(), key=lambda kv: kv[1][0])
    peaks, peak_src = measured_peaks()
    nbytes = {"eigh": nk * (16 * 64 * 2 + 8 * 8), "fourier_f64": 16 * 64 * 343 + nk * (24 + 16 * 64)}.get(dom_name)
    roof = None
    if nbytes and dom_cnt:
        ach = nbytes / (dom_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(ach / peaks["hbm_gbs"], 5), "traffic": None, "peak_source": f"{peak_src} hbm copy",
                "launch_ms": round(dom_ms / dom_cnt, 4), "algorithmic_bytes_per_launch": nbytes,
                "note": "4096 matrices of order 8 and a 351 KB operator: the step is latency / launch bound"}
    # e2e: host k list in, eigenvalues + eigenvectors out
    xk_h = torch.from_numpy(np.ascontiguousarray(xks.T)).pin_memory()
    E, U = B.get_el_eigen_batched(itp, xk_d, prec=B.PREC_FP64)
    hE = torch.empty(E.shape, dtype=E.dtype).pin_memory()
    hU = torch.empty(U.shape, dtype=U.dtype).pin_memory()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        E, U = B.get_el_eigen_batched(itp, xk_h.to("cuda", non_blocking=True), prec=B.PREC_FP64)
        hE.copy_(E, non_blocking=True)
        hU.copy_(U, non_blocking=True)
    e1.record(s)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / args.steps
    cpu = None
    if not args.no_cpu:
        from oracle import epb_oracle as O

        t0 = time.perf_counter()
        hk = O.fourier_batched(ham.op_r, 64, ham.irvec, xks[:, :1024])
        O.eigen_batched(np.asfortranarray(hk.reshape(8, 8, -1, order="F")))
        dt = time.perf_counter() - t0
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": 1024 / dt, "unit": "k-points/s", "cores": cores, "kind": "port",
               "sample": f"1024 of the 4096 k: ZGEMM Fourier + per-k ZHEEV, {dt:.2f} s"}
    # the headline is the FP64 path (config 1 is the plain FP64 interpolation); the mixed path (FP64 H(k),
    # FP32 Jacobi + FP64 refinement) is reported beside it with its eigenvalue deviation
    ms = res["fp64"][0]
    line = {"metric": BANDS_METRIC, "value": nk / (ms * 1e-3), "unit": "k-points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; H(R) ~ CN(0,1) exp(-|R|/1.5))",
            "config": {"workload": "config1: nw=8, R 7^3 (343), 4096 random k, E + U", "nk": nk,
                       "l2": "inputs fit in L2 (351 KB operator); the whole step is launch-bound"},
            "mixed_ms_per_step": round(res["mixed"][0], 3), "mixed_value": nk / (res["mixed"][0] * 1e-3),
            "max_abs_eig_dev_mixed_vs_fp64_ry": dev, "roofline": roof, "cpu_baseline": cpu,
            "gpu_launches": launches, "clocks": clocks, "profile_one_step": profile,
            "e2e": {"value": nk / (ms_e2e * 1e-3), "unit": "k-points/s", "h2d_bytes_per_step": xk_h.numel() * 8,
                    "d2h_bytes_per_step": hE.numel() * 8 + hU.numel() * 16, "ms_per_step": round(ms_e2e, 3)},
            "impl": "epb"}
    print(json.dumps(line), flush=True)


EIGH_METRIC = "uneven batched Hermitian eigensolves/s (n in 4..96, 5% planted clusters), eigenvalues + vectors"


def eigh_generate(count, torch, seed=3):
    """Config-3 batch on the device: CN(0,1) symmetrised, or Q diag(e) Q^H with a planted cluster."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(np.arange(4, 97, 4), count).astype(np.int64)
    planted = rng.random(count) < 0.05
    a_off = np.zeros(count, np.int64)
    a_off[1:] = np.cumsum(sizes * sizes)[:-1]
    e_off = np.zeros(count, np.int64)
    e_off[1:] = np.cumsum(sizes)[:-1]
    total = int((sizes * sizes).sum())
    A = torch.empty(total, dtype=torch.complex128, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(seed)
    for n in np.unique(sizes):
        for plant in (False, True):
            idx = np.nonzero((sizes == n) & (planted == plant))[0]
            if len(idx) == 0:
                continue
            for c0 in range(0, len(idx), 8192):
                ii = idx[c0:c0 + 8192]
                m = len(ii)
                X = torch.randn((m, n, n), dtype=torch.complex128, device="cuda", generator=g)
                if not plant:
                    H = (X + X.conj().transpose(1, 2)) * 0.5
                else:
                    Q, _ = torch.linalg.qr(X)
                    ev = torch.sort(torch.randn((m, n), dtype=torch.float64, device="cuda", generator=g) * float(np.sqrt(n)),
                                    dim=1).values
                    c = int(rng.integers(2, 5))
                    st = int(rng.integers(0, n - c + 1))
                    ev[:, st:st + c] = ev[:, st:st + 1] + 1e-10 * torch.arange(c, device="cuda", dtype=torch.float64)
                    H = (Q * ev[:, None, :].to(torch.complex128)) @ Q.conj().transpose(1, 2)
                    H = (H + H.conj().transpose(1, 2)) * 0.5
                base = torch.from_numpy(a_off[ii]).cuda()[:, None] + torch.arange(n * n, device="cuda")[None, :]
                A[base.reshape(-1)] = H.reshape(-1)
                del X, H
    return sizes, a_off, e_off, A


def run_eigh(args):
    import torch

    from epb200 import _lib

    torch.cuda.set_device(0)
    prec = _lib.PREC_FP64 if args.prec == "fp64" else _lib.PREC_MIXED
    t0 = time.perf_counter()
    sizes, a_off, e_off, A0 = eigh_generate(args.count, torch)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    A = torch.empty_like(A0)
    n_d = torch.from_numpy(sizes.astype(np.int32)).cuda()
    ao_d = torch.from_numpy(a_off).cuda()
    eo_d = torch.from_numpy(e_off).cuda()
    E = torch.empty(int(sizes.sum()), dtype=torch.float64, device="cuda")
    ctx = _lib.default_context()
    L = _lib.lib()

    def solve():
        return L.epb_eigh_varlen(ctx.h, A.data_ptr(), ao_d.data_ptr(), n_d.data_ptr(), args.count, E.data_ptr(),
                                 eo_d.data_ptr(), b"V", prec)

    s = torch.cuda.current_stream()
    for _ in range(args.warmup):
        A.copy_(A0)
        _lib.check(solve())
    torch.cuda.synchronize()
    clk = clocks_start()
    tot_ms = 0.0
    l0 = ctx.launch_count()
    for _ in range(args.steps):
        A.copy_(A0)  # the solve overwrites its input: restored outside the timed region
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        st = solve()
        e1.record(s)
        torch.cuda.synchronize()
        _lib.check(st)
        tot_ms += e0.elapsed_time(e1)
    clocks = clocks_stop(clk, 0)
    launches = ctx.launch_count() - l0
    ms = tot_ms / args.steps
    ctx.profile(True)
    A.copy_(A0)
    _lib.check(solve())
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    profile = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in prof.items() if v[1]}
    # e2e through the public call with host buffers, on the first (at most) 100 000 matrices of the batch:
    # pinned host matrices in, eigenvalues and eigenvectors back to pinned host memory, all timed
    ne = min(args.count, 100000)
    abytes = int(a_off[ne - 1] + sizes[ne - 1] ** 2)
    ebytes = int(e_off[ne - 1] + sizes[ne - 1])
    A_h = A0[:abytes].cpu().pin_memory()
    U_h = torch.empty_like(A_h).pin_memory()
    E_h = torch.empty(ebytes, dtype=torch.float64).pin_memory()
    e2e_ms = 0.0
    for it in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        A[:abytes].copy_(A_h, non_blocking=True)
        st = L.epb_eigh_varlen(ctx.h, A.data_ptr(), ao_d.data_ptr(), n_d.data_ptr(), ne, E.data_ptr(), eo_d.data_ptr(),
                               b"V", prec)
        U_h.copy_(A[:abytes], non_blocking=True)
        E_h.copy_(E[:ebytes], non_blocking=True)
        e1.record(s)
        torch.cuda.synchronize()
        _lib.check(st)
        if it >= args.warmup:
            e2e_ms += e0.elapsed_time(e1)
    e2e_ms /= args.steps
    e2e = {"value": ne / (e2e_ms * 1e-3), "unit": "matrices/s", "h2d_bytes_per_step": 16 * abytes,
           "d2h_bytes_per_step": 16 * abytes + 8 * ebytes, "ms_per_step": round(e2e_ms, 3),
           "sample": f"the first {ne} matrices of the batch (pinned host buffers)"}
    del A_h, U_h, E_h
    # accuracy spot check on a sample vs LAPACK (host)
    from oracle import epb_oracle as O

    Eh = E.cpu().numpy()
    Ah = A0.cpu().numpy() if args.count <= 20000 else None
    worst = 0.0
    sample = np.random.default_rng(9).choice(args.count, 64, replace=False)
    for b in sample:
        n, ao, eo = int(sizes[b]), int(a_off[b]), int(e_off[b])
        h = (A0[ao:ao + n * n].cpu().numpy() if Ah is None else Ah[ao:ao + n * n]).reshape(n, n, order="F")
        ref = O._zheev(h.copy(), "N")[0]
        worst = max(worst, float(np.max(np.abs(Eh[eo:eo + n] - ref))))
    # algorithmic bytes: every matrix read and its eigenvectors written (16 n^2 each) + 8 n eigenvalues
    nbytes = float((32 * sizes * sizes + 8 * sizes).sum())
    peaks, psrc = measured_peaks()
    ach = nbytes / (ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "eigh (all size classes)", "achieved": round(ach, 2), "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": round(ach / peaks["hbm_gbs"], 5), "traffic": None,
            "peak_source": f"{psrc} hbm copy; the solve is FP32/FP64 CUDA-core compute bound (about 90 flop/B)"}
    # compute roofline: 40 n^3 real flops per matrix (the dense Hermitian eigensolve with vectors counted as
    # tridiagonalisation + implicit QR + back-transformation in complex arithmetic), against a live FFMA peak
    flops = float((40.0 * sizes.astype(np.float64) ** 3).sum())
    fp32 = measure_fp32_simt_peak(torch)
    ach_f = flops / (ms * 1e-3) / 1e12
    roof_c = {"bound": "fp32 simt", "kernel": "eigh (all size classes)", "achieved": round(ach_f, 3), "peak": round(fp32, 2),
              "unit": "TFLOP/s", "frac": round(ach_f / fp32, 4),
              "peak_source": "measured live: cuBLAS SGEMM 8192^3, TF32 off",
              "note": "algorithmic flops 40 n^3 per matrix; the Jacobi solves do several times more"}
    cpu = None
    if not args.no_cpu:
        t0 = time.perf_counter()
        nd = 0
        for b in range(400):
            n, ao = int(sizes[b]), int(a_off[b])
            h = A0[ao:ao + n * n].cpu().numpy().reshape(n, n, order="F")
            O._zheev(h, "V")
            nd += 1
        dt = time.perf_counter() - t0
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": nd / dt, "unit": "matrices/s", "cores": cores, "kind": "port",
               "sample": f"first {nd} matrices of the batch, LAPACK ZHEEV (scipy), {dt:.1f} s"}
    line = {"metric": EIGH_METRIC, "value": args.count / (ms * 1e-3), "unit": "matrices/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64" if prec == _lib.PREC_MIXED else "f64",
            "data": "synthetic (seeded, generated on the device)",
            "config": {"workload": f"config3 uneven batched eigensolve: {args.count} matrices, n in 4..96, 5% planted "
                                   "2-4-fold clusters spaced 1e-10", "precision": args.prec,
                       "input_bytes": int(16 * (sizes * sizes).sum()), "generation_s": round(t_gen, 1),
                       "l2": "inputs larger than L2"},
            "autotuned_classes": {l.split()[0]: ("L2-scratch solver instance" if l.split()[1] == "1" else
                                                 "shared-memory / 512-thread solver")
                                  for l in ctx.tune_text().splitlines() if l.startswith("eigh_varlen/")},
            "max_abs_eig_err_vs_lapack_sample64": worst, "roofline": roof, "roofline_compute": roof_c,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "impl": "epb", "profile_one_step": profile}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "eigh":
        run_eigh(a)
    elif a.workload == "bands":
        run_bands(a)
    elif a.workload == "bte":
        run_bte(a)
    elif a.workload == "outerq":
        run_outerq(a)
    elif a.workload == "epw":
        run_epw(a)
    elif a.workload == "filter":
        if a.nq == NQ:
            a.nq = 8192
        run_filter(a)
    else:
        run_epb(a)
