#!/usr/bin/env python
"""Localizations/s of the batched Poisson-MLE PSF estimator on B200.

One step = one pass of the hot path over one batch: LM fit (centre-of-mass start) +
Fisher/CRLB + chi-square for every ROI of the batch, which is what photonpy's
EstimationQueue runs per batch (Estimate then ChiSquareAndCRLB).

Default workload: 2D Gaussian free-sigma MLE (XYIBgSigmaXY), 1,000,000 float32 ROIs of
16x16 px per GPU, photonpy's Python defaults (LM lambda 1e-18, 50 iterations), seeded
synthetic Poisson data. The inputs (1.02 GB) exceed the 126 MB L2, so no L2 flush is needed
between steps.

  value   device-resident throughput (inputs already in HBM), CUDA events on the launch stream
  e2e     the same through the C ABI (PB200_EstimateCRLB) with pinned HOST buffers; the
          host->device copy of the ROIs and the device->host copy of the results are inside
          the timed region (wall clock around the synchronous call)
  roofline  the fit kernel is bound by the FP32 FMA pipe (not tensor cores, not HBM):
          achieved = algorithmic FLOPs (photonpy_b200/roofline.py) / kernel time, peak =
          FP32 FMA throughput measured in the same run by PB200_Fp32ProbeLaunch
  cpu_baseline  photonpy's own C++ CPU estimator (oracle/_ref, built from the reference
          sources) on a bounded sample of the same ROIs, all host cores

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]
Multi-GPU: one process per GPU (torchrun); each rank fits its own batch (weak scaling, no
collective on the data path); the step time is the max over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "localizations/s (1 B200, fused vs plain GPU vs host CPU) at CPU-oracle tolerance"
UNIT = "localizations/s"
MAX_IT = 50
LAMBDA = 1e-18


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sigmaxy", choices=["sigmaxy", "xyibg", "astig", "spline", "mixed", "frames"])
    ap.add_argument("--tile", type=int, default=0,
                    help="mixed workload: ROIs a group takes per claim (0: the autotuner picks it and the "
                         "register budget)")
    ap.add_argument("--n", type=int, default=None, help="ROIs per GPU (default: the workload's size)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per ROI (0 = library default)")
    ap.add_argument("--standalone-min", type=int, default=None, dest="standalone_min",
                    help="mixed workload: ROIs per SM from which a bucket runs as launches of its own "
                         "(default: the library's)")
    ap.add_argument("--threads", type=int, default=0, help="threads per block (0 = library default)")
    ap.add_argument("--variant", type=int, default=None, help="Gaussian kernel family (0 column-blocked, 1 generic)")
    ap.add_argument("--xy-step", type=float, default=1.0, dest="xy_step",
                    help="spline workload: xy step of the 26x26x41 calibration in ROI pixels (1: photonpy's one "
                         "voxel per pixel; 0.5: the oversampled extension, whose CPU baseline is the oracle port)")
    ap.add_argument("--B", type=float, default=0.0, dest="astig_B",
                    help="astig workload: quartic term B of sigma(z) (0: photonpy's 4-coefficient form; the "
                         "reference cannot express B != 0, so its CPU baseline is then the oracle port)")
    return ap.parse_args()


WORKLOADS = {
    "sigmaxy": dict(n=1_000_000, desc="XYIBgSigmaXY 16x16 free-sigma 2D Gaussian MLE + CRLB"),
    "xyibg": dict(n=1_000_000, desc="XYIBg 10x10 fixed-sigma 2D Gaussian MLE + CRLB"),
    "astig": dict(n=1_000_000, desc="XYZIBg 12x12 astigmatic 3D Gaussian MLE + CRLB (reference 4-term form)"),
    "spline": dict(n=500_000, desc="CSpline XYZIBg 13x13 cubic-spline 3D MLE + CRLB"),
    "mixed": dict(n=4_000_000, desc="mixed batch: ROI sizes {7,9,11,16} p={.2,.3,.3,.2}, 50% XYIBg / 30% "
                                    "XYIBgSigmaXY / 20% astig XYZIBg, LM + CRLB"),
    "frames": dict(n=200, desc="camera frames 512x512 (60 spots each, sigma 1.5 px) -> spot detection -> 9x9 ROIs "
                               "-> XYIBg fit + CRLB"),
}


# seed of each workload's batch (rank r of the GPU arm draws with seed + 1000 r)
BASE_SEED = {"sigmaxy": 2, "xyibg": 1, "astig": 3, "spline": 4}


def make_data(workload, n, seed, device=None, astig_B=0.0, xy_step=1.0):
    from photonpy_b200 import synth
    synth.use_torch(device, seed)
    if workload == "sigmaxy":
        return synth.sigmaxy(n, seed=seed)
    if workload == "xyibg":
        return synth.xyibg(n, seed=seed)
    if workload == "astig":
        return synth.astig(n, seed=seed, B=astig_B)
    if workload == "spline":
        d = synth.spline(n, seed=seed, B=astig_B)
        zstack, zr = synth.astig_zstack(shape_xy=26, nz=41, zrange_um=(-0.4, 0.4), B=astig_B, step_px=xy_step)
        d["zstack"], d["spline_zrange"], d["xy_step"] = zstack, zr, xy_step
        return d
    raise ValueError(workload)


def workload_desc(args, w):
    if args.workload == "astig" and args.astig_B:
        return w["desc"].replace("(reference 4-term form)", f"(quartic term B = {args.astig_B:g}, FP64-oracle extension)")
    if args.workload == "spline":
        step = "1 px (photonpy's form)" if args.xy_step == 1.0 else f"{args.xy_step:g} px (oversampled extension)"
        return w["desc"] + f", 26x26x41 calibration, xy step {step}, z step 20 nm" + (
            f", astig model with B = {args.astig_B:g}" if args.astig_B else "")
    return w["desc"]


def make_estimator(pb, ctx, d):
    G = pb.GaussianPSFMethods(ctx)
    k = d["kind"]
    if k == "XYIBg":
        return G.CreatePSF_XYIBg(d["R"], d["sigma"], True)
    if k == "XYIBgSigmaXY":
        return G.CreatePSF_XYIBgSigmaXY(d["R"], d["sigma"], True)
    if k == "XYZIBg":
        cx, cy = d["astig"]
        if cx[4] != 0 or cy[4] != 0:
            return G.CreatePSF_XYZIBg(d["R"], pb.Gauss3D_CalibrationB(cx, cy, d["zrange"]), True)
        return G.CreatePSF_XYZIBg(d["R"], pb.Gauss3D_Calibration(cx[:4], cy[:4], d["zrange"]), True)
    if k == "CSpline":
        sm = pb.CSplineMethods(ctx)
        coefs = sm.ComputeSplineCoeff(d["zstack"], border=1)
        calib = pb.CSplineCalibration(d["spline_zrange"][0], d["spline_zrange"][1], coefs)
        e = sm.CreatePSF_XYZIBg(d["R"], calib, sm.FlatBg, True, xyStep=d.get("xy_step", 1.0))
        e._calib = calib
        return e
    raise ValueError(k)


def ref_estimator(d):
    from oracle import ref_lib
    k = d["kind"]
    if k in ("XYIBg", "XYIBgSigmaXY"):
        return ref_lib.RefEstimator(k, d["R"], sigma=d["sigma"])
    if k == "XYZIBg":
        cx, cy = d["astig"]
        return ref_lib.RefEstimator(k, d["R"], astig=(cx[:4], cy[:4]), zrange=d["zrange"])
    if k == "CSpline":
        coefs = ref_lib.spline_compute(d["zstack"], border=1)
        return ref_lib.RefEstimator(k, d["R"], coefs=coefs, spline_zrange=d["spline_zrange"])
    raise ValueError(k)


def oracle_model(d):
    from oracle import oracle as O
    k = d["kind"]
    if k == "XYIBg":
        return O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    if k == "XYIBgSigmaXY":
        return O.Model(O.XYIBG_SIGMAXY, d["R"], sigma=d["sigma"])
    if k == "XYZIBg":
        cx, cy = d["astig"]
        return O.Model(O.XYZIBG, d["R"], astig_x=cx, astig_y=cy, zrange=d["zrange"])
    if k == "CSpline":
        return O.Model(O.CSPLINE, d["R"], coefs=O.spline_compute(d["zstack"], border=1),
                       spline_zrange=d["spline_zrange"], spline_xy_step=d.get("xy_step", 1.0))
    raise ValueError(k)


def cpu_localize(d, samples, keep=False):
    """photonpy's CPU estimator (reference build) — or the oracle port when it is absent —
    on `samples`: Estimate + ChiSquareAndCRLB, in chunks of 20k spots (the reference starts one
    thread per spot). Returns (seconds, kind), plus (params, iterations, crlb) with keep."""
    from oracle import ref_lib
    out = ([], [], [])
    t0 = time.perf_counter()
    if ref_lib.available() and not beyond_reference_model(d):
        est = ref_estimator(d)
        for s in range(0, len(samples), 20000):
            chunk = samples[s:s + 20000]
            p, it, _ = est.estimate(chunk, trace_len=0)
            crlb, _ = est.crlb_chisq(p, chunk)
            if keep:
                for lst, v in zip(out, (p, it, crlb)):
                    lst.append(v)
        est.close()
        kind = "reference"
    else:
        m = oracle_model(d)
        for s in range(0, len(samples), 20000):
            chunk = samples[s:s + 20000]
            p, it = m.fit(chunk)
            crlb, _ = m.crlb(p, chunk)
            if keep:
                for lst, v in zip(out, (p, it, crlb)):
                    lst.append(v)
        kind = "port"
    dt = time.perf_counter() - t0
    if keep:
        return dt, kind, tuple(np.concatenate(v) for v in out)
    return dt, kind


def beyond_reference_model(d):
    """Workloads photonpy's models cannot express: the astig workload with B != 0, the spline
    workload with a calibration sampled finer than one ROI pixel."""
    if d["kind"] == "CSpline":
        return d.get("xy_step", 1.0) != 1.0
    return d["kind"] == "XYZIBg" and (d["astig"][0][4] != 0 or d["astig"][1][4] != 0)


def cpu_baseline(d, budget_s):
    """The CPU estimator timed on the first ROIs of the batch (about budget_s of work); also
    returns its results on those ROIs (params, iterations, crlb) for the parity check."""
    samples = d["samples"]
    n0 = min(len(samples), 2000)
    t, kind = cpu_localize(d, samples[:n0])
    rate = n0 / max(t, 1e-6)
    n = int(min(len(samples), max(n0, rate * budget_s)))
    t, kind, res = cpu_localize(d, samples[:n], keep=True)
    return dict(value=n / t, unit=UNIT, cores=os.cpu_count(), kind=kind,
                sample=f"first {n} ROIs of the same batch ({d['kind']} {d['R']}x{d['R']}), "
                       f"Estimate + ChiSquareAndCRLB, {t:.1f} s"), res


POS_TOL = {"XYIBg": (1e-3, 1e-3), "XYIBgSigmaXY": (1e-3, 1e-3), "XYZIBg": (1e-3, 1e-3, 1.0),
           "CSpline": (1e-3, 1e-3, 1e-3)}


def parity_summary(kind, ref, ours, maxit=MAX_IT):
    """Agreement of the GPU results with the CPU estimator's on the same ROIs, stratified by
    converged (both iteration counts <= maxit) and capped (the reference hit the cap): fractions
    of spots with positions within 1e-3 px (z: 1 nm astig, 1e-3 um spline), I and bg within 1e-4
    relative, CRLB within 1e-4 relative, iteration counts equal, converged flags equal."""
    (rp, rit, rcrlb), (p, it, crlb) = ref, ours
    tol = np.array(POS_TOL[kind])
    npos = len(tol)
    pos_ok = np.all(np.abs(p[:, :npos] - rp[:, :npos]) <= tol, axis=1)
    phot = np.abs(p[:, npos:npos + 2] - rp[:, npos:npos + 2]) / np.maximum(np.abs(rp[:, npos:npos + 2]), 1e-6)
    phot_ok = np.all(phot <= 1e-4, axis=1)
    crlb_ok = np.all(np.abs(crlb - rcrlb) <= 1e-4 * np.abs(rcrlb), axis=1)
    conv_ref, conv = rit <= maxit, it <= maxit
    both = conv_ref & conv
    capped = ~conv_ref

    def frac(m, sel):
        return float(np.mean(m[sel])) if sel.any() else None

    out = dict(n=int(len(it)), capped_ref=float(np.mean(capped)), it_match=float(np.mean(it == rit)),
               conv_flag_match=float(np.mean(conv == conv_ref)))
    for name, sel in (("converged", both), ("capped", capped)):
        out[name] = {"n": int(sel.sum()), "pos_within_1e-3": frac(pos_ok, sel), "I_bg_within_1e-4": frac(phot_ok, sel),
                     "crlb_within_1e-4": frac(crlb_ok, sel), "it_match": frac(it == rit, sel)}
    return out


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smmax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwth=parts[6], swth=parts[7], swpc=parts[8]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 200] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwth", "hw_thermal_slowdown"), ("swth", "sw_thermal_slowdown"),
                              ("swpc", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return dict(sm_mhz=statistics.median(r["sm"] for r in load), sm_max_mhz=max(r["smmax"] for r in rows),
                     power_w_max=max(r["power"] for r in rows), samples=len(rows), reasons=sorted(reasons))


def fp32_peak(pb, torch):
    """Measured FP32 FMA throughput (TFLOP/s) on this GPU: best of 3 probe launches."""
    L = pb.load_library()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = torch.zeros(sms * 8, device="cuda")
    stream = torch.cuda.current_stream()
    best = 0.0
    for it in (2000, 8000, 8000, 8000):
        s, e = torch.cuda.Event(True), torch.cuda.Event(True)
        s.record()
        flops = L.PB200_Fp32ProbeLaunch(sms * 8, 256, it, out.data_ptr(), stream.cuda_stream)
        e.record()
        torch.cuda.synchronize()
        if flops > 0:
            best = max(best, flops / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


HBM_FALLBACK_GBS = 6650.0  # an earlier copy-bandwidth measurement on this pool's B200s


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def hbm_peak(peaks):
    """(GB/s, source): the measured copy bandwidth, else the fallback figure."""
    if peaks.get("hbm_gbs"):
        return float(peaks["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    return HBM_FALLBACK_GBS, "of fallback (no MEASURED_PEAKS.json)"


def traffic_from_profile(workload):
    """DRAM bytes per fit launch from the committed ncu summary, scaled to the batch."""
    p = os.path.join(ROOT, "profiles", f"fit_{workload}_traffic.json")
    try:
        return json.load(open(p))
    except Exception:
        return None


def run_reference(args):
    """Reference arm: photonpy's own CPU estimator on the host cores, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    # the same draws as rank 0 of the GPU arm: same seed, and the Poisson stream from the same
    # torch generator on the GPU when one is present (the data path only; the fits run on the CPU)
    try:
        import torch
        device = "cuda" if torch.cuda.is_available() else None
    except ImportError:
        device = None
    d = make_data(args.workload, args.n or w["n"], seed=BASE_SEED[args.workload], device=device, astig_B=args.astig_B,
                  xy_step=args.xy_step)
    from oracle import ref_lib
    n_cal = 2000
    t, kind = cpu_localize(d, d["samples"][:n_cal])
    per_step = int(min(len(d["samples"]), max(n_cal, n_cal / t * 6.0)))
    for _ in range(args.warmup):
        cpu_localize(d, d["samples"][:min(per_step, 5000)])
    times = []
    for k in range(args.steps):
        off = (k * per_step) % max(1, len(d["samples"]) - per_step + 1)
        t, kind = cpu_localize(d, d["samples"][off:off + per_step])
        times.append(t)
    ms = 1e3 * float(np.mean(times))
    value = per_step / (ms * 1e-3)
    line = dict(impl="reference", metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic (seeded Poisson ROIs)",
                config=dict(workload=workload_desc(args, w), roi_size=d["R"], model=d["kind"], rois_per_step=per_step,
                            batch=len(d["samples"]), seed=BASE_SEED[args.workload],
                            draws="torch generator on the GPU, as the GPU arm" if device else "numpy (no GPU)",
                            lm_iterations=MAX_IT, lm_lambda=LAMBDA),
                cpu_baseline=dict(value=value, unit=UNIT, cores=os.cpu_count(), kind=kind,
                                  sample=f"{per_step} ROIs per step ({d['kind']} {d['R']}x{d['R']}), "
                                         f"Estimate + ChiSquareAndCRLB, reference {'build' if ref_lib.available() else 'port'}"),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def mixed_estimator(pb, ctx, g):
    G = pb.GaussianPSFMethods(ctx)
    if g["kind"] == "XYIBg":
        return G.CreatePSF_XYIBg(g["R"], g["sigma"], True)
    if g["kind"] == "XYIBgSigmaXY":
        return G.CreatePSF_XYIBgSigmaXY(g["R"], g["sigma"], True)
    cx, cy = g["astig"]
    return G.CreatePSF_XYZIBg(g["R"], pb.Gauss3D_Calibration(cx[:4], cy[:4], g["zrange"]), True)


def run_mixed(args):
    """Mixed workload: one graph-replayed MixedBatch run (buckets as launches of their own on
    forked streams, or in the persistent mixed kernel, as the autotuner picks unless --tile is
    given) vs one launch per (model, ROI size) bucket in sequence on one stream (plain),
    device-resident inputs; CPU and reference-GPU baselines."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import roofline, synth
    from photonpy_b200.mixed import MixedBatch, set_standalone_min, standalone_min
    w = WORKLOADS["mixed"]
    n = args.n or w["n"]
    synth.use_torch("cuda", 5)
    groups = synth.mixed(n, seed=5)
    ctx = pb.Context()
    ests = [mixed_estimator(pb, ctx, g) for g in groups]
    xs = [torch.from_numpy(g["samples"]).cuda() for g in groups]
    if args.standalone_min is not None:
        set_standalone_min(args.standalone_min)
    tuned = None
    tile, threads = args.tile, args.threads or 256
    if tile <= 0:
        from photonpy_b200.autotune import tune_mixed
        tuned = tune_mixed(list(zip(ests, xs)), standalone_mins=(0, None) if args.standalone_min is None
                           else (args.standalone_min,))
        tile, threads = tuned["tile"], tuned["threads"]
        set_standalone_min(tuned["standalone_min"])
    mb = MixedBatch(list(zip(ests, xs)), tile_rois=tile, threads=threads)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        mb.run(s)
        s.synchronize()
        mb.capture(s)

    def timed(fn, k):
        for _ in range(max(args.warmup, 3)):
            fn()
        s.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(s)
        for _ in range(k):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    with torch.cuda.stream(s):
        with ClockSampler(0) as clk:
            ms_fused = timed(lambda: mb.run(s), args.steps)
            n0 = pb.launch_count()
            mb.run(s)  # launches of one step, counted outside the timed loop (which has warm-up runs)
            launches = (pb.launch_count() - n0) * args.steps
        n0 = pb.launch_count()
        mb.run_plain(s)
        plain_launches = pb.launch_count() - n0
        ms_plain = timed(lambda: mb.run_plain(s), args.steps)
        ms_plain_default = timed(lambda: mb.run_plain(s, lanes=None), args.steps)
        ms_plain_4 = timed(lambda: mb.run_plain(s, lanes=4), args.steps)
        mb.run(s)  # results of the fused path for the flop count below
    flops = 0.0
    for g, r in zip(groups, mb.results()):
        flops += roofline.localization_flops(g["kind"], g["R"], r["iterations"].cpu().numpy(), MAX_IT)
    peak = fp32_peak(pb, torch)
    # baselines on a bounded proportional sample: reference CPU estimator and the reference's own
    # one-thread-per-ROI GPU kernels (through its host API, copies included)
    cpu = ref_gpu = None
    from oracle import ref_lib
    if ref_lib.available() and not args.no_cpu_baseline:
        frac = min(1.0, 60000 / n)
        tot, t_cpu, t_gpu = 0, 0.0, 0.0
        for g in groups:
            m = max(1, int(len(g["samples"]) * frac))
            sub = dict(g, samples=g["samples"][:m])
            dt, kind = cpu_localize(sub, sub["samples"])
            t_cpu += dt
            est = ref_gpu_estimator(g)
            t0 = time.perf_counter()
            p, _, _ = est.estimate(sub["samples"], trace_len=0)
            est.crlb_chisq(p, sub["samples"])
            t_gpu += time.perf_counter() - t0
            est.close()
            tot += m
        cpu = dict(value=tot / t_cpu, unit=UNIT, cores=os.cpu_count(), kind="reference",
                   sample=f"{tot} ROIs ({frac:.3%} of every bucket), Estimate + ChiSquareAndCRLB")
        ref_gpu = dict(value=tot / t_gpu, unit=UNIT,
                       what="photonpy's own one-thread-per-ROI CUDA kernels built for sm_100a, one call per "
                            "bucket through its host API (host copies included)", sample=f"{tot} ROIs")
    line = dict(
        metric=METRIC, value=n / (ms_fused * 1e-3), unit=UNIT, n_gpus=1, steps=args.steps, warmup=max(args.warmup, 3),
        ms_per_step=ms_fused, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
        data="synthetic (seeded Poisson ROIs, photonpy_b200.synth)",
        config=dict(workload=w["desc"], rois=n, buckets=len(groups), tile_rois=tile, threads_per_block=threads,
                    autotuned=(tuned["timings"] if tuned else None),
                    lanes_per_roi=dict(zip([f"{g['kind']}_{g['R']}" for g in groups], mb.lanes())),
                    standalone_min_rois_per_sm=standalone_min(),
                    standalone_buckets=[f"{g['kind']}_{g['R']}" for g, a in zip(groups, mb.standalone()) if a],
                    graph_replay=True, lm_iterations=MAX_IT, lm_lambda=LAMBDA,
                    l2="inputs of %.2f GB per step exceed the 126 MB L2" % (sum(x.numel() for x in xs) * 4 / 1e9)),
        plain_gpu=dict(value=n / (ms_plain * 1e-3), ms_per_step=ms_plain, launches_per_step=plain_launches,
                       what="the LM, Fisher and CRLB launches of every (model, ROI size) bucket with the "
                            "fused form's lanes per ROI (the same results bit for bit)"),
        plain_gpu_default_config=dict(value=n / (ms_plain_default * 1e-3), ms_per_step=ms_plain_default,
                                      what="the same per-bucket launches at each estimator's default "
                                           "configuration (2 lanes per ROI for the 7 and 9 px buckets)"),
        plain_gpu_4_lanes=dict(value=n / (ms_plain_4 * 1e-3), ms_per_step=ms_plain_4,
                               what="the same per-bucket launches with 4 lanes per ROI for every bucket"),
        fused_over_plain=ms_plain / ms_fused,
        roofline=dict(bound="fp32", achieved=flops / (ms_fused * 1e-3) / 1e12, peak=peak, unit="TFLOP/s",
                      frac=flops / (ms_fused * 1e-3) / 1e12 / peak if peak else None, traffic=None,
                      peak_source="FP32 FMA probe measured in this run"),
        cpu_baseline=cpu, reference_gpu_plain=ref_gpu, gpu_launches=int(launches), clocks=clk.summary())
    print(json.dumps(line), flush=True)
    mb.close()
    ctx.Destroy()


def run_frames(args):
    """Frames workload: spot detection + ROI cut-out + fused fit of device-resident frames
    (value), the same from pinned host frames (e2e), photonpy's spot-extraction queue API
    (SpotExtractionQueue_Create + ImgProc_AddFrameU16, host frames in, ROIs out), and baselines:
    the reference's own queue (its CUDA detector) and the C restatement of the detector on one
    host core."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import spotdetect, synth
    w = WORKLOADS["frames"]
    n = args.n or w["n"]
    H = W = 512
    R = 9
    d = synth.frames(n, h=H, w=W, spots_per_frame=60, seed=21, sigma=1.5, margin=4)
    frames_u16 = d["frames"].astype(np.uint16)
    ctx = pb.Context()
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(R, 1.5, True)
    sd = spotdetect.SpotDetector(1.5, R, 7.0)
    sm = spotdetect.SpotDetectionMethods(ctx)
    x = torch.from_numpy(d["frames"]).cuda()
    K = 256
    stream = torch.cuda.current_stream()

    def step():
        return spotdetect.localize_frames(x, sd, est, R, K)

    def detect_only():
        return sm.DetectDevice(x, sd, R, K)

    for _ in range(max(args.warmup, 3)):
        out = step()
        detect_only()
    torch.cuda.synchronize()

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        r = None
        for _ in range(k):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, r

    with ClockSampler(0) as clk:
        t_w = time.perf_counter()
        while time.perf_counter() - t_w < 0.6:  # keep the GPU busy while nvidia-smi starts sampling
            step()
        torch.cuda.synchronize()
        n0 = pb.launch_count()
        ms, out = timed(step, args.steps)
        launches = pb.launch_count() - n0
        ms_det, _ = timed(detect_only, args.steps)
    nspots = int(out["params"].shape[0])

    e2e = None
    if not args.no_e2e:
        h_frames = torch.from_numpy(frames_u16.view(np.int16)).pin_memory()  # the 16-bit pixels as stored

        def e2e_step():
            xd = h_frames.to("cuda", non_blocking=True).to(torch.int32).bitwise_and_(0xFFFF).to(torch.float32)
            r = spotdetect.localize_frames(xd, sd, est, R, K)
            return r["params"].cpu(), r["crlb"].cpu(), r["frame"].cpu()

        for _ in range(2):
            e2e_step()
        tt = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            e2e_step()
            tt.append(time.perf_counter() - t0)
        et = float(np.mean(tt))
        e2e = dict(value=n / et, unit="frames/s", ms_per_step=1e3 * et, h2d_bytes_per_step=int(frames_u16.nbytes),
                   d2h_bytes_per_step=int(nspots * (2 * 4 * 4 + 8)),
                   api="photonpy_b200.spotdetect.localize_frames on frames copied from pinned host memory")

    # photonpy's queue API: 16-bit host frames pushed one by one, ROIs popped from the ROI queue
    q, rq = sm.CreateQueue((H, W), [R, R], sd)
    for f in frames_u16[:16]:  # warm-up: buffers, worker thread
        q.PushFrameU16(f)
    while q.NumFinishedFrames() < 16 or not q.IsIdle():
        time.sleep(0.001)
    rq.Fetch()
    t0 = time.perf_counter()
    for f in frames_u16:
        q.PushFrameU16(f)
    while q.NumFinishedFrames() < 16 + n or not q.IsIdle():
        time.sleep(0.001)
    info, _ = rq.Fetch()
    t_queue = time.perf_counter() - t0
    q.Destroy()
    queue = dict(value=n / t_queue, unit="frames/s", rois=int(len(info)),
                 api="SpotExtractionQueue_Create + ImgProc_AddFrameU16 (host 16-bit frames in, ROIs out; no fit)")

    cpu = ref_gpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        m = min(n, 12)
        t0 = time.perf_counter()
        for f in range(m):
            O.detect_spots(d["frames"][f], 5, 10, 7, R, 7.0, max_spots=H * W)
        dt = time.perf_counter() - t0
        cpu = dict(value=m / dt, unit="frames/s", cores=1, kind="port",
                   sample=f"{m} frames, spot detection only (the C restatement of photonpy's CUDA detector; "
                          "photonpy has no CPU detector)")
        from oracle import ref_lib
        if ref_lib.available() and hasattr(ref_lib.lib(), "SpotExtractionQueue_Create"):
            m = min(n, 60)
            t0 = time.perf_counter()
            rinfo, _ = ref_lib.spot_queue(frames_u16[:m], 5, 10, 7, R, 7.0)
            dt = time.perf_counter() - t0
            ref_gpu = dict(value=m / dt, unit="frames/s", rois=int(len(rinfo)), sample=f"{m} frames",
                           what="photonpy's own spot-extraction queue (its CUDA detector, 2 detection threads) "
                                "built for sm_100a, host 16-bit frames in, ROIs out; no fit")
    peaks = measured_peaks()
    hbm, hbm_src = hbm_peak(peaks)
    frame_bytes = 4.0 * n * H * W
    achieved = frame_bytes / (ms_det * 1e-3) / 1e9
    line = dict(
        metric="frames/s (1 B200): spot detection + ROI extraction + XYIBg fit + CRLB", value=n / (ms * 1e-3),
        unit="frames/s", n_gpus=1, steps=args.steps, warmup=max(args.warmup, 3), ms_per_step=ms,
        higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
        data="synthetic (seeded Poisson frames, photonpy_b200.synth.frames)",
        config=dict(workload=w["desc"], frames=n, frame_shape=[H, W], spots=nspots, roi_size=R,
                    max_spots_per_frame=K, lm_iterations=MAX_IT, lm_lambda=LAMBDA,
                    l2="frames of %.0f MB per step exceed the 126 MB L2" % (frame_bytes / 1e6)),
        detection=dict(ms_per_step=ms_det, value=n / (ms_det * 1e-3), unit="frames/s"),
        roofline=dict(bound="hbm", achieved=achieved, peak=hbm, unit="GB/s",
                      frac=achieved / hbm if hbm else None, traffic=None,
                      note="detection (4 kernels) over the frame bytes read, " + hbm_src + "; the filter kernel "
                           "is bound by instruction issue, not by HBM (profiles/spot_detect_512x512x200.md)"),
        e2e=e2e, queue_api=queue, cpu_baseline=cpu, reference_gpu_queue=ref_gpu, gpu_launches=int(launches),
        clocks=clk.summary())
    print(json.dumps(line), flush=True)
    est.Destroy()
    ctx.Destroy()


def reference_gpu_plain(d, m=50_000):
    """photonpy's own plain GPU form (its one-thread-per-ROI CUDA kernels built for sm_100a)
    through its host API, Estimate + ChiSquareAndCRLB, on the first m ROIs of the batch; host
    copies included, as photonpy always has them."""
    from oracle import ref_lib
    if not ref_lib.available() or d["kind"] not in ("XYIBg", "XYIBgSigmaXY", "XYZIBg") or beyond_reference_model(d):
        return None
    sub = d["samples"][:m]
    est = ref_gpu_estimator(d)
    try:
        p, _, _ = est.estimate(sub[:1000], trace_len=0)  # warm-up
        t0 = time.perf_counter()
        p, _, _ = est.estimate(sub, trace_len=0)
        est.crlb_chisq(p, sub)
        dt = time.perf_counter() - t0
    finally:
        est.close()
    return dict(value=len(sub) / dt, unit=UNIT, sample=f"first {len(sub)} ROIs of the batch",
                what="photonpy's own one-thread-per-ROI CUDA kernels built for sm_100a, through its host API "
                     "(Estimate + ChiSquareAndCRLB, host copies included)")


def ref_gpu_estimator(d):
    from oracle import ref_lib
    k = d["kind"]
    if k in ("XYIBg", "XYIBgSigmaXY"):
        return ref_lib.RefEstimator(k, d["R"], cuda=True, sigma=d["sigma"])
    cx, cy = d["astig"]
    return ref_lib.RefEstimator(k, d["R"], cuda=True, astig=(cx[:4], cy[:4]), zrange=d["zrange"])


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "mixed":
        run_mixed(args)
        return
    if args.workload == "frames":
        run_frames(args)
        return
    import torch
    import torch.distributed as dist
    import photonpy_b200 as pb
    from photonpy_b200 import roofline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pb.load_library().CudaSetDevice(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    w = WORKLOADS[args.workload]
    n = args.n or w["n"]
    d = make_data(args.workload, n, seed=BASE_SEED[args.workload] + 1000 * rank, device=f"cuda:{local}",
                  astig_B=args.astig_B, xy_step=args.xy_step)
    smp = d["samples"]
    K = roofline.K_OF[d["kind"]]

    ctx = pb.Context()
    est = make_estimator(pb, ctx, d)
    est.SetKernelConfig(args.lanes, args.threads, variant=args.variant)
    x = torch.from_numpy(smp).cuda()
    peak_fp32 = fp32_peak(pb, torch)

    def step():
        return est.EstimateDevice(x, with_crlb=True)

    for _ in range(max(args.warmup, 3)):
        out = step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_w = time.perf_counter()
        while time.perf_counter() - t_w < 0.6:  # keep the GPU busy while nvidia-smi starts sampling
            step()
            torch.cuda.synchronize()
        n_launch0 = pb.launch_count()
        ev0.record(stream)
        for _ in range(args.steps):
            out = step()
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = pb.launch_count() - n_launch0
    ms = ev0.elapsed_time(ev1) / args.steps
    # the dominant kernel alone: the LM launch (the same instance and arguments, without the
    # Fisher and CRLB launches that follow it in a step), timed the same way
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    est.EstimateDevice(x, with_crlb=False)
    ev2.record(stream)
    for _ in range(args.steps):
        est.EstimateDevice(x, with_crlb=False)
    ev3.record(stream)
    torch.cuda.synchronize()
    lm_ms = ev2.elapsed_time(ev3) / args.steps
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n / (ms_max * 1e-3)

    its = out["iterations"].cpu().numpy()
    flops = roofline.localization_flops(d["kind"], d["R"], its, MAX_IT)
    achieved_tflops = flops / (ms * 1e-3) / 1e12
    flops_lm = roofline.lm_flops(d["kind"], d["R"], its, MAX_IT)
    achieved_lm = flops_lm / (lm_ms * 1e-3) / 1e12
    bytes_roi = roofline.hbm_bytes_per_roi(d["kind"], d["R"])
    hbm_gbs = bytes_roi * n / (ms * 1e-3) / 1e9
    peaks = measured_peaks()

    # ---- e2e through the C ABI with pinned host buffers --------------------------------
    e2e = None
    if not args.no_e2e:
        import ctypes as ct
        h_smp = torch.empty(smp.shape, dtype=torch.float32, pin_memory=True)
        h_smp.numpy()[...] = smp
        h_par = torch.empty((n, K), dtype=torch.float32, pin_memory=True)
        h_its = torch.empty(n, dtype=torch.int32, pin_memory=True)
        h_crlb = torch.empty((n, K), dtype=torch.float32, pin_memory=True)
        h_chi = torch.empty(n, dtype=torch.float32, pin_memory=True)
        L = pb.load_library()
        fn = L.PB200_EstimateCRLB
        fn.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                       ct.c_void_p, ct.c_void_p]

        def e2e_step():
            fn(est.inst, n, h_smp.data_ptr(), None, None, h_par.data_ptr(), h_its.data_ptr(), h_crlb.data_ptr(),
               h_chi.data_ptr())
        from photonpy_b200.lib import check_error

        for _ in range(2):
            e2e_step()
        check_error("PB200_EstimateCRLB")
        if world > 1:
            dist.barrier()
        tt = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            e2e_step()
            tt.append(time.perf_counter() - t0)
        check_error("PB200_EstimateCRLB")
        et = torch.tensor([float(np.mean(tt))], device="cuda")
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        h2d = smp.nbytes
        d2h = n * (4 * K * 2 + 8)
        e2e = dict(value=world * n / float(et.item()), unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                   ms_per_step=1e3 * float(et.item()), api="PB200_EstimateCRLB (C ABI, pinned host buffers)")
        # The host-to-device copy of the step's ROIs alone (one copy of the same pinned buffer,
        # CUDA events): with the fits overlapping the copies, an end-to-end step cannot be
        # shorter than the longer of this copy and the device-resident step.
        d_copy = torch.empty(h_smp.shape, dtype=torch.float32, device="cuda")
        for _ in range(2):
            d_copy.copy_(h_smp, non_blocking=True)
        torch.cuda.synchronize()
        ev4, ev5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev4.record()
        for _ in range(3):
            d_copy.copy_(h_smp, non_blocking=True)
        ev5.record()
        ev5.synchronize()
        copy_ms = ev4.elapsed_time(ev5) / 3
        del d_copy
        bound_ms = max(copy_ms, ms)
        e2e["bound"] = dict(h2d_copy_ms=copy_ms, h2d_gbs=h2d / (copy_ms * 1e-3) / 1e9, device_step_ms=ms,
                            bound_ms=bound_ms, frac=bound_ms / e2e["ms_per_step"],
                            what="max(host-to-device copy of the ROIs alone, device-resident step) / e2e step")
        # results through the host path equal the device path
        assert np.array_equal(h_par.numpy(), out["params"].cpu().numpy())

    cpu = ref_gpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_res = cpu_baseline(d, args.cpu_seconds)
        m = len(ref_res[1])
        ours = (out["params"][:m].cpu().numpy(), out["iterations"][:m].cpu().numpy(), out["crlb"][:m].cpu().numpy())
        parity = parity_summary(d["kind"], ref_res, ours)
        parity["sample"] = f"the first {m} ROIs of the timed batch, against the CPU estimator ({cpu['kind']})"
        ref_gpu = reference_gpu_plain(d)

    if rank == 0:
        tr = traffic_from_profile(args.workload)
        traffic = traffic_lm = None
        if tr:
            traffic = tr["dram_bytes_per_roi"] * n
            traffic_lm = tr["lm_dram_bytes_per_roi"] * n
        line = dict(
            metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=max(args.warmup, 3),
            ms_per_step=ms_max, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
            data="synthetic (seeded Poisson ROIs, photonpy_b200.synth)",
            config=dict(workload=workload_desc(args, w), model=d["kind"], roi_size=d["R"], rois_per_gpu=n,
                        global_rois=world * n,
                        lm_iterations=MAX_IT, lm_lambda=LAMBDA, mean_iterations=float(np.minimum(its, MAX_IT).mean()),
                        kernel_config=list(est.GetKernelConfig()),
                        l2="inputs of %.2f GB per step exceed the 126 MB L2; no flush needed" % (smp.nbytes / 1e9),
                        parallelism=f"dp{world} (independent ROI shards, no collective)"),
            roofline=dict(bound="fp32", achieved=achieved_lm, peak=peak_fp32, unit="TFLOP/s",
                          frac=achieved_lm / peak_fp32 if peak_fp32 else None, traffic=traffic_lm,
                          kernel="the LM launch (gauss_fit_kernel / fit_kernel, PASS_LM), 1 launch per step",
                          peak_source="FP32 FMA probe measured in this run (PB200_Fp32ProbeLaunch)",
                          flops_per_launch=flops_lm, kernel_ms=lm_ms),
            roofline_step=dict(bound="fp32", achieved=achieved_tflops, peak=peak_fp32, unit="TFLOP/s",
                               frac=achieved_tflops / peak_fp32 if peak_fp32 else None, traffic=traffic,
                               what="the whole step (LM, Fisher and FP64 CRLB launches)",
                               flops_per_step=flops, step_ms=ms),
            roofline_hbm=dict(bound="hbm", achieved=hbm_gbs, peak=hbm_peak(peaks)[0], unit="GB/s",
                              frac=hbm_gbs / hbm_peak(peaks)[0],
                              note="algorithmic ROI-stream bytes, " + hbm_peak(peaks)[1]),
            e2e=e2e, cpu_baseline=cpu, parity=parity, reference_gpu_plain=ref_gpu, gpu_launches=int(launches),
            clocks=clk.summary(),
        )
        print(json.dumps(line), flush=True)
    est.Destroy()
    ctx.Destroy()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
