"""Autotuner for the fit kernels' launch choices.

For one estimator (model, ROI size, LM settings) it times the fused fit + CRLB over the
candidate kernel configurations — kernel family (column-blocked / generic table), lanes per
ROI (4, 8, 16, 32) and threads per block — on a batch of device-resident ROIs and keeps the
fastest. For a MixedBatch it tunes the claim size (ROIs a group takes per claim) and the kernel's
register budget. Results are cached per GPU model in a JSON file
(``$PB200_AUTOTUNE_CACHE`` or ``~/.cache/photonpy_b200/autotune.json``) so later runs apply
them without timing.
"""
from __future__ import annotations

import json
import math
import os
import threading

_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("PB200_AUTOTUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "photonpy_b200",
                                                                  "autotune.json")


def load_cache(path=None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path=None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def estimator_key(gpu: str, model: int, roisize: int, iterations: int, lam: float) -> str:
    return f"{gpu}|model{model}|R{roisize}|it{iterations}|lam{lam:g}"


def candidates(model: int, roisize: int):
    """(variant, lanes, threads) triples valid for this model and ROI size."""
    out = []
    variants = (1,) if model == 5 else (0, 1)
    for v in variants:
        for g in ((2, 4, 8, 16, 32) if v == 0 else (4, 8, 16, 32)):
            if v == 0 and math.ceil(roisize / g) > (2 if g == 32 else (5 if g == 2 else 4)):
                continue
            if g > roisize * roisize:
                continue
            for t in (128, 256):
                out.append((v, g, t))
    return out


def choose_best(timings: dict):
    """timings: {config: ms} -> (config, ms) with the smallest time (ties: first seen)."""
    best = None
    for cfg, ms in timings.items():
        if ms is None or not math.isfinite(ms):
            continue
        if best is None or ms < best[1]:
            best = (cfg, ms)
    if best is None:
        raise RuntimeError("no candidate configuration ran")
    return best


def _synthetic_rois(est, n, seed=0):
    """Poisson ROIs of the estimator's own model at plausible parameters (centre +- 1 px)."""
    import torch
    from .lib import load_library  # noqa: F401
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    R = int(est.sampleshape[0])
    K = est.numparams
    lo, hi = est.ParamLimits()
    th = torch.empty((n, K), device="cuda")
    u = lambda: torch.rand(n, device="cuda", generator=g)  # noqa: E731
    c = (R - 1) / 2
    th[:, 0] = c - 1 + 2 * u()
    th[:, 1] = c - 1 + 2 * u()
    names = est.param_names
    for k, name in enumerate(names):
        if name == "I":
            th[:, k] = torch.exp(math.log(300) + (math.log(8000) - math.log(300)) * u())
        elif name == "bg":
            th[:, k] = 1 + 15 * u()
        elif name in ("sigma", "sx", "sy"):
            th[:, k] = 1.2 + 1.0 * u()
        elif name == "z":
            mid, half = (float(lo[k]) + float(hi[k])) / 2, (float(hi[k]) - float(lo[k])) / 2
            th[:, k] = mid + half * 0.6 * (2 * u() - 1)
    consts = None
    if est.numconst:
        consts = (1.2 + 0.6 * torch.rand((n, est.numconst), device="cuda", generator=g)).contiguous()
    ev = est.ExpectedValueDevice(th.contiguous(), constants=consts)
    return torch.poisson(ev, generator=g).contiguous(), consts


def tune_estimator(est, samples=None, constants=None, n=65536, reps=3, use_cache=True, write_cache=True,
                   cache_file=None):
    """Time every candidate kernel configuration for `est`, apply the fastest and return
    dict(config=(variant, lanes, threads), ms=..., timings={...}, cached=bool)."""
    import torch
    from .autograd import model_id
    model = model_id(est)
    R = int(est.sampleshape[0])
    lm = est.GetLevMarParams()
    gpu = torch.cuda.get_device_name()
    key = estimator_key(gpu, model, R, lm.iterations, lm.lambda_)
    with _lock:
        cache = load_cache(cache_file) if use_cache else {}
    if use_cache and key in cache:
        v, g, t = cache[key]["config"]
        est.SetKernelConfig(g, t, variant=v)
        return dict(config=(v, g, t), ms=cache[key]["ms"], timings=None, cached=True)
    if samples is None:
        samples, constants = _synthetic_rois(est, n)
    timings = {}
    for v, g, t in candidates(model, R):
        try:
            est.SetKernelConfig(g, t, variant=v)
            for _ in range(2):
                est.EstimateDevice(samples, constants=constants, with_crlb=True)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record()
            for _ in range(reps):
                est.EstimateDevice(samples, constants=constants, with_crlb=True)
            e1.record()
            e1.synchronize()
            timings[(v, g, t)] = e0.elapsed_time(e1) / reps
        except Exception:
            timings[(v, g, t)] = None
    (v, g, t), ms = choose_best(timings)
    est.SetKernelConfig(g, t, variant=v)
    if write_cache:
        with _lock:
            cache = load_cache(cache_file)
            cache[key] = dict(config=[v, g, t], ms=ms)
            save_cache(cache, cache_file)
    return dict(config=(v, g, t), ms=ms, timings={str(k): ms_ for k, ms_ in timings.items()}, cached=False)


def tune_mixed(buckets, tiles=(1, 2, 4, 8), budgets=(256, 129, 128), reps=3, standalone_mins=(0, None)):
    """Time MixedBatch configurations for these buckets: for each threshold of standalone_mins
    (ROIs per SM from which a bucket runs as launches of its own; None = every bucket in the
    persistent mixed kernel), the persistent kernel's claim sizes and register budgets when it
    has buckets. Returns dict(standalone_min=..., tile=..., threads=..., ms=..., timings={...});
    the caller calls mixed.set_standalone_min(standalone_min) and builds its MixedBatch with
    tile and threads. The process-wide threshold is restored before returning."""
    import torch
    from .mixed import MixedBatch, set_standalone_min, standalone_min
    never = 1 << 30
    saved = standalone_min()
    s = torch.cuda.Stream()
    timings = {}
    try:
        with torch.cuda.stream(s):
            for smin in standalone_mins:
                set_standalone_min(never if smin is None else smin)
                for thr in budgets:
                    for tile in tiles:
                        mb = MixedBatch(buckets, tile_rois=tile, threads=thr)
                        all_alone = all(mb.standalone())
                        try:
                            _time_mixed(mb, s, reps, timings, (smin, tile, thr))
                        finally:
                            mb.close()
                        if all_alone:  # no bucket in the persistent kernel: tile and budget do not matter
                            break
                    if all_alone:
                        break
    finally:
        set_standalone_min(saved)
    (smin, tile, thr), ms = choose_best(timings)
    return dict(standalone_min=never if smin is None else smin, tile=tile, threads=thr, ms=ms,
                timings={str(k): v for k, v in timings.items()})


def _time_mixed(mb, s, reps, timings, key):
    import torch
    mb.run(s)
    s.synchronize()
    mb.capture(s)
    for _ in range(2):
        mb.run(s)
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record(s)
    for _ in range(reps):
        mb.run(s)
    e1.record(s)
    e1.synchronize()
    timings[key] = e0.elapsed_time(e1) / reps
