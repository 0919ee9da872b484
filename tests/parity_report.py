"""Parity report of the CUDA estimator against the reference's own estimator (needs a GPU).

    python tests/parity_report.py [--synthetic N] [--json out.json] [--variant V] [--lanes G]
                                  [--cache ref.npz]

Cases: every golden set (tests/golden/*.npz, fitted by the reference's C++ CPU estimator) and,
with --synthetic N, N seeded ROIs of each benchmark workload (XYIBg 10x10, XYIBgSigmaXY 16x16,
astigmatic XYZIBg 12x12, cubic spline 13x13) fitted here by the reference's CPU build
(oracle/_ref; --cache keeps those fits between runs).

For every case it reports, against the reference CPU fit and stratified by converged / capped
(reference iteration count <= 50):
  * this library: iteration-count match, converged-flag match, converged spots with positions
    within 1e-3 px (z: 1 nm astig, 1e-3 um spline) and I/bg within 1e-4 relative;
  * the floor: the same statistics for the reference's own CUDA build (its one-thread-per-ROI
    kernels, oracle/_ref with cuda=True) against its CPU build -- how much the reference's
    results move from rounding alone (CUDA's erff/expf, FMA contraction);
  * golden sets only: CRLB within 1e-4 relative at the reference's parameters, and the
    90th-percentile position error against the FP64 oracle (same algorithm in double precision,
    iterated to its own convergence) of the reference and of this library.
The kernel variant and lanes per ROI can be chosen (SetKernelConfig), and the library build with
PHOTONPY_B200_LIBRARY. tests/test_gpu_parity.py asserts floors on the same statistics.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import GOLDEN_SETS, load_golden  # noqa: E402
from helpers import (SYNTHETIC, cuda_estimator, golden_name, oracle_model, parity_stats, ref_estimator,  # noqa: E402
                     ref_fit, split_params, synthetic_case)


def load_cases(synthetic_n, cache):
    cases = [(name, load_golden(name), True) for name in GOLDEN_SETS]
    if synthetic_n:
        cached = dict(np.load(cache, allow_pickle=False)) if cache and os.path.exists(cache) else {}
        store = {}
        for name in SYNTHETIC:
            g = synthetic_case(name, synthetic_n)
            key = f"{name}_{synthetic_n}"
            if key + "_params" in cached:
                g["params"], g["iterations"] = cached[key + "_params"], cached[key + "_iterations"]
            else:
                est = ref_estimator(golden_name(name), g, cuda=False)
                t0 = time.perf_counter()
                g["params"], g["iterations"] = ref_fit(est, g["samples"])
                print(f"# reference CPU fit of {name}: {synthetic_n} ROIs in {time.perf_counter() - t0:.1f} s",
                      file=sys.stderr)
                est.close()
            store[key + "_params"], store[key + "_iterations"] = g["params"], g["iterations"]
            cases.append((name, g, False))
        if cache:
            np.savez(cache, **{**cached, **store})
    return cases


def report(ctx, synthetic_n=0, variant=None, lanes=0, ref_gpu=True, cache=None):
    from oracle import ref_lib
    ref_gpu = ref_gpu and ref_lib.available()
    out = {}
    for name, g, golden in load_cases(synthetic_n, cache):
        gname = golden_name(name)
        est = cuda_estimator(gname, g, ctx)
        if variant is not None or lanes:
            est.SetKernelConfig(lanes, 0, variant=variant)
        c = g.get("constants")
        params, _, _, its = est.Estimate(g["samples"], constants=c, return_iterations=True)
        row = dict(n=len(its), ours=parity_stats(gname, g["params"], g["iterations"], params, its),
                   kernel_config=list(est.GetKernelConfig()))
        if ref_gpu:
            rg = ref_estimator(gname, g, cuda=True)
            p_gpu, it_gpu = ref_fit(rg, g["samples"], constants=c, chunk=1 << 20)
            rg.close()
            row["ref_gpu"] = parity_stats(gname, g["params"], g["iterations"], p_gpu, it_gpu)
            row["ours_vs_ref_gpu"] = parity_stats(gname, p_gpu, it_gpu, params, its)
        if golden:
            crlb, _ = est.CRLBAndChiSquare(g["params"], g["samples"], constants=c)
            row["crlb_ok"] = float(np.mean(np.all(np.abs(crlb - g["crlb"]) <= 1e-4 * np.abs(g["crlb"]), axis=1)))
            m = oracle_model(name, g)
            p64, it64 = m.fit(g["samples"], constants=c, fp64=True, iterations=200, lambda_=1e-18)
            pos, _ = split_params(name, params.shape[1])
            both = (g["iterations"] <= 50) & (its <= 50) & (it64 <= 200)
            q = (lambda e: float(np.quantile(e, 0.9)) if e.size else None)
            row["p90_fp64_ref"] = q(np.abs(g["params"][both][:, pos] - p64[both][:, pos]).max(axis=1))
            row["p90_fp64_ours"] = q(np.abs(params[both][:, pos] - p64[both][:, pos]).max(axis=1))
        out[name] = row
        est.Destroy()
    return out


def markdown(rows):
    pct = (lambda v: "-" if v is None else f"{100 * v:.2f}%")
    lines = ["| case | spots | ref capped | iteration match | floor: ref GPU it-match | converged flag match | "
             "floor: ref GPU flag match | converged: pos ok | converged: I/bg ok | CRLB within 1e-4 | "
             "p90 pos err vs FP64: ref / ours |",
             "|---|---|---|---|---|---|---|---|---|---|---|"]
    for name, r in rows.items():
        o, f = r["ours"], r.get("ref_gpu", {})
        fp = "-" if r.get("p90_fp64_ref") is None else f"{r['p90_fp64_ref']:.2e} / {r['p90_fp64_ours']:.2e}"
        lines.append(f"| {name} | {r['n']} | {pct(o['frac_capped_ref'])} | {pct(o['it_match'])} | "
                     f"{pct(f.get('it_match'))} | {pct(o['conv_flag_match'])} | {pct(f.get('conv_flag_match'))} | "
                     f"{pct(o['pos_ok_converged'])} | {pct(o['phot_ok_converged'])} | {pct(r.get('crlb_ok'))} | {fp} |")
    return "\n".join(lines)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--synthetic", type=int, default=0, help="ROIs per benchmark workload (0: golden sets only)")
    ap.add_argument("--json", default=None)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--cache", default=None, help="npz file keeping the reference CPU fits of the synthetic cases")
    ap.add_argument("--no-ref-gpu", action="store_true")
    a = ap.parse_args()
    import photonpy_b200 as pb
    ctx = pb.Context()
    rows = report(ctx, a.synthetic, a.variant, a.lanes, not a.no_ref_gpu, a.cache)
    ctx.Destroy()
    print(markdown(rows))
    if a.json:
        json.dump(dict(library=pb.library_path(), variant=a.variant, lanes=a.lanes, rows=rows), open(a.json, "w"),
                  indent=1)
