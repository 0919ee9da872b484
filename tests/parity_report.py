"""Parity report of the CUDA estimator against the reference's golden vectors (needs a GPU).

    python tests/parity_report.py            # markdown table on stdout

For every golden set (tests/golden/*.npz, produced by the reference's own C++ CPU estimator)
it fits the same ROIs with the CUDA path and reports, stratified by converged / capped
(reference iteration count <= 50):
  * iteration-count match and converged-flag match,
  * converged spots with positions within 1e-3 px (z: 1 nm astig, 1e-3 um spline) and I/bg
    within 1e-4 relative, and the largest position difference,
  * CRLB within 1e-4 relative (at the reference's parameters),
  * the 90th-percentile position error against the FP64 oracle (same algorithm in double
    precision, iterated to its own convergence) of the reference and of the CUDA path, over the
    spots all three converged on ("-" when there are none).
It is the source of the parity table of the design notes; tests/test_gpu_parity.py asserts
floors on the same statistics.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import GOLDEN_SETS, load_golden  # noqa: E402
from helpers import cuda_estimator, oracle_model, parity_stats, split_params  # noqa: E402


def report(ctx):
    rows = []
    for name in GOLDEN_SETS:
        g = load_golden(name)
        est = cuda_estimator(name, g, ctx)
        c = g.get("constants")
        params, _, _, its = est.Estimate(g["samples"], constants=c, return_iterations=True)
        st = parity_stats(name, g["params"], g["iterations"], params, its)
        crlb, _ = est.CRLBAndChiSquare(g["params"], g["samples"], constants=c)
        crlb_ok = float(np.mean(np.all(np.abs(crlb - g["crlb"]) <= 1e-4 * np.abs(g["crlb"]), axis=1)))
        m = oracle_model(name, g)
        p64, it64 = m.fit(g["samples"], constants=c, fp64=True, iterations=200, lambda_=1e-18)
        pos, _ = split_params(name, params.shape[1])
        both = (g["iterations"] <= 50) & (its <= 50) & (it64 <= 200)
        e_ref = np.abs(g["params"][both][:, pos] - p64[both][:, pos]).max(axis=1)
        e_cuda = np.abs(params[both][:, pos] - p64[both][:, pos]).max(axis=1)
        q = (lambda e: float(np.quantile(e, 0.9)) if e.size else float("nan"))
        rows.append((name, st, crlb_ok, q(e_ref), q(e_cuda)))
        est.Destroy()
    out = ["| golden set | spots | ref capped | iteration match | converged flag match | converged: pos ok | "
           "converged: I/bg ok | max pos diff (converged) | CRLB within 1e-4 | p90 pos err vs FP64: ref | "
           "p90 pos err vs FP64: CUDA |",
           "|---|---|---|---|---|---|---|---|---|---|---|"]
    for name, st, cok, er, ec in rows:
        out.append(f"| {name} | {st['n']} | {100 * st['frac_capped_ref']:.1f}% | {100 * st['it_match']:.2f}% | "
                   f"{100 * st['conv_flag_match']:.2f}% | {100 * st['pos_ok_converged']:.2f}% | "
                   f"{100 * st['phot_ok_converged']:.2f}% | {st['max_dpos_converged']:.2e} | {100 * cok:.1f}% | "
                   f"{'-' if er != er else f'{er:.2e}'} | {'-' if ec != ec else f'{ec:.2e}'} |")
    return "\n".join(out)


if __name__ == "__main__":
    import photonpy_b200 as pb
    ctx = pb.Context()
    print(report(ctx))
    ctx.Destroy()
