"""Generate the golden fixtures in tests/golden/ from the reference's own CPU estimator.

Run in a container that has the reference sources (the GPU box does not):
    oracle/build_ref.sh            # builds oracle/_ref/libphotonpy_ref.so from the reference
    python tests/golden/make_golden.py

Inputs are seeded synthetic ROIs (photonpy_b200.synth). Every output array is what the
reference's C ABI (Estimator_Estimate, Estimator_ChiSquareAndCRLB,
Estimator_ComputeDerivatives, CSpline_Compute; cuda=False) returned for them, with the
Python API's default LM settings (lambda 1e-18, 50 iterations; estimator.py:151).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_lib  # noqa: E402
from photonpy_b200 import synth  # noqa: E402

N_TRACE = 40
N_DERIV = 16


def _fit_and_save(name, est, data, constants=None, extra=None):
    smp = data["samples"]
    params, its, trace = est.estimate(smp, constants=constants, trace_len=50)
    crlb, chisq = est.crlb_chisq(params, smp, constants=constants)
    crlb_truth, _ = est.crlb_chisq(data["truth"], None, constants=constants)
    deriv, ev = est.derivatives(data["truth"][:N_DERIV], constants=None if constants is None else constants[:N_DERIV])
    out = dict(samples=smp, truth=data["truth"], params=params, iterations=its, trace=trace[:N_TRACE],
               crlb=crlb, chisq=chisq, crlb_truth=crlb_truth, deriv=deriv, ev=ev, roisize=np.int32(data["R"]))
    if constants is not None:
        out["constants"] = constants
    out.update(extra or {})
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    capped = float(np.mean(its > 50))
    print(f"{name}: n={len(smp)} mean it={its.mean():.2f} capped={capped:.3f}")


def main(only=None):
    """Writes every golden set, or only those named in `only`."""
    if not ref_lib.available():
        raise SystemExit("build the reference first: oracle/build_ref.sh")
    want = (lambda name: only is None or name in only)
    if want("tiltedbg_r11"):
        d = synth.tilted(300, seed=113)
        e = ref_lib.RefEstimator("XYITiltedBg", d["R"])
        _fit_and_save("tiltedbg_r11", e, d, constants=d["constants"])
    if want("tiltedsxy_r11"):
        d = synth.tilted(300, seed=114, free_sigma=True)
        e = ref_lib.RefEstimator("XYITiltedBgSigmaXY", d["R"], sigma=d["sigma"])
        _fit_and_save("tiltedsxy_r11", e, d, extra=dict(sigma=np.float32(d["sigma"])))
    if want("spline_tilted_r13") or want("spline_bgimage_r13"):
        # the spline modes CSPLINE_TILTEDBG (1) and CSPLINE_BGIMAGE (2) on the spline_r13 calibration
        zstack, zr = synth.astig_zstack(shape_xy=24, nz=21, zrange_um=(-0.4, 0.4))
        coefs = ref_lib.spline_compute(zstack, border=1)
        if want("spline_tilted_r13"):
            d = synth.spline_background(300, "tilted", seed=118)
            e = ref_lib.RefEstimator("CSpline", d["R"], coefs=coefs, spline_zrange=zr, spline_mode=1)
            _fit_and_save("spline_tilted_r13", e, d, extra=dict(zstack=zstack, spline_zrange=np.float32(zr)))
        if want("spline_bgimage_r13"):
            d = synth.spline_background(300, "bgimage", seed=119)
            e = ref_lib.RefEstimator("CSpline", d["R"], coefs=coefs, spline_zrange=zr, spline_mode=2)
            _fit_and_save("spline_bgimage_r13", e, d, constants=d["constants"],
                          extra=dict(zstack=zstack, spline_zrange=np.float32(zr)))
    if want("intensitybg_r9"):
        # Gauss2D_EstimateIntensityBg: spots at known positions; sigma given per spot as [n][2]
        # with distinct values, so the reference's flat indexing of it (GaussianPSF.cu:225) is pinned
        d = synth.xyibg(300, seed=115, R=9, xy=(3.0, 5.0))
        rng = np.random.default_rng(116)
        sig = rng.uniform(1.3, 1.7, size=(300, 2)).astype(np.float32)
        xy = d["truth"][:, :2] + rng.normal(0, 0.05, size=(300, 2)).astype(np.float32)
        ibg, crlb = ref_lib.estimate_intensity_bg(d["samples"], xy, sig, 100)
        np.savez_compressed(os.path.join(HERE, "intensitybg_r9.npz"), samples=d["samples"], truth=d["truth"],
                            xy=xy.astype(np.float32), sigma=sig, ibg=ibg, ibg_crlb=crlb, max_iterations=np.int32(100),
                            roisize=np.int32(9))
        print(f"intensitybg_r9: n=300 I mean={ibg[:, 0].mean():.1f}")
    if only is not None and not ({"xyibg_r10", "constsigma_r9", "sigma_r11", "sigmaxy_r16", "astig_r12",
                                  "spline_r13"} & set(only)):
        return

    d = synth.xyibg(400, seed=101)
    e = ref_lib.RefEstimator("XYIBg", d["R"], sigma=d["sigma"])
    _fit_and_save("xyibg_r10", e, d, extra=dict(sigma=np.float32(d["sigma"])))

    d = synth.constsigma(300, seed=111)
    e = ref_lib.RefEstimator("XYIBgConstSigma", d["R"])
    _fit_and_save("constsigma_r9", e, d, constants=d["constants"])

    d = synth.sigma1(300, seed=112)
    e = ref_lib.RefEstimator("XYIBgSigma", d["R"], sigma=d["sigma"])
    _fit_and_save("sigma_r11", e, d, extra=dict(sigma=np.float32(d["sigma"])))

    d = synth.sigmaxy(400, seed=102)
    e = ref_lib.RefEstimator("XYIBgSigmaXY", d["R"], sigma=d["sigma"])
    _fit_and_save("sigmaxy_r16", e, d, extra=dict(sigma=np.float32(d["sigma"])))

    d = synth.astig(400, seed=103)
    cx, cy = d["astig"]
    zr = d["zrange"]
    e = ref_lib.RefEstimator("XYZIBg", d["R"], astig=(cx[:4], cy[:4]), zrange=zr)
    _fit_and_save("astig_r12", e, d, extra=dict(astig_x=np.float32(cx), astig_y=np.float32(cy),
                                                zrange=np.float32(zr)))

    # Cubic spline: z-stack of the astig model (z in um), coefficients by the reference's
    # CSpline_Compute with border 1 (one voxel per ROI pixel, one spline segment per z step).
    zstack, zr = synth.astig_zstack(shape_xy=24, nz=21, zrange_um=(-0.4, 0.4))
    coefs = ref_lib.spline_compute(zstack, border=1)
    rng = np.random.default_rng(7)
    pick = rng.choice(coefs.size, 4096, replace=False)
    d = synth.spline(300, seed=104)
    e = ref_lib.RefEstimator("CSpline", d["R"], coefs=coefs, spline_zrange=zr)
    _fit_and_save("spline_r13", e, d, extra=dict(
        zstack=zstack, spline_zrange=np.float32(zr), coefs_sha256=np.bytes_(hashlib.sha256(coefs.tobytes()).hexdigest()),
        coefs_shape=np.int32(coefs.shape), coefs_pick=pick.astype(np.int64), coefs_pick_values=coefs.reshape(-1)[pick]))


if __name__ == "__main__":
    main(sys.argv[1:] or None)
