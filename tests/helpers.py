"""Shared test helpers: build the CUDA estimator and the oracle model for a golden set."""
import hashlib

import numpy as np

from oracle import oracle as O


def oracle_model(name, g):
    R = int(g["roisize"])
    if name.startswith("xyibg"):
        return O.Model(O.XYIBG, R, sigma=tuple(g["sigma"]))
    if name.startswith("constsigma"):
        return O.Model(O.XYIBG_CONSTSIGMA, R)
    if name.startswith("sigma_"):
        return O.Model(O.XYIBG_SIGMA, R, sigma=tuple(g["sigma"]))
    if name.startswith("sigmaxy"):
        return O.Model(O.XYIBG_SIGMAXY, R, sigma=tuple(g["sigma"]))
    if name.startswith("astig"):
        return O.Model(O.XYZIBG, R, astig_x=g["astig_x"], astig_y=g["astig_y"], zrange=tuple(g["zrange"]))
    if name.startswith("spline"):
        coefs = O.spline_compute(g["zstack"], border=1)
        mid = O.CSPLINE_TILTED if "tilted" in name else (O.CSPLINE_BGIMAGE if "bgimage" in name else O.CSPLINE)
        return O.Model(mid, R, coefs=coefs, spline_zrange=tuple(g["spline_zrange"]))
    if name.startswith("tiltedbg"):
        return O.Model(O.XYITILTEDBG, R)
    if name.startswith("tiltedsxy"):
        return O.Model(O.XYITILTEDBG_SIGMAXY, R, sigma=tuple(g["sigma"]))
    raise KeyError(name)


def cuda_estimator(name, g, ctx):
    import photonpy_b200 as pb
    R = int(g["roisize"])
    if name.startswith("xyibg"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(R, tuple(g["sigma"]), True)
    if name.startswith("constsigma"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(R, None, True)
    if name.startswith("sigma_"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigma(R, float(g["sigma"][0]), True)
    if name.startswith("sigmaxy"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(R, tuple(g["sigma"]), True)
    if name.startswith("astig"):
        c = pb.Gauss3D_Calibration(list(g["astig_x"][:4]), list(g["astig_y"][:4]), list(g["zrange"]))
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(R, c, True)
    if name.startswith("spline"):
        sm = pb.CSplineMethods(ctx)
        coefs = sm.ComputeSplineCoeff(g["zstack"], border=1)
        calib = pb.CSplineCalibration(float(g["spline_zrange"][0]), float(g["spline_zrange"][1]), coefs)
        mode = sm.TiltedBg if "tilted" in name else (sm.BgImage if "bgimage" in name else sm.FlatBg)
        est = sm.CreatePSF_XYZIBg(R, calib, mode, True)
        est._keep = calib
        return est
    if name.startswith("tiltedbg"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYITiltedBg(R, True)
    if name.startswith("tiltedsxy"):
        return pb.GaussianPSFMethods(ctx).CreatePSF_XYITiltedBgSigmaXY(R, tuple(g["sigma"]), True)
    raise KeyError(name)


def coefs_sha(coefs):
    return hashlib.sha256(np.ascontiguousarray(coefs, dtype=np.float32).tobytes()).hexdigest()


def pos_tol(name):
    """Position tolerance: 1e-3 px for x/y; z: 1 nm (astig, z in nm) or 1e-3 um (spline)."""
    if name.startswith("astig"):
        return np.array([1e-3, 1e-3, 1.0])
    if name.startswith("spline"):
        return np.array([1e-3, 1e-3, 1e-3])
    return np.array([1e-3, 1e-3])


def split_params(name, K):
    """indices of (position params, photometric params I/bg)"""
    if name.startswith("astig") or name.startswith("spline"):
        return [0, 1, 2], [3, 4]
    return [0, 1], [2, 3]


def parity_stats(name, ref_params, ref_its, params, its, maxit=50):
    """Agreement of one result set with the reference, stratified by converged/capped."""
    pos, phot = split_params(name, ref_params.shape[1])
    tol = pos_tol(name)
    dpos = np.abs(params[:, pos] - ref_params[:, pos])
    pos_ok = np.all(dpos <= tol[None, :], axis=1)
    rel = np.abs(params[:, phot] - ref_params[:, phot]) / np.maximum(np.abs(ref_params[:, phot]), 1e-6)
    phot_ok = np.all(rel <= 1e-4, axis=1)
    conv_ref = ref_its <= maxit
    conv = its <= maxit
    both = conv_ref & conv
    return dict(
        n=len(its),
        it_match=float(np.mean(its == ref_its)),
        conv_flag_match=float(np.mean(conv == conv_ref)),
        pos_ok=float(np.mean(pos_ok)),
        phot_ok=float(np.mean(phot_ok)),
        pos_ok_converged=float(np.mean(pos_ok[both])) if both.any() else 1.0,
        phot_ok_converged=float(np.mean(phot_ok[both])) if both.any() else 1.0,
        frac_capped_ref=float(np.mean(~conv_ref)),
        max_dpos_converged=float(dpos[both].max()) if both.any() else 0.0,
    )


def ref_estimator(name, g, cuda):
    """The reference's own estimator (oracle/_ref build) for a golden set; cuda selects its GPU
    kernels, else its CPU path (the one the golden vectors come from)."""
    from oracle import ref_lib
    R = int(g["roisize"])
    if name.startswith("xyibg"):
        return ref_lib.RefEstimator("XYIBg", R, cuda=cuda, sigma=tuple(g["sigma"]))
    if name.startswith("constsigma"):
        return ref_lib.RefEstimator("XYIBgConstSigma", R, cuda=cuda)
    if name.startswith("sigma_"):
        return ref_lib.RefEstimator("XYIBgSigma", R, cuda=cuda, sigma=tuple(g["sigma"]))
    if name.startswith("sigmaxy"):
        return ref_lib.RefEstimator("XYIBgSigmaXY", R, cuda=cuda, sigma=tuple(g["sigma"]))
    if name.startswith("astig"):
        return ref_lib.RefEstimator("XYZIBg", R, cuda=cuda, astig=(g["astig_x"][:4], g["astig_y"][:4]),
                                    zrange=tuple(g["zrange"]))
    if name.startswith("spline"):
        mode = 1 if "tilted" in name else (2 if "bgimage" in name else 0)
        coefs = ref_lib.spline_compute(g["zstack"], border=1)
        return ref_lib.RefEstimator("CSpline", R, cuda=cuda, coefs=coefs, spline_zrange=tuple(g["spline_zrange"]),
                                    spline_mode=mode)
    if name.startswith("tiltedbg"):
        return ref_lib.RefEstimator("XYITiltedBg", R, cuda=cuda)
    if name.startswith("tiltedsxy"):
        return ref_lib.RefEstimator("XYITiltedBgSigmaXY", R, cuda=cuda, sigma=tuple(g["sigma"]))
    raise KeyError(name)


def ref_fit(est, samples, constants=None, chunk=20000):
    """(params, iterations) of a reference estimator, in chunks (its CPU path starts one thread
    per spot)."""
    ps, its = [], []
    for s in range(0, len(samples), chunk):
        c = None if constants is None else constants[s:s + chunk]
        p, it, _ = est.estimate(samples[s:s + chunk], constants=c, trace_len=0)
        ps.append(p)
        its.append(it)
    return np.concatenate(ps), np.concatenate(its)


# Benchmark workloads as parity cases: XYIBg 10x10, XYIBgSigmaXY 16x16, astigmatic XYZIBg 12x12
# and the cubic spline 13x13 on a 26x26x41 z-stack, drawn as the benchmark draws them.
SYNTHETIC = ["xyibg_10", "sigmaxy_16", "astig_12", "spline_13"]


def synthetic_case(name, n):
    """Seeded ROIs of a benchmark workload, in the layout of a golden set (without the
    reference's fit, which the caller adds)."""
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    if name == "xyibg_10":
        d = synth.xyibg(n, seed=1)
        return dict(samples=d["samples"], roisize=d["R"], sigma=np.float32(d["sigma"]))
    if name == "sigmaxy_16":
        d = synth.sigmaxy(n, seed=2)
        return dict(samples=d["samples"], roisize=d["R"], sigma=np.float32(d["sigma"]))
    if name == "astig_12":
        d = synth.astig(n, seed=3)
        cx, cy = d["astig"]
        return dict(samples=d["samples"], roisize=d["R"], astig_x=np.float32(cx), astig_y=np.float32(cy),
                    zrange=np.float32(d["zrange"]))
    if name == "spline_13":
        d = synth.spline(n, seed=4)
        zstack, zr = synth.astig_zstack(shape_xy=26, nz=41, zrange_um=(-0.4, 0.4))
        return dict(samples=d["samples"], roisize=d["R"], zstack=zstack, spline_zrange=np.float32(zr))
    raise KeyError(name)


def golden_name(case):
    """Golden-set name whose estimator factory fits a synthetic case."""
    return {"xyibg_10": "xyibg_r10", "sigmaxy_16": "sigmaxy_r16", "astig_12": "astig_r12",
            "spline_13": "spline_r13"}.get(case, case)
