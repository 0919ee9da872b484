"""photonpy's own Python binding, unmodified, over libphotonpy_b200.so.

oracle/build_ref.sh copies photonpy's `photonpy/cpp/{lib,context,estimator,gaussian,cspline,
estim_queue}.py` next to the reference build (oracle/_ref/photonpy_cpp, git-ignored). This test
puts them in a throw-away `photonpy.cpp` package with empty package `__init__` stubs (photonpy's
own `photonpy/__init__.py` imports its whole SMLM pipeline) and places this library at the path
photonpy's loader opens (`photonpy/x64/Release/photonpy.dll`, photonpy/cpp/lib.py:41-66), so
not a line of photonpy's binding changes. `matplotlib.pyplot`, which photonpy/cpp/lib.py imports
for plotting only, is not installed here and is stubbed. photonpy's `SMLM.Close` frees the
library through `ctypes.windll` (Windows only), so the context is built on an SMLM object it
does not own, as photonpy's API allows (photonpy/cpp/context.py:11-14).

Through that binding the golden sets are fitted (Estimate), and CRLBAndChiSquare,
ExpectedValue, Derivatives, the spline coefficients (ComputeSplineCoeff) and the estimation
queue (EstimQueue) are run; every result must equal this package's own binding bit for bit.
"""
import importlib
import os
import shutil
import sys
import types

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PY_SRC = os.path.join(ROOT, "oracle", "_ref", "photonpy_cpp")


@pytest.fixture(scope="module")
def photonpy(tmp_path_factory):
    if not os.path.isdir(PY_SRC):
        pytest.skip("photonpy's binding is not beside the reference build (run oracle/build_ref.sh)")
    import photonpy_b200 as pb
    base = tmp_path_factory.mktemp("photonpy_dropin")
    pkg = base / "photonpy"
    cpp = pkg / "cpp"
    rel = pkg / "x64" / "Release"
    cpp.mkdir(parents=True)
    rel.mkdir(parents=True)
    (pkg / "__init__.py").write_text("")
    (cpp / "__init__.py").write_text("")
    for f in sorted(os.listdir(PY_SRC)):
        if f.endswith(".py"):
            shutil.copy(os.path.join(PY_SRC, f), cpp / f)
    os.symlink(pb.library_path(), rel / "photonpy.dll")
    saved = {k: v for k, v in sys.modules.items() if k.split(".")[0] in ("photonpy", "matplotlib")}
    for k in saved:
        del sys.modules[k]
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.path.insert(0, str(base))
    try:
        mods = types.SimpleNamespace(**{m: importlib.import_module("photonpy.cpp." + m) for m in
                                        ("lib", "context", "estimator", "gaussian", "cspline", "estim_queue")})
        mods.smlm = mods.lib.SMLM()
        assert os.path.samefile(mods.smlm.lib_path, pb.library_path())
        yield mods
    finally:
        sys.path.remove(str(base))
        for k in [k for k in sys.modules if k.split(".")[0] in ("photonpy", "matplotlib")]:
            del sys.modules[k]
        sys.modules.update(saved)


def _pair(photonpy, ctx, name, g):
    """(photonpy's binding, this package's binding) estimators of one golden set."""
    import photonpy_b200 as pb
    rctx = photonpy.context.Context(photonpy.smlm)
    R = int(g["roisize"])
    if name.startswith("sigmaxy"):
        a = photonpy.gaussian.GaussianPSFMethods(rctx).CreatePSF_XYIBgSigmaXY(R, list(g["sigma"]), True)
        b = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(R, tuple(g["sigma"]), True)
    elif name.startswith("xyibg"):
        a = photonpy.gaussian.GaussianPSFMethods(rctx).CreatePSF_XYIBg(R, tuple(g["sigma"]), True)
        b = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(R, tuple(g["sigma"]), True)
    elif name.startswith("astig"):
        ca = photonpy.gaussian.Gauss3D_Calibration(list(g["astig_x"][:4]), list(g["astig_y"][:4]), list(g["zrange"]))
        cb = pb.Gauss3D_Calibration(list(g["astig_x"][:4]), list(g["astig_y"][:4]), list(g["zrange"]))
        a = photonpy.gaussian.GaussianPSFMethods(rctx).CreatePSF_XYZIBg(R, ca, True)
        b = pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(R, cb, True)
    elif name.startswith("spline"):
        sa = photonpy.cspline.CSplineMethods(rctx)
        sb = pb.CSplineMethods(ctx)
        coefs_a = sa.ComputeSplineCoeff(g["zstack"], border=1)
        coefs_b = sb.ComputeSplineCoeff(g["zstack"], border=1)
        assert np.array_equal(coefs_a, coefs_b)
        zr = g["spline_zrange"]
        ca = photonpy.cspline.CSplineCalibration(float(zr[0]), float(zr[1]), coefs_a)
        cb = pb.CSplineCalibration(float(zr[0]), float(zr[1]), coefs_b)
        a = sa.CreatePSF_XYZIBg(R, ca, sa.FlatBg, True)
        b = sb.CreatePSF_XYZIBg(R, cb, sb.FlatBg, True)
        a._keep, b._keep = ca, cb
    else:
        raise KeyError(name)
    return rctx, a, b


@pytest.mark.parametrize("name", ["xyibg_r10", "sigmaxy_r16", "astig_r12", "spline_r13"])
def test_photonpy_binding_equals_package_binding(photonpy, ctx, name):
    g = load_golden(name)
    rctx, a, b = _pair(photonpy, ctx, name, g)
    assert a.param_names == b.param_names and a.numparams == b.numparams
    assert np.array_equal(a.limits, b.limits)
    smp = g["samples"]
    pa, da, ta = a.Estimate(smp)
    pb_, db, tb, its = b.Estimate(smp, return_iterations=True)
    assert np.array_equal(pa, pb_)
    assert da.shape == db.shape == (len(smp), 0)
    assert [len(t) for t in ta] == list(np.minimum(its, 50))
    assert all(np.array_equal(x, y) for x, y in zip(ta, tb))
    ca, xa = a.CRLBAndChiSquare(pa, smp)
    cb, xb = b.CRLBAndChiSquare(pa, smp)
    assert np.array_equal(ca, cb) and np.array_equal(xa, xb)
    assert np.all(np.isfinite(ca))
    truth = g["truth"][:16]
    assert np.array_equal(a.ExpectedValue(truth), b.ExpectedValue(truth))
    dA, eA = a.Derivatives(truth)
    dB, eB = b.Derivatives(truth)
    assert np.array_equal(dA, dB) and np.array_equal(eA, eB)
    # the golden reference fit, for scale: converged positions within 1e-3 px of photonpy's CPU
    conv = (g["iterations"] <= 50) & (its <= 50)
    assert np.quantile(np.abs(pa[conv, :2] - g["params"][conv, :2]).max(1), 0.95) < 1e-3
    a.Destroy()
    b.Destroy()
    rctx.Destroy()


def test_photonpy_estim_queue_equals_direct_fit(photonpy, ctx):
    g = load_golden("sigmaxy_r16")
    rctx, a, b = _pair(photonpy, ctx, "sigmaxy_r16", g)
    smp = g["samples"]
    n = len(smp)
    direct, _, _ = a.Estimate(smp)
    crlb_direct = b.CRLBAndChiSquare(direct, smp)[0]
    q = photonpy.estim_queue.EstimQueue(a, batchSize=64, maxQueueLenInBatches=1 << 20)
    ids = np.arange(n, dtype=np.int32)[::-1].copy()
    q.Schedule(smp[::-1], ids=ids)
    q.WaitUntilDone()
    r = q.GetResults()
    assert len(r.ids) == n
    order = np.argsort(r.ids)
    assert np.array_equal(r.ids[order], np.arange(n))
    assert np.array_equal(r.estim[order], direct)
    assert np.array_equal(r.crlb[order], crlb_direct)
    q.Destroy()
    a.Destroy()
    b.Destroy()
    rctx.Destroy()
