"""Fisher matrix and CRLB entry points on the GPU against the FP64 oracle.

Estimator.FisherMatrix runs the fit kernels' Fisher pass (FP32 sums) and Estimator.CRLB inverts
it in FP64 on the GPU; photonpy computes both in numpy from downloaded derivative stacks
(photonpy/cpp/estimator.py:205-220, 249-253). The FP64 oracle restates the same sums and the
reference's LUP inverse in double precision (oracle/psf_oracle_impl.h, ComputeChiSquareAndCRLB).
NumDeriv / NumCRLB are checked against the analytic Derivatives / CRLB they approximate.
"""
import numpy as np
import pytest

from conftest import GOLDEN_SETS, load_golden
from helpers import cuda_estimator, oracle_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", GOLDEN_SETS)
def test_fisher_matrix_and_crlb_match_fp64_oracle(name, ctx):
    g = load_golden(name)
    est = cuda_estimator(name, g, ctx)
    c = g.get("constants")
    p = g["params"]
    fi = est.FisherMatrix(p, constants=c)
    K = est.numparams
    assert fi.shape == (len(p), K, K) and fi.dtype == np.float32
    assert np.array_equal(fi, np.transpose(fi, (0, 2, 1)))
    crlb64, _, fi64 = oracle_model(name, g).crlb(p, g["samples"], constants=c, fp64=True, return_fisher=True)
    # entries relative to sqrt(FI_ii FI_jj): FP32 sums of a few hundred positive terms
    d = np.sqrt(np.abs(np.diagonal(fi64, axis1=1, axis2=2)))
    scale = d[:, :, None] * d[:, None, :] + 1e-30
    err = (np.abs(fi - fi64) / scale).max(axis=(1, 2))
    assert np.quantile(err, 0.99) < 2e-5, (name, np.quantile(err, [0.5, 0.99, 1]))
    crlb = est.CRLB(p, constants=c)
    ok = np.all(np.isfinite(crlb64), axis=1)
    assert np.array_equal(np.all(np.isfinite(crlb), axis=1), ok)
    rel = np.abs(crlb[ok] - crlb64[ok]) / crlb64[ok]
    assert np.quantile(rel.max(axis=1), 0.99) < 1e-4, (name, np.quantile(rel, [0.5, 0.99, 1]))
    # the same values as the CRLB of the fused path and of CRLBAndChiSquare
    assert np.array_equal(crlb, est.CRLBAndChiSquare(p, constants=c))
    est.Destroy()


@pytest.mark.parametrize("name", ["xyibg_r10", "sigmaxy_r16", "astig_r12", "spline_r13"])
def test_numerical_derivatives(name, ctx):
    """NumDeriv is the float32 central difference of ExpectedValue (checked bit for bit against the
    difference formed here from separate ExpectedValue calls), and on the position columns, with
    a step that float32 parameters resolve, it approximates the analytic Derivatives."""
    g = load_golden(name)
    est = cuda_estimator(name, g, ctx)
    truth = g["truth"][:24]
    K = truth.shape[1]
    eps = 1e-2
    nd, ev = est.NumDeriv(truth, eps=eps)
    assert np.array_equal(ev, est.ExpectedValue(truth))
    for k in range(K):
        hi, lo = truth.copy(), truth.copy()
        hi[:, k] += np.float32(eps)
        lo[:, k] -= np.float32(eps)
        want = (est.ExpectedValue(hi) - est.ExpectedValue(lo)) / np.float32(2 * eps)
        assert np.array_equal(nd[:, k], want), k
    deriv, _ = est.Derivatives(truth)
    scale = np.abs(deriv[:, :2]).max(axis=(2, 3), keepdims=True)
    assert np.quantile(np.abs(nd[:, :2] - deriv[:, :2]) / scale, 0.99) < 2e-3
    est.Destroy()


@pytest.mark.parametrize("name", ["xyibg_r10", "sigmaxy_r16", "astig_r12", "spline_r13"])
def test_numerical_crlb_from_analytic_derivatives(name, ctx):
    """NumCRLB over the analytic Derivatives (FP64 host sums) agrees with the GPU's CRLB."""
    g = load_golden(name)
    est = cuda_estimator(name, g, ctx)
    truth = g["truth"][:24]
    crlb = est.CRLB(truth)
    ncrlb = est.NumCRLB(truth, useNumDeriv=False)
    assert np.quantile(np.abs(ncrlb - crlb) / crlb, 0.99) < 1e-4
    est.Destroy()


def test_model_constants_match_device_arithmetic():
    """The set-up constants and the host-computed fixed-sigma scales equal what the device's IEEE
    square root and division give, so the fixed-sigma model's results do not depend on where
    they were computed."""
    import ctypes as ct
    import photonpy_b200 as pb
    L = pb.load_library()
    sig = np.concatenate([np.linspace(0.5, 5.0, 4001), np.random.default_rng(5).uniform(0.3, 50, 4000)]).astype(
        np.float32)
    bad = ct.c_int(-1)
    L.PB200_CheckModelConstants.argtypes = [ct.c_int, ct.c_void_p, ct.POINTER(ct.c_int)]
    assert L.PB200_CheckModelConstants(len(sig), sig.ctypes.data, ct.byref(bad)) == 0
    assert bad.value == 0
