"""Seeded synthetic ROI batches for tests and benchmarks.

Ground truth is drawn with ``numpy.random.default_rng(seed)``, the pixel
expectation is evaluated in FP64 from the pixel-integrated (erf-difference)
Gaussian PSF that photonpy's models describe (GaussianPSFModels.h:63-98), and
observed pixels are Poisson draws stored as float32. The same arrays feed the
CUDA estimator, the reference's CPU estimator and the oracle.

Workloads (distributions as stated in each generator):
  * ``xyibg``      10x10, sigma 1.5 fixed, x,y~U[4,6], I~U[500,5000], bg~U[2,10]
  * ``sigmaxy``    16x16 free sigma_x/sigma_y, x,y~U[6.5,8.5], sigma~U[1.2,2.2],
                   I log-uniform [200,20000], bg~U[1,20], initial sigma 1.7
  * ``astig``      12x12 astigmatic 3D, z~U[-400,400] nm, s0 1.3 px, c 150 nm,
                   d 400 nm, A 0.1 (and optional B), I log-uniform [500,1e4], bg~U[2,15]
  * ``spline``     13x13 cubic-spline PSF built from a z-stack of the astig model
                   (z in micrometres), z~U[-0.38,0.38] um
  * ``mixed``      sizes {7,9,11,16} p={.2,.3,.3,.2}; 50% XYIBg, 30% SigmaXY, 20% astig;
                   x,y re-centred at (R-1)/2 +- 1 px
  * ``tilted``     11x11 tilted background bg + bgx (x - R/2) + bgy (y - R/2), bgx,bgy~U[-0.15,0.15],
                   per-spot sigma constants~U[1.2,1.8] (XYITiltedBg), or free sigma_x/sigma_y
                   ~U[1.2,2.0] (XYITiltedBgSigmaXY, initial sigma 1.6)
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf

SQRT2 = math.sqrt(2.0)


def _delta(pix, centre, sigma):
    """Pixel-integrated 1D Gaussian, shape [n, R] (FP64)."""
    s = SQRT2 * sigma[:, None]
    a = (pix[None, :] - centre[:, None] + 0.5) / s
    b = (pix[None, :] - centre[:, None] - 0.5) / s
    return 0.5 * erf(a) - 0.5 * erf(b)


def gauss2d_ev(R, x, y, I, bg, sx, sy):
    """Expected pixel values [n, R, R] of bg + I * DeltaX * DeltaY (FP64)."""
    pix = np.arange(R, dtype=np.float64)
    dx = _delta(pix, np.asarray(x, np.float64), np.asarray(sx, np.float64))
    dy = _delta(pix, np.asarray(y, np.float64), np.asarray(sy, np.float64))
    return np.asarray(bg)[:, None, None] + np.asarray(I)[:, None, None] * dy[:, :, None] * dx[:, None, :]


def astig_sigma(z, s0, gamma, d, A, B=0.0):
    """sigma(z) = s0*sqrt(1 + tz^2/d^2 + A*tz^3/d^2 + B*tz^4/d^4), tz = z - gamma (the
    reference's 4-coefficient form, GaussianPSFModels.h:698-702, plus an optional B term)."""
    tz = np.asarray(z, np.float64) - gamma
    return s0 * np.sqrt(1 + tz ** 2 / d ** 2 + A * tz ** 3 / d ** 2 + B * tz ** 4 / d ** 4)


def astig_calib_nm(A=0.1, B=0.0, s0=1.3, c=150.0, d=400.0, zrange=(-600.0, 600.0)):
    """Config-3 calibration expressed in the reference's coefficients (z in nm).

    The workload writes sigma = s0*sqrt(1 + t^2 + A t^3 + B t^4) with t = (z -+ c)/d.
    In the reference's form A multiplies tz^3/d^2, hence A_ref = A/d.
    Returns (x[5], y[5], zrange) with (s0, gamma, d, A_ref, B)."""
    x = [s0, c, d, A / d, B]
    y = [s0, -c, d, A / d, B]
    return x, y, tuple(zrange)


_TORCH = {"device": None, "gen": None}


def use_torch(device, seed):
    """Route Poisson draws and expected values of the generators below through torch on
    `device` (much faster for million-ROI batches); None restores numpy. Ground truth is
    still drawn with numpy's seeded generator; the Poisson stream comes from a torch
    generator seeded with `seed`."""
    if device is None:
        _TORCH["device"] = None
        _TORCH["gen"] = None
        return
    import torch
    _TORCH["device"] = torch.device(device)
    g = torch.Generator(device=_TORCH["device"])
    g.manual_seed(int(seed))
    _TORCH["gen"] = g


def _gauss2d_poisson_torch(R, x, y, I, bg, sx, sy):
    import torch
    dev = _TORCH["device"]
    f64 = dict(device=dev, dtype=torch.float64)
    pix = torch.arange(R, **f64)

    def delta(c, s):
        c = torch.tensor(np.array(c, np.float64), **f64)[:, None]
        s = torch.tensor(np.array(s, np.float64), **f64)[:, None] * SQRT2
        return 0.5 * torch.special.erf((pix[None] - c + 0.5) / s) - 0.5 * torch.special.erf((pix[None] - c - 0.5) / s)

    dx = delta(x, sx)
    dy = delta(y, sy)
    ev = torch.tensor(np.array(bg, np.float64), **f64)[:, None, None] + \
        torch.tensor(np.array(I, np.float64), **f64)[:, None, None] * dy[:, :, None] * dx[:, None, :]
    return torch.poisson(ev, generator=_TORCH["gen"]).to(torch.float32).cpu().numpy()


def _poisson(rng, ev, chunk=1 << 22):
    out = np.empty(ev.shape, np.float32)
    flat_in = ev.reshape(-1)
    flat_out = out.reshape(-1)
    for s in range(0, flat_in.size, chunk):
        flat_out[s:s + chunk] = rng.poisson(flat_in[s:s + chunk])
    return out


def _gauss_samples(rng, R, x, y, I, bg, sx, sy, chunk):
    """Poisson ROIs for the given truth arrays, generated chunk by chunk."""
    sx = np.broadcast_to(np.asarray(sx, np.float64), np.shape(x))
    sy = np.broadcast_to(np.asarray(sy, np.float64), np.shape(x))
    if _TORCH["device"] is not None:
        ch = 1 << 18
        return _gen_chunks(len(x), ch, lambda a, b: _gauss2d_poisson_torch(R, x[a:b], y[a:b], I[a:b], bg[a:b],
                                                                          sx[a:b], sy[a:b]))
    return _gen_chunks(len(x), chunk, lambda a, b: _poisson(rng, gauss2d_ev(R, x[a:b], y[a:b], I[a:b], bg[a:b],
                                                                          sx[a:b], sy[a:b])))


def _gen_chunks(n, chunk, fn):
    parts = [fn(s, min(n, s + chunk)) for s in range(0, n, chunk)]
    return np.concatenate(parts, axis=0) if parts else None


def xyibg(n, seed=1, R=10, sigma=1.5, xy=(4.0, 6.0)):
    rng = np.random.default_rng(seed)
    x = rng.uniform(*xy, n)
    y = rng.uniform(*xy, n)
    I = rng.uniform(500, 5000, n)
    bg = rng.uniform(2, 10, n)
    truth = np.stack([x, y, I, bg], 1).astype(np.float32)
    smp = _gauss_samples(rng, R, x, y, I, bg, sigma, sigma, 65536)
    return dict(kind="XYIBg", R=R, sigma=(sigma, sigma), samples=smp, truth=truth)


def constsigma(n, seed=11, R=9, sig=(1.2, 1.8)):
    rng = np.random.default_rng(seed)
    x = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    y = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    I = rng.uniform(500, 5000, n)
    bg = rng.uniform(2, 10, n)
    sx = rng.uniform(*sig, n)
    sy = rng.uniform(*sig, n)
    truth = np.stack([x, y, I, bg], 1).astype(np.float32)
    consts = np.stack([sx, sy], 1).astype(np.float32)
    smp = _poisson(rng, gauss2d_ev(R, x, y, I, bg, sx, sy))
    return dict(kind="XYIBgConstSigma", R=R, samples=smp, truth=truth, constants=consts)


def tilted(n, seed=13, R=11, free_sigma=False, init_sigma=1.6):
    """Tilted-background Gaussian spots (GaussianPSFModels.h:228-304, 474-558). Truth rows are
    (x, y, I, bg, bgx, bgy) for the per-spot-sigma model, (x, y, I, bg, bgx, bgy, sx, sy) for
    the free-sigma one; the expectation always includes the tilt."""
    rng = np.random.default_rng(seed)
    c = (R - 1) / 2
    x = rng.uniform(c - 1, c + 1, n)
    y = rng.uniform(c - 1, c + 1, n)
    I = rng.uniform(500, 5000, n)
    bg = rng.uniform(2, 10, n)
    bgx = rng.uniform(-0.15, 0.15, n)
    bgy = rng.uniform(-0.15, 0.15, n)
    if free_sigma:
        sx = rng.uniform(1.2, 2.0, n)
        sy = rng.uniform(1.2, 2.0, n)
    else:
        sx = rng.uniform(1.2, 1.8, n)
        sy = rng.uniform(1.2, 1.8, n)
    pix = np.arange(R, dtype=np.float64) - R * 0.5
    ev = gauss2d_ev(R, x, y, I, bg, sx, sy) + bgx[:, None, None] * pix[None, None, :] + \
        bgy[:, None, None] * pix[None, :, None]
    smp = _poisson(rng, ev)
    if free_sigma:
        truth = np.stack([x, y, I, bg, bgx, bgy, sx, sy], 1).astype(np.float32)
        return dict(kind="XYITiltedBgSigmaXY", R=R, sigma=(init_sigma, init_sigma), samples=smp, truth=truth)
    truth = np.stack([x, y, I, bg, bgx, bgy], 1).astype(np.float32)
    consts = np.stack([sx, sy], 1).astype(np.float32)
    return dict(kind="XYITiltedBg", R=R, samples=smp, truth=truth, constants=consts)


def sigma1(n, seed=12, R=11, init_sigma=1.5):
    rng = np.random.default_rng(seed)
    x = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    y = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    I = rng.uniform(500, 5000, n)
    bg = rng.uniform(2, 10, n)
    s = rng.uniform(1.2, 2.0, n)
    truth = np.stack([x, y, I, bg, s], 1).astype(np.float32)
    smp = _poisson(rng, gauss2d_ev(R, x, y, I, bg, s, s))
    return dict(kind="XYIBgSigma", R=R, sigma=(init_sigma, init_sigma), samples=smp, truth=truth)


def sigmaxy(n, seed=2, R=16, init_sigma=1.7, xy=(6.5, 8.5)):
    rng = np.random.default_rng(seed)
    x = rng.uniform(*xy, n)
    y = rng.uniform(*xy, n)
    sx = rng.uniform(1.2, 2.2, n)
    sy = rng.uniform(1.2, 2.2, n)
    I = np.exp(rng.uniform(math.log(200), math.log(20000), n))
    bg = rng.uniform(1, 20, n)
    truth = np.stack([x, y, I, bg, sx, sy], 1).astype(np.float32)
    smp = _gauss_samples(rng, R, x, y, I, bg, sx, sy, 32768)
    return dict(kind="XYIBgSigmaXY", R=R, sigma=(init_sigma, init_sigma), samples=smp, truth=truth)


def astig(n, seed=3, R=12, A=0.1, B=0.0, zr=(-400.0, 400.0), xy=None, zrange=(-600.0, 600.0)):
    rng = np.random.default_rng(seed)
    cx, cy, zrange = astig_calib_nm(A=A, B=B, zrange=zrange)
    lo, hi = xy if xy is not None else ((R - 1) / 2 - 1, (R - 1) / 2 + 1)
    x = rng.uniform(lo, hi, n)
    y = rng.uniform(lo, hi, n)
    z = rng.uniform(*zr, n)
    I = np.exp(rng.uniform(math.log(500), math.log(1e4), n))
    bg = rng.uniform(2, 15, n)
    sx = astig_sigma(z, *cx)
    sy = astig_sigma(z, *cy)
    truth = np.stack([x, y, z, I, bg], 1).astype(np.float32)
    smp = _gauss_samples(rng, R, x, y, I, bg, sx, sy, 65536)
    return dict(kind="XYZIBg", R=R, astig=(cx, cy), zrange=zrange, samples=smp, truth=truth)


def astig_zstack(shape_xy=26, nz=41, zrange_um=(-0.4, 0.4), A=0.1, B=0.0, step_px=1.0):
    """Z-stack [nz, Y, X] of the astig model (z in micrometres), centred at (X-1)/2 in
    units of the output grid, each slice normalised to sum 1 (in ROI pixel units)."""
    cx, cy, _ = astig_calib_nm(A=A, B=B)
    cx = [cx[0], cx[1] * 1e-3, cx[2] * 1e-3, cx[3] * 1e3, cx[4]]
    cy = [cy[0], cy[1] * 1e-3, cy[2] * 1e-3, cy[3] * 1e3, cy[4]]
    zs = np.linspace(zrange_um[0], zrange_um[1], nz)
    X = shape_xy
    # Grid point g sits at ROI-pixel offset (g - (X-1)/2) * step_px from the PSF centre.
    offs = (np.arange(X) - (X - 1) / 2) * step_px
    out = np.zeros((nz, X, X), np.float64)
    for k, z in enumerate(zs):
        sx = astig_sigma(z, *cx)
        sy = astig_sigma(z, *cy)
        # pixel-integrated over one ROI pixel centred at each grid offset
        dx = 0.5 * erf((offs + 0.5) / (SQRT2 * sx)) - 0.5 * erf((offs - 0.5) / (SQRT2 * sx))
        dy = 0.5 * erf((offs + 0.5) / (SQRT2 * sy)) - 0.5 * erf((offs - 0.5) / (SQRT2 * sy))
        sl = dy[:, None] * dx[None, :]
        out[k] = sl / sl.sum() * (step_px ** 2 if step_px != 1.0 else 1.0)
    return out.astype(np.float32), (float(zs[0]), float(zs[-1]))


def spline(n, seed=4, R=13, zr=(-0.38, 0.38), A=0.1, B=0.0):
    """ROIs drawn from the astig model with z in micrometres (the PSF the spline calibrates)."""
    rng = np.random.default_rng(seed)
    cx, cy, _ = astig_calib_nm(A=A, B=B)
    cx = [cx[0], cx[1] * 1e-3, cx[2] * 1e-3, cx[3] * 1e3, cx[4]]
    cy = [cy[0], cy[1] * 1e-3, cy[2] * 1e-3, cy[3] * 1e3, cy[4]]
    x = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    y = rng.uniform((R - 1) / 2 - 1, (R - 1) / 2 + 1, n)
    z = rng.uniform(*zr, n)
    I = np.exp(rng.uniform(math.log(500), math.log(1e4), n))
    bg = rng.uniform(2, 15, n)
    sx = astig_sigma(z, *cx)
    sy = astig_sigma(z, *cy)
    truth = np.stack([x, y, z, I, bg], 1).astype(np.float32)
    smp = _gauss_samples(rng, R, x, y, I, bg, sx, sy, 65536)
    return dict(kind="CSpline", R=R, samples=smp, truth=truth)


def spline_background(n, mode, seed=6, R=13, zr=(-0.38, 0.38), A=0.1):
    """Spline-workload spots on a tilted background (mode "tilted": truth (x, y, z, I, bg, bgx,
    bgy), bgx,bgy~U[-0.15,0.15]) or on a per-spot background image (mode "bgimage": truth
    (x, y, z, I, bg), constants = an image [R, R] with values in [0.5, 1.5] that bg scales)."""
    rng = np.random.default_rng(seed)
    cx, cy, _ = astig_calib_nm(A=A)
    cx = [cx[0], cx[1] * 1e-3, cx[2] * 1e-3, cx[3] * 1e3, cx[4]]
    cy = [cy[0], cy[1] * 1e-3, cy[2] * 1e-3, cy[3] * 1e3, cy[4]]
    c = (R - 1) / 2
    x = rng.uniform(c - 1, c + 1, n)
    y = rng.uniform(c - 1, c + 1, n)
    z = rng.uniform(*zr, n)
    I = np.exp(rng.uniform(math.log(500), math.log(1e4), n))
    bg = rng.uniform(2, 15, n)
    ev = gauss2d_ev(R, x, y, I, np.zeros(n), astig_sigma(z, *cx), astig_sigma(z, *cy))
    pix = np.arange(R, dtype=np.float64) - R * 0.5
    if mode == "tilted":
        bgx = rng.uniform(-0.15, 0.15, n)
        bgy = rng.uniform(-0.15, 0.15, n)
        ev += bg[:, None, None] + bgx[:, None, None] * pix[None, None, :] + bgy[:, None, None] * pix[None, :, None]
        truth = np.stack([x, y, z, I, bg, bgx, bgy], 1).astype(np.float32)
        return dict(kind="CSplineTilted", R=R, samples=_poisson(rng, ev), truth=truth)
    gx = rng.uniform(-0.5, 0.5, n)[:, None, None] * pix[None, None, :] / (R * 0.5)
    gy = rng.uniform(-0.5, 0.5, n)[:, None, None] * pix[None, :, None] / (R * 0.5)
    img = (1.0 + 0.5 * (gx + gy)).astype(np.float32)
    ev += bg[:, None, None] * img
    truth = np.stack([x, y, z, I, bg], 1).astype(np.float32)
    return dict(kind="CSplineBgImage", R=R, samples=_poisson(rng, ev), truth=truth,
                constants=img.reshape(n, R * R))


def frames(n, h=128, w=160, spots_per_frame=20, seed=8, sigma=1.5, I=(300, 3000), bg=(3.0, 8.0), margin=2):
    """Camera frames [n, h, w] with Gaussian spots at random positions (at least `margin` px
    from the border) on a flat background, Poisson noise. Returns dict(frames, truth) with truth
    rows (frame, x, y, I, bg)."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, h, w), np.float32)
    truth = []
    px, py = np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64)
    for f in range(n):
        b = rng.uniform(*bg)
        x = rng.uniform(margin, w - 1 - margin, spots_per_frame)
        y = rng.uniform(margin, h - 1 - margin, spots_per_frame)
        inten = rng.uniform(*I, spots_per_frame)
        dx = _delta(px, x, np.full(spots_per_frame, sigma))
        dy = _delta(py, y, np.full(spots_per_frame, sigma))
        ev = b + np.einsum("s,sy,sx->yx", inten, dy, dx)
        out[f] = rng.poisson(ev)
        for k in range(spots_per_frame):
            truth.append((f, x[k], y[k], inten[k], b))
    return dict(frames=out, truth=np.array(truth, np.float64))


MIXED_SIZES = (7, 9, 11, 16)
MIXED_SIZE_P = (0.2, 0.3, 0.3, 0.2)
MIXED_MODELS = ("XYIBg", "XYIBgSigmaXY", "XYZIBg")
MIXED_MODEL_P = (0.5, 0.3, 0.2)


def mixed(n, seed=5):
    """Mixed-size, mixed-model batch. Returns a list of groups, one per (model, size):
    dict(kind, R, index (positions in the mixed order), samples, truth, ...)."""
    rng = np.random.default_rng(seed)
    size_idx = rng.choice(len(MIXED_SIZES), n, p=MIXED_SIZE_P)
    model_idx = rng.choice(len(MIXED_MODELS), n, p=MIXED_MODEL_P)
    groups = []
    sub_seed = seed * 1000
    for mi, kind in enumerate(MIXED_MODELS):
        for si, R in enumerate(MIXED_SIZES):
            sel = np.nonzero((model_idx == mi) & (size_idx == si))[0]
            if sel.size == 0:
                continue
            sub_seed += 1
            xy = ((R - 1) / 2 - 1, (R - 1) / 2 + 1)
            if kind == "XYIBg":
                g = xyibg(sel.size, seed=sub_seed, R=R, xy=xy)
            elif kind == "XYIBgSigmaXY":
                g = sigmaxy(sel.size, seed=sub_seed, R=R, xy=xy)
            else:
                g = astig(sel.size, seed=sub_seed, R=R, xy=xy)
            g["index"] = sel
            groups.append(g)
    return groups
