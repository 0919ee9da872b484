"""Mixed batches: several (model, ROI size) buckets fitted in one run (a CUDA-graph replay).

photonpy fits one estimator — one model and one ROI size — per call (its EstimationQueue
holds one estimator per queue, EstimationQueue.h:27-108). A ``MixedBatch`` binds several
estimators with their device-resident ROIs; one ``run()`` fits all of them: buckets of at
least ``standalone_min()`` ROIs per SM with the single-model launches, each on a stream forked
from the run's stream, and the others with two persistent launches (the LM pass, then the
Fisher/CRLB pass) in which ROI groups claim ``tile_rois`` consecutive ROIs at a time from
per-bucket counters; ``capture()`` records that run into a CUDA graph for replay.
``run_plain()`` is the one-launch-per-bucket form of the same work, in sequence on one stream,
for comparison.
"""
from __future__ import annotations

import ctypes as ct

from .lib import check_error, load_library


def _bind(L):
    vp = ct.c_void_p
    L.PB200_MixedPlanCreate.argtypes = [ct.c_int, vp, vp, vp, vp, vp, vp, vp, vp, ct.c_int, ct.c_int]
    L.PB200_MixedPlanCreate.restype = vp
    L.PB200_MixedPlanRun.argtypes = [vp, vp]
    L.PB200_MixedPlanRun.restype = ct.c_int
    L.PB200_MixedPlanCapture.argtypes = [vp, vp]
    L.PB200_MixedPlanCapture.restype = ct.c_int
    L.PB200_MixedPlanInfo.argtypes = [vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]
    L.PB200_MixedPlanInfo.restype = ct.c_int
    L.PB200_MixedPlanDestroy.argtypes = [vp]
    L.PB200_MixedPlanLanes.argtypes = [vp, ct.c_int, vp]
    L.PB200_MixedPlanLanes.restype = ct.c_int
    L.PB200_MixedPlanStandalone.argtypes = [vp, ct.c_int, vp]
    L.PB200_MixedPlanStandalone.restype = ct.c_int
    L.PB200_SetMixedStandaloneMin.argtypes = [ct.c_int]
    L.PB200_SetMixedStandaloneMin.restype = None
    L.PB200_GetMixedStandaloneMin.argtypes = []
    L.PB200_GetMixedStandaloneMin.restype = ct.c_int
    return L


def _ptr_array(tensors):
    arr = (ct.c_void_p * len(tensors))()
    for i, t in enumerate(tensors):
        arr[i] = None if t is None else t.data_ptr()
    return arr


def set_standalone_min(rois_per_sm):
    """ROIs per SM from which a bucket of the MixedBatch objects created afterwards runs as
    launches of its own, on a stream forked from the run's stream (default 0: every bucket; None
    restores it; a value above any bucket size keeps every bucket in the persistent kernel).
    Process-wide."""
    _bind(load_library()).PB200_SetMixedStandaloneMin(-1 if rois_per_sm is None else int(rois_per_sm))


def standalone_min():
    return int(_bind(load_library()).PB200_GetMixedStandaloneMin())


class MixedBatch:
    """buckets: list of (Estimator, samples [n, R, R] float32 CUDA tensor[, constants tensor])."""

    def __init__(self, buckets, tile_rois=1, threads=256, with_crlb=True):
        import torch
        self._L = _bind(load_library())
        self.buckets = []
        for b in buckets:
            est, smp = b[0], b[1]
            consts = b[2] if len(b) > 2 else None
            assert smp.is_cuda and smp.dtype == torch.float32 and smp.is_contiguous()
            n, K = smp.shape[0], est.numparams
            out = dict(params=torch.empty((n, K), device=smp.device),
                       iterations=torch.empty(n, dtype=torch.int32, device=smp.device))
            if with_crlb:
                out["crlb"] = torch.empty((n, K), device=smp.device)
                out["chisq"] = torch.empty(n, device=smp.device)
            self.buckets.append(dict(est=est, samples=smp, constants=consts, out=out))
        nb = len(self.buckets)
        ests = (ct.c_void_p * nb)(*[b["est"].inst for b in self.buckets])
        counts = (ct.c_int * nb)(*[b["samples"].shape[0] for b in self.buckets])
        self._arrays = dict(
            ests=ests, counts=counts,
            smp=_ptr_array([b["samples"] for b in self.buckets]),
            consts=_ptr_array([b["constants"] for b in self.buckets]),
            params=_ptr_array([b["out"]["params"] for b in self.buckets]),
            its=_ptr_array([b["out"]["iterations"] for b in self.buckets]),
            crlb=_ptr_array([b["out"].get("crlb") for b in self.buckets]),
            chisq=_ptr_array([b["out"].get("chisq") for b in self.buckets]))
        a = self._arrays
        self.plan = self._L.PB200_MixedPlanCreate(nb, a["ests"], a["counts"], a["smp"], a["consts"], a["params"],
                                                  a["its"], a["crlb"], a["chisq"], int(tile_rois), int(threads))
        if not self.plan:
            check_error("MixedPlanCreate")
            raise RuntimeError("MixedPlanCreate failed")
        self.tile_rois, self.threads, self.with_crlb = tile_rois, threads, with_crlb
        self.captured = False

    def info(self):
        nt, tiles, stride = ct.c_int(), ct.c_int(), ct.c_int()
        self._L.PB200_MixedPlanInfo(self.plan, ct.byref(nt), ct.byref(tiles), ct.byref(stride))
        return dict(tasks=nt.value, tiles=tiles.value, smem_floats_per_group=stride.value)

    def _stream(self, stream):
        import torch
        return (stream if stream is not None else torch.cuda.current_stream()).cuda_stream

    def run(self, stream=None):
        rc = self._L.PB200_MixedPlanRun(self.plan, ct.c_void_p(self._stream(stream)))
        if rc != 0:
            check_error("MixedPlanRun")
        return self

    def capture(self, stream):
        """Record one run into a CUDA graph on `stream` (a non-default torch stream); later
        run() calls replay the graph."""
        rc = self._L.PB200_MixedPlanCapture(self.plan, ct.c_void_p(stream.cuda_stream))
        if rc != 0:
            check_error("MixedPlanCapture")
        self.captured = True
        return self

    def lanes(self):
        """Lanes per ROI each bucket runs with in the fused launches (4, or 2 for large 7..10 px
        buckets)."""
        arr = (ct.c_int * len(self.buckets))()
        if self._L.PB200_MixedPlanLanes(self.plan, len(self.buckets), arr) != 0:
            check_error("MixedPlanLanes")
        return list(arr)

    def standalone(self):
        """Per bucket: True when it runs as launches of its own (the single-model kernels, at least
        standalone_min() ROIs per SM), False when the persistent mixed kernel fits it."""
        arr = (ct.c_int * len(self.buckets))()
        if self._L.PB200_MixedPlanStandalone(self.plan, len(self.buckets), arr) != 0:
            check_error("MixedPlanStandalone")
        return [bool(v) for v in arr]

    def run_plain(self, stream=None, lanes="plan"):
        """The same work as single-model launches, bucket by bucket (LM, Fisher and CRLB
        launches each). lanes="plan" uses the lanes per ROI the fused launches chose for each
        bucket (lanes()), which gives run()'s results bit for bit; None keeps each estimator's own
        kernel configuration (2 lanes per ROI for 7..10 pixel Gaussians by default); an int
        runs every bucket with that many lanes per ROI."""
        plan_lanes = self.lanes() if lanes == "plan" else None
        for i, b in enumerate(self.buckets):
            est, o = b["est"], b["out"]
            saved = est.kernel_config_setting()
            g = plan_lanes[i] if plan_lanes is not None else lanes
            if g is not None:
                est.SetKernelConfig(g, 0, variant=0)
            try:
                est.EstimateDevice(b["samples"], constants=b["constants"], with_crlb=self.with_crlb, stream=stream,
                                   out=o)
            finally:
                est.SetKernelConfig(*saved)
        return self

    def results(self):
        return [b["out"] for b in self.buckets]

    def close(self):
        if getattr(self, "plan", None):
            self._L.PB200_MixedPlanDestroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
