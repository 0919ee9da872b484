"""Estimation queue — counterpart of photonpy/cpp/estim_queue.py over the EstimQueue_* C ABI.

``EstimQueue(estim, batchSize, maxQueueLenInBatches, numStreams, keepSamples)`` accepts ROIs
from host memory in any amount (``Schedule``), fits them in the background on the GPU with
the fused LM + CRLB + chi-square kernels, and hands back whole finished batches
(``GetResults`` -> ``EstimQueue_Results``). Results are not kept in scheduling order: sort
them with ``SortByID`` as photonpy's users do (photonpy/smlm/process_movie.py:190).

The C ABI counts its queue limit in spots; this wrapper passes maxQueueLenInBatches *
batchSize, which is what the reference's keyword name says.
"""
from __future__ import annotations

import copy
import ctypes as ct
import time

import numpy as np
import numpy.ctypeslib as ctl

from .estimator import Estimator
from .lib import NullableFloatArrayType, NullableIntArrayType, check_error


class EstimQueue_Results:
    """The results a queue hands back (the attributes and methods of photonpy's
    EstimQueue_Results, photonpy/cpp/estim_queue.py:14-74): per-spot arrays estim [n, K],
    diagnostics [n, numDiag], crlb [n, K], roipos [n, dims], iterations [n], chisq [n], ids [n] and,
    when the queue keeps them, samples [n, *sampleshape]; all selections act on every one of them."""

    _PER_SPOT = ("estim", "diagnostics", "crlb", "roipos", "iterations", "chisq", "ids", "samples")

    def __init__(self, param_names, sampleshape, estim, diag, crlb, iterations, chisq, roipos, samples, ids):
        self.param_names = param_names
        self.sampleshape = sampleshape
        self.estim, self.diagnostics, self.crlb = estim, diag, crlb
        self.iterations, self.chisq, self.roipos = iterations, chisq, roipos
        self.ids, self.samples = ids, samples

    def CRLB(self):
        return self.crlb

    def Filter(self, indices):
        """Keep the spots selected by `indices` (a boolean mask or an index array, in the order
        given) in every per-spot array; returns the index array."""
        indices = np.asarray(indices)
        if indices.dtype == bool:
            indices = np.flatnonzero(indices)
        for name in self._PER_SPOT:
            arr = getattr(self, name)
            if arr is not None:
                setattr(self, name, arr[indices])
        return indices

    def SortByID(self, isUnique=False):
        """Order the spots by ascending id and return the permutation applied (old index of each
        new position). isUnique: the ids are exactly 0..n-1, so the permutation is their inverse."""
        if isUnique:
            perm = np.empty(len(self.ids), dtype=np.int64)
            perm[np.asarray(self.ids)] = np.arange(len(self.ids))
        else:
            perm = np.argsort(self.ids, kind="stable")
        return self.Filter(perm)

    def FilterXY(self, minX, minY, maxX, maxY):
        """Keep the spots whose x and y lie strictly inside (minX, maxX) x (minY, maxY)."""
        x, y = self.estim[:, 0], self.estim[:, 1]
        return self.Filter((x > minX) & (x < maxX) & (y > minY) & (y < maxY))

    def Clone(self):
        return copy.deepcopy(self)

    def ColIdx(self, *names):
        """Column index of each named parameter (a scalar for one name)."""
        idx = [self.param_names.index(n) for n in names]
        return idx[0] if len(idx) == 1 else np.array(idx, dtype=np.int64)


# EstimatorResult (Estimators/EstimationQueue.h:21-25)
EstimResultDType = np.dtype([('id', '<i4'), ('chisq', '<f4'), ('iterations', '<i4')])


class EstimQueue:
    """photonpy/cpp/estim_queue.py:76-255: same constructor, methods and context manager."""

    def __init__(self, estim: Estimator, batchSize=256, maxQueueLenInBatches=5, numStreams=-1, keepSamples=False,
                 ctx=None):
        self.ctx = estim.ctx if ctx is None else ctx
        lib = self.ctx.smlm.lib
        self.estim = estim
        self.batchSize = batchSize
        self.keepSamples = keepSamples
        Inst = ct.c_void_p
        self._EstimQueue_Create = lib.EstimQueue_Create
        self._EstimQueue_Create.argtypes = [Inst, ct.c_int32, ct.c_int32, ct.c_bool, ct.c_int32, ct.c_void_p]
        self._EstimQueue_Create.restype = Inst
        self._EstimQueue_Delete = lib.EstimQueue_Delete
        self._EstimQueue_Delete.argtypes = [Inst]
        self._EstimQueue_Schedule = lib.EstimQueue_Schedule
        self._EstimQueue_Schedule.argtypes = [
            Inst, ct.c_int32,
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),  # ids
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),  # samples
            NullableFloatArrayType,  # initial
            NullableFloatArrayType,  # constants
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),  # roipos
        ]
        self._EstimQueue_Flush = lib.EstimQueue_Flush
        self._EstimQueue_Flush.argtypes = [Inst]
        self._EstimQueue_IsIdle = lib.EstimQueue_IsIdle
        self._EstimQueue_IsIdle.argtypes = [Inst]
        self._EstimQueue_IsIdle.restype = ct.c_bool
        self._EstimQueue_GetResultCount = lib.EstimQueue_GetResultCount
        self._EstimQueue_GetResultCount.argtypes = [Inst]
        self._EstimQueue_GetResultCount.restype = ct.c_int32
        self._EstimQueue_GetQueueLength = lib.EstimQueue_GetQueueLength
        self._EstimQueue_GetQueueLength.argtypes = [Inst]
        self._EstimQueue_GetQueueLength.restype = ct.c_int32
        self._EstimQueue_GetResults = lib.EstimQueue_GetResults
        self._EstimQueue_GetResults.argtypes = [
            Inst, ct.c_int32,
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),  # estim
            NullableFloatArrayType,  # diag
            NullableFloatArrayType,  # crlb
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),  # roipos
            NullableFloatArrayType,  # samples
            ctl.ndpointer(EstimResultDType, flags="aligned, c_contiguous"),  # results
        ]
        self._EstimQueue_GetResults.restype = ct.c_int32
        self.param_names = estim.param_names
        self.inst = self._EstimQueue_Create(estim.inst, batchSize, int(maxQueueLenInBatches) * int(batchSize),
                                            keepSamples, numStreams, self.ctx.inst if self.ctx else None)
        if not self.inst:
            check_error("EstimQueue_Create")
            raise RuntimeError("Unable to create PSF MLE Queue with given PSF")

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.Destroy()

    def Destroy(self):
        if self.inst:
            self._EstimQueue_Delete(self.inst)
            self.inst = None

    def Flush(self):
        self._EstimQueue_Flush(self.inst)
        check_error("EstimQueue_Flush")

    def WaitUntilDone(self):
        self.Flush()
        while not self.IsIdle():
            time.sleep(0.002)

    def IsIdle(self):
        r = self._EstimQueue_IsIdle(self.inst)
        check_error("EstimQueue_IsIdle")
        return r

    def Schedule(self, samples, roipos=None, ids=None, initial=None, constants=None):
        samples = np.ascontiguousarray(samples, dtype=np.float32)
        numspots = len(samples)
        if roipos is None:
            roipos = np.zeros((numspots, self.estim.indexdims), dtype=np.int32)
        if constants is not None:
            constants = np.ascontiguousarray(constants, dtype=np.float32)
            if constants.size != numspots * self.estim.numconst:
                raise ValueError(f'Estimator is expecting constants array with shape '
                                 f'{(numspots, self.estim.numconst)}. Given: {constants.shape}')
        else:
            assert self.estim.numconst == 0
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=np.float32)
            assert np.array_equal(initial.shape, [numspots, self.estim.numparams])
        roipos = np.ascontiguousarray(roipos, dtype=np.int32)
        if not np.array_equal(roipos.shape, [numspots, self.estim.indexdims]):
            raise ValueError(f'Incorrect shape for ROI positions: {roipos.shape} given, '
                             f'expecting {[numspots, self.estim.indexdims]}')
        assert self.estim.samplecount * numspots == samples.size
        if ids is None:
            ids = np.zeros(numspots, dtype=np.int32)
        else:
            assert len(ids) == len(samples)
            ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._EstimQueue_Schedule(self.inst, numspots, ids, samples, initial, constants, roipos)
        check_error("EstimQueue_Schedule")

    def GetQueueLength(self):
        return self._EstimQueue_GetQueueLength(self.inst)

    def GetResultCount(self):
        return self._EstimQueue_GetResultCount(self.inst)

    def GetResults(self, maxResults=None, getSampleData=False) -> EstimQueue_Results:
        count = self._EstimQueue_GetResultCount(self.inst)
        if maxResults is not None and count > maxResults:
            count = maxResults
        K = self.estim.NumParams()
        estim = np.zeros((count, K), dtype=np.float32)
        diag = np.zeros((count, self.estim.NumDiag()), dtype=np.float32)
        crlb = np.zeros((count, K), dtype=np.float32)
        roipos = np.zeros((count, self.estim.indexdims), dtype=np.int32)
        results = np.zeros(count, dtype=EstimResultDType)
        samples = np.zeros((count, *self.estim.sampleshape), dtype=np.float32) if getSampleData else None
        copied = self._EstimQueue_GetResults(self.inst, count, estim, diag, crlb, roipos, samples, results)
        check_error("EstimQueue_GetResults")
        if copied != count:  # maxResults cut a batch: only whole batches are returned
            estim, diag, crlb, roipos, results = estim[:copied], diag[:copied], crlb[:copied], roipos[:copied], \
                results[:copied]
            samples = None if samples is None else samples[:copied]
        return EstimQueue_Results(self.param_names, self.estim.sampleshape, estim, diag, crlb, results['iterations'],
                                  results['chisq'], roipos, samples, results['id'])
