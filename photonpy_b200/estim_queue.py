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
    """Results of a queue (photonpy/cpp/estim_queue.py:14-74)."""

    def __init__(self, param_names, sampleshape, estim, diag, crlb, iterations, chisq, roipos, samples, ids):
        self.estim = estim
        self.sampleshape = sampleshape
        self.diagnostics = diag
        self.crlb = crlb
        self.roipos = roipos
        self.iterations = iterations
        self.chisq = chisq
        self.ids = ids
        self.samples = samples
        self.param_names = param_names

    def CRLB(self):
        return self.crlb

    def SortByID(self, isUnique=False):
        """Reorder by spot id; with isUnique the ids must be a permutation of 0..n-1."""
        if isUnique:
            order = np.arange(len(self.ids))
            order[self.ids] = order * 1
        else:
            order = np.argsort(self.ids, kind="stable")
        self.Filter(order)
        return order

    def Filter(self, indices):
        if indices.dtype == bool:
            indices = np.nonzero(indices)[0]
        if len(indices) != len(self.ids):
            print(f"Removing {len(self.ids) - len(indices)}/{len(self.ids)}")
        self.estim = self.estim[indices]
        self.diagnostics = self.diagnostics[indices]
        self.crlb = self.crlb[indices]
        self.roipos = self.roipos[indices]
        self.iterations = self.iterations[indices]
        self.chisq = self.chisq[indices]
        self.ids = self.ids[indices]
        if self.samples is not None:
            self.samples = self.samples[indices]
        return indices

    def FilterXY(self, minX, minY, maxX, maxY):
        return self.Filter(np.where(np.logical_and(np.logical_and(self.estim[:, 0] > minX, self.estim[:, 1] > minY),
                                                   np.logical_and(self.estim[:, 0] < maxX,
                                                                  self.estim[:, 1] < maxY)))[0])

    def Clone(self):
        return copy.deepcopy(self)

    def ColIdx(self, *names):
        return np.squeeze(np.array([self.param_names.index(n) for n in names], dtype=np.int64))


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
