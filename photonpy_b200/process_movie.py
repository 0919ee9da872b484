"""Movie processing — counterpart of the detection/localization functions of
photonpy/smlm/process_movie.py.

``detect_spots`` streams 16-bit frames through the spot-extraction queue and writes the ROIs
to a file in photonpy's format: repeated pairs of ``numpy.save`` arrays, the ``ROIInfoDType``
records of a batch and its pixels [n, (sumframes,) roisize, roisize] (process_movie.py:30-60).
``load_rois_iterator`` / ``load_rois`` read such a file back (process_movie.py:67-95) and
``localize_rois`` fits the ROIs through an ``EstimQueue`` (process_movie.py:134-202), and
``extract_rois_iterator`` cuts predefined ROIs out of a movie (process_movie.py:96-131).
``create_calib_obj`` takes scalars or arrays (photonpy also reads TIFF calibration movies, which
needs tifffile; pass the arrays instead).
"""
from __future__ import annotations

import time

import numpy as np

from . import spotdetect
from .calib import GainOffset_Calib, GainOffsetImage_Calib
from .context import Context
from .estim_queue import EstimQueue


def end_of_file(f):
    curpos = f.tell()
    f.seek(0, 2)
    file_size = f.tell()
    f.seek(curpos, 0)
    return curpos == file_size


def detect_spots(sdcfg, calib, movie, sumframes, output_fn, batch_size, ctx: Context, numThreads=3):
    """Spot detection over a movie (an iterable of 2D frames), ROIs written to output_fn.
    Returns (number of ROIs, number of frames)."""
    sm = spotdetect.SpotDetectionMethods(ctx)
    with Context(ctx.smlm) as lq_ctx, open(output_fn, "wb") as f:
        roishape = [sdcfg.roisize, sdcfg.roisize]
        numframes = 0
        numrois = 0
        q = rq = None

        def save_rois(rois_info, pixels):
            nonlocal numrois
            np.save(f, rois_info, allow_pickle=False)
            np.save(f, pixels, allow_pickle=False)
            numrois += len(rois_info)

        for i, img in enumerate(movie):
            if i == 0:
                q, rq = sm.CreateQueue(img.shape, roishape, sdcfg, calib=calib, sumframes=sumframes, ctx=lq_ctx,
                                       numThreads=numThreads)
            q.PushFrameU16(img)
            numframes += 1
            if rq.Length() > batch_size:
                save_rois(*rq.Fetch())
        if q is not None:
            while q.NumFinishedFrames() < numframes // sumframes:
                time.sleep(0.01)
            if rq.Length() > 0:
                save_rois(*rq.Fetch())
        return numrois, numframes


def load_rois_iterator(rois_fn, maxrois=None):
    """Load the ROIs of a detect_spots file batch by batch."""
    with open(rois_fn, "rb") as f:
        total = 0
        while not end_of_file(f):
            rois_info = np.load(f)
            pixels = np.load(f)
            if maxrois is not None:
                if len(pixels) + total >= maxrois:
                    rem = maxrois - total
                    yield rois_info[:rem], pixels[:rem]
                    return
            total += len(pixels)
            yield rois_info, pixels


def load_rois(rois_fn, maxrois=None):
    rois_info = []
    pixels = []
    for ri, px in load_rois_iterator(rois_fn, maxrois):
        rois_info.append(ri)
        pixels.append(px)
    return np.concatenate(rois_info), np.concatenate(pixels)


def extract_rois_iterator(movie, roipos, roiframe, calib, roisize, ctx: Context, minBatchSize):
    """Boxes of predefined ROIs from a movie (an iterable of 16-bit frames): roipos [n, 2] ROI
    corners, given to the extractor as its cornerpos (x, y) records, roiframe [n] the frame of
    each. Yields (rois, frames) batches of at least minBatchSize records (the last one may be
    smaller). photonpy's version of this function calls a PushFrame method its frame processor
    does not have; here the frames go in through PushFrameU16."""
    from .image_proc import ROIExtractor
    roilist = np.zeros(len(roipos), dtype=ROIExtractor.ROIType)
    roilist["cornerpos"] = roipos
    roilist["startframe"] = roiframe
    roilist["numframes"] = 1
    with Context(ctx.smlm) as ex_ctx:
        q = None
        for i, img in enumerate(movie):
            if i == 0:
                q = ROIExtractor(img.shape, roilist, 1, roisize, calib, ex_ctx)
            q.PushFrameU16(img)
            resultcount = q.GetResultCount()
            if resultcount > minBatchSize:
                yield q.GetResults(resultcount)
        if q is None:
            return
        while not q.IsIdle():
            time.sleep(0.005)
            resultcount = q.GetResultCount()
            if resultcount > minBatchSize:
                yield q.GetResults(resultcount)
        resultcount = q.GetResultCount()
        if resultcount > 0:
            yield q.GetResults(resultcount)


def localize_rois(rois_data_source, psf, initial_estim=None, constants=None, prog_cb=None, total=None):
    """Fits ROIs with the PSF through an EstimQueue. rois_data_source: a detect_spots file name or
    an iterable of (rois_info, pixels). Returns the EstimQueue_Results in ROI order, with
    ``ids`` set to the frame numbers. prog_cb(result count) may return False to cancel (None is
    then returned)."""
    if isinstance(rois_data_source, str):
        iterator = load_rois_iterator(rois_data_source)
    else:
        iterator = rois_data_source
    framenums = []
    with EstimQueue(psf, batchSize=1024) as queue:
        count = 0

        def progupdate():
            if prog_cb is None:
                return True
            return prog_cb(queue.GetResultCount())

        for rois_info, pixels in iterator:
            roipos = np.zeros((len(rois_info), 2))
            roipos[:, 0] = rois_info["y"]
            roipos[:, 1] = rois_info["x"]
            framenums.append(rois_info["id"])
            initial = initial_estim[count:count + len(pixels)] if initial_estim is not None else None
            batch_constants = constants[count:count + len(pixels)] if constants is not None else None
            queue.Schedule(pixels, ids=np.arange(count, count + len(pixels)), roipos=roipos, initial=initial,
                           constants=batch_constants)
            count += len(pixels)
            if not progupdate():
                return None
        queue.Flush()
        while not queue.IsIdle():
            time.sleep(0.005)
            progupdate()
        progupdate()
        r = queue.GetResults(getSampleData=False)
        r.SortByID(isUnique=True)  # back to the ROI order
        r.ids = np.concatenate(framenums) if framenums else np.zeros(0, dtype=np.int32)
    return r


def create_calib_obj(gain, offset, imgshape, ctx):
    """Gain/offset camera calibration from scalars or per-pixel arrays."""
    if isinstance(gain, str) or isinstance(offset, str):
        raise NotImplementedError("calibration movies from TIFF files: load them and pass the arrays")
    if isinstance(offset, np.ndarray):
        if not isinstance(gain, np.ndarray):
            gain = np.ones(imgshape) * gain
        return GainOffsetImage_Calib(gain, offset, ctx)
    return GainOffset_Calib(gain, offset, ctx)


def _summed_movie(movie, sumframes):
    img = None
    f = 0
    for m in movie:
        if f == 0:
            img = m.copy()
        else:
            img += m
        f += 1
        if f == sumframes:
            img_ = img
            img = None
            f = 0
            yield img_
