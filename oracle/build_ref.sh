#!/usr/bin/env bash
# Builds the reference photonpy estimator (CPU path + its own one-thread-per-ROI
# CUDA kernels for sm_100a) from the reference sources, as a checker and as the
# timed CPU baseline. Output: oracle/_ref/libphotonpy_ref.so (git-ignored).
#
# The reference is an MSVC project. GCC needs a handful of mechanical fixes
# (header case, MSVC-only `typename` placement, two-phase lookup in unused
# templates). They are applied by the sed/perl lines below to a throw-away copy
# under oracle/_ref/src, which is deleted again after the build so that only
# the shared library remains. No reference source is kept in the repository.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT
#    or: PHOTONPY_REFERENCE_ROOT=<photonpy checkout> oracle/build_ref.sh
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${PHOTONPY_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "usage: $0 REFERENCE_ROOT (or set PHOTONPY_REFERENCE_ROOT)" >&2
  exit 2
fi
SRC_ROOT="$REF/cpp/SMLMLib"
OUT="$HERE/_ref"
TMP="$OUT/src"
if [ ! -d "$SRC_ROOT" ]; then
  echo "reference sources not found at $SRC_ROOT" >&2
  exit 1
fi
# photonpy's own Python binding of the estimator, unmodified, beside the library (git-ignored
# like it): the drop-in test loads it over libphotonpy_b200.so. PB_REF_PYTHON_ONLY=1 stops here.
PY_OUT="$OUT/photonpy_cpp"
mkdir -p "$PY_OUT"
for f in lib context estimator gaussian cspline estim_queue; do
  cp "$REF/photonpy/cpp/$f.py" "$PY_OUT/$f.py"
done
if [ "${PB_REF_PYTHON_ONLY:-0}" = 1 ]; then
  echo "copied photonpy's binding to $PY_OUT"
  exit 0
fi
rm -rf "$TMP"
mkdir -p "$TMP"
cp -r "$SRC_ROOT"/. "$TMP"/
cd "$TMP"

# 1. case-sensitive include name
ln -sf DLLMacros.h dllmacros.h
# 2. Windows.h / force-included compatibility shim (written here, not copied)
cat > Windows.h << 'H'
#pragma once
#define OutputDebugString(x) ((void)0)
#define OutputDebugStringA(x) ((void)0)
H
cat > msvc_compat.h << 'H'
#pragma once
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdarg>
#include <stdexcept>
#include <thread>
#include <vector>
#include <future>
#include <mutex>
#include <list>
#include <memory>
#include <algorithm>
#include <string>
#define __declspec(x)
#define strcpy_s(d, n, s) strncpy(d, s, n)
#define vsprintf_s(buf, n, fmt, args) vsnprintf(buf, n, fmt, args)
#define sprintf_s snprintf
H
# 3. MSVC accepts `typename` before names that are not dependent-nested; GCC does not.
find . \( -name '*.h' -o -name '*.cu' -o -name '*.cpp' \) -print0 | xargs -0 perl -0pi -e '
  s/\btypename\s+(\w+)(?=\s+[A-Za-z_])(?!\s*::)/$1/g;
  s/\(typename Params\*\)/(Params*)/g;
  s/\btypename\s+(\w+<[^<>;]*>)(?!\s*::)/$1/g;
  s/typename\s+(ChiSquareAndCRLB<Params>)/$1/g;
  s/typename\s+(Vector<T,\s*d>\s+ApplyMatrix)/$1/g;
'
# 4. spots the generic rule cannot see
perl -0pi -e 's/Estimator\* CreateGaussianPSF\(int roisize, bool cuda, TModel::Calibration calib/Estimator* CreateGaussianPSF(int roisize, bool cuda, typename TModel::Calibration calib/' Estimators/Gaussian/GaussianPSF.cu
perl -0pi -e 's/return get_param_arg</return typename get_param_arg</g' palala.h
perl -0pi -e 's/template<typename T>(\s*)friend vector3 operator\/\(T a, vector3<T> b\)/template<typename U>$1friend vector3 operator\/(U a, vector3<U> b)/' MathUtils.h
perl -0pi -e 's/template<typename T>(\s*)PinnedArray\(const DeviceArray<T>& src\)/PinnedArray(const DeviceArray<T>\& src)/' CudaUtils.h
# 5. two-phase lookup errors inside templates that are never instantiated
perl -0pi -e 's/T x = sample\[smpIndex\] \+= readnoiseVG2\[smpIndex\];/T x = sample[smpIndex] + readnoiseVG2[smpIndex];/' Estimators/Estimation.h
sed -i '/OneOverSqrt2PiSigma3Y = /,/ComputeInitialEstimate/{s/\bimgw\b/Width()/g}' Estimators/Gaussian/GaussianPSFModels.h
perl -0pi -e 's/\bheight\(\)/Height()/g; s/\bwidth\(\)/Width()/g' Estimators/Gaussian/GaussianPSFModels.h
# members of a dependent base class named without this-> (the frame-queue templates)
perl -0pi -e 's/= GetFinishedFrame\(\);/= this->GetFinishedFrame();/; s/\tRecycleOutput\(std::move\(f\)\);/\tthis->RecycleOutput(std::move(f));/; s/auto output = GetNewOutputFrame\(\);/auto output = this->GetNewOutputFrame();/; s/\tAddToFinished\(std::move\(output\)\);/\tthis->AddToFinished(std::move(output));/; s/CopyToHost\(output->h_filtered\.data\(\), stream\)/CopyToHost(output->h_filtered.data(), this->stream)/; s/cudaStreamSynchronize\(stream\);/cudaStreamSynchronize(this->stream);/g' ImgFilterQueueImpl.h
# a braced size that matches two DeviceImage constructors
perl -0pi -e 's/original\(\{ imgsize\.x, imgsize\.y\*sumframes \}\)/original(imgsize.x, imgsize.y*sumframes)/' ImgFilterQueue.cu
# the index-list generator names a predicate that SpotDetector.h defines after including it
perl -0pi -e 's/#include "SpotIndexListGenerator.h"\n//; s/(struct SpotLocationList)/#include "SpotIndexListGenerator.h"\n\n$1/' SpotDetection/SpotDetector.h

NVCC=${NVCC:-nvcc}
FLAGS=(-x cu -std=c++17 -O3 -Xcompiler -fPIC,-fpermissive,-w,-O3 --expt-extended-lambda --expt-relaxed-constexpr
       -gencode arch=compute_100a,code=sm_100a -I. -IEstimators -include msvc_compat.h -DNDEBUG)
SRCS=(Estimators/Estimator.cpp StringUtils.cpp Context.cpp DebugImageCallback.cpp Rendering.cpp CudaUtils.cu
      Estimators/EstimatorImpl.cu Estimators/Gaussian/GaussianPSF.cu Estimators/CSpline/CubicSplinePSF.cu
      Estimators/EstimationQueue.cpp Estimators/GLRT_PSF.cu SpotDetection/SpotDetector.cu
      ImgFilterQueue.cu ROIQueue.cpp CameraCalibration.cu ImageProcessor.cpp)
OBJS=()
pids=()
for s in "${SRCS[@]}"; do
  o="$OUT/$(basename "${s%.*}").o"
  OBJS+=("$o")
  "$NVCC" "${FLAGS[@]}" -c "$s" -o "$o" &
  pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
if [ $rc -ne 0 ]; then echo "reference build failed" >&2; exit 1; fi
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a "${OBJS[@]}" -o "$OUT/libphotonpy_ref.so" -lcudart -lpthread
rm -f "${OBJS[@]}"
cd "$OUT"
rm -rf "$TMP"
echo "built $OUT/libphotonpy_ref.so"
