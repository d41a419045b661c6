/* ORACLE — test infrastructure only.
 * Force-included (-include) when the reference world simulator's kernels are
 * compiled for the correctly rounded comparison (no fast math, no FMA
 * contraction): every expf/logf/cosf/sinf/hypotf call in the reference
 * sources, host or device, resolves to a correctly rounded binary32 function. The device
 * implementation is the library's nsx::expf_cr / nsx::logf_cr (and the
 * trigonometric and hypot functions beside them), whose results the oracle's
 * sweeps check against an independent binary128 evaluation; a correctly rounded result is unique, so any
 * correct implementation gives the same bits. */
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <random>
#ifdef __CUDACC__
#include <cub/device/device_select.cuh>       /* library headers that declare expf/logf themselves */
#include <thrust/iterator/counting_iterator.h>
#include <cuda/std/cmath>
#endif
#include "ns_crmath.h"
#define expf(x) nsx::expf_cr(x)
#define logf(x) nsx::logf_cr(x)
#define cosf(x) nsx::cosf_cr(x)
#define sinf(x) nsx::sinf_cr(x)
#define hypotf(x, y) nsx::hypotf_cr(x, y)
