// noalloc.cu — scalar FP64 synthesis whose scratch is a fixed, library-owned device array.
//
// Who needs this: hosts that cannot or must not allocate device memory between
// transforms. A time-stepping model that runs inside another runtime's memory pool
// (CUDA.jl, a game/visualisation engine, an embedded controller) may be forbidden
// from calling cudaMalloc, and cudaMalloc/cudaFree can implicitly synchronize the
// device or fail part-way through a long run when memory is fragmented. Such callers
// pass only their input coefficients and output grid; the Fourier scratch between
// the Legendre and FFT stages lives in `g_noalloc_scratch` below, a static device
// array that exists on every GPU that loads this library until the process exits.
#include "kernels.cuh"

namespace shtb {

// Upper bound of the scratch: nfields * (mmax/mres + 1) * 2 * ceil(nlat/2) * 16 bytes
// must fit (e.g. lmax 511 on 512 x 1024: 8 fields; lmax 255 on 256 x 512: 32 fields).
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The host-side name g_noalloc_scratch only stands in for the symbol: passing it to a
// kernel would hand the GPU a host address. Its device address is looked up here, with
// the plan's device current, when a plan is created (shtb_plan_create), and kept in the
// plan. Looking it up loads this file's module, which is when the driver reserves the
// array on that device; doing it at plan creation keeps that reservation (and any
// failure of it) out of the transform calls.
cudaError_t noalloc_scratch_address(void** out) {
  *out = nullptr;
  return cudaGetSymbolAddress(out, g_noalloc_scratch);
}

}  // namespace shtb

using namespace shtb;

extern "C" int shtb_synthesis_noalloc(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, void* stream) {
  if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan is NULL");
  if (nf < 1) return set_error(SHTB_ERR_BAD_ARG, "nfields must be >= 1");
  if (ltr < 0) ltr = p->lmax;
  if (ltr > p->lmax)
    return set_error(SHTB_ERR_BAD_ARG, "lcap must satisfy 0 <= lcap <= lmax=" + std::to_string(p->lmax));
  if (!alm || !f) return set_error(SHTB_ERR_BAD_ARG, "NULL buffer pointer");
  if ((((uintptr_t)alm) & 15u) || (((uintptr_t)f) & 15u))
    return set_error(SHTB_ERR_ALIGN, "buffers must be 16-byte aligned");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device) return set_error(SHTB_ERR_BAD_ARG, "the current CUDA device differs from the plan's device");
  const size_t need = (size_t)nf * p->nm * 2 * p->npair * 16;
  if (need > kNoAllocScratchBytes)
    return set_error(SHTB_ERR_WORKSPACE, "shtb_synthesis_noalloc needs " + std::to_string(need) +
                                             " bytes of scratch for this plan and nfields; its static scratch holds " +
                                             std::to_string(kNoAllocScratchBytes) +
                                             " bytes (use shtb_synthesis with a caller workspace)");
  void* W = p->noalloc_scratch;
  if (!W)
    return set_error(SHTB_ERR_CUDA, "shtb_synthesis_noalloc: the static scratch was not available when the plan "
                                    "was created: " + p->noalloc_err);
  int rc = SHTB_OK;
  // The Legendre stage writes every scratch entry the FFT stage reads, so nothing is cleared.
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = std::min(p->mmax, ltr);
  CoefSrc src{(const double2*)alm, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 1 : 0, 1.0, 1.0};
  if ((rc = launch_leg_syn64(p, src, F, W, nf, ltr, mlim, st))) return rc;
  return launch_fft_syn<double, double>(p, W, (double*)f, nullptr, 1, nf, mlim, p->phi_inv_scale / p->nlon, 0, 0, st);
}
