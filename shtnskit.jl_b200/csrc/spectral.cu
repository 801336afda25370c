// spectral.cu — diagonal operators on dense spectral coefficients.
//
// One elementwise kernel covers the reference's dense diagonal operators:
//   SHTB_SPEC_NEG_LL      out = -l(l+1) in
//       divergence_from_spheroidal / vorticity_from_toroidal (src/sphtor_transforms.jl:771-783,
//       :865-877), laplacian_kernel! / gpu_apply_laplacian! (ext/GPUCommon.jl:1501-1512,
//       ext/SHTnsKitGPUExt.jl:2382-2389), turbo_apply_laplacian! (ext/SHTnsKitLoopVecExt.jl:286-305)
//   SHTB_SPEC_INV_NEG_LL  out = -(in / (l(l+1)))
//       spheroidal_from_divergence / toroidal_from_vorticity (src/sphtor_transforms.jl:817-831,
//       :911-925)
// Entries with m % mres != 0 or l < max(1, m) become zero, whatever the input holds
// there. The factor is the integer l(l+1) converted to the element type, and the
// inverse divides each component by it (no reciprocal), as the reference computes it.
#include "internal.cuh"
#include "kernels.cuh"

namespace shtb {

template <typename C, typename R>
__global__ void spectral_op_kernel(int lmax, int mmax, int mres, const C* __restrict__ in, C* out, int op) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y, k = blockIdx.z;
  if (l > lmax) return;
  const long long o = ((long long)k * (mmax + 1) + m) * (lmax + 1) + l;
  C v;
  v.x = (R)0;
  v.y = (R)0;
  if (m % mres == 0 && l >= max(1, m)) {
    const C x = in[o];
    const R ll = (R)((long long)l * (l + 1));
    if (op == SHTB_SPEC_NEG_LL) {
      v.x = -ll * x.x;
      v.y = -ll * x.y;
    } else {
      v.x = -(x.x / ll);
      v.y = -(x.y / ll);
    }
  }
  out[o] = v;
}

}  // namespace shtb

using namespace shtb;

static bool is_aligned16(const void* q) { return ((uintptr_t)q & 15u) == 0; }

extern "C" int shtb_spectral_op(const shtb_plan* p, int op, const void* in, void* out, int nf, int dtype,
                                void* stream) {
  if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan is NULL");
  if (nf < 1) return set_error(SHTB_ERR_BAD_ARG, "nfields must be >= 1");
  if (op != SHTB_SPEC_NEG_LL && op != SHTB_SPEC_INV_NEG_LL) return set_error(SHTB_ERR_BAD_ARG, "unknown spectral op");
  if (dtype != SHTB_F64 && dtype != SHTB_F32) return set_error(SHTB_ERR_BAD_ARG, "unknown dtype");
  if (!in || !out) return set_error(SHTB_ERR_BAD_ARG, "NULL buffer pointer");
  if (!is_aligned16(in) || !is_aligned16(out)) return set_error(SHTB_ERR_ALIGN, "buffers must be 16-byte aligned");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device) return set_error(SHTB_ERR_BAD_ARG, "the current CUDA device differs from the plan's device");
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid((p->lmax + 1 + 127) / 128, p->mmax + 1, nf);
  prof_begin(st);
  if (dtype == SHTB_F64)
    spectral_op_kernel<double2, double><<<grid, 128, 0, st>>>(p->lmax, p->mmax, p->mres, (const double2*)in,
                                                               (double2*)out, op);
  else
    spectral_op_kernel<float2, float><<<grid, 128, 0, st>>>(p->lmax, p->mmax, p->mres, (const float2*)in,
                                                             (float2*)out, op);
  SHTB_LAUNCHED("spectral operator kernel");
  return SHTB_OK;
}
