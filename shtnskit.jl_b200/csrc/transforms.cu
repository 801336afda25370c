// transforms.cu — C-ABI entry points: validation, workspace layout and the
// kernel sequence of every transform and adjoint.
//
// Scalar synthesis  : coefficients --(Legendre, E/O)--> W --(unfold + inverse FFT)--> grid
// Scalar analysis   : grid --(FFT + fold + weights)--> W --(Legendre GEMM)--> coefficients
// Vector transforms : the spheroidal/toroidal pair is rewritten as two scalar
//   contractions over degrees m..ltr+1 using
//     sin(theta) dP_l/dtheta = l d_{l+1} P_{l+1} - (l+1) d_l P_{l-1},
//     d_l = sqrt((l^2 - m^2) / (4 l^2 - 1))              (src/legendre.jl:478-555)
//   so (Gtheta, Gphi) = (1/sin theta) sum_j P_j U_j with U built from S, T
//   (sphtor_pre64), and analysis recombines the two scalar sums (sphtor_post64).
#include <cmath>

#include "kernels.cuh"

namespace shtb {

// ---------------------------------------------------------------------------
// vector coefficient transforms
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fct(const PlanDev& P, const Factors& F, long long poff, int l, int m, int div_ll) {
  double s = (m == 0) ? F.mf0 : F.mf1;
  if (F.fac) s *= F.fac[poff + (l - m)];
  if (F.sc_mode) {
    const double q = F.sc[l + (long long)(P.lmax + 1) * m];
    s = (F.sc_mode == 1) ? s * q : s / q;
  }
  if (div_ll) s /= ((double)l * (double)(l + 1));
  return s;
}

__device__ __forceinline__ double2 imul(double2 v, double s) {  // i * s * v
  return make_double2(-s * v.y, s * v.x);
}

__global__ void sphtor_pre64_kernel(PlanDev P, const double2* __restrict__ S, const double2* __restrict__ T,
                                    double2* __restrict__ U, long long ldu, int ltr, Factors F, int div_ll,
                                    const double* __restrict__ dco) {
  const int im = blockIdx.y, m = im * P.mres, k = blockIdx.z;
  const int j = m + blockIdx.x * blockDim.x + threadIdx.x;
  const int jend = min(ltr + 1, P.lrec);
  if (j > jend) return;
  const long long poff = P.off[im];
  const long long ld = (long long)(P.lmax + 1) * (P.mmax + 1);
  const double2* Sk = S + (long long)k * ld + (long long)m * (P.lmax + 1);
  const double2* Tk = T + (long long)k * ld + (long long)m * (P.lmax + 1);
  const int lo = max(1, m);
  auto sv = [&](const double2* A, int l) -> double2 {
    if (l < lo || l > ltr) return make_double2(0.0, 0.0);
    const double s = fct(P, F, poff, l, m, div_ll);
    const double2 v = A[l];
    return make_double2(v.x * s, v.y * s);
  };
  const double cj = P.cfac[poff + (j - m)];
  const double dj = dco[poff + (j - m)];
  const double dj1 = (j + 1 <= P.lrec) ? dco[poff + (j + 1 - m)] : 0.0;
  const double am = (double)(j - 1) * dj, bp = (double)(j + 2) * dj1;
  const double2 sm1 = sv(Sk, j - 1), sp1 = sv(Sk, j + 1), s0 = sv(Sk, j);
  const double2 tm1 = sv(Tk, j - 1), tp1 = sv(Tk, j + 1), t0 = sv(Tk, j);
  const double2 it = imul(t0, (double)m), is = imul(s0, (double)m);
  double2 ut, up;
  ut.x = cj * (am * sm1.x - bp * sp1.x - it.x);
  ut.y = cj * (am * sm1.y - bp * sp1.y - it.y);
  up.x = cj * (is.x + am * tm1.x - bp * tp1.x);
  up.y = cj * (is.y + am * tm1.y - bp * tp1.y);
  U[(2LL * k) * ldu + poff + (j - m)] = ut;
  U[(2LL * k + 1) * ldu + poff + (j - m)] = up;
}

__global__ void sphtor_post64_kernel(PlanDev P, const double2* __restrict__ V, long long ldu, double2* __restrict__ S,
                                     double2* __restrict__ T, int ltr, Factors F, int div_ll,
                                     const double* __restrict__ dco) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y, k = blockIdx.z;
  if (l > P.lmax) return;
  const long long ld = (long long)(P.lmax + 1) * (P.mmax + 1);
  const long long o = (long long)k * ld + (long long)m * (P.lmax + 1) + l;
  const int lo = max(1, m);
  if ((m % P.mres) != 0 || m > ltr || l < lo || l > ltr) {
    S[o] = make_double2(0.0, 0.0);
    T[o] = make_double2(0.0, 0.0);
    return;
  }
  const int im = m / P.mres;
  const long long poff = P.off[im];
  const int jend = ltr + 1;
  const double2* Vt = V + (2LL * k) * ldu + poff - m;
  const double2* Vp = V + (2LL * k + 1) * ldu + poff - m;
  auto at = [&](const double2* A, int j) -> double2 {
    return (j >= m && j <= jend) ? A[j] : make_double2(0.0, 0.0);
  };
  const double pre = fct(P, F, poff, l, m, div_ll);
  const double cl = P.cfac[poff + (l - m)], cl1 = P.cfac[poff + (l + 1 - m)];
  const double clm1 = (l - 1 >= m) ? P.cfac[poff + (l - 1 - m)] : 0.0;
  const double dl = dco[poff + (l - m)], dl1 = dco[poff + (l + 1 - m)];
  const double A = (double)l * dl1 * cl1, B = (double)(l + 1) * dl * clm1, C = (double)m * cl;
  const double2 tp = at(Vt, l + 1), tm = at(Vt, l - 1), t0 = at(Vt, l);
  const double2 pp = at(Vp, l + 1), pm = at(Vp, l - 1), p0 = at(Vp, l);
  const double2 ip = imul(p0, C), itt = imul(t0, C);
  S[o] = make_double2(pre * (A * tp.x - B * tm.x - ip.x), pre * (A * tp.y - B * tm.y - ip.y));
  T[o] = make_double2(pre * (itt.x + A * pp.x - B * pm.x), pre * (itt.y + A * pp.y - B * pm.y));
}

__global__ void zero_columns64_kernel(PlanDev P, double2* __restrict__ a, int mlim) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y, k = blockIdx.z;
  if (l > P.lmax) return;
  if ((m % P.mres) != 0 || m > mlim)
    a[(long long)k * (P.lmax + 1) * (P.mmax + 1) + (long long)m * (P.lmax + 1) + l] = make_double2(0.0, 0.0);
}

int launch_sphtor_pre64(const shtb_plan* p, const double2* S, const double2* T, double2* U, int nf, int ltr,
                        const Factors& F, int div_ll, cudaStream_t st) {
  const int mlim = std::min(p->mmax, ltr);
  const int nmu = mlim / p->mres + 1;
  dim3 grid((p->lrec + 1 + 127) / 128, nmu, nf);
  prof_begin(st);
  sphtor_pre64_kernel<<<grid, 128, 0, st>>>(p->dev, S, T, U, p->hoff[p->nm], ltr, F, div_ll, p->d_dcoef);
  SHTB_LAUNCHED("sphtor pre-combine kernel");
  return SHTB_OK;
}

int launch_sphtor_post64(const shtb_plan* p, const double2* V, double2* S, double2* T, int nf, int ltr,
                         const Factors& F, int div_ll, cudaStream_t st) {
  dim3 grid((p->lmax + 1 + 127) / 128, p->mmax + 1, nf);
  prof_begin(st);
  sphtor_post64_kernel<<<grid, 128, 0, st>>>(p->dev, V, p->hoff[p->nm], S, T, ltr, F, div_ll, p->d_dcoef);
  SHTB_LAUNCHED("sphtor post-combine kernel");
  return SHTB_OK;
}

int launch_zero_columns64(const shtb_plan* p, double2* a, int nf, int mlim, cudaStream_t st) {
  dim3 grid((p->lmax + 1 + 127) / 128, p->mmax + 1, nf);
  prof_begin(st);
  zero_columns64_kernel<<<grid, 128, 0, st>>>(p->dev, a, mlim);
  SHTB_LAUNCHED("zero columns kernel");
  return SHTB_OK;
}

}  // namespace shtb

using namespace shtb;

// ---------------------------------------------------------------------------
// validation and workspace
// ---------------------------------------------------------------------------
static size_t wbytes_fourier(const shtb_plan* p, int nfw, size_t celem) {
  return (size_t)nfw * p->nm * 2 * p->npair * celem;
}
static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

extern "C" size_t shtb_workspace_bytes(const shtb_plan* p, int op, int nfields, int dtype, int precision) {
  if (!p || nfields < 1) return 0;
  const size_t celem = (precision == SHTB_PREC_MIXED) ? 8 : 16;
  (void)dtype;
  switch (op) {
    case SHTB_OP_SYNTHESIS:
    case SHTB_OP_ANALYSIS:
      if (precision == SHTB_PREC_MIXED) return mixed_workspace_bytes(p, op, nfields);
      return align256(wbytes_fourier(p, nfields, celem));
    case SHTB_OP_SYNTHESIS_SPHTOR:
    case SHTB_OP_ANALYSIS_SPHTOR:
      return align256(wbytes_fourier(p, 2 * nfields, celem)) + align256((size_t)2 * nfields * p->hoff[p->nm] * 16);
    default:
      return 0;
  }
}

static bool aligned16(const void* q) { return ((uintptr_t)q & 15u) == 0; }

static int check_common(const shtb_plan* p, int nf, int* ltr, int dtype, int precision, const void* work,
                        size_t wb, int op) {
  if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan is NULL");
  if (nf < 1) return set_error(SHTB_ERR_BAD_ARG, "nfields must be >= 1");
  if (*ltr < 0) *ltr = p->lmax;
  if (*ltr > p->lmax)
    return set_error(SHTB_ERR_BAD_ARG, "lcap must satisfy 0 <= lcap <= lmax=" + std::to_string(p->lmax));
  if (precision != SHTB_PREC_FP64 && precision != SHTB_PREC_MIXED)
    return set_error(SHTB_ERR_BAD_ARG, "unknown precision");
  if (dtype != SHTB_F64 && dtype != SHTB_F32) return set_error(SHTB_ERR_BAD_ARG, "unknown dtype");
  if (precision == SHTB_PREC_FP64 && dtype != SHTB_F64)
    return set_error(SHTB_ERR_UNSUPPORTED, "the FP64 path takes double buffers (dtype SHTB_F64)");
  if (precision == SHTB_PREC_MIXED && dtype != SHTB_F32)
    return set_error(SHTB_ERR_UNSUPPORTED, "the mixed-precision path takes float buffers (dtype SHTB_F32)");
  const size_t need = shtb_workspace_bytes(p, op, nf, dtype, precision);
  if (!work || wb < need)
    return set_error(SHTB_ERR_WORKSPACE, "workspace of " + std::to_string(need) + " bytes required, got " +
                                             std::to_string(wb));
  if (((uintptr_t)work & 255u) != 0) return set_error(SHTB_ERR_ALIGN, "workspace must be 256-byte aligned");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device)
    return set_error(SHTB_ERR_BAD_ARG, "the current CUDA device differs from the plan's device");
  return SHTB_OK;
}

static int check_ptrs(std::initializer_list<const void*> ps) {
  for (const void* q : ps) {
    if (!q) return set_error(SHTB_ERR_BAD_ARG, "NULL buffer pointer");
    if (!aligned16(q)) return set_error(SHTB_ERR_ALIGN, "buffers must be 16-byte aligned");
  }
  return SHTB_OK;
}

static Factors fac_none() { return Factors{nullptr, nullptr, 0, 1.0, 1.0}; }

// Mixed-precision entry points live in mixed.cu.
namespace shtb {
int mixed_synthesis(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, void* work, cudaStream_t st,
                    int packed);
int mixed_analysis(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, void* work, cudaStream_t st,
                   int packed);
}

// ---------------------------------------------------------------------------
// scalar
// ---------------------------------------------------------------------------
// packed = 1: coefficients in the SHTns LM layout (nlm per field) instead of dense columns.
static int scalar_synthesis(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, int dtype, int precision,
                            void* work, size_t wb, void* stream, int packed) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_SYNTHESIS);
  if (rc) return rc;
  if ((rc = check_ptrs({alm, f}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = std::min(p->mmax, ltr);
  if (precision == SHTB_PREC_MIXED) return mixed_synthesis(p, alm, f, nf, ltr, work, st, packed);
  CoefSrc src = packed ? CoefSrc{(const double2*)alm, lm_count(p->lmax, p->mmax, p->mres), 0, 2}
                       : CoefSrc{(const double2*)alm, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 1 : 0, 1.0, 1.0};
  if ((rc = launch_leg_syn64(p, src, F, work, nf, ltr, mlim, st))) return rc;
  return launch_fft_syn<double, double>(p, work, (double*)f, nullptr, 1, nf, mlim, p->phi_inv_scale / p->nlon, 0, 0, st);
}

static int scalar_analysis(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, int dtype, int precision,
                           void* work, size_t wb, void* stream, int packed) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_ANALYSIS);
  if (rc) return rc;
  if ((rc = check_ptrs({alm, f}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = std::min(p->mmax, ltr);
  if (precision == SHTB_PREC_MIXED) return mixed_analysis(p, f, alm, nf, ltr, work, st, packed);
  if ((rc = launch_fft_ana<double, double>(p, (const double*)f, nullptr, 1, work, nf, mlim, p->ana_scale, 1, 0, st)))
    return rc;
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 2 : 0, 1.0, 1.0};
  if (packed) {
    // every order's block is written for l <= ltr; degrees above ltr and orders above it start cleared
    const long long nlm = lm_count(p->lmax, p->mmax, p->mres);
    if (ltr < p->lmax)
      SHTB_TRY_CUDA(cudaMemsetAsync(alm, 0, (size_t)nlm * nf * sizeof(double2), st), "packed output clear");
    CoefSink dst{(double2*)alm, nlm, 0, 2};
    return launch_leg_ana64(p, work, nf, ltr, mlim, dst, F, 0, st);
  }
  CoefSink dst{(double2*)alm, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  if ((rc = launch_leg_ana64(p, work, nf, ltr, mlim, dst, F, 1, st))) return rc;
  if (p->mres > 1 || mlim < p->mmax) return launch_zero_columns64(p, (double2*)alm, nf, mlim, st);
  return SHTB_OK;
}

// Complex grids (FP64): synthesis with real_output = false, analysis of complex fields.
extern "C" int shtb_synthesis_cplx(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, void* work,
                                   size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_SYNTHESIS);
  if (rc) return rc;
  if ((rc = check_ptrs({alm, f}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = std::min(p->mmax, ltr);
  CoefSrc src{(const double2*)alm, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 1 : 0, 1.0, 1.0};
  if ((rc = launch_leg_syn64(p, src, F, work, nf, ltr, mlim, st))) return rc;
  return launch_fft_cplx64(p, 1, work, f, nf, mlim, p->phi_inv_scale / p->nlon, st);
}

extern "C" int shtb_analysis_cplx(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, void* work,
                                  size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_ANALYSIS);
  if (rc) return rc;
  if ((rc = check_ptrs({alm, f}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = std::min(p->mmax, ltr);
  if ((rc = launch_fft_cplx64(p, 0, f, work, nf, mlim, p->ana_scale, st))) return rc;
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 2 : 0, 1.0, 1.0};
  CoefSink dst{(double2*)alm, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  if ((rc = launch_leg_ana64(p, work, nf, ltr, mlim, dst, F, 1, st))) return rc;
  if (p->mres > 1 || mlim < p->mmax) return launch_zero_columns64(p, (double2*)alm, nf, mlim, st);
  return SHTB_OK;
}

extern "C" int shtb_synthesis(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, int dtype,
                              int precision, void* work, size_t wb, void* stream) {
  return scalar_synthesis(p, alm, f, nf, ltr, dtype, precision, work, wb, stream, 0);
}

extern "C" int shtb_analysis(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, int dtype,
                             int precision, void* work, size_t wb, void* stream) {
  return scalar_analysis(p, f, alm, nf, ltr, dtype, precision, work, wb, stream, 0);
}

extern "C" int shtb_synthesis_packed(const shtb_plan* p, const void* qlm, void* f, int nf, int ltr, int dtype,
                                     int precision, void* work, size_t wb, void* stream) {
  return scalar_synthesis(p, qlm, f, nf, ltr, dtype, precision, work, wb, stream, 1);
}

extern "C" int shtb_analysis_packed(const shtb_plan* p, const void* f, void* qlm, int nf, int ltr, int dtype,
                                    int precision, void* work, size_t wb, void* stream) {
  return scalar_analysis(p, f, qlm, nf, ltr, dtype, precision, work, wb, stream, 1);
}

// ---------------------------------------------------------------------------
// vector
// ---------------------------------------------------------------------------
static int vec_synthesis(const shtb_plan* p, const void* S, const void* T, void* Vt, void* Vp, int nf, int ltr,
                         const Factors& Fpre, int div_ll, double gscale, int use_w, int spow, void* work,
                         cudaStream_t st) {
  const int mlim = std::min(p->mmax, ltr);
  char* W = (char*)work;
  double2* U = (double2*)(W + align256(wbytes_fourier(p, 2 * nf, 16)));
  int rc = launch_sphtor_pre64(p, (const double2*)S, (const double2*)T, U, nf, ltr, Fpre, div_ll, st);
  if (rc) return rc;
  CoefSrc src{U, p->hoff[p->nm], 0, 1};
  if ((rc = launch_leg_syn64(p, src, fac_none(), W, 2 * nf, ltr + 1, mlim, st))) return rc;
  return launch_fft_syn<double, double>(p, W, (double*)Vt, (double*)Vp, 2, 2 * nf, mlim, gscale, use_w, spow, st);
}

static int vec_analysis(const shtb_plan* p, const void* Vt, const void* Vp, void* S, void* T, int nf, int ltr,
                        const Factors& Fpost, int div_ll, double wscale, int use_w, int spow, void* work,
                        cudaStream_t st) {
  const int mlim = std::min(p->mmax, ltr);
  char* W = (char*)work;
  double2* V = (double2*)(W + align256(wbytes_fourier(p, 2 * nf, 16)));
  int rc = launch_fft_ana<double, double>(p, (const double*)Vt, (const double*)Vp, 2, W, 2 * nf, mlim, wscale,
                                          use_w, spow, st);
  if (rc) return rc;
  CoefSink dst{V, p->hoff[p->nm], 0, 1};
  if ((rc = launch_leg_ana64(p, W, 2 * nf, ltr + 1, mlim, dst, fac_none(), 0, st))) return rc;
  return launch_sphtor_post64(p, V, (double2*)S, (double2*)T, nf, ltr, Fpost, div_ll, st);
}

extern "C" int shtb_synthesis_sphtor(const shtb_plan* p, const void* S, const void* T, void* Vt, void* Vp, int nf,
                                     int ltr, int dtype, int precision, void* work, size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_SYNTHESIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({S, T, Vt, Vp}))) return rc;
  if (precision != SHTB_PREC_FP64) return set_error(SHTB_ERR_UNSUPPORTED, "vector transforms run on the FP64 path");
  Factors F{nullptr, p->d_scale, p->d_scale ? 1 : 0, 1.0, 1.0};
  // (1/sin) from the dtheta identity; Robert form multiplies by sin again
  return vec_synthesis(p, S, T, Vt, Vp, nf, ltr, F, 0, p->phi_inv_scale / p->nlon, 0, p->robert ? 0 : 1, work,
                       (cudaStream_t)stream);
}

extern "C" int shtb_analysis_sphtor(const shtb_plan* p, const void* Vt, const void* Vp, void* S, void* T, int nf,
                                    int ltr, int dtype, int precision, void* work, size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_ANALYSIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({S, T, Vt, Vp}))) return rc;
  if (precision != SHTB_PREC_FP64) return set_error(SHTB_ERR_UNSUPPORTED, "vector transforms run on the FP64 path");
  Factors F{nullptr, p->d_scale, p->d_scale ? 2 : 0, 1.0, 1.0};
  return vec_analysis(p, Vt, Vp, S, T, nf, ltr, F, 1, p->ana_scale, 1, p->robert ? 2 : 1, work,
                      (cudaStream_t)stream);
}

// Divergence/vorticity spectra: S = -div / (l(l+1)) enters the sphtor synthesis as the
// factor -1 / (l(l+1)) of the pre-combine kernel; div = -l(l+1) S leaves the analysis as
// the factor -1 in place of its 1 / (l(l+1)).
extern "C" int shtb_synthesis_divvort(const shtb_plan* p, const void* D, const void* Z, void* Vt, void* Vp, int nf,
                                      int ltr, int dtype, int precision, void* work, size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_SYNTHESIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({D, Z, Vt, Vp}))) return rc;
  if (precision != SHTB_PREC_FP64) return set_error(SHTB_ERR_UNSUPPORTED, "vector transforms run on the FP64 path");
  Factors F{nullptr, p->d_scale, p->d_scale ? 1 : 0, -1.0, -1.0};
  return vec_synthesis(p, D, Z, Vt, Vp, nf, ltr, F, 1, p->phi_inv_scale / p->nlon, 0, p->robert ? 0 : 1, work,
                       (cudaStream_t)stream);
}

extern "C" int shtb_analysis_divvort(const shtb_plan* p, const void* Vt, const void* Vp, void* D, void* Z, int nf,
                                     int ltr, int dtype, int precision, void* work, size_t wb, void* stream) {
  int rc = check_common(p, nf, &ltr, dtype, precision, work, wb, SHTB_OP_ANALYSIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({D, Z, Vt, Vp}))) return rc;
  if (precision != SHTB_PREC_FP64) return set_error(SHTB_ERR_UNSUPPORTED, "vector transforms run on the FP64 path");
  Factors F{nullptr, p->d_scale, p->d_scale ? 2 : 0, -1.0, -1.0};
  return vec_analysis(p, Vt, Vp, D, Z, nf, ltr, F, 0, p->ana_scale, 1, p->robert ? 2 : 1, work,
                      (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// adjoints (src/core_transforms.jl:477-652, src/sphtor_transforms.jl:385-452)
// ---------------------------------------------------------------------------
extern "C" int shtb_synthesis_adjoint(const shtb_plan* p, const void* ybar, void* abar, int nf, void* work,
                                      size_t wb, void* stream) {
  int ltr = -1;
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_ANALYSIS);
  if (rc) return rc;
  if ((rc = check_ptrs({ybar, abar}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = p->mmax;
  // abar[l,m] = wm * (phi_inv_scale/nlon) * sum_i P(x_i) FFT(ybar)[i,m] * s_lm,  wm = 1 (m=0), 2 (m>0)
  if ((rc = launch_fft_ana<double, double>(p, (const double*)ybar, nullptr, 1, work, nf, mlim, 1.0, 0, 0, st)))
    return rc;
  const double phiadj = p->phi_inv_scale / p->nlon;
  CoefSink dst{(double2*)abar, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 1 : 0, phiadj, 2.0 * phiadj};
  if ((rc = launch_leg_ana64(p, work, nf, p->lmax, mlim, dst, F, 1, st))) return rc;
  if (p->mres > 1) return launch_zero_columns64(p, (double2*)abar, nf, mlim, st);
  return SHTB_OK;
}

extern "C" int shtb_analysis_adjoint(const shtb_plan* p, const void* abar, void* fbar, int nf, void* work,
                                     size_t wb, void* stream) {
  int ltr = -1;
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_SYNTHESIS);
  if (rc) return rc;
  if ((rc = check_ptrs({abar, fbar}))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int mlim = p->mmax;
  // fbar = Re ifft(F), F[i,m] = phiadj' w_i sum_l P A/s (no Hermitian fill): bins m>0 enter once,
  // so they are halved relative to the Hermitian synthesis kernel.
  const double phiadj = p->nlon * p->ana_scale;
  CoefSrc src{(const double2*)abar, (long long)(p->lmax + 1) * (p->mmax + 1), (long long)(p->lmax + 1), 0};
  Factors F{p->dev.cfac, p->d_scale, p->d_scale ? 2 : 0, phiadj, 0.5 * phiadj};
  if ((rc = launch_leg_syn64(p, src, F, work, nf, p->lmax, mlim, st))) return rc;
  return launch_fft_syn<double, double>(p, work, (double*)fbar, nullptr, 1, nf, mlim, 1.0 / p->nlon, 1, 0, st);
}

extern "C" int shtb_synthesis_sphtor_adjoint(const shtb_plan* p, const void* Vtbar, const void* Vpbar, void* Sbar,
                                             void* Tbar, int nf, void* work, size_t wb, void* stream) {
  int ltr = -1;
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_ANALYSIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({Vtbar, Vpbar, Sbar, Tbar}))) return rc;
  const double phiadj = p->phi_inv_scale / p->nlon;
  Factors F{nullptr, p->d_scale, p->d_scale ? 1 : 0, phiadj, 2.0 * phiadj};
  // Robert: cotangent * sin, then the 1/sin of the identity: net weight 1
  return vec_analysis(p, Vtbar, Vpbar, Sbar, Tbar, nf, p->lmax, F, 0, 1.0, 0, p->robert ? 0 : 1, work,
                      (cudaStream_t)stream);
}

extern "C" int shtb_analysis_sphtor_adjoint(const shtb_plan* p, const void* Sbar, const void* Tbar, void* Vtbar,
                                            void* Vpbar, int nf, void* work, size_t wb, void* stream) {
  int ltr = -1;
  int rc = check_common(p, nf, &ltr, SHTB_F64, SHTB_PREC_FP64, work, wb, SHTB_OP_SYNTHESIS_SPHTOR);
  if (rc) return rc;
  if ((rc = check_ptrs({Sbar, Tbar, Vtbar, Vpbar}))) return rc;
  const double phiadj = p->nlon * p->ana_scale;
  Factors F{nullptr, p->d_scale, p->d_scale ? 2 : 0, phiadj, 0.5 * phiadj};
  return vec_synthesis(p, Sbar, Tbar, Vtbar, Vpbar, nf, p->lmax, F, 1, 1.0 / p->nlon, 1, p->robert ? 2 : 1, work,
                       (cudaStream_t)stream);
}
