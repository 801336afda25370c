// fft.cu — longitude FFT kernels fused with the equatorial fold/unfold.
//
// Synthesis (shtb_fft_syn): W[k][im][E|O][pair] -> grid rows north/south.
// Analysis  (shtb_fft_ana): grid rows north/south -> W[k][im][E|O][pair], weighted.
#include "fft.cuh"
#include "kernels.cuh"

namespace shtb {

template <typename T>
__device__ __forceinline__ T pair_factor(const PlanDev& P, int pair, double scale, int use_w, int spow) {
  double g = scale;
  if (use_w) g *= P.w[pair];
  if (spow) {
    const double s = P.sint[pair];
    g = (s > 0.0) ? g / (spow == 1 ? s : s * s) : 0.0;
  }
  return (T)g;
}

template <typename T, typename GT, int EMAX>
__global__ void __launch_bounds__(1024) fft_syn_kernel(PlanDev P, FFTDesc fd, const typename V2<T>::type* __restrict__ W,
                                                       GT* __restrict__ out0, GT* __restrict__ out1, int ncomp,
                                                       int mlim, int H, double gscale, int use_w, int spow,
                                                       const typename V2<T>::type* __restrict__ tw) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = N + 1;
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* gfac = reinterpret_cast<T*>(Z + (fd.direct ? 2 : 1) * H * S);
  const int p0 = blockIdx.x * H;
  const int k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  for (int idx = threadIdx.x; idx < H * S; idx += blockDim.x) {
    V z;
    z.x = 0; z.y = 0;
    Z[idx] = z;
  }
  for (int h = threadIdx.x; h < H; h += blockDim.x)
    gfac[h] = (p0 + h < npair) ? pair_factor<T>(P, p0 + h, gscale, use_w, spow) : (T)0;
  __syncthreads();
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H, pair = p0 + h;
    if (pair >= npair) continue;
    const int m = im * P.mres;
    const size_t base = ((size_t)k * P.nm + im) * 2 * npair + pair;
    const V E = W[base], O = W[base + npair];
    V XN = cadd(E, O), XS = csub(E, O);
    if (m == 0) {
      V z;
      z.x = XN.x; z.y = XS.x;
      Z[h * S] = z;
    } else {
      V a, b;
      a.x = XN.x - XS.y; a.y = XN.y + XS.x;
      b.x = XN.x + XS.y; b.y = XS.x - XN.y;
      Z[h * S + m] = a;
      Z[h * S + N - m] = b;
    }
  }
  __syncthreads();
  fft_rows<T, V, EMAX>(Z, scratch, H, S, fd, tw, +1);
  GT* out = (ncomp == 2 && (k & 1)) ? out1 : out0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  for (int idx = threadIdx.x; idx < N * H; idx += blockDim.x) {
    const int j = idx / H, h = idx - j * H, pair = p0 + h;
    if (pair >= npair) continue;
    const V z = Z[h * S + j];
    const T g = gfac[h];
    out[fbase + (size_t)j * nlat + pair] = (GT)(z.x * g);
    const int south = nlat - 1 - pair;
    if (south != pair) out[fbase + (size_t)j * nlat + south] = (GT)(z.y * g);
  }
}

template <typename T, typename GT, int EMAX>
__global__ void __launch_bounds__(1024) fft_ana_kernel(PlanDev P, FFTDesc fd, const GT* __restrict__ in0,
                                                       const GT* __restrict__ in1, int ncomp,
                                                       typename V2<T>::type* __restrict__ W, int mlim, int H,
                                                       double wscale, int use_w, int spow,
                                                       const typename V2<T>::type* __restrict__ tw) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = N + 1;
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* wfac = reinterpret_cast<T*>(Z + (fd.direct ? 2 : 1) * H * S);
  const int p0 = blockIdx.x * H;
  const int k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  const GT* in = (ncomp == 2 && (k & 1)) ? in1 : in0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  for (int h = threadIdx.x; h < H; h += blockDim.x)
    wfac[h] = (p0 + h < npair) ? pair_factor<T>(P, p0 + h, wscale, use_w, spow) : (T)0;
  for (int idx = threadIdx.x; idx < N * H; idx += blockDim.x) {
    const int j = idx / H, h = idx - j * H, pair = p0 + h;
    V z;
    z.x = 0; z.y = 0;
    if (pair < npair) {
      z.x = (T)in[fbase + (size_t)j * nlat + pair];
      const int south = nlat - 1 - pair;
      if (south != pair) z.y = (T)in[fbase + (size_t)j * nlat + south];
    }
    Z[h * S + j] = z;
  }
  __syncthreads();
  fft_rows<T, V, EMAX>(Z, scratch, H, S, fd, tw, -1);
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H, pair = p0 + h;
    if (pair >= npair) continue;
    const int m = im * P.mres;
    const V Zm = Z[h * S + m];
    V Zc = Z[h * S + (m == 0 ? 0 : N - m)];
    Zc.y = -Zc.y;
    const V sum = cadd(Zm, Zc), d = csub(Zm, Zc);
    V XN, XS;
    XN.x = sum.x * (T)0.5; XN.y = sum.y * (T)0.5;
    XS.x = d.y * (T)0.5;   XS.y = -d.x * (T)0.5;
    const T wt = wfac[h];
    const size_t base = ((size_t)k * P.nm + im) * 2 * npair + pair;
    W[base] = cscale(cadd(XN, XS), wt);
    W[base + npair] = cscale(csub(XN, XS), wt);
  }
}

static int fft_config(const FFTDesc& fd, size_t celem, int npair, int* H, int* threads, size_t* smem) {
  const int N = fd.n;
  constexpr int EMAX = 16;
  int h = std::max(1, std::min(16, 4096 / N));
  h = std::min(h, npair);
  const int S = N + 1;
  auto need = [&](int hh) { return (size_t)hh * S * celem * (fd.direct ? 2 : 1) + (size_t)hh * 8 + 16; };
  while (h > 1 && need(h) > 96 * 1024) --h;
  int t = (int)std::min<long long>(1024, std::max<long long>(256, ((long long)h * N + EMAX - 1) / EMAX));
  t = (t + 31) / 32 * 32;
  if ((long long)h * N > (long long)EMAX * t) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the FFT kernel");
  *H = h;
  *threads = t;
  *smem = need(h);
  return SHTB_OK;
}

template <typename T, typename GT>
int launch_fft_syn(const shtb_plan* p, const void* W, GT* out0, GT* out1, int ncomp, int nfw, int mlim,
                   double gscale, int use_w, int spow, cudaStream_t st) {
  using V = typename V2<T>::type;
  int H, threads;
  size_t smem;
  int rc = fft_config(p->fft, sizeof(V), p->npair, &H, &threads, &smem);
  if (rc) return rc;
  auto kern = fft_syn_kernel<T, GT, 16>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  prof_begin(st);
  kern<<<grid, threads, smem, st>>>(p->dev, p->fft, (const V*)W, out0, out1, ncomp, mlim, H, gscale, use_w, spow, tw);
  SHTB_LAUNCHED("fft synthesis kernel");
  return SHTB_OK;
}

template <typename T, typename GT>
int launch_fft_ana(const shtb_plan* p, const GT* in0, const GT* in1, int ncomp, void* W, int nfw, int mlim,
                   double wscale, int use_w, int spow, cudaStream_t st) {
  using V = typename V2<T>::type;
  int H, threads;
  size_t smem;
  int rc = fft_config(p->fft, sizeof(V), p->npair, &H, &threads, &smem);
  if (rc) return rc;
  auto kern = fft_ana_kernel<T, GT, 16>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  prof_begin(st);
  kern<<<grid, threads, smem, st>>>(p->dev, p->fft, in0, in1, ncomp, (V*)W, mlim, H, wscale, use_w, spow, tw);
  SHTB_LAUNCHED("fft analysis kernel");
  return SHTB_OK;
}

template int launch_fft_syn<double, double>(const shtb_plan*, const void*, double*, double*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<double, double>(const shtb_plan*, const double*, const double*, int, void*, int, int, double, int, int, cudaStream_t);
template int launch_fft_syn<float, float>(const shtb_plan*, const void*, float*, float*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<float, float>(const shtb_plan*, const float*, const float*, int, void*, int, int, double, int, int, cudaStream_t);

}  // namespace shtb
