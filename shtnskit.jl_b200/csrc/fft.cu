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

template <typename T, typename GT, bool GENERIC>
__global__ void __launch_bounds__(256) fft_syn_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rev,
                                                      const typename V2<T>::type* __restrict__ W,
                                                       GT* __restrict__ out0, GT* __restrict__ out1, int ncomp,
                                                       int mlim, int H, double gscale, int use_w, int spow,
                                                       const typename V2<T>::type* __restrict__ tw) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = fft_row_stride(N);
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
  // batched loads (U items in flight per thread) for memory-level parallelism
  constexpr int U = 4;
  for (int base0 = threadIdx.x; base0 < nmu * H; base0 += blockDim.x * U) {
    V Ev[U], Ov[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      Ev[u].x = Ev[u].y = Ov[u].x = Ov[u].y = 0;
      if (idx < nmu * H) {
        const int im = idx / H, h = idx - im * H, pair = p0 + h;
        if (pair < npair) {
          const size_t base = ((size_t)k * P.nm + im) * 2 * npair + pair;
          Ev[u] = W[base];
          Ov[u] = W[base + npair];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      if (idx >= nmu * H) continue;
      const int im = idx / H, h = idx - im * H, pair = p0 + h;
      if (pair >= npair) continue;
      const int m = im * P.mres;
      const V XN = cadd(Ev[u], Ov[u]), XS = csub(Ev[u], Ov[u]);
      if (m == 0) {
        V z;
        z.x = XN.x; z.y = XS.x;
        Z[h * S] = z;
      } else {
        V a, b;
        a.x = XN.x - XS.y; a.y = XN.y + XS.x;
        b.x = XN.x + XS.y; b.y = XS.x - XN.y;
        Z[h * S + fft_pad(m)] = a;
        Z[h * S + fft_pad(N - m)] = b;
      }
    }
  }
  __syncthreads();
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, +1);
  GT* out = (ncomp == 2 && (k & 1)) ? out1 : out0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  for (int idx = threadIdx.x; idx < N * H; idx += blockDim.x) {
    const int j = idx / H, h = idx - j * H, pair = p0 + h;
    if (pair >= npair) continue;
    const V z = Z[h * S + fft_pad(rev[j])];
    const T g = gfac[h];
    out[fbase + (size_t)j * nlat + pair] = (GT)(z.x * g);
    const int south = nlat - 1 - pair;
    if (south != pair) out[fbase + (size_t)j * nlat + south] = (GT)(z.y * g);
  }
}

template <typename T, typename GT, bool GENERIC>
__global__ void __launch_bounds__(256) fft_ana_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rev,
                                                      const GT* __restrict__ in0,
                                                       const GT* __restrict__ in1, int ncomp,
                                                       typename V2<T>::type* __restrict__ W, int mlim, int H,
                                                       double wscale, int use_w, int spow,
                                                       const typename V2<T>::type* __restrict__ tw) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = fft_row_stride(N);
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
  constexpr int U = 8;
  for (int base0 = threadIdx.x; base0 < N * H; base0 += blockDim.x * U) {
    T vn[U], vs[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      vn[u] = vs[u] = (T)0;
      if (idx < N * H) {
        const int j = idx / H, h = idx - j * H, pair = p0 + h;
        if (pair < npair) {
          vn[u] = (T)in[fbase + (size_t)j * nlat + pair];
          const int south = nlat - 1 - pair;
          if (south != pair) vs[u] = (T)in[fbase + (size_t)j * nlat + south];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      if (idx < N * H) {
        const int j = idx / H, h = idx - j * H;
        V z;
        z.x = vn[u];
        z.y = vs[u];
        Z[h * S + fft_pad(j)] = z;
      }
    }
  }
  __syncthreads();
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, -1);
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H, pair = p0 + h;
    if (pair >= npair) continue;
    const int m = im * P.mres;
    const V Zm = Z[h * S + fft_pad(rev[m])];
    V Zc = Z[h * S + fft_pad(rev[m == 0 ? 0 : N - m])];
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
  const int S = fft_row_stride(N);
  // enough latitude pairs for 32-byte (FP64) / 32-byte (FP32) row segments, up to 16
  int h = std::min(16, std::max(celem == 16 ? 2 : 4, 4096 / std::max(N, 1)));
  h = std::max(1, std::min(h, npair));
  auto need = [&](int hh) { return (size_t)hh * S * celem * (fd.direct ? 2 : 1) + (size_t)hh * 8 + 16; };
  while (h > 1 && need(h) > 100 * 1024) --h;
  if (need(h) > 220 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the shared-memory FFT");
  *H = h;
  *threads = 256;
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
  bool generic = p->fft.direct;
  for (int i = 0; i < p->fft.nrad; ++i) {
    const int r = p->fft.rad[i];
    generic = generic || !(r == 2 || r == 3 || r == 4 || r == 5 || r == 8);
  }
  auto kern = generic ? fft_syn_kernel<T, GT, true> : fft_syn_kernel<T, GT, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  prof_begin(st);
  kern<<<grid, threads, smem, st>>>(p->dev, p->fft, p->d_rev, (const V*)W, out0, out1, ncomp, mlim, H, gscale, use_w, spow, tw);
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
  bool generic = p->fft.direct;
  for (int i = 0; i < p->fft.nrad; ++i) {
    const int r = p->fft.rad[i];
    generic = generic || !(r == 2 || r == 3 || r == 4 || r == 5 || r == 8);
  }
  auto kern = generic ? fft_ana_kernel<T, GT, true> : fft_ana_kernel<T, GT, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  prof_begin(st);
  kern<<<grid, threads, smem, st>>>(p->dev, p->fft, p->d_rev, in0, in1, ncomp, (V*)W, mlim, H, wscale, use_w, spow, tw);
  SHTB_LAUNCHED("fft analysis kernel");
  return SHTB_OK;
}

template int launch_fft_syn<double, double>(const shtb_plan*, const void*, double*, double*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<double, double>(const shtb_plan*, const double*, const double*, int, void*, int, int, double, int, int, cudaStream_t);
template int launch_fft_syn<float, float>(const shtb_plan*, const void*, float*, float*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<float, float>(const shtb_plan*, const float*, const float*, int, void*, int, int, double, int, int, cudaStream_t);

}  // namespace shtb
