// fft.cu — longitude FFT kernels fused with the equatorial fold/unfold.
//
// Synthesis (fft_syn_kernel): W[k][im][E|O][pair] -> grid rows north/south.
// Analysis  (fft_ana_kernel): grid rows north/south -> W[k][im][E|O][pair], weighted.
//
// A CTA owns H consecutive latitude pairs of one field (H templated so the per-pair
// values live in registers). Global traffic moves in whole segments: a longitude row
// j of the grid contributes H north values (contiguous) and H south values
// (contiguous, reversed order), loaded/stored as 16-byte vectors when the grid's
// latitude count allows; W is read/written per order m as H contiguous complex values.
// The FFT itself (fft.cuh) leaves bins in digit-reversed positions, so the synthesis
// output loop walks shared memory in storage order q and writes longitude rinv[q].
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

// 16-byte vector of grid values
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };

template <typename T, int NV>
__device__ __forceinline__ void load_seg(const T* __restrict__ src, T* v) {
  using VT = typename Vec16<T>::type;
  constexpr int L = Vec16<T>::n;
#pragma unroll
  for (int c = 0; c < NV / L; ++c) {
    const VT x = *reinterpret_cast<const VT*>(src + c * L);
    const T* xs = reinterpret_cast<const T*>(&x);
#pragma unroll
    for (int u = 0; u < L; ++u) v[c * L + u] = xs[u];
  }
}
template <typename T, int NV>
__device__ __forceinline__ void store_seg(T* __restrict__ dst, const T* v) {
  using VT = typename Vec16<T>::type;
  constexpr int L = Vec16<T>::n;
#pragma unroll
  for (int c = 0; c < NV / L; ++c) {
    VT x;
    T* xs = reinterpret_cast<T*>(&x);
#pragma unroll
    for (int u = 0; u < L; ++u) xs[u] = v[c * L + u];
    *reinterpret_cast<VT*>(dst + c * L) = x;
  }
}

template <typename T, int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_syn_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rinv,
                                                      const typename V2<T>::type* __restrict__ W, T* __restrict__ out0,
                                                      T* __restrict__ out1, int ncomp, int mlim, double gscale,
                                                      int use_w, int spow, const typename V2<T>::type* __restrict__ tw,
                                                      const typename V2<T>::type* __restrict__ twp) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = fft_row_stride(N);
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* gfac = reinterpret_cast<T*>(Z + ((GENERIC && fd.direct) ? 2 : 1) * H * S);
  const int p0 = blockIdx.x * H;
  const int k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  const int hv = min(H, npair - p0);
  // Bins the order loop below does not write (|m| > mlim, or m off the mres lattice)
  // must be zero; with mres == 1 those are the bins mlim < q < N - mlim.
  {
    const int zlo = (P.mres == 1) ? mlim + 1 : 0, zhi = (P.mres == 1) ? N - mlim : N;
    const int zn = zhi - zlo;
    if (zn > 0) {
      V z;
      z.x = 0; z.y = 0;
      for (int idx = threadIdx.x; idx < H * zn; idx += blockDim.x) {
        const int h = idx / zn, q = idx - h * zn;
        Z[h * S + fft_pad(zlo + q)] = z;
      }
    }
  }
  for (int h = threadIdx.x; h < H; h += blockDim.x) gfac[h] = (h < hv) ? pair_factor<T>(P, p0 + h, gscale, use_w, spow) : (T)0;
  __syncthreads();
  const int nmu = mlim / P.mres + 1;
  // one (im, pair) item per thread; consecutive threads read consecutive pairs of one m
  constexpr int U = 4;
  for (int base0 = threadIdx.x; base0 < nmu * H; base0 += blockDim.x * U) {
    V Ev[U], Ov[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      Ev[u].x = Ev[u].y = Ov[u].x = Ov[u].y = 0;
      if (idx < nmu * H) {
        const int im = idx / H, h = idx - im * H;
        if (h < hv) {
          const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p0 + h;
          Ev[u] = W[base];
          Ov[u] = W[base + npair];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = base0 + u * blockDim.x;
      if (idx >= nmu * H) continue;
      const int im = idx / H, h = idx - im * H;
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
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, +1);
  T* out = (ncomp == 2 && (k & 1)) ? out1 : out0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  constexpr int L = Vec16<T>::n;
  const bool vec = (H % L == 0) && (hv == H) && (nlat % L == 0);
  constexpr int QU = 4;   // longitudes per thread per round; their rinv entries load together
  for (int q0 = threadIdx.x; q0 < N; q0 += QU * blockDim.x) {
    int jq[QU];
#pragma unroll
    for (int u = 0; u < QU; ++u) {
      const int q = q0 + u * blockDim.x;
      jq[u] = (q < N) ? rinv[q] : 0;
    }
#pragma unroll
    for (int u = 0; u < QU; ++u) {
      const int q = q0 + u * blockDim.x;
      if (q >= N) break;
      T vn[H], vs[H];
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const V z = Z[h * S + fft_pad(q)];
        vn[h] = z.x * gfac[h];
        vs[h] = z.y * gfac[h];
      }
      T* row = out + fbase + (size_t)jq[u] * nlat;
      if constexpr (H % L == 0) {
        if (vec) {
          T rs[H];
#pragma unroll
          for (int h = 0; h < H; ++h) rs[h] = vs[H - 1 - h];
          store_seg<T, H>(row + p0, vn);
          store_seg<T, H>(row + (nlat - p0 - H), rs);
          continue;
        }
      }
#pragma unroll
      for (int h = 0; h < H; ++h) {
        if (h >= hv) continue;
        const int pair = p0 + h;
        row[pair] = vn[h];
        const int south = nlat - 1 - pair;
        if (south != pair) row[south] = vs[h];
      }
    }
  }
}

template <typename T, int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_ana_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rev,
                                                      const T* __restrict__ in0, const T* __restrict__ in1, int ncomp,
                                                      typename V2<T>::type* __restrict__ W, int mlim, double wscale,
                                                      int use_w, int spow, const typename V2<T>::type* __restrict__ tw,
                                                      const typename V2<T>::type* __restrict__ twp) {
  using V = typename V2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = fd.n, S = fft_row_stride(N);
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* wfac = reinterpret_cast<T*>(Z + ((GENERIC && fd.direct) ? 2 : 1) * H * S);
  const int p0 = blockIdx.x * H;
  const int k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  const int hv = min(H, npair - p0);
  const T* in = (ncomp == 2 && (k & 1)) ? in1 : in0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  for (int h = threadIdx.x; h < H; h += blockDim.x) wfac[h] = (h < hv) ? pair_factor<T>(P, p0 + h, wscale, use_w, spow) : (T)0;
  constexpr int L = Vec16<T>::n;
  const bool vec = (H % L == 0) && (hv == H) && (nlat % L == 0);
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const T* row = in + fbase + (size_t)j * nlat;
    T vn[H], vs[H];
    bool done = false;
    if constexpr (H % L == 0) {
      if (vec) {
        T rs[H];
        load_seg<T, H>(row + p0, vn);
        load_seg<T, H>(row + (nlat - p0 - H), rs);
#pragma unroll
        for (int h = 0; h < H; ++h) vs[h] = rs[H - 1 - h];
        done = true;
      }
    }
    if (!done) {
#pragma unroll
      for (int h = 0; h < H; ++h) {
        vn[h] = vs[h] = (T)0;
        if (h < hv) {
          const int pair = p0 + h;
          vn[h] = row[pair];
          const int south = nlat - 1 - pair;
          if (south != pair) vs[h] = row[south];
        }
      }
    }
#pragma unroll
    for (int h = 0; h < H; ++h) {
      V z;
      z.x = vn[h];
      z.y = vs[h];
      Z[h * S + fft_pad(j)] = z;
    }
  }
  __syncthreads();
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, -1);
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H;
    if (h >= hv) continue;
    const int m = im * P.mres;
    const V Zm = Z[h * S + fft_pad(rev[m])];
    V Zc = Z[h * S + fft_pad(rev[m == 0 ? 0 : N - m])];
    Zc.y = -Zc.y;
    const V sum = cadd(Zm, Zc), d = csub(Zm, Zc);
    V XN, XS;
    XN.x = sum.x * (T)0.5; XN.y = sum.y * (T)0.5;
    XS.x = d.y * (T)0.5;   XS.y = -d.x * (T)0.5;
    const T wt = wfac[h];
    const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p0 + h;
    W[base] = cscale(cadd(XN, XS), wt);
    W[base + npair] = cscale(csub(XN, XS), wt);
  }
}

// H latitude pairs per CTA: the largest power of two <= 16 whose shared-memory
// footprint stays within ~200 KB (one CTA of 512 threads per SM). Two CTAs of 256
// threads with half the pairs measured slower on B200: their grid segments shrink to
// 16 bytes and each FFT has half the threads.
static int fft_pick_h(const FFTDesc& fd, size_t celem, int npair) {
  const size_t S = (size_t)fft_row_stride(fd.n);
  int h = 16;
  while (h > 1 && (size_t)h * S * celem * (fd.direct ? 2 : 1) + 16 * 8 > 200 * 1024) h >>= 1;
  while (h > 1 && h / 2 >= npair) h >>= 1;
  return h;
}

static size_t fft_smem(const FFTDesc& fd, size_t celem, int h) {
  return (size_t)h * fft_row_stride(fd.n) * celem * (fd.direct ? 2 : 1) + (size_t)h * 8 + 16;
}

static bool fft_generic(const shtb_plan* p) {
  bool g = p->fft.direct;
  for (int i = 0; i < p->fft.nrad; ++i) {
    const int r = p->fft.rad[i];
    g = g || !(r == 2 || r == 3 || r == 4 || r == 5 || r == 8);
  }
  return g;
}

template <typename T, int H>
static int launch_syn_h(const shtb_plan* p, const void* W, T* out0, T* out1, int ncomp, int nfw, int mlim,
                        double gscale, int use_w, int spow, cudaStream_t st) {
  using V = typename V2<T>::type;
  const size_t smem = fft_smem(p->fft, sizeof(V), H);
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the shared-memory FFT");
  auto kern = fft_generic(p) ? fft_syn_kernel<T, H, true> : fft_syn_kernel<T, H, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  const V* twp = std::is_same<T, double>::value ? (const V*)p->d_twp64 : (const V*)p->d_twp32;
  prof_begin(st);
  kern<<<grid, 512, smem, st>>>(p->dev, p->fft, p->d_rinv, (const V*)W, out0, out1, ncomp, mlim, gscale, use_w, spow, tw,
                                twp);
  SHTB_LAUNCHED("fft synthesis kernel");
  return SHTB_OK;
}

template <typename T, int H>
static int launch_ana_h(const shtb_plan* p, const T* in0, const T* in1, int ncomp, void* W, int nfw, int mlim,
                        double wscale, int use_w, int spow, cudaStream_t st) {
  using V = typename V2<T>::type;
  const size_t smem = fft_smem(p->fft, sizeof(V), H);
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the shared-memory FFT");
  auto kern = fft_generic(p) ? fft_ana_kernel<T, H, true> : fft_ana_kernel<T, H, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  const V* tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  const V* twp = std::is_same<T, double>::value ? (const V*)p->d_twp64 : (const V*)p->d_twp32;
  prof_begin(st);
  kern<<<grid, 512, smem, st>>>(p->dev, p->fft, p->d_rev, in0, in1, ncomp, (V*)W, mlim, wscale, use_w, spow, tw, twp);
  SHTB_LAUNCHED("fft analysis kernel");
  return SHTB_OK;
}

template <typename T, typename GT>
int launch_fft_syn(const shtb_plan* p, const void* W, GT* out0, GT* out1, int ncomp, int nfw, int mlim,
                   double gscale, int use_w, int spow, cudaStream_t st) {
  static_assert(std::is_same<T, GT>::value, "grid and compute types match");
  switch (fft_pick_h(p->fft, sizeof(typename V2<T>::type), p->npair)) {
    case 16: return launch_syn_h<T, 16>(p, W, out0, out1, ncomp, nfw, mlim, gscale, use_w, spow, st);
    case 8: return launch_syn_h<T, 8>(p, W, out0, out1, ncomp, nfw, mlim, gscale, use_w, spow, st);
    case 4: return launch_syn_h<T, 4>(p, W, out0, out1, ncomp, nfw, mlim, gscale, use_w, spow, st);
    case 2: return launch_syn_h<T, 2>(p, W, out0, out1, ncomp, nfw, mlim, gscale, use_w, spow, st);
    default: return launch_syn_h<T, 1>(p, W, out0, out1, ncomp, nfw, mlim, gscale, use_w, spow, st);
  }
}

template <typename T, typename GT>
int launch_fft_ana(const shtb_plan* p, const GT* in0, const GT* in1, int ncomp, void* W, int nfw, int mlim,
                   double wscale, int use_w, int spow, cudaStream_t st) {
  static_assert(std::is_same<T, GT>::value, "grid and compute types match");
  switch (fft_pick_h(p->fft, sizeof(typename V2<T>::type), p->npair)) {
    case 16: return launch_ana_h<T, 16>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, st);
    case 8: return launch_ana_h<T, 8>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, st);
    case 4: return launch_ana_h<T, 4>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, st);
    case 2: return launch_ana_h<T, 2>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, st);
    default: return launch_ana_h<T, 1>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, st);
  }
}

template int launch_fft_syn<double, double>(const shtb_plan*, const void*, double*, double*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<double, double>(const shtb_plan*, const double*, const double*, int, void*, int, int, double, int, int, cudaStream_t);
template int launch_fft_syn<float, float>(const shtb_plan*, const void*, float*, float*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<float, float>(const shtb_plan*, const float*, const float*, int, void*, int, int, double, int, int, cudaStream_t);

}  // namespace shtb
