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
#include <cstring>

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

// Everything one FFT launch needs about one transform; the grouped kernels stage it in
// shared memory per work item.
template <typename T>
struct FFTJob {
  PlanDev P;
  FFTDesc fd;
  const int* perm;                        // rinv (synthesis) or rev (analysis)
  const typename V2<T>::type* Win;        // synthesis: Fourier buffer in
  typename V2<T>::type* Wout;             // analysis: Fourier buffer out
  T* g0;                                  // grid (synthesis out / analysis in), component 0
  T* g1;                                  // component 1 when ncomp == 2
  int ncomp, mlim, use_w, spow;
  int wtile;                              // analysis: 1 = write W as the GEMM's B tile images
  int nf;                                 //   (FP32), nf fields
  double scale;                           // synthesis: grid factor; analysis: weight factor
  const typename V2<T>::type* tw;
  const typename V2<T>::type* twp;
};

// Analysis B tile images: region (im, parity, K-step of 8 latitude pairs) =
// ((im * 2 + par) * nks8 + p / 8); field k in block k / 64 (see btile_off).
__device__ __forceinline__ size_t btile_base(int im, int par, int p, int k, int npair, int nf) {
  const size_t nks8 = (size_t)(npair + 7) / 8;
  return (((size_t)im * 2 + par) * nks8 + (p >> 3)) * (size_t)btile_nfp(nf) * 16 + (size_t)(k >> 6) * 1024;
}

// First DIF pass (radix R, span N/R) read straight from the grid: group (row h, j)
// takes longitudes j + q span of latitude pair p0 + h as z = f_north + i f_south.
// Consecutive threads take consecutive rows, so a warp's loads for one q cover whole
// 32-byte runs of latitudes.
template <typename T, typename V, int R, int H>
__device__ __forceinline__ void dif_first_from_grid(V* X, int S, int N, const T* __restrict__ in, int nlat, int p0,
                                                    int hv, const V* __restrict__ twp, int sh) {
  const int span = N / R;
  for (int b = threadIdx.x; b < H * span; b += blockDim.x) {
    const int h = b % H, j = b / H;
    const int pair = p0 + h, south = nlat - 1 - pair;
    const bool vn = h < hv, vs = vn && south != pair;
    V u[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const size_t off = (size_t)(j + q * span) * nlat;
      u[q].x = vn ? in[off + pair] : (T)0;
      u[q].y = vs ? in[off + south] : (T)0;
    }
    dft_small<T, V, R>(u, -1, nullptr, 0, R);
    if (j != 0) {
#pragma unroll
      for (int q = 1; q < R; ++q) u[q] = cmul(u[q], twp[(q - 1) * span + j]);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) X[h * S + fft_pad(j + q * span, sh)] = u[q];
  }
}

// Last DIF pass (radix R, span 1) written straight to the grid: group (row h, block)
// holds the storage positions block R + q, i.e. longitudes rinv[block R + q]; the
// per-pair factor g[h] is applied on the way out.
template <typename T, typename V, int R, int H>
__device__ __forceinline__ void dif_last_to_grid(const V* X, int S, int N, T* __restrict__ out, int nlat, int p0,
                                                 int hv, const int* __restrict__ rinv, const T* g, int sh) {
  const int ngrp = N / R;
  for (int b = threadIdx.x; b < H * ngrp; b += blockDim.x) {
    const int h = b % H, blk = b / H;
    V u[R];
#pragma unroll
    for (int q = 0; q < R; ++q) u[q] = X[h * S + fft_pad(blk * R + q, sh)];
    dft_small<T, V, R>(u, +1, nullptr, 0, R);
    if (h < hv) {
      const int pair = p0 + h, south = nlat - 1 - pair;
      const T gh = g[h];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        T* row = out + (size_t)rinv[blk * R + q] * nlat;
        row[pair] = u[q].x * gh;
        if (south != pair) row[south] = u[q].y * gh;
      }
    }
  }
}

// Latitude pairs p0 .. p0+H-1 of field k.
// Fourier-buffer loads of the synthesis (each value read once) that leave no line in L1, so
// the twiddle and permutation tables stay there.
__device__ __forceinline__ float2 ld_once(const float2* p) {
  float2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_once(const double2* p) {
  double2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

template <typename T, int H, bool GENERIC>
__device__ __forceinline__ void fft_syn_body(const FFTJob<T>& J, int p0, int k, unsigned char* smem_raw) {
  const PlanDev& P = J.P;
  const FFTDesc& fd = J.fd;
  const int* __restrict__ rinv = J.perm;
  const typename V2<T>::type* __restrict__ W = J.Win;
  T* __restrict__ out0 = J.g0;
  T* __restrict__ out1 = J.g1;
  const int ncomp = J.ncomp, mlim = J.mlim, use_w = J.use_w, spow = J.spow;
  const double gscale = J.scale;
  const typename V2<T>::type* __restrict__ tw = J.tw;
  const typename V2<T>::type* __restrict__ twp = J.twp;
  using V = typename V2<T>::type;
  const int sh = fft_padsh(fd, sizeof(V)), N = fd.n, S = fft_row_stride(N, sh);
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* gfac = reinterpret_cast<T*>(Z + ((GENERIC && fd.direct) ? 2 : 1) * H * S);
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
        Z[h * S + fft_pad(zlo + q, sh)] = z;
      }
    }
  }
  for (int h = threadIdx.x; h < H; h += blockDim.x) gfac[h] = (h < hv) ? pair_factor<T>(P, p0 + h, gscale, use_w, spow) : (T)0;
  __syncthreads();
  const int nmu = mlim / P.mres + 1;
  // one (im, pair) item per thread; consecutive threads read consecutive pairs of one m
  // FP32: all of a thread's (order, pair) items for H = 8 in flight together; FP64 keeps 4 (registers)
  constexpr int U = sizeof(T) == 4 ? 16 : 4;
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
          Ev[u] = ld_once(W + base);
          Ov[u] = ld_once(W + base + npair);
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
        Z[h * S + fft_pad(m, sh)] = a;
        Z[h * S + fft_pad(N - m, sh)] = b;
      }
    }
  }
  __syncthreads();
  T* out = (ncomp == 2 && (k & 1)) ? out1 : out0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  if (const int rl = fft_fusable_radix(fd, fd.nrad - 1)) {
    // all passes but the last in shared memory; the last one writes the grid
    fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, +1, 0, fd.nrad - 1);
    T* o = out + fbase;
    switch (rl) {
      case 16: dif_last_to_grid<T, V, 16, H>(Z, S, N, o, nlat, p0, hv, rinv, gfac, sh); break;
      case 8: dif_last_to_grid<T, V, 8, H>(Z, S, N, o, nlat, p0, hv, rinv, gfac, sh); break;
      case 4: dif_last_to_grid<T, V, 4, H>(Z, S, N, o, nlat, p0, hv, rinv, gfac, sh); break;
      default: dif_last_to_grid<T, V, 2, H>(Z, S, N, o, nlat, p0, hv, rinv, gfac, sh); break;
    }
    return;
  }
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, +1);
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
        const V z = Z[h * S + fft_pad(q, sh)];
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

// Latitude pairs p0 .. p0+H-1 of field k.
template <typename T, int H, bool GENERIC>
__device__ __forceinline__ void fft_ana_body(const FFTJob<T>& J, int p0, int k, unsigned char* smem_raw) {
  const PlanDev& P = J.P;
  const FFTDesc& fd = J.fd;
  const int* __restrict__ rev = J.perm;
  const T* __restrict__ in0 = J.g0;
  const T* __restrict__ in1 = J.g1;
  typename V2<T>::type* __restrict__ W = J.Wout;
  const int ncomp = J.ncomp, mlim = J.mlim, use_w = J.use_w, spow = J.spow;
  const double wscale = J.scale;
  const typename V2<T>::type* __restrict__ tw = J.tw;
  const typename V2<T>::type* __restrict__ twp = J.twp;
  using V = typename V2<T>::type;
  const int sh = fft_padsh(fd, sizeof(V)), N = fd.n, S = fft_row_stride(N, sh);
  V* Z = reinterpret_cast<V*>(smem_raw);
  V* scratch = Z + H * S;
  T* wfac = reinterpret_cast<T*>(Z + ((GENERIC && fd.direct) ? 2 : 1) * H * S);
  const int npair = P.npair, nlat = P.nlat;
  const int hv = min(H, npair - p0);
  const T* in = (ncomp == 2 && (k & 1)) ? in1 : in0;
  const size_t kk = (ncomp == 2) ? (size_t)(k >> 1) : (size_t)k;
  const size_t fbase = kk * (size_t)nlat * N;
  for (int h = threadIdx.x; h < H; h += blockDim.x) wfac[h] = (h < hv) ? pair_factor<T>(P, p0 + h, wscale, use_w, spow) : (T)0;
  if (const int r0 = fft_fusable_radix(fd, 0)) {
    // the first pass reads the grid; the remaining passes run in shared memory
    __syncthreads();   // wfac
    const T* src = in + fbase;
    switch (r0) {
      case 16: dif_first_from_grid<T, V, 16, H>(Z, S, N, src, nlat, p0, hv, twp + fd.twoff[0], sh); break;
      case 8: dif_first_from_grid<T, V, 8, H>(Z, S, N, src, nlat, p0, hv, twp + fd.twoff[0], sh); break;
      case 4: dif_first_from_grid<T, V, 4, H>(Z, S, N, src, nlat, p0, hv, twp + fd.twoff[0], sh); break;
      default: dif_first_from_grid<T, V, 2, H>(Z, S, N, src, nlat, p0, hv, twp + fd.twoff[0], sh); break;
    }
    __syncthreads();
    fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, -1, 1);
  } else {
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
      Z[h * S + fft_pad(j, sh)] = z;
    }
  }
  __syncthreads();
  fft_rows<T, V, GENERIC>(Z, scratch, H, S, fd, tw, twp, -1);
  }
  const int nmu = mlim / P.mres + 1;
  if constexpr (H % 4 == 0) {
    if (J.wtile && hv == H) {
      // B tile images, four pairs per thread: a K-slot quad of rows 2f and 2f+1 is one
      // 32-byte run, written as two 16-byte stores per parity
      float* Wf = reinterpret_cast<float*>(W);
      const int fl = k & 63;
      constexpr int NQ = H / 4;
      for (int idx = threadIdx.x; idx < nmu * NQ; idx += blockDim.x) {
        const int im = idx / NQ, qd = idx - im * NQ;
        const int m = im * P.mres;
        const int pm = fft_pad(rev[m], sh), pc = fft_pad(rev[m == 0 ? 0 : N - m], sh);
        float4 ex, ey, ox, oy;
        float* e0 = &ex.x; float* e1 = &ey.x; float* q0 = &ox.x; float* q1 = &oy.x;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int h = 4 * qd + u;
          const V Zm = Z[h * S + pm];
          V Zc = Z[h * S + pc];
          Zc.y = -Zc.y;
          const V sum = cadd(Zm, Zc), d = csub(Zm, Zc);
          V XN, XS;
          XN.x = sum.x * (T)0.5; XN.y = sum.y * (T)0.5;
          XS.x = d.y * (T)0.5;   XS.y = -d.x * (T)0.5;
          const T wt = wfac[h];
          const V E = cscale(cadd(XN, XS), wt), O = cscale(csub(XN, XS), wt);
          e0[u] = (float)E.x; e1[u] = (float)E.y; q0[u] = (float)O.x; q1[u] = (float)O.y;
        }
        const int p = p0 + 4 * qd, kk = p & 7;
        float* d0 = Wf + btile_base(im, 0, p, k, npair, J.nf) + btile_off(2 * fl, kk);
        float* d1 = Wf + btile_base(im, 1, p, k, npair, J.nf) + btile_off(2 * fl, kk);
        reinterpret_cast<float4*>(d0)[0] = ex;   // row 2f
        reinterpret_cast<float4*>(d0)[1] = ey;   // row 2f+1 (next 16 bytes)
        reinterpret_cast<float4*>(d1)[0] = ox;
        reinterpret_cast<float4*>(d1)[1] = oy;
      }
    }
  }
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    if constexpr (H % 4 == 0) {
      if (J.wtile && hv == H) break;
    }
    const int im = idx / H, h = idx - im * H;
    if (h >= hv) continue;
    const int m = im * P.mres;
    const V Zm = Z[h * S + fft_pad(rev[m], sh)];
    V Zc = Z[h * S + fft_pad(rev[m == 0 ? 0 : N - m], sh)];
    Zc.y = -Zc.y;
    const V sum = cadd(Zm, Zc), d = csub(Zm, Zc);
    V XN, XS;
    XN.x = sum.x * (T)0.5; XN.y = sum.y * (T)0.5;
    XS.x = d.y * (T)0.5;   XS.y = -d.x * (T)0.5;
    const T wt = wfac[h];
    const V E = cscale(cadd(XN, XS), wt), O = cscale(csub(XN, XS), wt);
    if (J.wtile) {
      float* Wf = reinterpret_cast<float*>(W);
      const int p = p0 + h;
      const size_t b0 = btile_base(im, 0, p, k, npair, J.nf), b1 = btile_base(im, 1, p, k, npair, J.nf);
      const int kk = p & 7, fl = k & 63;
      const float v[4] = {(float)E.x, (float)E.y, (float)O.x, (float)O.y};
      const size_t o[4] = {b0 + btile_off(2 * fl, kk), b0 + btile_off(2 * fl + 1, kk), b1 + btile_off(2 * fl, kk),
                           b1 + btile_off(2 * fl + 1, kk)};
#pragma unroll
      for (int q = 0; q < 4; ++q) Wf[o[q]] = v[q];
    } else {
      const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p0 + h;
      W[base] = E;
      W[base + npair] = O;
    }
  }
  if (J.wtile && p0 <= npair - 1 && npair - 1 < p0 + H) {
    // the block holding the last pair also zeroes the padding pairs npair .. npair8-1
    float* Wf = reinterpret_cast<float*>(W);
    const int pad = ((npair + 7) & ~7) - npair;
    for (int idx = threadIdx.x; idx < nmu * pad; idx += blockDim.x) {
      const int im = idx / pad, p = npair + idx - im * pad;
      const int kk = p & 7, fl = k & 63;
      for (int par = 0; par < 2; ++par) {
        const size_t b = btile_base(im, par, p, k, npair, J.nf);
        for (int c = 0; c < 2; ++c) Wf[b + btile_off(2 * fl + c, kk)] = 0.f;
      }
    }
  }
}

template <typename T, int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_syn_kernel(const __grid_constant__ FFTJob<T> J) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fft_syn_body<T, H, GENERIC>(J, blockIdx.x * H, blockIdx.y, smem_raw);
}

template <typename T, int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_ana_kernel(const __grid_constant__ FFTJob<T> J) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // B tile image output: blockIdx.x = field, blockIdx.y = pair block, so the fields' CTAs
  // that fill one B tile region (all fields of 8 pairs) run together and its lines
  // complete in L2; Fourier-buffer output: blockIdx.x = pair block, blockIdx.y = field.
  if (J.wtile)
    fft_ana_body<T, H, GENERIC>(J, blockIdx.y * H, blockIdx.x, smem_raw);
  else
    fft_ana_body<T, H, GENERIC>(J, blockIdx.x * H, blockIdx.y, smem_raw);
}

// Persistent FFTs over many independent transforms; item = (transform, first latitude
// pair, field), list sorted by decreasing row length. Each CTA claims the next item from
// the device counter *queue (zero at launch) when it finishes one. Shared memory is sized
// for the longest row of the group.
template <typename T, int H, bool GENERIC, bool SYN>
__global__ void __launch_bounds__(512) fft_group_kernel(const FFTJob<T>* __restrict__ jobs,
                                                        const int4* __restrict__ items, int nitems,
                                                        int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FFTJob<T> sj;
  __shared__ int4 s_it;
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = atomicAdd(queue, 1);
      s_it = (i < nitems) ? items[i] : make_int4(-1, 0, 0, 0);
      if (i < nitems) sj = jobs[s_it.x];
    }
    __syncthreads();
    const int4 it = s_it;
    if (it.x < 0) break;
    if (SYN)
      fft_syn_body<T, H, GENERIC>(sj, it.y, it.z, smem_raw);
    else
      fft_ana_body<T, H, GENERIC>(sj, it.y, it.z, smem_raw);
    __syncthreads();   // sj, s_it and the shared rows are rewritten for the next item
  }
}

// Floats of the analysis B tile images.
size_t fft_btile_floats(const shtb_plan* p, int nf) {
  return (size_t)p->nm * 2 * ((p->npair + 7) / 8) * btile_nfp(nf) * 16;
}

template <typename T>
static FFTJob<T> fft_job(const shtb_plan* p, const int* perm, const typename V2<T>::type* Win,
                         typename V2<T>::type* Wout, T* g0, T* g1, int ncomp, int mlim, double scale, int use_w,
                         int spow, int wtile = 0, int nf = 0) {
  using V = typename V2<T>::type;
  FFTJob<T> J;
  J.P = p->dev;
  J.fd = p->fft;
  J.perm = perm;
  J.Win = Win;
  J.Wout = Wout;
  J.g0 = g0;
  J.g1 = g1;
  J.ncomp = ncomp;
  J.mlim = mlim;
  J.use_w = use_w;
  J.spow = spow;
  J.wtile = wtile;
  J.nf = nf;
  J.scale = scale;
  J.tw = std::is_same<T, double>::value ? (const V*)p->d_tw64 : (const V*)p->d_tw32;
  J.twp = std::is_same<T, double>::value ? (const V*)p->d_twp64 : (const V*)p->d_twp32;
  return J;
}

// H latitude pairs per CTA: the largest power of two <= 16 whose shared-memory
// footprint stays within ~200 KB (one CTA of 512 threads per SM). Two CTAs of 256
// threads with half the pairs measured slower on B200: their grid segments shrink to
// 16 bytes and each FFT has half the threads.
static int fft_pick_h(const FFTDesc& fd, size_t celem, int npair) {
  const size_t S = (size_t)fft_row_stride(fd.n, fft_padsh(fd, celem));
  int h = 16;
  while (h > 1 && (size_t)h * S * celem * (fd.direct ? 2 : 1) + 16 * 8 > 200 * 1024) h >>= 1;
  while (h > 1 && h / 2 >= npair) h >>= 1;
  return h;
}

static size_t fft_smem(const FFTDesc& fd, size_t celem, int h) {
  return (size_t)h * fft_row_stride(fd.n, fft_padsh(fd, celem)) * celem * (fd.direct ? 2 : 1) + (size_t)h * 8 + 16;
}

static bool fft_generic(const shtb_plan* p) {
  bool g = p->fft.direct;
  for (int i = 0; i < p->fft.nrad; ++i) {
    const int r = p->fft.rad[i];
    g = g || !(r == 2 || r == 3 || r == 4 || r == 5 || r == 8 || r == 16);
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
  const FFTJob<T> J = fft_job<T>(p, p->d_rinv, (const V*)W, nullptr, out0, out1, ncomp, mlim, gscale, use_w, spow);
  prof_begin(st);
  kern<<<grid, 512, smem, st>>>(J);
  SHTB_LAUNCHED("fft synthesis kernel");
  return SHTB_OK;
}

template <typename T, int H>
static int launch_ana_h(const shtb_plan* p, const T* in0, const T* in1, int ncomp, void* W, int nfw, int mlim,
                        double wscale, int use_w, int spow, int wtile, cudaStream_t st) {
  using V = typename V2<T>::type;
  const size_t smem = fft_smem(p->fft, sizeof(V), H);
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the shared-memory FFT");
  auto kern = fft_generic(p) ? fft_ana_kernel<T, H, true> : fft_ana_kernel<T, H, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
  dim3 grid((p->npair + H - 1) / H, nfw);
  if (wtile) grid = dim3(nfw, (p->npair + H - 1) / H);
  const FFTJob<T> J = fft_job<T>(p, p->d_rev, nullptr, (V*)W, const_cast<T*>(in0), const_cast<T*>(in1), ncomp, mlim,
                                 wscale, use_w, spow, wtile, nfw);
  prof_begin(st);
  kern<<<grid, 512, smem, st>>>(J);
  SHTB_LAUNCHED("fft analysis kernel");
  return SHTB_OK;
}

template <typename T, typename GT>
int launch_fft_syn(const shtb_plan* p, const void* W, GT* out0, GT* out1, int ncomp, int nfw, int mlim,
                   double gscale, int use_w, int spow, cudaStream_t st) {
  static_assert(std::is_same<T, GT>::value, "grid and compute types match");
  if constexpr (std::is_same<T, float>::value) {
    if (ncomp == 1 && !use_w && !spow && fft2_applicable(p))
      return launch_fft2_syn(p, W, (float*)out0, nfw, mlim, gscale, st);
  }
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
                   double wscale, int use_w, int spow, cudaStream_t st, int wtile) {
  static_assert(std::is_same<T, GT>::value, "grid and compute types match");
  if constexpr (std::is_same<T, float>::value) {
    if (ncomp == 1 && use_w && !spow && wtile && fft2_applicable(p))
      return launch_fft2_ana(p, (const float*)in0, W, nfw, mlim, wscale, st);
  }
  switch (fft_pick_h(p->fft, sizeof(typename V2<T>::type), p->npair)) {
    case 16: return launch_ana_h<T, 16>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, wtile, st);
    case 8: return launch_ana_h<T, 8>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, wtile, st);
    case 4: return launch_ana_h<T, 4>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, wtile, st);
    case 2: return launch_ana_h<T, 2>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, wtile, st);
    default: return launch_ana_h<T, 1>(p, in0, in1, ncomp, W, nfw, mlim, wscale, use_w, spow, wtile, st);
  }
}

template int launch_fft_syn<double, double>(const shtb_plan*, const void*, double*, double*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<double, double>(const shtb_plan*, const double*, const double*, int, void*, int, int, double, int, int, cudaStream_t, int);
template int launch_fft_syn<float, float>(const shtb_plan*, const void*, float*, float*, int, int, int, double, int, int, cudaStream_t);
template int launch_fft_ana<float, float>(const shtb_plan*, const float*, const float*, int, void*, int, int, double, int, int, cudaStream_t, int);

// ---------------------------------------------------------------- complex grids (FP64)
// Complex-valued grids have no Hermitian symmetry, so each latitude row is its own complex
// sequence: a CTA holds the north and south rows of H latitude pairs (2H sequences).
// Synthesis with complex output (real_output = false, src/core_transforms.jl:293-344):
// bins m >= 0 of the north row are E + O, of the south row E - O, every other bin zero
// (no Hermitian fill), inverse FFT, times gscale. Analysis of a complex field: forward
// FFT of both rows, E = w (X_N + X_S), O = w (X_N - X_S) from their bins m >= 0.
template <int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_syn_cplx_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rinv,
                                                           const double2* __restrict__ tw,
                                                           const double2* __restrict__ twp,
                                                           const double2* __restrict__ W, double2* __restrict__ out,
                                                           int mlim, double gscale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int sh = fft_padsh(fd, sizeof(double2)), N = fd.n, S = fft_row_stride(N, sh);
  double2* Z = reinterpret_cast<double2*>(smem_raw);
  double2* scratch = Z + 2 * H * S;
  const int p0 = blockIdx.x * H, k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  const int hv = min(H, npair - p0);
  for (int idx = threadIdx.x; idx < 2 * H * N; idx += blockDim.x) Z[(idx / N) * S + fft_pad(idx % N, sh)] = make_double2(0.0, 0.0);
  __syncthreads();
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H, m = im * P.mres;
    if (h >= hv) continue;
    const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p0 + h;
    const double2 E = W[base], O = W[base + npair];
    Z[(2 * h) * S + fft_pad(m, sh)] = cadd(E, O);
    Z[(2 * h + 1) * S + fft_pad(m, sh)] = csub(E, O);
  }
  __syncthreads();
  fft_rows<double, double2, GENERIC>(Z, scratch, 2 * H, S, fd, tw, twp, +1);
  // storage position q holds longitude rinv[q]; threads take the 2H rows of one position
  for (int idx = threadIdx.x; idx < 2 * H * N; idx += blockDim.x) {
    const int r = idx % (2 * H), q = idx / (2 * H), h = r >> 1;
    if (h >= hv) continue;
    const int pair = p0 + h, row = (r & 1) ? nlat - 1 - pair : pair;
    if ((r & 1) && row == pair) continue;   // the equator row of odd nlat is its north row
    out[((size_t)k * N + rinv[q]) * nlat + row] = cscale(Z[r * S + fft_pad(q, sh)], gscale);
  }
}

template <int H, bool GENERIC>
__global__ void __launch_bounds__(512) fft_ana_cplx_kernel(PlanDev P, FFTDesc fd, const int* __restrict__ rev,
                                                           const double2* __restrict__ tw,
                                                           const double2* __restrict__ twp,
                                                           const double2* __restrict__ in, double2* __restrict__ W,
                                                           int mlim, double wscale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int sh = fft_padsh(fd, sizeof(double2)), N = fd.n, S = fft_row_stride(N, sh);
  double2* Z = reinterpret_cast<double2*>(smem_raw);
  double2* scratch = Z + 2 * H * S;
  const int p0 = blockIdx.x * H, k = blockIdx.y;
  const int npair = P.npair, nlat = P.nlat;
  const int hv = min(H, npair - p0);
  // threads take the 2H rows of one longitude (contiguous runs of the grid)
  for (int idx = threadIdx.x; idx < 2 * H * N; idx += blockDim.x) {
    const int r = idx % (2 * H), j = idx / (2 * H), h = r >> 1;
    double2 v = make_double2(0.0, 0.0);
    if (h < hv) {
      const int pair = p0 + h, row = (r & 1) ? nlat - 1 - pair : pair;
      if (!((r & 1) && row == pair)) v = in[((size_t)k * N + j) * nlat + row];
    }
    Z[r * S + fft_pad(j, sh)] = v;
  }
  __syncthreads();
  fft_rows<double, double2, GENERIC>(Z, scratch, 2 * H, S, fd, tw, twp, -1);
  const int nmu = mlim / P.mres + 1;
  for (int idx = threadIdx.x; idx < nmu * H; idx += blockDim.x) {
    const int im = idx / H, h = idx - im * H, m = im * P.mres;
    if (h >= hv) continue;
    const double wt = wscale * P.w[p0 + h];
    const double2 XN = Z[(2 * h) * S + fft_pad(rev[m], sh)], XS = Z[(2 * h + 1) * S + fft_pad(rev[m], sh)];
    const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p0 + h;
    W[base] = cscale(cadd(XN, XS), wt);
    W[base + npair] = cscale(csub(XN, XS), wt);
  }
}

// Latitude pairs per CTA for complex rows: the largest H <= 8 whose 2H padded rows fit
// ~200 KB of shared memory.
static int fft_pick_h_cplx(const FFTDesc& fd, int npair) {
  const size_t S = (size_t)fft_row_stride(fd.n, fft_padsh(fd, sizeof(double2)));
  int h = 8;
  while (h > 1 && (size_t)2 * h * S * sizeof(double2) * (fd.direct ? 2 : 1) > 200 * 1024) h >>= 1;
  while (h > 1 && h / 2 >= npair) h >>= 1;
  return h;
}

template <int H>
static int launch_cplx_h(const shtb_plan* p, int syn, const void* src, void* dst, int nf, int mlim, double scale,
                         cudaStream_t st) {
  const size_t smem = (size_t)2 * H * fft_row_stride(p->fft.n, fft_padsh(p->fft, sizeof(double2))) * sizeof(double2) *
                      (p->fft.direct ? 2 : 1);
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "nlon too large for the complex-row FFT");
  const bool gen = fft_generic(p);
  dim3 grid((p->npair + H - 1) / H, nf);
  prof_begin(st);
  if (syn) {
    auto kern = gen ? fft_syn_cplx_kernel<H, true> : fft_syn_cplx_kernel<H, false>;
    SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
    kern<<<grid, 512, smem, st>>>(p->dev, p->fft, p->d_rinv, p->d_tw64, p->d_twp64, (const double2*)src,
                                  (double2*)dst, mlim, scale);
    SHTB_LAUNCHED("fft synthesis kernel");
  } else {
    auto kern = gen ? fft_ana_cplx_kernel<H, true> : fft_ana_cplx_kernel<H, false>;
    SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fft smem attr");
    kern<<<grid, 512, smem, st>>>(p->dev, p->fft, p->d_rev, p->d_tw64, p->d_twp64, (const double2*)src,
                                  (double2*)dst, mlim, scale);
    SHTB_LAUNCHED("fft analysis kernel");
  }
  return SHTB_OK;
}

int launch_fft_cplx64(const shtb_plan* p, int syn, const void* src, void* dst, int nf, int mlim, double scale,
                      cudaStream_t st) {
  switch (fft_pick_h_cplx(p->fft, p->npair)) {
    case 8: return launch_cplx_h<8>(p, syn, src, dst, nf, mlim, scale, st);
    case 4: return launch_cplx_h<4>(p, syn, src, dst, nf, mlim, scale, st);
    case 2: return launch_cplx_h<2>(p, syn, src, dst, nf, mlim, scale, st);
    default: return launch_cplx_h<1>(p, syn, src, dst, nf, mlim, scale, st);
  }
}

// ---------------------------------------------------------------- grouped transforms
// Host-side pieces of the persistent grouped FP32 FFTs.

size_t fft_job_bytes_f32() { return sizeof(FFTJob<float>); }

void fft_fill_job_f32(const shtb_plan* p, int syn, const void* W, void* grid, int nf, void* host_job) {
  const int mlim = std::min(p->mmax, p->lmax);
  FFTJob<float> J = syn ? fft_job<float>(p, p->d_rinv, (const float2*)W, nullptr, (float*)grid, nullptr, 1, mlim,
                                         p->phi_inv_scale / p->nlon, 0, 0)
                        : fft_job<float>(p, p->d_rev, nullptr, (float2*)const_cast<void*>(W), (float*)grid, nullptr, 1,
                                         mlim, p->ana_scale, 1, 0, 1, nf);
  std::memcpy(host_job, &J, sizeof(J));
}

size_t fft_group_smem_f32(const shtb_plan* p, int h) { return fft_smem(p->fft, sizeof(float2), h); }

bool fft_plan_generic(const shtb_plan* p) { return fft_generic(p); }

template <int H, bool GENERIC>
static int launch_fft_group_h(int syn, const void* jobs, const int4* items, int nitems, int grid, size_t smem,
                              int* queue, cudaStream_t st) {
  auto kern = syn ? fft_group_kernel<float, H, GENERIC, true> : fft_group_kernel<float, H, GENERIC, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "group fft smem attr");
  kern<<<grid, 512, smem, st>>>((const FFTJob<float>*)jobs, items, nitems, queue);
  count_launch();
  SHTB_TRY_CUDA(cudaGetLastError(), "group fft launch");
  return SHTB_OK;
}

int launch_fft_group_f32(int syn, int h, bool generic, const void* jobs, const int4* items, int nitems, int grid,
                         size_t smem, int* queue, cudaStream_t st) {
  if (nitems <= 0) return SHTB_OK;
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "group FFT tile does not fit in shared memory");
#define SHTB_GFFT(H_)                                                                                 \
  if (h == H_) return generic ? launch_fft_group_h<H_, true>(syn, jobs, items, nitems, grid, smem, queue, st) \
                              : launch_fft_group_h<H_, false>(syn, jobs, items, nitems, grid, smem, queue, st);
  SHTB_GFFT(16) SHTB_GFFT(8) SHTB_GFFT(4) SHTB_GFFT(2)
#undef SHTB_GFFT
  return set_error(SHTB_ERR_BAD_ARG, "group FFT: unsupported pairs per CTA");
}

}  // namespace shtb
