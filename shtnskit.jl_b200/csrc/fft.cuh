// fft.cuh — shared-memory mixed-radix FFT along longitude.
//
// Each CTA transforms H latitude pairs (north row i, south row nlat-1-i) of one
// field. A pair is packed into ONE complex sequence z = f_north + i f_south of
// length nlon, so a complex FFT of nlon points yields both real transforms.
// The pair packing is also the equatorial fold: the analysis side writes
// E = w (X_N + X_S) and O = w (X_N - X_S) directly, and the synthesis side reads
// E/O and forms X_N = E + O, X_S = E - O.
//
// The transform is an in-place decimation-in-frequency mixed-radix FFT
// (radices 16, 8, 4, 2, 3, 5 and generic odd radices up to 13): every pass updates
// disjoint groups of r elements where they lie, so one shared buffer and one
// barrier per pass suffice for any thread count. The result comes out in
// mixed-radix digit-reversed order; callers read bin k at position rev[k]
// (a plan table). Indices are skewed by pad(n) = n + n/8 to spread the strided
// accesses of the late passes over the shared-memory banks.
//
// Sign conventions follow FFTW/Julia (src/fftutils.jl:280-305): forward
// F_k = sum_j f_j exp(-2 pi i j k / N), inverse without the 1/N (the caller's
// per-row factor carries it).
#pragma once

#include <cuda_runtime.h>

#include "internal.cuh"

namespace shtb {

template <typename T> struct V2;
template <> struct V2<double> { using type = double2; };
template <> struct V2<float> { using type = float2; };

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename V, typename T> __device__ __forceinline__ V cscale(V a, T s) { a.x *= s; a.y *= s; return a; }
// multiply by (dir * i): dir = -1 forward, +1 inverse
template <typename V> __device__ __forceinline__ V crot(V a, int dir) {
  V r;
  if (dir > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

__device__ __forceinline__ int fft_pad(int n, int sh) { return n + (n >> sh); }
__host__ __device__ inline int fft_row_stride(int n, int sh) { return n + (n >> sh) + 1; }
// Skew of a row of complex elements of celem bytes: the plan's choice for FP32 (8-byte
// elements); FP64 rows (16-byte elements) measured fastest with i + i/8 at every length.
__host__ __device__ inline int fft_padsh(const FFTDesc& fd, size_t celem) { return celem == 8 ? fd.padsh : 3; }
// Radix of pass s when the grid I/O can take it over (power-of-two radices), else 0.
__host__ __device__ inline int fft_fusable_radix(const FFTDesc& fd, int s) {
  if (fd.direct || fd.nrad < 2) return 0;
  const int r = fd.rad[s];
  return (r == 2 || r == 4 || r == 8 || r == 16) ? r : 0;
}

// In-register DFT of RADIX points in direction dir. Generic odd radices use the
// twiddle table tw[t] = exp(-2 pi i t / N) with step twstep = N / radix.
template <typename T, typename V, int RADIX>
__device__ __forceinline__ void dft_small(V* u, int dir, const V* __restrict__ tw, int twstep, int radix_rt) {
  if constexpr (RADIX == 2) {
    V a = u[0], b = u[1];
    u[0] = cadd(a, b);
    u[1] = csub(a, b);
  } else if constexpr (RADIX == 3) {
    const T h = (T)0.86602540378443864676;
    V t = cadd(u[1], u[2]);
    V s = cscale(crot(csub(u[1], u[2]), dir), h);
    V a = u[0];
    u[0] = cadd(a, t);
    V b = csub(a, cscale(t, (T)0.5));
    u[1] = cadd(b, s);
    u[2] = csub(b, s);
  } else if constexpr (RADIX == 4) {
    V t0 = cadd(u[0], u[2]), t1 = csub(u[0], u[2]);
    V t2 = cadd(u[1], u[3]), t3 = crot(csub(u[1], u[3]), dir);
    u[0] = cadd(t0, t2);
    u[2] = csub(t0, t2);
    u[1] = cadd(t1, t3);
    u[3] = csub(t1, t3);
  } else if constexpr (RADIX == 5) {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    V a1 = cadd(u[1], u[4]), a2 = cadd(u[2], u[3]);
    V b1 = csub(u[1], u[4]), b2 = csub(u[2], u[3]);
    V x0 = u[0];
    u[0] = cadd(x0, cadd(a1, a2));
    V p1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
    V p2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
    // forward: X1 = p1 - i(s1 b1 + s2 b2), X2 = p2 - i(s2 b1 - s1 b2)
    V q1 = crot(cadd(cscale(b1, s1), cscale(b2, s2)), dir);
    V q2 = crot(csub(cscale(b1, s2), cscale(b2, s1)), dir);
    u[1] = cadd(p1, q1);
    u[4] = csub(p1, q1);
    u[2] = cadd(p2, q2);
    u[3] = csub(p2, q2);
  } else if constexpr (RADIX == 8) {
    V e[4] = {u[0], u[2], u[4], u[6]}, o[4] = {u[1], u[3], u[5], u[7]};
    dft_small<T, V, 4>(e, dir, tw, twstep, 4);
    dft_small<T, V, 4>(o, dir, tw, twstep, 4);
    const T r = (T)0.70710678118654752440;
    // w8^k = exp(dir * 2 pi i k / 8)
    V w1, w3;
    w1.x = r; w1.y = dir > 0 ? r : -r;
    w3.x = -r; w3.y = dir > 0 ? r : -r;
    V o1 = cmul(o[1], w1), o2 = crot(o[2], dir), o3 = cmul(o[3], w3);
    u[0] = cadd(e[0], o[0]); u[4] = csub(e[0], o[0]);
    u[1] = cadd(e[1], o1);   u[5] = csub(e[1], o1);
    u[2] = cadd(e[2], o2);   u[6] = csub(e[2], o2);
    u[3] = cadd(e[3], o3);   u[7] = csub(e[3], o3);
  } else if constexpr (RADIX == 16) {
    // 16 = 4 x 4: DFT4 over n1 of x[4 n1 + n2], twiddle W16^(n2 k1), DFT4 over n2;
    // X[k1 + 4 k2] lands in u[k1 + 4 k2]
    V a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      V t[4] = {u[n2], u[n2 + 4], u[n2 + 8], u[n2 + 12]};
      dft_small<T, V, 4>(t, dir, tw, twstep, 4);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    // W16^e = exp(dir 2 pi i e / 16) for e = n2 k1 in {1, 2, 3, 4, 6, 9}
    const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, r2 = (T)0.70710678118654752440;
    const T sd = dir > 0 ? (T)1 : (T)-1;
    V w1, w2, w3, w6, w9;
    w1.x = c1;  w1.y = sd * s1;
    w2.x = r2;  w2.y = sd * r2;
    w3.x = s1;  w3.y = sd * c1;
    w6.x = -r2; w6.y = sd * r2;
    w9.x = -c1; w9.y = -sd * s1;
    a[1][1] = cmul(a[1][1], w1); a[1][2] = cmul(a[1][2], w2); a[1][3] = cmul(a[1][3], w3);
    a[2][1] = cmul(a[2][1], w2); a[2][2] = crot(a[2][2], dir); a[2][3] = cmul(a[2][3], w6);
    a[3][1] = cmul(a[3][1], w3); a[3][2] = cmul(a[3][2], w6); a[3][3] = cmul(a[3][3], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      V t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      dft_small<T, V, 4>(t, dir, tw, twstep, 4);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) u[k1 + 4 * k2] = t[k2];
    }
  } else {
    V out[RADIX];
#pragma unroll
    for (int a = 0; a < RADIX; ++a) {
      V acc;
      acc.x = 0; acc.y = 0;
      if (a < radix_rt) {
#pragma unroll
        for (int q = 0; q < RADIX; ++q) {
          if (q < radix_rt) {
            V wv = tw[((a * q) % radix_rt) * twstep];
            if (dir > 0) wv.y = -wv.y;
            acc = cadd(acc, cmul(u[q], wv));
          }
        }
      }
      out[a] = acc;
    }
#pragma unroll
    for (int a = 0; a < RADIX; ++a) u[a] = out[a];
  }
}

// One DIF pass of radix r on sub-transforms of length Ns (all F rows, stride S):
// for j < Ns/r, element group {base + j + q*Ns/r}: DFT_r, then twiddle
// W_Ns^(j*q) on output q, read from this pass's table twp[(q-1)*span + j].
// Group indices are split with multiply-high divisions (magic_div_mul), and each
// thread loads two groups before computing either so their loads overlap.
template <typename T, typename V, int RADIX>
__device__ __forceinline__ void dif_group_load(const V* X, int S, int N, int span, unsigned mrow, unsigned mspan,
                                               int per_row, int r, int b, V* u, int& rowoff, int& base, int& j,
                                               int sh) {
  const int f = mrow ? (int)__umulhi((unsigned)b, mrow) : b;
  const int t = b - f * per_row;
  const int blk = mspan ? (int)__umulhi((unsigned)t, mspan) : t;
  j = t - blk * span;
  base = blk * span * r + j;
  rowoff = f * S;
#pragma unroll
  for (int q = 0; q < RADIX; ++q)
    if (q < r) u[q] = X[rowoff + fft_pad(base + q * span, sh)];
}

template <typename T, typename V, int RADIX>
__device__ __forceinline__ void dif_group_finish(V* X, int span, int r, const V* __restrict__ tw, int N,
                                                 const V* __restrict__ twp, int dir, V* u, int rowoff, int base, int j,
                                                 int sh) {
  dft_small<T, V, RADIX>(u, dir, tw, N / r, r);
  if (j != 0) {
#pragma unroll
    for (int q = 1; q < RADIX; ++q) {
      if (q < r) {
        V wv = twp[(q - 1) * span + j];
        if (dir > 0) wv.y = -wv.y;
        u[q] = cmul(u[q], wv);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < RADIX; ++q)
    if (q < r) X[rowoff + fft_pad(base + q * span, sh)] = u[q];
}

template <typename T, typename V, int RADIX>
__device__ __forceinline__ void dif_pass(V* X, int F, int N, int S, int Ns, int radix_rt, const V* __restrict__ tw,
                                         const V* __restrict__ twp, unsigned mrow, unsigned mspan, int dir, int sh) {
  const int r = (RADIX >= 7) ? radix_rt : RADIX;
  const int span = Ns / r;            // distance between group members
  const int per_row = N / r;          // groups per row
  const int total = F * per_row;
  const int bd = blockDim.x;
  // two groups in flight for FP32 radices <= 8; FP64 and the generic radix keep one (registers)
  constexpr bool kTwo = (RADIX <= 8) && (sizeof(T) == 4);
  const int step = kTwo ? 2 * bd : bd;
  for (int b = threadIdx.x; b < total; b += step) {
    V u0[RADIX], u1[kTwo ? RADIX : 1];
    int ro0, ba0, j0, ro1 = 0, ba1 = 0, j1 = 0;
    const bool two = kTwo && (b + bd < total);
    dif_group_load<T, V, RADIX>(X, S, N, span, mrow, mspan, per_row, r, b, u0, ro0, ba0, j0, sh);
    if constexpr (kTwo) {
      if (two) dif_group_load<T, V, RADIX>(X, S, N, span, mrow, mspan, per_row, r, b + bd, u1, ro1, ba1, j1, sh);
    }
    dif_group_finish<T, V, RADIX>(X, span, r, tw, N, twp, dir, u0, ro0, ba0, j0, sh);
    if constexpr (kTwo) {
      if (two) dif_group_finish<T, V, RADIX>(X, span, r, tw, N, twp, dir, u1, ro1, ba1, j1, sh);
    }
  }
  __syncthreads();
}

// Full in-place FFT of F rows (natural-order input; output bin k at rev[k]), or its
// passes s0 .. s1-1 only (s1 < 0: to the end) when the caller fuses the first or the
// last pass with its global loads or stores. `scratch` (same size as X) is used only in
// direct mode (a prime factor above 13).
template <typename T, typename V, bool GENERIC>
__device__ void fft_rows(V* X, V* scratch, int F, int S, const FFTDesc& fd, const V* __restrict__ tw,
                         const V* __restrict__ twp, int dir, int s0 = 0, int s1 = -1) {
  const int N = fd.n, sh = fft_padsh(fd, sizeof(V));
  if (GENERIC && fd.direct) {
    // O(N^2) DFT into scratch, written at natural positions (rev = identity in direct mode)
    for (int idx = threadIdx.x; idx < F * N; idx += blockDim.x) {
      const int f = idx / N, k = idx - f * N;
      V acc;
      acc.x = 0; acc.y = 0;
      int t = 0;
      for (int n = 0; n < N; ++n) {
        V wv = tw[t];
        if (dir > 0) wv.y = -wv.y;
        acc = cadd(acc, cmul(X[(size_t)f * S + fft_pad(n, sh)], wv));
        t += k;
        if (t >= N) t -= N;
      }
      scratch[(size_t)f * S + fft_pad(k, sh)] = acc;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < F * N; idx += blockDim.x) {
      const int f = idx / N, k = idx - f * N;
      X[(size_t)f * S + fft_pad(k, sh)] = scratch[(size_t)f * S + fft_pad(k, sh)];
    }
    __syncthreads();
    return;
  }
  int Ns = N;
  for (int s = 0; s < s0; ++s) Ns /= fd.rad[s];
  const int send = s1 < 0 ? fd.nrad : s1;
  for (int s = s0; s < send; ++s) {
    const int r = fd.rad[s];
    const V* tp = twp + fd.twoff[s];
    const unsigned mr = fd.mrow[s], ms = fd.mspan[s];
    switch (r) {
      case 2: dif_pass<T, V, 2>(X, F, N, S, Ns, 2, tw, tp, mr, ms, dir, sh); break;
      case 3: dif_pass<T, V, 3>(X, F, N, S, Ns, 3, tw, tp, mr, ms, dir, sh); break;
      case 4: dif_pass<T, V, 4>(X, F, N, S, Ns, 4, tw, tp, mr, ms, dir, sh); break;
      case 5: dif_pass<T, V, 5>(X, F, N, S, Ns, 5, tw, tp, mr, ms, dir, sh); break;
      case 8: dif_pass<T, V, 8>(X, F, N, S, Ns, 8, tw, tp, mr, ms, dir, sh); break;
      case 16: dif_pass<T, V, 16>(X, F, N, S, Ns, 16, tw, tp, mr, ms, dir, sh); break;
      default:
        if constexpr (GENERIC) dif_pass<T, V, 13>(X, F, N, S, Ns, r, tw, tp, mr, ms, dir, sh);
        break;
    }
    Ns /= r;
  }
}

}  // namespace shtb
