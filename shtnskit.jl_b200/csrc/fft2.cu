// fft2.cu — FP32 longitude FFTs on packed pairs of sequences (f32x2).
//
// The general kernels (fft.cu) transform one complex sequence z = f_north + i f_south per
// latitude pair with scalar FP32 arithmetic. Here a thread carries the same point of TWO
// sequences (latitude pairs 2q and 2q + 1 of the CTA) at once, in structure-of-arrays form
//   re = (Re z_a, Re z_b), im = (Im z_a, Im z_b)
// so every add, multiply and FMA of the butterflies is one f32x2 instruction for both
// (sm_100 packed FP32: the FP32 pipe's full rate at half the instructions), shared memory
// moves 16 bytes per point-pair, and the grid side reads and writes the two adjacent
// latitudes of a row as one 8-byte access. The algorithm is the one of fft.cuh: an
// in-place decimation-in-frequency FFT (radices 16, 8, 4, 2) whose first pass (analysis)
// or last pass (synthesis) runs against the grid, with the equatorial fold into even/odd
// parts at the Fourier side.
//
// Scope: power-of-two nlon from 64 to 2048 and nlat a multiple of 4 (every latitude has
// its mirror, the south rows of two pairs are adjacent, and pair-pairs start on 16-byte
// boundaries of the Fourier buffer); other sizes use the general kernels.
// One CTA transforms 2 HP latitude pairs (HP pair-pairs) of one field with 128 HP threads.
#include <algorithm>
#include <cstring>

#include "fft.cuh"
#include "kernels.cuh"

namespace shtb {
namespace f2 {

typedef unsigned long long u64;

__device__ __forceinline__ u64 pk(float2 v) {
  u64 r;
  memcpy(&r, &v, 8);
  return r;
}
__device__ __forceinline__ float2 up(u64 v) {
  float2 r;
  memcpy(&r, &v, 8);
  return r;
}
__device__ __forceinline__ u64 add2(u64 a, u64 b) {
  u64 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b) {
  u64 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
  u64 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
  u64 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ u64 neg2(u64 a) { return sub2(0ull, a); }
__device__ __forceinline__ u64 bc(float v) { return pk(make_float2(v, v)); }

// The same point of two sequences.
struct C2 {
  u64 re, im;
};
__device__ __forceinline__ C2 cadd(C2 a, C2 b) { return C2{add2(a.re, b.re), add2(a.im, b.im)}; }
__device__ __forceinline__ C2 csub(C2 a, C2 b) { return C2{sub2(a.re, b.re), sub2(a.im, b.im)}; }
// a * (dir i): dir = -1 forward, +1 inverse
template <int DIR>
__device__ __forceinline__ C2 crot(C2 a) {
  return DIR > 0 ? C2{neg2(a.im), a.re} : C2{a.im, neg2(a.re)};
}
// a * (c + i s) with c, s broadcast
__device__ __forceinline__ C2 cmulc(C2 a, u64 c, u64 s) {
  return C2{fma2(a.im, neg2(s), mul2(a.re, c)), fma2(a.re, s, mul2(a.im, c))};
}
// a * w^(DIR < 0 ? 1 : -1) for the table twiddle w = (c, s) = exp(-2 pi i e / Ns), broadcast
// to both sequences
template <int DIR>
__device__ __forceinline__ C2 ctw(C2 a, float2 w) {
  const u64 c = pk(make_float2(w.x, w.x)), s = pk(make_float2(w.y, w.y));
  return DIR < 0 ? C2{fma2(a.im, neg2(s), mul2(a.re, c)), fma2(a.re, s, mul2(a.im, c))}
                 : C2{fma2(a.im, s, mul2(a.re, c)), fma2(a.re, neg2(s), mul2(a.im, c))};
}

// In-register DFT of R points (R = 2, 4, 8, 16), output in natural order.
template <int R, int DIR>
__device__ __forceinline__ void dft(C2* u) {
  if constexpr (R == 2) {
    const C2 a = u[0], b = u[1];
    u[0] = cadd(a, b);
    u[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const C2 t0 = cadd(u[0], u[2]), t1 = csub(u[0], u[2]);
    const C2 t2 = cadd(u[1], u[3]), t3 = crot<DIR>(csub(u[1], u[3]));
    u[0] = cadd(t0, t2);
    u[2] = csub(t0, t2);
    u[1] = cadd(t1, t3);
    u[3] = csub(t1, t3);
  } else if constexpr (R == 8) {
    C2 e[4] = {u[0], u[2], u[4], u[6]}, o[4] = {u[1], u[3], u[5], u[7]};
    dft<4, DIR>(e);
    dft<4, DIR>(o);
    // w8^k = exp(dir 2 pi i k / 8): k = 1: r (1 + dir i), k = 3: r (-1 + dir i)
    const u64 r = bc(0.70710678118654752440f), nr = bc(-0.70710678118654752440f), ds = bc(DIR > 0 ? 0.70710678118654752440f : -0.70710678118654752440f);
    const C2 o1 = cmulc(o[1], r, ds), o2 = crot<DIR>(o[2]), o3 = cmulc(o[3], nr, ds);
    u[0] = cadd(e[0], o[0]);
    u[4] = csub(e[0], o[0]);
    u[1] = cadd(e[1], o1);
    u[5] = csub(e[1], o1);
    u[2] = cadd(e[2], o2);
    u[6] = csub(e[2], o2);
    u[3] = cadd(e[3], o3);
    u[7] = csub(e[3], o3);
  } else {
    static_assert(R == 16, "radix");
    // 16 = 4 x 4: DFT4 over n1 of x[4 n1 + n2], twiddle W16^(n2 k1), DFT4 over n2
    C2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      C2 t[4] = {u[n2], u[n2 + 4], u[n2 + 8], u[n2 + 12]};
      dft<4, DIR>(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    const float sd = DIR > 0 ? 1.f : -1.f;
    const u64 c1 = bc(0.92387953251128675613f), s1 = bc(sd * 0.38268343236508977173f);
    const u64 r2 = bc(0.70710678118654752440f), sr2 = bc(sd * 0.70710678118654752440f), nr2 = bc(-0.70710678118654752440f);
    const u64 c3 = bc(0.38268343236508977173f), s3 = bc(sd * 0.92387953251128675613f);
    const u64 c9 = bc(-0.92387953251128675613f), s9 = bc(-sd * 0.38268343236508977173f);
    a[1][1] = cmulc(a[1][1], c1, s1);
    a[1][2] = cmulc(a[1][2], r2, sr2);
    a[1][3] = cmulc(a[1][3], c3, s3);
    a[2][1] = cmulc(a[2][1], r2, sr2);
    a[2][2] = crot<DIR>(a[2][2]);
    a[2][3] = cmulc(a[2][3], nr2, sr2);
    a[3][1] = cmulc(a[3][1], c3, s3);
    a[3][2] = cmulc(a[3][2], nr2, sr2);
    a[3][3] = cmulc(a[3][3], c9, s9);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      C2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      dft<4, DIR>(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) u[k1 + 4 * k2] = t[k2];
    }
  }
}

// Shared-memory index of point n of pair-pair hp (HP pair-pairs per CTA, 16 bytes each).
// Synthesis (SW false): HP point-pairs per n and HP more after every 8 n, which keeps every
// pass's quarter-warp accesses (8 lanes: the HP pair-pairs of 8 / HP consecutive groups) on
// distinct banks. Analysis (SW true, HP = 4): no padding; a 128-byte row holds points 2r and
// 2r + 1 in the halves given by the parity of n ^ (n >> 3) ^ (n >> 7), so a quarter warp
// covers all 8 slots of a row pair when its two points differ by 1 from an even point (the
// first pass and the span-8 pass), by 8 from a multiple of 16 (the span-1 pass) or by 128
// without a carry into bit 7 (bins at digit-reversed positions, which the padded layout
// puts on the same banks). The smaller tile leaves the L1 more room beside it (FFT
// analysis 0.429 -> 0.420 ms at nlon 2048 x 64; the synthesis measured slower with it).
template <int HP, bool SW>
__device__ __forceinline__ int sidx(int n, int hp) {
  if constexpr (SW) {
    static_assert(HP == 4, "row layout of four pair-pairs");
    return (((n >> 1) << 1) | ((n ^ (n >> 3) ^ (n >> 7)) & 1)) * HP + hp;
  } else {
    return (n + (n >> 3)) * HP + hp;
  }
}
// Elements of the larger (synthesis) layout; the analysis uses the first N HP of them.
template <int HP>
__host__ __device__ inline int smem_elems(int N) { return (N + (N >> 3)) * HP; }
template <int HP>
__host__ __device__ inline int smem_elems_ana(int N) { return N * HP; }

__device__ __forceinline__ float4 ld4(const float4* X, int i) { return X[i]; }
__device__ __forceinline__ C2 ldc(const float4* X, int i) {
  const float4 v = X[i];
  return C2{pk(make_float2(v.x, v.y)), pk(make_float2(v.z, v.w))};
}
__device__ __forceinline__ void stc(float4* X, int i, C2 c) {
  const float2 r = up(c.re), m = up(c.im);
  X[i] = make_float4(r.x, r.y, m.x, m.y);
}

// One in-shared-memory DIF pass of radix R over span S (twiddled unless S == 1).
template <int HP, int R, int DIR>
__device__ __forceinline__ void pass_smem(float4* X, int N, int S, const float2* __restrict__ tw) {
  const int ngrp = HP * (N / R);
  for (int gi = threadIdx.x; gi < ngrp; gi += blockDim.x) {
    const int hp = gi % HP, grp = gi / HP;
    const int j = grp & (S - 1), base = (grp - j) * R + j;
    C2 u[R];
#pragma unroll
    for (int q = 0; q < R; ++q) u[q] = ldc(X, sidx<HP, (DIR < 0)>(base + q * S, hp));
    dft<R, DIR>(u);
    if (j != 0) {
#pragma unroll
      for (int q = 1; q < R; ++q) u[q] = ctw<DIR>(u[q], tw[(q - 1) * S + j]);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) stc(X, sidx<HP, (DIR < 0)>(base + q * S, hp), u[q]);
  }
}

template <int HP, int DIR>
__device__ __forceinline__ void run_pass(float4* X, int N, int R, int S, const float2* tw) {
  switch (R) {
    case 16: pass_smem<HP, 16, DIR>(X, N, S, tw); break;
    case 8: pass_smem<HP, 8, DIR>(X, N, S, tw); break;
    case 4: pass_smem<HP, 4, DIR>(X, N, S, tw); break;
    default: pass_smem<HP, 2, DIR>(X, N, S, tw); break;
  }
}

struct Job {
  PlanDev P;
  FFTDesc fd;
  const int* perm;          // rev (analysis) or rinv (synthesis)
  const float2* tw;         // per-pass twiddles (c, s), layout of FFTDesc::twoff
  const float2* Win;        // synthesis: Fourier buffer
  float* Wout;              // analysis: B tile images of the mixed analysis GEMM
  float* grid;
  int nf, mlim;
  double scale;             // synthesis: grid factor; analysis: weight factor
};

// ------------------------------------------------------------------------------ analysis
// Fourier-buffer loads of the synthesis (read once) that leave no line in L1, which keeps the
// twiddle and permutation tables there (FFT synthesis 0.409 -> 0.398 ms at nlon 2048 x 64
// fields). The analysis's 8-byte grid loads are faster with L1 allocation (0.430 vs 0.588 ms).
__device__ __forceinline__ float4 ld_once4(const float2* p) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
template <int HP, int R0>
__device__ __forceinline__ void first_from_grid(float4* X, const Job& J, const float* __restrict__ in, int p0) {
  const int N = J.fd.n, S = N / R0, nlat = J.P.nlat, npair = J.P.npair;
  const float2* tw = J.tw + J.fd.twoff[0];
  const int ngrp = HP * S;
  for (int gi = threadIdx.x; gi < ngrp; gi += blockDim.x) {
    const int hp = gi % HP, j = gi / HP;
    const int pa = p0 + 2 * hp;                    // pairs pa, pa + 1
    const bool va = pa < npair, vb = pa + 1 < npair;
    C2 u[R0];
#pragma unroll
    for (int q = 0; q < R0; ++q) {
      const float* row = in + (size_t)(j + q * S) * nlat;
      float2 nn = make_float2(0.f, 0.f), ss = make_float2(0.f, 0.f);
      if (vb) {
        nn = *reinterpret_cast<const float2*>(row + pa);
        const float2 s2 = *reinterpret_cast<const float2*>(row + nlat - 2 - pa);   // (south b, south a)
        ss = make_float2(s2.y, s2.x);
      } else if (va) {
        nn.x = row[pa];
        ss.x = row[nlat - 1 - pa];
      }
      u[q] = C2{pk(nn), pk(ss)};
    }
    dft<R0, -1>(u);
    if (j != 0) {
#pragma unroll
      for (int q = 1; q < R0; ++q) u[q] = ctw<-1>(u[q], tw[(q - 1) * S + j]);
    }
#pragma unroll
    for (int q = 0; q < R0; ++q) stc(X, sidx<HP, true>(j + q * S, hp), u[q]);
  }
}

// B tile images (btile_base / btile_off of fft.cu): region (im, parity, K-step of 8 pairs)
__device__ __forceinline__ size_t f2_btile_base(int im, int par, int p, int k, int npair, int nf) {
  const size_t nks8 = (size_t)(npair + 7) / 8;
  return (((size_t)im * 2 + par) * nks8 + (p >> 3)) * (size_t)btile_nfp(nf) * 16 + (size_t)(k >> 6) * 1024;
}

// Pairs p0 .. p0 + 2 HP - 1 of field k.
template <int HP>
__device__ __forceinline__ void ana_body(const Job& J, int k, int p0, float4* X, float* wfac) {
  const PlanDev& P = J.P;
  const int N = J.fd.n, npair = P.npair;
  for (int h = threadIdx.x; h < 2 * HP; h += blockDim.x) {
    const int p = p0 + h;
    wfac[h] = (p < npair) ? (float)(J.scale * P.w[p]) : 0.f;
  }
  const float* in = J.grid + (size_t)k * P.nlat * N;
  switch (J.fd.rad[0]) {
    case 16: first_from_grid<HP, 16>(X, J, in, p0); break;
    case 8: first_from_grid<HP, 8>(X, J, in, p0); break;
    case 4: first_from_grid<HP, 4>(X, J, in, p0); break;
    default: first_from_grid<HP, 2>(X, J, in, p0); break;
  }
  __syncthreads();
  int S = N / J.fd.rad[0];
  for (int s = 1; s < J.fd.nrad; ++s) {
    const int R = J.fd.rad[s];
    S /= R;
    run_pass<HP, -1>(X, N, R, S, J.tw + J.fd.twoff[s]);
    __syncthreads();
  }
  // epilogue: E = w (X_N + X_S), O = w (X_N - X_S) with X_N = (Z_m + conj Z_{N-m}) / 2 and
  // X_S = -i (Z_m - conj Z_{N-m}) / 2, for both pairs of a pair-pair, into the B images
  // Lanes 2j and 2j + 1 hold pair-pairs hp and hp + 1 (4 consecutive pairs) of one order:
  // after one exchange the even lane stores the 4 pairs of the real row and the odd lane
  // those of the imaginary row, two adjacent 16-byte core-matrix rows, so every store of a
  // warp fills whole 32-byte sectors. Pairs past npair carry zero weights and store zeros
  // into the padding of their K-step.
  static_assert(HP % 2 == 0, "pair-pairs go in lane pairs");
  const int nmu = J.mlim / P.mres + 1, nitem = nmu * HP;
  const int fl = k & 63, lane = threadIdx.x & 31;
  const bool odd = lane & 1;
  for (int base = threadIdx.x - lane; base < nitem; base += blockDim.x) {
    const int idx = base + lane;
    const bool valid = idx < nitem;
    const int hp = idx % HP, im = valid ? idx / HP : 0, m = im * P.mres;
    const int pa = p0 + 2 * hp;
    const C2 zm = ldc(X, sidx<HP, true>(J.perm[m], hp));
    const C2 zc = ldc(X, sidx<HP, true>(J.perm[m == 0 ? 0 : N - m], hp));
    const u64 sre = add2(zm.re, zc.re), sim = sub2(zm.im, zc.im);   // Z_m + conj Z_c
    const u64 dre = sub2(zm.re, zc.re), dim = add2(zm.im, zc.im);   // Z_m - conj Z_c
    const u64 hw = pk(make_float2(0.5f * wfac[2 * hp], 0.5f * wfac[2 * hp + 1]));
    const u64 Ere = mul2(hw, add2(sre, dim)), Eim = mul2(hw, sub2(sim, dre));
    const u64 Ore = mul2(hw, sub2(sre, dim)), Oim = mul2(hw, add2(sim, dre));
    // the even lane keeps its real parts and takes its partner's; the odd lane the reverse
    const u64 eo = __shfl_xor_sync(0xffffffffu, odd ? Ere : Eim, 1);
    const u64 oo = __shfl_xor_sync(0xffffffffu, odd ? Ore : Oim, 1);
    if (!valid) continue;
    const float2 e0 = up(odd ? eo : Ere), e1 = up(odd ? Eim : eo);
    const float2 o0 = up(odd ? oo : Ore), o1 = up(odd ? Oim : oo);
    const int pe = pa - (odd ? 2 : 0);     // first of the 4 pairs, a multiple of 4
    const int off = btile_off(2 * fl + (odd ? 1 : 0), pe & 7);
    *reinterpret_cast<float4*>(J.Wout + f2_btile_base(im, 0, pe, k, npair, J.nf) + off) = make_float4(e0.x, e0.y, e1.x, e1.y);
    *reinterpret_cast<float4*>(J.Wout + f2_btile_base(im, 1, pe, k, npair, J.nf) + off) = make_float4(o0.x, o0.y, o1.x, o1.y);
  }
  if (p0 <= npair - 1 && npair - 1 < p0 + 2 * HP) {
    // the CTA holding the last pair also zeroes the padding pairs npair .. npair8-1
    const int pad = ((npair + 7) & ~7) - npair;
    for (int idx = threadIdx.x; idx < nmu * pad; idx += blockDim.x) {
      const int im = idx / pad, p = npair + idx - im * pad;
      const int kk = p & 7;
      for (int par = 0; par < 2; ++par) {
        float* b = J.Wout + f2_btile_base(im, par, p, k, npair, J.nf);
        b[btile_off(2 * fl, kk)] = 0.f;
        b[btile_off(2 * fl + 1, kk)] = 0.f;
      }
    }
  }
}

template <int HP>
__global__ void __launch_bounds__(128 * HP, 4 / HP) ana_kernel(const __grid_constant__ Job J) {
  extern __shared__ __align__(16) float4 X[];
  __shared__ float wfac[2 * HP];
  ana_body<HP>(J, blockIdx.x, blockIdx.y * (2 * HP), X, wfac);
}

// ----------------------------------------------------------------------------- synthesis
template <int HP, int RL>
__device__ __forceinline__ void last_to_grid(const float4* X, const Job& J, float* __restrict__ out, int p0,
                                             const float* gfac) {
  const int N = J.fd.n, nlat = J.P.nlat, npair = J.P.npair;
  const int ngrp = HP * (N / RL);
  for (int gi = threadIdx.x; gi < ngrp; gi += blockDim.x) {
    const int hp = gi % HP, blk = gi / HP;
    C2 u[RL];
#pragma unroll
    for (int q = 0; q < RL; ++q) u[q] = ldc(X, sidx<HP, false>(blk * RL + q, hp));
    dft<RL, +1>(u);
    const int pa = p0 + 2 * hp;
    if (pa >= npair) continue;
    const bool vb = pa + 1 < npair;
    const u64 g = pk(make_float2(gfac[2 * hp], gfac[2 * hp + 1]));
#pragma unroll
    for (int q = 0; q < RL; ++q) {
      float* row = out + (size_t)J.perm[blk * RL + q] * nlat;
      const float2 nn = up(mul2(u[q].re, g)), ss = up(mul2(u[q].im, g));
      if (vb) {
        *reinterpret_cast<float2*>(row + pa) = nn;
        *reinterpret_cast<float2*>(row + nlat - 2 - pa) = make_float2(ss.y, ss.x);
      } else {
        row[pa] = nn.x;
        row[nlat - 1 - pa] = ss.x;
      }
    }
  }
}

// Pairs p0 .. p0 + 2 HP - 1 of field k.
template <int HP>
__device__ __forceinline__ void syn_body(const Job& J, int k, int p0, float4* X, float* gfac) {
  const PlanDev& P = J.P;
  const int N = J.fd.n, npair = P.npair;
  const int mlim = J.mlim;
  // bins the order loop does not write are zero: mlim < q < N - mlim (mres == 1), all
  // others when orders are sparse
  {
    const int zlo = (P.mres == 1) ? mlim + 1 : 0, zhi = (P.mres == 1) ? N - mlim : N;
    const int zn = zhi - zlo;
    for (int idx = threadIdx.x; idx < zn * HP; idx += blockDim.x)
      X[sidx<HP, false>(zlo + idx / HP, idx % HP)] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int h = threadIdx.x; h < 2 * HP; h += blockDim.x) gfac[h] = (float)J.scale;
  __syncthreads();
  // Z_m = X_N + i X_S, Z_{N-m} = conj X_N + i conj X_S with X_N = E + O, X_S = E - O. A
  // thread's items are (order, pair-pair) idx, idx + blockDim, ...; kU of them have their
  // Fourier-buffer loads in flight together.
  constexpr int kU = 8;
  const int nmu = mlim / P.mres + 1, nitem = nmu * HP;
  for (int i0 = threadIdx.x; i0 < nitem; i0 += kU * blockDim.x) {
    float4 ev[kU], ov[kU];   // (re a, im a, re b, im b)
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int idx = i0 + u * blockDim.x;
      ev[u] = ov[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (idx < nitem) {
        const int hp = idx % HP, im = idx / HP;
        const int pa = p0 + 2 * hp;
        const size_t base = ((size_t)k * P.nm + im) * 2 * npair + pa;
        if (pa + 1 < npair) {
          ev[u] = ld_once4(J.Win + base);
          ov[u] = ld_once4(J.Win + base + npair);
        } else if (pa < npair) {
          const float2 e = J.Win[base], o = J.Win[base + npair];
          ev[u].x = e.x; ev[u].y = e.y;
          ov[u].x = o.x; ov[u].y = o.y;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int idx = i0 + u * blockDim.x;
      if (idx >= nitem) break;
      const int hp = idx % HP, m = (idx / HP) * P.mres;
      const u64 ere = pk(make_float2(ev[u].x, ev[u].z)), eim = pk(make_float2(ev[u].y, ev[u].w));
      const u64 ore = pk(make_float2(ov[u].x, ov[u].z)), oim = pk(make_float2(ov[u].y, ov[u].w));
      const u64 nre = add2(ere, ore), nim = add2(eim, oim);   // X_N
      const u64 sre = sub2(ere, ore), sim = sub2(eim, oim);   // X_S
      if (m == 0) {
        const float2 a = up(nre), b = up(sre);
        X[sidx<HP, false>(0, hp)] = make_float4(a.x, a.y, b.x, b.y);
      } else {
        stc(X, sidx<HP, false>(m, hp), C2{sub2(nre, sim), add2(nim, sre)});
        stc(X, sidx<HP, false>(N - m, hp), C2{add2(nre, sim), sub2(sre, nim)});
      }
    }
  }
  __syncthreads();
  int S = N;
  for (int s = 0; s + 1 < J.fd.nrad; ++s) {
    const int R = J.fd.rad[s];
    S /= R;
    run_pass<HP, +1>(X, N, R, S, J.tw + J.fd.twoff[s]);
    __syncthreads();
  }
  float* out = J.grid + (size_t)k * P.nlat * N;
  switch (J.fd.rad[J.fd.nrad - 1]) {
    case 16: last_to_grid<HP, 16>(X, J, out, p0, gfac); break;
    case 8: last_to_grid<HP, 8>(X, J, out, p0, gfac); break;
    case 4: last_to_grid<HP, 4>(X, J, out, p0, gfac); break;
    default: last_to_grid<HP, 2>(X, J, out, p0, gfac); break;
  }
}

template <int HP>
__global__ void __launch_bounds__(128 * HP, 4 / HP) syn_kernel(const __grid_constant__ Job J) {
  extern __shared__ __align__(16) float4 X[];
  __shared__ float gfac[2 * HP];
  syn_body<HP>(J, blockIdx.y, blockIdx.x * (2 * HP), X, gfac);
}

// Persistent FFTs of many transforms (uneven batches): item = (transform, first pair of a
// block of 2 HP pairs, field), list sorted by decreasing row length; each CTA claims the
// next item from the device counter *queue (zero at launch) when it finishes one. Shared
// memory is sized for the longest row of the group.
template <int HP, bool SYN>
__global__ void __launch_bounds__(128 * HP, 4 / HP) group_kernel(const Job* __restrict__ jobs,
                                                                const int4* __restrict__ items, int nitems,
                                                                int* __restrict__ queue) {
  extern __shared__ __align__(16) float4 X[];
  __shared__ float fac[2 * HP];
  __shared__ Job sj;
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
      syn_body<HP>(sj, it.z, it.y, X, fac);
    else
      ana_body<HP>(sj, it.z, it.y, X, fac);
    __syncthreads();   // sj, s_it, fac and X are rewritten for the next item
  }
}

}  // namespace f2

// Whether the packed-pair kernels take this plan's FP32 FFTs.
bool fft2_applicable(const shtb_plan* p) {
  const FFTDesc& fd = p->fft;
  if (fd.direct || fd.nrad < 2 || (p->nlat & 3)) return false;   // npair even: 16-byte pair loads
  if (fd.n < 64 || fd.n > 2048 || (fd.n & (fd.n - 1))) return false;
  for (int s = 0; s < fd.nrad; ++s)
    if (!(fd.rad[s] == 2 || fd.rad[s] == 4 || fd.rad[s] == 8 || fd.rad[s] == 16)) return false;
  return p->d_twp32 != nullptr;
}

static f2::Job fft2_job(const shtb_plan* p, const int* perm, double scale, int nf, int mlim) {
  f2::Job J;
  J.P = p->dev;
  J.fd = p->fft;
  J.perm = perm;
  J.tw = p->d_twp32;
  J.Win = nullptr;
  J.Wout = nullptr;
  J.grid = nullptr;
  J.nf = nf;
  J.mlim = mlim;
  J.scale = scale;
  return J;
}

// Pair-pairs per CTA: 4 (8 latitude pairs, 512 threads, one CTA per SM). Two CTAs of 2
// pair-pairs per SM measured slower (0.56 vs 0.51 ms analysis, 0.51 vs 0.43 ms synthesis
// at nlon 2048, 64 fields).
constexpr int kFft2HP = 4;

int launch_fft2_ana(const shtb_plan* p, const float* grid, void* W, int nf, int mlim, double wscale, cudaStream_t st) {
  constexpr int HP = kFft2HP;
  const size_t smem = (size_t)f2::smem_elems_ana<HP>(p->fft.n) * 16;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(f2::ana_kernel<HP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "fft2 smem attr");
  f2::Job J = fft2_job(p, p->d_rev, wscale, nf, mlim);
  J.grid = const_cast<float*>(grid);
  J.Wout = (float*)W;
  // blockIdx.x = field, blockIdx.y = block of 2 HP pairs: the fields' CTAs that fill one B
  // tile region run together
  dim3 grd(nf, (p->npair + 2 * HP - 1) / (2 * HP));
  prof_begin(st);
  f2::ana_kernel<HP><<<grd, 128 * HP, smem, st>>>(J);
  SHTB_LAUNCHED("fft analysis kernel");
  return SHTB_OK;
}

// ---------------------------------------------------------------- grouped transforms
size_t fft2_job_bytes() { return sizeof(f2::Job); }

int fft2_group_pairs() { return 2 * kFft2HP; }

size_t fft2_group_smem(const shtb_plan* p) { return (size_t)f2::smem_elems<kFft2HP>(p->fft.n) * 16; }

void fft2_fill_job(const shtb_plan* p, int syn, const void* W, void* grid, int nf, void* host_job) {
  const int mlim = std::min(p->mmax, p->lmax);
  f2::Job J = syn ? fft2_job(p, p->d_rinv, p->phi_inv_scale / p->nlon, nf, mlim)
                  : fft2_job(p, p->d_rev, p->ana_scale, nf, mlim);
  J.grid = (float*)grid;
  if (syn)
    J.Win = (const float2*)W;
  else
    J.Wout = (float*)const_cast<void*>(W);
  std::memcpy(host_job, &J, sizeof(J));
}

int launch_fft2_group(int syn, const void* jobs, const int4* items, int nitems, int grid, size_t smem, int* queue,
                      cudaStream_t st) {
  if (nitems <= 0) return SHTB_OK;
  constexpr int HP = kFft2HP;
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "group FFT tile does not fit in shared memory");
  auto kern = syn ? f2::group_kernel<HP, true> : f2::group_kernel<HP, false>;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "group fft2 smem attr");
  kern<<<grid, 128 * HP, smem, st>>>((const f2::Job*)jobs, items, nitems, queue);
  count_launch();
  SHTB_TRY_CUDA(cudaGetLastError(), "group fft2 launch");
  return SHTB_OK;
}

int launch_fft2_syn(const shtb_plan* p, const void* W, float* grid, int nf, int mlim, double gscale, cudaStream_t st) {
  constexpr int HP = kFft2HP;
  const size_t smem = (size_t)f2::smem_elems<HP>(p->fft.n) * 16;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(f2::syn_kernel<HP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "fft2 smem attr");
  f2::Job J = fft2_job(p, p->d_rinv, gscale, nf, mlim);
  J.Win = (const float2*)W;
  J.grid = grid;
  dim3 grd((p->npair + 2 * HP - 1) / (2 * HP), nf);
  prof_begin(st);
  f2::syn_kernel<HP><<<grd, 128 * HP, smem, st>>>(J);
  SHTB_LAUNCHED("fft synthesis kernel");
  return SHTB_OK;
}

}  // namespace shtb
