// legendre64.cu — FP64 associated-Legendre contraction kernels.
//
// Both directions work per order m on latitude PAIRS (i, nlat-1-i) folded by
// equatorial symmetry: P_l^m(-x) = (-1)^(l-m) P_l^m(x), so every contraction is
// split into degrees of even (E) and odd (O) parity l-m.
//
// P_l^m is never stored: it is regenerated by the c-scaled three-term recurrence
//   r_l = alpha_l x r_{l-1} - r_{l-2},   P_l^m = c_l r_l
// (one DMUL + one DFMA per value), started from per-(m, latitude) records that
// already carry the reference's extended-range sectoral seed. The c_l factors
// are folded into the coefficients on the way in (synthesis) or out (analysis).
//
// Synthesis (leg_syn64_kernel): each thread owns TP latitude pairs and walks l
// with the recurrence in registers; a CTA stages FB fields of coefficients per
// 32-degree chunk in shared memory (read back as broadcasts) and accumulates
// E and O sums for every field.
//
// Analysis (leg_ana64_kernel): a CTA owns a 64-degree tile of one m and a block
// of columns (field re/im parts) and reduces over all latitude pairs in chunks
// of 32. Warp 0 regenerates the P panel of the next chunk from the tile's
// recurrence checkpoint while the CTA multiplies the current one: a
// register-tiled FP64 GEMM (4 E rows + 4 O rows by TC columns per thread) fed
// from double-buffered shared memory (cp.async for the Fourier panel).
#include <climits>

#include "kernels.cuh"

namespace shtb {

__device__ __forceinline__ double factor_at(const PlanDev& P, const Factors& F, long long poff, int l, int m) {
  double s = (m == 0) ? F.mf0 : F.mf1;
  if (F.fac) s *= F.fac[poff + (l - m)];
  if (F.sc_mode) {
    const double q = F.sc[l + (long long)(P.lmax + 1) * m];
    s = (F.sc_mode == 1) ? s * q : s / q;
  }
  return s;
}

// ---------------------------------------------------------------------------
// synthesis
// ---------------------------------------------------------------------------
template <int FB, int TP, int NT>
__global__ void __launch_bounds__(NT) leg_syn64_kernel(PlanDev P, CoefSrc src, Factors F, double2* __restrict__ W,
                                                       int nf, int row_end) {
  constexpr int LC = 32;
  __shared__ double2 As[LC][FB];
  __shared__ double alph[LC];
  __shared__ int smin;
  const int im = blockIdx.y, m = im * P.mres;
  const int kb = blockIdx.z * FB;
  const int pb = blockIdx.x * (TP * NT);
  const int npair = P.npair;
  const long long poff = P.off[im];
  double xt[TP], ra[TP], rb[TP], r0[TP], r1[TP];
  int l0[TP];
  int lmin = INT_MAX;
#pragma unroll
  for (int t = 0; t < TP; ++t) {
    const int p = pb + t * NT + threadIdx.x;
    if (p < npair) {
      xt[t] = P.x[p];
      l0[t] = P.l0[(size_t)im * npair + p];
      const double2 v = P.r01[(size_t)im * npair + p];
      r0[t] = v.x;
      r1[t] = v.y;
    } else {
      xt[t] = 0.0;
      l0[t] = INT_MAX / 2;
      r0[t] = r1[t] = 0.0;
    }
    ra[t] = rb[t] = 0.0;
    lmin = min(lmin, l0[t]);
  }
  for (int o = 16; o > 0; o >>= 1) lmin = min(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
  if (threadIdx.x == 0) smin = INT_MAX;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicMin(&smin, lmin);
  __syncthreads();
  const int lend = min(row_end, P.lrec);
  int lbeg = max(smin, m);
  lbeg -= (lbeg - m) & 1;
  double2 accE[TP][FB], accO[TP][FB];
#pragma unroll
  for (int t = 0; t < TP; ++t)
#pragma unroll
    for (int f = 0; f < FB; ++f) {
      accE[t][f] = make_double2(0.0, 0.0);
      accO[t][f] = make_double2(0.0, 0.0);
    }
  const long long cbase = src.packed == 1 ? (poff - m)
                          : src.packed == 2 ? lm_base(P.lmax, P.mres, m) : (long long)m * src.ld_m;
  for (int lc = lbeg; lc <= lend; lc += LC) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < LC * FB; idx += NT) {
      const int j = idx % LC, f = idx / LC, l = lc + j, k = kb + f;
      double2 v = make_double2(0.0, 0.0);
      if (l <= lend && k < nf) {
        v = src.ptr[(long long)k * src.ld_k + cbase + l];
        const double s = factor_at(P, F, poff, l, m);
        v.x *= s;
        v.y *= s;
      }
      As[j][f] = v;
    }
    for (int idx = threadIdx.x; idx < LC; idx += NT) {
      const int l = lc + idx;
      alph[idx] = (l <= lend) ? P.alpha[poff + (l - m)] : 0.0;
    }
    __syncthreads();
    const int nr = min(LC, lend - lc + 1);
#define SYN_STEP(JJ, ACC)                                                        \
  {                                                                              \
    const int l = lc + (JJ);                                                     \
    const double a = alph[(JJ)];                                                 \
    _Pragma("unroll") for (int t = 0; t < TP; ++t) {                             \
      double r = fma(a * xt[t], ra[t], -rb[t]);                                  \
      r = (l == l0[t]) ? r0[t] : r;                                              \
      r = (l == l0[t] + 1) ? r1[t] : r;                                          \
      rb[t] = ra[t];                                                             \
      ra[t] = r;                                                                 \
    }                                                                            \
    _Pragma("unroll") for (int f = 0; f < FB; ++f) {                             \
      const double2 c = As[(JJ)][f];                                             \
      _Pragma("unroll") for (int t = 0; t < TP; ++t) {                           \
        ACC[t][f].x = fma(ra[t], c.x, ACC[t][f].x);                              \
        ACC[t][f].y = fma(ra[t], c.y, ACC[t][f].y);                              \
      }                                                                          \
    }                                                                            \
  }
#pragma unroll 2
    for (int j = 0; j < nr; j += 2) {
      SYN_STEP(j, accE);
      SYN_STEP(j + 1, accO);
    }
#undef SYN_STEP
  }
#pragma unroll
  for (int t = 0; t < TP; ++t) {
    const int p = pb + t * NT + threadIdx.x;
    if (p >= npair) continue;
#pragma unroll
    for (int f = 0; f < FB; ++f) {
      const int k = kb + f;
      if (k >= nf) continue;
      const size_t base = ((size_t)k * P.nm + im) * 2 * npair + p;
      W[base] = accE[t][f];
      W[base + npair] = accO[t][f];
    }
  }
}

int launch_leg_syn64(const shtb_plan* p, const CoefSrc& src, const Factors& F, void* W, int nf, int row_end,
                     int mlim, cudaStream_t st) {
  constexpr int NT = 128, TP = 2;
  const int nmu = mlim / p->mres + 1;
  auto go = [&](auto kern, int FB) -> int {
    dim3 grid((p->npair + TP * NT - 1) / (TP * NT), nmu, (nf + FB - 1) / FB);
    prof_begin(st);
    kern<<<grid, NT, 0, st>>>(p->dev, src, F, (double2*)W, nf, row_end);
    SHTB_LAUNCHED("legendre synthesis kernel");
    return SHTB_OK;
  };
  if (nf >= 8) return go(leg_syn64_kernel<8, TP, NT>, 8);
  if (nf >= 4) return go(leg_syn64_kernel<4, TP, NT>, 4);
  if (nf >= 2) return go(leg_syn64_kernel<2, TP, NT>, 2);
  return go(leg_syn64_kernel<1, TP, NT>, 1);
}

// ---------------------------------------------------------------------------
// analysis
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

constexpr int kKC = 32;       // latitude pairs per K chunk
constexpr int kRS = 82;       // Rs row stride (doubles): 64 rows, 2 pad doubles after every 8 rows, +2

template <int CT>
__host__ __device__ constexpr int ana_bs() { return CT + 2; }

template <int CT, int TC>
constexpr size_t ana64_smem() {
  constexpr int RG = 8, CG = CT / TC, KS = 256 / (RG * CG);
  constexpr size_t main = (size_t)2 * kKC * kRS * 8 + (size_t)2 * 2 * kKC * ana_bs<CT>() * 8 + 64 * 8;
  constexpr size_t red = (KS > 1) ? (size_t)KS * 64 * CT * 8 : 0;
  return main > red ? main : red;
}

template <int CT, int TC>
__global__ void __launch_bounds__(256, 1) leg_ana64_kernel(PlanDev P, const double2* __restrict__ W, int nf,
                                                           int row_end, int mlim, CoefSink dst, Factors F,
                                                           int zero_fill) {
  constexpr int NT = 256, RG = 8, TRP = 4, CG = CT / TC, KS = NT / (RG * CG), KPT = kKC / KS;
  constexpr int BS = ana_bs<CT>(), NFB = CT / 2;
  static_assert(RG * TRP == 32, "64-row tiles");
  static_assert(KS * RG * CG == NT, "thread layout");
  static_assert(TC % 2 == 0, "complex column pairs");
  extern __shared__ __align__(16) double sm[];
  double* Rs = sm;                               // [2][kKC][kRS]
  double* Bs = sm + 2 * kKC * kRS;               // [2][2][kKC][BS]
  double* alph = Bs + 2 * 2 * kKC * BS;          // [64]
  const int2 tile = P.tiles[blockIdx.x];
  const int im = tile.x, t0 = tile.y, m = im * P.mres;
  const int lend = min(row_end, P.lrec);
  if (m > mlim || t0 > lend) return;
  const int kb = blockIdx.y * NFB;
  const int npair = P.npair;
  const long long poff = P.off[im];
  const int tid = threadIdx.x;
  const int rg = tid % RG, cg = (tid / RG) % CG, ks = tid / (RG * CG);
  const int lane = tid & 31;
  const bool producer = tid < 32;

  for (int i = tid; i < 64; i += NT) {
    const int l = t0 + i;
    alph[i] = (l <= P.lrec) ? P.alpha[poff + (l - m)] : 0.0;
  }
  __syncthreads();

  auto produce = [&](int c, int buf) {
    const int pair = c * kKC + lane;
    double x = 0.0, ra = 0.0, rb = 0.0, r0 = 0.0, r1 = 0.0;
    int l0 = INT_MAX / 2;
    if (pair < npair) {
      x = P.x[pair];
      const double2 stv = P.ckpt[(size_t)blockIdx.x * npair + pair];
      ra = stv.x;
      rb = stv.y;
      l0 = P.l0[(size_t)im * npair + pair];
      const double2 v = P.r01[(size_t)im * npair + pair];
      r0 = v.x;
      r1 = v.y;
    }
    double* R = Rs + (size_t)(buf * kKC + lane) * kRS;
#pragma unroll 4
    for (int rr = 0; rr < 64; rr += 2) {
      double re, ro;
      {
        const int l = t0 + rr;
        double r = fma(alph[rr] * x, ra, -rb);
        r = (l == l0) ? r0 : r;
        r = (l == l0 + 1) ? r1 : r;
        rb = ra;
        ra = r;
        re = r;
      }
      {
        const int l = t0 + rr + 1;
        double r = fma(alph[rr + 1] * x, ra, -rb);
        r = (l == l0) ? r0 : r;
        r = (l == l0 + 1) ? r1 : r;
        rb = ra;
        ra = r;
        ro = r;
      }
      // rows (rr, rr+1) = (E row rr/2, O row rr/2) side by side; 16 bytes of padding per 8 rows
      *reinterpret_cast<double2*>(R + rr + 2 * (rr >> 3)) = make_double2(re, ro);
    }
  };
  auto loadB = [&](int c, int buf) {
    double* B = Bs + (size_t)buf * 2 * kKC * BS;
    for (int idx = tid; idx < kKC * CT; idx += NT) {
      const int kk = idx % kKC, rest = idx / kKC, fl = rest % NFB, par = rest / NFB;
      const int pair = c * kKC + kk, kf = kb + fl;
      double* d = B + ((size_t)par * kKC + kk) * BS + 2 * fl;
      if (pair < npair && kf < nf) {
        cp_async16(d, W + (((size_t)kf * P.nm + im) * 2 + par) * npair + pair);
      } else {
        d[0] = 0.0;
        d[1] = 0.0;
      }
    }
    cp_async_commit();
  };

  double accE[TRP][TC], accO[TRP][TC];
#pragma unroll
  for (int i = 0; i < TRP; ++i)
#pragma unroll
    for (int c = 0; c < TC; ++c) accE[i][c] = accO[i][c] = 0.0;

  const int nchunks = (npair + kKC - 1) / kKC;
  loadB(0, 0);
  if (producer) produce(0, 0);
  cp_async_wait_all();
  __syncthreads();
  int buf = 0;
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      loadB(c + 1, buf ^ 1);
      if (producer) produce(c + 1, buf ^ 1);
    }
    const double* R = Rs + (size_t)buf * kKC * kRS;
    const double* B = Bs + (size_t)buf * 2 * kKC * BS;
#pragma unroll 4
    for (int kk = 0; kk < KPT; ++kk) {
      const int k = ks * KPT + kk;
      double rE[TRP], rO[TRP], bE[TC], bO[TC];
#pragma unroll
      for (int i = 0; i < TRP; ++i) {
        const double2 eo = *reinterpret_cast<const double2*>(R + k * kRS + 10 * rg + 2 * i);
        rE[i] = eo.x;
        rO[i] = eo.y;
      }
#pragma unroll
      for (int q = 0; q < TC; q += 2) {
        const double2 e = *reinterpret_cast<const double2*>(B + (size_t)k * BS + cg * TC + q);
        const double2 o = *reinterpret_cast<const double2*>(B + ((size_t)kKC + k) * BS + cg * TC + q);
        bE[q] = e.x; bE[q + 1] = e.y;
        bO[q] = o.x; bO[q + 1] = o.y;
      }
#pragma unroll
      for (int i = 0; i < TRP; ++i)
#pragma unroll
        for (int q = 0; q < TC; ++q) {
          accE[i][q] = fma(rE[i], bE[q], accE[i][q]);
          accO[i][q] = fma(rO[i], bO[q], accO[i][q]);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    buf ^= 1;
  }

  if constexpr (KS > 1) {
    // reduce the K-split partial tiles: red[ks][row 64][CT]
    double* red = sm;
#pragma unroll
    for (int i = 0; i < TRP; ++i)
#pragma unroll
      for (int q = 0; q < TC; ++q) {
        const int rp = rg * TRP + i, col = cg * TC + q;
        red[((size_t)ks * 64 + 2 * rp) * CT + col] = accE[i][q];
        red[((size_t)ks * 64 + 2 * rp + 1) * CT + col] = accO[i][q];
      }
    __syncthreads();
    if (ks == 0) {
#pragma unroll
      for (int i = 0; i < TRP; ++i)
#pragma unroll
        for (int q = 0; q < TC; ++q) {
          const int rp = rg * TRP + i, col = cg * TC + q;
          double se = 0.0, so = 0.0;
          for (int s = 0; s < KS; ++s) {
            se += red[((size_t)s * 64 + 2 * rp) * CT + col];
            so += red[((size_t)s * 64 + 2 * rp + 1) * CT + col];
          }
          accE[i][q] = se;
          accO[i][q] = so;
        }
    }
  }

  const long long dbase = dst.packed == 1 ? (poff - m)
                          : dst.packed == 2 ? lm_base(P.lmax, P.mres, m) : (long long)m * dst.ld_m;
  const int lcap = dst.packed == 1 ? lend : min(lend, P.lmax);
  if (ks == 0) {
#pragma unroll
    for (int i = 0; i < TRP; ++i) {
      const int rp = rg * TRP + i;
#pragma unroll
      for (int par = 0; par < 2; ++par) {
        const int l = t0 + 2 * rp + par;
        if (l > lcap) continue;
        const double s = factor_at(P, F, poff, l, m);
#pragma unroll
        for (int q = 0; q < TC; q += 2) {
          const int kf = kb + (cg * TC + q) / 2;
          if (kf >= nf) continue;
          const double re = par ? accO[i][q] : accE[i][q];
          const double imv = par ? accO[i][q + 1] : accE[i][q + 1];
          dst.ptr[(long long)kf * dst.ld_k + dbase + l] = make_double2(re * s, imv * s);
        }
      }
    }
  }
  if (zero_fill && !dst.packed && t0 == m) {
    const int nz_lo = m, nz_hi = P.lmax - lcap;  // rows [0, m) and (lcap, lmax]
    const int nrow = nz_lo + max(nz_hi, 0);
    for (int idx = tid; idx < nrow * NFB; idx += NT) {
      const int r = idx % nrow, fl = idx / nrow, kf = kb + fl;
      if (kf >= nf) continue;
      const int l = (r < nz_lo) ? r : lcap + 1 + (r - nz_lo);
      dst.ptr[(long long)kf * dst.ld_k + (long long)m * dst.ld_m + l] = make_double2(0.0, 0.0);
    }
  }
}

int launch_leg_ana64(const shtb_plan* p, const void* W, int nf, int row_end, int mlim, const CoefSink& dst,
                     const Factors& F, int zero_fill, cudaStream_t st) {
  auto go = [&](auto kern, size_t smem, int nfb) -> int {
    SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "analysis smem attr");
    dim3 grid(p->dev.ntiles, (nf + nfb - 1) / nfb);
    prof_begin(st);
    kern<<<grid, 256, smem, st>>>(p->dev, (const double2*)W, nf, row_end, mlim, dst, F, zero_fill);
    SHTB_LAUNCHED("legendre analysis kernel");
    return SHTB_OK;
  };
  if (nf > 32) return go(leg_ana64_kernel<128, 4>, ana64_smem<128, 4>(), 64);
  if (nf > 16) return go(leg_ana64_kernel<64, 4>, ana64_smem<64, 4>(), 32);
  if (nf > 8) return go(leg_ana64_kernel<32, 4>, ana64_smem<32, 4>(), 16);
  if (nf > 4) return go(leg_ana64_kernel<16, 4>, ana64_smem<16, 4>(), 8);
  if (nf > 2) return go(leg_ana64_kernel<8, 4>, ana64_smem<8, 4>(), 4);
  if (nf > 1) return go(leg_ana64_kernel<4, 4>, ana64_smem<4, 4>(), 2);
  return go(leg_ana64_kernel<2, 2>, ana64_smem<2, 2>(), 1);
}

}  // namespace shtb
