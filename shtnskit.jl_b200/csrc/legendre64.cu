// legendre64.cu — FP64 associated-Legendre contraction kernels on the FP64 tensor cores.
//
// Both directions work per order m on latitude PAIRS (i, nlat-1-i) folded by
// equatorial symmetry: P_l^m(-x) = (-1)^(l-m) P_l^m(x), so every contraction is
// split into degrees of even (E) and odd (O) parity l-m. Per order and parity each
// direction is a dense GEMM whose P operand is regenerated on the fly:
//   synthesis  W[pair, col] = sum_l P_l(x_pair) a[l, col]     (K = degrees)
//   analysis   a[l, col]    = sum_pair P_l(x_pair) W[pair, col] (K = latitude pairs)
// with col = (field, re|im).
//
// P_l^m is never stored in global memory: four producer warps per CTA regenerate the
// panels of the coming K chunks into a ring of shared-memory stages with the c-scaled
// three-term recurrence
//   r_l = alpha_l x r_{l-1} - r_{l-2},   P_l^m = c_l r_l
// (one DMUL + one DFMA per value), started from per-(m, pair) records that carry the
// reference's extended-range sectoral seed (values below 2^-480 are zero until the
// record's first degree l0) and, inside the degree range, from the plan's recurrence
// checkpoints (every ckstep degrees), so the panel of a chunk is many short independent
// chains rather than one long one; they fill the same stage with the chunk's coefficient
// or Fourier panel by cp.async. Eight consumer warps multiply each stage with FP64 MMAs
// (mma.sync m16n8k4 .f64: 512 FMAs per instruction, the DFMA units' full rate at an
// eighth of the issue slots of DFMA code), operands from shared memory, accumulators in
// registers. Stages are handed over on mbarriers (full: panels written and copies landed;
// empty: every consumer warp done), so the producers run up to a ring's depth ahead and
// their latency-bound recurrence, which shares the FP64 pipe with the MMAs, never holds
// the consumers at a CTA-wide barrier. Every wait is bounded (pipe.cuh).
//
// Per-(l, m) multipliers (c_l, normalization, phi scales) are folded into the P panel
// (synthesis) or applied at the store (analysis). Chunks whose P values are all zero
// (every pair of the chunk still below its record's first degree, near the poles at
// high m) are skipped: adding their zeros changes nothing.
#include <climits>

#include "kernels.cuh"
#include "pipe.cuh"

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

// D (16x8) += A (16x4, row-major) B (4x8, column-major), FP64. Fragments per lane
// (g = lane / 4, t = lane % 4): a0 = A[g][t], a1 = A[g + 8][t]; b0 = B[t][g];
// d0, d1 = D[g][2t], D[g][2t + 1]; d2, d3 = D[g + 8][2t], D[g + 8][2t + 1].
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

constexpr int kConsumerWarps = 8;

// Consumer warp layout shared by both directions: per parity an output tile of 64 rows
// by NCOL columns, split over kConsumerWarps / 2 warps as RG row groups x CG column
// groups; a warp holds MT x NT fragments of 16 x 8.
template <int NCOL>
struct WarpTile {
  static constexpr int WPP = kConsumerWarps / 2;   // warps per parity
  static constexpr int RG = NCOL >= 64 ? 2 : 4, CG = WPP / RG;
  static constexpr int MT = 64 / RG / 16, NT = NCOL / CG / 8;
  static constexpr int NF = NCOL / 2;   // fields per CTA
  static_assert(MT >= 1 && NT >= 1 && RG * CG == WPP, "warp tile");
};

constexpr int kProducerWarps = 4;   // one per SM sub-partition, so the recurrence's FP64 work
                                    // spreads over all four FP64 pipes
constexpr int kLegThreads = 32 * (kConsumerWarps + kProducerWarps);

// ---------------------------------------------------------------------------
// synthesis: CTA = (64 pairs, order m, NCOL/2 fields), K chunks of 16 degrees
// ---------------------------------------------------------------------------
constexpr int kSynPairs = 64;
constexpr int kSynDeg = 16;                    // degrees per chunk (8 per parity)
constexpr int kSynPS = kSynPairs + 4;          // P panel row stride (doubles), = 4 mod 16
constexpr int kSynCS = 2 * (kSynDeg / 2) + 8;  // coefficient field stride (doubles), = 8 mod 16
constexpr int kSynStages = 4;

template <int NCOL>
struct SynSmem {
  static constexpr int NF = WarpTile<NCOL>::NF;
  static constexpr int PBUF = 2 * (kSynDeg / 2) * kSynPS;   // [parity][8 degrees][pairs]
  static constexpr int CBUF = 2 * NF * kSynCS;              // [parity][field][8 degrees x re|im]
  static constexpr int STAGE = PBUF + CBUF;                 // doubles
  static constexpr int BAR = kSynStages * STAGE;            // then full[S], empty[S], flags
  // stages, barriers, abort flag and two pair minima, then alpha and the folded factor of
  // every degree m..lend
  static size_t bytes(int ndeg) { return (size_t)BAR * 8 + 2 * kSynStages * 8 + 16 + (size_t)2 * ndeg * 8; }
};

template <int NCOL>
__global__ void __launch_bounds__(kLegThreads, 1)
    leg_syn64_kernel(PlanDev P, CoefSrc src, Factors F, double2* __restrict__ W, int nf, int row_end, int* err) {
  using WT = WarpTile<NCOL>;
  using SM = SynSmem<NCOL>;
  constexpr int NF = WT::NF, S = kSynStages;
  extern __shared__ __align__(16) double sm[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + SM::BAR);
  unsigned long long* empty = full + S;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + S);
  int* sLmin = reinterpret_cast<int*>(empty + S) + 1;
  double* sAl = reinterpret_cast<double*>(empty + S + 2);
  const int im = blockIdx.y, m = im * P.mres;
  const int p0 = blockIdx.x * kSynPairs;
  const int kb = blockIdx.z * NF;
  const int npair = P.npair;
  const long long poff = P.off[im];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool producer = warp >= kConsumerWarps;
  const int lend = min(row_end, P.lrec);
  const int ndeg = max(lend - m + 1, 0);
  double* sFa = sAl + ndeg;

  if (tid == 0) {
    for (int q = 0; q < S; ++q) {
      pipe_bar_init(&full[q], 64);   // one group of two producer warps fills a stage
      pipe_bar_init(&empty[q], kConsumerWarps);
    }
    *abort_flag = 0;
    pipe_bar_init_fence();
  }
  for (int i = tid; i < ndeg; i += kLegThreads) {
    sAl[i] = P.alpha[poff + i];
    sFa[i] = factor_at(P, F, poff, m + i, m);
  }
  // producer state: the producer warps form two groups that fill alternate chunks; in
  // each group, thread q = 32 (w % 2) + lane takes pair p0 + q
  double px = 0.0, pr0 = 0.0, pr1 = 0.0;
  int pl0 = INT_MAX / 2;
  const int pw = warp - kConsumerWarps, pgroup = pw >> 1, pq = 32 * (pw & 1) + lane;
  const int pp = p0 + pq;
  if (producer) {
    if (pp < npair) {
      px = P.x[pp];
      pl0 = P.l0[(size_t)im * npair + pp];
      const double2 v = P.r01[(size_t)im * npair + pp];
      pr0 = v.x;
      pr1 = v.y;
    }
    int mn = pl0;
    for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if (lane == 0 && pw < 2) sLmin[pw] = mn;
  }
  __syncthreads();
  const int lmin = max(min(sLmin[0], sLmin[1]), m);
  // chunks start at degrees m + 16 k (even l - m first)
  const int lbeg = m + ((lmin - m) / kSynDeg) * kSynDeg;
  const int nchunks = (lend >= lbeg) ? (lend - lbeg) / kSynDeg + 1 : 0;
  const long long cbase = src.packed == 1 ? (poff - m)
                          : src.packed == 2 ? lm_base(P.lmax, P.mres, m) : (long long)m * src.ld_m;

  if (producer) {
    for (int c = pgroup; c < nchunks; c += 2) {
      const int st = c % S;
      if (c >= S && !pipe_wait(&empty[st], ((c / S) - 1) & 1, abort_flag, err)) break;
      double* Pn = sm + st * SM::STAGE;
      double* C = Pn + SM::PBUF;
      const int lc = lbeg + c * kSynDeg;
      // coefficients: 8 consecutive threads fill one (parity, field) row of 8 degrees
      for (int idx = pq; idx < NF * kSynDeg; idx += 64) {
        const int s = 2 * (idx & 7) + ((idx >> 3) & 1), fl = idx / kSynDeg;
        const int l = lc + s, kf = kb + fl;
        const bool ok = (l <= lend) && (kf < nf);
        const double2* gp = ok ? src.ptr + (long long)kf * src.ld_k + cbase + l : src.ptr;
        pipe_cp16(C + ((s & 1) * NF + fl) * kSynCS + 2 * (s >> 1), gp, ok ? 16u : 0u);
      }
      pipe_arrive_cp_async(&full[st]);
      // P panel column of pair pp, the per-degree factors folded in (zero past lend): the
      // chain starts at the checkpoint at or below lc
      const int ks = (lc - m) / P.ckstep, lk = m + ks * P.ckstep;
      double ra = 0.0, rb = 0.0;
      if (pp < npair) {
        const double2 v = P.ckpt[(size_t)(P.ckbase[im] + ks) * npair + pp];
        ra = v.x;
        rb = v.y;
      }
      for (int l = lk; l < lc; ++l) {   // only when the checkpoints are sparser than a chunk
        double r = fma(sAl[l - m] * px, ra, -rb);
        r = (l == pl0) ? pr0 : r;
        r = (l == pl0 + 1) ? pr1 : r;
        rb = ra;
        ra = r;
      }
#pragma unroll
      for (int s = 0; s < kSynDeg; ++s) {
        const int l = lc + s;
        const bool in = l <= lend;
        const double a = in ? sAl[l - m] : 0.0, f = in ? sFa[l - m] : 0.0;
        double r = fma(a * px, ra, -rb);
        r = (l == pl0) ? pr0 : r;
        r = (l == pl0 + 1) ? pr1 : r;
        rb = ra;
        ra = r;
        Pn[((s & 1) * (kSynDeg / 2) + (s >> 1)) * kSynPS + pq] = r * f;
      }
      pipe_arrive(&full[st]);
    }
    pipe_cp_wait_all();   // no copy of this thread is in flight when the CTA exits
    return;
  }

  // consumer warp geometry
  const int par = warp / WT::WPP, rg = (warp % WT::WPP) / WT::CG, cg = warp % WT::CG;
  const int rowbase = rg * (64 / WT::RG), colbase = cg * (NCOL / WT::CG);
  const int g = lane >> 2, t = lane & 3;
  // first degree any pair of this warp's rows needs
  int wlmin = INT_MAX / 2;
  {
    const int pr = p0 + rowbase + lane;
    if (lane < 64 / WT::RG && pr < npair) wlmin = P.l0[(size_t)im * npair + pr];
    for (int o = 16; o > 0; o >>= 1) wlmin = min(wlmin, __shfl_xor_sync(0xffffffffu, wlmin, o));
  }
  double acc[WT::MT][WT::NT][4];
#pragma unroll
  for (int i = 0; i < WT::MT; ++i)
#pragma unroll
    for (int j = 0; j < WT::NT; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  for (int c = 0; c < nchunks; ++c) {
    const int st = c % S;
    if (!pipe_wait(&full[st], (c / S) & 1, abort_flag, err)) break;
    const int lc = lbeg + c * kSynDeg;
    if (lc + kSynDeg - 1 >= wlmin) {
      const double* Pn = sm + st * SM::STAGE + par * (kSynDeg / 2) * kSynPS;
      const double* C = sm + st * SM::STAGE + SM::PBUF + par * NF * kSynCS;
#pragma unroll
      for (int ks = 0; ks < kSynDeg / 8; ++ks) {
        double a[WT::MT][2], b[WT::NT];
#pragma unroll
        for (int i = 0; i < WT::MT; ++i) {
          const double* pa = Pn + (ks * 4 + t) * kSynPS + rowbase + i * 16 + g;
          a[i][0] = pa[0];
          a[i][1] = pa[8];
        }
#pragma unroll
        for (int j = 0; j < WT::NT; ++j) {
          const int col = colbase + j * 8 + g;
          b[j] = C[(col >> 1) * kSynCS + 2 * (ks * 4 + t) + (col & 1)];
        }
#pragma unroll
        for (int i = 0; i < WT::MT; ++i)
#pragma unroll
          for (int j = 0; j < WT::NT; ++j) dmma_16x8x4(acc[i][j], a[i][0], a[i][1], b[j]);
      }
    }
    __syncwarp();
    if (lane == 0) pipe_arrive(&empty[st]);
  }
  if (*abort_flag) return;
#pragma unroll
  for (int i = 0; i < WT::MT; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int pr = p0 + rowbase + i * 16 + g + 8 * h;
      if (pr >= npair) continue;
#pragma unroll
      for (int j = 0; j < WT::NT; ++j) {
        const int kf = kb + (colbase + j * 8) / 2 + t;
        if (kf >= nf) continue;
        W[(((size_t)kf * P.nm + im) * 2 + par) * npair + pr] = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
      }
    }
}

template <int NCOL>
static int launch_syn_ncol(const shtb_plan* p, const CoefSrc& src, const Factors& F, void* W, int nf, int row_end,
                           int mlim, cudaStream_t st) {
  auto kern = leg_syn64_kernel<NCOL>;
  // shared memory for the longest order (m = 0)
  const int ndeg = std::min(row_end, p->lrec) + 1;
  const size_t smem = SynSmem<NCOL>::bytes(ndeg);
  if (smem > 227 * 1024) return set_error(SHTB_ERR_UNSUPPORTED, "lmax too large for the FP64 synthesis kernel");
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "synthesis smem attr");
  constexpr int NF = WarpTile<NCOL>::NF;
  dim3 grid((p->npair + kSynPairs - 1) / kSynPairs, mlim / p->mres + 1, (nf + NF - 1) / NF);
  prof_begin(st);
  kern<<<grid, kLegThreads, smem, st>>>(p->dev, src, F, (double2*)W, nf, row_end, p->d_err);
  SHTB_LAUNCHED("legendre synthesis kernel");
  return SHTB_OK;
}

int launch_leg_syn64(const shtb_plan* p, const CoefSrc& src, const Factors& F, void* W, int nf, int row_end,
                     int mlim, cudaStream_t st) {
  if (nf > 32) return launch_syn_ncol<128>(p, src, F, W, nf, row_end, mlim, st);
  if (nf > 16) return launch_syn_ncol<64>(p, src, F, W, nf, row_end, mlim, st);
  if (nf > 8) return launch_syn_ncol<32>(p, src, F, W, nf, row_end, mlim, st);
  if (nf > 4) return launch_syn_ncol<16>(p, src, F, W, nf, row_end, mlim, st);
  return launch_syn_ncol<8>(p, src, F, W, nf, row_end, mlim, st);
}

// ---------------------------------------------------------------------------
// analysis: CTA = (128 degrees of order m, NCOL/2 fields), K chunks of kAnaPairs pairs
// ---------------------------------------------------------------------------
constexpr int kAnaPairs = 16;                    // latitude pairs per chunk
constexpr int kAnaAS = kAnaPairs + 4;            // P panel row stride (doubles), = 4 mod 16
constexpr int kAnaBS = 2 * kAnaPairs + 8;        // Fourier panel field stride (doubles), = 8 mod 16
constexpr int kAnaMaxChunks = 512;               // npair <= 8192
constexpr int kAnaStages = 3;

template <int NCOL>
struct AnaSmem {
  static constexpr int NF = WarpTile<NCOL>::NF;
  static constexpr int ABUF = 2 * 64 * kAnaAS;   // [parity][64 rows][pairs]
  static constexpr int BBUF = 2 * NF * kAnaBS;   // [parity][field][pairs x re|im]
  static constexpr int STAGE = ABUF + BBUF;
  static constexpr int ALPH = kAnaStages * STAGE;          // alpha of the tile's 128 degrees
  static constexpr int BAR = ALPH + kAnaTile;              // then full[S], empty[S], flags, chunk list
  static size_t bytes() { return (size_t)BAR * 8 + 2 * kAnaStages * 8 + 16 + (kAnaMaxChunks + 8) * 4; }
};

template <int NCOL>
__global__ void __launch_bounds__(kLegThreads, 1)
    leg_ana64_kernel(PlanDev P, const double2* __restrict__ W, int nf, int row_end, int mlim, CoefSink dst, Factors F,
                     int zero_fill, int* err) {
  using WT = WarpTile<NCOL>;
  using SM = AnaSmem<NCOL>;
  constexpr int NF = WT::NF, S = kAnaStages;
  extern __shared__ __align__(16) double sm[];
  double* salph = sm + SM::ALPH;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + SM::BAR);
  unsigned long long* empty = full + S;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + S);
  int* slist = reinterpret_cast<int*>(empty + S) + 4;   // nonzero chunks, then their count
  const int4 tile = P.atiles[blockIdx.x];
  const int im = tile.x, t0 = tile.y, ck0 = tile.z, m = im * P.mres;
  const int lend = min(row_end, P.lrec);
  if (m > mlim || t0 > lend) return;
  const int kb = blockIdx.y * NF;
  const int npair = P.npair;
  const long long poff = P.off[im];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool producer = warp >= kConsumerWarps;
  const int tlast = min(t0 + kAnaTile - 1, lend);

  if (tid == 0) {
    for (int q = 0; q < S; ++q) {
      pipe_bar_init(&full[q], 32 * kProducerWarps);
      pipe_bar_init(&empty[q], kConsumerWarps);
    }
    *abort_flag = 0;
    pipe_bar_init_fence();
  }
  for (int i = tid; i < kAnaTile; i += kLegThreads) {
    const int l = t0 + i;
    salph[i] = (l <= lend) ? P.alpha[poff + (l - m)] : 0.0;
  }
  // chunks with a nonzero P value: some pair's first significant degree is <= tlast
  const int nch = (npair + kAnaPairs - 1) / kAnaPairs;
  if (warp == 0) {
    int cnt = 0;
    for (int c0 = 0; c0 < nch; c0 += 32) {
      const int c = c0 + lane;
      bool nz = false;
      if (c < nch) {
        int mn = INT_MAX;
        for (int q = 0; q < kAnaPairs; ++q) {
          const int p = c * kAnaPairs + q;
          if (p < npair) mn = min(mn, P.l0[(size_t)im * npair + p]);
        }
        nz = mn <= tlast;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, nz);
      if (nz) slist[cnt + __popc(bal & ((1u << lane) - 1u))] = c;
      cnt += __popc(bal);
    }
    if (lane == 0) slist[kAnaMaxChunks] = cnt;
  }
  __syncthreads();
  const int nz = slist[kAnaMaxChunks];

  if (producer) {
    // every producer thread takes part in every chunk: thread q = 32 w + lane runs the chain
    // of pair q % 16 over the tile's checkpoint segment q / 16 (ckstep degrees)
    const int ptid = tid - 32 * kConsumerWarps, pq = ptid % kAnaPairs, seg = ptid / kAnaPairs;
    const int cs = P.ckstep, nseg = kAnaTile / cs;
    const bool chain = seg < nseg && t0 + seg * cs <= P.lrec;
    for (int ci = 0; ci < nz; ++ci) {
      const int st = ci % S;
      if (ci >= S && !pipe_wait(&empty[st], ((ci / S) - 1) & 1, abort_flag, err)) break;
      const int c = slist[ci];
      double* A = sm + st * SM::STAGE;
      double* B = A + SM::ABUF;
      for (int idx = ptid; idx < 2 * NF * kAnaPairs; idx += 32 * kProducerWarps) {
        const int q = idx % kAnaPairs, rest = idx / kAnaPairs, fl = rest % NF, pr = rest / NF;
        const int pair = c * kAnaPairs + q, kf = kb + fl;
        const bool ok = pair < npair && kf < nf;
        const double2* gp = ok ? W + (((size_t)kf * P.nm + im) * 2 + pr) * npair + pair : W;
        pipe_cp16(B + (pr * NF + fl) * kAnaBS + 2 * q, gp, ok ? 16u : 0u);
      }
      pipe_arrive_cp_async(&full[st]);
      if (seg < nseg) {
        const int p = c * kAnaPairs + pq;
        double x = 0.0, ra = 0.0, rb = 0.0, r0 = 0.0, r1 = 0.0;
        int l0 = INT_MAX / 2;
        if (p < npair && chain) {
          x = P.x[p];
          const double2 stv = P.ckpt[(size_t)(ck0 + seg) * npair + p];
          ra = stv.x;
          rb = stv.y;
          l0 = P.l0[(size_t)im * npair + p];
          const double2 v = P.r01[(size_t)im * npair + p];
          r0 = v.x;
          r1 = v.y;
        }
        const int d0 = seg * cs;
        double* Ar = A + pq;
#pragma unroll 4
        for (int s = 0; s < cs; ++s) {
          const int d = d0 + s, l = t0 + d;
          double r = fma(salph[d] * x, ra, -rb);
          r = (l == l0) ? r0 : r;
          r = (l == l0 + 1) ? r1 : r;
          rb = ra;
          ra = r;
          Ar[((d & 1) * 64 + (d >> 1)) * kAnaAS] = r;
        }
      }
      pipe_arrive(&full[st]);
    }
    pipe_cp_wait_all();   // no copy of this thread is in flight when the CTA exits
    return;
  }

  const int par = warp / WT::WPP, rg = (warp % WT::WPP) / WT::CG, cg = warp % WT::CG;
  const int rowbase = rg * (64 / WT::RG), colbase = cg * (NCOL / WT::CG);
  const int g = lane >> 2, t = lane & 3;
  double acc[WT::MT][WT::NT][4];
#pragma unroll
  for (int i = 0; i < WT::MT; ++i)
#pragma unroll
    for (int j = 0; j < WT::NT; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  // 16-row fragments whose first degree lies past lend hold no output: no MMAs for them
  // (m-tiles are in increasing degree order, so live[0] false means none is live)
  bool live[WT::MT];
#pragma unroll
  for (int i = 0; i < WT::MT; ++i) live[i] = t0 + 2 * (rowbase + i * 16) + par <= lend;

  for (int ci = 0; ci < nz; ++ci) {
    const int st = ci % S;
    if (!pipe_wait(&full[st], (ci / S) & 1, abort_flag, err)) break;
    const double* A = sm + st * SM::STAGE + par * 64 * kAnaAS;
    const double* B = sm + st * SM::STAGE + SM::ABUF + par * NF * kAnaBS;
#pragma unroll
    for (int ks = 0; ks < kAnaPairs / 4 && live[0]; ++ks) {
      double a[WT::MT][2], b[WT::NT];
#pragma unroll
      for (int i = 0; i < WT::MT; ++i) {
        const double* pa = A + (rowbase + i * 16 + g) * kAnaAS + ks * 4 + t;
        a[i][0] = pa[0];
        a[i][1] = pa[8 * kAnaAS];
      }
#pragma unroll
      for (int j = 0; j < WT::NT; ++j) {
        const int col = colbase + j * 8 + g;
        b[j] = B[(col >> 1) * kAnaBS + 2 * (ks * 4 + t) + (col & 1)];
      }
#pragma unroll
      for (int i = 0; i < WT::MT; ++i)
        if (live[i]) {
#pragma unroll
          for (int j = 0; j < WT::NT; ++j) dmma_16x8x4(acc[i][j], a[i][0], a[i][1], b[j]);
        }
    }
    __syncwarp();
    if (lane == 0) pipe_arrive(&empty[st]);
  }
  if (*abort_flag) return;

  const long long dbase = dst.packed == 1 ? (poff - m)
                          : dst.packed == 2 ? lm_base(P.lmax, P.mres, m) : (long long)m * dst.ld_m;
  const int lcap = dst.packed == 1 ? lend : min(lend, P.lmax);
#pragma unroll
  for (int i = 0; i < WT::MT; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = rowbase + i * 16 + g + 8 * h;
      const int l = t0 + 2 * row + par;
      if (l > lcap) continue;
      const double s = factor_at(P, F, poff, l, m);
#pragma unroll
      for (int j = 0; j < WT::NT; ++j) {
        const int kf = kb + (colbase + j * 8) / 2 + t;
        if (kf >= nf) continue;
        dst.ptr[(long long)kf * dst.ld_k + dbase + l] = make_double2(acc[i][j][2 * h] * s, acc[i][j][2 * h + 1] * s);
      }
    }
  if (zero_fill && !dst.packed && t0 == m) {
    const int nz_lo = m, nz_hi = P.lmax - lcap;  // rows [0, m) and (lcap, lmax]
    const int nrow = nz_lo + max(nz_hi, 0);
    for (int idx = tid; idx < nrow * NF; idx += 32 * kConsumerWarps) {
      const int r = idx % nrow, fl = idx / nrow, kf = kb + fl;
      if (kf >= nf) continue;
      const int l = (r < nz_lo) ? r : lcap + 1 + (r - nz_lo);
      dst.ptr[(long long)kf * dst.ld_k + (long long)m * dst.ld_m + l] = make_double2(0.0, 0.0);
    }
  }
}

template <int NCOL>
static int launch_ana_ncol(const shtb_plan* p, const void* W, int nf, int row_end, int mlim, const CoefSink& dst,
                           const Factors& F, int zero_fill, cudaStream_t st) {
  if ((p->npair + kAnaPairs - 1) / kAnaPairs > kAnaMaxChunks)
    return set_error(SHTB_ERR_UNSUPPORTED, "nlat too large for the FP64 analysis kernel");
  auto kern = leg_ana64_kernel<NCOL>;
  const size_t smem = AnaSmem<NCOL>::bytes();
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "analysis smem attr");
  constexpr int NF = WarpTile<NCOL>::NF;
  dim3 grid(p->dev.natiles, (nf + NF - 1) / NF);
  prof_begin(st);
  kern<<<grid, kLegThreads, smem, st>>>(p->dev, (const double2*)W, nf, row_end, mlim, dst, F, zero_fill, p->d_err);
  SHTB_LAUNCHED("legendre analysis kernel");
  return SHTB_OK;
}

int launch_leg_ana64(const shtb_plan* p, const void* W, int nf, int row_end, int mlim, const CoefSink& dst,
                     const Factors& F, int zero_fill, cudaStream_t st) {
  if (nf > 32) return launch_ana_ncol<128>(p, W, nf, row_end, mlim, dst, F, zero_fill, st);
  if (nf > 16) return launch_ana_ncol<64>(p, W, nf, row_end, mlim, dst, F, zero_fill, st);
  if (nf > 8) return launch_ana_ncol<32>(p, W, nf, row_end, mlim, dst, F, zero_fill, st);
  if (nf > 4) return launch_ana_ncol<16>(p, W, nf, row_end, mlim, dst, F, zero_fill, st);
  return launch_ana_ncol<8>(p, W, nf, row_end, mlim, dst, F, zero_fill, st);
}

}  // namespace shtb
