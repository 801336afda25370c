// mixed.cu — mixed-precision Legendre stage on the 5th-generation tensor cores.
//
// Per order m both directions are dense GEMMs over one parity class of degrees:
//   synthesis  E[pair, col] = sum_j  P[m+2j,   pair] * a[m+2j,   col]    (O: degrees m+2j+1)
//   analysis   a[m+2j, col] = sum_pair P[m+2j, pair] * E[pair, col]      (O likewise)
// with col = (field, re|im). Each GEMM runs as tcgen05.mma kind::tf32 with FP32
// accumulation in TMEM, using the 3xTF32 split x = hi + lo (both rounded to
// nearest TF32): x*y ~ hi_x hi_y + hi_x lo_y + lo_x hi_y.
//
// P comes from a per-plan FP32 table of P_l^m(x_pair), l = m..lmax+1, grouped by
// (m, parity) as rows of padded latitude pairs. The table is written once by
// mixed_table_kernel from the FP64 recurrence (extended-range seeds and FP64
// recurrence coefficients), so every P value is the FP64 result rounded once.
//
// CTA organisation (544 threads, one parity class per CTA): warps 0-7 are two
// producer groups of 128 threads that load operands, split them into hi/lo and
// store K-major tiles (no swizzle) into an 8-stage shared-memory ring,
// alternating stages; warp 8 allocates TMEM and one of its threads issues the
// MMAs (tcgen05.commit releases each stage). The tensor core accumulates only
// kChunk K-steps into one of two TMEM buffers (hi*hi and the small cross terms
// in separate accumulators); warps 9-16 drain each finished chunk with
// tcgen05.ld into round-to-nearest FP32 register sums. Long accumulation chains
// inside the tensor core round toward zero and would bias sums of many terms;
// short chunks keep that bias below 1e-6 relative at any lmax.
// Every mbarrier wait is bounded (2 s of %globaltimer); a timeout sets the
// plan's error word and the CTA drains and exits.
#include <climits>

#include "kernels.cuh"

namespace shtb {
namespace mx {

constexpr int kM = 128;          // UMMA M
constexpr int kK = 8;            // TF32 K per instruction
constexpr int kStages = 8;
constexpr int kChunk = 4;          // K-steps accumulated in TMEM before promotion
constexpr int kThreads = 544;       // 8 producer warps, 1 MMA warp, 8 promotion warps
constexpr int kTileBytesA = kM * kK * 4;  // 4 KB
constexpr unsigned long long kWaitNs = 2000000000ull;

struct Args {
  PlanDev P;
  const float* tab;
  const long long* seg;      // [2*nm+1] first table row of segment (im, parity); rows hold npp pairs
  int npp;
  const float2* cin;         // synthesis: coefficients; analysis: unused
  const float2* Win;         // analysis: Fourier buffer [f][nm][2][npair]
  float2* Wout;              // synthesis: Fourier buffer
  float2* cout;              // analysis: coefficients
  long long ld_k;            // coefficient field stride (complex elements)
  const double* sc;          // normalization scale table (dense) or null
  int sc_mode;               // 0 none, 1 multiply, 2 divide
  float mf0, mf1;
  int nf, lend, lcap;
  const int2* tiles;         // analysis tiles (im, j0)
  int* err;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false after a timeout or once another thread of the CTA gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, volatile int* abort_flag,
                                          int* err) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_test(bar, parity)) {
    if (*abort_flag) return false;
    if (gtimer() - t0 > kWaitNs) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ float tf32_rn(float x) {
  unsigned u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return __uint_as_float(u);
}

// K-major, no-swizzle tile: 8-row core matrices of 16-byte rows; the two 16-byte
// K halves of a core-matrix pair are 128 bytes apart (LBO), 8-row groups 256 bytes (SBO).
__device__ __forceinline__ int tile_off(int r, int khalf) { return (r >> 3) * 256 + khalf * 128 + (r & 7) * 16; }

__device__ __forceinline__ unsigned long long sdesc(const void* p) {
  const unsigned a = smem_u32(p);
  return (unsigned long long)((a >> 4) & 0x3FFF) | ((unsigned long long)(128 >> 4) << 16) |
         ((unsigned long long)(256 >> 4) << 32) | (1ull << 46);
}

template <int N>
__device__ __forceinline__ unsigned idesc_tf32() {
  // F32 accumulate, A/B TF32, both K-major, N>>3 at bit 17, M>>4 at bit 24
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                         unsigned accum) {
  const unsigned z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Split 8 consecutive K values of one row into hi/lo tiles.
__device__ __forceinline__ void store_split8(unsigned char* hi, unsigned char* lo, int row, const float* v) {
  float4 h0, h1, l0, l1;
  h0.x = tf32_rn(v[0]); h0.y = tf32_rn(v[1]); h0.z = tf32_rn(v[2]); h0.w = tf32_rn(v[3]);
  h1.x = tf32_rn(v[4]); h1.y = tf32_rn(v[5]); h1.z = tf32_rn(v[6]); h1.w = tf32_rn(v[7]);
  l0.x = tf32_rn(v[0] - h0.x); l0.y = tf32_rn(v[1] - h0.y); l0.z = tf32_rn(v[2] - h0.z); l0.w = tf32_rn(v[3] - h0.w);
  l1.x = tf32_rn(v[4] - h1.x); l1.y = tf32_rn(v[5] - h1.y); l1.z = tf32_rn(v[6] - h1.z); l1.w = tf32_rn(v[7] - h1.w);
  *reinterpret_cast<float4*>(hi + tile_off(row, 0)) = h0;
  *reinterpret_cast<float4*>(hi + tile_off(row, 1)) = h1;
  *reinterpret_cast<float4*>(lo + tile_off(row, 0)) = l0;
  *reinterpret_cast<float4*>(lo + tile_off(row, 1)) = l1;
}

__device__ __forceinline__ float coef_factor(const Args& a, int l, int m) {
  double s = (m == 0) ? (double)a.mf0 : (double)a.mf1;
  if (a.sc_mode) {
    const double q = a.sc[l + (long long)(a.P.lmax + 1) * m];
    s = (a.sc_mode == 1) ? s * q : s / q;
  }
  return (float)s;
}

template <int N>
struct Smem {
  static constexpr int kTileB = N * kK * 4;
  // per stage: A_hi, A_lo, B_hi, B_lo (one parity class per CTA)
  static constexpr int kStage = 2 * kTileBytesA + 2 * kTileB;
  static constexpr int kBar = kStages * kStage;
  static constexpr int kBytes = kBar + (2 * kStages + 4) * 8 + 16;
};

__device__ __forceinline__ void store_split4(unsigned char* hi, unsigned char* lo, int row, int khalf, const float* v) {
  float4 h, l;
  h.x = tf32_rn(v[0]); h.y = tf32_rn(v[1]); h.z = tf32_rn(v[2]); h.w = tf32_rn(v[3]);
  l.x = tf32_rn(v[0] - h.x); l.y = tf32_rn(v[1] - h.y); l.z = tf32_rn(v[2] - h.z); l.w = tf32_rn(v[3] - h.w);
  *reinterpret_cast<float4*>(hi + tile_off(row, khalf)) = h;
  *reinterpret_cast<float4*>(lo + tile_off(row, khalf)) = l;
}

// MODE 0: synthesis, MODE 1: analysis. N = columns per CTA (2 x fields).
// blockIdx.x = 2 * tile + parity; one CTA accumulates one parity class.
template <int MODE, int N>
__global__ void __launch_bounds__(kThreads, 1) mixed_gemm_kernel(const __grid_constant__ Args a) {
  using S = Smem<N>;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + S::kBar);
  unsigned long long* empty = full + kStages;
  unsigned long long* accf = empty + kStages;   // [2] chunk accumulated in TMEM buffer b
  unsigned long long* acce = accf + 2;          // [2] TMEM buffer b drained by the promotion warps
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(acce + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const PlanDev& P = a.P;
  const int npair = P.npair;
  const int par = blockIdx.x & 1, tile = blockIdx.x >> 1;
  int im, p0 = 0, j0 = 0;
  if (MODE == 0) {
    im = blockIdx.y;
    p0 = tile * kM;
  } else {
    const int2 t = a.tiles[tile];
    im = t.x;
    j0 = t.y;
  }
  const int m = im * P.mres;
  const int kb = blockIdx.z * (N / 2);
  // degrees of this parity class in [m, lend]
  const int J = (a.lend >= m + par) ? (a.lend - m - par) / 2 + 1 : 0;
  const long long sg = a.seg[2 * im + par];
  const long long ln = a.seg[2 * im + par + 1] - sg;
  const int nks = (MODE == 0) ? (J + kK - 1) / kK : (npair + kK - 1) / kK;
  const int nch = (nks + kChunk - 1) / kChunk;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 128);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 256);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(4 * N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot;
  // TMEM: buffer b holds the hi*hi chunk sum at column 2bN and the cross terms at 2bN + N

  if (warp < 8) {
    // ------------------------------------------------------------- producers
    const int g = warp >> 2, t = tid & 127;
    const int bf = t >> 1, bh = t & 1;           // B: field bf, K half bh (4 values)
    const bool bact = bf < N / 2;
    float va[kK], vb[2][4];
    auto load = [&](int ks) {
      if (MODE == 0) {
        const int pr = p0 + t;
#pragma unroll
        for (int k = 0; k < kK; ++k) {
          const int j = ks * kK + k;
          va[k] = (j < ln) ? a.tab[(sg + j) * a.npp + pr] : 0.f;
        }
      } else {
        const int j = j0 + t;
        if (j < ln) {
          const float4* q = reinterpret_cast<const float4*>(a.tab + (sg + j) * a.npp + ks * kK);
          const float4 x0 = q[0], x1 = q[1];
          va[0] = x0.x; va[1] = x0.y; va[2] = x0.z; va[3] = x0.w;
          va[4] = x1.x; va[5] = x1.y; va[6] = x1.z; va[7] = x1.w;
        } else {
#pragma unroll
          for (int k = 0; k < kK; ++k) va[k] = 0.f;
        }
      }
      const int kf = kb + bf;
#pragma unroll
      for (int k = 0; k < 4; ++k) vb[0][k] = vb[1][k] = 0.f;
      if (bact && kf < a.nf) {
        if (MODE == 0) {
          const float2* c = a.cin + (long long)kf * a.ld_k + (long long)m * (P.lmax + 1);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int l = m + 2 * (ks * kK + 4 * bh + k) + par;
            if (l <= a.lend) {
              float2 v = c[l];
              const float s = coef_factor(a, l, m);
              vb[0][k] = v.x * s;
              vb[1][k] = v.y * s;
            }
          }
        } else {
          const float2* w = a.Win + (((long long)kf * P.nm + im) * 2 + par) * npair;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int pr = ks * kK + 4 * bh + k;
            if (pr < npair) {
              const float2 v = w[pr];
              vb[0][k] = v.x;
              vb[1][k] = v.y;
            }
          }
        }
      }
    };
    if (g < nks) load(g);
    for (int ks = g; ks < nks; ks += 2) {
      const int b = ks % kStages;
      if (ks >= kStages)
        if (!mbar_wait(&empty[b], ((ks / kStages) - 1) & 1, abort_flag, a.err)) break;
      unsigned char* st = sm + (size_t)b * S::kStage;
      store_split8(st, st + kTileBytesA, t, va);
      if (bact) {
        unsigned char* bh_ = st + 2 * kTileBytesA;
        unsigned char* bl_ = bh_ + S::kTileB;
        store_split4(bh_, bl_, 2 * bf, bh, vb[0]);
        store_split4(bh_, bl_, 2 * bf + 1, bh, vb[1]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[b]);
      if (ks + 2 < nks) load(ks + 2);
    }
  } else if (warp == 8) {
    // ------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const unsigned idesc = idesc_tf32<N>();
      bool ok = true;
      for (int c = 0; c < nch && ok; ++c) {
        const int bb = c & 1;
        if (c >= 2 && !mbar_wait(&acce[bb], ((c >> 1) - 1) & 1, abort_flag, a.err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned dH = tmem + 2 * bb * N, dX = dH + N;
        const int k1 = min(nks, (c + 1) * kChunk);
        for (int ks = c * kChunk; ks < k1; ++ks) {
          const int b = ks % kStages;
          if (!mbar_wait(&full[b], (ks / kStages) & 1, abort_flag, a.err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char* st = sm + (size_t)b * S::kStage;
          const unsigned long long ah = sdesc(st), al = sdesc(st + kTileBytesA);
          const unsigned long long bh_ = sdesc(st + 2 * kTileBytesA), bl_ = sdesc(st + 2 * kTileBytesA + S::kTileB);
          const unsigned acc = (ks == c * kChunk) ? 0u : 1u;
          mma_tf32(dH, ah, bh_, idesc, acc);
          mma_tf32(dX, ah, bl_, idesc, acc);
          mma_tf32(dX, al, bh_, idesc, 1u);
          mma_commit(&empty[b]);
        }
        mma_commit(&accf[bb]);
      }
    }
  } else {
    // ------------------------------------------------------------- promotion warps (9..16)
    const int q = warp & 3;                        // TMEM lane quadrant this warp may access
    const int h = (warp - 9) >> 2;                 // column half
    const int row = 32 * q + lane;
    const unsigned lane_base = (unsigned)(32 * q) << 16;
    float acc[N / 2];
#pragma unroll
    for (int i = 0; i < N / 2; ++i) acc[i] = 0.f;
    bool ok = true;
    for (int c = 0; c < nch; ++c) {
      const int bb = c & 1;
      if (ok) ok = mbar_wait(&accf[bb], (c >> 1) & 1, abort_flag, a.err);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      __syncwarp();
      const unsigned dH = tmem + lane_base + 2 * bb * N + h * (N / 2), dX = dH + N;
#pragma unroll
      for (int i = 0; i < N / 2; i += 16) {
        float vh[16], vx[16];
        tmem_ld16(dH + i, vh);
        tmem_ld16(dX + i, vx);
#pragma unroll
        for (int u = 0; u < 16; ++u) acc[i + u] += vh[u] + vx[u];
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&acce[bb]);
      if (!ok) break;
    }
    if (ok) {
#pragma unroll
      for (int qq = 0; qq < N / 4; ++qq) {
        const int kf = kb + h * (N / 4) + qq;
        if (kf >= a.nf) continue;
        if (MODE == 0) {
          const int pr = p0 + row;
          if (pr < npair) a.Wout[(((size_t)kf * P.nm + im) * 2 + par) * npair + pr] = make_float2(acc[2 * qq], acc[2 * qq + 1]);
        } else {
          const int l = m + 2 * (j0 + row) + par;
          if (l <= a.lcap) {
            const float s = coef_factor(a, l, m);
            a.cout[(long long)kf * a.ld_k + (long long)m * (P.lmax + 1) + l] = make_float2(acc[2 * qq] * s, acc[2 * qq + 1] * s);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 8) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(4 * N));
  }
}

// Table: P_l^m(x_pair) as FP32 at row seg[2 im + (l-m)%2] + (l-m)/2, column pair.
__global__ void mixed_table_kernel(PlanDev P, float* __restrict__ tab, const long long* __restrict__ seg, int npp) {
  const int pair = blockIdx.x * blockDim.x + threadIdx.x;
  const int im = blockIdx.y;
  if (pair >= P.npair) return;
  const int m = im * P.mres;
  const long long poff = P.off[im];
  const double x = P.x[pair];
  const int l0 = P.l0[(size_t)im * P.npair + pair];
  const double2 r01 = P.r01[(size_t)im * P.npair + pair];
  double ra = 0.0, rb = 0.0;
  for (int l = m; l <= P.lrec; ++l) {
    double r;
    if (l == l0)
      r = r01.x;
    else if (l == l0 + 1)
      r = r01.y;
    else
      r = fma(P.alpha[poff + (l - m)] * x, ra, -rb);
    rb = ra;
    ra = r;
    const int par = (l - m) & 1, j = (l - m) >> 1;
    tab[(seg[2 * im + par] + j) * npp + pair] = (float)(P.cfac[poff + (l - m)] * r);
  }
}

}  // namespace mx

using namespace mx;

static int ensure_table(const shtb_plan* cp, cudaStream_t st) {
  shtb_plan* p = const_cast<shtb_plan*>(cp);
  std::lock_guard<std::mutex> lk(p->tab_mu);
  if (p->d_tab) return SHTB_OK;
  const int nm = p->nm, LR = p->lrec;
  p->npp = (p->npair + kM - 1) / kM * kM;
  p->htab_seg.assign(2 * nm + 1, 0);
  long long rows = 0;
  for (int im = 0; im < nm; ++im) {
    const int m = im * p->mres;
    for (int par = 0; par < 2; ++par) {
      p->htab_seg[2 * im + par] = rows;
      const int cnt = (LR - m - par >= 0) ? (LR - m - par) / 2 + 1 : 0;
      rows += (cnt + kK - 1) / kK * kK;
    }
  }
  p->htab_seg[2 * nm] = rows;
  const size_t tb = (size_t)rows * p->npp * 4;
  void* mem = nullptr;
  cudaError_t e = cudaMalloc(&mem, tb + (2 * nm + 1) * 8 + 256);
  if (e != cudaSuccess) return set_error(SHTB_ERR_OOM, std::string("mixed table: ") + cudaGetErrorString(e));
  float* tab = (float*)mem;
  long long* dseg = (long long*)((char*)mem + (tb + 255) / 256 * 256);
  e = cudaMemcpyAsync(dseg, p->htab_seg.data(), (2 * nm + 1) * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tab, 0, tb, st);
  if (e != cudaSuccess) {
    cudaFree(mem);
    return set_error(SHTB_ERR_CUDA, std::string("mixed table init: ") + cudaGetErrorString(e));
  }
  dim3 grid((p->npair + 127) / 128, nm);
  mixed_table_kernel<<<grid, 128, 0, st>>>(p->dev, tab, dseg, p->npp);
  count_launch();
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(mem);
    return set_error(SHTB_ERR_CUDA, std::string("mixed table kernel: ") + cudaGetErrorString(e));
  }
  p->d_tab = tab;
  p->d_tab_seg = dseg;
  p->tab_bytes = tb;
  return SHTB_OK;
}

template <int MODE, int N>
static int launch_gemm(const shtb_plan* p, const Args& a, dim3 grid, cudaStream_t st) {
  auto kern = mixed_gemm_kernel<MODE, N>;
  const int smem = Smem<N>::kBytes;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "mixed smem attr");
  prof_begin(st);
  kern<<<grid, kThreads, smem, st>>>(a);
  SHTB_LAUNCHED(MODE == 0 ? "tc gemm synthesis kernel" : "tc gemm analysis kernel");
  return SHTB_OK;
}

template <int MODE>
static int dispatch_gemm(const shtb_plan* p, const Args& a, int nf, dim3 grid_xy, cudaStream_t st) {
  if (nf > 32) { dim3 g(grid_xy.x, grid_xy.y, (nf + 63) / 64); return launch_gemm<MODE, 128>(p, a, g, st); }
  if (nf > 16) { dim3 g(grid_xy.x, grid_xy.y, 1); return launch_gemm<MODE, 64>(p, a, g, st); }
  if (nf > 8) { dim3 g(grid_xy.x, grid_xy.y, 1); return launch_gemm<MODE, 32>(p, a, g, st); }
  dim3 g(grid_xy.x, grid_xy.y, 1);
  return launch_gemm<MODE, 16>(p, a, g, st);
}

__global__ void zero_outside_kernel32(PlanDev P, float2* __restrict__ a, long long ld_k, int mlim, int lcap) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y, k = blockIdx.z;
  if (l > P.lmax) return;
  if ((m % P.mres) != 0 || m > mlim || l < m || l > lcap)
    a[(long long)k * ld_k + (long long)m * (P.lmax + 1) + l] = make_float2(0.f, 0.f);
}

static Args base_args(const shtb_plan* p) {
  Args a{};
  a.P = p->dev;
  a.tab = p->d_tab;
  a.seg = p->d_tab_seg;
  a.npp = p->npp;
  a.ld_k = (long long)(p->lmax + 1) * (p->mmax + 1);
  a.sc = p->d_scale;
  a.err = p->d_err;
  a.mf0 = a.mf1 = 1.f;
  return a;
}

int mixed_synthesis(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, void* work, cudaStream_t st) {
  int rc = ensure_table(p, st);
  if (rc) return rc;
  const int mlim = std::min(p->mmax, ltr);
  Args a = base_args(p);
  a.cin = (const float2*)alm;
  a.Wout = (float2*)work;
  a.sc_mode = p->d_scale ? 1 : 0;
  a.nf = nf;
  a.lend = ltr;
  a.lcap = ltr;
  dim3 g(2 * ((p->npair + kM - 1) / kM), mlim / p->mres + 1);
  if ((rc = dispatch_gemm<0>(p, a, nf, g, st))) return rc;
  return launch_fft_syn<float, float>(p, work, (float*)f, nullptr, 1, nf, mlim, p->phi_inv_scale / p->nlon, 0, 0, st);
}

int mixed_analysis(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, void* work, cudaStream_t st) {
  int rc = ensure_table(p, st);
  if (rc) return rc;
  const int mlim = std::min(p->mmax, ltr);
  if ((rc = launch_fft_ana<float, float>(p, (const float*)f, nullptr, 1, work, nf, mlim, p->ana_scale, 1, 0, st)))
    return rc;
  // analysis tiles: 128 degrees of each parity per tile
  std::vector<int2>& tl = const_cast<shtb_plan*>(p)->hmx_tiles;
  const int key = ltr;
  if (p->mx_tiles_key != key) {
    tl.clear();
    for (int im = 0; im * p->mres <= mlim; ++im) {
      const int m = im * p->mres;
      const int JE = (ltr - m) / 2 + 1;
      for (int j0 = 0; j0 < JE; j0 += kM) tl.push_back(make_int2(im, j0));
    }
    shtb_plan* pm = const_cast<shtb_plan*>(p);
    if (pm->d_mx_tiles) cudaFree(pm->d_mx_tiles);
    pm->d_mx_tiles = nullptr;
    SHTB_TRY_CUDA(cudaMalloc(&pm->d_mx_tiles, tl.size() * sizeof(int2)), "mixed tiles");
    SHTB_TRY_CUDA(cudaMemcpyAsync(pm->d_mx_tiles, tl.data(), tl.size() * sizeof(int2), cudaMemcpyHostToDevice, st),
                  "mixed tiles upload");
    pm->mx_tiles_key = key;
  }
  Args a = base_args(p);
  a.Win = (const float2*)work;
  a.cout = (float2*)alm;
  a.sc_mode = p->d_scale ? 2 : 0;
  a.nf = nf;
  a.lend = ltr;
  a.lcap = ltr;
  a.tiles = p->d_mx_tiles;
  dim3 g(2 * (unsigned)tl.size(), 1);
  if ((rc = dispatch_gemm<1>(p, a, nf, g, st))) return rc;
  dim3 zg((p->lmax + 1 + 127) / 128, p->mmax + 1, nf);
  prof_begin(st);
  zero_outside_kernel32<<<zg, 128, 0, st>>>(p->dev, (float2*)alm, a.ld_k, mlim, ltr);
  SHTB_LAUNCHED("zero fill kernel");
  return SHTB_OK;
}

}  // namespace shtb
