// mixed.cu — mixed-precision Legendre stage on the 5th-generation tensor cores.
//
// Per order m both directions are dense GEMMs over one parity class of degrees:
//   synthesis  E[pair, col] = sum_j  P[m+2j,   pair] * a[m+2j,   col]    (O: degrees m+2j+1)
//   analysis   a[m+2j, col] = sum_pair P[m+2j, pair] * E[pair, col]      (O likewise)
// with col = (field, re|im). Each GEMM runs as tcgen05.mma kind::f16 (K = 16, A and B f16)
// with FP32 accumulation in TMEM, on the split x = hi + lo of both operands into f16
// values (hi rounded to nearest, lo = the rounded remainder: 22 significant bits):
// x*y ~ hi_x hi_y + hi_x lo_y + lo_x hi_y. f16 has 5 exponent bits, so both operands are
// scaled by powers of two first: P by 2^s for the whole plan (its largest values near
// 2^15), B per row by 2^e so that the row's largest magnitude lies in [2^14, 2^15) (per
// segment in the synthesis, per chunk in the analysis); the promotion undoes both exactly.
//
// P comes from a per-plan table of P_l^m(x_pair), l = m..lmax+1, grouped by (m, parity)
// into segments of R rows (degrees, padded to a multiple of 16) by npp latitude pairs
// (padded to a multiple of 128). mixed_table_kernel writes it once from the FP64
// recurrence (extended-range seeds and FP64 recurrence coefficients), rounded once to
// FP32, scaled and split into f16 hi/lo. It is stored twice, as the byte images of the A
// tiles the two GEMMs load (synthesis 128 pairs x 16 degrees, analysis 128 degrees x 16
// pairs; hi and lo tiles of 4 KB each in the K-major no-swizzle core-matrix order), so one
// bulk copy (cp.async.bulk, completing on an mbarrier) fills a stage's A operand. The
// synthesis B images (coefficients) arrive split the same way from mixed_pack_kernel; the
// analysis B images (Fourier coefficients) arrive in FP32 from the FFT and are split in
// shared memory.
//
// CTA organisation (one parity class per CTA; at N = 128: 27 warps, 864 threads): one
// thread of the loader warp (25) fills a shared-memory ring of chunk stages (8 image
// K-steps of A and B each) with bulk copies; in the analysis, warps 0-7 split each
// chunk's B tiles in place; one thread of warp 8 (which allocates TMEM) issues the MMAs
// from shared memory, 12 per chunk, into one of 4 TMEM accumulators and commits once per
// chunk; warps 9-24 drain each finished chunk with tcgen05.ld into round-to-nearest FP32
// register sums and store the tile; warp 26 writes the analysis output's structural
// zeros (degrees below m and above lcap). Long accumulation chains inside
// the tensor core round toward zero and would bias sums of many terms; short chunks keep
// that bias below 1e-6 relative at any lmax.
// Every mbarrier wait is bounded (2 s of %globaltimer); a timeout sets the
// plan's error word and the CTA drains and exits.
#include <cuda_fp16.h>

#include <climits>
#include <cstring>

#include "kernels.cuh"

namespace shtb {
namespace mx {

constexpr int kM = 128;          // UMMA M
constexpr int kK = 8;            // K-step of the FP32 tile images (8 x 4 bytes = 16 f16 values)
constexpr int kTileBytesA = kM * kK * 4;  // 4 KB
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr int kChunk = 8;        // image K-steps (4 f16 K-steps, 12 MMAs) accumulated before promotion
constexpr int kScR = 16;         // ring of per-chunk B column scales
constexpr int kSegRows = 16;     // table segment padding (degrees): one f16 K-step
// Warp roles: splitters [0, kSW), MMA issuer kSW, promotion [kSW + 1, kSW + 1 + kPW), loader
// kSW + 1 + kPW, and at N >= 64 a clearing warp after it. The promotion warps (kPW of them,
// four per TMEM lane quadrant) each drain and store a quarter (kPW = 16, N >= 64) or a half
// (kPW = 8) of a tile's columns; the clearing warp writes the analysis output's structural
// zeros (l < m, l > lcap), which the promotion warps do themselves below N = 64.
constexpr int kSW = 8;
constexpr int kMmaWarp = kSW, kPromo0 = kSW + 1;
template <int N>
constexpr int kPW = (N >= 64) ? 16 : 8;
template <int N>
constexpr int kLoaderWarp = kPromo0 + kPW<N>;
template <int N>
constexpr int kZW = (N >= 64) ? 1 : 0;
template <int N>
constexpr int kThreads = 32 * (kLoaderWarp<N> + 1 + kZW<N>);
constexpr int kAcc = 4;          // TMEM chunk accumulators

struct Args {
  PlanDev P;
  const float* tab;          // tile images of this direction (synthesis or analysis)
  const long long* seg;      // [2*nm+1] first table row of segment (im, parity); rows hold npp pairs
  int npp;
  // live-chunk masks of the tile list's entries ([entry][parity]; bit c: chunk c's A image
  // has a nonzero value; chunks from 64 on always run), or null (every chunk runs)
  const unsigned long long* tmask;
  const float2* cin;         // synthesis: coefficients (input of the B packing)
  float* bimg;               // B tile images: synthesis f16 hi/lo pairs written by the packing,
                             //   analysis FP32 written by the FFT (converted in shared memory)
  float* bsc;                // synthesis: factor 2^-(e + s) of each (segment, B row) undoing the
                             //   f16 scaling ([2 nm][2 nfp])
  float2* Wout;              // synthesis: Fourier buffer
  float2* cout;              // analysis: coefficients
  long long ld_k;            // coefficient field stride (complex elements)
  const double* sc;          // normalization scale table (dense) or null
  int sc_mode;               // 0 none, 1 multiply, 2 divide
  float mf0, mf1;
  int nf, lend, lcap;
  const int2* tiles;         // tiles (im, p0) of the synthesis, (im, j0) of the analysis
  int* err;
  int cpacked;               // coefficients in the packed LM layout (field stride ld_k = nlm)
  unsigned long long wait_ns;  // limit of every bounded mbarrier wait (kWaitNs unless a test shortens it)
  int skip_chunk;            // test hook: CTA 0's loader leaves this chunk's copies unissued (-1: none)
};

// First coefficient of order m of one field: dense column m, or the order's packed LM block.
__device__ __forceinline__ long long coef_col(const Args& a, int m) {
  return a.cpacked ? lm_base(a.P.lmax, a.P.mres, m) : (long long)m * (a.P.lmax + 1);
}

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
__device__ __forceinline__ void mbar_arrive_cnt(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
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
// Bounded wait: false after a timeout (limit ns) or once another thread of the CTA gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, volatile int* abort_flag,
                                          int* err, unsigned long long limit) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_test(bar, parity)) {
    if (*abort_flag) return false;
    if (gtimer() - t0 > limit) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}
// Bounded wait used after an abort, for this thread's own asynchronous work (bulk copies it
// issued, MMAs it committed) to land before the CTA frees TMEM and exits; it ignores the
// abort flag. false after kWaitNs.
__device__ __forceinline__ bool mbar_wait_drain(unsigned long long* bar, unsigned parity) {
  const unsigned long long t0 = gtimer();
  while (!mbar_test(bar, parity))
    if (gtimer() - t0 > kWaitNs) return false;
  return true;
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
__device__ __forceinline__ unsigned idesc_f16() {
  // F32 accumulate, A/B F16, both K-major, N>>3 at bit 17, M>>4 at bit 24
  return (1u << 4) | ((unsigned)(N >> 3) << 17) | ((unsigned)(kM >> 4) << 24);
}

// A and B from shared memory (K = 16).
__device__ __forceinline__ void mma_f16_ss(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                           unsigned accum) {
  const unsigned z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ unsigned h2_bits(__half2 h) {
  unsigned u;
  memcpy(&u, &h, 4);
  return u;
}

// (a, b) = hi + lo as f16 pairs (a in the low half): hi rounded to nearest, lo the
// remainders (exact in FP32) rounded to nearest.
__device__ __forceinline__ void split_h2(float a, float b, unsigned& hi, unsigned& lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  hi = h2_bits(h);
  lo = h2_bits(__floats2half2_rn(a - hf.x, b - hf.y));
}

// fp16x3: the table holds P * 2^s with s the largest exponent <= 14 such that
// 2^s sqrt(2 (2L + 1) / (4 pi)) <= 2^15, L = lmax + 1. |P_l^m| <= sqrt((2l + 1) / (4 pi)),
// so every scaled value and its f16 hi part stay below 2^15 (f16 maximum 65504) with a
// factor sqrt(2) to spare.
__device__ __forceinline__ int f16_table_exp(int lmax) {
  const long long q = 2LL * (lmax + 1) + 1;
  int s = 14;
  while (s > 0 && (q << (2 * s)) > 6746518852LL) --s;   // floor(2^31 pi)
  return s;
}

__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// NC consecutive TMEM columns of this thread's lane (32x32b shape), completed by the
// wait::ld in the same asm statement so no use of the registers can precede it.
template <int NC>
__device__ __forceinline__ void tmem_ld(unsigned taddr, float* v);
template <>
__device__ __forceinline__ void tmem_ld<8>(unsigned taddr, float* v) {
  unsigned r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
template <>
__device__ __forceinline__ void tmem_ld<16>(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy global -> this CTA's shared memory (no multicast), completing on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
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
  // One stage holds a chunk: kChunk image K-steps of A, then of B (one parity class per
  // CTA), each operand filled by one bulk copy. Image K-steps 2g and 2g + 1 hold the f16
  // hi and lo tiles of f16 K-step g (the analysis converts its FP32 B tiles in place).
  static constexpr int kStageA = kChunk * kTileBytesA;
  static constexpr int kStage = kChunk * (kTileBytesA + kTileB);
  // Ring depth: up to 192 KB of stages per CTA (110 KB for each of the two 16-column CTAs
  // of an SM).
  static constexpr int kSt = ((N == 16) ? 112640 : 196608) / kStage < 14 ? ((N == 16) ? 112640 : 196608) / kStage : 14;
  static constexpr int kLd = 2 * kSt;   // copy barriers: chunk gc's copies complete on ldfull[gc % kLd]
  static constexpr int kFull = 16;   // per-chunk conversion barriers (analysis)
  static constexpr int kRel = 16;    // chunk-release barriers
  static constexpr int kBar = kSt * kStage;
  // barriers: full[kFull], ldfull[kLd], ldb[kLd], rel[kRel], acce[kAcc]; then TMEM slot,
  // abort flag, then the FP32 column scales of the last kScR chunks
  static constexpr int kScOff = (kBar + (kFull + 2 * kLd + kRel + kAcc) * 8 + 16 + 15) & ~15;
  static constexpr int kBytes = kScOff + kScR * N * 4;
  // grouped kernels only: a ring of kQ claimed tile indices with its full/empty barriers
  static constexpr int kQ = 8;
  static constexpr int kQOff = (kBytes + 15) & ~15;
  static constexpr int kBytesQ = kQOff + kQ * (8 + 8 + 4);
  // TMEM: chunk accumulator b at columns [b N, (b + 1) N), b < kAcc
  static constexpr int kTmemNeed = kAcc * N;
  static constexpr int kTmemCols = kTmemNeed <= 32 ? 32 : kTmemNeed <= 64 ? 64 : kTmemNeed <= 128 ? 128
                                   : kTmemNeed <= 256 ? 256 : 512;
  static_assert(kTmemNeed <= 512, "TMEM columns");
  static_assert(kSt <= kRel, "release barriers");
  // a phase of full, rel or the scale ring is reused only after the promotion of the
  // chunk kFull (kRel, kScR) earlier: the loader runs at most kSt chunks ahead of the
  // MMAs, which run at most kAcc chunks ahead of the promotion
  static_assert(kSt + kAcc <= kScR && kSt + kAcc <= kFull && kSt + kAcc <= kRel, "barrier and scale rings");
};

// Narrow tiles (N = 16: up to 8 fields) leave the tensor core mostly idle, so two CTAs
// share an SM to overlap one tile's load latency with the other's work.
template <int N>
constexpr int kCtasPerSm = (N <= 16) ? 2 : 1;

// Coordinates of one GEMM tile: order index im, first latitude pair p0 (synthesis) or
// first degree index j0 (analysis), parity class par, first field kb.
struct TileCoord {
  int im, p0, j0, par, kb;
};

// Shared-memory barriers of a GEMM CTA (initialised once per CTA).
struct Bars {
  unsigned long long *full, *ldfull, *ldb, *rel, *acce;
  unsigned* tmem_slot;
  volatile int* abort_flag;
  float* fsc;   // analysis: [kScR][N] factors 2^-(row scale + table scale) of chunk gc % kScR
};

template <int N>
__device__ __forceinline__ Bars gemm_bars(unsigned char* sm) {
  using S = Smem<N>;  // barriers follow the stage ring
  Bars B;
  B.full = reinterpret_cast<unsigned long long*>(sm + S::kBar);   // [kFull] chunk gc split (A in TMEM)
  B.ldfull = B.full + S::kFull;   // [kLd] bulk copies of chunk q landed (q % kLd; the analysis: its A)
  B.ldb = B.ldfull + S::kLd;      // [kLd] analysis: the B copy of chunk q landed (q % kLd)
  B.rel = B.ldb + S::kLd;         // [kRel] MMAs of chunk q done (q % kRel)
  B.acce = B.rel + S::kRel;       // [kAcc] TMEM chunk accumulator b drained by the promotion warps
  B.tmem_slot = reinterpret_cast<unsigned*>(B.acce + kAcc);
  B.abort_flag = reinterpret_cast<volatile int*>(B.tmem_slot + 1);
  B.fsc = reinterpret_cast<float*>(sm + S::kScOff);
  return B;
}

// K-steps of a tile (the same count in every role).
template <int MODE>
__device__ __forceinline__ int tile_ksteps(const Args& a, const TileCoord& tc) {
  const int m = tc.im * a.P.mres;
  const int J = (a.lend >= m + tc.par) ? (a.lend - m - tc.par) / 2 + 1 : 0;
  return (MODE == 0) ? (J + kK - 1) / kK : (a.P.npair + kK - 1) / kK;
}

// Barrier setup and TMEM allocation, once per CTA.
template <int N>
__device__ __forceinline__ unsigned gemm_cta_setup(const Bars& B) {
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    // two arrivals per splitter warp and chunk
    for (int s = 0; s < Smem<N>::kFull; ++s) mbar_init(&B.full[s], 2 * kSW);
    for (int s = 0; s < Smem<N>::kLd; ++s) {
      mbar_init(&B.ldfull[s], 1);
      mbar_init(&B.ldb[s], 1);
    }
    for (int s = 0; s < Smem<N>::kRel; ++s) mbar_init(&B.rel[s], 1);
    for (int b = 0; b < kAcc; ++b) mbar_init(&B.acce[b], kPW<N>);   // one arrival per promotion warp
    *B.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(B.tmem_slot)),
                 "r"(Smem<N>::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *B.tmem_slot;
}

template <int N>
__device__ __forceinline__ void gemm_cta_teardown(unsigned tmem) {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if ((threadIdx.x >> 5) == kMmaWarp) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Smem<N>::kTmemCols));
  }
}

// GEMM tiles. MODE 0: synthesis, MODE 1: analysis; N = columns per CTA (2 x fields).
//
// A CTA runs a sequence of tiles (tile i = blockIdx.x, blockIdx.x + gridDim.x, ...), and
// each role walks that sequence on its own: the loader and splitters run ahead into the
// next tile while the promotion warps still drain and store the previous one. c0,
// counted identically by every role, numbers the chunks of the tiles before the current
// one and fixes every stage index, accumulator and barrier phase.
//
// Synchronisation: chunk gc (kChunk image K-steps, fewer at the end of a tile) occupies
// shared-memory stage gc % kSt and TMEM accumulator gc % kAcc. The loader's bulk copies
// complete on ldfull[gc % kLd]; the analysis splitters convert the chunk's B tiles and
// arrive on full[gc % kFull]; the MMA issuer waits for one of the two, issues the chunk's
// 3 (kChunk / 2) MMAs back to back and commits once, to rel[gc % kRel]. Each mbarrier
// wait costs a few hundred cycles even when the phase has completed, so the MMA issuer
// waits on two barriers per chunk only. rel releases the chunk's stage (loader) and
// hands its accumulator to the promotion warps, whose arrival on acce[gc % kAcc] frees
// it for chunk gc + kAcc. The ring sizes keep every waiter from seeing a barrier two
// phases ahead.
struct TileInfo {
  int m, nks, nch;          // K-steps; chunks with a nonzero A block (the ones every role runs)
  int nall;                 // chunks of the tile's K range
  unsigned long long live;  // chunk c < 64 runs iff bit c is set (chunks from 64 on always run)
  long long sg, ln;   // table segment start and rows of (im, par)
  int arows;          // rows of the A tile image (128, fewer in the last analysis tile)
  unsigned bstr;      // bytes from one K-step's B tile to the next in a stage
  unsigned bbytes;    // bytes of one K-step's B tile image (this CTA's fields)
};

__device__ __forceinline__ bool chunk_live(const TileInfo& T, int c) { return c >= 64 || ((T.live >> c) & 1ull); }

template <int MODE>
__device__ __forceinline__ TileInfo tile_info(const Args& a, const TileCoord& tc, unsigned long long live) {
  TileInfo T;
  T.m = tc.im * a.P.mres;
  T.sg = a.seg[2 * tc.im + tc.par];
  T.ln = a.seg[2 * tc.im + tc.par + 1] - T.sg;
  T.nks = tile_ksteps<MODE>(a, tc);
  T.nall = (T.nks + kChunk - 1) / kChunk;
  // A chunk (64 degree rows x 128 pairs in the synthesis, 128 degree rows x 64 pairs in the
  // analysis) whose P image is all zero adds exact zeros: no role runs it.
  T.live = live;
  T.nch = __popcll(T.nall >= 64 ? T.live : T.live & ((1ull << T.nall) - 1)) + max(T.nall - 64, 0);
  T.arows = (MODE == 0) ? kM : min(kM, (int)T.ln - tc.j0);
  // B images of consecutive K-steps are contiguous when all fields fit one 64-field block
  const int nfp = btile_nfp(a.nf);
  T.bstr = (nfp <= 64) ? (unsigned)nfp * 64 : (unsigned)(kM / 2) * 64;
  T.bbytes = (unsigned)min(64, nfp - tc.kb) * 64;
  return T;
}

// One thread fills the shared-memory ring, kSt chunks ahead, with one bulk copy per
// operand and chunk (the A image, f16 hi/lo tile pairs, and the B image: f16 pairs in the
// synthesis, FP32 in the analysis, converted in place by the splitters) when the B images
// of the chunk are contiguous, one per K-step for B otherwise.
template <int MODE, int N>
__device__ __forceinline__ bool loader_tile(const Args& a, const TileCoord& tc, const TileInfo& T, unsigned char* sm,
                                            const Bars& B, unsigned c0, unsigned& issued) {
  using S = Smem<N>;
  const int npair = a.P.npair;
  // A tile images: synthesis [ptile][ks] blocks of 4 KB after the segment start;
  // analysis [jtile][ks] blocks of rows*32 bytes (rows = 128, fewer in the last jtile)
  const float* aseg = a.tab + T.sg * a.npp;
  const float* a0 = (MODE == 0) ? aseg + (long long)(tc.p0 / kM) * (T.ln / kK) * (kM * kK) : aseg + (long long)tc.j0 * a.npp;
  const unsigned abytes = (unsigned)T.arows * kK * 4;
  // B tile images: region rb + ks of nfp x 16 floats, this CTA's block of 64 fields
  const int nfp = btile_nfp(a.nf);
  const long long rb = (MODE == 0) ? T.sg / kK : (long long)(tc.im * 2 + tc.par) * ((npair + kK - 1) / kK);
  const float* bsrc = a.bimg + rb * nfp * 16 + (long long)(tc.kb >> 6) * 1024;
  const unsigned bbytes = T.bbytes;
  const bool bcontig = nfp <= 64;
  int* err = a.err;
  for (int c = 0, q = 0; c < T.nall; ++c) {
    if (!chunk_live(T, c)) continue;
    const unsigned gc = c0 + q++;
    const int st = gc % S::kSt;
    if (gc >= S::kSt) {
      const unsigned q = gc - S::kSt;   // the chunk that last used this stage
      if (!mbar_wait(&B.rel[q % S::kRel], (q / S::kRel) & 1, B.abort_flag, err, a.wait_ns)) return false;
    }
    const int k0 = c * kChunk, nk = min(kChunk, T.nks - k0);
    issued = gc + 1;
    if (blockIdx.x == 0 && (int)gc == a.skip_chunk) continue;   // test hook: this chunk never lands
    unsigned char* sa = sm + (size_t)st * S::kStage;
    unsigned char* sb = sa + S::kStageA;
    unsigned long long* bar = &B.ldfull[gc % S::kLd];
    // the analysis's B copy goes first, on its own barrier, so that the splitters start
    // converting while the A copy is still on its way
    unsigned long long* barb = (MODE == 1) ? &B.ldb[gc % S::kLd] : bar;
    // A tiles come in hi/lo pairs, and so do the synthesis B tiles (the analysis loads its
    // FP32 B tiles and treats a missing last odd one as zeros)
    const int na = (nk + 1) & ~1, nb = (MODE == 0) ? na : nk;
    if (MODE == 1) {
      mbar_expect_tx(barb, (unsigned)nb * bbytes);
      mbar_expect_tx(bar, (unsigned)na * abytes);
    } else {
      mbar_expect_tx(bar, (unsigned)na * abytes + (unsigned)nb * bbytes);
    }
    if (bcontig) {
      bulk_g2s(sb, bsrc + (long long)k0 * nfp * 16, nb * bbytes, barb);
    } else {
      for (int s = 0; s < nb; ++s) bulk_g2s(sb + s * S::kTileB, bsrc + (long long)(k0 + s) * nfp * 16, bbytes, barb);
    }
    bulk_g2s(sa, a0 + (long long)k0 * T.arows * kK, na * abytes, bar);
  }
  return true;
}

// Analysis splitters. The FFT writes B as FP32 tile images; image K-steps 2g and 2g + 1 of
// a chunk form f16 K-step g (K = 16), whose hi tile takes the place of FP32 tile 2g and lo
// tile that of 2g + 1 (the table holds A in that form already). kTpr threads per row, each
// owning whole f16 K-steps g = v, v + kTpr, ...: each row of the chunk is scaled by the power
// of two 2^e that brings its largest magnitude into [2^14, 2^15), split into f16 hi + lo and
// written in place (the same core-matrix byte order: 16-byte rows of 8 f16 values), one
// 16-byte store per FP32 K-step half for hi and one for lo; a thread's writes land only in
// its own two FP32 tiles. A thread with at most 32 values keeps them in registers between
// the row maximum and the conversion; with more it reads them twice (maximum, then
// conversion). Lane layout: the 8 lanes of a quarter warp take 8 consecutive rows of one
// core-matrix group (so every 16-byte access of a quarter warp covers one 128-byte run),
// and a row's kTpr threads sit 8 lanes apart (partners by xor 8, 16). The factor
// 2^-(e + s) that undoes this and the table's scale 2^s goes to the chunk's entry of the
// scale ring. A missing odd K-step at the end of a tile converts as zeros. Below N = 128
// the splitter warps form two groups that take the chunks in turn (group gc % 2), so
// conversions of consecutive chunks overlap; at N = 128 all eight convert every chunk
// (2 threads per row), which halves a conversion's latency. A group reaches chunk gc after
// its own previous chunk, possibly before the loader has refilled the stage; the copy
// barriers form a ring of 2 kSt (a multiple of the group count), so the previous phase of
// chunk gc's barrier belongs to chunk gc - 2 kSt, the group's own, whose copies it saw
// land: its wait cannot match an older phase.
template <int MODE, int N>
__device__ __forceinline__ bool splitter_tile(const Args& a, const TileInfo& T, unsigned char* sm, const Bars& B,
                                                  unsigned c0) {
  using S = Smem<N>;
  // splitter groups: one at N = 128 (2 threads per row, 32 values each, converted in one
  // pass from registers), two otherwise
  constexpr int kSG = (N == 128) ? 1 : 2;
  static_assert(S::kLd % kSG == 0, "copy-barrier ring a multiple of the groups");
  constexpr int kGT = 32 * kSW / kSG;                                    // threads per group
  constexpr int kTpr = (kGT >= 4 * N) ? 4 : (kGT >= N) ? kGT / N : 1;     // threads per B row (1, 2 or 4)
  constexpr int kRpt = (kGT >= N) ? 1 : N / kGT;                         // B rows per thread
  constexpr int kGpt = kChunk / 2 / kTpr;                                // f16 K-steps per thread
  constexpr int kRpw = 8 * (4 / kTpr);                                   // rows per warp
  static_assert((kChunk / 2) % kTpr == 0 && (kTpr == 1 || kTpr == 2 || kTpr == 4), "splitter layout");
  const int tid = threadIdx.x % kGT, grp = threadIdx.x / kGT, lane = tid & 31;
  const int slot = lane >> 3, v = slot % kTpr;
  const int row_w = (tid >> 5) * kRpw + 8 * (slot / kTpr) + (lane & 7);   // this thread's row (first pass)
  const int nrows = min((int)(T.bbytes >> 5), N);     // B rows loaded (2 per field)
  const int sa = f16_table_exp(a.P.lmax);
  for (int c = 0, q = 0; c < T.nall; ++c) {
    if (!chunk_live(T, c)) continue;
    const unsigned gc = c0 + q++;
    if ((int)(gc % kSG) != grp) continue;
    const int nk = min(kChunk, T.nks - c * kChunk), nk2 = (nk + 1) >> 1;
    const bool ok = mbar_wait(&B.ldb[gc % S::kLd], (gc / S::kLd) & 1, B.abort_flag, a.err, a.wait_ns);
    if (!__all_sync(0xffffffffu, ok)) return false;
    unsigned char* Bs = sm + (size_t)(gc % S::kSt) * S::kStage + S::kStageA;
#pragma unroll
    for (int ri = 0; ri < kRpt; ++ri) {
      const int r = row_w + ri * (kGT / kTpr);
      const bool rowok = r < nrows;
      int e;
      if constexpr (kGpt * 16 <= 32) {
        // one pass: the thread's values (kGpt f16 K-steps, both FP32 tiles 2g, 2g + 1, two
        // 16-byte halves each) stay in registers between the row maximum and the conversion
        float4 x[kGpt][4];
        unsigned mx = 0;
#pragma unroll
        for (int j = 0; j < kGpt; ++j) {
          const int g = v + j * kTpr;
#pragma unroll
          for (int w = 0; w < 2; ++w) {
            const bool have = rowok && 2 * g + w < nk;   // a missing odd K-step converts as zeros
            const unsigned char* src = Bs + (2 * g + w) * T.bstr + tile_off(r, 0);
            x[j][2 * w] = have ? *reinterpret_cast<const float4*>(src) : make_float4(0.f, 0.f, 0.f, 0.f);
            x[j][2 * w + 1] = have ? *reinterpret_cast<const float4*>(src + 128) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
              const float4 y = x[j][2 * w + hh];
              mx = max(mx, max(max(__float_as_uint(y.x) & 0x7fffffffu, __float_as_uint(y.y) & 0x7fffffffu),
                               max(__float_as_uint(y.z) & 0x7fffffffu, __float_as_uint(y.w) & 0x7fffffffu)));
            }
          }
        }
#pragma unroll
        for (int o = 8; o < 8 * kTpr; o <<= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        e = min(141 - (int)(mx >> 23), 100);
        const float su = __int_as_float((e + 127) << 23);
        if (rowok) {
#pragma unroll
          for (int j = 0; j < kGpt; ++j) {
            const int g = v + j * kTpr;
            if (g < nk2) {
              unsigned char* b0 = Bs + 2 * g * T.bstr + tile_off(r, 0);
#pragma unroll
              for (int w = 0; w < 2; ++w) {
                uint4 hi, lo;
                split_h2(x[j][2 * w].x * su, x[j][2 * w].y * su, hi.x, lo.x);
                split_h2(x[j][2 * w].z * su, x[j][2 * w].w * su, hi.y, lo.y);
                split_h2(x[j][2 * w + 1].x * su, x[j][2 * w + 1].y * su, hi.z, lo.z);
                split_h2(x[j][2 * w + 1].z * su, x[j][2 * w + 1].w * su, hi.w, lo.w);
                *reinterpret_cast<uint4*>(b0 + w * 128) = hi;
                *reinterpret_cast<uint4*>(b0 + T.bstr + w * 128) = lo;
              }
            }
          }
        }
      } else {
        // two passes (more values than registers). pass 1: the row's largest magnitude over the thread's f16 K-steps (FP32 K-steps 2g,
        // 2g + 1 for g = v, v + kTpr, ...), reduced over the row's threads
        unsigned mx = 0;
#pragma unroll
        for (int j = 0; j < kGpt; ++j) {
          const int g = v + j * kTpr;
#pragma unroll
          for (int w = 0; w < 2; ++w) {
            const int st = 2 * g + w;
            if (rowok && st < nk) {
              const unsigned char* src = Bs + st * T.bstr + tile_off(r, 0);
              const float4 x0 = *reinterpret_cast<const float4*>(src);
              const float4 x1 = *reinterpret_cast<const float4*>(src + 128);
              mx = max(mx, max(max(__float_as_uint(x0.x) & 0x7fffffffu, __float_as_uint(x0.y) & 0x7fffffffu),
                               max(__float_as_uint(x0.z) & 0x7fffffffu, __float_as_uint(x0.w) & 0x7fffffffu)));
              mx = max(mx, max(max(__float_as_uint(x1.x) & 0x7fffffffu, __float_as_uint(x1.y) & 0x7fffffffu),
                               max(__float_as_uint(x1.z) & 0x7fffffffu, __float_as_uint(x1.w) & 0x7fffffffu)));
            }
          }
        }
#pragma unroll
        for (int o = 8; o < 8 * kTpr; o <<= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        // max * 2^e in [2^14, 2^15) (e at most 100: rows below 2^-86 keep the f16 subnormal steps)
        e = min(141 - (int)(mx >> 23), 100);
        const float su = __int_as_float((e + 127) << 23);
        // pass 2: each f16 K-step g reads and writes only its own two FP32 tiles 2g, 2g + 1
        // (hi of both into 2g, lo of both into 2g + 1), so it converts in place right after
        // reading them
        if (rowok) {
#pragma unroll
          for (int j = 0; j < kGpt; ++j) {
            const int g = v + j * kTpr;
            if (g < nk2) {
              unsigned char* b0 = Bs + 2 * g * T.bstr + tile_off(r, 0);
              float4 x[4];
#pragma unroll
              for (int w = 0; w < 2; ++w) {
                const bool have = 2 * g + w < nk;   // a missing odd K-step converts as zeros
                const unsigned char* src = b0 + w * T.bstr;
                x[2 * w] = have ? *reinterpret_cast<const float4*>(src) : make_float4(0.f, 0.f, 0.f, 0.f);
                x[2 * w + 1] = have ? *reinterpret_cast<const float4*>(src + 128) : make_float4(0.f, 0.f, 0.f, 0.f);
              }
#pragma unroll
              for (int w = 0; w < 2; ++w) {
                uint4 hi, lo;
                split_h2(x[2 * w].x * su, x[2 * w].y * su, hi.x, lo.x);
                split_h2(x[2 * w].z * su, x[2 * w].w * su, hi.y, lo.y);
                split_h2(x[2 * w + 1].x * su, x[2 * w + 1].y * su, hi.z, lo.z);
                split_h2(x[2 * w + 1].z * su, x[2 * w + 1].w * su, hi.w, lo.w);
                // FP32 K-step 2g + w -> khalf w of the hi tile (2g) and of the lo tile (2g + 1)
                *reinterpret_cast<uint4*>(b0 + w * 128) = hi;
                *reinterpret_cast<uint4*>(b0 + T.bstr + w * 128) = lo;
              }
            }
          }
        }
      }
      if (rowok && v == 0) B.fsc[(gc % kScR) * N + r] = __int_as_float((127 - e - sa) << 23);
    }
    // the chunk's A copy has landed too before the MMAs may run (they wait only on full)
    const bool oka = mbar_wait(&B.ldfull[gc % S::kLd], (gc / S::kLd) & 1, B.abort_flag, a.err, a.wait_ns);
    if (!__all_sync(0xffffffffu, oka)) return false;
    // the B tiles written here are read by the MMAs (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive_cnt(&B.full[gc % S::kFull], 2 * kSG);
  }
  return true;
}

// One thread issues the MMAs, a chunk at a time, and commits once per chunk. It waits for
// the chunk's bulk copies (synthesis) or its B conversion (analysis, which follows them).
template <int MODE, int N>
__device__ __forceinline__ bool mma_tile(const Args& a, const TileInfo& T, unsigned char* sm, const Bars& B,
                                         unsigned tmem, unsigned c0, int& committed) {
  using S = Smem<N>;
  const unsigned idesc = idesc_f16<N>();
  constexpr unsigned long long kStageDesc = S::kStage >> 4;   // descriptor address step per stage
  const unsigned long long a0 = sdesc(sm), b0 = sdesc(sm + S::kStageA);
  const unsigned long long akDesc = ((unsigned)T.arows * kK * 4) >> 4;   // per image K-step: A
  const unsigned long long bkDesc = T.bstr >> 4;                         // and B
  for (int c = 0, q = 0; c < T.nall; ++c) {
    if (!chunk_live(T, c)) continue;
    const unsigned gc = c0 + q++;
    const int bb = gc % kAcc;
    if (gc >= kAcc && !mbar_wait(&B.acce[bb], ((gc / kAcc) - 1) & 1, B.abort_flag, a.err, a.wait_ns)) return false;
    const int k0 = c * kChunk, k1 = min(T.nks, k0 + kChunk);
    const bool ready = (MODE == 0) ? mbar_wait(&B.ldfull[gc % S::kLd], (gc / S::kLd) & 1, B.abort_flag, a.err, a.wait_ns)
                                   : mbar_wait(&B.full[gc % S::kFull], (gc / S::kFull) & 1, B.abort_flag, a.err, a.wait_ns);
    if (!ready) return false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // The accumulator rounds every addition toward zero at its current magnitude, so
    // the small cross terms (hi*lo, lo*hi) of the whole chunk go in first, while the
    // sum is still small, and the hi*hi products last. f16 K-step g: A and B hi in image
    // K-step 2g, lo in 2g + 1.
    const unsigned dH = tmem + bb * N;
    const unsigned long long sc = (unsigned long long)(gc % S::kSt) * kStageDesc;
    const unsigned long long as = a0 + sc, bs = b0 + sc;
    const int nk2 = (k1 - k0 + 1) >> 1;
    for (int g = 0; g < nk2; ++g) {
      const unsigned long long ah = as + 2 * g * akDesc, bh = bs + 2 * g * bkDesc;
      mma_f16_ss(dH, ah, bh + bkDesc, idesc, g == 0 ? 0u : 1u);
      mma_f16_ss(dH, ah + akDesc, bh, idesc, 1u);
    }
    for (int g = 0; g < nk2; ++g) mma_f16_ss(dH, as + 2 * g * akDesc, bs + 2 * g * bkDesc, idesc, 1u);
    mma_commit(&B.rel[gc % S::kRel]);
    committed = (int)gc;
  }
  return true;
}

// The first analysis tile of each order also clears that order's degrees l < m and
// lcap < l <= lmax (dense layout; a packed output is cleared before the call); the two
// parity tiles take half of the fields each. Threads t = t0, t0 + nt, ... of the clearing role.
template <int N>
__device__ __forceinline__ void clear_tile(const Args& a, const TileCoord& tc, int t0, int nt) {
  if (tc.j0 != 0 || a.cpacked) return;
  const PlanDev& P = a.P;
  const int m = tc.im * P.mres, kb = tc.kb, par = tc.par;
  const int nfl = min(N / 2, a.nf - kb), hf = (nfl + 1) / 2;
  const int f0 = par ? hf : 0, f1 = par ? nfl : hf;
  const int lcap = a.lcap, ntail = P.lmax - lcap, per = m + ntail;
  const long long ld = a.ld_k;
  float2* col0 = a.cout + (long long)m * (P.lmax + 1);
  for (int fi = f0; fi < f1; ++fi) {
    float2* col = col0 + (long long)(kb + fi) * ld;
    for (int r = t0; r < per; r += nt) col[r < m ? r : lcap + 1 + (r - m)] = make_float2(0.f, 0.f);
  }
}

// Promotion warps: drain each chunk into round-to-nearest FP32 sums, then store the tile
// (the analysis also clears l < m and l > lcap in the first tile of an order). The
// analysis undoes its per-chunk B scales chunk by chunk; the synthesis sums in units of
// its per-(segment, row) scales and multiplies once, at the store.
template <int MODE, int N>
__device__ __forceinline__ bool promo_tile(const Args& a, const TileCoord& tc, const TileInfo& T, const Bars& B,
                                           unsigned tmem, unsigned c0) {
  using S = Smem<N>;
  const PlanDev& P = a.P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3;                        // TMEM lane quadrant this warp may access
  const int h = (warp - kPromo0) >> 2;           // column group of kCols columns
  const int row = 32 * q + lane;
  const unsigned lane_base = (unsigned)(32 * q) << 16;
  constexpr int kCols = N / (kPW<N> / 4);          // columns of this thread's TMEM lane
  constexpr int kLd = (kCols < 16) ? kCols : 16;  // columns per TMEM load
  float acc[kCols];
#pragma unroll
  for (int i = 0; i < kCols; ++i) acc[i] = 0.f;
  bool ok = true;
  for (int c = 0; c < T.nch; ++c) {
    const unsigned gc = c0 + c;
    const int bb = gc % kAcc;
    // analysis: the chunk's column scales, written by the splitters before they arrived
    // on full (complete long before the chunk's MMAs are)
    if (MODE == 1 && ok) ok = mbar_wait(&B.full[gc % S::kFull], (gc / S::kFull) & 1, B.abort_flag, a.err, a.wait_ns);
    if (ok) ok = mbar_wait(&B.rel[gc % S::kRel], (gc / S::kRel) & 1, B.abort_flag, a.err, a.wait_ns);
    ok = __all_sync(0xffffffffu, ok);   // warp-uniform: the TMEM loads are warp-collective
    if (!ok) return false;              // the chunk's MMAs may not have run: leave TMEM alone
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned dH = tmem + lane_base + bb * N + h * kCols;
    const float4* fs = reinterpret_cast<const float4*>(B.fsc + (gc % kScR) * N + h * kCols);
#pragma unroll
    for (int i = 0; i < kCols; i += kLd) {
      float v[kLd];
      tmem_ld<kLd>(dH + i, v);
      if constexpr (MODE == 1) {
#pragma unroll
        for (int u = 0; u < kLd; u += 4) {
          const float4 f = fs[(i + u) >> 2];   // exact powers of two: fma rounds once, like the add
          acc[i + u] = fmaf(v[u], f.x, acc[i + u]);
          acc[i + u + 1] = fmaf(v[u + 1], f.y, acc[i + u + 1]);
          acc[i + u + 2] = fmaf(v[u + 2], f.z, acc[i + u + 2]);
          acc[i + u + 3] = fmaf(v[u + 3], f.w, acc[i + u + 3]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < kLd; ++u) acc[i + u] += v[u];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(&B.acce[bb]);
  }
  // Every Args field and the scale factor are read before the first store: the stores
  // go through generic pointers, after which the compiler would reload them.
  const int npair = P.npair, im = tc.im, par = tc.par, m = T.m, kb = tc.kb;
  const int nf = a.nf, kf0 = kb + h * (kCols / 2);
  const int nq = min(kCols / 2, nf - kf0);
  if (MODE == 0) {
    const int pr = tc.p0 + row;
    if (pr < npair) {
      const size_t fstride = (size_t)P.nm * 2 * npair;
      const float2* fsc = reinterpret_cast<const float2*>(a.bsc + (2 * im + par) * 2 * btile_nfp(nf)) + kf0;
      float2* w = a.Wout + (((size_t)kf0 * P.nm + im) * 2 + par) * npair + pr;
#pragma unroll
      for (int qq = 0; qq < kCols / 2; ++qq)
        if (qq < nq) {
          const float2 f = fsc[qq];
          w[qq * fstride] = make_float2(acc[2 * qq] * f.x, acc[2 * qq + 1] * f.y);
        }
    }
  } else {
    const int l = m + 2 * (tc.j0 + row) + par;
    if (l <= a.lcap) {
      const float s = coef_factor(a, l, m);
      const long long ld = a.ld_k;
      float2* c = a.cout + (long long)kf0 * ld + coef_col(a, m) + l;
#pragma unroll
      for (int qq = 0; qq < kCols / 2; ++qq)
        if (qq < nq) c[qq * ld] = make_float2(acc[2 * qq] * s, acc[2 * qq + 1] * s);
    }
  }
  if (MODE == 1 && kZW<N> == 0) clear_tile<N>(a, tc, tid - kPromo0 * 32, 32 * kPW<N>);
  return true;
}

// Tile-index ring of the grouped kernels. The loader thread claims tile indices from the
// launch's device counter (atomicAdd: the list is sorted by decreasing cost, so the CTAs
// take the longest remaining tile whenever they have room) and publishes each in slot
// t % kQ of the ring, -1 once the list is exhausted; the other roles read the slots in the
// same order. full[s]: one arrival (the loader's, after writing the index); empty[s]: one
// arrival per consumer (each splitter and promotion warp and the MMA thread) after reading.
struct TileQueue {
  unsigned long long *full, *empty;
  volatile int* ids;
};
template <int N>
__device__ __forceinline__ TileQueue tile_queue(unsigned char* sm) {
  using S = Smem<N>;
  TileQueue Q;
  Q.full = reinterpret_cast<unsigned long long*>(sm + S::kQOff);
  Q.empty = Q.full + S::kQ;
  Q.ids = reinterpret_cast<volatile int*>(Q.empty + S::kQ);
  return Q;
}
template <int MODE, int N>
constexpr unsigned kQueueConsumers = (MODE == 1 ? kSW + kZW<N> : 0) + 1 + kPW<N>;

// Runs the tiles of src (args(i), coord(i), n): i = blockIdx.x, blockIdx.x + gridDim.x, ...
// for a static source; for a dynamic one (Src::kDynamic, the grouped kernels) the tiles
// the loader claims from src.queue, in claim order.
template <int MODE, int N, class Src>
__device__ __forceinline__ void gemm_tiles(const Src& src, unsigned char* sm, const Bars& B, unsigned tmem) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the synthesis B images arrive converted: its splitter warps have no work
  const bool loader = (warp == kLoaderWarp<N> && lane == 0), splitter = (MODE == 1 && warp < kSW),
             mma = (warp == kMmaWarp && lane == 0), promo = (warp >= kPromo0 && warp < kPromo0 + kPW<N>),
             clear = (MODE == 1 && kZW<N> == 1 && warp == kLoaderWarp<N> + 1);
  const bool role = loader || splitter || mma || promo || clear;
  unsigned c0 = 0;
  unsigned issued = 0;   // loader: chunks 0 .. issued-1 had their copies issued (all but a skipped one)
  int committed = -1;    // MMA issuer: last chunk committed
  int skip = -1;
  int i = blockIdx.x;
  TileCoord tc_next{};
  unsigned long long live_next = ~0ull;
  if constexpr (!Src::kDynamic) {
    if (i < src.n) {
      tc_next = src.coord(i);
      live_next = src.live(i);
    }
  }
  for (unsigned t = 0; role; ++t) {
    if constexpr (Src::kDynamic) {
      using S = Smem<N>;
      const TileQueue Q = tile_queue<N>(sm);
      const unsigned s = t % S::kQ;
      if (loader) {
        if (t >= (unsigned)S::kQ &&
            !mbar_wait(&Q.empty[s], ((t / S::kQ) - 1) & 1, B.abort_flag, src.err(), kWaitNs))
          break;
        const int c = atomicAdd(src.queue, 1);
        i = (c < src.n) ? c : -1;
        Q.ids[s] = i;
        mbar_arrive(&Q.full[s]);
      } else {
        bool ok = mbar_wait(&Q.full[s], (t / S::kQ) & 1, B.abort_flag, src.err(), kWaitNs);
        if (!mma) ok = __all_sync(0xffffffffu, ok);   // splitter and promotion warps: warp-uniform
        if (!ok) break;
        i = Q.ids[s];
        if (!mma) __syncwarp();
        if (mma || lane == 0) mbar_arrive(&Q.empty[s]);
      }
      if (i < 0) break;
    } else {
      if (i >= src.n) break;
    }
    const Args& a = src.args(i);
    TileCoord tc;
    unsigned long long live = ~0ull;
    if constexpr (!Src::kDynamic) {
      // this tile's list entry and mask were loaded one tile ahead; start the next tile's
      // loads now, so no role waits for them at a tile boundary
      tc = tc_next;
      live = live_next;
      const int in = i + (int)gridDim.x;
      if (in < src.n) {
        tc_next = src.coord(in);
        live_next = src.live(in);
      }
    } else {
      tc = src.coord(i);
      live = src.live(i);
    }
    const TileInfo T = tile_info<MODE>(a, tc, live);
    if (blockIdx.x == 0) skip = a.skip_chunk;
    bool ok;
    if (loader)
      ok = loader_tile<MODE, N>(a, tc, T, sm, B, c0, issued);
    else if (splitter)
      ok = splitter_tile<MODE, N>(a, T, sm, B, c0);
    else if (mma)
      ok = mma_tile<MODE, N>(a, T, sm, B, tmem, c0, committed);
    else if (clear)
      clear_tile<N>(a, tc, lane, 32), ok = true;
    else
      ok = promo_tile<MODE, N>(a, tc, T, B, tmem, c0);
    if (!ok) break;
    if (promo) src.tile_done(i);
    c0 += T.nch;
    if constexpr (!Src::kDynamic) i += gridDim.x;
  }
  // Every thread of the CTA: after this barrier the abort flag is final.
  __syncthreads();
  if (!*B.abort_flag) return;
  // After an abort nothing of this CTA's may still run asynchronously when it frees TMEM
  // and exits. The loader's copies in flight are among its last kSt chunks (it issues
  // chunk gc only after chunk gc - kSt was consumed), each completing on its own copy
  // barrier (a ring of 2 kSt); the MMA issuer's last commit completes after all its MMAs.
  using S = Smem<N>;
  if (loader) {
    for (unsigned gc = issued > (unsigned)S::kSt ? issued - S::kSt : 0u; gc < issued; ++gc)
      if ((int)gc != skip) {
        mbar_wait_drain(&B.ldfull[gc % S::kLd], (gc / S::kLd) & 1);
        if (MODE == 1) mbar_wait_drain(&B.ldb[gc % S::kLd], (gc / S::kLd) & 1);
      }
  } else if (mma && committed >= 0) {
    mbar_wait_drain(&B.rel[committed % S::kRel], (committed / S::kRel) & 1);
  }
}

// One coefficient of the synthesis B images: a_lm times the per-(l, m) factors, zero
// beyond lend.
__device__ __forceinline__ float2 pack_value(const Args& a, const float2* c, int l, int m, bool scaled) {
  float2 v = make_float2(0.f, 0.f);
  if (l <= a.lend) {
    v = c[l];
    if (scaled) {
      const float sc = coef_factor(a, l, m);
      v.x *= sc;
      v.y *= sc;
    }
  }
  return v;
}

// Synthesis B tile images of order im, fields k0..k0+3 (one 8-row core-matrix group; rows
// of fields >= nf are written as zeros), as f16 hi/lo pairs; one block of kPackThreads
// threads. Rows are the degrees l = m + par + 2j of one parity; degree row j lies in f16
// K-step j/16 of its segment, whose hi tile is image region seg(im, par)/8 + 2 (j/16) and lo
// tile the region after it (element k16 = j % 16 of a row at byte tile_off(row, k16 / 8) +
// 2 (k16 % 8)). Each (field, parity, re|im) row is scaled by the power of two 2^e that
// brings its largest magnitude into [2^14, 2^15), and bsc receives 2^-(e + s), s the
// table's exponent. Unit b = 16 consecutive degrees l = m + 16 b + q, i.e. degrees
// j = 8b..8b+7 of each parity. 64 threads per field stage 64 units of its coefficient
// column in shared memory (coalesced loads) and find the row maxima; then each thread
// converts one (unit, parity, row) run of 8 values, so that 8 consecutive lanes store the
// 8 rows' 16-byte runs as one 128-byte line (hi, then lo). Orders longer than one staging
// pass are read twice (maximum pass, store pass). Every row of the segment is written, zero
// beyond lend, so the last K-steps of each segment read zeros. All threads of the block call
// it (it synchronises them).
constexpr int kPackFields = 4;
constexpr int kPackThreads = 64 * kPackFields;
constexpr int kPackRow = 18;                        // float2 per staged unit: 16 values + skew
constexpr int kPackField = 64 * kPackRow + 2;       // float2 per field buffer (+16 bytes of skew)
__device__ __forceinline__ void pack_stage(const Args& a, const float2* c, int m, int b0, int nb, bool scaled,
                                           float2* fb) {
  for (int i = threadIdx.x & 63; i < 64 * 16; i += 64) {
    const int b = b0 + i / 16;
    fb[(i / 16) * kPackRow + i % 16] =
        (c != nullptr && b < nb) ? pack_value(a, c, m + 16 * b0 + i, m, scaled) : make_float2(0.f, 0.f);
  }
}
__device__ __forceinline__ void pack_fields(const Args& a, int im, int k0) {
  __shared__ __align__(16) float2 buf[kPackFields * kPackField];
  __shared__ unsigned smx[kPackFields][2][4];   // [field][warp of the field][row (par, re|im)]
  __shared__ float ssu[kPackFields][4];         // scale 2^e of each (field, par, re|im) row
  const PlanDev& P = a.P;
  const int t = threadIdx.x, fi = t >> 6, tt = t & 63, lane = t & 31;
  const int m = im * P.mres;
  const int nfp = btile_nfp(a.nf);
  const int k = k0 + fi;
  const float2* c = (k < a.nf) ? a.cin + (long long)k * a.ld_k + coef_col(a, m) : nullptr;
  const bool scaled = a.sc_mode || a.mf0 != 1.f || a.mf1 != 1.f;
  const long long sg0 = a.seg[2 * im], sg1 = a.seg[2 * im + 1];
  const int R0 = (int)(sg1 - sg0), R1 = (int)(a.seg[2 * im + 2] - sg1);
  const int nb = R0 / 8;   // units; R1 <= R0
  const int npass = (nb + 63) / 64;
  float2* fb = buf + fi * kPackField;
  unsigned mx[4] = {0u, 0u, 0u, 0u};
  for (int ps = 0; ps < npass; ++ps) {
    if (ps > 0) __syncthreads();
    pack_stage(a, c, m, ps * 64, nb, scaled, fb);
    __syncthreads();
    const float4* u = reinterpret_cast<const float4*>(fb + tt * kPackRow);
#pragma unroll
    for (int q = 0; q < 8; ++q) {   // float4 q = degrees 2q (even parity) and 2q + 1
      const float4 v = u[q];
      mx[0] = max(mx[0], __float_as_uint(v.x) & 0x7fffffffu);
      mx[1] = max(mx[1], __float_as_uint(v.y) & 0x7fffffffu);
      mx[2] = max(mx[2], __float_as_uint(v.z) & 0x7fffffffu);
      mx[3] = max(mx[3], __float_as_uint(v.w) & 0x7fffffffu);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx[r] = max(mx[r], __shfl_xor_sync(0xffffffffu, mx[r], o));
    if (lane == 0) smx[fi][tt >> 5][r] = mx[r];
  }
  __syncthreads();
  if (tt < 4) {
    const int r = tt;
    const unsigned v = max(smx[fi][0][r], smx[fi][1][r]);
    // max 2^e in [2^14, 2^15) (e at most 100: rows below 2^-86 keep the f16 subnormal steps)
    const int e = min(141 - (int)(v >> 23), 100);
    ssu[fi][r] = __int_as_float((e + 127) << 23);
    if (k < a.nf)
      a.bsc[(2 * im + (r >> 1)) * 2 * nfp + 2 * k + (r & 1)] =
          __int_as_float((127 - e - f16_table_exp(P.lmax)) << 23);
  }
  __syncthreads();
  const long long lo = (long long)nfp * 64;   // bytes from a hi tile to its lo tile
  const int row0 = 2 * (k0 & 63);             // first image row of the group
  for (int ps = 0; ps < npass; ++ps) {
    if (npass > 1) {   // the last staged pass is still in shared memory when npass == 1
      __syncthreads();
      pack_stage(a, c, m, ps * 64, nb, scaled, fb);
      __syncthreads();
    }
    // item = (unit bl of the pass, parity, row rho): 8 consecutive lanes take the 8 rows
    for (int idx = t; idx < 64 * 2 * 8; idx += kPackThreads) {
      const int rho = idx & 7, par = (idx >> 3) & 1, bl = idx >> 4;
      const int b = ps * 64 + bl;
      if (b >= nb || 8 * b >= (par ? R1 : R0)) continue;
      const int f = rho >> 1, ri = rho & 1;
      const float* z = reinterpret_cast<const float*>(buf + f * kPackField + bl * kPackRow) + 2 * par + ri;
      const float su = ssu[f][2 * par + ri];
      uint4 h, l;
      split_h2(z[0] * su, z[4] * su, h.x, l.x);
      split_h2(z[8] * su, z[12] * su, h.y, l.y);
      split_h2(z[16] * su, z[20] * su, h.z, l.z);
      split_h2(z[24] * su, z[28] * su, h.w, l.w);
      unsigned char* d = reinterpret_cast<unsigned char*>(a.bimg + ((par ? sg1 : sg0) / kK + 2 * (b / 2)) * nfp * 16 +
                                                          (long long)(k0 >> 6) * 1024) +
                         tile_off(row0 + rho, b & 1);
      *reinterpret_cast<uint4*>(d) = h;
      *reinterpret_cast<uint4*>(d + lo) = l;
    }
  }
  __syncthreads();   // buf, smx and ssu are reused by the next call
}

// blockIdx.x = order, blockIdx.y = group of kPackFields fields.
__global__ void __launch_bounds__(kPackThreads) mixed_pack_kernel(const __grid_constant__ Args a) {
  pack_fields(a, blockIdx.x, blockIdx.y * kPackFields);
}

// The same images for one field k (the grouped transforms' packing: members of 1..8
// fields, where 4-field blocks would mostly write padding rows); one block of kPack1Threads
// threads. Rows are the degrees l = m + par + 2j of one parity; degree row j
// lies in f16 K-step j/16 of its segment, whose hi tile is image region seg(im, par)/8 +
// 2 (j/16) and lo tile the region after it (element k16 = j % 16 of a row at byte
// tile_off(row, k16 / 8) + 2 (k16 % 8)). Each (parity, re|im) row is scaled by the power of
// two 2^e that brings its largest magnitude into [2^14, 2^15), and bsc receives
// 2^-(e + s), s the table's exponent. Thread work unit b = 16 consecutive degrees
// l = m + 16 b + q: the 8 degrees j = 8b..8b+7 of each parity, i.e. one 16-byte run of each
// of its 4 rows, stored hi and lo with one 16-byte store each. The block stages
// kPack1Threads units at a time in shared memory (coalesced loads of the coefficient
// column; each thread then reads its unit as 16-byte words); orders longer than one
// staging pass are read twice (maximum pass, store pass). Every row of the segment is
// written, zero beyond lend, so the last K-steps of each segment read zeros. All threads
// of the block call it (it synchronises them).
constexpr int kPack1Threads = 64;
__device__ __forceinline__ void pack_stage1(const Args& a, const float2* c, int m, int b0, int nb, bool scaled,
                                           float2 (*buf)[kPackRow]) {
  for (int i = threadIdx.x; i < kPack1Threads * 16; i += kPack1Threads) {
    const int b = b0 + i / 16;
    buf[i / 16][i % 16] = (b < nb) ? pack_value(a, c, m + 16 * b0 + i, m, scaled) : make_float2(0.f, 0.f);
  }
}
__device__ __forceinline__ void pack_field1(const Args& a, int im, int k) {
  __shared__ __align__(16) float2 buf[kPack1Threads][kPackRow];
  __shared__ unsigned smx[kPack1Threads / 32][4];
  const PlanDev& P = a.P;
  const int t = threadIdx.x, lane = t & 31;
  const int m = im * P.mres;
  const int nfp = btile_nfp(a.nf), fl = k & 63;
  const float2* c = a.cin + (long long)k * a.ld_k + coef_col(a, m);
  const bool scaled = a.sc_mode || a.mf0 != 1.f || a.mf1 != 1.f;
  const long long sg[2] = {a.seg[2 * im], a.seg[2 * im + 1]};
  const int R[2] = {(int)(sg[1] - sg[0]), (int)(a.seg[2 * im + 2] - sg[1])};
  const int nb = R[0] / 8;   // units; R[1] <= R[0]
  const int npass = (nb + kPack1Threads - 1) / kPack1Threads;
  unsigned mx[4] = {0u, 0u, 0u, 0u};   // rows (par, re|im)
  for (int ps = 0; ps < npass; ++ps) {
    if (ps > 0) __syncthreads();
    pack_stage1(a, c, m, ps * kPack1Threads, nb, scaled, buf);
    __syncthreads();
    const float4* u = reinterpret_cast<const float4*>(buf[t]);
#pragma unroll
    for (int q = 0; q < 8; ++q) {   // float4 q = degrees 2q (even parity) and 2q + 1
      const float4 v = u[q];
      mx[0] = max(mx[0], __float_as_uint(v.x) & 0x7fffffffu);
      mx[1] = max(mx[1], __float_as_uint(v.y) & 0x7fffffffu);
      mx[2] = max(mx[2], __float_as_uint(v.z) & 0x7fffffffu);
      mx[3] = max(mx[3], __float_as_uint(v.w) & 0x7fffffffu);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx[r] = max(mx[r], __shfl_xor_sync(0xffffffffu, mx[r], o));
    if (lane == 0) smx[t >> 5][r] = mx[r];
  }
  __syncthreads();
  float su[4];
  const int sa = f16_table_exp(P.lmax);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    unsigned v = 0u;
#pragma unroll
    for (int w = 0; w < kPack1Threads / 32; ++w) v = max(v, smx[w][r]);
    // max 2^e in [2^14, 2^15) (e at most 100: rows below 2^-86 keep the f16 subnormal steps)
    const int e = min(141 - (int)(v >> 23), 100);
    su[r] = __int_as_float((e + 127) << 23);
    if (t == 0) a.bsc[(2 * im + (r >> 1)) * 2 * nfp + 2 * k + (r & 1)] = __int_as_float((127 - e - sa) << 23);
  }
  const long long lo = (long long)nfp * 64;   // bytes from a hi tile to its lo tile
  for (int ps = 0; ps < npass; ++ps) {
    if (npass > 1) {   // the last staged pass is still in shared memory when npass == 1
      __syncthreads();
      pack_stage1(a, c, m, ps * kPack1Threads, nb, scaled, buf);
      __syncthreads();
    }
    const int b = ps * kPack1Threads + t;
    if (b >= nb) continue;
    const float4* u = reinterpret_cast<const float4*>(buf[t]);
    float y[4][8];   // rows (par, re|im) x j % 8
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 v = u[q];
      y[0][q] = v.x * su[0];
      y[1][q] = v.y * su[1];
      y[2][q] = v.z * su[2];
      y[3][q] = v.w * su[3];
    }
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      if (8 * b >= R[par]) continue;
      unsigned char* base = reinterpret_cast<unsigned char*>(a.bimg + (sg[par] / kK + 2 * (b / 2)) * nfp * 16 +
                                                             (long long)(k >> 6) * 1024);
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const float* z = y[2 * par + ri];
        uint4 h, l;
        split_h2(z[0], z[1], h.x, l.x);
        split_h2(z[2], z[3], h.y, l.y);
        split_h2(z[4], z[5], h.z, l.z);
        split_h2(z[6], z[7], h.w, l.w);
        unsigned char* d = base + tile_off(2 * fl + ri, b & 1);
        *reinterpret_cast<uint4*>(d) = h;
        *reinterpret_cast<uint4*>(d + lo) = l;
      }
    }
  }
  __syncthreads();   // buf and smx are reused by the next call
}

// Persistent packing for grouped transforms: item = (transform, order), all its fields,
// claimed in list order from the device counter *queue (zero at launch).
__global__ void __launch_bounds__(kPack1Threads) mixed_pack_group_kernel(const Args* __restrict__ targs,
                                                                       const int2* __restrict__ items, int nitems,
                                                                       int* __restrict__ queue) {
  __shared__ Args sa;
  __shared__ int s_item, s_order;
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = atomicAdd(queue, 1);
      s_item = i;
      if (i < nitems) {
        const int2 it = items[i];
        s_order = it.y;
        sa = targs[it.x];
      }
    }
    __syncthreads();
    const int item = s_item, order = s_order, nf = sa.nf;
    __syncthreads();   // everyone holds the item before thread 0 may claim the next one
    if (item >= nitems) break;
    for (int k = 0; k < nf; ++k) pack_field1(sa, order, k);   // ends with __syncthreads
  }
}

// Tiles of one transform: tile i = (list index * nz + z) * 2 + par over the tile list
// (synthesis (im, p0), analysis (im, j0), in order of decreasing work), z = block of N/2
// fields.
template <int MODE, int N>
struct SingleSrc {
  static constexpr bool kDynamic = false;
  const Args& a;
  int n, nz;
  __device__ const Args& args(int) const { return a; }
  __device__ void tile_done(int) const {}
  __device__ unsigned long long live(int i) const { return a.tmask ? a.tmask[((i >> 1) / nz) * 2 + (i & 1)] : ~0ull; }
  __device__ TileCoord coord(int i) const {
    TileCoord tc;
    tc.par = i & 1;
    int r = i >> 1;
    tc.kb = (r % nz) * (N / 2);
    const int2 t = a.tiles[r / nz];   // (im, first pair) or (im, first degree row)
    tc.im = t.x;
    tc.p0 = (MODE == 0) ? t.y : 0;
    tc.j0 = (MODE == 0) ? 0 : t.y;
    return tc;
  }
};

// ntiles: tile list length * nz * 2.
template <int MODE, int N>
__global__ void __launch_bounds__(kThreads<N>, kCtasPerSm<N>) mixed_gemm_kernel(const __grid_constant__ Args a, int ntiles,
                                                                             int nz) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const Bars B = gemm_bars<N>(sm);
  const unsigned tmem = gemm_cta_setup<N>(B);
  const SingleSrc<MODE, N> src{a, ntiles, nz};
  gemm_tiles<MODE, N>(src, sm, B, tmem);
  gemm_cta_teardown<N>(tmem);
}

// Tiles of many independent transforms: item = (transform, im, p0 or j0, parity), list
// sorted by decreasing cost and claimed through the device counter queue (zero at launch).
// done[t] receives the %globaltimer value at which the last tile of transform t was
// stored (the maximum over its tiles).
template <int MODE>
struct GroupSrc {
  static constexpr bool kDynamic = true;
  const Args* targs;
  const int4* items;
  const unsigned long long* masks;   // live-chunk mask of each item, or null
  int n;
  unsigned long long* done;
  int* queue;
  __device__ int* err() const { return targs[0].err; }
  __device__ const Args& args(int i) const { return targs[items[i].x]; }
  __device__ unsigned long long live(int i) const { return masks ? masks[i] : ~0ull; }
  __device__ TileCoord coord(int i) const {
    const int4 it = items[i];
    TileCoord tc;
    tc.im = it.y;
    tc.par = it.w;
    tc.kb = 0;
    tc.p0 = (MODE == 0) ? it.z : 0;
    tc.j0 = (MODE == 0) ? 0 : it.z;
    return tc;
  }
  // called by each promotion warp after its stores of tile i
  __device__ void tile_done(int i) const {
    if (!done) return;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) atomicMax(done + items[i].x, gtimer());
  }
};

// Persistent GEMM over the tiles of many transforms, claimed from the counter *queue.
template <int MODE, int N>
__global__ void __launch_bounds__(kThreads<N>, kCtasPerSm<N>) mixed_gemm_group_kernel(const Args* __restrict__ targs,
                                                                                   const int4* __restrict__ items,
                                                                                   const unsigned long long* __restrict__ masks,
                                                                                   int nitems,
                                                                                   unsigned long long* __restrict__ done,
                                                                                   int* __restrict__ queue) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const Bars B = gemm_bars<N>(sm);
  if (threadIdx.x == 0) {   // made visible by the fence and barrier of gemm_cta_setup
    const TileQueue Q = tile_queue<N>(sm);
    for (int s = 0; s < Smem<N>::kQ; ++s) {
      mbar_init(&Q.full[s], 1);
      mbar_init(&Q.empty[s], kQueueConsumers<MODE, N>);
    }
  }
  const unsigned tmem = gemm_cta_setup<N>(B);
  const GroupSrc<MODE> src{targs, items, masks, nitems, done, queue};
  gemm_tiles<MODE, N>(src, sm, B, tmem);
  gemm_cta_teardown<N>(tmem);
}

// Table: P_l^m(x_pair) as FP32, degree row j = (l-m)/2 of segment (im, (l-m)%2), written
// into both tile images (layout described at the top of this file).
__global__ void mixed_table_kernel(PlanDev P, float* __restrict__ tabS, float* __restrict__ tabA,
                                   const long long* __restrict__ seg, int npp, unsigned char* __restrict__ nzb, int nrb,
                                   int npb) {
  const int pair = blockIdx.x * blockDim.x + threadIdx.x;
  const int im = blockIdx.y;
  if (pair >= P.npair) return;
  const int m = im * P.mres;
  const long long poff = P.off[im];
  const double x = P.x[pair];
  const int l0 = P.l0[(size_t)im * P.npair + pair];
  const double2 r01 = P.r01[(size_t)im * P.npair + pair];
  const int pt = pair / kM, pr = pair % kM;
  const float asc = (float)(1 << f16_table_exp(P.lmax));   // exact scaling
  double ra = 0.0, rb = 0.0;
  unsigned long long nzm[2] = {0ull, 0ull};   // 64-row blocks of each parity with a nonzero value
  unsigned char* nzf = nzb + (long long)(2 * im) * nrb * npb + pair / 64;
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
    const long long sg = seg[2 * im + par];
    const int R = (int)(seg[2 * im + par + 1] - sg);
    const float v = (float)(P.cfac[poff + (l - m)] * r) * asc;
    const int jt = j / kM, rr = j % kM, rows = min(kM, R - jt * kM);
    // f16 hi/lo of P 2^s: image K-step pair (2g, 2g + 1) holds the hi and lo tiles of f16
    // K-step g, element k16 of a row at byte tile_off(row, k16 / 8) + 2 (k16 % 8).
    // synthesis: tile (pt, degree j / 16), row pr; analysis: tile (j / 128, pair / 16) of
    // rows = min(128, R - 128 (j / 128)), row j % 128
    const __half h = __float2half_rn(v), lo = __float2half_rn(v - __half2float(h));
    const int js = j % 16, ps = pair % 16;
    unsigned char* ds = reinterpret_cast<unsigned char*>(tabS + sg * npp) +
                        ((long long)pt * (R / kK) + 2 * (j / 16)) * kTileBytesA + tile_off(pr, js >> 3) + 2 * (js & 7);
    unsigned char* da = reinterpret_cast<unsigned char*>(tabA + sg * npp + (long long)jt * kM * npp) +
                        (long long)(2 * (pair / 16)) * rows * kK * 4 + tile_off(rr, ps >> 3) + 2 * (ps & 7);
    *reinterpret_cast<__half*>(ds) = h;
    *reinterpret_cast<__half*>(ds + kTileBytesA) = lo;
    *reinterpret_cast<__half*>(da) = h;
    *reinterpret_cast<__half*>(da + rows * kK * 4) = lo;
    if ((__half_as_ushort(h) | __half_as_ushort(lo)) & 0x7fffu) {
      const int b = j / 64;
      if (b < 64)
        nzm[par] |= 1ull << b;
      else
        nzf[((long long)par * nrb + b) * npb] = 1;
    }
  }
  for (int par = 0; par < 2; ++par)
    for (unsigned long long bits = nzm[par]; bits; bits &= bits - 1)
      nzf[((long long)par * nrb + __ffsll((long long)bits) - 1) * npb] = 1;
}

// Live-chunk masks from the block flags: synthesis tile (im, par, pair tile pt) chunk c =
// degree rows 64 c.. of pair blocks 2 pt, 2 pt + 1; analysis tile (im, par, degree tile jt)
// chunk c = pairs 64 c.. of row blocks 2 jt, 2 jt + 1. One thread per (segment, tile).
__global__ void mixed_mask_kernel(const unsigned char* __restrict__ nzb, int nseg, int nrb, int npb, int njt,
                                  unsigned long long* __restrict__ mskS, unsigned long long* __restrict__ mskA) {
  const int ntp = npb / 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nseg * (ntp + njt)) return;
  const int sgi = i / (ntp + njt), r = i - sgi * (ntp + njt);
  const unsigned char* f = nzb + (long long)sgi * nrb * npb;
  unsigned long long live = 0ull;
  if (r < ntp) {
    for (int c = 0; c < 64 && c < nrb; ++c)
      if (f[c * npb + 2 * r] | f[c * npb + 2 * r + 1]) live |= 1ull << c;
    mskS[(long long)sgi * ntp + r] = live;
  } else {
    const int jt = r - ntp;
    for (int c = 0; c < 64 && c < npb; ++c)
      if (f[(2 * jt) * npb + c] | f[(2 * jt + 1) * npb + c]) live |= 1ull << c;
    mskA[(long long)sgi * njt + jt] = live;
  }
}

}  // namespace mx

using namespace mx;

// Segment starts of the P table: rows (degrees m+par, m+par+2, .., lrec) of every
// (order, parity), each segment padded to a multiple of kSegRows rows (one f16 K-step of
// 16 degrees). Returns the row count.
static long long table_segments(const shtb_plan* p, std::vector<long long>* seg) {
  const int nm = p->nm, LR = p->lrec;
  if (seg) seg->assign(2 * nm + 1, 0);
  long long rows = 0;
  for (int im = 0; im < nm; ++im) {
    const int m = im * p->mres;
    for (int par = 0; par < 2; ++par) {
      if (seg) (*seg)[2 * im + par] = rows;
      const int cnt = (LR - m - par >= 0) ? (LR - m - par) / 2 + 1 : 0;
      rows += (cnt + kSegRows - 1) / kSegRows * kSegRows;
    }
  }
  if (seg) (*seg)[2 * nm] = rows;
  return rows;
}

static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Synthesis workspace: Fourier buffer [f][nm][2][npair] (float2), then the B tile
// images (table rows x nfp x 2 floats).
static size_t syn_w_bytes(const shtb_plan* p, int nf) { return align256((size_t)nf * p->nm * 2 * p->npair * 8); }
// ... then the per-(segment, row) scales of the images ([2 nm][2 nfp] floats).
static size_t syn_img_only(const shtb_plan* p, int nf) {
  return align256((size_t)table_segments(p, nullptr) * btile_nfp(nf) * 2 * 4);
}
static size_t syn_img_bytes(const shtb_plan* p, int nf) {
  return syn_img_only(p, nf) + align256((size_t)p->nm * 2 * 2 * btile_nfp(nf) * 4);
}

static int ensure_table(const shtb_plan* cp, cudaStream_t st) {
  shtb_plan* p = const_cast<shtb_plan*>(cp);
  std::lock_guard<std::mutex> lk(p->tab_mu);
  if (p->d_tab) return SHTB_OK;
  const int nm = p->nm;
  p->npp = (p->npair + kM - 1) / kM * kM;
  const long long rows = table_segments(p, &p->htab_seg);
  const size_t tb = (size_t)rows * p->npp * 4;   // one image
  long long rmax = 0;
  for (int s = 0; s < 2 * nm; ++s) rmax = std::max(rmax, p->htab_seg[s + 1] - p->htab_seg[s]);
  const int njt = (int)((rmax + kM - 1) / kM), nrb = 2 * njt + 1, npb = p->npp / 64;
  const size_t nzbytes = (size_t)2 * nm * nrb * npb;
  const size_t segoff = (2 * tb + 255) / 256 * 256, nzoff = (segoff + (2 * nm + 1) * 8 + 255) / 256 * 256;
  const size_t msoff = (nzoff + nzbytes + 255) / 256 * 256, ntp = p->npp / kM;
  const size_t maoff = msoff + (size_t)2 * nm * ntp * 8, mend = maoff + (size_t)2 * nm * njt * 8;
  void* mem = nullptr;
  cudaError_t e = cudaMalloc(&mem, mend);
  if (e != cudaSuccess) return set_error(SHTB_ERR_OOM, std::string("mixed table: ") + cudaGetErrorString(e));
  float* tab = (float*)mem;
  float* taba = (float*)((char*)mem + tb);
  long long* dseg = (long long*)((char*)mem + segoff);
  unsigned char* dnz = (unsigned char*)mem + nzoff;
  e = cudaMemcpyAsync(dseg, p->htab_seg.data(), (2 * nm + 1) * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tab, 0, 2 * tb, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dnz, 0, nzbytes, st);
  if (e != cudaSuccess) {
    cudaFree(mem);
    return set_error(SHTB_ERR_CUDA, std::string("mixed table init: ") + cudaGetErrorString(e));
  }
  dim3 grid((p->npair + 127) / 128, nm);
  mixed_table_kernel<<<grid, 128, 0, st>>>(p->dev, tab, taba, dseg, p->npp, dnz, nrb, npb);
  count_launch();
  unsigned long long* msk_s = (unsigned long long*)((char*)mem + msoff);
  unsigned long long* msk_a = (unsigned long long*)((char*)mem + maoff);
  const int nmask = 2 * nm * (int)(ntp + njt);
  mixed_mask_kernel<<<(nmask + 127) / 128, 128, 0, st>>>(dnz, 2 * nm, nrb, npb, njt, msk_s, msk_a);
  count_launch();
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(mem);
    return set_error(SHTB_ERR_CUDA, std::string("mixed table kernel: ") + cudaGetErrorString(e));
  }
  p->d_tab = tab;
  p->d_tab_ana = taba;
  p->d_tab_seg = dseg;
  p->hmsk_s.resize((size_t)2 * nm * ntp);
  p->hmsk_a.resize((size_t)2 * nm * njt);
  e = cudaMemcpy(p->hmsk_s.data(), msk_s, p->hmsk_s.size() * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(p->hmsk_a.data(), msk_a, p->hmsk_a.size() * 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaFree(mem);
    return set_error(SHTB_ERR_CUDA, std::string("mixed table masks: ") + cudaGetErrorString(e));
  }
  p->d_tab_msk_s = msk_s;
  p->d_tab_msk_a = msk_a;
  p->tab_njt = njt;
  p->tab_bytes = mend;
  return SHTB_OK;
}

static int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// ntiles tiles per block of N/2 fields; persistent CTAs, at most the resident number.
template <int MODE, int N>
static int launch_gemm(const shtb_plan* p, const Args& a, int ntiles, int nz, cudaStream_t st) {
  auto kern = mixed_gemm_kernel<MODE, N>;
  const int smem = Smem<N>::kBytes;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "mixed smem attr");
  const int total = ntiles * nz;
  const int grid = std::max(1, std::min(total, sm_count() * kCtasPerSm<N>));
  prof_begin(st);
  kern<<<grid, kThreads<N>, smem, st>>>(a, total, nz);
  SHTB_LAUNCHED(MODE == 0 ? "tc gemm synthesis kernel" : "tc gemm analysis kernel");
  return SHTB_OK;
}

// ntiles: tiles per block of fields (tile list length x 2 parities).
template <int MODE>
static int dispatch_gemm(const shtb_plan* p, const Args& a, int nf, int ntiles, cudaStream_t st) {
  if (nf > 32) return launch_gemm<MODE, 128>(p, a, ntiles, (nf + 63) / 64, st);
  if (nf > 16) return launch_gemm<MODE, 64>(p, a, ntiles, 1, st);
  if (nf > 8) return launch_gemm<MODE, 32>(p, a, ntiles, 1, st);
  return launch_gemm<MODE, 16>(p, a, ntiles, 1, st);
}

// Clears whole order columns the analysis GEMM does not visit (m not a multiple of
// mres, or m > min(mmax, lcap)); one block per (m, field).
__global__ void zero_columns_kernel32(PlanDev P, float2* __restrict__ a, long long ld_k, int mlim) {
  const int m = blockIdx.x, k = blockIdx.y;
  if ((m % P.mres) == 0 && m <= mlim) return;
  float2* col = a + (long long)k * ld_k + (long long)m * (P.lmax + 1);
  for (int l = threadIdx.x; l <= P.lmax; l += blockDim.x) col[l] = make_float2(0.f, 0.f);
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
  a.wait_ns = p->dbg_wait_ns ? p->dbg_wait_ns : kWaitNs;
  a.skip_chunk = p->dbg_skip_chunk;
  return a;
}

// GEMM tile list of one direction for truncation degree ltr, built once per (direction, ltr)
// and kept on the plan until it is destroyed, so a list handed to a kernel is never freed
// under it (calls from several host threads share the cache under the plan's table mutex):
// synthesis (im, first pair), analysis (im, first degree row), each entry with the
// live-chunk masks of both parities, ordered by decreasing count of live chunks (the
// persistent CTAs take tiles blockIdx.x, + gridDim.x, ..., so every round holds tiles of
// similar cost).
static int gemm_tiles_list(const shtb_plan* cp, int mode, int ltr, int mlim, cudaStream_t st,
                           shtb_plan::MxTileList* out) {
  shtb_plan* p = const_cast<shtb_plan*>(cp);
  std::lock_guard<std::mutex> lk(p->tab_mu);
  auto it = p->mx_lists[mode].find(ltr);
  if (it != p->mx_lists[mode].end()) {
    *out = it->second;
    return SHTB_OK;
  }
  std::vector<int2> tl;
  std::vector<int> cost;
  std::vector<unsigned long long> msk;   // [entry][parity]
  const int ntp = p->npp / kM, njt = p->tab_njt;
  auto live = [](unsigned long long mk, int nall) {
    return __builtin_popcountll(nall >= 64 ? mk : mk & ((1ull << nall) - 1)) + std::max(nall - 64, 0);
  };
  for (int im = 0; im * p->mres <= mlim; ++im) {
    const int m = im * p->mres;
    if (mode == 0) {
      for (int pt = 0; pt * kM < p->npair; ++pt) {
        int c = 0;
        for (int par = 0; par < 2; ++par) {
          const int J = (ltr >= m + par) ? (ltr - m - par) / 2 + 1 : 0;
          const unsigned long long mk = p->hmsk_s[(size_t)(2 * im + par) * ntp + pt];
          c += live(mk, ((J + kK - 1) / kK + kChunk - 1) / kChunk);
          msk.push_back(mk);
        }
        tl.push_back(make_int2(im, pt * kM));
        cost.push_back(c);
      }
    } else {
      const int JE = (ltr - m) / 2 + 1;
      const int nall = ((p->npair + kK - 1) / kK + kChunk - 1) / kChunk;
      for (int j0 = 0; j0 < JE; j0 += kM) {
        int c = 0;
        for (int par = 0; par < 2; ++par) {
          const unsigned long long mk = p->hmsk_a[(size_t)(2 * im + par) * njt + j0 / kM];
          c += live(mk, nall);
          msk.push_back(mk);
        }
        tl.push_back(make_int2(im, j0));
        cost.push_back(c);
      }
    }
  }
  std::vector<int> ord(tl.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<int2> sorted(tl.size());
  std::vector<unsigned long long> smsk(msk.size());
  for (size_t i = 0; i < ord.size(); ++i) {
    sorted[i] = tl[ord[i]];
    smsk[2 * i] = msk[2 * ord[i]];
    smsk[2 * i + 1] = msk[2 * ord[i] + 1];
  }
  shtb_plan::MxTileList L;
  L.count = (int)sorted.size();
  cudaError_t e = cudaMalloc(&L.tiles, std::max<size_t>(1, sorted.size()) * sizeof(int2));
  if (e == cudaSuccess) e = cudaMalloc(&L.masks, std::max<size_t>(1, smsk.size()) * 8);
  // pageable sources: each copy has read its source when the call returns
  if (e == cudaSuccess && L.count)
    e = cudaMemcpyAsync(L.tiles, sorted.data(), sorted.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && L.count)
    e = cudaMemcpyAsync(L.masks, smsk.data(), smsk.size() * 8, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    if (L.tiles) cudaFree(L.tiles);
    if (L.masks) cudaFree(L.masks);
    return set_error(SHTB_ERR_CUDA, std::string("mixed tiles: ") + cudaGetErrorString(e));
  }
  p->mx_lists[mode][ltr] = L;
  *out = L;
  return SHTB_OK;
}

int mixed_synthesis(const shtb_plan* p, const void* alm, void* f, int nf, int ltr, void* work, cudaStream_t st,
                    int packed) {
  const int mlim = std::min(p->mmax, ltr);
  int rc;
  if (simt_applicable(p, nf)) {   // one or two fields: recurrence on the FP64 pipes, no table
    if ((rc = launch_simt_syn(p, alm, work, nf, ltr, mlim, packed, st))) return rc;
    return launch_fft_syn<float, float>(p, work, (float*)f, nullptr, 1, nf, mlim, p->phi_inv_scale / p->nlon, 0, 0, st);
  }
  if ((rc = ensure_table(p, st))) return rc;
  Args a = base_args(p);
  a.cin = (const float2*)alm;
  if (packed) {
    a.cpacked = 1;
    a.ld_k = lm_count(p->lmax, p->mmax, p->mres);
  }
  a.Wout = (float2*)work;
  a.bimg = (float*)((char*)work + syn_w_bytes(p, nf));
  a.bsc = (float*)((char*)a.bimg + syn_img_only(p, nf));
  a.sc_mode = p->d_scale ? 1 : 0;
  a.nf = nf;
  a.lend = ltr;
  a.lcap = ltr;
  prof_begin(st);
  mixed_pack_kernel<<<dim3(mlim / p->mres + 1, (nf + kPackFields - 1) / kPackFields), kPackThreads, 0, st>>>(a);
  SHTB_LAUNCHED("tc gemm B packing kernel");
  shtb_plan::MxTileList tl;
  if ((rc = gemm_tiles_list(p, 0, ltr, mlim, st, &tl))) return rc;
  a.tiles = tl.tiles;
  a.tmask = tl.masks;
  if ((rc = dispatch_gemm<0>(p, a, nf, 2 * tl.count, st))) return rc;
  return launch_fft_syn<float, float>(p, work, (float*)f, nullptr, 1, nf, mlim, p->phi_inv_scale / p->nlon, 0, 0, st);
}

size_t mixed_workspace_bytes(const shtb_plan* p, int op, int nf) {
  if (op == SHTB_OP_SYNTHESIS) return syn_w_bytes(p, nf) + syn_img_bytes(p, nf);
  return align256(fft_btile_floats(p, nf) * 4);
}

int mixed_analysis(const shtb_plan* p, const void* f, void* alm, int nf, int ltr, void* work, cudaStream_t st,
                   int packed) {
  const int mlim = std::min(p->mmax, ltr);
  int rc;
  if ((rc = ensure_table(p, st))) return rc;
  const long long nlm = lm_count(p->lmax, p->mmax, p->mres);
  if (packed && ltr < p->lmax)   // degrees above ltr are no tile's output
    SHTB_TRY_CUDA(cudaMemsetAsync(alm, 0, (size_t)nlm * nf * sizeof(float2), st), "packed output clear");
  if ((rc = launch_fft_ana<float, float>(p, (const float*)f, nullptr, 1, work, nf, mlim, p->ana_scale, 1, 0, st, 1)))
    return rc;
  // analysis tiles: 128 degrees of each parity per tile
  shtb_plan::MxTileList tl;
  if ((rc = gemm_tiles_list(p, 1, ltr, mlim, st, &tl))) return rc;
  Args a = base_args(p);
  a.tab = p->d_tab_ana;
  a.bimg = (float*)work;
  a.cout = (float2*)alm;
  a.sc_mode = p->d_scale ? 2 : 0;
  a.nf = nf;
  a.lend = ltr;
  a.lcap = ltr;
  a.tiles = tl.tiles;
  a.tmask = tl.masks;
  if (packed) {
    a.cpacked = 1;
    a.ld_k = nlm;
  }
  if ((rc = dispatch_gemm<1>(p, a, nf, 2 * tl.count, st))) return rc;
  if (!packed && (p->mres > 1 || mlim < p->mmax)) {
    dim3 zg(p->mmax + 1, nf);
    prof_begin(st);
    zero_columns_kernel32<<<zg, 256, 0, st>>>(p->dev, (float2*)alm, a.ld_k, mlim);
    SHTB_LAUNCHED("zero fill kernel");
  }
  return SHTB_OK;
}

// ---------------------------------------------------------------- grouped transforms
// Host-side pieces of the persistent grouped GEMMs (uneven batches of transforms with
// up to 8 fields each, N = 16 columns).

int mixed_prepare(const shtb_plan* p, cudaStream_t st) { return ensure_table(p, st); }

size_t mixed_args_bytes() { return sizeof(Args); }

void mixed_fill_args(const shtb_plan* p, int mode, const void* in, void* out, int nf, void* host_args) {
  Args a = base_args(p);
  if (mode == 0) {
    a.cin = (const float2*)in;
    a.Wout = (float2*)out;
    a.bimg = (float*)((char*)out + syn_w_bytes(p, nf));
    a.bsc = (float*)((char*)a.bimg + syn_img_only(p, nf));
    a.sc_mode = p->d_scale ? 1 : 0;
  } else {
    a.tab = p->d_tab_ana;
    a.bimg = (float*)const_cast<void*>(in);
    a.cout = (float2*)out;
    a.sc_mode = p->d_scale ? 2 : 0;
  }
  a.nf = nf;
  a.lend = a.lcap = p->lmax;
  a.wait_ns = kWaitNs;   // the test hook of shtb_plan_debug_waits applies to single-plan calls only
  a.skip_chunk = -1;
  std::memcpy(host_args, &a, sizeof(Args));
}

unsigned long long mixed_group_tile(const shtb_plan* p, int mode, int im, int t0, int par, int* ksteps) {
  const int m = im * p->mres;
  const int J = (p->lmax >= m + par) ? (p->lmax - m - par) / 2 + 1 : 0;
  const int nks = mode == 0 ? (J + kK - 1) / kK : (p->npair + kK - 1) / kK, nall = (nks + kChunk - 1) / kChunk;
  unsigned long long mk = ~0ull;
  if (mode == 0 && !p->hmsk_s.empty()) mk = p->hmsk_s[(size_t)(2 * im + par) * (p->npp / kM) + t0 / kM];
  if (mode == 1 && !p->hmsk_a.empty()) mk = p->hmsk_a[(size_t)(2 * im + par) * p->tab_njt + t0 / kM];
  const int live = __builtin_popcountll(nall >= 64 ? mk : mk & ((1ull << nall) - 1)) + std::max(nall - 64, 0);
  *ksteps = std::min(nks, live * kChunk);
  return mk;
}

int mixed_group_tile_rows() { return kM; }

int launch_pack_group(const void* targs, const int2* items, int nitems, int grid, int* queue, cudaStream_t st) {
  if (nitems <= 0) return SHTB_OK;
  mixed_pack_group_kernel<<<grid, kPack1Threads, 0, st>>>((const Args*)targs, items, nitems, queue);
  count_launch();
  SHTB_TRY_CUDA(cudaGetLastError(), "group pack launch");
  return SHTB_OK;
}

int launch_gemm_group(int mode, const void* targs, const int4* items, const unsigned long long* masks, int nitems,
                      int grid, unsigned long long* done, int* queue, cudaStream_t st) {
  if (nitems <= 0) return SHTB_OK;
  const int smem = Smem<16>::kBytesQ;
  if (mode == 0) {
    auto kern = mixed_gemm_group_kernel<0, 16>;
    SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "group gemm smem attr");
    kern<<<grid, kThreads<16>, smem, st>>>((const Args*)targs, items, masks, nitems, done, queue);
  } else {
    auto kern = mixed_gemm_group_kernel<1, 16>;
    SHTB_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "group gemm smem attr");
    kern<<<grid, kThreads<16>, smem, st>>>((const Args*)targs, items, masks, nitems, done, queue);
  }
  count_launch();
  SHTB_TRY_CUDA(cudaGetLastError(), "group gemm launch");
  return SHTB_OK;
}

}  // namespace shtb
