// simt.cu — mixed-precision Legendre synthesis for batches of one or two fields, with the
// recurrence regenerated on the fly on the FP64 pipes.
//
// The tensor-core synthesis GEMM of mixed.cu reads the plan's P table image (4 bytes per
// value) once per transform whatever the number of fields, so with one or two fields that
// stream, not the arithmetic, sets its time: 4 bytes of table for 2 or 4 output columns. Here
// each thread runs the c-scaled three-term recurrence of its own latitude pair in FP64,
//   r_l = alpha_l x r_{l-1} - r_{l-2},   P_l^m = c_l r_l,
// from the plan's start records (values below 2^-480 are zero until the record's first
// degree l0), so P is never read from memory: 2 FP64 operations per value plus the
// multiply-adds of the fields. Thread = latitude pair, CTA = 128 pairs of one order; the
// order's coefficients (times c_l and the per-(l, m) factors, in FP64) are staged in shared
// memory and read as broadcasts; E and O sums in FP64. Output: the Fourier buffer
// W[field][im][E|O][pair] (FP32) that the FFT synthesis reads, as the GEMM writes it.
//
// The analysis keeps the tensor-core GEMM: its sums run over latitude pairs, across threads,
// and a version of this kernel that reduced them across each CTA per block of degrees ran
// several times slower than the GEMM on one-field batches (latency-bound chains at a few
// warps per SM).
#include <climits>
#include <cstring>

#include "kernels.cuh"

namespace shtb {
namespace sx {

constexpr int kSynThreads = 128;

struct Args {
  PlanDev P;
  const double* sc;       // normalization scale table (dense) or null
  int sc_mode;            // 0 none, 1 multiply
  const float2* cin;      // coefficients, field stride ld_k
  float2* Wout;           // Fourier buffer
  long long ld_k;
  int cpacked;            // coefficients in the packed LM layout (ld_k = nlm)
  int nf, lend;
};

__device__ __forceinline__ double coef_factor(const Args& a, int l, int m) {
  double s = 1.0;
  if (a.sc_mode) {
    const double q = a.sc[l + (long long)(a.P.lmax + 1) * m];
    s = q;
  }
  return s;
}

// ------------------------------------------------------------------------- synthesis
// Order index im, pairs 128 pb .. 128 pb + 127. smem: alpha of the order's degrees, then the
// folded coefficients [degree][field] (syn_smem_bytes of the plan's lmax). All threads of the
// CTA call it (it synchronises them).
__host__ __device__ inline size_t syn_smem_bytes(int lmax, int nf) {
  return (size_t)((lmax + 2) & ~1) * 8 + (size_t)(lmax + 1) * nf * 16 + 64;
}

template <int NF>
__device__ __forceinline__ void syn_body(const Args& a, int im, int pb, double* smem) {
  const PlanDev& P = a.P;
  const int m = im * P.mres;
  const int lend = a.lend, ndeg = lend - m + 1;
  const long long poff = P.off[im];
  double* sAl = smem;
  double2* sC = reinterpret_cast<double2*>(smem + ((ndeg + 1) & ~1));
  for (int d = threadIdx.x; d < ndeg; d += kSynThreads) sAl[d] = P.alpha[poff + d];
  for (int i = threadIdx.x; i < ndeg * NF; i += kSynThreads) {
    const int d = i / NF, k = i - d * NF, l = m + d;
    double2 v = make_double2(0.0, 0.0);
    if (k < a.nf) {
      const long long col = a.cpacked ? lm_base(P.lmax, P.mres, m) : (long long)m * (P.lmax + 1);
      const float2 c = a.cin[(long long)k * a.ld_k + col + l];
      const double f = P.cfac[poff + d] * coef_factor(a, l, m);
      v = make_double2(c.x * f, c.y * f);
    }
    sC[i] = v;
  }
  const int npair = P.npair, pair = pb * kSynThreads + threadIdx.x;
  int l0 = INT_MAX / 2;
  double x = 0.0, s0 = 0.0, s1 = 0.0;
  if (pair < npair) {
    x = P.x[pair];
    l0 = P.l0[(size_t)im * npair + pair];
    const double2 v = P.r01[(size_t)im * npair + pair];
    s0 = v.x;
    s1 = v.y;
  }
  // each warp starts at its own pairs' first significant degree (below it every value is
  // zero) and a warp with no pair of the plan skips the degree loop
  int mn = l0;
  for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  __syncthreads();   // the staged alpha and coefficients
  const int lbeg = max(mn, m);
  const bool warp_live = pb * kSynThreads + (threadIdx.x & ~31) < npair;
  double2 accE[NF], accO[NF];
#pragma unroll
  for (int k = 0; k < NF; ++k) accE[k] = accO[k] = make_double2(0.0, 0.0);
  double ra = 0.0, rb = 0.0;
  // one degree into acc (E for even l - m, O for odd): the parity is static in the unrolled
  // loop below, so the accumulators stay in registers
  auto step = [&](int l, double2 (&acc)[NF]) {
    const int d = l - m;
    double r = fma(sAl[d] * x, ra, -rb);
    r = (l == l0) ? s0 : r;
    r = (l == l0 + 1) ? s1 : r;
    rb = ra;
    ra = r;
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      const double2 c = sC[d * NF + k];
      acc[k].x = fma(r, c.x, acc[k].x);
      acc[k].y = fma(r, c.y, acc[k].y);
    }
  };
  if (warp_live) {
    int l = lbeg;
    if (((l - m) & 1) && l <= lend) step(l++, accO);
    for (; l + 1 <= lend; l += 2) {
      step(l, accE);
      step(l + 1, accO);
    }
    if (l <= lend) step(l, accE);
  }
  if (pair < npair) {
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      if (k >= a.nf) break;
      float2* w = a.Wout + (((size_t)k * P.nm + im) * 2) * npair + pair;
      w[0] = make_float2((float)accE[k].x, (float)accE[k].y);
      w[npair] = make_float2((float)accO[k].x, (float)accO[k].y);
    }
  }
  __syncthreads();   // shared memory is reused by the caller's next item
}

// blockIdx.x = block of 128 pairs, blockIdx.y = order index.
template <int NF>
__global__ void __launch_bounds__(kSynThreads) syn_kernel(const __grid_constant__ Args a) {
  extern __shared__ __align__(16) double smem[];
  syn_body<NF>(a, blockIdx.y, blockIdx.x, smem);
}

// Persistent kernel over the items of many transforms (uneven batches), one item per warp:
// item = (transform, order index, block of 32 latitude pairs), list sorted by decreasing
// work and claimed by each warp from the device counter *queue (zero at launch). A warp
// stages its order's recurrence coefficients and FP64 coefficients in its own shared-memory
// slice, kGroupChunk degrees at a time, so warps never wait for one another (a CTA-wide item
// ends with a barrier at which the warps nearer the poles, which start at higher degrees,
// wait for the others). Per thread the arithmetic is that of syn_body, so the results are
// the same bit for bit.
constexpr int kGroupChunk = 128;
constexpr size_t kGroupWarpDoubles = kGroupChunk + kGroupChunk * 2 * 2;   // alpha, then [degree][NF <= 2] double2

template <int NF>
__device__ __forceinline__ void syn_warp_item(const Args& a, int im, int pb, double* wsm) {
  const PlanDev& P = a.P;
  const int lane = threadIdx.x & 31;
  const int m = im * P.mres;
  const int lend = a.lend, ndeg = lend - m + 1;
  const long long poff = P.off[im];
  double* sAl = wsm;
  double2* sC = reinterpret_cast<double2*>(wsm + kGroupChunk);
  const int npair = P.npair, pair = pb * 32 + lane;
  int l0 = INT_MAX / 2;
  double x = 0.0, s0 = 0.0, s1 = 0.0;
  if (pair < npair) {
    x = P.x[pair];
    l0 = P.l0[(size_t)im * npair + pair];
    const double2 v = P.r01[(size_t)im * npair + pair];
    s0 = v.x;
    s1 = v.y;
  }
  int mn = l0;
  for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  const int dbeg = max(mn, m) - m;   // first degree (relative to m) with a nonzero value
  const long long col = a.cpacked ? lm_base(P.lmax, P.mres, m) : (long long)m * (P.lmax + 1);
  double2 accE[NF], accO[NF];
#pragma unroll
  for (int k = 0; k < NF; ++k) accE[k] = accO[k] = make_double2(0.0, 0.0);
  double ra = 0.0, rb = 0.0;
  for (int d0 = dbeg; d0 < ndeg; d0 += kGroupChunk) {
    const int nd = min(kGroupChunk, ndeg - d0);
    __syncwarp();   // the previous chunk's values are read
    for (int d = lane; d < nd; d += 32) sAl[d] = P.alpha[poff + d0 + d];
    for (int i = lane; i < nd * NF; i += 32) {
      const int d = i / NF, k = i - d * NF, l = m + d0 + d;
      double2 v = make_double2(0.0, 0.0);
      if (k < a.nf) {
        const float2 c = a.cin[(long long)k * a.ld_k + col + l];
        const double f = P.cfac[poff + d0 + d] * coef_factor(a, l, m);
        v = make_double2(c.x * f, c.y * f);
      }
      sC[i] = v;
    }
    __syncwarp();
    auto step = [&](int l, double2 (&acc)[NF]) {
      const int d = l - m - d0;
      double r = fma(sAl[d] * x, ra, -rb);
      r = (l == l0) ? s0 : r;
      r = (l == l0 + 1) ? s1 : r;
      rb = ra;
      ra = r;
#pragma unroll
      for (int k = 0; k < NF; ++k) {
        const double2 c = sC[d * NF + k];
        acc[k].x = fma(r, c.x, acc[k].x);
        acc[k].y = fma(r, c.y, acc[k].y);
      }
    };
    int l = m + d0;
    const int le = m + d0 + nd - 1;
    if (((l - m) & 1) && l <= le) step(l++, accO);
    for (; l + 1 <= le; l += 2) {
      step(l, accE);
      step(l + 1, accO);
    }
    if (l <= le) step(l, accE);
  }
  if (pair < npair) {
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      if (k >= a.nf) break;
      float2* w = a.Wout + (((size_t)k * P.nm + im) * 2) * npair + pair;
      w[0] = make_float2((float)accE[k].x, (float)accE[k].y);
      w[npair] = make_float2((float)accO[k].x, (float)accO[k].y);
    }
  }
}

__global__ void __launch_bounds__(kSynThreads, 8) syn_group_kernel(const Args* __restrict__ targs,
                                                                const int4* __restrict__ items, int nitems,
                                                                int* __restrict__ queue) {
  extern __shared__ __align__(16) double smem[];
  double* wsm = smem + (threadIdx.x >> 5) * kGroupWarpDoubles;
  const int lane = threadIdx.x & 31;
  for (;;) {
    int i = 0;
    if (lane == 0) i = atomicAdd(queue, 1);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= nitems) break;
    const int4 it = items[i];
    const Args& a = targs[it.x];
    if (a.nf == 1)
      syn_warp_item<1>(a, it.y, it.z, wsm);
    else
      syn_warp_item<2>(a, it.y, it.z, wsm);
  }
}

}  // namespace sx

// ---------------------------------------------------------------------------- host
bool simt_applicable(const shtb_plan* p, int nf) { return nf >= 1 && nf <= 2; }

static sx::Args simt_args(const shtb_plan* p, const void* alm, void* W, int nf, int ltr, int packed) {
  sx::Args a;
  a.P = p->dev;
  a.sc = p->d_scale;
  a.sc_mode = p->d_scale ? 1 : 0;
  a.cin = (const float2*)alm;
  a.Wout = (float2*)W;
  a.cpacked = packed;
  a.ld_k = packed ? lm_count(p->lmax, p->mmax, p->mres) : (long long)(p->lmax + 1) * (p->mmax + 1);
  a.nf = nf;
  a.lend = ltr;
  return a;
}

// Coefficients (FP32, dense or packed LM) -> Fourier buffer W (FP32), orders 0..mlim.
int launch_simt_syn(const shtb_plan* p, const void* alm, void* W, int nf, int ltr, int mlim, int packed,
                    cudaStream_t st) {
  const sx::Args a = simt_args(p, alm, W, nf, ltr, packed);
  const int nmu = mlim / p->mres + 1;
  const size_t smem = sx::syn_smem_bytes(p->lmax, nf);
  dim3 grid((p->npair + sx::kSynThreads - 1) / sx::kSynThreads, nmu);
  prof_begin(st);
  if (nf == 1) {
    SHTB_TRY_CUDA(cudaFuncSetAttribute(sx::syn_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "simt smem attr");
    sx::syn_kernel<1><<<grid, sx::kSynThreads, smem, st>>>(a);
  } else {
    SHTB_TRY_CUDA(cudaFuncSetAttribute(sx::syn_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "simt smem attr");
    sx::syn_kernel<2><<<grid, sx::kSynThreads, smem, st>>>(a);
  }
  SHTB_LAUNCHED("simt legendre synthesis kernel");
  return SHTB_OK;
}

// ------------------------------------------------------------- grouped transforms
size_t simt_args_bytes() { return sizeof(sx::Args); }

void simt_fill_args(const shtb_plan* p, const void* alm, void* W, int nf, void* host_args) {
  const sx::Args a = simt_args(p, alm, W, nf, p->lmax, 0);
  std::memcpy(host_args, &a, sizeof(a));
}

int simt_syn_pair_blocks(const shtb_plan* p) { return (p->npair + 31) / 32; }   // per-warp items of the group kernel

size_t simt_group_syn_smem(const shtb_plan*) { return (sx::kSynThreads / 32) * sx::kGroupWarpDoubles * sizeof(double); }

int launch_simt_group(const void* targs, const int4* items, int nitems, int grid, size_t smem, int* queue,
                      cudaStream_t st) {
  if (nitems <= 0) return SHTB_OK;
  SHTB_TRY_CUDA(cudaFuncSetAttribute(sx::syn_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "simt group smem attr");
  sx::syn_group_kernel<<<grid, sx::kSynThreads, smem, st>>>((const sx::Args*)targs, items, nitems, queue);
  count_launch();
  SHTB_TRY_CUDA(cudaGetLastError(), "simt group launch");
  return SHTB_OK;
}

}  // namespace shtb
