// internal.cuh — plan layout, error plumbing and small device helpers shared by
// the translation units of libshtb200.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shtb200.h"

namespace shtb {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);   // records msg, returns code
int check_cuda(cudaError_t e, const char* what);    // SHTB_OK or SHTB_ERR_CUDA
void count_launch(int n = 1);
// Per-kernel CUDA-event timing on the launching stream (off unless enabled by
// shtb_profile_enable); prof_begin/prof_end bracket one launch.
void prof_begin(cudaStream_t st);
void prof_end(const char* name, cudaStream_t st);
// Device address, on the current device, of the static scratch array that the
// allocation-free synthesis uses (cudaGetSymbolAddress; loads the module holding it).
cudaError_t noalloc_scratch_address(void** out);

#define SHTB_TRY_CUDA(expr, what)                                   \
  do {                                                              \
    int _rc = ::shtb::check_cuda((expr), (what));                   \
    if (_rc != SHTB_OK) return _rc;                                 \
  } while (0)

#define SHTB_LAUNCHED(what)                                         \
  do {                                                              \
    ::shtb::prof_end((what), st);                                   \
    ::shtb::count_launch();                                         \
    int _rc = ::shtb::check_cuda(cudaGetLastError(), (what));       \
    if (_rc != SHTB_OK) return _rc;                                 \
  } while (0)

// Degrees of one FP64 analysis tile (64 of each parity).
constexpr int kAnaTile = 128;
// Largest checkpoint table the plan keeps (bytes); the spacing grows from 16 degrees
// until the table fits.
constexpr size_t kCkptBudget = size_t(2) << 30;

// ---------------------------------------------------------------------------
// device view of a plan (passed by value to kernels)
// ---------------------------------------------------------------------------
struct PlanDev {
  int lmax, mmax, mres, nlat, nlon, nm, npair, lrec;  // lrec = lmax + 1
  const double* x;         // [nlat] north first
  const double* w;         // [nlat]
  const double* sint;      // [nlat]
  const long long* off;    // [nm+1] packed (im, l) offsets, l in [m, lrec]
  const double* alpha;     // packed: r_l = alpha_l x r_{l-1} - r_{l-2}
  const double* cfac;      // packed: P_l = c_l r_l
  const int* l0;           // [nm*npair] first significant degree per (im, pair)
  const double2* r01;      // [nm*npair] (r_{l0}, r_{l0+1})
  // recurrence checkpoints every ckstep degrees: entry (ckbase[im] + k) * npair + pair holds
  // the state (r_{t-1}, r_{t-2}) before degree t = m + k * ckstep
  const double2* ckpt;
  const int* ckbase;       // [nm]
  int ckstep;              // 16, 32, 64 or 128 (a divisor of kAnaTile)
  // FP64 analysis tiles of kAnaTile degrees: (im, t0, checkpoint index of t0, 0)
  const int4* atiles;
  int natiles;
};

// FFT description for nlon
struct FFTDesc {
  int n;
  int nrad;
  int rad[24];
  bool direct;             // a prime factor above the largest register radix: O(N^2) DFT
  int padsh;               // shared-memory index skew: element i at i + (i >> padsh)
  int twoff[24];           // pass s twiddles start at twoff[s] in the per-pass table
  unsigned mrow[24];       // floor(2^32 / (n / rad[s])) + 1, or 0 when n / rad[s] == 1
  unsigned mspan[24];      // the same for the group span Ns / rad[s]
};

// B operand tile images of the mixed-precision GEMMs: one region of nfp x 16 floats per
// K-step (nfp = fields rounded up to 4, so tiles have whole 8-row core-matrix groups);
// fields in blocks of 64 (1024 floats), block rows 2f (real) and 2f+1 (imaginary) in the
// K-major no-swizzle core-matrix order, 8 K values per row. btile_off gives the float
// offset of (row, K slot kk) inside a block. The analysis images hold FP32 values (from the
// FFT); the synthesis images hold f16 hi/lo tile pairs in the same bytes (16 K values per
// row and region, hi in even regions, lo in odd ones).
__host__ __device__ inline int btile_nfp(int nf) { return (nf + 3) & ~3; }
__host__ __device__ inline int btile_off(int row, int kk) {
  return (row >> 3) * 64 + (kk >> 2) * 32 + (row & 7) * 4 + (kk & 3);
}

// Start of order m's block in the packed LM layout of SHTns (src/layout.jl:143-162):
// LM_index(l, m) = lm_base(m) + l with im = m / mres.
__host__ __device__ inline long long lm_base(int lmax, int mres, int m) {
  const long long im = m / mres;
  return (im * (2LL * lmax + 2 - (im + 1) * mres)) >> 1;
}
// Number of packed LM coefficients (nlm_calc, src/layout.jl:88-101).
__host__ __device__ inline long long lm_count(int lmax, int mmax, int mres) {
  long long s = 0;
  for (int m = 0; m <= mmax && m <= lmax; m += mres) s += lmax - m + 1;
  return s;
}

// floor(v / d) for v * d < 2^32 with the multiplier m = floor(2^32 / d) + 1 (m = 0 means d = 1)
__host__ __device__ inline unsigned magic_div_mul(unsigned d) {
  return d <= 1 ? 0u : (unsigned)((1ull << 32) / d + 1);
}

}  // namespace shtb

struct shtb_plan {
  int lmax, mmax, mres, nlat, nlon, nm, npair, lrec;
  int robert;
  int device;
  double phi_inv_scale, ana_scale;
  bool canonical;
  std::vector<double> hx, hw, hsint;
  std::vector<double> hscale;             // (lmax+1)*(mmax+1), empty if canonical
  std::vector<long long> hoff;            // [nm+1]
  shtb::FFTDesc fft;
  // device memory
  void* dmem = nullptr;                   // one allocation for every small table
  size_t dbytes = 0;
  shtb::PlanDev dev{};
  const double* d_scale = nullptr;        // s_lm table (device) or null
  const double2* d_tw64 = nullptr;        // exp(-2 pi i t / nlon)
  const float2* d_tw32 = nullptr;
  const int* d_rev = nullptr;             // FFT output position of bin k (digit reversal)
  const int* d_rinv = nullptr;            // natural index stored at FFT position q (inverse of d_rev)
  const double2* d_twp64 = nullptr;       // per-pass twiddles: pass s, factor q (1..r-1), index j < span:
  const float2* d_twp32 = nullptr;        //   entry twoff[s] + (q-1)*span + j = exp(-2 pi i j q / Ns)
  const double* d_dcoef = nullptr;        // packed d(l,m) = sqrt((l^2-m^2)/(4l^2-1)), l in [m, lrec]
  int* d_err = nullptr;                   // device status word (bounded waits that gave up)
  // device address of the allocation-free synthesis's static scratch array on this
  // plan's device, resolved at plan creation (null, with the reason, if that failed)
  void* noalloc_scratch = nullptr;
  std::string noalloc_err;
  // test hook of the mixed GEMMs' bounded waits (shtb_plan_debug_waits): limit in ns
  // (0: the default 2 s) and a chunk CTA 0's loader leaves unissued (-1: none)
  unsigned long long dbg_wait_ns = 0;
  int dbg_skip_chunk = -1;
  // mixed-precision path: FP32 table of P_l^m grouped by (m, parity), built on first use
  std::mutex tab_mu;
  float* d_tab = nullptr;                 // synthesis tile images (start of the table allocation)
  float* d_tab_ana = nullptr;             // analysis tile images
  const long long* d_tab_seg = nullptr;
  // per-tile live-chunk masks of the GEMMs (chunks whose P image is all zero are skipped):
  // synthesis [2 nm][npp / 128], analysis [2 nm][tab_njt]
  const unsigned long long* d_tab_msk_s = nullptr;
  const unsigned long long* d_tab_msk_a = nullptr;
  int tab_njt = 0;
  size_t tab_bytes = 0;
  int npp = 0;
  std::vector<long long> htab_seg;
  std::vector<unsigned long long> hmsk_s, hmsk_a;   // host copies of the live-chunk masks
  // GEMM tile lists (analysis: (im, j0); synthesis: (im, p0)) for truncation degree key
  // GEMM tile lists of the mixed path per direction (0 synthesis, 1 analysis) and truncation
  // degree, kept until the plan is destroyed: device entries and live-chunk masks
  struct MxTileList {
    int2* tiles = nullptr;
    unsigned long long* masks = nullptr;
    int count = 0;
  };
  std::map<int, MxTileList> mx_lists[2];
};
