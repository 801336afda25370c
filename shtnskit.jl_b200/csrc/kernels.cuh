// kernels.cuh — launchers shared between translation units.
#pragma once

#include <algorithm>
#include <type_traits>

#include "internal.cuh"

namespace shtb {

// Coefficient-side operands of the Legendre stage. Element (l, im, k) lives at
//   ptr[k * ld_k + base(im) + l],  base(im) = packed ? off[im] - m : m * ld_m.
// packed: 0 dense (lmax+1, mmax+1) columns of stride ld_m; 1 the plan's internal packed
// (im, l <= lrec) layout; 2 the SHTns LM layout (lm_base). ld_k: field stride.
struct CoefSrc {
  const double2* ptr;
  long long ld_k, ld_m;
  int packed;
};
struct CoefSink {
  double2* ptr;
  long long ld_k, ld_m;
  int packed;
};

// Per-(l, m) multipliers applied where coefficients enter (synthesis) or leave
// (analysis) the Legendre stage: fac (packed, e.g. c_l) * sc[l,m]^(+1|-1) * mf(m).
struct Factors {
  const double* fac;   // packed over (im, l), or null
  const double* sc;    // dense (lmax+1)x(mmax+1) normalization scale, or null
  int sc_mode;         // 0 none, 1 multiply, 2 divide
  double mf0, mf1;     // factor for m == 0 and for m > 0
};

template <typename T, typename GT>
int launch_fft_syn(const shtb_plan* p, const void* W, GT* out0, GT* out1, int ncomp, int nfw, int mlim,
                   double gscale, int use_w, int spow, cudaStream_t st);
// wtile = 1 writes W as the mixed analysis GEMM's B tile images (FP32 only).
template <typename T, typename GT>
int launch_fft_ana(const shtb_plan* p, const GT* in0, const GT* in1, int ncomp, void* W, int nfw, int mlim,
                   double wscale, int use_w, int spow, cudaStream_t st, int wtile = 0);

// FP64 FFTs of complex grids (each latitude row its own sequence): syn = 1 takes the
// Fourier buffer to a complex grid (bins m >= 0 only, times scale), syn = 0 a complex grid
// to the Fourier buffer (weights w times scale).
int launch_fft_cplx64(const shtb_plan* p, int syn, const void* src, void* dst, int nf, int mlim, double scale,
                      cudaStream_t st);

int launch_leg_syn64(const shtb_plan* p, const CoefSrc& src, const Factors& F, void* W, int nf, int row_end,
                     int mlim, cudaStream_t st);
int launch_leg_ana64(const shtb_plan* p, const void* W, int nf, int row_end, int mlim, const CoefSink& dst,
                     const Factors& F, int zero_fill, cudaStream_t st);

// Vector coefficient transforms around the scalar Legendre stage.
int launch_sphtor_pre64(const shtb_plan* p, const double2* S, const double2* T, double2* U, int nf, int ltr,
                        const Factors& F, int div_ll, cudaStream_t st);
int launch_sphtor_post64(const shtb_plan* p, const double2* V, double2* S, double2* T, int nf, int ltr,
                         const Factors& F, int div_ll, cudaStream_t st);
int launch_zero_columns64(const shtb_plan* p, double2* a, int nf, int mlim, cudaStream_t st);

// FP32 FFTs on packed pairs of latitude pairs (fft2.cu) for power-of-two nlon <= 2048 and
// nlat a multiple of 4: the mixed path's analysis into B tile images, and its synthesis.
bool fft2_applicable(const shtb_plan* p);
int launch_fft2_ana(const shtb_plan* p, const float* grid, void* W, int nf, int mlim, double wscale, cudaStream_t st);
int launch_fft2_syn(const shtb_plan* p, const void* W, float* grid, int nf, int mlim, double gscale, cudaStream_t st);

// Floats of one analysis B tile image of the mixed path (hi and lo images back to back).
size_t fft_btile_floats(const shtb_plan* p, int nf);
// Bytes of the mixed path's workspace for op (SHTB_OP_SYNTHESIS or SHTB_OP_ANALYSIS).
size_t mixed_workspace_bytes(const shtb_plan* p, int op, int nf);

// Grouped (uneven-batch) execution: persistent launches over the tiles of many plans.
int mixed_prepare(const shtb_plan* p, cudaStream_t st);
size_t mixed_args_bytes();
void mixed_fill_args(const shtb_plan* p, int mode, const void* in, void* out, int nf, void* host_args);
// Live-chunk mask of GEMM tile (mode, im, first pair or degree row t0, par) of a prepared
// plan, with the K-steps its live chunks hold (the tile's cost).
unsigned long long mixed_group_tile(const shtb_plan* p, int mode, int im, int t0, int par, int* ksteps);
int mixed_group_tile_rows();
int launch_gemm_group(int mode, const void* targs, const int4* items, const unsigned long long* masks, int nitems,
                      int grid, unsigned long long* done, int* queue, cudaStream_t st);
int launch_pack_group(const void* targs, const int2* items, int nitems, int grid, int* queue, cudaStream_t st);
size_t fft_job_bytes_f32();
void fft_fill_job_f32(const shtb_plan* p, int syn, const void* W, void* grid, int nf, void* host_job);
size_t fft_group_smem_f32(const shtb_plan* p, int h);
bool fft_plan_generic(const shtb_plan* p);
int launch_fft_group_f32(int syn, int h, bool generic, const void* jobs, const int4* items, int nitems, int grid,
                         size_t smem, int* queue, cudaStream_t st);
// Mixed-precision Legendre synthesis on the FP64 pipes for one or two fields (simt.cu):
// coefficients (dense or packed LM) -> Fourier buffer.
bool simt_applicable(const shtb_plan* p, int nf);
int launch_simt_syn(const shtb_plan* p, const void* alm, void* W, int nf, int ltr, int mlim, int packed,
                    cudaStream_t st);
size_t simt_args_bytes();
void simt_fill_args(const shtb_plan* p, const void* alm, void* W, int nf, void* host_args);
int simt_syn_pair_blocks(const shtb_plan* p);
size_t simt_group_syn_smem(const shtb_plan* p);
int launch_simt_group(const void* targs, const int4* items, int nitems, int grid, size_t smem, int* queue,
                      cudaStream_t st);
// the packed-pair FP32 FFTs of fft2_applicable members (2 HP latitude pairs per item)
size_t fft2_job_bytes();
int fft2_group_pairs();
size_t fft2_group_smem(const shtb_plan* p);
void fft2_fill_job(const shtb_plan* p, int syn, const void* W, void* grid, int nf, void* host_job);
int launch_fft2_group(int syn, const void* jobs, const int4* items, int nitems, int grid, size_t smem, int* queue,
                      cudaStream_t st);

}  // namespace shtb
