// plan.cu — plan construction: host-side validation and tables, device setup
// kernel for the per-(m, latitude) recurrence start records and the analysis
// checkpoints, Gauss-Legendre nodes, error plumbing.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>

#include "internal.cuh"

namespace shtb {

static thread_local std::string g_last_error;
static thread_local uint64_t g_launches = 0;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SHTB_OK;
  return set_error(SHTB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void count_launch(int n) { g_launches += (uint64_t)n; }

// Constants of the extended-range seed (SHTnsKit src/legendre.jl:203-215):
// a scaled value p with exponent e stands for p * 2^e, rescaled by 2^960.
__device__ __constant__ double kInvSqrt4Pi = 0.28209479177387814;

__device__ inline double plm_a(int l, int m) {
  return sqrt(((double)(2 * l - 1) * (double)(2 * l + 1)) / ((double)(l - m) * (double)(l + m)));
}
__device__ inline double plm_b(int l, int m) {
  return sqrt(((double)(2 * l + 1) * (double)(l - 1 - m) * (double)(l - 1 + m)) /
              ((double)(2 * l - 3) * (double)(l - m) * (double)(l + m)));
}

// One thread per (im, latitude pair): the sectoral seed with its power-of-two
// exponent (legendre.jl:252-271), the scaled recurrence until the exponent
// returns to zero (legendre.jl:287-322), then the c-scaled recurrence
//   r_l = alpha_l x r_{l-1} - r_{l-2}
// through lrec, recording the state in front of every ckstep-th degree.
// Values whose exponent is still negative are below 2^-480 and are dropped.
__global__ void plan_setup_kernel(PlanDev P, const double* __restrict__ seedfac, int* __restrict__ l0_out,
                                  double2* __restrict__ r01_out, double2* __restrict__ ckpt_out) {
  const int pair = blockIdx.x * blockDim.x + threadIdx.x;
  const int im = blockIdx.y;
  if (pair >= P.npair) return;
  const int m = im * P.mres;
  const int LR = P.lrec;
  const double x = P.x[pair];
  const double s = sqrt(fmax(0.0, (1.0 - x) * (1.0 + x)));
  const double TINY = 0x1p-480, HUGE_ = 0x1p480, UP = 0x1p960, DOWN = 0x1p-960;
  double pmm = kInvSqrt4Pi;
  int e = 0;
  for (int k = 1; k <= m; k += 8) {
    const int kend = min(k + 7, m);
    for (int j = k; j <= kend; ++j) pmm = (seedfac[j] * s) * pmm;
    while (fabs(pmm) < TINY && pmm != 0.0) {
      pmm *= UP;
      e -= 960;
    }
  }
  const long long base = P.off[im];
  int l0;
  double r0 = 0.0, r1 = 0.0;
  if (e == 0) {
    l0 = m;
    r0 = pmm;
    r1 = sqrt((double)(2 * m + 3)) * x * pmm;
  } else {
    double p2 = pmm, p1 = sqrt((double)(2 * m + 3)) * x * pmm;
    int l = m + 2;
    bool ok = false;
    while (l <= LR) {
      const double p = plm_a(l, m) * x * p1 - plm_b(l, m) * p2;
      p2 = p1;
      p1 = p;
      ++l;
      const double mag = fmax(fabs(p2), fabs(p1));
      if (mag > HUGE_) {
        p2 *= DOWN;
        p1 *= DOWN;
        e += 960;
        if (e == 0) {
          ok = true;
          break;
        }
      } else if (mag < TINY && mag != 0.0) {
        p2 *= UP;
        p1 *= UP;
        e -= 960;
      }
    }
    if (ok) {
      l0 = l - 2;
      r0 = p2 / P.cfac[base + (l0 - m)];
      r1 = p1 / P.cfac[base + (l0 + 1 - m)];
    } else {
      l0 = INT_MAX / 2;
    }
  }
  l0_out[(size_t)im * P.npair + pair] = l0;
  r01_out[(size_t)im * P.npair + pair] = make_double2(r0, r1);
  // checkpoints: state before degrees m + ckstep * k
  const int tb = P.ckbase[im];
  double ra = 0.0, rb = 0.0;
  for (int l = m; l <= LR; ++l) {
    if (((l - m) % P.ckstep) == 0)
      ckpt_out[(size_t)(tb + (l - m) / P.ckstep) * P.npair + pair] = make_double2(ra, rb);
    double r;
    if (l == l0)
      r = r0;
    else if (l == l0 + 1)
      r = r1;
    else
      r = fma(P.alpha[base + (l - m)] * x, ra, -rb);
    rb = ra;
    ra = r;
  }
}

static bool factor_fft(int n, FFTDesc& d) {
  d.n = n;
  d.nrad = 0;
  d.direct = false;
  int k = n;
  // prefer radix 16, 8 and 4, then 2, 3, 5, 7 and small odd primes up to 16: fewer
  // passes over shared memory
  while (k % 16 == 0 && d.nrad < 24) { d.rad[d.nrad++] = 16; k /= 16; }
  while (k % 8 == 0 && d.nrad < 24) { d.rad[d.nrad++] = 8; k /= 8; }
  while (k % 4 == 0 && d.nrad < 24) { d.rad[d.nrad++] = 4; k /= 4; }
  while (k % 2 == 0 && d.nrad < 24) { d.rad[d.nrad++] = 2; k /= 2; }
  const int odd[] = {3, 5, 7, 11, 13};
  for (int p : odd)
    while (k % p == 0 && d.nrad < 24) { d.rad[d.nrad++] = p; k /= p; }
  if (k != 1) {
    d.direct = true;
    d.nrad = 0;
  }
  // FP32 rows: skew i + i/16 leaves every pass of a power-of-two length free of bank
  // conflicts; mixed radices (odd last passes) do better with i + i/8 (fft_padsh).
  d.padsh = ((n & (n - 1)) == 0) ? 4 : 3;
  int off = 0, Ns = n;
  for (int s = 0; s < d.nrad; ++s) {
    const int r = d.rad[s], span = Ns / r;
    d.twoff[s] = off;
    d.mrow[s] = magic_div_mul((unsigned)(n / r));
    d.mspan[s] = magic_div_mul((unsigned)span);
    off += (r - 1) * span;
    Ns = span;
  }
  return true;
}

// Per-pass twiddle table (layout of FFTDesc::twoff): entry twoff[s] + (q-1)*span + j.
static int fft_pass_twiddles(const FFTDesc& d, std::vector<double2>& out) {
  out.clear();
  int Ns = d.n;
  for (int s = 0; s < d.nrad; ++s) {
    const int r = d.rad[s], span = Ns / r;
    for (int q = 1; q < r; ++q)
      for (int j = 0; j < span; ++j) {
        const long long e = ((long long)j * q) % Ns;
        const double ang = -2.0 * (double)e / (double)Ns;   // in units of pi
        out.push_back(make_double2(std::cos(M_PI * ang), std::sin(M_PI * ang)));
      }
    Ns = span;
  }
  if (out.empty()) out.push_back(make_double2(1.0, 0.0));
  return (int)out.size();
}

}  // namespace shtb

using namespace shtb;

extern "C" int shtb_version(void) { return 100; }

extern "C" const char* shtb_last_error(void) { return g_last_error.c_str(); }

extern "C" uint64_t shtb_launch_count(int reset) {
  uint64_t v = g_launches;
  if (reset) g_launches = 0;
  return v;
}

// Newton iteration on P_n, tolerance 1e-15, at most 50 steps (legendre.jl:956-1003),
// returned north pole first (config.jl:639).
extern "C" int shtb_gauss_nodes(int n, double* x, double* w) {
  if (n <= 0) return set_error(SHTB_ERR_BAD_ARG, "n must be positive");
  if (!x || !w) return set_error(SHTB_ERR_BAD_ARG, "null output pointer");
  std::vector<double> xs(n), ws(n);
  const int half = (n + 1) / 2;
  for (int k = 1; k <= half; ++k) {
    double z = std::cos(M_PI * (k - 0.25) / (n + 0.5));
    for (int it = 0; it < 50; ++it) {
      double pnm1 = 1.0, pn = z;
      for (int l = 2; l <= n; ++l) {
        const double pnp1 = ((2.0 * l - 1) * z * pn - (l - 1.0) * pnm1) / l;
        pnm1 = pn;
        pn = pnp1;
      }
      const double pd = n * (z * pn - pnm1) / (z * z - 1.0);
      const double z1 = z;
      z -= pn / pd;
      if (std::fabs(z - z1) < 1e-15) break;
    }
    double pnm1 = 1.0, pn = z;
    for (int l = 2; l <= n; ++l) {
      const double pnp1 = ((2.0 * l - 1) * z * pn - (l - 1.0) * pnm1) / l;
      pnm1 = pn;
      pn = pnp1;
    }
    const double pd = n * (z * pn - pnm1) / (z * z - 1.0);
    xs[k - 1] = -z;
    xs[n - k] = z;
    const double wk = 2.0 / ((1.0 - z * z) * pd * pd);
    ws[k - 1] = wk;
    ws[n - k] = wk;
  }
  for (int i = 0; i < n; ++i) {
    x[i] = xs[n - 1 - i];
    w[i] = ws[n - 1 - i];
  }
  return SHTB_OK;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

extern "C" int shtb_plan_create(shtb_plan** out, int lmax, int mmax, int mres, int nlat, int nlon,
                                const double* x, const double* w, const double* coeff_scale,
                                double phi_inv_scale, double analysis_phi_scale, int robert_form) {
  if (!out) return set_error(SHTB_ERR_BAD_ARG, "plan output pointer is NULL");
  *out = nullptr;
  // _validate_spectral_layout (src/config.jl:465-481), Gauss grid
  if (lmax < 0) return set_error(SHTB_ERR_BAD_ARG, "lmax must be >= 0, got " + std::to_string(lmax));
  if (mmax < 0) return set_error(SHTB_ERR_BAD_ARG, "mmax must be >= 0, got " + std::to_string(mmax));
  if (mmax > lmax)
    return set_error(SHTB_ERR_BAD_ARG, "mmax must be <= lmax, got mmax=" + std::to_string(mmax) +
                                           ", lmax=" + std::to_string(lmax));
  if (mres < 1) return set_error(SHTB_ERR_BAD_ARG, "mres must be >= 1, got " + std::to_string(mres));
  if (nlat < 1) return set_error(SHTB_ERR_BAD_ARG, "nlat must be >= 1, got " + std::to_string(nlat));
  if (nlat < lmax + 1)
    return set_error(SHTB_ERR_BAD_ARG,
                     "Gauss-Legendre quadrature requires nlat >= lmax+1, got nlat=" +
                         std::to_string(nlat) + " and lmax=" + std::to_string(lmax));
  if (nlon < 2 * mmax + 1)
    return set_error(SHTB_ERR_BAD_ARG, "nlon must be >= 2*mmax+1 = " + std::to_string(2 * mmax + 1) +
                                           " to resolve every azimuthal order, got nlon=" +
                                           std::to_string(nlon));
  if (!x || !w) return set_error(SHTB_ERR_BAD_ARG, "x and w must be host arrays of nlat values");
  if (nlon > 8192) return set_error(SHTB_ERR_UNSUPPORTED, "nlon above 8192 is not supported");
  for (int i = 0; i < nlat; ++i) {
    if (!(x[i] >= -1.0 && x[i] <= 1.0)) return set_error(SHTB_ERR_BAD_ARG, "x must lie in [-1, 1]");
    if (i > 0 && !(x[i] < x[i - 1])) return set_error(SHTB_ERR_BAD_ARG, "x must be strictly decreasing (north first)");
  }
  for (int i = 0; i < nlat / 2; ++i)
    if (std::fabs(x[i] + x[nlat - 1 - i]) > 1e-12)
      return set_error(SHTB_ERR_BAD_ARG, "latitudes must be symmetric about the equator");

  shtb_plan* p = new (std::nothrow) shtb_plan();
  if (!p) return set_error(SHTB_ERR_OOM, "host allocation failed");
  p->lmax = lmax;
  p->mmax = mmax;
  p->mres = mres;
  p->nlat = nlat;
  p->nlon = nlon;
  p->nm = mmax / mres + 1;
  p->npair = (nlat + 1) / 2;
  p->lrec = lmax + 1;
  p->robert = robert_form ? 1 : 0;
  p->phi_inv_scale = phi_inv_scale;
  p->ana_scale = analysis_phi_scale;
  p->hx.assign(x, x + nlat);
  p->hw.assign(w, w + nlat);
  p->hsint.resize(nlat);
  for (int i = 0; i < nlat; ++i) p->hsint[i] = std::sqrt(std::max(0.0, (1.0 - x[i]) * (1.0 + x[i])));
  p->canonical = (coeff_scale == nullptr);
  if (coeff_scale) p->hscale.assign(coeff_scale, coeff_scale + (size_t)(lmax + 1) * (mmax + 1));
  cudaGetDevice(&p->device);
  factor_fft(nlon, p->fft);

  const int nm = p->nm, npair = p->npair, LR = p->lrec;
  p->hoff.resize(nm + 1);
  long long acc = 0;
  for (int im = 0; im < nm; ++im) {
    p->hoff[im] = acc;
    acc += LR - im * mres + 1;
  }
  p->hoff[nm] = acc;
  const long long npk = acc;
  // checkpoint spacing: the finest of 16, 32, 64, 128 degrees whose table fits the budget
  int ckstep = 16;
  auto nseg_total = [&](int cs) {
    long long n = 0;
    for (int im = 0; im < nm; ++im) n += (LR - im * mres + cs) / cs;
    return n;
  };
  while (ckstep < kAnaTile && (size_t)nseg_total(ckstep) * npair * 16 > kCkptBudget) ckstep *= 2;
  std::vector<int> ckbase(nm);
  int nseg = 0;
  for (int im = 0; im < nm; ++im) {
    ckbase[im] = nseg;
    nseg += (LR - im * mres + ckstep) / ckstep;
  }
  std::vector<int4> atiles;
  for (int im = 0; im < nm; ++im) {
    const int m = im * mres;
    for (int t0 = m; t0 <= LR; t0 += kAnaTile) atiles.push_back(make_int4(im, t0, ckbase[im] + (t0 - m) / ckstep, 0));
  }
  const int natiles = (int)atiles.size();
  std::vector<double> alpha(npk, 0.0), cfac(npk, 1.0), dco(npk, 0.0);
  for (int im = 0; im < nm; ++im) {
    const int m = im * mres;
    const long long b = p->hoff[im];
    for (int l = m; l <= LR; ++l) {
      const long long k = b + (l - m);
      if (l >= m + 2) {
        const double bl = std::sqrt(((double)(2 * l + 1) * (double)(l - 1 - m) * (double)(l - 1 + m)) /
                                    ((double)(2 * l - 3) * (double)(l - m) * (double)(l + m)));
        const double al = std::sqrt(((double)(2 * l - 1) * (double)(2 * l + 1)) / ((double)(l - m) * (double)(l + m)));
        cfac[k] = bl * cfac[k - 2];
        alpha[k] = al * cfac[k - 1] / cfac[k];
      }
      dco[k] = (l == 0 || l == m) ? 0.0 : std::sqrt(std::max(0.0, (double)(l * l - m * m) / (double)(4 * l * l - 1)));
    }
  }
  std::vector<double> seedfac(mmax + 2, 0.0);
  for (int j = 1; j <= mmax; ++j) seedfac[j] = -std::sqrt((double)(2 * j + 1) / (double)(2 * j));
  std::vector<double2> tw(nlon);
  for (int t = 0; t < nlon; ++t) {
    // exact symmetric angles: reduce t/N to [0, 1/8] octant-free form via sincospi
    const double ang = -2.0 * (double)t / (double)nlon;  // in units of pi
    tw[t] = make_double2(std::cos(M_PI * ang), std::sin(M_PI * ang));
  }
  std::vector<int> rev(nlon);
  for (int k = 0; k < nlon; ++k) {
    if (p->fft.direct) { rev[k] = k; continue; }
    int pos = 0, kk = k, Ns = nlon;
    for (int s = 0; s < p->fft.nrad; ++s) {
      const int r = p->fft.rad[s];
      const int d = kk % r;
      kk /= r;
      Ns /= r;
      pos += d * Ns;
    }
    rev[k] = pos;
  }
  std::vector<int> rinv(nlon);
  for (int k = 0; k < nlon; ++k) rinv[rev[k]] = k;
  std::vector<float2> tw32(nlon);
  for (int t = 0; t < nlon; ++t) tw32[t] = make_float2((float)tw[t].x, (float)tw[t].y);
  std::vector<double2> twp;
  const int ntwp = fft_pass_twiddles(p->fft, twp);
  std::vector<float2> twp32(ntwp);
  for (int t = 0; t < ntwp; ++t) twp32[t] = make_float2((float)twp[t].x, (float)twp[t].y);

  // one device allocation for all tables
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = align_up(o + bytes, 256); return r; };
  const size_t o_x = take(nlat * 8), o_w = take(nlat * 8), o_s = take(nlat * 8);
  const size_t o_off = take((nm + 1) * 8), o_alpha = take(npk * 8), o_c = take(npk * 8), o_d = take(npk * 8);
  const size_t o_l0 = take((size_t)nm * npair * 4), o_r01 = take((size_t)nm * npair * 16);
  const size_t o_ck = take((size_t)nseg * npair * 16), o_ckbase = take((size_t)nm * 4);
  const size_t o_atiles = take((size_t)natiles * 16);
  const size_t o_scale = coeff_scale ? take((size_t)(lmax + 1) * (mmax + 1) * 8) : 0;
  const size_t o_tw = take((size_t)nlon * 16), o_tw32 = take((size_t)nlon * 8);
  const size_t o_seed = take((mmax + 2) * 8), o_rev = take((size_t)nlon * 4), o_rinv = take((size_t)nlon * 4);
  const size_t o_twp = take((size_t)ntwp * 16), o_twp32 = take((size_t)ntwp * 8);
  const size_t o_err = take(16);
  p->dbytes = o;
  cudaError_t ce = cudaMalloc(&p->dmem, o);
  if (ce != cudaSuccess) {
    delete p;
    return set_error(SHTB_ERR_OOM, std::string("plan tables: ") + cudaGetErrorString(ce));
  }
  char* D = (char*)p->dmem;
  auto up = [&](size_t off, const void* src, size_t bytes) {
    return cudaMemcpy(D + off, src, bytes, cudaMemcpyHostToDevice);
  };
  ce = cudaSuccess;
  if (ce == cudaSuccess) ce = up(o_x, x, nlat * 8);
  if (ce == cudaSuccess) ce = up(o_w, w, nlat * 8);
  if (ce == cudaSuccess) ce = up(o_s, p->hsint.data(), nlat * 8);
  if (ce == cudaSuccess) ce = up(o_off, p->hoff.data(), (nm + 1) * 8);
  if (ce == cudaSuccess) ce = up(o_alpha, alpha.data(), npk * 8);
  if (ce == cudaSuccess) ce = up(o_c, cfac.data(), npk * 8);
  if (ce == cudaSuccess) ce = up(o_d, dco.data(), npk * 8);
  if (ce == cudaSuccess) ce = up(o_ckbase, ckbase.data(), (size_t)nm * 4);
  if (ce == cudaSuccess) ce = up(o_atiles, atiles.data(), (size_t)natiles * 16);
  if (ce == cudaSuccess && coeff_scale) ce = up(o_scale, coeff_scale, (size_t)(lmax + 1) * (mmax + 1) * 8);
  if (ce == cudaSuccess) ce = up(o_tw, tw.data(), (size_t)nlon * 16);
  if (ce == cudaSuccess) ce = up(o_tw32, tw32.data(), (size_t)nlon * 8);
  if (ce == cudaSuccess) ce = up(o_seed, seedfac.data(), (mmax + 2) * 8);
  if (ce == cudaSuccess) ce = up(o_rev, rev.data(), (size_t)nlon * 4);
  if (ce == cudaSuccess) ce = up(o_rinv, rinv.data(), (size_t)nlon * 4);
  if (ce == cudaSuccess) ce = up(o_twp, twp.data(), (size_t)ntwp * 16);
  if (ce == cudaSuccess) ce = up(o_twp32, twp32.data(), (size_t)ntwp * 8);
  if (ce != cudaSuccess) {
    cudaFree(p->dmem);
    delete p;
    return set_error(SHTB_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(ce));
  }
  PlanDev& dv = p->dev;
  dv.lmax = lmax; dv.mmax = mmax; dv.mres = mres; dv.nlat = nlat; dv.nlon = nlon;
  dv.nm = nm; dv.npair = npair; dv.lrec = LR;
  dv.x = (const double*)(D + o_x);
  dv.w = (const double*)(D + o_w);
  dv.sint = (const double*)(D + o_s);
  dv.off = (const long long*)(D + o_off);
  dv.alpha = (const double*)(D + o_alpha);
  dv.cfac = (const double*)(D + o_c);
  dv.l0 = (const int*)(D + o_l0);
  dv.r01 = (const double2*)(D + o_r01);
  dv.ckpt = (const double2*)(D + o_ck);
  dv.ckbase = (const int*)(D + o_ckbase);
  dv.ckstep = ckstep;
  dv.atiles = (const int4*)(D + o_atiles);
  dv.natiles = natiles;
  p->d_scale = coeff_scale ? (const double*)(D + o_scale) : nullptr;
  p->d_tw64 = (const double2*)(D + o_tw);
  p->d_tw32 = (const float2*)(D + o_tw32);
  p->d_dcoef = (const double*)(D + o_d);
  p->d_rev = (const int*)(D + o_rev);
  p->d_rinv = (const int*)(D + o_rinv);
  p->d_twp64 = (const double2*)(D + o_twp);
  p->d_twp32 = (const float2*)(D + o_twp32);
  p->d_err = (int*)(D + o_err);
  if (ce == cudaSuccess) ce = cudaMemset(D + o_err, 0, 16);

  dim3 grid((npair + 127) / 128, nm);
  plan_setup_kernel<<<grid, 128>>>(dv, (const double*)(D + o_seed), (int*)(D + o_l0), (double2*)(D + o_r01),
                                   (double2*)(D + o_ck));
  count_launch();
  ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) {
    cudaFree(p->dmem);
    delete p;
    return set_error(SHTB_ERR_CUDA, std::string("plan setup kernel: ") + cudaGetErrorString(ce));
  }
  // the allocation-free synthesis's scratch on this device (shtb_synthesis_noalloc); a
  // failure here only disables that entry point
  ce = noalloc_scratch_address(&p->noalloc_scratch);
  if (ce != cudaSuccess || !p->noalloc_scratch) {
    p->noalloc_scratch = nullptr;
    p->noalloc_err = cudaGetErrorString(ce);
    cudaGetLastError();
  }
  *out = p;
  return SHTB_OK;
}

extern "C" int shtb_plan_destroy(shtb_plan* p) {
  if (!p) return SHTB_OK;
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device) cudaSetDevice(p->device);
  cudaError_t e = cudaFree(p->dmem);
  if (p->d_tab) cudaFree(p->d_tab);
  for (auto& lists : p->mx_lists)
    for (auto& kv : lists) {
      if (kv.second.tiles) cudaFree(kv.second.tiles);
      if (kv.second.masks) cudaFree(kv.second.masks);
    }
  if (dev >= 0 && dev != p->device) cudaSetDevice(dev);
  delete p;
  return check_cuda(e, "plan destroy");
}

extern "C" size_t shtb_plan_table_bytes(const shtb_plan* p) { return p ? p->dbytes + p->tab_bytes : 0; }

// Synchronizes the device and reports whether any kernel of this plan gave up a
// bounded wait since the last call (the status word is cleared).
extern "C" int shtb_plan_status(const shtb_plan* p) {
  if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan is NULL");
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(SHTB_ERR_CUDA, std::string("plan status: ") + cudaGetErrorString(e));
  if (h) {
    cudaMemset(p->d_err, 0, sizeof(int));
    return set_error(SHTB_ERR_TIMEOUT, "a device wait exceeded its time limit; results of the affected call are invalid");
  }
  return SHTB_OK;
}

// Test hook for the failure path of the bounded device waits: shortens the mixed GEMM
// kernels' wait limit and makes CTA 0's loader leave one chunk's copies unissued, so the
// wait for that chunk runs out, the CTA drains its own copies and MMAs, frees TMEM and
// exits, and shtb_plan_status reports SHTB_ERR_TIMEOUT. Nothing faults or hangs.
extern "C" int shtb_plan_debug_waits(shtb_plan* p, uint64_t wait_ns, int skip_chunk) {
  if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan is NULL");
  if (wait_ns > 10000000000ull) return set_error(SHTB_ERR_BAD_ARG, "wait_ns must be <= 10 s");
  p->dbg_wait_ns = wait_ns;
  p->dbg_skip_chunk = skip_chunk < 0 ? -1 : skip_chunk;
  return SHTB_OK;
}

// ---------------------------------------------------------------------------
// per-kernel event timing
// ---------------------------------------------------------------------------
namespace shtb {
struct ProfRec {
  std::string name;
  cudaEvent_t a, b;
};
static thread_local bool g_prof_on = false;
static thread_local std::vector<ProfRec> g_prof_recs;
static thread_local cudaEvent_t g_prof_pending = nullptr;

void prof_begin(cudaStream_t st) {
  if (!g_prof_on) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, st);
  g_prof_pending = e;
}

void prof_end(const char* name, cudaStream_t st) {
  if (!g_prof_on || !g_prof_pending) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, st);
  g_prof_recs.push_back(ProfRec{name, g_prof_pending, e});
  g_prof_pending = nullptr;
}
}  // namespace shtb

extern "C" int shtb_profile_enable(int on) {
  using namespace shtb;
  if (on && !g_prof_on) {
    for (auto& r : g_prof_recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    g_prof_recs.clear();
  }
  g_prof_on = on != 0;
  return SHTB_OK;
}

// Aggregates the recorded launches per kernel name (synchronizes their events).
// names: max*64 bytes, NUL-terminated entries. Returns the number of kernel kinds.
extern "C" int shtb_profile_read(int max, char* names, double* total_ms, int* count) {
  using namespace shtb;
  std::vector<std::string> keys;
  std::vector<double> tot;
  std::vector<int> cnt;
  for (auto& r : g_prof_recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) != cudaSuccess) return set_error(SHTB_ERR_CUDA, "profile event sync failed");
    cudaEventElapsedTime(&ms, r.a, r.b);
    size_t i = 0;
    while (i < keys.size() && keys[i] != r.name) ++i;
    if (i == keys.size()) { keys.push_back(r.name); tot.push_back(0.0); cnt.push_back(0); }
    tot[i] += ms;
    cnt[i] += 1;
  }
  const int n = (int)keys.size();
  for (int i = 0; i < n && i < max; ++i) {
    std::strncpy(names + 64 * i, keys[i].c_str(), 63);
    names[64 * i + 63] = 0;
    total_ms[i] = tot[i];
    count[i] = cnt[i];
  }
  return n;
}
