/*
 * sht_oracle.c — C restatement of SHTnsKit.jl's CPU scalar transforms.
 *
 * TEST INFRASTRUCTURE AND CPU BASELINE ONLY: used by tests/ as a fast checker and
 * by bench.py as the timed CPU baseline ("port" of the reference's CPU path).
 * The product (the CUDA library) never links or calls it.
 *
 * Algorithm (paths within the SHTnsKit.jl project):
 *   - per (m, latitude) the full orthonormal + Condon-Shortley row P̄_l^m(x_i),
 *     l = m..lmax, with the 2^-480 / 2^960 extended-range sectoral seed
 *     (src/legendre.jl:233-322) — no equatorial symmetry, as the reference;
 *   - m processed in the zig-zag order 0, M, 1, M-1, ... (src/buffer_utils.jl:16-25)
 *     with static scheduling (src/core_transforms.jl:734-746, :808-869);
 *   - batches reuse each P̄ row across fields (src/batch_transforms.jl:403-425, :519-536);
 *   - synthesis: F[i,m] = phi_inv_scale * sum_l P̄ a, Hermitian fill, inverse FFT,
 *     real part (src/core_transforms.jl:294-344); analysis: FFT then
 *     a_lm = analysis_phi_scale * sum_i w_i P̄ F[i,m] (src/core_transforms.jl:169-207).
 * The longitude FFT is a plain recursive mixed-radix (2, 3, 5, generic) FFT written
 * here (the reference uses FFTW). Canonical normalization only. Threads are
 * POSIX threads with a static block partition (the reference's `:static`).
 *
 * Layouts: grid f[i + nlat*j + nlat*nlon*k]; coefficients complex
 * a[l + (lmax+1)*m + (lmax+1)*(mmax+1)*k] as interleaved (re, im) doubles.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <pthread.h>
#include <string.h>
#include <unistd.h>

typedef double complex cplx;

static const double INV_SQRT_4PI = 0.28209479177387814;

/* ---------------------------------------------------------------- P̄ rows */
static void plm_norm_row(double* P, double x, int lmax, int m) {
  for (int l = 0; l <= lmax; ++l) P[l] = 0.0;
  if (lmax < m) return;
  const double s = sqrt(fmax(0.0, (1.0 - x) * (1.0 + x)));
  const double TINY = ldexp(1.0, -480), HUGE_ = ldexp(1.0, 480), UP = ldexp(1.0, 960), DOWN = ldexp(1.0, -960);
  double pmm = INV_SQRT_4PI;
  int e = 0;
  for (int k = 1; k <= m; k += 8) {
    const int kend = k + 7 < m ? k + 7 : m;
    for (int j = k; j <= kend; ++j) pmm = (-sqrt((double)(2 * j + 1) / (double)(2 * j)) * s) * pmm;
    while (fabs(pmm) < TINY && pmm != 0.0) {
      pmm *= UP;
      e -= 960;
    }
  }
  int l = m + 2;
  if (e != 0) {
    double factor = ldexp(1.0, e);
    P[m] = pmm * factor;
    if (lmax == m) return;
    double p2 = pmm, p1 = sqrt((double)(2 * m + 3)) * x * pmm;
    P[m + 1] = p1 * factor;
    while (l <= lmax) {
      const double a = sqrt(((double)(2 * l - 1) * (double)(2 * l + 1)) / ((double)(l - m) * (double)(l + m)));
      const double b = sqrt(((double)(2 * l + 1) * (double)(l - 1 - m) * (double)(l - 1 + m)) /
                            ((double)(2 * l - 3) * (double)(l - m) * (double)(l + m)));
      const double p = a * x * p1 - b * p2;
      P[l] = p * factor;
      p2 = p1;
      p1 = p;
      ++l;
      const double mag = fmax(fabs(p2), fabs(p1));
      if (mag > HUGE_) {
        p2 *= DOWN;
        p1 *= DOWN;
        e += 960;
        if (e == 0) break;
        factor = ldexp(1.0, e);
      } else if (mag < TINY && mag != 0.0) {
        p2 *= UP;
        p1 *= UP;
        e -= 960;
        factor = ldexp(1.0, e);
      }
    }
  } else {
    P[m] = pmm;
    if (lmax == m) return;
    P[m + 1] = sqrt((double)(2 * m + 3)) * x * pmm;
  }
  for (; l <= lmax; ++l) {
    const double a = sqrt(((double)(2 * l - 1) * (double)(2 * l + 1)) / ((double)(l - m) * (double)(l + m)));
    const double b = sqrt(((double)(2 * l + 1) * (double)(l - 1 - m) * (double)(l - 1 + m)) /
                          ((double)(2 * l - 3) * (double)(l - m) * (double)(l + m)));
    P[l] = a * x * P[l - 1] - b * P[l - 2];
  }
}

/* ---------------------------------------------------------------- FFT */
/* out[k] = sum_j in[j*stride] * exp(sign*2*pi*i*j*k/n), recursive mixed radix */
static void fft_rec(const cplx* in, cplx* out, int n, int stride, int sign, cplx* tmp) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int r = 0;
  const int primes[] = {4, 2, 3, 5};
  for (int t = 0; t < 4; ++t)
    if (n % primes[t] == 0) { r = primes[t]; break; }
  if (r == 0) { /* generic: smallest factor, or direct DFT for a prime */
    for (int p = 7; p * p <= n; p += 2)
      if (n % p == 0) { r = p; break; }
    if (r == 0) {
      for (int k = 0; k < n; ++k) {
        cplx acc = 0;
        for (int j = 0; j < n; ++j) {
          const double ang = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / n;
          acc += in[(size_t)j * stride] * (cos(ang) + I * sin(ang));
        }
        out[k] = acc;
      }
      return;
    }
  }
  const int m = n / r;
  /* sub-transforms of the r decimated sequences into out[q*m ...] */
  for (int q = 0; q < r; ++q) fft_rec(in + (size_t)q * stride, out + (size_t)q * m, m, stride * r, sign, tmp);
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < r; ++q) {
      const double ang = sign * 2.0 * M_PI * (double)q * k / n;
      tmp[q] = out[(size_t)q * m + k] * (cos(ang) + I * sin(ang));
    }
    for (int s = 0; s < r; ++s) {
      cplx acc = 0;
      for (int q = 0; q < r; ++q) {
        const double ang = sign * 2.0 * M_PI * (double)((q * s) % r) / r;
        acc += tmp[q] * (cos(ang) + I * sin(ang));
      }
      tmp[r + s] = acc;
    }
    for (int s = 0; s < r; ++s) out[(size_t)s * m + k] = tmp[r + s];
  }
}

static void balanced_m_order(int mmax, int mres, int* order, int* n_out) {
  const int n = mmax / mres + 1;
  for (int i = 0; i < n; ++i) order[i] = ((i % 2 == 0) ? i / 2 : (n - 1) - i / 2) * mres;
  *n_out = n;
}

/* ---------------------------------------------------------------- threads */
typedef void (*range_fn)(void* ctx, long long lo, long long hi, int tid);
typedef struct {
  range_fn fn;
  void* ctx;
  long long lo, hi;
  int tid;
} job_t;
static void* job_run(void* a) {
  job_t* j = (job_t*)a;
  j->fn(j->ctx, j->lo, j->hi, j->tid);
  return NULL;
}
static int g_threads = 0;
static int resolve_threads(int nthreads) {
  if (nthreads > 0) return nthreads;
  if (g_threads > 0) return g_threads;
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}
/* static partition of [0, n) into nthreads contiguous blocks */
static void parallel_for(long long n, int nthreads, range_fn fn, void* ctx) {
  const int T = nthreads < 1 ? 1 : nthreads;
  pthread_t th[256];
  job_t jobs[256];
  const int nt = T > 256 ? 256 : T;
  for (int t = 0; t < nt; ++t) {
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].lo = n * t / nt;
    jobs[t].hi = n * (t + 1) / nt;
    jobs[t].tid = t;
    if (t > 0) pthread_create(&th[t], NULL, job_run, &jobs[t]);
  }
  job_run(&jobs[0]);
  for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
}

/* ---------------------------------------------------------------- transforms */
typedef struct {
  int lmax, mmax, nlat, nlon, nf;
  const double* x;
  const double* w;
  const cplx* a_in;
  cplx* a_out;
  const double* f_in;
  double* f_out;
  cplx* F;
  const int* order;
  double scale;
} job_ctx;

static void syn_legendre(void* c, long long lo, long long hi, int tid) {
  job_ctx* J = (job_ctx*)c;
  (void)tid;
  const size_t lda = (size_t)(J->lmax + 1) * (J->mmax + 1);
  double* P = (double*)malloc(sizeof(double) * (J->lmax + 1));
  for (long long idx = lo; idx < hi; ++idx) {
    const int m = J->order[idx];
    for (int i = 0; i < J->nlat; ++i) {
      plm_norm_row(P, J->x[i], J->lmax, m);
      for (int k = 0; k < J->nf; ++k) {
        const cplx* ak = J->a_in + k * lda + (size_t)m * (J->lmax + 1);
        cplx acc = 0;
        for (int l = m; l <= J->lmax; ++l) acc += P[l] * ak[l];
        J->F[((size_t)k * (J->mmax + 1) + m) * J->nlat + i] = J->scale * acc;
      }
    }
  }
  free(P);
}

static void syn_fft(void* c, long long lo, long long hi, int tid) {
  job_ctx* J = (job_ctx*)c;
  (void)tid;
  const int nlon = J->nlon, nlat = J->nlat, mmax = J->mmax;
  cplx* row = (cplx*)malloc(sizeof(cplx) * nlon);
  cplx* res = (cplx*)malloc(sizeof(cplx) * nlon);
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * 2 * (nlon + 1));
  for (long long ki = lo; ki < hi; ++ki) {
    const int k = (int)(ki / nlat), i = (int)(ki % nlat);
    for (int j = 0; j < nlon; ++j) row[j] = 0;
    for (int m = 0; m <= mmax; ++m) row[m] = J->F[((size_t)k * (mmax + 1) + m) * nlat + i];
    for (int m = 1; m <= mmax; ++m) row[nlon - m] = conj(row[m]);
    fft_rec(row, res, nlon, 1, +1, tmp);
    for (int j = 0; j < nlon; ++j) J->f_out[(size_t)k * nlat * nlon + (size_t)j * nlat + i] = creal(res[j]) / nlon;
  }
  free(row);
  free(res);
  free(tmp);
}

static void ana_fft(void* c, long long lo, long long hi, int tid) {
  job_ctx* J = (job_ctx*)c;
  (void)tid;
  const int nlon = J->nlon, nlat = J->nlat, mmax = J->mmax;
  cplx* row = (cplx*)malloc(sizeof(cplx) * nlon);
  cplx* res = (cplx*)malloc(sizeof(cplx) * nlon);
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * 2 * (nlon + 1));
  for (long long ki = lo; ki < hi; ++ki) {
    const int k = (int)(ki / nlat), i = (int)(ki % nlat);
    for (int j = 0; j < nlon; ++j) row[j] = J->f_in[(size_t)k * nlat * nlon + (size_t)j * nlat + i];
    fft_rec(row, res, nlon, 1, -1, tmp);
    for (int m = 0; m <= mmax; ++m) J->F[((size_t)k * (mmax + 1) + m) * nlat + i] = res[m];
  }
  free(row);
  free(res);
  free(tmp);
}

static void ana_legendre(void* c, long long lo, long long hi, int tid) {
  job_ctx* J = (job_ctx*)c;
  (void)tid;
  const size_t lda = (size_t)(J->lmax + 1) * (J->mmax + 1);
  double* P = (double*)malloc(sizeof(double) * (J->lmax + 1));
  for (long long idx = lo; idx < hi; ++idx) {
    const int m = J->order[idx];
    for (int i = 0; i < J->nlat; ++i) {
      plm_norm_row(P, J->x[i], J->lmax, m);
      const double wi = J->w[i] * J->scale;
      for (int k = 0; k < J->nf; ++k) {
        const cplx Fi = J->F[((size_t)k * (J->mmax + 1) + m) * J->nlat + i];
        cplx* ak = J->a_out + k * lda + (size_t)m * (J->lmax + 1);
        for (int l = m; l <= J->lmax; ++l) ak[l] += (wi * P[l]) * Fi;
      }
    }
  }
  free(P);
}

int oracle_synthesis_batch(int lmax, int mmax, int mres, int nlat, int nlon, const double* x, const double* alm,
                           double* f, int nf, double phi_inv_scale, int nthreads) {
  const int T = resolve_threads(nthreads);
  job_ctx J;
  memset(&J, 0, sizeof J);
  J.lmax = lmax; J.mmax = mmax; J.nlat = nlat; J.nlon = nlon; J.nf = nf;
  J.x = x; J.a_in = (const cplx*)alm; J.f_out = f; J.scale = phi_inv_scale;
  J.F = (cplx*)calloc((size_t)nf * nlat * (mmax + 1), sizeof(cplx)); /* F[k][m][i] */
  int* order = (int*)malloc(sizeof(int) * (mmax + 1));
  int nm;
  balanced_m_order(mmax, mres, order, &nm);
  J.order = order;
  parallel_for(nm, T, syn_legendre, &J);
  parallel_for((long long)nf * nlat, T, syn_fft, &J);
  free(J.F);
  free(order);
  return 0;
}

int oracle_analysis_batch(int lmax, int mmax, int mres, int nlat, int nlon, const double* x, const double* w,
                          const double* f, double* alm, int nf, double ana_scale, int nthreads) {
  const int T = resolve_threads(nthreads);
  job_ctx J;
  memset(&J, 0, sizeof J);
  J.lmax = lmax; J.mmax = mmax; J.nlat = nlat; J.nlon = nlon; J.nf = nf;
  J.x = x; J.w = w; J.f_in = f; J.a_out = (cplx*)alm; J.scale = ana_scale;
  J.F = (cplx*)malloc((size_t)nf * nlat * (mmax + 1) * sizeof(cplx));
  parallel_for((long long)nf * nlat, T, ana_fft, &J);
  memset(alm, 0, sizeof(cplx) * (size_t)(lmax + 1) * (mmax + 1) * nf);
  int* order = (int*)malloc(sizeof(int) * (mmax + 1));
  int nm;
  balanced_m_order(mmax, mres, order, &nm);
  J.order = order;
  parallel_for(nm, T, ana_legendre, &J);
  free(J.F);
  free(order);
  return 0;
}

int oracle_max_threads(void) { return resolve_threads(0); }
