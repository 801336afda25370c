// group.cu — uneven batches: many independent mixed-precision scalar transforms, each
// with its own plan (lmax, Gauss grid, nlon) and 1..8 fields, run as four persistent
// launches (B packing, order-GEMM synthesis, FFT synthesis, FFT analysis, order-GEMM
// analysis).
//
// Every stage owns a list of work items over all members — GEMM tiles (member, order,
// first latitude pair or degree, parity) and FFT tiles (member, first latitude pair,
// field) — sorted by decreasing cost. A stage launches min(items, SMs x CTAs per SM)
// CTAs and CTA i runs items i, i + gridDim.x, ...: the longest tiles start first and
// the short ones fill in behind them, so a batch of mixed sizes keeps every SM busy
// without one launch per member. The six launches of a roundtrip (a start marker plus
// the five stages) are captured once into a CUDA graph and replayed.
//
// Per-member latency: the start marker records %globaltimer; the analysis GEMM stores,
// per member, the time its last tile finished.
//
// Launch-shape autotuning times every FFT shape (latitude pairs per CTA; 1, 2 or 4 CTAs
// per SM, the extra CTAs queueing behind the resident ones) on the bound buffers and
// keeps the fastest; the shape changes no result.
#include <algorithm>
#include <numeric>
#include <vector>

#include "kernels.cuh"

namespace shtb {

__global__ void group_start_kernel(unsigned long long* done, int n, unsigned long long* t0) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) done[i] = 0;
  if (threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *t0 = t;
  }
}

static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace shtb

using namespace shtb;

struct shtb_group {
  int n = 0, device = -1, nsm = 148;
  std::vector<const shtb_plan*> plans;
  std::vector<int> nf;
  std::vector<size_t> woff;             // byte offset of member t's Fourier buffer
  size_t argsz = 0, jobsz = 0;
  // device memory: [args syn | args ana | jobs syn | jobs ana | done | t0 | gemm items | W]
  unsigned char* dmem = nullptr;
  unsigned char *d_args_syn = nullptr, *d_args_ana = nullptr, *d_jobs_syn = nullptr, *d_jobs_ana = nullptr;
  unsigned long long *d_done = nullptr, *d_t0 = nullptr;
  int4 *d_items_syn = nullptr, *d_items_ana = nullptr;
  int2* d_items_pack = nullptr;
  int n_syn = 0, n_ana = 0, n_pack = 0;
  unsigned char* d_w = nullptr;
  int4* d_items_fft = nullptr;          // rebuilt when the FFT shape changes
  int n_fft = 0;
  // launch shape
  int fft_h = 8, fft_ctas = 148, gemm_ctas_syn = 148, gemm_ctas_ana = 148;
  bool generic = false;
  size_t fft_smem = 0;
  bool bound = false;
  // graph
  cudaStream_t priv = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void group_free(shtb_group* g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->ev_in) cudaEventDestroy(g->ev_in);
  if (g->ev_out) cudaEventDestroy(g->ev_out);
  if (g->priv) cudaStreamDestroy(g->priv);
  if (g->d_items_fft) cudaFree(g->d_items_fft);
  if (g->dmem) cudaFree(g->dmem);
  delete g;
}

static void drop_graph(shtb_group* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  g->exec = nullptr;
}

// FFT tiles for a given number of latitude pairs per CTA, longest rows first.
static int build_fft_items(shtb_group* g, int h) {
  std::vector<int4> it;
  std::vector<int> cost;
  for (int t = 0; t < g->n; ++t) {
    const shtb_plan* p = g->plans[t];
    for (int p0 = 0; p0 < p->npair; p0 += h)
      for (int k = 0; k < g->nf[t]; ++k) {
        it.push_back(make_int4(t, p0, k, 0));
        cost.push_back(p->nlon);
      }
  }
  std::vector<int> ord(it.size());
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int4> sorted(it.size());
  for (size_t i = 0; i < ord.size(); ++i) sorted[i] = it[ord[i]];
  if (g->d_items_fft) cudaFree(g->d_items_fft);
  g->d_items_fft = nullptr;
  SHTB_TRY_CUDA(cudaMalloc(&g->d_items_fft, std::max<size_t>(1, sorted.size()) * sizeof(int4)), "group fft items");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_items_fft, sorted.data(), sorted.size() * sizeof(int4), cudaMemcpyHostToDevice),
                "group fft items upload");
  g->n_fft = (int)sorted.size();
  return SHTB_OK;
}

static size_t group_fft_smem(const shtb_group* g, int h) {
  size_t s = 0;
  for (const shtb_plan* p : g->plans) s = std::max(s, fft_group_smem_f32(p, h));
  return s;
}

static int set_fft_shape(shtb_group* g, int h, int ctas) {
  int rc = build_fft_items(g, h);
  if (rc) return rc;
  g->fft_h = h;
  g->fft_smem = group_fft_smem(g, h);
  g->fft_ctas = std::max(1, std::min(ctas, g->n_fft));
  drop_graph(g);
  return SHTB_OK;
}

static int group_launch_stages(shtb_group* g, int op, cudaStream_t st) {
  int rc;
  if (op != SHTB_OP_ANALYSIS) {
    group_start_kernel<<<1, 256, 0, st>>>(g->d_done, g->n, g->d_t0);
    count_launch();
    SHTB_TRY_CUDA(cudaGetLastError(), "group start marker");
    if ((rc = launch_pack_group(g->d_args_syn, g->d_items_pack, g->n_pack, std::min(g->n_pack, 24 * g->nsm), st)))
      return rc;
    if ((rc = launch_gemm_group(0, g->d_args_syn, g->d_items_syn, g->n_syn, g->gemm_ctas_syn, nullptr, st))) return rc;
    if ((rc = launch_fft_group_f32(1, g->fft_h, g->generic, g->d_jobs_syn, g->d_items_fft, g->n_fft, g->fft_ctas,
                                   g->fft_smem, st)))
      return rc;
  }
  if (op != SHTB_OP_SYNTHESIS) {
    if ((rc = launch_fft_group_f32(0, g->fft_h, g->generic, g->d_jobs_ana, g->d_items_fft, g->n_fft, g->fft_ctas,
                                   g->fft_smem, st)))
      return rc;
    if ((rc = launch_gemm_group(1, g->d_args_ana, g->d_items_ana, g->n_ana, g->gemm_ctas_ana, g->d_done, st))) return rc;
  }
  return SHTB_OK;
}

static int check_device(const shtb_group* g) {
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != g->device) return set_error(SHTB_ERR_BAD_ARG, "the current CUDA device differs from the group's device");
  return SHTB_OK;
}

extern "C" int shtb_group_create(shtb_group** out, const shtb_plan* const* plans, int n, const int* nfields) {
  if (!out) return set_error(SHTB_ERR_BAD_ARG, "out is NULL");
  *out = nullptr;
  if (n < 1 || !plans || !nfields) return set_error(SHTB_ERR_BAD_ARG, "a group needs n >= 1 plans and field counts");
  int dev = -1;
  SHTB_TRY_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  for (int t = 0; t < n; ++t) {
    const shtb_plan* p = plans[t];
    if (!p) return set_error(SHTB_ERR_BAD_ARG, "plan " + std::to_string(t) + " is NULL");
    if (p->device != dev) return set_error(SHTB_ERR_BAD_ARG, "plan " + std::to_string(t) + " lives on another device");
    if (p->mres != 1) return set_error(SHTB_ERR_UNSUPPORTED, "group members need mres == 1");
    if (nfields[t] < 1 || nfields[t] > 8)
      return set_error(SHTB_ERR_BAD_ARG, "group members take 1..8 fields, got " + std::to_string(nfields[t]));
  }
  shtb_group* g = new (std::nothrow) shtb_group();
  if (!g) return set_error(SHTB_ERR_OOM, "group");
  g->n = n;
  g->device = dev;
  g->plans.assign(plans, plans + n);
  g->nf.assign(nfields, nfields + n);
  cudaDeviceGetAttribute(&g->nsm, cudaDevAttrMultiProcessorCount, dev);
  auto fail = [&](int rc) {
    group_free(g);
    return rc;
  };
  for (int t = 0; t < n; ++t) {
    int rc = mixed_prepare(plans[t], 0);
    if (rc) return fail(rc);
    g->generic = g->generic || fft_plan_generic(plans[t]);
  }
  // GEMM tiles, most K-steps first
  const int TM = mixed_group_tile_rows();
  std::vector<int4> syn, ana;
  std::vector<int> csyn, cana;
  for (int t = 0; t < n; ++t) {
    const shtb_plan* p = plans[t];
    const int mlim = std::min(p->mmax, p->lmax);
    for (int im = 0; im <= mlim; ++im) {
      for (int par = 0; par < 2; ++par) {
        for (int p0 = 0; p0 < p->npair; p0 += TM) {
          syn.push_back(make_int4(t, im, p0, par));
          csyn.push_back(mixed_group_ksteps(p, 0, im, par));
        }
        const int JE = (p->lmax - im) / 2 + 1;
        for (int j0 = 0; j0 < JE; j0 += TM) {
          ana.push_back(make_int4(t, im, j0, par));
          cana.push_back(mixed_group_ksteps(p, 1, im, par));
        }
      }
    }
  }
  auto sort_items = [](std::vector<int4>& it, const std::vector<int>& cost) {
    std::vector<int> ord(it.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int4> s(it.size());
    for (size_t i = 0; i < ord.size(); ++i) s[i] = it[ord[i]];
    it.swap(s);
  };
  sort_items(syn, csyn);
  sort_items(ana, cana);
  std::vector<int2> pack;   // (member, order) for the synthesis B packing, most degrees first
  {
    std::vector<int4> tmp;
    std::vector<int> cost;
    for (int t = 0; t < n; ++t)
      for (int im = 0; im <= std::min(plans[t]->mmax, plans[t]->lmax); ++im) {
        tmp.push_back(make_int4(t, im, 0, 0));
        cost.push_back(plans[t]->lmax - im);
      }
    sort_items(tmp, cost);
    for (const int4& v : tmp) pack.push_back(make_int2(v.x, v.y));
  }
  g->n_pack = (int)pack.size();
  g->n_syn = (int)syn.size();
  g->n_ana = (int)ana.size();
  // two GEMM CTAs of 16 columns fit on an SM
  g->gemm_ctas_syn = std::max(1, std::min(2 * g->nsm, g->n_syn));
  g->gemm_ctas_ana = std::max(1, std::min(2 * g->nsm, g->n_ana));
  // one device allocation
  g->argsz = mixed_args_bytes();
  g->jobsz = fft_job_bytes_f32();
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = align256(o + b); return r; };
  const size_t o_as = take(n * g->argsz), o_aa = take(n * g->argsz), o_js = take(n * g->jobsz), o_ja = take(n * g->jobsz);
  const size_t o_done = take(n * 8), o_t0 = take(8), o_is = take(syn.size() * sizeof(int4)),
               o_ia = take(ana.size() * sizeof(int4)), o_ip = take(pack.size() * sizeof(int2));
  g->woff.resize(n);
  size_t wbytes = 0;
  for (int t = 0; t < n; ++t) {
    g->woff[t] = wbytes;
    wbytes = align256(wbytes + std::max(mixed_workspace_bytes(plans[t], SHTB_OP_SYNTHESIS, g->nf[t]),
                                        mixed_workspace_bytes(plans[t], SHTB_OP_ANALYSIS, g->nf[t])));
  }
  const size_t o_w = take(wbytes);
  cudaError_t e = cudaMalloc(&g->dmem, o);
  if (e != cudaSuccess) return fail(set_error(SHTB_ERR_OOM, std::string("group buffers: ") + cudaGetErrorString(e)));
  g->d_args_syn = g->dmem + o_as;
  g->d_args_ana = g->dmem + o_aa;
  g->d_jobs_syn = g->dmem + o_js;
  g->d_jobs_ana = g->dmem + o_ja;
  g->d_done = (unsigned long long*)(g->dmem + o_done);
  g->d_t0 = (unsigned long long*)(g->dmem + o_t0);
  g->d_items_syn = (int4*)(g->dmem + o_is);
  g->d_items_ana = (int4*)(g->dmem + o_ia);
  g->d_items_pack = (int2*)(g->dmem + o_ip);
  g->d_w = g->dmem + o_w;
  e = cudaMemcpy(g->d_items_syn, syn.data(), syn.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_items_ana, ana.data(), ana.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_items_pack, pack.data(), pack.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(g->d_done, 0, n * 8);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->priv, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(set_error(SHTB_ERR_CUDA, std::string("group setup: ") + cudaGetErrorString(e)));
  // default FFT shape: the most latitude pairs per CTA that fit in ~200 KB
  int h = 16;
  while (h > 2 && group_fft_smem(g, h) > 200 * 1024) h >>= 1;
  int rc = set_fft_shape(g, h, g->nsm);
  if (rc) return fail(rc);
  *out = g;
  return SHTB_OK;
}

extern "C" int shtb_group_destroy(shtb_group* g) {
  if (!g) return SHTB_OK;
  group_free(g);
  return SHTB_OK;
}

extern "C" int shtb_group_bind(shtb_group* g, void* const* alm_in, void* const* grid, void* const* alm_out) {
  if (!g) return set_error(SHTB_ERR_BAD_ARG, "group is NULL");
  if (!alm_in || !grid || !alm_out) return set_error(SHTB_ERR_BAD_ARG, "NULL buffer array");
  int rc = check_device(g);
  if (rc) return rc;
  std::vector<unsigned char> as(g->n * g->argsz), aa(g->n * g->argsz), js(g->n * g->jobsz), ja(g->n * g->jobsz);
  for (int t = 0; t < g->n; ++t) {
    if (!alm_in[t] || !grid[t] || !alm_out[t])
      return set_error(SHTB_ERR_BAD_ARG, "NULL buffer for member " + std::to_string(t));
    if ((((uintptr_t)alm_in[t]) | ((uintptr_t)grid[t]) | ((uintptr_t)alm_out[t])) & 15u)
      return set_error(SHTB_ERR_ALIGN, "buffers must be 16-byte aligned");
    const shtb_plan* p = g->plans[t];
    void* W = g->d_w + g->woff[t];
    mixed_fill_args(p, 0, alm_in[t], W, g->nf[t], as.data() + t * g->argsz);
    mixed_fill_args(p, 1, W, alm_out[t], g->nf[t], aa.data() + t * g->argsz);
    fft_fill_job_f32(p, 1, W, grid[t], g->nf[t], js.data() + t * g->jobsz);
    fft_fill_job_f32(p, 0, W, grid[t], g->nf[t], ja.data() + t * g->jobsz);
  }
  SHTB_TRY_CUDA(cudaMemcpy(g->d_args_syn, as.data(), as.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_args_ana, aa.data(), aa.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs_syn, js.data(), js.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs_ana, ja.data(), ja.size(), cudaMemcpyHostToDevice), "group bind");
  g->bound = true;
  drop_graph(g);
  return SHTB_OK;
}

extern "C" int shtb_group_launch(shtb_group* g, int op, void* stream) {
  if (!g) return set_error(SHTB_ERR_BAD_ARG, "group is NULL");
  if (!g->bound) return set_error(SHTB_ERR_BAD_ARG, "group buffers are not bound");
  if (op != -1 && op != SHTB_OP_SYNTHESIS && op != SHTB_OP_ANALYSIS) return set_error(SHTB_ERR_BAD_ARG, "unknown op");
  int rc = check_device(g);
  if (rc) return rc;
  return group_launch_stages(g, op, (cudaStream_t)stream);
}

extern "C" int shtb_group_roundtrip(shtb_group* g, void* stream) {
  if (!g) return set_error(SHTB_ERR_BAD_ARG, "group is NULL");
  if (!g->bound) return set_error(SHTB_ERR_BAD_ARG, "group buffers are not bound");
  int rc = check_device(g);
  if (rc) return rc;
  if (!g->exec) {
    const uint64_t before = shtb_launch_count(0);
    SHTB_TRY_CUDA(cudaStreamBeginCapture(g->priv, cudaStreamCaptureModeThreadLocal), "group capture begin");
    rc = group_launch_stages(g, -1, g->priv);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g->priv, &graph);
    count_launch(-(int)(shtb_launch_count(0) - before));   // capturing runs no kernel
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return set_error(SHTB_ERR_CUDA, std::string("group capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      g->exec = nullptr;
      return set_error(SHTB_ERR_CUDA, std::string("group graph instantiate: ") + cudaGetErrorString(ei));
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  SHTB_TRY_CUDA(cudaEventRecord(g->ev_in, st), "group event");
  SHTB_TRY_CUDA(cudaStreamWaitEvent(g->priv, g->ev_in, 0), "group wait");
  SHTB_TRY_CUDA(cudaGraphLaunch(g->exec, g->priv), "group graph launch");
  count_launch(6);   // start marker, B packing and four stage kernels
  SHTB_TRY_CUDA(cudaEventRecord(g->ev_out, g->priv), "group event");
  SHTB_TRY_CUDA(cudaStreamWaitEvent(st, g->ev_out, 0), "group wait");
  return SHTB_OK;
}

extern "C" int shtb_group_autotune(shtb_group* g, void* stream) {
  if (!g) return set_error(SHTB_ERR_BAD_ARG, "group is NULL");
  if (!g->bound) return set_error(SHTB_ERR_BAD_ARG, "group buffers are not bound");
  int rc = check_device(g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  SHTB_TRY_CUDA(cudaStreamSynchronize(st), "group autotune sync");
  cudaEvent_t e0, e1;
  SHTB_TRY_CUDA(cudaEventCreate(&e0), "event");
  SHTB_TRY_CUDA(cudaEventCreate(&e1), "event");
  float best = 1e30f;
  int bh = g->fft_h, bc = g->fft_ctas;
  for (int h : {16, 8, 4}) {
    if (group_fft_smem(g, h) > 200 * 1024) continue;
    for (int mult : {1, 2, 4}) {
      if ((rc = set_fft_shape(g, h, g->nsm * mult))) break;
      float ms_min = 1e30f;
      for (int rep = 0; rep < 3 && !rc; ++rep) {
        cudaEventRecord(e0, g->priv);
        rc = group_launch_stages(g, -1, g->priv);
        cudaEventRecord(e1, g->priv);
        if (!rc && cudaEventSynchronize(e1) == cudaSuccess) {
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          ms_min = std::min(ms_min, ms);
        }
      }
      if (rc) break;
      if (ms_min < best) {
        best = ms_min;
        bh = h;
        bc = g->fft_ctas;
      }
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  SHTB_TRY_CUDA(cudaStreamSynchronize(g->priv), "group autotune");
  return set_fft_shape(g, bh, bc);
}

extern "C" int shtb_group_config(const shtb_group* g, int* fft_pairs, int* fft_ctas, int* gemm_ctas) {
  if (!g) return set_error(SHTB_ERR_BAD_ARG, "group is NULL");
  if (fft_pairs) *fft_pairs = g->fft_h;
  if (fft_ctas) *fft_ctas = g->fft_ctas;
  if (gemm_ctas) *gemm_ctas = g->gemm_ctas_syn;
  return SHTB_OK;
}

extern "C" int shtb_group_latency_ns(const shtb_group* g, uint64_t* ns) {
  if (!g || !ns) return set_error(SHTB_ERR_BAD_ARG, "NULL argument");
  std::vector<unsigned long long> done(g->n);
  unsigned long long t0 = 0;
  SHTB_TRY_CUDA(cudaMemcpy(done.data(), g->d_done, g->n * 8, cudaMemcpyDeviceToHost), "group latency read");
  SHTB_TRY_CUDA(cudaMemcpy(&t0, g->d_t0, 8, cudaMemcpyDeviceToHost), "group latency read");
  for (int t = 0; t < g->n; ++t) ns[t] = done[t] > t0 ? (uint64_t)(done[t] - t0) : 0;
  return SHTB_OK;
}
