// group.cu — uneven batches: many independent mixed-precision scalar transforms, each
// with its own plan (lmax, Gauss grid, nlon) and 1..8 fields, run as persistent stage
// launches: B packing and order-GEMM synthesis for members with three or more fields, the
// FP64-pipe synthesis (simt.cu) for members with one or two, FFT synthesis, FFT analysis and
// order-GEMM analysis.
//
// Every stage owns a list of work items over all members — GEMM tiles (member, order,
// first latitude pair or degree, parity, with the tile's live-chunk mask: chunks whose P
// image is all zero are skipped), FP64-pipe items (member, order, block of 32 latitude
// pairs, one per warp) and FFT tiles (member, first latitude pair, field) — sorted by
// decreasing cost, and a device work counter (zeroed by a memset at the start of every
// roundtrip). A stage launches min(items, SMs x CTAs per SM) persistent CTAs; each claims
// the next item with an atomicAdd on the counter whenever it has room for one, so the
// longest tiles start first and the short ones fill in behind whichever CTA frees up first,
// and a batch of mixed sizes keeps every SM busy without one launch per member. Members
// whose FFTs the packed-pair kernels take (fft2_applicable) run them in a second persistent
// FFT kernel per direction, forked beside the general one, and the FP64-pipe synthesis is
// forked beside the packing and GEMM synthesis, so every member's results equal its
// single-plan calls bit for bit. The memset and the launches of a roundtrip (a start marker
// plus the stages) are captured once into a CUDA graph and replayed.
//
// Per-member latency: the start marker records %globaltimer; the analysis GEMM stores,
// per member, the time its last tile finished.
//
// Launch-shape autotuning times, on the bound buffers, every FFT shape (latitude pairs per
// CTA; 1, 2 or 4 CTAs per SM, the extra CTAs queueing behind the resident ones), then one
// or two GEMM CTAs per SM for the synthesis and for the analysis GEMM, and keeps the
// fastest; the shape changes no result.
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

// work counters: pack, GEMM syn, FFT syn, FFT ana, GEMM ana, fft2 syn, fft2 ana, FP64-pipe syn
constexpr int kGroupQueues = 8;

}  // namespace shtb

using namespace shtb;

struct shtb_group {
  int n = 0, device = -1, nsm = 148;
  std::vector<const shtb_plan*> plans;
  std::vector<int> nf;
  std::vector<size_t> woff;             // byte offset of member t's Fourier buffer
  std::vector<char> f2;                 // member runs the packed-pair FFTs (fft2_applicable)
  std::vector<char> simt;               // member's Legendre synthesis runs on the FP64 pipes (simt_applicable)
  size_t sargsz = 0;
  unsigned char* d_sargs = nullptr;
  int4* d_items_ssyn = nullptr;
  int n_ssyn = 0, ssyn_ctas = 148;
  size_t ssyn_smem = 0;
  size_t argsz = 0, jobsz = 0, job2sz = 0;
  // device memory: [args syn | args ana | jobs syn | jobs ana | done | t0 | gemm items | W]
  unsigned char* dmem = nullptr;
  unsigned char *d_args_syn = nullptr, *d_args_ana = nullptr, *d_jobs_syn = nullptr, *d_jobs_ana = nullptr;
  unsigned char *d_jobs2_syn = nullptr, *d_jobs2_ana = nullptr;
  int4* d_items_fft2 = nullptr;         // packed-pair FFT items (members with f2 set)
  int n_fft2 = 0, fft2_ctas = 148;
  size_t fft2_smem = 0;
  unsigned long long *d_done = nullptr, *d_t0 = nullptr;
  int* d_queue = nullptr;               // work counters (kGroupQueues)
  int4 *d_items_syn = nullptr, *d_items_ana = nullptr;
  unsigned long long *d_masks_syn = nullptr, *d_masks_ana = nullptr;   // live-chunk mask per GEMM item
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
  cudaStream_t priv = nullptr, aux = nullptr;   // aux: the packed-pair FFTs, forked beside the others
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr, ev_join = nullptr;
  int graph_kernels = 0;
  cudaGraphExec_t exec = nullptr;
};

static void group_free(shtb_group* g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->ev_in) cudaEventDestroy(g->ev_in);
  if (g->ev_out) cudaEventDestroy(g->ev_out);
  if (g->ev_fork) cudaEventDestroy(g->ev_fork);
  if (g->ev_join) cudaEventDestroy(g->ev_join);
  if (g->priv) cudaStreamDestroy(g->priv);
  if (g->aux) cudaStreamDestroy(g->aux);
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
    if (g->f2[t]) continue;
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
  for (int t = 0; t < g->n; ++t)
    if (!g->f2[t]) s = std::max(s, fft_group_smem_f32(g->plans[t], h));
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

// One FFT stage: the packed-pair kernel of the fft2 members on the aux stream, forked from
// and joined back into st, beside the general kernel of the others on st.
static int group_fft_stage(shtb_group* g, int syn, int* q_gen, int* q_f2, cudaStream_t st) {
  int rc;
  const bool fork = g->n_fft2 > 0 && g->n_fft > 0;
  if (fork) {
    SHTB_TRY_CUDA(cudaEventRecord(g->ev_fork, st), "group fork");
    SHTB_TRY_CUDA(cudaStreamWaitEvent(g->aux, g->ev_fork, 0), "group fork");
  }
  if ((rc = launch_fft2_group(syn, syn ? g->d_jobs2_syn : g->d_jobs2_ana, g->d_items_fft2, g->n_fft2, g->fft2_ctas,
                              g->fft2_smem, q_f2, fork ? g->aux : st)))
    return rc;
  if ((rc = launch_fft_group_f32(syn, g->fft_h, g->generic, syn ? g->d_jobs_syn : g->d_jobs_ana, g->d_items_fft,
                                 g->n_fft, g->fft_ctas, g->fft_smem, q_gen, st)))
    return rc;
  if (fork) {
    SHTB_TRY_CUDA(cudaEventRecord(g->ev_join, g->aux), "group join");
    SHTB_TRY_CUDA(cudaStreamWaitEvent(st, g->ev_join, 0), "group join");
  }
  return SHTB_OK;
}

// The Legendre synthesis stage: the FP64-pipe kernel of the one- and two-field members on the
// aux stream, forked from and joined back into st, beside the packing and tensor-core GEMM of
// the others on st.
static int group_synthesis_stage(shtb_group* g, int* q, cudaStream_t st) {
  int rc;
  const bool fork = g->n_ssyn > 0 && g->n_syn > 0;
  if (fork) {
    SHTB_TRY_CUDA(cudaEventRecord(g->ev_fork, st), "group fork");
    SHTB_TRY_CUDA(cudaStreamWaitEvent(g->aux, g->ev_fork, 0), "group fork");
  }
  if ((rc = launch_simt_group(g->d_sargs, g->d_items_ssyn, g->n_ssyn, g->ssyn_ctas, g->ssyn_smem, q + 7,
                              fork ? g->aux : st)))
    return rc;
  if ((rc = launch_pack_group(g->d_args_syn, g->d_items_pack, g->n_pack, std::min(g->n_pack, 24 * g->nsm), q, st)))
    return rc;
  if ((rc = launch_gemm_group(0, g->d_args_syn, g->d_items_syn, g->d_masks_syn, g->n_syn, g->gemm_ctas_syn, nullptr, q + 1, st)))
    return rc;
  if (fork) {
    SHTB_TRY_CUDA(cudaEventRecord(g->ev_join, g->aux), "group join");
    SHTB_TRY_CUDA(cudaStreamWaitEvent(st, g->ev_join, 0), "group join");
  }
  return SHTB_OK;
}

static int group_launch_stages(shtb_group* g, int op, cudaStream_t st) {
  int rc;
  int* q = g->d_queue;
  SHTB_TRY_CUDA(cudaMemsetAsync(q, 0, kGroupQueues * sizeof(int), st), "group work counters");
  if (op != SHTB_OP_ANALYSIS) {
    group_start_kernel<<<1, 256, 0, st>>>(g->d_done, g->n, g->d_t0);
    count_launch();
    SHTB_TRY_CUDA(cudaGetLastError(), "group start marker");
    if ((rc = group_synthesis_stage(g, q, st))) return rc;
    if ((rc = group_fft_stage(g, 1, q + 2, q + 5, st))) return rc;
  }
  if (op != SHTB_OP_SYNTHESIS) {
    if ((rc = group_fft_stage(g, 0, q + 3, q + 6, st))) return rc;
    if ((rc = launch_gemm_group(1, g->d_args_ana, g->d_items_ana, g->d_masks_ana, g->n_ana, g->gemm_ctas_ana, g->d_done, q + 4, st)))
      return rc;
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
  g->f2.resize(n);
  g->simt.resize(n);
  for (int t = 0; t < n; ++t) {
    g->simt[t] = simt_applicable(plans[t], nfields[t]) ? 1 : 0;
    int rc = mixed_prepare(plans[t], 0);   // the analysis GEMM reads the plan's P table
    if (rc) return fail(rc);
    g->f2[t] = fft2_applicable(plans[t]) ? 1 : 0;
    if (!g->f2[t]) g->generic = g->generic || fft_plan_generic(plans[t]);
  }
  // packed-pair FFT items: blocks of fft2_group_pairs() pairs, longest rows first
  std::vector<int4> f2items;
  {
    std::vector<int> cost;
    const int hp = fft2_group_pairs();
    for (int t = 0; t < n; ++t) {
      if (!g->f2[t]) continue;
      g->fft2_smem = std::max(g->fft2_smem, fft2_group_smem(plans[t]));
      for (int p0 = 0; p0 < plans[t]->npair; p0 += hp)
        for (int k = 0; k < nfields[t]; ++k) {
          f2items.push_back(make_int4(t, p0, k, 0));
          cost.push_back(plans[t]->nlon);
        }
    }
    std::vector<int> ord(f2items.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int4> sorted(f2items.size());
    for (size_t i = 0; i < ord.size(); ++i) sorted[i] = f2items[ord[i]];
    f2items.swap(sorted);
  }
  g->n_fft2 = (int)f2items.size();
  g->fft2_ctas = std::max(1, std::min(g->nsm, g->n_fft2));
  // GEMM tiles with their live-chunk masks, most live K-steps first
  const int TM = mixed_group_tile_rows();
  std::vector<int4> syn, ana;
  std::vector<unsigned long long> msyn, mana;
  std::vector<int> csyn, cana;
  // FP64-pipe synthesis items of the one- and two-field members, most work first
  std::vector<int4> ssyn;
  std::vector<int> cssyn;
  for (int t = 0; t < n; ++t) {
    if (!g->simt[t]) continue;
    const shtb_plan* p = plans[t];
    const int mlim = std::min(p->mmax, p->lmax);
    g->ssyn_smem = std::max(g->ssyn_smem, simt_group_syn_smem(p));
    for (int im = 0; im <= mlim; ++im)
      for (int pb = 0; pb < simt_syn_pair_blocks(p); ++pb) {
        ssyn.push_back(make_int4(t, im, pb, 0));
        cssyn.push_back(p->lmax - im + 1);
      }
  }
  for (int t = 0; t < n; ++t) {
    const shtb_plan* p = plans[t];
    const int mlim = std::min(p->mmax, p->lmax);
    for (int im = 0; im <= mlim; ++im) {
      for (int par = 0; par < 2; ++par) {
        for (int p0 = 0; !g->simt[t] && p0 < p->npair; p0 += TM) {
          int c = 0;
          msyn.push_back(mixed_group_tile(p, 0, im, p0, par, &c));
          syn.push_back(make_int4(t, im, p0, par));
          csyn.push_back(c);
        }
        const int JE = (p->lmax - im) / 2 + 1;
        for (int j0 = 0; j0 < JE; j0 += TM) {
          int c = 0;
          mana.push_back(mixed_group_tile(p, 1, im, j0, par, &c));
          ana.push_back(make_int4(t, im, j0, par));
          cana.push_back(c);
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
  auto sort_masked = [](std::vector<int4>& it, std::vector<unsigned long long>& mk, const std::vector<int>& cost) {
    std::vector<int> ord(it.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int4> s(it.size());
    std::vector<unsigned long long> sm(mk.size());
    for (size_t i = 0; i < ord.size(); ++i) {
      s[i] = it[ord[i]];
      sm[i] = mk[ord[i]];
    }
    it.swap(s);
    mk.swap(sm);
  };
  sort_masked(syn, msyn, csyn);
  sort_masked(ana, mana, cana);
  sort_items(ssyn, cssyn);
  std::vector<int2> pack;   // (member, order) for the synthesis B packing, most degrees first
  {
    std::vector<int4> tmp;
    std::vector<int> cost;
    for (int t = 0; t < n; ++t)
      for (int im = 0; !g->simt[t] && im <= std::min(plans[t]->mmax, plans[t]->lmax); ++im) {
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
  g->n_ssyn = (int)ssyn.size();
  g->ssyn_ctas = std::max(1, std::min(8 * g->nsm, g->n_ssyn));   // 128-thread CTAs, several per SM
  g->sargsz = simt_args_bytes();
  // one device allocation
  g->argsz = mixed_args_bytes();
  g->jobsz = fft_job_bytes_f32();
  g->job2sz = fft2_job_bytes();
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = align256(o + b); return r; };
  const size_t o_as = take(n * g->argsz), o_aa = take(n * g->argsz), o_js = take(n * g->jobsz), o_ja = take(n * g->jobsz);
  const size_t o_j2s = take(n * g->job2sz), o_j2a = take(n * g->job2sz),
               o_i2 = take(std::max<size_t>(1, f2items.size()) * sizeof(int4));
  const size_t o_done = take(n * 8), o_t0 = take(8), o_q = take(kGroupQueues * sizeof(int)),
               o_is = take(syn.size() * sizeof(int4)),
               o_ia = take(ana.size() * sizeof(int4)), o_ip = take(pack.size() * sizeof(int2)),
               o_ms = take(msyn.size() * 8), o_ma = take(mana.size() * 8);
  const size_t o_sas = take(n * g->sargsz), o_iss = take(ssyn.size() * sizeof(int4));
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
  g->d_jobs2_syn = g->dmem + o_j2s;
  g->d_jobs2_ana = g->dmem + o_j2a;
  g->d_items_fft2 = (int4*)(g->dmem + o_i2);
  g->d_done = (unsigned long long*)(g->dmem + o_done);
  g->d_t0 = (unsigned long long*)(g->dmem + o_t0);
  g->d_queue = (int*)(g->dmem + o_q);
  g->d_items_syn = (int4*)(g->dmem + o_is);
  g->d_items_ana = (int4*)(g->dmem + o_ia);
  g->d_masks_syn = (unsigned long long*)(g->dmem + o_ms);
  g->d_masks_ana = (unsigned long long*)(g->dmem + o_ma);
  g->d_items_pack = (int2*)(g->dmem + o_ip);
  g->d_sargs = g->dmem + o_sas;
  g->d_items_ssyn = (int4*)(g->dmem + o_iss);
  g->d_w = g->dmem + o_w;
  e = cudaMemcpy(g->d_items_syn, syn.data(), syn.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_items_ana, ana.data(), ana.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !msyn.empty()) e = cudaMemcpy(g->d_masks_syn, msyn.data(), msyn.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !mana.empty()) e = cudaMemcpy(g->d_masks_ana, mana.data(), mana.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_items_pack, pack.data(), pack.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_items_ssyn, ssyn.data(), ssyn.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !f2items.empty())
    e = cudaMemcpy(g->d_items_fft2, f2items.data(), f2items.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(g->d_done, 0, n * 8);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->priv, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->aux, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming);
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
  std::vector<unsigned char> as(g->n * g->argsz), aa(g->n * g->argsz), js(g->n * g->jobsz), ja(g->n * g->jobsz),
      j2s(g->n * g->job2sz), j2a(g->n * g->job2sz), sas(g->n * g->sargsz);
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
    if (g->f2[t]) {
      fft2_fill_job(p, 1, W, grid[t], g->nf[t], j2s.data() + t * g->job2sz);
      fft2_fill_job(p, 0, W, grid[t], g->nf[t], j2a.data() + t * g->job2sz);
    }
    if (g->simt[t]) simt_fill_args(p, alm_in[t], W, g->nf[t], sas.data() + t * g->sargsz);
  }
  SHTB_TRY_CUDA(cudaMemcpy(g->d_args_syn, as.data(), as.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_args_ana, aa.data(), aa.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs_syn, js.data(), js.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs_ana, ja.data(), ja.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs2_syn, j2s.data(), j2s.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_jobs2_ana, j2a.data(), j2a.size(), cudaMemcpyHostToDevice), "group bind");
  SHTB_TRY_CUDA(cudaMemcpy(g->d_sargs, sas.data(), sas.size(), cudaMemcpyHostToDevice), "group bind");
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
    g->graph_kernels = (int)(shtb_launch_count(0) - before);
    count_launch(-g->graph_kernels);   // capturing runs no kernel
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
  count_launch(g->graph_kernels);   // start marker, B packing, GEMMs and the FFT kernels
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
  // best of three roundtrips with the current shape
  auto time_shape = [&](float& ms_min) {
    ms_min = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, g->priv);
      const int r = group_launch_stages(g, -1, g->priv);
      cudaEventRecord(e1, g->priv);
      if (r) return r;
      if (cudaEventSynchronize(e1) == cudaSuccess) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms_min = std::min(ms_min, ms);
      }
    }
    return SHTB_OK;
  };
  float best = 1e30f;
  int bh = g->fft_h, bc = g->fft_ctas;
  for (int h : {16, 8, 4}) {
    if (g->n_fft == 0) {   // only packed-pair FFTs: their shape is fixed
      if ((rc = time_shape(best))) break;
      break;
    }
    if (group_fft_smem(g, h) > 200 * 1024) continue;
    for (int mult : {1, 2, 4}) {
      float ms;
      if ((rc = set_fft_shape(g, h, g->nsm * mult)) || (rc = time_shape(ms))) break;
      if (ms < best) {
        best = ms;
        bh = h;
        bc = g->fft_ctas;
      }
    }
    if (rc) break;
  }
  if (!rc && g->n_fft > 0) rc = set_fft_shape(g, bh, bc);
  // GEMM CTAs per SM (the kernel's resources allow two), synthesis then analysis
  for (int which = 0; which < 2 && !rc; ++which) {
    int& ctas = which == 0 ? g->gemm_ctas_syn : g->gemm_ctas_ana;
    const int nitems = which == 0 ? g->n_syn : g->n_ana;
    if (nitems == 0) continue;
    int keep = ctas;
    for (int mult : {1, 2}) {
      const int c = std::max(1, std::min(mult * g->nsm, nitems));
      if (c == keep) continue;
      const int prev = ctas;
      ctas = c;
      float ms;
      if ((rc = time_shape(ms))) break;
      if (ms < best) {
        best = ms;
        keep = c;
      } else {
        ctas = prev;
      }
    }
    ctas = keep;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  SHTB_TRY_CUDA(cudaStreamSynchronize(g->priv), "group autotune");
  drop_graph(g);
  return SHTB_OK;
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
