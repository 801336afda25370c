/*
 * shtb200.h — C ABI of the B200-native spherical harmonic transform library.
 *
 * Every entry point takes plain pointers, sizes and an opaque plan; no C++ or
 * torch types cross this boundary. Device pointers are CUDA device addresses
 * on the plan's device; the stream is a cudaStream_t passed as void* (NULL =
 * legacy default stream). Calls are asynchronous on that stream.
 *
 * Layouts are the reference's Julia column-major ones:
 *   grid         f[i, j, k]   at i + nlat*j + nlat*nlon*k   (latitude north->south fastest)
 *   coefficients a[l, m, k]   at l + (lmax+1)*m + (lmax+1)*(mmax+1)*k, complex = (re, im) pair
 * Entries with l < m are ignored on input and written as zero on output.
 *
 * Reference interfaces replaced (SHTnsKit.jl v3.0.0, paths within that project):
 *   shtb_plan_create        per-config device tables built by `_cuda_scalar_tables` /
 *                           `_cuda_vector_tables` (ext/SHTnsKitGPUExt.jl:495-557) from an
 *                           `SHTConfig` (src/config.jl:170-206, create_gauss_config :633-655)
 *   shtb_synthesis          `_gpu_adapter_synthesis(::CUDAAdapter, cfg, alm; real_output=true)`
 *                           (ext/SHTnsKitGPUExt.jl:788-836); CPU semantics src/core_transforms.jl:271-344
 *   shtb_analysis           `_gpu_adapter_analysis` (ext/SHTnsKitGPUExt.jl:750-786, :828-831);
 *                           CPU semantics src/core_transforms.jl:169-207
 *   shtb_synthesis_sphtor   `_gpu_adapter_synthesis_sphtor` (ext/SHTnsKitGPUExt.jl:927-992);
 *                           CPU semantics src/sphtor_transforms.jl:162-241
 *   shtb_analysis_sphtor    `_gpu_adapter_analysis_sphtor` (ext/SHTnsKitGPUExt.jl:859-910, :987-989);
 *                           CPU semantics src/sphtor_transforms.jl:252-289
 *   batched calls (nfields > 1) replace `analysis_batch(::GPU, ...)` / `synthesis_batch`
 *                           (ext/SHTnsKitGPUExt.jl:1845-1975; src/batch_transforms.jl:312-660)
 *   *_adjoint               the pullbacks of the ChainRules rrules
 *                           (ext/SHTnsKitAdvancedADExt.jl:55-91, :198-246) which call
 *                           `_adjoint_synthesis` (src/core_transforms.jl:477-519),
 *                           `_adjoint_analysis` (:611-652), `_adjoint_synthesis_sphtor` (:537-597),
 *                           `_adjoint_analysis_sphtor` (src/sphtor_transforms.jl:385-452)
 *   shtb_gauss_nodes        `gausslegendre` (src/legendre.jl:956-1003) with the north-first
 *                           reversal of create_gauss_config (src/config.jl:639)
 */
#ifndef SHTB200_H
#define SHTB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (every entry point returns one) ---- */
#define SHTB_OK               0
#define SHTB_ERR_BAD_ARG     -1   /* invalid scalar argument (maps to ArgumentError)        */
#define SHTB_ERR_BAD_SHAPE   -2   /* size/layout mismatch (maps to DimensionMismatch)        */
#define SHTB_ERR_ALIGN       -3   /* pointer not 16-byte aligned                             */
#define SHTB_ERR_OOM         -4   /* device allocation for plan tables failed                */
#define SHTB_ERR_CUDA        -5   /* CUDA runtime error (maps to BackendUnavailableError)    */
#define SHTB_ERR_TIMEOUT     -6   /* a bounded device wait gave up                           */
#define SHTB_ERR_UNSUPPORTED -7   /* valid request this build does not implement             */
#define SHTB_ERR_WORKSPACE   -8   /* workspace pointer NULL or smaller than required         */

/* ---- element types of the caller's buffers ---- */
#define SHTB_F64 0   /* grids double, coefficients complex double */
#define SHTB_F32 1   /* grids float,  coefficients complex float  */

/* ---- arithmetic paths ---- */
#define SHTB_PREC_FP64  0   /* plain FP64 drop-in (relative L2 <= 1e-12 vs the FP64 CPU result) */
#define SHTB_PREC_MIXED 1   /* FP32 buffers; Legendre contraction on tensor cores as fp16x3
                               products (f16 hi/lo splits of power-of-two-scaled operands,
                               hi*hi + hi*lo + lo*hi) with FP32 accumulation; nodes, weights,
                               seeds and recurrence in FP64 (relative L2 <= 1e-6 vs FP64)    */

/* ---- operation ids for shtb_workspace_bytes ---- */
#define SHTB_OP_SYNTHESIS        0
#define SHTB_OP_ANALYSIS         1
#define SHTB_OP_SYNTHESIS_SPHTOR 2
#define SHTB_OP_ANALYSIS_SPHTOR  3

typedef struct shtb_plan shtb_plan;

/* Library version (major*10000 + minor*100 + patch). */
int shtb_version(void);

/* Message of the last failing call on this host thread ("" if none). */
const char* shtb_last_error(void);

/* Gauss-Legendre nodes x (descending, north pole first) and weights w, n > 0. Host memory. */
int shtb_gauss_nodes(int n, double* x, double* w);

/*
 * Build a plan on the current CUDA device.
 *   x, w          host arrays of nlat Gauss nodes/weights, north pole first
 *   coeff_scale   host (lmax+1)*(mmax+1) column-major array s[l,m] with
 *                 a_canonical = s * a_configured (src/normalization.jl:142-147), or NULL
 *                 for the canonical orthonormal + Condon-Shortley convention
 *   phi_inv_scale       synthesis bin scale (nlon under phi_scale=:dft, src/SHTnsKit.jl:141-159)
 *   analysis_phi_scale  analysis factor (2*pi/nlon under :dft, src/SHTnsKit.jl:177)
 *   robert_form   nonzero: vector fields carry the sin(theta) factor
 * Validation mirrors `_validate_spectral_layout` (src/config.jl:465-481).
 */
int shtb_plan_create(shtb_plan** plan, int lmax, int mmax, int mres, int nlat, int nlon,
                     const double* x, const double* w, const double* coeff_scale,
                     double phi_inv_scale, double analysis_phi_scale, int robert_form);
int shtb_plan_destroy(shtb_plan* plan);

/* Device bytes held by the plan's tables. */
size_t shtb_plan_table_bytes(const shtb_plan* plan);

/*
 * Synchronizes the device; returns SHTB_ERR_TIMEOUT if a kernel of this plan gave
 * up a bounded device wait since the last call (and clears the condition), else SHTB_OK.
 */
int shtb_plan_status(const shtb_plan* plan);

/*
 * Test hook for failure detection (no counterpart in the reference). For this plan's
 * mixed-precision (SHTB_PREC_MIXED) calls: wait_ns replaces the 2 s limit of the tensor-core
 * kernels' bounded device waits (0 restores it), and skip_chunk >= 0 makes the loader of the
 * first CTA leave that chunk's copies unissued, so the wait for it runs out. The kernel then
 * drains its own copies and MMAs in flight, frees its tensor memory and returns;
 * shtb_plan_status reports SHTB_ERR_TIMEOUT and the plan stays usable. skip_chunk < 0 turns
 * the skip off.
 */
int shtb_plan_debug_waits(shtb_plan* plan, uint64_t wait_ns, int skip_chunk);

/* Workspace bytes a call needs for nfields fields (caller allocates, >= 256-byte aligned). */
size_t shtb_workspace_bytes(const shtb_plan* plan, int op, int nfields, int dtype, int precision);

/*
 * Scalar synthesis, real output: f = Re(ifft(Hermitian-filled bins)) for nfields fields.
 * ltr truncates degrees (ltr < 0 means lmax).
 */
int shtb_synthesis(const shtb_plan* plan, const void* alm, void* f, int nfields, int ltr,
                   int dtype, int precision, void* work, size_t work_bytes, void* stream);

/* Scalar analysis of real grids. */
int shtb_analysis(const shtb_plan* plan, const void* f, void* alm, int nfields, int ltr,
                  int dtype, int precision, void* work, size_t work_bytes, void* stream);

/*
 * Complex grids, FP64 (complex double grids f[i, j, k], coefficients as shtb_synthesis):
 *   shtb_synthesis_cplx  synthesis with real_output = false: f = ifft of the bins m >= 0
 *                        without the Hermitian fill (`synthesis(cfg, alm; real_output=false)`,
 *                        `synthesis_cplx`, src/core_transforms.jl:271-344; CUDA adapter
 *                        ext/SHTnsKitGPUExt.jl:788-826 with real_output=false)
 *   shtb_analysis_cplx   analysis of a complex-valued field from its bins m >= 0
 *                        (src/core_transforms.jl:169-207; ext/SHTnsKitGPUExt.jl:750-786 on a
 *                        complex CuArray)
 * Workspace: SHTB_OP_SYNTHESIS / SHTB_OP_ANALYSIS with SHTB_F64, SHTB_PREC_FP64.
 */
int shtb_synthesis_cplx(const shtb_plan* plan, const void* alm, void* f, int nfields, int ltr,
                        void* work, size_t work_bytes, void* stream);
int shtb_analysis_cplx(const shtb_plan* plan, const void* f, void* alm, int nfields, int ltr,
                       void* work, size_t work_bytes, void* stream);

/* Spheroidal/toroidal synthesis to (Vt, Vp), real output. */
int shtb_synthesis_sphtor(const shtb_plan* plan, const void* S, const void* T, void* Vt, void* Vp,
                          int nfields, int ltr, int dtype, int precision,
                          void* work, size_t work_bytes, void* stream);

/* Spheroidal/toroidal analysis of real (Vt, Vp). */
int shtb_analysis_sphtor(const shtb_plan* plan, const void* Vt, const void* Vp, void* S, void* T,
                         int nfields, int ltr, int dtype, int precision,
                         void* work, size_t work_bytes, void* stream);

/*
 * Scalar transforms on coefficients in the packed LM layout of SHTns: per field a vector of
 * nlm = sum over m = 0, mres, ..., mmax of (lmax - m + 1) complex values, order m's block
 * starting at LM_index(0, m) = (im (2 lmax + 2 - (im + 1) mres)) / 2 (src/layout.jl:88-162),
 * fields nlm apart. The gather/scatter is the transform's own coefficient addressing, not a
 * separate pass.
 *   shtb_synthesis_packed  synthesis_packed / synthesis_packed_l (src/transforms.jl:144-155,
 *                          :209-227); ltr < lmax ignores the packed coefficients above ltr
 *   shtb_analysis_packed   analysis_packed / analysis_packed_l (src/transforms.jl:125-136,
 *                          :183-203); coefficients above ltr come out zero
 * Arguments, workspace (SHTB_OP_SYNTHESIS / SHTB_OP_ANALYSIS), precisions and errors as
 * shtb_synthesis / shtb_analysis.
 */
int shtb_synthesis_packed(const shtb_plan* plan, const void* qlm, void* f, int nfields, int ltr,
                          int dtype, int precision, void* work, size_t work_bytes, void* stream);
int shtb_analysis_packed(const shtb_plan* plan, const void* f, void* qlm, int nfields, int ltr,
                         int dtype, int precision, void* work, size_t work_bytes, void* stream);

/*
 * Vector transforms with divergence/vorticity spectra on the spectral side, the diagonal
 * factor applied where the coefficients enter (synthesis) or leave (analysis) the Legendre
 * stage instead of in a separate pass:
 *   shtb_synthesis_divvort(div, vort) = synthesis_sphtor(spheroidal_from_divergence(div),
 *                                                        toroidal_from_vorticity(vort))
 *   shtb_analysis_divvort(Vt, Vp)     = (divergence_from_spheroidal(S), vorticity_from_toroidal(T))
 *                                       with (S, T) = analysis_sphtor(Vt, Vp)
 * (src/sphtor_transforms.jl:771-783, :817-831, :865-877, :911-925 composed with
 * :162-241 / :252-289). No single reference entry point; arguments, workspace
 * (SHTB_OP_SYNTHESIS_SPHTOR / SHTB_OP_ANALYSIS_SPHTOR) and errors as the sphtor calls. FP64.
 */
int shtb_synthesis_divvort(const shtb_plan* plan, const void* div, const void* vort, void* Vt, void* Vp,
                           int nfields, int ltr, int dtype, int precision,
                           void* work, size_t work_bytes, void* stream);
int shtb_analysis_divvort(const shtb_plan* plan, const void* Vt, const void* Vp, void* div, void* vort,
                          int nfields, int ltr, int dtype, int precision,
                          void* work, size_t work_bytes, void* stream);

/*
 * Diagonal spectral operators on dense (lmax+1, mmax+1) coefficients of nfields fields
 * (dtype SHTB_F64: complex double, SHTB_F32: complex float), no workspace:
 *   SHTB_SPEC_NEG_LL      out = -l(l+1) in: divergence_from_spheroidal!,
 *                         vorticity_from_toroidal! (src/sphtor_transforms.jl:771-783, :865-877),
 *                         laplacian_kernel! / gpu_apply_laplacian! (ext/GPUCommon.jl:1501-1512,
 *                         ext/SHTnsKitGPUExt.jl:2382-2389)
 *   SHTB_SPEC_INV_NEG_LL  out = -(in / (l(l+1))): spheroidal_from_divergence!,
 *                         toroidal_from_vorticity! (src/sphtor_transforms.jl:817-831, :911-925)
 * Entries with m % mres != 0 or l < max(1, m) are written as zero. out may be in itself;
 * otherwise the two must not overlap.
 */
#define SHTB_SPEC_NEG_LL     0
#define SHTB_SPEC_INV_NEG_LL 1
int shtb_spectral_op(const shtb_plan* plan, int op, const void* in, void* out, int nfields, int dtype,
                     void* stream);

/*
 * Adjoints (Zygote convention g = 2 dL/d(conj a)), FP64 only, real spatial cotangents.
 *   shtb_synthesis_adjoint:        ybar (grid)  -> abar (coefficients)
 *   shtb_analysis_adjoint:         abar         -> fbar (grid, real projection)
 *   shtb_synthesis_sphtor_adjoint: (Vtbar, Vpbar) -> (Sbar, Tbar)
 *   shtb_analysis_sphtor_adjoint:  (Sbar, Tbar)   -> (Vtbar, Vpbar) (real projection)
 * Workspace: same as the forward operation of the same shape.
 */
int shtb_synthesis_adjoint(const shtb_plan* plan, const void* ybar, void* abar, int nfields,
                           void* work, size_t work_bytes, void* stream);
int shtb_analysis_adjoint(const shtb_plan* plan, const void* abar, void* fbar, int nfields,
                          void* work, size_t work_bytes, void* stream);
int shtb_synthesis_sphtor_adjoint(const shtb_plan* plan, const void* Vtbar, const void* Vpbar,
                                  void* Sbar, void* Tbar, int nfields,
                                  void* work, size_t work_bytes, void* stream);
int shtb_analysis_sphtor_adjoint(const shtb_plan* plan, const void* Sbar, const void* Tbar,
                                 void* Vtbar, void* Vpbar, int nfields,
                                 void* work, size_t work_bytes, void* stream);

/*
 * Scalar FP64 synthesis that allocates no device memory and takes no workspace.
 * No counterpart in the reference: it exists for hosts that must not call cudaMalloc
 * between transforms (code running inside another runtime's memory pool, or long runs
 * where an allocation could synchronize the device or fail). Same inputs, outputs and
 * results as shtb_synthesis with dtype SHTB_F64 and precision SHTB_PREC_FP64.
 * Scratch: a 32 MiB array owned by the library on every GPU that loads it (until process
 * exit); calls needing more (nfields * (mmax/mres+1) * 2 * ceil(nlat/2) * 16 bytes) return
 * SHTB_ERR_WORKSPACE. shtb_plan_create looks up the array's device address on the plan's
 * device and keeps it in the plan; with CUDA's lazy module loading that lookup is when the
 * driver reserves the 32 MiB on that device, so the reservation (and an out-of-memory
 * failure of it, reported by this call as SHTB_ERR_CUDA) happens at plan creation, where
 * allocation is expected, never inside a transform. All calls share the array: calls that
 * overlap on the GPU (other streams or other host threads) race and must be serialized.
 */
int shtb_synthesis_noalloc(const shtb_plan* plan, const void* alm, void* f, int nfields, int ltr,
                           void* stream);

/*
 * Uneven batches: n independent mixed-precision (FP32 buffers, fp16x3 tensor-core
 * Legendre stage) scalar transforms, each with its own plan (its own lmax, Gauss grid
 * and nlon) and 1..8 fields. No single counterpart in the reference, whose transforms
 * run one configuration per call (src/core_transforms.jl, src/batch_transforms.jl):
 * a group runs every member's tiles in one persistent launch per stage (B packing and
 * order-GEMM synthesis for members of three or more fields, the FP64-pipe synthesis for
 * one- or two-field members, FFT synthesis, FFT analysis, order-GEMM analysis), work items
 * sorted by cost and claimed by the CTAs (or warps) from a device work counter, the stage
 * launches captured once in a CUDA graph and replayed.
 * Members must use lcap = lmax and mres = 1. Buffers (device pointers, per member):
 * alm_in and alm_out are (lmax+1, mmax+1, nfields) complex FP32 (Julia column-major),
 * grid is (nlat, nlon, nfields) FP32. Results equal those of shtb_synthesis /
 * shtb_analysis with SHTB_PREC_MIXED on the same member, bit for bit.
 */
typedef struct shtb_group shtb_group;
int shtb_group_create(shtb_group** out, const shtb_plan* const* plans, int n, const int* nfields);
int shtb_group_destroy(shtb_group* group);
/* Bind per-member device buffers (arrays of n pointers); invalidates the captured graph. */
int shtb_group_bind(shtb_group* group, void* const* alm_in, void* const* grid, void* const* alm_out);
/* synthesis alm_in -> grid, then analysis grid -> alm_out, as one graph launch on stream. */
int shtb_group_roundtrip(shtb_group* group, void* stream);
/* The same stages launched directly (no graph); op = SHTB_OP_SYNTHESIS, SHTB_OP_ANALYSIS or -1 (both). */
int shtb_group_launch(shtb_group* group, int op, void* stream);
/* Time the candidate launch shapes on the bound buffers and keep the fastest (blocking):
 * FFT latitude pairs per CTA x FFT CTAs per SM, then GEMM CTAs per SM of each GEMM stage. */
int shtb_group_autotune(shtb_group* group, void* stream);
/* Launch shape in use: FFT latitude pairs per CTA, FFT CTAs, CTAs of the synthesis GEMM. */
int shtb_group_config(const shtb_group* group, int* fft_pairs, int* fft_ctas, int* gemm_ctas);
/* After the last roundtrip completed: per-member completion time in ns after its start (n values). */
int shtb_group_latency_ns(const shtb_group* group, uint64_t* ns);

/* Number of kernels the library launched on this host thread since the last reset. */
uint64_t shtb_launch_count(int reset);

/*
 * Per-kernel timing: while enabled, every launch on this host thread is bracketed
 * by CUDA events on its stream. shtb_profile_read synchronizes the recorded events
 * and returns the number of distinct kernel names (names: max*64 bytes).
 * Enabling clears earlier records.
 */
int shtb_profile_enable(int on);
int shtb_profile_read(int max, char* names, double* total_ms, int* count);

#ifdef __cplusplus
}
#endif
#endif /* SHTB200_H */
