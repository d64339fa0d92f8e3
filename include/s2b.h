/*
 * s2b.h -- C ABI of the B200 spin spherical-harmonic / Wigner transform library.
 *
 * Plain pointers and sizes only. Every entry point returns an int status
 * (S2B_OK == 0) and never exits the process; s2b_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Device buffers are caller-owned. Inputs are never modified. The transform
 * calls (s2b_inverse, s2b_forward, s2b_wigner_*, s2b_precompute_*) are
 * stream-ordered on the given cudaStream_t (passed as void*) and perform no
 * device allocation and no host synchronisation, so they can be captured in a
 * CUDA graph once the plan exists. Several host threads may call one plan at
 * once, each with its own workspace and stream (spin plans with spin != 0 and
 * Wigner plans fork to streams the plan owns; the fork is made atomic per
 * plan). Plan creation allocates the plan's tables;
 * s2b_kernel_build with S2B_BF16X3 allocates and frees a temporary table.
 *
 * Array layouts (row-major, innermost last), for B = desc.batch maps:
 *   flm   [B][L][2L-1]           complex, index [l][L-1+m]
 *   f     [B][ntheta][nphi]      equiangular (mw, mwss, dh, gl)
 *         [B][12*nside^2]        healpix, ring-ordered
 *   f is complex, or real when desc.reality != 0.
 *   complex = interleaved (re, im); double for S2B_F64, float for S2B_F32.
 *   flmn  [B][2N-1][L][2L-1]     Wigner coefficients, index [N-1+n][l][L-1+m]
 *   f_so3 [B][2N-1][ntheta][nphi] (or [B][2N-1][12 nside^2])
 *
 * Reference interfaces these replace (upstream astro-informatics/s2fft):
 *   s2b_inverse  <- s2fft/transforms/spherical.py:21-109 (inverse, method dispatch)
 *                   + transforms/otf_recursions.py:15-171 (inverse_latitudinal_step)
 *   s2b_forward  <- s2fft/transforms/spherical.py:352-464 (forward, incl. iter refinement)
 *                   + transforms/otf_recursions.py:432-588 (forward_latitudinal_step)
 *   s2b_plan_create <- lib/src/extensions.cc:115-149 (build_healpix_fft_descriptor,
 *                   plan cache init) and recursions/price_mcewen.py:118-255
 *                   (generate_precomputes_jax: per-plan recursion tables)
 *   s2b_wigner_inverse / s2b_wigner_forward
 *                <- s2fft/transforms/wigner.py:13-107, 346-439
 *   s2b_kernel_build <- s2fft/precompute_transforms/construct.py:16-161
 *                   (spin_spherical_kernel)
 *   s2b_precompute_inverse / s2b_precompute_forward
 *                <- s2fft/precompute_transforms/spherical.py:87-149, 314-380
 */
#ifndef S2B_H
#define S2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum s2b_status {
  S2B_OK = 0,
  S2B_ERR_INVALID = 1,   /* bad descriptor or argument                   */
  S2B_ERR_CUDA = 2,      /* a CUDA runtime call failed                    */
  S2B_ERR_WORKSPACE = 3, /* workspace missing or too small                */
  S2B_ERR_ALIGN = 4,     /* a pointer is NULL or not 16-byte aligned      */
  S2B_ERR_TIMEOUT = 5,   /* a bounded device wait gave up (status word)   */
  S2B_ERR_INTERNAL = 6
};

enum s2b_sampling { S2B_MW = 0, S2B_MWSS = 1, S2B_DH = 2, S2B_GL = 3, S2B_HEALPIX = 4 };

/* S2B_F64: everything in double.
 * S2B_F32: recursion and projection in float; recursion seeds, exponent
 *          bookkeeping, lambda(theta, m) and quadrature weights in double. */
/* S2B_BF16X3: as S2B_F32, except that the precompute contractions (forward and
 *          inverse) run on the tcgen05 tensor cores with 3-term bf16 split operands
 *          (hi*hi + hi*lo + lo*hi) and FP32 accumulation; their kernel tables are the
 *          packed bf16 layouts produced by s2b_kernel_build (spin plans, every sampling). */
enum s2b_precision { S2B_F64 = 0, S2B_F32 = 1, S2B_BF16X3 = 2 };

typedef struct s2b_desc {
  int L;          /* harmonic band-limit                                  */
  int spin;       /* spin s (Wigner: ignored, set by N)                   */
  int nside;      /* HEALPix resolution (healpix only)                    */
  int sampling;   /* enum s2b_sampling                                    */
  int reality;    /* signal is real (spin 0 only)                         */
  int L_lower;    /* harmonic lower bound                                 */
  int precision;  /* enum s2b_precision                                   */
  int batch;      /* maps per execute call                                */
  int iter;       /* forward: Jacobi refinement iterations                */
  int N;          /* Wigner directional band-limit (0 = spin transform)   */
} s2b_desc;

typedef struct s2b_plan s2b_plan;

/* Library version, e.g. 100 for 0.1.0. */
int s2b_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* s2b_last_error(void);

/* Build a plan (host + device tables) on the current device. Synchronous. */
int s2b_plan_create(const s2b_desc* desc, s2b_plan** plan);
int s2b_plan_destroy(s2b_plan* plan);

/* Bytes of device workspace an execute call needs (0 allowed); forward selects the
 * call: 0 s2b_inverse, 1 s2b_forward, 2 s2b_inverse_adjoint, 3 s2b_forward_adjoint. */
int s2b_workspace_size(const s2b_plan* plan, int forward, size_t* bytes);

/* Spin spherical-harmonic transforms. */
int s2b_inverse(s2b_plan* plan, const void* flm, void* f, void* workspace,
                size_t workspace_bytes, void* stream);
int s2b_forward(s2b_plan* plan, const void* f, void* flm, void* workspace,
                size_t workspace_bytes, void* stream);

/* Adjoints (conjugate transposes) of the spin transforms, for reverse-mode
 * differentiation: for a complex-linear map y = A x the gradient of a real
 * loss is A^H applied to the gradient of y. Layouts as s2b_inverse /
 * s2b_forward (g_f has the shape of f, g_flm of flm); complex plans only
 * (reality = 0); s2b_forward_adjoint is the adjoint of the single-pass forward
 * (desc.iter is ignored). Workspace: s2b_workspace_size(plan, 2 | 3, ...).
 * Replace the custom VJP rules of s2fft/transforms/spherical.py:306-324 and
 * 711-729 (latitudinal steps) together with JAX's autodiff of the ring FFTs and
 * the MW/MWSS resampling (s2fft/utils/resampling.py). */
int s2b_inverse_adjoint(s2b_plan* plan, const void* g_f, void* g_flm, void* workspace,
                        size_t workspace_bytes, void* stream);
int s2b_forward_adjoint(s2b_plan* plan, const void* g_flm, void* g_f, void* workspace,
                        size_t workspace_bytes, void* stream);

/* HEALPix ring FFTs alone (plan with sampling S2B_HEALPIX; spin is ignored):
 *   f [B][12 nside^2] (complex, or real when desc.reality) <-> ftm [B][4 nside - 1][2L]
 * complex, column c holding m = c - L: per ring FFT (no normalisation), fftshift and
 * periodic extension to 2L columns; the inverse folds each row onto its ring length and
 * inverse-FFTs without normalisation. No ring phase shifts. For real maps the rings of 2L
 * pixels keep m >= 0 only, and the inverse returns real maps (Hermitian spectra).
 * Replace s2fft/utils/healpix_ffts.py:187-423 (healpix_fft / healpix_ifft) and the XLA
 * custom call lib/src/extensions.cc:26-100 (healpix_fft_cuda: healpix_forward /
 * healpix_backward), which leaves reality aside. No workspace. */
int s2b_healpix_fft(s2b_plan* plan, const void* f, void* ftm, void* stream);
int s2b_healpix_ifft(s2b_plan* plan, const void* ftm, void* f, void* stream);

/* Wigner transforms on SO(3) (plan with desc.N > 0; desc.spin is ignored):
 *   flmn [B][2N-1][L][2L-1] <-> f [B][2N-1][ntheta][nphi] (or [B][2N-1][12 nside^2]);
 *   f real when desc.reality (then flmn obeys the SO(3) conjugate symmetry).
 * Replace s2fft/transforms/wigner.py:13-107 (inverse) and 346-439 (forward). */
int s2b_wigner_inverse(s2b_plan* plan, const void* flmn, void* f, void* workspace,
                       size_t workspace_bytes, void* stream);
int s2b_wigner_forward(s2b_plan* plan, const void* f, void* flmn, void* workspace,
                       size_t workspace_bytes, void* stream);

/* Precompute-kernel path (spin plans only). The kernel table has the upstream
 * layout K [ntheta_k][L][M] with M = 2L-1 (or L when reality), real in the
 * plan precision (complex for HEALPix, phases folded in); forward tables carry
 * the quadrature weights and, for mw/mwss, the 2L+1 rings of the MWSS grid at 2L.
 * s2b_kernel_size     <- s2fft/precompute_transforms/construct.py:16-161 (table size)
 * s2b_kernel_build    <- construct.py:16-161 (spin_spherical_kernel), built on the device
 * s2b_precompute_inverse <- s2fft/precompute_transforms/spherical.py:87-149
 * s2b_precompute_forward <- s2fft/precompute_transforms/spherical.py:314-380
 * Workspace: s2b_workspace_size(plan, forward, ...). */
int s2b_kernel_size(const s2b_plan* plan, int forward, size_t* bytes);
int s2b_kernel_build(s2b_plan* plan, int forward, void* kernel, void* stream);
int s2b_precompute_inverse(s2b_plan* plan, const void* kernel, const void* flm, void* f,
                           void* workspace, size_t workspace_bytes, void* stream);
int s2b_precompute_forward(s2b_plan* plan, const void* kernel, const void* f, void* flm,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Adjoints (conjugate transposes) of the precompute transforms for reverse-mode
 * differentiation, with the same kernel table and workspace as the call they invert the
 * direction of: g_flm = A^H g_f for A = s2b_precompute_inverse, g_f = A^H g_flm for
 * A = s2b_precompute_forward. Complex plans (reality = 0) with float or double tables
 * (not S2B_BF16X3). Replace JAX's autodiff of upstream's precompute einsums and FFTs
 * (s2fft/precompute_transforms/spherical.py:87-149, 314-380). */
int s2b_precompute_inverse_adjoint(s2b_plan* plan, const void* kernel, const void* g_f,
                                   void* g_flm, void* workspace, size_t workspace_bytes,
                                   void* stream);
int s2b_precompute_forward_adjoint(s2b_plan* plan, const void* kernel, const void* g_flm,
                                   void* g_f, void* workspace, size_t workspace_bytes,
                                   void* stream);

/* Device status of the plan (synchronous): *status != 0 after a bounded
 * wait inside a kernel ran out (the kernel then skipped its work); returns
 * S2B_ERR_TIMEOUT in that case. No upstream counterpart (upstream exits the
 * process on CUDA errors, lib/include/hresult.h:26-33). */
int s2b_plan_status(s2b_plan* plan, int* status);

/* Launch shape of the latitudinal kernels for later calls on this plan (and its
 * sub-plans): key 0 = forward tile (value 0: 16 rings per warp in float / 8 in double;
 * 1: half of that, twice the CTAs), key 1 = inverse tile (value bit 0: one ring per
 * lane instead of two in float; bit 1: start values read from global memory instead of
 * staged in shared memory), key 2 = inverse segments along m (value 1, 2, 4 or 8: each
 * CTA's m-range split into that many independently restarted parts; default 8), key 3 =
 * forward segments along m (same values; used by the equator-symmetric spin-0 forward).
 * Results agree to rounding; only the speed differs, which
 * depends on band-limit, batch and sampling. Used by the autotuner of the batched
 * front-end. No upstream counterpart. */
int s2b_plan_set_tuning(s2b_plan* plan, int key, int value);

/* The CUDA device ordinal a plan was created on (the device current at
 * s2b_plan_create). Every execute call on a spin or Wigner plan returns
 * S2B_ERR_INVALID, before launching anything, when the current device differs.
 * No upstream counterpart (upstream's plan cache is per process,
 * lib/include/plan_cache.h:15-44). */
int s2b_plan_device(const s2b_plan* plan, int* device);

/* Testing hook: overwrite the device ordinal recorded in the plan (and its
 * Wigner sub-plans), so that the device check above can be exercised on a
 * machine with one GPU. Never needed in normal use. No upstream counterpart. */
int s2b_debug_set_plan_device(s2b_plan* plan, int device);

/* Instrumentation: number of device allocations (cudaMalloc) the library has
 * made since it was loaded: plan tables, and the temporary table of
 * s2b_kernel_build with S2B_BF16X3. Execute calls add nothing to it. No
 * upstream counterpart. */
long long s2b_device_alloc_count(void);

/* Instrumentation: record the caller's cudaEvent_t objects (passed as void*)
 * immediately before and after the latitudinal (recursion + projection) kernel
 * of every later inverse (forward = 0) or forward (forward = 1) call on this
 * plan. NULL events switch recording off. No upstream counterpart; used by the
 * benchmark to time the dominant kernel on the launching stream. */
int s2b_plan_set_events(s2b_plan* plan, int forward, void* ev_begin, void* ev_end);

/* Spin inverse transform for callers that may not allocate device memory:
 * code running inside a host application or framework that owns every device
 * allocation (a plugin handed only its input and output buffers, a custom
 * call whose memory budget was fixed ahead of time), or code on a path where
 * an allocation would synchronise the device. Same plan, layouts, result and
 * errors as s2b_inverse, but instead of a caller-provided workspace it uses a
 * fixed scratch array of S2B_NOALLOC_SCRATCH_BYTES that the library holds on
 * every GPU it is loaded on, until the process exits. It calls no
 * cudaMalloc/cudaFree or other allocating routine.
 *   - Plans whose inverse workspace (s2b_workspace_size(plan, 0, ...)) exceeds
 *     S2B_NOALLOC_SCRATCH_BYTES are rejected with S2B_ERR_WORKSPACE. 32 MiB
 *     covers one mw-sampled map up to L ~ 1000 in float32 and L ~ 700 in
 *     float64; dh, with twice the rings, reaches about 5/6 of that.
 *   - The current device must be the plan's (else S2B_ERR_INVALID). The
 *     first call on a device looks up the array's device address with
 *     cudaGetSymbolAddress and keeps it; make that first call before any
 *     stream capture on that device. The kept address is not valid after a
 *     cudaDeviceReset of that device: do not call this entry point on a
 *     device after resetting it.
 *   - Every call on a device shares the one array: calls that can overlap on
 *     the GPU (different streams, threads or plans without ordering between
 *     them) race and corrupt each other's results. Order them on one stream.
 *   - Leftover contents from earlier calls are harmless: each call zeroes
 *     the accumulation rows it sums into and overwrites the rest before use.
 * No counterpart in the reference: upstream transforms always receive their
 * temporaries from the JAX/XLA allocator. */
#define S2B_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int s2b_inverse_noalloc(s2b_plan* plan, const void* flm, void* f, void* stream);

/* Uneven batches: the spin transforms of several plans (different L, spin,
 * sampling, nside, batch; one device and one precision) in one call. Entry k
 * transforms with plans[k] exactly as s2b_inverse / s2b_forward would (same
 * layouts, results and refinement iterations), from in[k] to out[k] with the
 * workspace ws[k] of ws_bytes[k] >= s2b_workspace_size(plans[k], 0 or 1)
 * bytes. The stages around the latitudinal kernels run per plan on a few
 * streams the batch owns (forked from and joined back to `stream`); the
 * latitudinal kernels of all entries run as persistent launches, one per
 * kernel variant (spin 0 or not, tile shape), whose CTAs pull (plan, tile)
 * items from a device counter. Stream-ordered and capturable in a CUDA graph
 * like the single-plan calls; the batch object may not be used by two calls
 * at once. The plans must outlive the batch. s2b_batch_create allocates the
 * counters and creates the streams and events.
 * No upstream counterpart: upstream transforms one (L, spin, sampling) per
 * call (s2fft/transforms/spherical.py:21-109, 352-464); these are those calls,
 * fused across entries. */
typedef struct s2b_batch s2b_batch;
int s2b_batch_create(s2b_plan* const* plans, int nplans, s2b_batch** batch);
int s2b_batch_destroy(s2b_batch* batch);
int s2b_batch_inverse(s2b_batch* batch, const void* const* flm, void* const* f,
                      void* const* workspace, const size_t* ws_bytes, void* stream);
int s2b_batch_forward(s2b_batch* batch, const void* const* f, void* const* flm,
                      void* const* workspace, const size_t* ws_bytes, void* stream);
/* Schedule of a batch's calls. key 0: waves (1 to 4; default 1). The entries are
 * dealt round-robin into waves; the per-plan stages of one wave (ring FFTs, which
 * are memory-bound) run on the batch's streams while the persistent latitudinal
 * launches of the next wave run on `stream`. key 1: CTAs per SM of the persistent
 * launches (0, the default: as many as fit), which leaves room on each SM for the
 * overlapping stages. Results do not depend on either. */
int s2b_batch_set_option(s2b_batch* batch, int key, int value);

/* Rotation of spherical-harmonic coefficients by the Euler angles (alpha, beta, gamma):
 *   flm'[l, m] = exp(-i m alpha) sum_n d^l_{m,n}(beta) exp(-i n gamma) flm[l, n],
 * replaces s2fft.utils.rotation.rotate_flms (s2fft/utils/rotation.py:9-64). flm and out
 * are [batch][L][2L-1] complex (double for precision S2B_F64, float for S2B_F32); the
 * arithmetic is double in both. dl == NULL: the Wigner-d values at beta are generated
 * on the device by the three-term recurrence in the degree of every (m, n) (upstream
 * builds the planes with Risbo's recursion, s2fft/recursions/risbo.py:4-120; the two
 * agree to rounding), L <= 8192; otherwise dl holds them in the layout of upstream's
 * generate_rotate_dls, [L][2L-1][2L-1] float64 with d^l_{m,n} at [l][L-1+m][L-1+n].
 * The workspace (s2b_rotate_workspace_size(L) bytes, caller-owned) holds the
 * recurrence coefficients, the start values and the phase tables. Results do not
 * depend on the launch order (fixed-order sums). Stream-ordered; no allocation. */
size_t s2b_rotate_workspace_size(int L);
int s2b_rotate_flms(int L, int batch, int precision, double alpha, double beta, double gamma,
                    const void* flm, void* out, const double* dl, void* ws, size_t ws_bytes,
                    void* stream);

/* The planes d^l_{m,n}(beta), 0 <= l < L, in the layout of upstream's
 * generate_rotate_dls (s2fft/utils/rotation.py:75-96): dl[l][L-1+m][L-1+n] float64,
 * zero where |m| > l or |n| > l; every entry is written. L <= 8192. */
int s2b_rotate_dls(int L, double beta, double* dl, void* ws, size_t ws_bytes, void* stream);

/* Fourier-Wigner transforms on SO(3) and the spin-subset lifting ops (mw / mwss only).
 * A plan holds the FFT tables of one (L, N, sampling, precision), N the azimuthal
 * band-limit of the full transforms (1 <= N <= L; the subset ops take any plan of the L,
 * sampling and precision); it is independent of the batch and of the spin subset. Layouts (complex interleaved, double for S2B_F64,
 * float for S2B_F32):
 *   flmn  [batch][2N-1][L][2L-1]            f [batch][2N-1][ntheta][nphi] (real if reality)
 *   spin-subset coefficients [batch][nspins][L][2L-1], maps [batch][nspins][ntheta][nphi],
 *   SO(3) signals for s2b_fw_so3_to_subset [batch][ngamma][ntheta][nphi].
 * delta = [L][2L-1][2L-1] float64 planes Delta^l_{a,b} = d^l_{a,b}(pi/2) (upstream layout,
 * e.g. from s2b_rotate_dls(L, pi/2, ...)); quads = [4L-3] complex128 upsampled quadrature
 * weights (s2b_fw_quads). Spins satisfy |spin| <= L-1 (slice n = -spin; a slice with |n|
 * > L-1 comes out zero). Pointers 16-byte aligned, workspace 256-byte aligned, of
 * s2b_fw_workspace_size bytes for the operation (enum s2b_fw_op). Stream-ordered; no
 * allocation or synchronisation outside plan creation.
 * Replace upstream:
 *   s2b_fw_plan_create / s2b_fw_quads
 *            <- s2fft/precompute_transforms/construct.py:614-639 (fourier_wigner_kernel)
 *   s2b_fw_inverse  <- s2fft/precompute_transforms/fourier_wigner.py:13-88
 *   s2b_fw_forward  <- s2fft/precompute_transforms/fourier_wigner.py:177-333
 *   s2b_fw_subset_to_s2  <- s2fft/precompute_transforms/custom_ops.py:5-83
 *   s2b_fw_s2_to_subset  <- s2fft/precompute_transforms/custom_ops.py:251-333
 *   s2b_fw_so3_to_subset <- s2fft/precompute_transforms/custom_ops.py:168-205 */
typedef struct s2b_fw_plan s2b_fw_plan;
enum s2b_fw_op {
  S2B_FW_INVERSE = 0,
  S2B_FW_FORWARD = 1,
  S2B_FW_SUBSET_TO_S2 = 2,
  S2B_FW_S2_TO_SUBSET = 3,
  S2B_FW_SO3_TO_SUBSET = 4
};
int s2b_fw_plan_create(int L, int N, int sampling, int precision, s2b_fw_plan** plan);
int s2b_fw_plan_destroy(s2b_fw_plan* plan);
int s2b_fw_quads(s2b_fw_plan* plan, void* quads, void* stream);
/* reality is used by the full transforms, nspins by the subset ops. */
size_t s2b_fw_workspace_size(const s2b_fw_plan* plan, int op, int batch, int reality,
                             int nspins);
/* Full transforms with the plan's N. */
int s2b_fw_inverse(s2b_fw_plan* plan, int batch, int reality, const double* delta,
                   const void* flmn, void* f, void* workspace, size_t workspace_bytes,
                   void* stream);
int s2b_fw_forward(s2b_fw_plan* plan, int batch, int reality, const double* delta,
                   const void* quads, const void* f, void* flmn, void* workspace,
                   size_t workspace_bytes, void* stream);
/* Adjoints (conjugate transposes) of s2b_fw_inverse / s2b_fw_forward for reverse-mode
 * differentiation (complex signals): g_flmn = A^H g_f, g_f = A^H g_flmn, with the plan's N,
 * the same delta / quads and the workspace of the transform they adjoin (reality = 0).
 * Replace JAX's autodiff of upstream's fourier_wigner.py:13-333. */
int s2b_fw_inverse_adjoint(s2b_fw_plan* plan, int batch, const double* delta, const void* g_f,
                           void* g_flmn, void* workspace, size_t workspace_bytes, void* stream);
int s2b_fw_forward_adjoint(s2b_fw_plan* plan, int batch, const double* delta, const void* quads,
                           const void* g_flmn, void* g_f, void* workspace,
                           size_t workspace_bytes, void* stream);
/* spins: device int32 [nspins]. */
int s2b_fw_subset_to_s2(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                        const double* delta, const void* flmn, void* f, void* workspace,
                        size_t workspace_bytes, void* stream);
int s2b_fw_s2_to_subset(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                        const double* delta, const void* quads, const void* f, void* flmn,
                        void* workspace, size_t workspace_bytes, void* stream);
int s2b_fw_so3_to_subset(s2b_fw_plan* plan, int batch, int ngamma, int nspins,
                         const int* spins, const double* delta, const void* quads,
                         const void* f, void* flmn, void* workspace, size_t workspace_bytes,
                         void* stream);

/* Adjoints of the three spin-subset ops (complex): same plan, spins, delta / quads and
 * workspace as the op, input and output exchanged (g_flmn = A^H g_f for subset_to_s2,
 * g_f = A^H g_flmn for s2_to_subset and so3_to_subset). Replace JAX's autodiff of
 * upstream's custom_ops.py:5-333. */
int s2b_fw_subset_to_s2_adjoint(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                                const double* delta, const void* g_f, void* g_flmn,
                                void* workspace, size_t workspace_bytes, void* stream);
int s2b_fw_s2_to_subset_adjoint(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                                const double* delta, const void* quads, const void* g_flmn,
                                void* g_f, void* workspace, size_t workspace_bytes,
                                void* stream);
int s2b_fw_so3_to_subset_adjoint(s2b_fw_plan* plan, int batch, int ngamma, int nspins,
                                 const int* spins, const double* delta, const void* quads,
                                 const void* g_flmn, void* g_f, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* Peak-rate probe: a fused multiply-add chain kernel (float when fp64 == 0,
 * double otherwise) over `blocks` CTAs of 256 threads, `iters` iterations of 8
 * independent FMA chains per thread, writing one value per thread to `out`
 * (blocks*256 elements). No upstream counterpart. */
int s2b_fma_probe(int fp64, int blocks, int iters, void* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* S2B_H */
