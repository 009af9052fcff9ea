/*
 * surfacelets_b200 — C ABI of the B200 (sm_100a) surfacelet analyze/synthesize
 * library.
 *
 * This is the drop-in boundary for the device path of hakkelt/Surfacelets.jl.
 * Each entry point below replaces one method of the reference's
 * AbstractMultiscaleTransforms interface for `NSSurfacelet` and the decimated
 * `Surfacelet`; the citation in front of each declaration names the reference
 * method (file:line in the Surfacelets.jl tree) whose behaviour it takes over.
 *
 * Conventions
 *   - Every function returns an int status: SFL_OK (0) or a negative code.
 *     SFL_ERR_ARGUMENT maps to Julia's ArgumentError and SFL_ERR_DIMENSION to
 *     DimensionMismatch; sfl_last_error() holds the message (thread-local), in
 *     the reference's own wording.
 *   - Volumes are column-major (axis 1 fastest), real float32 or complex
 *     float32 with interleaved real/imaginary parts.  Complex data runs as two
 *     real channels through the same kernels, so the transform is exactly
 *     real-linear (bit for bit).
 *   - NSSurfacelet coefficients are one (n1, n2, n3, S) array: subband i
 *     (1-based, lowpass first) is the contiguous volume at element offset
 *     (i-1)*n1*n2*n3.  Surfacelet coefficients are one flat vector with each
 *     subband a contiguous column-major block at the offset sfl_subband_info
 *     reports (the reference's SubbandVector).
 *   - Data pointers passed to sfl_analyze & co. are device pointers; `stream`
 *     is a cudaStream_t (NULL = the legacy default stream).  Calls are
 *     asynchronous with respect to the host unless stated otherwise.
 *   - A plan owns its tables and scratch.  It is not reentrant: one call at a
 *     time per plan (the reference's workspaces have the same rule,
 *     src/transforms/ns_surfacelet.jl:51-53, src/transforms/surfacelet.jl:40-44).
 */
#ifndef SURFACELETS_B200_H
#define SURFACELETS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SFL_OK 0
#define SFL_DONE 1               /* a stream has no further subband */
#define SFL_ERR_ARGUMENT (-1)    /* ArgumentError */
#define SFL_ERR_DIMENSION (-2)   /* DimensionMismatch */
#define SFL_ERR_CUDA (-3)        /* a CUDA call failed */
#define SFL_ERR_ALLOC (-4)       /* device memory could not be allocated */
#define SFL_ERR_STATE (-5)       /* call out of order (streaming) */
#define SFL_ERR_UNSUPPORTED (-6) /* a size or option this library does not handle */
#define SFL_ERR_TIMEOUT (-7)     /* a bounded device wait of an earlier call on the plan ran out */

#define SFL_MAX_SCALES 16

#define SFL_REAL32 0
#define SFL_COMPLEX64 1

#define SFL_KIND_NS 0
#define SFL_KIND_DECIMATED 1
#define SFL_KIND_NDFB 2        /* standalone directional bank (make_ndfb / make_hourglass) */

/* NSSurfacelet(; scales, direction_levels, bernstein_order, halfband_order,
 *              transition, tight) — src/types/transforms.jl:86-113.
 * direction_levels[j] for j = 0 .. scales-1, coarsest scale first. */
typedef struct {
    int32_t scales;
    int32_t direction_levels[SFL_MAX_SCALES];
    int32_t bernstein_order;
    int32_t halfband_order;
    double transition;
    int32_t tight;
} sfl_ns_params;

/* make_ndfb(dims; levels, bernstein_order, halfband_order, tight, transition)
 * — src/directional/ndfb.jl:91-104; levels = 0 is make_hourglass
 * (src/directional/hourglass.jl:149-170).  3 * 2^levels full-size subbands,
 * index ((i-1) na + (p-1)) nb + q (src/directional/ndfb.jl:184-190). */
typedef struct {
    int32_t levels;
    int32_t bernstein_order;
    int32_t halfband_order;
    double transition;
    int32_t tight;
} sfl_ndfb_params;

/* Surfacelet(; scales, direction_levels, pyramid_ratio, checkerboard_order,
 *            diamond_length, kaiser_beta, diamond_power) —
 * src/types/transforms.jl:222-261.  levels[j][K][m] is the level matrix of
 * scale j (coarsest first): the number of checkerboard stages along axis m
 * inside hourglass K (diagonal ignored).  Integer levels convert with
 * sfl_surf_levels_from_int. */
typedef struct {
    int32_t scales;
    int32_t levels[SFL_MAX_SCALES][3][3];
    double pyramid_ratio;
    int32_t checkerboard_order;
    int32_t diamond_length;
    double kaiser_beta;
    int32_t diamond_power;
} sfl_surf_params;

typedef struct sfl_plan sfl_plan;

/* Message of the last failed call on this thread ("" when none). */
const char* sfl_last_error(void);

/* Library version string. */
const char* sfl_version(void);

/* ── Parameter and layout queries (host only, no device needed) ─────────── */

/* Constructor validation of NSSurfacelet: src/types/transforms.jl:93-104. */
int sfl_ns_check_params(const sfl_ns_params* p);

/* Size validation of make_workspace, including the empty-scale refusal:
 * src/transforms/ns_surfacelet.jl:98-115. */
int sfl_ns_check_size(const sfl_ns_params* p, const int32_t dims[3]);

/* nsubbands(t, dims): src/transforms/ns_surfacelet.jl:527. */
int sfl_ns_nsubbands(const sfl_ns_params* p, int32_t* n);

/* subband_layout(t, dims): (scale, direction) per subband, lowpass (0, 0)
 * first; arrays of nsubbands entries.  src/transforms/ns_surfacelet.jl:518-525. */
int sfl_ns_layout(const sfl_ns_params* p, int32_t* scale, int32_t* direction);

/* Integer directional level L to a level matrix: src/types/transforms.jl:270-278. */
int sfl_surf_levels_from_int(int32_t L, int32_t out[3][3]);

/* Constructor validation of Surfacelet: src/types/transforms.jl:231-251. */
int sfl_surf_check_params(const sfl_surf_params* p);

/* Subband sizes and layout, with the reference's size validation
 * (src/transforms/surfacelet.jl:230-308).  *n receives the subband count;
 * sizes (3 per subband), scale, hourglass and wedge may be NULL. */
int sfl_surf_layout(const sfl_surf_params* p, const int32_t dims[3], int32_t* n,
                    int32_t* sizes, int32_t* scale, int32_t* hourglass, int32_t* wedge);

/* surfacelet_redundancy(t, dims): src/transforms/surfacelet.jl:220-222. */
int sfl_surf_redundancy(const sfl_surf_params* p, const int32_t dims[3], double* r);

/* ── Plans (make_workspace) ─────────────────────────────────────────────── */

/* make_workspace(t::NSSurfacelet, T, dims): src/transforms/ns_surfacelet.jl:88-123.
 * Designs the masks in float64, stores them as float32 on the current device
 * and allocates the scratch.  dtype is SFL_REAL32 or SFL_COMPLEX64. */
int sfl_ns_plan_create(const sfl_ns_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out);

/* The standalone directional bank on the NSSurfacelet kernels: parameter
 * check (host only; "levels must be ≥ 0", "transition must be ≥ 0" as in
 * src/directional/ndfb.jl:98-99) and plan.  The plan takes sfl_analyze
 * (ndfb_decompose!, src/directional/ndfb.jl:276), sfl_synthesize
 * (ndfb_reconstruct!, :384), the adjoints and the streaming entry points
 * (ndfb_decompose(f, ...), :317); coefficients are (n1, n2, n3, 3 * 2^levels). */
int sfl_ndfb_check_params(const sfl_ndfb_params* p);
int sfl_ndfb_plan_create(const sfl_ndfb_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out);

/* make_workspace(t::Surfacelet, T, dims): src/transforms/surfacelet.jl:126-149. */
int sfl_surf_plan_create(const sfl_surf_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out);

/* Releases a plan and its device memory (synchronizes the device first). */
int sfl_plan_destroy(sfl_plan* plan);

/* transform(ws), size(ws), eltype(ws), nsubbands, coefficient count:
 * src/transforms/ns_surfacelet.jl:78-80, src/transforms/surfacelet.jl:63-65. */
int sfl_plan_info(const sfl_plan* plan, int32_t* kind, int32_t dims[3], int32_t* dtype,
                  int32_t* nsubbands, int64_t* ncoeffs);

/* subband(t, c, i): shape of subband i (1-based) and its element offset in
 * the coefficients.  src/transforms/ns_surfacelet.jl:539,
 * src/transforms/surfacelet.jl:444. */
int sfl_subband_info(const sfl_plan* plan, int32_t i, int32_t shape[3], int64_t* offset);

/* The plan's status word, written by kernels whose bounded waits ran out
 * (0 = fine, 1 = a bulk-copy barrier wait timed out).  It lives in mapped
 * host memory; this call synchronizes with the device first, and reset != 0
 * clears it.  Every compute call on an NS plan also checks it before
 * enqueueing anything: a nonzero word is reported once, as SFL_ERR_TIMEOUT
 * (the word is cleared, the call does nothing; the earlier call's results are
 * not valid).  No counterpart in the reference. */
int sfl_plan_status(sfl_plan* plan, int32_t* status, int32_t reset);

/* Self-test of the bounded waits: one kernel waits, with a short iteration
 * limit, on an mbarrier that nothing completes (no copy in flight), so the
 * wait runs out and the plan's status word records 1.  The next compute call
 * on the plan returns SFL_ERR_TIMEOUT once.  NS plans only.  No counterpart
 * in the reference. */
int sfl_plan_selftest_wait(sfl_plan* plan, void* stream);

/* Subbands a launch keeps in flight (NS: scratch holds that many spectra).
 * Default 8; only affects speed and scratch size. */
int sfl_plan_set_group(sfl_plan* plan, int32_t group);

/* NSSurfacelet kernel pipeline.  All give the same subbands to float32
 * rounding; they differ in speed only.
 *   SLABS (default where supported: axes 1 and 2 of length 64, 96, 128, 160
 *     or 256, axis 3 of length 16, 32, 64, 96, 128, 160 or 256): a line pass
 *     along axis 3 plus one pass per axis-3 slab, skipping the zero rows and
 *     columns of band-limited masks.
 *   LINES (default elsewhere): one line pass per axis.
 *   PLANES: retired (the plane-major pipeline was slower than SLABS at every
 *     size it supported); selecting it returns SFL_ERR_ARGUMENT.
 * Not while a streaming pass is open. */
#define SFL_PIPELINE_LINES 0
#define SFL_PIPELINE_PLANES 1
#define SFL_PIPELINE_SLABS 2
int sfl_plan_set_pipeline(sfl_plan* plan, int32_t pipeline);

/* The plan's pipeline and group.  No counterpart in the reference. */
int sfl_plan_tuning(const sfl_plan* plan, int32_t* pipeline, int32_t* group);

/* The tile of the slab pipeline's axis-3 analysis pass: subbands a CTA takes
 * (1, 2, 4 or 8; 0 = the default: the SFL_MASK_IPC environment variable if
 * set, else 8, halved per launch while the launch holds fewer CTAs than the
 * GPU has SMs).  A tile set here is used as given.
 * set != 0 writes *ipc, else reads it.  The autotuner picks it after the
 * pipeline and group.  NS plans only.  No counterpart in the reference. */
int sfl_plan_tile(sfl_plan* plan, int32_t set, int32_t* ipc);

/* Times analysis of x (into c, overwritten) followed by synthesis (into a
 * scratch volume of its own) under every pipeline that fits the size and
 * groups of 2, 4 and 8 subbands, then, on the slab pipeline, the axis-3 tile
 * of 1, 2 or 4 subbands a CTA against the default 8 (sfl_plan_tile); keeps the
 * fastest and records it for the process: NS and NDFB plans created later
 * with the same transform, size and element type start with it.
 * Synchronizes; reallocates the plan's scratch.  No-op for decimated plans.
 * No counterpart in the reference (its plans are FFTW-tuned instead). */
int sfl_plan_autotune(sfl_plan* plan, const void* x, void* c, void* stream);

/* ── Transforms ─────────────────────────────────────────────────────────── */

/* analyze!(c, t, x; workspace): src/transforms/ns_surfacelet.jl:551-566,
 * src/transforms/surfacelet.jl:446-454. */
int sfl_analyze(sfl_plan* plan, const void* x, void* c, void* stream);

/* synthesize!(x, t, c; workspace): src/transforms/ns_surfacelet.jl:568-581,
 * src/transforms/surfacelet.jl:456-464. */
int sfl_synthesize(sfl_plan* plan, const void* c, void* x, void* stream);

/* Adjoint of analyze (x = A^T c).  The reference has no adjoint entry point:
 * for a tight NSSurfacelet the inverse is the adjoint
 * (src/transforms/ns_surfacelet.jl:21-25) and this equals sfl_synthesize;
 * otherwise (tight = false, and the decimated transform, whose checkerboard
 * filters are biorthogonal, src/transforms/surfacelet.jl:24-26) it applies
 * the transposed analysis operator. */
int sfl_adjoint_analyze(sfl_plan* plan, const void* c, void* x, void* stream);

/* Adjoint of synthesize (c = S^T x); equals sfl_analyze for a tight NSSurfacelet. */
int sfl_adjoint_synthesize(sfl_plan* plan, const void* x, void* c, void* stream);

/* ── Streaming (NSSurfacelet only) ─────────────────────────────────────── */

/* Streaming analyze(f, t, x): src/transforms/ns_surfacelet.jl:474-479, 620-624.
 * begin transforms x once; each next writes the next subband (a volume of
 * the plan's dims and element type) to `band` and its 1-based index to
 * *index, in the reference's order: the directional subbands in increasing
 * index, then the lowpass (index 1).  next returns SFL_DONE after the last. */
int sfl_stream_analyze_begin(sfl_plan* plan, const void* x, void* stream);
int sfl_stream_analyze_next(sfl_plan* plan, void* band, int32_t* index, void* stream);

/* Streaming synthesize!(f, x, t): src/transforms/ns_surfacelet.jl:483-500,
 * 626-641.  next_index tells which subband the plan wants next (same order as
 * analysis; SFL_DONE when all were pushed); push consumes it; end writes x. */
int sfl_stream_synthesize_begin(sfl_plan* plan, void* stream);
int sfl_stream_synthesize_next_index(sfl_plan* plan, int32_t* index);
int sfl_stream_synthesize_push(sfl_plan* plan, const void* band, void* stream);
int sfl_stream_synthesize_end(sfl_plan* plan, void* x, void* stream);

/* ── Allocation-free single-subband analysis ─────────────────────────────
 * No counterpart in the reference.  Writes NSSurfacelet analysis subband
 * `index` (1-based, subband_layout order) of the real float32 volume x to
 * `band` (device memory of the plan's dims), and allocates nothing: its
 * scratch is a static 4 MiB device array inside the library, so it suits
 * callers that cannot allocate device memory when they transform
 * (allocation-free real-time loops, processes whose memory manager owns the
 * device).  Call it from ordinary host code: it launches kernels, so it may
 * not run inside a cudaLaunchHostFunc callback.  Create the plan (which
 * allocates the mask tables) beforehand, and make the first call for each
 * plan size at start-up too: the first call on a device looks up the
 * scratch's device address (cudaGetSymbolAddress), and under lazy module
 * loading a kernel's first launch loads its code; both belong before the
 * allocation-free phase.  The address is
 * cached per device for the process; do not call this again on a device
 * after cudaDeviceReset.  Limits: real plans only, and (n1/2+1)*n2*n3 <=
 * 262144 (e.g. 64^3); larger sizes return SFL_ERR_ARGUMENT.  All calls share
 * the scratch: calls that overlap on the GPU race, so order them (one
 * stream, or explicit synchronization). */
int sfl_ns_analyze_subband_static(sfl_plan* plan, const void* x, void* band, int32_t index, void* stream);

/* ── Design tables (host only; for tests and inspection) ──────────────────
 * Writes the float64 design table `name` (index selects one of several) of a
 * transform on `dims` to out (when not NULL) and its element count to *count.
 * Names (NS): "m1", "m2", "wedge" (index = ((scale-1)*3 + hourglass-1)*64*2
 * + plane*64 + wedge-1, plane 0 = a, 1 = b), "pa" (index = level*3 + axis),
 * "pl" (same), "group" (B_j times the hourglass factor of a plan's group
 * table; index = (scale-1)*3 + hourglass-1), "bandpass" (B_j; index = level,
 * 0 = finest), "hourglass" (the standalone bank's mask; index = hourglass-1).
 * Names (decimated): "ritf" (index = level*3 + K-1),
 * "irc" (complex as re/im pairs; index = ((level*3 + K-1)*32 + stage)*4 + which,
 * which 0,1 = analysis channel 0,1 and 2,3 = synthesis channel 0,1),
 * "pyr_prof" (index = level*3 + axis).  No counterpart in the reference's
 * interface: it exposes the internal tables of src/directional/*.jl. */
int sfl_ns_design_table(const sfl_ns_params* p, const int32_t dims[3], const char* name,
                        int32_t index, double* out, int64_t* count);
int sfl_surf_design_table(const sfl_surf_params* p, const int32_t dims[3], const char* name,
                          int32_t index, double* out, int64_t* count);
/* The float32 tables an NSSurfacelet or NDFB plan holds on the device (designed
 * there in float64): "group" (index = (scale-1)*3 + hourglass-1) and, for an
 * untight plan, "bandpass" (index = level, 0 = finest).  Writes H = (n1/2+1)
 * n2 n3 floats to the host buffer out (when not NULL) and H to *count.
 * Equal bit for bit to the float64 host design rounded to float32. */
int sfl_ns_plan_table(sfl_plan* plan, const char* name, int32_t index, float* out, int64_t* count);
/* The float32 tables a Surfacelet plan holds on the device (composed there in
 * float64 from the host's separable factors, src/directional/ritf.jl:89-108,
 * src/directional/irc.jl:49-67): "ritf" (V_K on the half-K grid; index =
 * level*3 + K-1) and "irc" (one stage's slice plane as re/im pairs; index as
 * in sfl_surf_design_table).  Writes the float count to *count and the values
 * to the host buffer out when not NULL.  No counterpart in the reference. */
int sfl_surf_plan_table(sfl_plan* plan, const char* name, int32_t index, float* out, int64_t* count);

/* ── Soft-threshold denoiser (NSSurfacelet and NDFB plans, Float32) ─────
 * No counterpart in the reference.  y = synthesize(soft(analyze(x), tau)),
 * soft(c) = sign(c) max(|c| - tau[s-1], 0) on subband s; tau is S float32
 * thresholds in device memory, by subband index.  On the slab pipeline the
 * coefficients never reach device memory (analysis, threshold and synthesis
 * of a subband meet in one slab pass); equal bit for bit to the three calls. */
int sfl_ns_denoise(sfl_plan* plan, const void* x, void* y, const float* tau, void* stream);

/* ── Item ranges (NSSurfacelet; sharding subbands across devices) ────────
 * No counterpart in the reference.  The subbands in stream order (stream_order
 * gives the subband index at each of the S positions) split into ranges:
 *   forward_spectrum   X = the spectrum of x, nch x spectrum_elems complex
 *                      float32 bins in the plan's internal layout (opaque);
 *   analyze_range      the subbands at positions [first, first + count) from
 *                      X into count consecutive volumes of c;
 *   accumulate_range   their synthesis contributions into the spectrum A
 *                      (clear != 0 zeroes A first);
 *   inverse_spectrum   x from an accumulated spectrum (A is overwritten).
 * Accumulated spectra add: the sum over devices of each device's
 * accumulation of its own ranges is the accumulation of all of them.  Slab
 * and line pipelines only; not while a stream is open.  X and A are
 * 16-byte aligned device buffers. */
int sfl_ns_spectrum_elems(const sfl_plan* plan, int64_t* elems);
int sfl_ns_stream_order(const sfl_plan* plan, int32_t* subband_index);
int sfl_ns_forward_spectrum(sfl_plan* plan, const void* x, void* X, void* stream);
int sfl_ns_analyze_range(sfl_plan* plan, const void* X, int32_t first, int32_t count, void* c, void* stream);
int sfl_ns_accumulate_range(sfl_plan* plan, const void* c, int32_t first, int32_t count, void* A, int32_t clear,
                            void* stream);
int sfl_ns_inverse_spectrum(sfl_plan* plan, void* A, void* x, void* stream);

/* ── bfloat16 coefficients (NSSurfacelet, Float32 volumes) ─────────────────
 * No counterpart in the reference.  c is (n1, n2, n3, S) bfloat16, column-
 * major like the float32 coefficients; scales holds S float32 (device
 * memory): subband s = scales[s-1] * c[..., s-1], each scale the power of two
 * at or above the subband's largest magnitude.  Half the coefficient memory
 * of float32 at bfloat16 accuracy (about 3 significant digits).  Slab and
 * line pipelines only. */
int sfl_ns_analyze_bf16(sfl_plan* plan, const void* x, void* c, float* scales, void* stream);
int sfl_ns_synthesize_bf16(sfl_plan* plan, const void* c, const float* scales, void* x, void* stream);

/* ── Batches ─────────────────────────────────────────────────────────────
 * Many transforms as one CUDA graph: batch_create runs each entry (plan,
 * operator, input, output) once eagerly, then captures the sequence
 * (distinct plans on up to eight concurrent branches, each plan dealt out,
 * largest work first, to the branch with the least work so far; the entries
 * of one plan keep their order, so an entry may consume an earlier one's
 * output) and
 * instantiates it; batch_run replays it on a stream with the same pointers,
 * whose contents may change between runs.  The plans must stay alive and
 * must not be used elsewhere while a run is in flight.  No counterpart in the
 * reference, whose batches are loops of plain calls. */
typedef struct sfl_batch sfl_batch;
#define SFL_OP_ANALYZE 0
#define SFL_OP_SYNTHESIZE 1
#define SFL_OP_ADJOINT_ANALYZE 2
#define SFL_OP_ADJOINT_SYNTHESIZE 3
#define SFL_OP_COPY_VOLUME 4   /* copy one volume of the plan's size (host <-> device, pinned host memory) */
int sfl_batch_create(int32_t n, sfl_plan* const* plans, const int32_t* ops, const void* const* inputs,
                     void* const* outputs, sfl_batch** out);
int sfl_batch_run(sfl_batch* batch, void* stream);
int sfl_batch_destroy(sfl_batch* batch);

/* ── Launch timing (benchmark instrumentation) ───────────────────────────
 * No counterpart in the reference.  While enabled, every kernel launch of the
 * library is bracketed by two CUDA events on its stream and filed under its
 * kernel tag; read sums the elapsed times of one tag (NULL = all), waiting
 * for the events.  tags writes the newline-separated tag list to buf. */
int sfl_profile_enable(int32_t on);
int sfl_profile_reset(void);
int sfl_profile_read(const char* tag, double* total_ms, int64_t* launches);
int sfl_profile_tags(char* buf, int64_t cap);
/* Algorithmic bytes (each input read once, each output written once) of the
 * profiled launches of a tag (all tags when tag is NULL), where the launch
 * site reports them. */
int sfl_profile_bytes(const char* tag, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* SURFACELETS_B200_H */
