/*
 * litho_b200.h — C ABI of liblitho_b200.so, the sm_100a imaging engine.
 *
 * The library computes the partially coherent aerial image of a thin mask
 * (the Abbe sum over source points, scalar or vector), its sum-of-coherent-
 * systems (SOCS) form, and the inverse-lithography adjoint, on one CUDA
 * device. It replaces the numpy hot path of Lithobat's imaging package
 * (litho_sim.expose / litho_sim.opc.ilt); each entry point names the
 * reference function it stands in for.
 *
 * Conventions
 *   - Every pointer named *_dev is device memory; everything else is host.
 *   - The caller owns every buffer, including the workspace. No entry point
 *     allocates or frees device memory; size the workspace with the matching
 *     *_workspace() call.
 *   - Work is enqueued on the given stream and returns without a host
 *     synchronisation. Entry points are re-entrant across streams as long as
 *     each call has its own workspace.
 *   - Return value: 0 on success, a negative LITHO_E* code for a rejected
 *     argument (nothing was launched), or a positive CUDA error code if a
 *     launch failed. litho_status_string() describes any of them.
 *   - Frequencies follow numpy's FFT ordering: signed bin k in [-N/2, N/2)
 *     is physical frequency k / (N * pixel_size).
 */
#ifndef LITHO_B200_H
#define LITHO_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LITHO_OK 0
#define LITHO_E_NULL -1          /* a required pointer is NULL               */
#define LITHO_E_SIZE -2          /* a size or count is out of range          */
#define LITHO_E_WORKSPACE -3     /* workspace smaller than *_workspace()     */
#define LITHO_E_BAND -4          /* band / coarse-grid geometry inconsistent */
#define LITHO_E_UNSUPPORTED -5   /* valid request this build does not serve  */
#define LITHO_E_ALIGN -6         /* a pointer is not 16-byte aligned         */
#define LITHO_E_DEVICE -7        /* device is not sm_100 or not reachable    */
#define LITHO_E_SCRATCH -8       /* needs more than the fixed no-allocation scratch */
#define LITHO_E_TIMEOUT 1000001  /* a bounded device wait gave up           */

/* Size of the fixed device scratch litho_abbe_noalloc() runs in. */
#define LITHO_NOALLOC_SCRATCH_BYTES (32u << 20)

/* ---- descriptors (plain data; layouts are fixed, see static sizes) ----- */

/* One optical state: the pupil of one clip at one image plane.
 * Replaces the arguments of expose/aerial_image.py:_pupil_phase (:142-166)
 * and expose/pupil.py:vector_coefficients (:292-369). */
typedef struct LithoPupil {
    double wavelength;    /* m                                              */
    double NA;
    double defocus;       /* m, this plane's defocus                        */
    double n_image;       /* image-space index of this plane                */
    double zernike[21];   /* waves; zernike[j-1] multiplies Noll Z_j        */
    int32_t exact_defocus;/* non-paraxial defocus OPD (pupil.py:214-221)    */
    int32_t vector;       /* 1: three field components (Ex, Ey, Ez)         */
    int32_t obliquity;    /* sqrt(cos theta) factor in the vector model     */
    int32_t has_zernike;  /* any zernike[] non-zero                         */
} LithoPupil;             /* 216 bytes */

/* One coherent system of the Abbe sum: a source point, an image plane and
 * (vector model) one incoherent polarisation state. Replaces one iteration of
 * the source loop in expose/aerial_image.py:_abbe_sum (:421-486). */
typedef struct LithoJob {
    double fsx, fsy;      /* source-point frequency offset, 1/m             */
    double jx, jy;        /* Jones vector of the state (vector model)       */
    double weight;        /* source weight x state weight                   */
    int32_t pupil;        /* index into the LithoPupil table                */
    int32_t clip;         /* which mask                                     */
    int32_t out;          /* which output image                             */
    int32_t cx, cy;       /* integer bin nearest the source offset          */
    int32_t ncomp;        /* 1 scalar, 3 vector                             */
    int32_t tab;          /* pupil-table slot; jobs of clips that share an  */
                          /* optical state and source point share a slot    */
} LithoJob;               /* 72 bytes */

/* A contiguous run of jobs, all for one output image, accumulated by one
 * thread block. */
typedef struct LithoItem {
    int32_t out, job_begin, job_end, pad;
} LithoItem;

/* Per-output normalisation (expose/aerial_image.py:normalisation_scale,
 * :217-241). mode 0: multiply by `scale` (clear, none, or 1 for raw output);
 * mode 1: peak normalisation, scale = dose / peak computed on the device. */
typedef struct LithoNorm {
    int32_t mode;
    float scale;          /* mode 0: the factor; mode 1: the dose           */
} LithoNorm;

/* The blank under a reflective (EUV) mask, for mask_model="multilayer"
 * (expose/m3d/provider.py:MultilayerSpectra, :190-295). The spectrum of
 * source point (fsx, fsy) at order frequency (FX, FY) is multiplied by the
 * blank's reflection r(theta), sin(theta) = |(tilt lambda fs / m + chief ray)
 * + lambda F / m| (provider.py:72-126, :260-264); the multiply is folded into
 * the pupil table. r is the linear interpolation, in theta, of |r| and of the
 * unwrapped arg r on an ascending angle table (clamped at its ends); orders
 * with sin(theta) > 1 get 0. One entry per LithoPupil when a plan sets
 * `mirrored`. */
typedef struct LithoMirror {
    double wavelength;    /* m                                              */
    double reduction;     /* mask-to-wafer demagnification                  */
    double tilt_sign;     /* source offset -> mask-side sine sign (-1)      */
    double sin_cx, sin_cy;/* chief-ray direction sines at the mask          */
    int32_t n_theta;      /* table length (>= 2); 0: thin mask, no multiply */
    int32_t pad;
    int64_t off_table;    /* bytes from the start of the LithoMirror array  */
                          /* to double[3][n_theta]: theta (rad), |r|, arg r */
} LithoMirror;            /* 56 bytes */

/* Geometry and counts of one Abbe batch. All clips share the grid. The
 * device "plan blob" holds the job/pupil/item/norm arrays at the byte
 * offsets given here (each 16-byte aligned). */
typedef struct LithoAbbePlan {
    int32_t n;            /* grid side N                                    */
    int32_t n_clips;      /* masks in the batch                             */
    int32_t n_out;        /* output images (clips x planes)                 */
    int32_t n_jobs;
    int32_t n_items;
    int32_t n_pupils;
    int32_t h;            /* half-width of a source point's disc, bins      */
    int32_t bm;           /* half-width of the mask band, bins              */
    int32_t L;            /* coarse grid side (>= 4h+1, power of two): 32 or */
                          /* 64 on chip; 128..1024 (<= n) wide-pupil engine */
    int32_t mask_complex; /* 0: float32 masks, 1: complex64 masks           */
    int32_t ncomp_max;    /* 1 or 3                                         */
    int32_t n_tab;        /* pupil-table slots (max LithoJob.tab + 1)       */
    double pixel_size;    /* m                                              */
    int64_t off_jobs, off_pupils, off_items, off_out_items, off_norm;
    int64_t off_slots;    /* int32[n_tab]: a job that owns each table slot  */
    int32_t mirrored;     /* 1: LithoMirror[n_pupils] at off_mirrors        */
    int32_t pad_m;
    int64_t off_mirrors;
} LithoAbbePlan;

/* One size group of an uneven batch (litho_uneven_run): a plan whose clips
 * share one grid side, its device buffers, and the work-queue sizes the
 * tuner picks (0 selects the default of each). Groups of the wide-pupil
 * engine (plan.L >= 128) run their coherent passes in the shared queue;
 * groups on the coarse grids of 32 / 64 points run litho_abbe_tabled(). */
typedef struct LithoUnevenGroup {
    LithoAbbePlan plan;
    const void* blob_host;    /* the plan blob in host memory (the schedule  */
                              /* reads its work items)                        */
    const void* blob_dev;     /* the same blob on the device                  */
    const void* table_dev;    /* litho_abbe_pupil_table() of the plan         */
    const void* masks_dev;    /* [n_clips][N][N]                              */
    float* image_dev;         /* [n_out][N][N]                                */
    float* peak_dev;          /* [n_out]                                      */
    void* workspace_dev;      /* litho_uneven_group_workspace() bytes         */
    size_t ws_bytes;
    int32_t slot_kib;         /* pass-A buffer slot target, KiB (0: 16        */
                              /* transforms per resident block, 16 MiB..1 GiB)*/
    int32_t n_slots;          /* slots in flight, >= 2 (2)                    */
    int32_t a_units;          /* warp transforms of 1024/L rows per pass-A    */
                              /* task (96)                                    */
    int32_t b_rows;           /* row blocks per pass-B task (2 at L = 128,    */
                              /* else 1)                                      */
} LithoUnevenGroup;           /* 200 bytes */

/* One task of the uneven work queue (written by litho_uneven_schedule). */
typedef struct LithoQueueTask {
    int32_t kind;             /* 0: pass A (row transforms), 1: pass B        */
    int32_t group;            /* wide group, in the schedule's order          */
    int32_t slot;             /* pass-A buffer slot                           */
    int32_t base;             /* first job of the slot's chunk                */
    int32_t first;            /* A: first job; B: work item                   */
    int32_t count;            /* A: jobs; B: first row block                  */
    int32_t rows;             /* B: row blocks                                */
    int32_t wait_ctr;         /* counter to wait for (-1: none)               */
    int32_t wait_value;       /* ... until it reaches this value              */
    int32_t done_ctr;         /* counter incremented when the task is done    */
} LithoQueueTask;             /* 40 bytes */

/* ---- library ----------------------------------------------------------- */

/* Human-readable text for a status code returned by any entry point. */
const char* litho_status_string(int status);

/* ABI version (major * 10000 + minor * 100 + patch). */
int litho_version(void);

/* sizeof() of the public structs, in declaration order: LithoPupil,
 * LithoJob, LithoItem, LithoNorm, LithoAbbePlan, LithoMirror,
 * LithoUnevenGroup, LithoQueueTask. Writes min(n, 8) values; returns how many
 * structs the ABI has. For binding generators. */
int litho_abi_sizes(int32_t* out, int n);

/* ---- Abbe imaging ------------------------------------------------------ */

/* Workspace bytes litho_abbe() needs for this plan. */
int litho_abbe_workspace(const LithoAbbePlan* plan, size_t* bytes);

/* litho_abbe() for callers that cannot allocate device memory for a
 * workspace (every device byte owned by another allocator, or a loop that
 * must not pay cudaMalloc's implicit synchronisation). It has no counterpart
 * in the reference, which allocates freely on the host. The kernels run in a
 * fixed LITHO_NOALLOC_SCRATCH_BYTES (32 MiB) buffer compiled into the
 * library, held on every GPU that loads it until exit; plans whose
 * litho_abbe_workspace() exceeds that are rejected with LITHO_E_SCRATCH
 * before anything is launched. The entry point allocates nothing. Its first
 * call on each device looks up that device's copy of the buffer
 * (cudaGetSymbolAddress), so make that first call before any stream capture.
 * All calls share the one buffer: calls that may overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. */
int litho_abbe_noalloc(const LithoAbbePlan* plan, const void* plan_blob_dev,
                       const void* mask_dev, float* image_dev, float* peak_dev,
                       cudaStream_t stream);

/* litho_abbe_status() for the fixed scratch of litho_abbe_noalloc() on the
 * current device: synchronise `stream` and return 0, or LITHO_E_TIMEOUT if a
 * bounded wait inside the last litho_abbe_noalloc() call on this device gave
 * up (its images and peaks are then invalid). No counterpart in the
 * reference; allocates nothing. */
int litho_abbe_noalloc_status(const LithoAbbePlan* plan, cudaStream_t stream);

/* Synchronise `stream` and return the device status word of the last
 * litho_abbe*() call that used this workspace: 0, or LITHO_E_TIMEOUT if a
 * bounded wait inside a kernel gave up (its outputs are then invalid). */
int litho_abbe_status(const LithoAbbePlan* plan, const void* workspace_dev, cudaStream_t stream);

/* Test hooks of the failure reporting (no counterpart in the reference, which
 * reports failures on the host only: app/worker.py:84-88). Every wait inside
 * a kernel is bounded; one that gives up drains its block's copies and MMAs
 * in flight, sets LITHO_E_TIMEOUT in the call's status word (the first word
 * of its workspace) and lets the block exit, so nothing hangs or faults.
 *
 * litho_set_wait_limit: the clock budget (cycles) of the waits that make
 * progress, on the current device; 0 restores the default (~2 s). Drain waits
 * keep the full budget. A short limit makes a pipeline report LITHO_E_TIMEOUT
 * with invalid outputs: for tests only. Synchronous.
 *
 * litho_wait_probe: one thread waits `cycles` (1 .. 4e9) on an mbarrier that
 * nothing arrives at and sets *status_dev = LITHO_E_TIMEOUT, exactly as a
 * pipeline wait that gives up. Pass a workspace's first word to check that a
 * status reader (litho_abbe_status and the like) sees it. */
int litho_set_wait_limit(long long cycles);
int litho_wait_probe(int* status_dev, long long cycles, cudaStream_t stream);

/* The clear throughput of every output in FP64, on the device: what an
 * unpatterned mask images to (expose/aerial_image.py:_abbe_sum, :464 for the
 * scalar model, :482-486 for the vector model, times the blank's specular
 * |r|^2 for a mirrored mask, :431-438): clear_out_dev[o] = sum over the
 * output's jobs of weight x [rho(DC) <= 1] x sum_c |V_c(DC)|^2 x |r|^2.
 * The `clear` normalisation divides the raw image by it. */
int litho_abbe_clear(const LithoAbbePlan* plan, const void* plan_blob_dev, double* clear_out_dev,
                     cudaStream_t stream);

/* Which engine litho_abbe() runs for this plan (no counterpart in the
 * reference, which has one dense path): info[0] = 1 for the on-chip coarse
 * grid (L = 32 or 64), 2 for the wide-pupil engine (L = 128..1024); info[1]
 * = the image synthesis: 0 direct with a normalising pass, 1 row-pair FFT,
 * 2 tcgen05 tensor cores (FP16 hi/lo planes), 3 the wide engine's own.
 * Writes min(n, 2) values. For tests and launch accounting. */
int litho_abbe_engine(const LithoAbbePlan* plan, int32_t* info, int n);

/* Bytes of the pupil table of a plan: n_tab x ncomp_max x (2h+1)^2 complex
 * float. The table depends on the optics and source only, not on the masks,
 * so a caller imaging many batches with the same plan builds it once. */
int litho_abbe_table_bytes(const LithoAbbePlan* plan, size_t* bytes);

/* Fill table_dev with every slot's pupil P (x V_c) on its (2h+1)^2 box:
 * expose/aerial_image.py:_pupil_geometry/_pupil_phase (:86-166) and
 * expose/pupil.py:vector_coefficients (:292-369), evaluated in FP64 with the
 * reference's exact aperture test rho <= 1, stored as complex float. */
int litho_abbe_pupil_table(const LithoAbbePlan* plan, const void* plan_blob_dev,
                           void* table_dev, cudaStream_t stream);

/* litho_abbe() with a table built by litho_abbe_pupil_table() for this plan. */
int litho_abbe_tabled(const LithoAbbePlan* plan, const void* plan_blob_dev,
                      const void* table_dev, const void* mask_dev, float* image_dev,
                      float* peak_dev, void* workspace_dev, size_t workspace_bytes,
                      cudaStream_t stream);

/* litho_abbe_tabled() for masks given as level maps: one byte per pixel,
 * mask_idx_dev[clip][y][x] indexing that clip's complex levels
 * levels_dev[clip][0 .. n_levels) (float2; an index >= n_levels takes the
 * last level). Binary and attenuated phase-shift masks have two levels (the
 * reference builds them as 0/1 arrays or as 1 and sqrt(T) e^{i phase},
 * mask/patterns.py), so the mask crosses the host link and HBM at 1 byte per
 * pixel instead of 8 (complex64), with the same images: the level values are
 * exactly the complex mask's values. Coarse-grid plans (plan.L <= 64) whose
 * band fits the register band transform; LITHO_E_UNSUPPORTED otherwise. The
 * plan's mask_complex is ignored. */
int litho_abbe_levels(const LithoAbbePlan* plan, const void* plan_blob_dev, const void* table_dev,
                      const uint8_t* mask_idx_dev, const void* levels_dev, int n_levels, float* image_dev,
                      float* peak_dev, void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);

/* The raw Abbe sum, normalised per output, for a batch of clips.
 * Replaces expose/aerial_image.py:_abbe_sum (:351-494) together with
 * compute_aerial_image (:502-548) and compute_aerial_planes (:551-587):
 *   image_dev[o]  = raw_o * s_o   (s_o from LithoNorm, raw if scale 1)
 *   peak_dev[o]   = max of raw_o (before scaling)
 * mask_dev: [n_clips][N][N] float32 or complex64 (row = y, column = x). */
int litho_abbe(const LithoAbbePlan* plan, const void* plan_blob_dev,
               const void* mask_dev, float* image_dev, float* peak_dev,
               void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);

/* litho_abbe() run `reps` times with CUDA events between its stages, for
 * measurement. stage_ms[0..6] receives the mean milliseconds of: pupil
 * table, mask band rows, mask band columns, coarse accumulation, coarse
 * reduction, then the peak pass and the writing synthesis pass (on grids
 * without the pair-FFT synthesis, and on the wide-pupil engine: synthesis,
 * then normalisation). Synchronises the stream. */
int litho_abbe_profile(const LithoAbbePlan* plan, const void* plan_blob_dev,
                       const void* table_dev /* NULL: built each run */, const void* mask_dev, float* image_dev, float* peak_dev,
                       void* workspace_dev, size_t workspace_bytes, cudaStream_t stream,
                       int reps, float* stage_ms);

/* ---- uneven batches ------------------------------------------------------
 * Clips of several grid sides imaged in one call: the reference images one
 * clip per compute_aerial_image() call whatever its size
 * (expose/aerial_image.py:502-548, batching transforms only within a clip in
 * _Batch, :312-348). Here every size group's coherent transforms on the
 * wide-pupil coarse grids run in ONE persistent kernel that drains a device
 * work queue of (chunk of jobs, pass A) and (work item, row block, pass B)
 * tasks across all groups; each task waits (bounded) on counters of earlier
 * tasks only, so the queue cannot deadlock. Usage: size every group's
 * workspace, build the schedule once on the host, copy the task list to the
 * device, then call litho_uneven_run() per batch (it is stream-ordered and
 * holds no host synchronisation, so it can be captured in a CUDA graph once
 * the device's twiddle tables exist, i.e. after one uncaptured call). */
int litho_uneven_group_workspace(const LithoUnevenGroup* group, size_t* bytes);

/* The task list of a batch: call with tasks == NULL for *n_tasks and
 * *n_counters, then with a buffer of max_tasks >= *n_tasks. Host only. */
int litho_uneven_schedule(const LithoUnevenGroup* groups, int n_groups, LithoQueueTask* tasks,
                          int max_tasks, int* n_tasks, int* n_counters);

/* Bytes of the queue's own workspace (status word, head, counters). */
int litho_uneven_queue_workspace(int n_counters, size_t* bytes);

/* Image every group: coarse-grid groups through litho_abbe_tabled(), then the
 * wide groups' band DFTs, the queue launch and their reductions, syntheses
 * and normalisations. Outputs as litho_abbe() per group. */
int litho_uneven_run(const LithoUnevenGroup* groups, int n_groups, const LithoQueueTask* tasks_dev,
                     int n_tasks, int n_counters, void* queue_workspace_dev, size_t queue_ws_bytes,
                     cudaStream_t stream);

/* Synchronise `stream` and return the queue's status word: 0, or
 * LITHO_E_TIMEOUT if a task's bounded wait gave up in the last run, or
 * LITHO_E_BAND if the task list held a task outside its group's buffers
 * (skipped); either way the images are invalid. Each group's own word:
 * litho_abbe_status(). */
int litho_uneven_status(const void* queue_workspace_dev, cudaStream_t stream);

/* Workspace bytes litho_abbe_plain() needs when it transforms `batch`
 * coherent systems (times their field components) at a time. */
int litho_abbe_plain_workspace(const LithoAbbePlan* plan, int batch, size_t* bytes);

/* The same images as litho_abbe(), by the plain per-source-point method:
 * every coherent system gets a full N x N spectrum in HBM, a row and a
 * column inverse FFT and a separate |E|^2 accumulate — the reference's
 * _abbe_sum loop and batched flush (expose/aerial_image.py:421-488, :336-348)
 * moved to the GPU unchanged. Power-of-two N in [16, 4096]. The comparison
 * baseline for the band-limited engine. */
int litho_abbe_plain(const LithoAbbePlan* plan, int batch, const void* plan_blob_dev,
                     const void* mask_dev, float* image_dev, float* peak_dev,
                     void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);

/* Workspace bytes of litho_plain_socs_forward() / litho_plain_socs_adjoint(). */
int litho_plain_socs_workspace(int n_clips, int n, size_t* bytes);

/* The plain SOCS forward of opc/ilt.py:socs_fields (:227-231) on full grids:
 * fields_out[k][c] = ifft2(phi_k fft2(mask_c)) (complex64, K x C x N x N),
 * I_out[c] = sum_k lambda_k |fields|^2; phi: K x nb band values at signed
 * bins (bkx, bky); lam_host: K host floats. Power-of-two N. The comparison
 * baseline for the band-limited ILT stages. */
int litho_plain_socs_forward(const float* masks_dev, int n_clips, int n, int K, const float2* phi_dev,
                             const float* lam_host, const int32_t* bkx_dev, const int32_t* bky_dev,
                             int nb, float2* fields_out_dev, float* I_out_dev, void* workspace_dev,
                             size_t workspace_bytes, cudaStream_t stream);

/* The plain adjoint of opc/ilt.py:socs_gradient (:262-266) on full grids:
 * grad_out[c] = 2 Re sum_k lambda_k ifft2(conj(phi_k) fft2(sens_c fields[k][c])). */
int litho_plain_socs_adjoint(const float2* fields_dev, const float* sens_dev, int n_clips, int n, int K,
                             const float2* phi_dev, const float* lam_host, const int32_t* bkx_dev,
                             const int32_t* bky_dev, int nb, float* grad_out_dev, void* workspace_dev,
                             size_t workspace_bytes, cudaStream_t stream);

/* ---- SOCS imaging and its gradient over a kernel table ------------------ */

/* Workspace bytes of litho_socs_forward(). */
int litho_socs_forward_workspace(int n_clips, int n, int K, int h, int mask_complex, size_t* bytes);

/* The SOCS image of a batch of masks: expose/hopkins.py:SOCSKernels.raw /
 * .image (:205-223), the intensity of opc/ilt.py:socs_fields (:227-231):
 *   raw_c = sum_k lambda_k |ifft2(phi_k fft2(mask_c))|^2,
 *   image_out[c] = raw_c x s_c, peak_out[c] = max raw_c,
 * s_c = norm_scale (norm_mode 0; 1 gives the raw sum) or norm_scale / peak
 * (norm_mode 1, peak normalisation with dose norm_scale).
 * table_dev: K x (2h+1)^2 complex64, kernel k's band value at signed bins
 * (kx, ky), |kx|, |ky| <= h, stored at [k][(ky + h)(2h + 1) + kx + h];
 * weights_dev: K doubles lambda_k on the device; mask_dev: [n_clips][n][n]
 * float32 (mask_complex 0) or complex64. Workspace 256-byte aligned; the job
 * list is built inside it on the device. */
int litho_socs_forward(const void* table_dev, const double* weights_dev, int K, int h, const void* mask_dev,
                       int mask_complex, int n_clips, int n, int norm_mode, float norm_scale, float* image_out_dev,
                       float* peak_out_dev, void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);

/* Workspace bytes of litho_socs_backward(). */
int litho_socs_backward_workspace(int n_clips, int n, int K, int h, size_t* bytes);

/* The gradient of sum_x sens_scale sens_c(x) raw_c(x) with respect to the
 * real mask m_c, raw_c the SOCS image of litho_socs_forward():
 * opc/ilt.py:socs_gradient (:235-266) applied to the fields of socs_fields
 * (:227-231), 2 Re sum_k lambda_k ifft2(conj(phi_k) fft2(g E_k)) with
 * g = sens_scale sens. Band-limited: the mask's band (|k| <= h), the
 * sensitivity's band (|g| <= 2h), the coarse-grid adjoint, one synthesis.
 * grad_out_dev: [n_clips][n][n] float32. The backward of litho_socs_forward
 * for autograd. */
int litho_socs_backward(const void* table_dev, const double* weights_dev, int K, int h, const float* mask_dev,
                        int n_clips, int n, const float* sens_dev, float sens_scale, float* grad_out_dev,
                        void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);

/* ---- the band TCC: SOCS image and adjoint boxes without per-kernel FFTs -- */

/* Bytes of the band TCC of a kernel set with n_band band points inside the
 * box |kx|, |ky| <= h; LITHO_E_UNSUPPORTED when it would not stay resident in
 * L2 (more than 96 MiB) or h > 31 (then use litho_coarse_image and
 * litho_socs_adjoint). */
int litho_socs_tcc_bytes(int n_band, int h, size_t* bytes);

/* Build the band TCC T(f, f') = sum_k lambda_k conj phi_k(f) phi_k(f') of the
 * K kept kernels (expose/hopkins.py:SOCSKernels, :144-198, truncated at K)
 * in FP64 and store it as complex64 in two layouts, with the band's index
 * maps. phi_dev: K x n_band complex128 (unit eigenvectors on the band, in
 * band order), lam_dev: K doubles, band_kx/ky_dev: signed bins of the band
 * points. *status_dev is set non-zero if a band point lies outside the box. */
int litho_socs_tcc_build(const void* phi_dev, const double* lam_dev, int K, const int32_t* band_kx_dev,
                         const int32_t* band_ky_dev, int n_band, int h, void* tcc_dev, size_t tcc_bytes,
                         int* status_dev, cudaStream_t stream);

/* The SOCS image band box of each clip from its mask band box (the
 * forward of opc/ilt.py:socs_fields, :227-231, and expose/hopkins.py:
 * SOCSKernels.raw, :215-217, on the band): B(g) = sum_f Tc(f + g, f) M(f + g)
 * conj M(f), Tc = conj T, |g| <= 2h. mask_box_dev: n_clips x (2h+1)^2
 * (F(m) / N^2); image_box_out_dev: n_clips x (4h+1)^2, the box of
 * litho_coarse_image() (synthesise with litho_band_synthesis, h' = 2h). */
int litho_socs_tcc_image(const void* tcc_dev, int n_band, int h, const void* mask_box_dev, int n_clips,
                         void* image_box_out_dev, cudaStream_t stream);

/* The gradient band box of sum_x G(x) I(x) (opc/ilt.py:socs_gradient,
 * :235-266): H(f) = A(f) + conj A(-f), A(f) = sum_f' T(f, f') M(f')
 * Gs(f - f'), |f| <= h. sens_box_dev: n_clips x (4h+1)^2, F(G) / N^2 (the
 * sens box of litho_socs_adjoint); grad_box_out_dev: n_clips x (2h+1)^2. */
int litho_socs_tcc_adjoint(const void* tcc_dev, int n_band, int h, const void* mask_box_dev,
                           const void* sens_box_dev, int n_clips, void* grad_box_out_dev, cudaStream_t stream);

/* ---- SOCS (Hopkins) decomposition ---------------------------------------- */

/* Workspace bytes of litho_socs_build() for n_source points and n_band band
 * frequencies. */
int litho_socs_workspace(int n_source, int n_band, size_t* bytes);

/* Eigen-decomposition of one optical state's transmission cross-coefficient.
 * Replaces expose/hopkins.py:SOCSKernels.build (:103-198) up to the
 * selection of kernels, via the dual form: with A[s][b] = sqrt(w_s)
 * exp(i W) on the band (zero where inside_dev[s*n_band+b] == 0, the
 * reference's hypot aperture test made by the caller), G = conj(A) A^T
 * (S x S) is assembled on the tensor cores (gram_mode 0: tcgen05 TF32 with
 * hi/lo operand splitting, FP32 accumulate, FP64 reduction) or in FP64 on
 * CUDA cores (gram_mode 1, a check), diagonalised by FP64 Jacobi, and
 *   phi_out[j][b] = (A^T u_j)[b]       (complex128, unnormalised)
 *   lambda_out[j] = |A^T u_j|^2        (the eigenvalue, FP64 Rayleigh quotient)
 * for every j < n_source, unsorted. phi_j / sqrt(lambda_j) are the TCC's
 * unit eigenvectors (the reference's kernels on the band). gram_out (may be
 * NULL) receives G, row-major with an even leading dimension >= n_source. */
int litho_socs_build(const LithoPupil* pupil_dev, const double* fsx_dev, const double* fsy_dev,
                     const double* w_dev, int n_source, const int32_t* band_kx_dev,
                     const int32_t* band_ky_dev, int n_band, const uint8_t* inside_dev, int n,
                     double pixel_size, int gram_mode, double2* phi_out_dev,
                     double* lambda_out_dev, double2* gram_out_dev, void* workspace_dev,
                     size_t workspace_bytes, cudaStream_t stream);

/* Copy, after litho_socs_build(), the diagonalised Gram matrix, its
 * eigenvector matrix (columns) and the Jacobi eigenvalues out of the
 * workspace (each n x n / n with n = n_source rounded up to even; any output
 * may be NULL). For checking the eigensolver. */
int litho_socs_debug(int n_source, int n_band, const void* workspace_dev, double2* H_out,
                     double2* V_out, double* evals_out, cudaStream_t stream);

/* Synchronise and report litho_socs_build()'s device status (0 or
 * LITHO_E_TIMEOUT) and the Jacobi sweeps it took. */
int litho_socs_status(int n_source, int n_band, const void* workspace_dev, int* sweeps,
                      cudaStream_t stream);

/* ---- band-limited transforms and the ILT adjoint --------------------------- */

/* Coarse-grid image band of a plan whose mask band box mb_dev (per clip,
 * (2 bm + 1)^2, from litho_band_spectrum with scale 1/N^2) is already known:
 * the accumulation and reduction stages of litho_abbe() alone. bbox_out:
 * per output (4h+1)^2 complex, ready for litho_band_synthesis(h' = 2h). */
int litho_coarse_image(const LithoAbbePlan* plan, const void* plan_blob_dev, const void* table_dev,
                       const void* mb_dev, void* bbox_out_dev, void* workspace_dev,
                       size_t workspace_bytes, cudaStream_t stream);

/* Workspace bytes of litho_band_spectrum(). */
int litho_band_spectrum_workspace(int n_fields, int n, int bm, size_t* bytes);

/* box_out[f][ky + bm][kx + bm] = scale * sum_{x,y} in[f][y][x] exp(-2 pi i (kx x + ky y) / N)
 * for |kx|, |ky| <= bm: the part of numpy.fft.fft2 a band-limited consumer
 * needs (the reference calls fft2 at opc/ilt.py:227, :263 and
 * expose/hopkins.py:215). in: float32 (is_complex 0) or complex64. */
int litho_band_spectrum(const void* in_dev, int is_complex, int n_fields, int n, int bm, float scale,
                        void* box_out_dev, void* workspace_dev, size_t workspace_bytes,
                        cudaStream_t stream);

/* Workspace bytes of litho_band_synthesis(). */
int litho_band_synthesis_workspace(int n_fields, int n, size_t* bytes);

/* out[f][y][x] = sum_{|kx|,|ky| <= h} box[f][ky + h][kx + h] exp(2 pi i (kx x + ky y) / N):
 * float32 output for Hermitian boxes (complex_out 0), complex64 otherwise —
 * numpy.fft.ifft2 (times N^2) of a band-limited spectrum (opc/ilt.py:228). */
int litho_band_synthesis(const void* box_dev, int n_fields, int n, int h, int complex_out,
                         void* out_dev, void* workspace_dev, size_t workspace_bytes,
                         cudaStream_t stream);

/* Workspace bytes of litho_socs_adjoint(). */
int litho_socs_adjoint_workspace(int n_clips, int n_items, int h, size_t* bytes);

/* The band of the SOCS adjoint (opc/ilt.py:socs_gradient, :235-266):
 *   grad_box[c] = H, H(f) = A(f) + conj(A(-f)),
 *   A(f) = sum_k lambda_k conj(phi_k(f)) [ (phi_k M_c) (*) G_c ](f),  |f| <= h,
 * with M_c = mask_box[c] ((2h+1)^2, F(m)/N^2), G_c = sens_box[c]
 * ((4h+1)^2, F(dJ/dI)/N^2), phi_k = table slot k, lambda_k = job weight, the
 * jobs/items of a litho_abbe plan with one job per (clip, kernel) and
 * bm == h <= 15. When field_box_dev is given (per job, (2h+1)^2: the band
 * spectrum of each coherent field, F(E_k)/N^2) it replaces phi_k M_c and
 * mask_box_dev may be NULL. litho_band_synthesis(grad_box, h, real) gives d/dm. */
int litho_socs_adjoint(const LithoAbbePlan* plan, const void* plan_blob_dev, const void* table_dev,
                       const void* mask_box_dev, const void* field_box_dev, const void* sens_box_dev,
                       void* grad_box_out_dev, void* workspace_dev, size_t workspace_bytes,
                       cudaStream_t stream);

/* Relaxed resist objective (opc/ilt.py:_Objective, :313-336) on an image that
 * is already blurred: signed = sign (scale img - level); z = sigmoid(a
 * signed) (argument clipped to +-60); dfield = sign (2/npix) (z - t) a z (1-z).
 * Writes dfield (dJ/d field), optionally signed, and per-block partial sums
 * of (z - t)^2 (cost_part) and of pattern errors (perr_part): n_part blocks
 * per field, partial arrays [n_fields][n_part]. */
int litho_ilt_objective(const float* img_dev, const float* target_dev, int n_fields, int n, float scale,
                        float level, float sign, float steepness_a, float* dfield_dev,
                        float* signed_out_dev, double* cost_part_dev, unsigned int* perr_part_dev,
                        int n_part, cudaStream_t stream);

/* litho_ilt_objective() that also finishes the sums on the device: the last
 * block of each field sums its partials in block order into cost_out[field]
 * = sum (z - t)^2 / npix (the _Objective cost, opc/ilt.py:331) and
 * perr_out[field] = the pattern-error count. counters_dev: n_fields words,
 * zero before the first call; every call leaves them zero again. */
int litho_ilt_objective_totals(const float* img_dev, const float* target_dev, int n_fields, int n, float scale,
                               float level, float sign, float steepness_a, float* dfield_dev,
                               float* signed_out_dev, double* cost_part_dev, unsigned int* perr_part_dev,
                               int n_part, unsigned int* counters_dev, double* cost_out_dev,
                               long long* perr_out_dev, cudaStream_t stream);

/* The raw SOCS image synthesised from its band box (side 2 g0 + 1 per field,
 * as litho_band_synthesis) with the objective of litho_ilt_objective_totals()
 * applied to every pixel as it is made, so the image itself is never stored:
 * the image and objective halves of opc/ilt.py:_Objective (:313-336) on the
 * band-limited image. Writes dfield, cost_out, perr_out (counters_dev as
 * litho_ilt_objective_totals()); target_dev 16-byte aligned. The workspace
 * query returns LITHO_E_UNSUPPORTED where the row-pair synthesis with its
 * target stage does not apply (n a power of two in [256, 1024], g0 <= 31). */
int litho_ilt_image_objective_workspace(int n_fields, int n, int g0, size_t* bytes);
int litho_ilt_image_objective(const void* image_box_dev, int n_fields, int n, int g0, const float* target_dev,
                              float scale, float level, float sign, float steepness_a, float* dfield_dev,
                              unsigned int* counters_dev, double* cost_out_dev, long long* perr_out_dev,
                              void* workspace, size_t ws_bytes, cudaStream_t stream);

/* litho_ilt_image_objective() without dJ/dfield: the band box of
 * band_scale x dJ/dfield on |k| <= band_half, (2 band_half + 1)^2 complex
 * per field (the sensitivity the adjoint needs, opc/ilt.py:_Objective
 * :313-336 into socs_gradient :262-266), is formed from each row pair as
 * the synthesis makes it, so dJ/dfield is neither stored nor read back. Same
 * values as litho_ilt_image_objective() followed by litho_band_spectrum() on
 * its dJ/dfield (same arithmetic in the same order). The workspace's first
 * word is a status (LITHO_E_TIMEOUT if a bounded wait of the band transform
 * gave up). counters: zero on entry, left at zero. */
int litho_ilt_image_objective_band_workspace(int n_fields, int n, int g0, int band_half, size_t* bytes);
int litho_ilt_image_objective_band(const void* image_box_dev, int n_fields, int n, int g0, const float* target_dev,
                                   float scale, float level, float sign, float steepness_a, int band_half,
                                   float band_scale, void* band_box_out_dev, unsigned int* counters_dev,
                                   double* cost_out_dev, long long* perr_out_dev, void* workspace_dev,
                                   size_t workspace_bytes, cudaStream_t stream);

/* TV (periodic neighbours) and discreteness penalties (opc/ilt.py:339-357):
 * adds their gradients to grad_dev and their costs to cost_part_dev. */
int litho_ilt_penalties(const float* mask_dev, int n_fields, int n, float w_tv, float w_disc,
                        float* grad_dev, double* cost_part_dev, int n_part, cudaStream_t stream);

/* mask = sigmoid(clip(beta field, +-60)) (opc/ilt.py:_mask_of, :368-378). */
int litho_ilt_mask(const float* field_dev, long long count, float beta, float* mask_dev,
                   cudaStream_t stream);

/* q = grad_m beta m (1 - m), the sigmoid's slope of opc/ilt.py:_grad_theta (:381-389). */
int litho_ilt_theta_grad(const float* grad_m_dev, const float* mask_dev, long long count, float beta,
                         float* q_dev, cudaStream_t stream);

/* dJ/dtheta, Adam and the next mask in one pass (opc/ilt.py:381-389,
 * 587-591, 368-378, without smoothing): m = sigmoid(beta theta),
 * q = g beta m (1 - m), Adam step `it` on theta (m1, m2 in place), mask =
 * sigmoid(beta_next theta). count a multiple of 4, 16-byte aligned arrays. */
int litho_ilt_update(const float* g_dev, long long count, float beta, float beta_next, float step, float b1,
                     float b2, float eps, int it, float* theta_dev, float* m1_dev, float* m2_dev, float* mask_dev,
                     cudaStream_t stream);
/* The step schedule of litho_ilt_update_sched(), in device memory, so that a
 * step recorded once (a CUDA graph) can be replayed: each call first sets
 * beta = beta_next, it = it + 1, beta_next = beta * growth, then runs
 * litho_ilt_update() with those values (run_ilt's beta annealing and Adam
 * counter, opc/ilt.py:582-596). Start it with beta = beta_next = the current
 * sharpness and it = the number of steps already taken. */
typedef struct LithoIltSched {
    double beta, beta_next, growth;
    int32_t it;
    float c1, c2;         /* Adam bias corrections 1 - b1^it, 1 - b2^it     */
    int32_t pad;          /* the update's block counter: 0 before the first */
                          /* call, left 0 by every call                     */
} LithoIltSched;          /* 40 bytes */

int litho_ilt_update_sched(const float* g_dev, long long count, LithoIltSched* sched_dev, float step, float b1,
                           float b2, float eps, float* theta_dev, float* m1_dev, float* m2_dev, float* mask_dev,
                           cudaStream_t stream);
/* One whole ILT iteration of n_clips clips in one call: the loop body of
 * opc/ilt.py:run_ilt (:576-596 -- dJ/dtheta, Adam, the beta anneal, mask_of)
 * and the objective with its adjoint (opc/ilt.py:_Objective :292-360 over
 * socs_fields / socs_gradient :208-266), for kernel bands whose band TCC
 * fits (litho_socs_tcc_bytes: h <= 15). The gradient is kept as its band
 * box grad_box_dev ((2h+1)^2 complex per clip, read and replaced); the step
 * synthesises it, runs litho_ilt_update_sched (sched_dev advanced, theta,
 * m1, m2 and mask_out_dev written), forms the mask's band box, the image
 * band box (litho_socs_tcc_image), the objective with the band box of dJ/dI
 * (litho_ilt_image_objective_band: cost_out_dev, perr_out_dev) and the new
 * gradient band box (litho_socs_tcc_adjoint). No blur, smoothing or
 * penalties (the fast form). steepness_a = steepness / |level|. Stream-
 * ordered, no host synchronisation, nothing allocated; the workspace is the
 * caller's (litho_ilt_step_workspace). litho_ilt_step_status synchronises
 * and returns the first non-zero status word of the last step (a bounded
 * wait that gave up), else 0. */
int litho_ilt_step_workspace(int n_clips, int n, int h, size_t* bytes);
int litho_ilt_step(const void* tcc_dev, int n_band, int h, int n_clips, int n, const float* target_dev,
                   float* theta_dev, float* m1_dev, float* m2_dev, LithoIltSched* sched_dev, void* grad_box_dev,
                   float* mask_out_dev, float scale, float level, float sign, float steepness_a, float step,
                   float b1, float b2, float eps, double* cost_out_dev, long long* perr_out_dev,
                   void* workspace_dev, size_t workspace_bytes, cudaStream_t stream);
int litho_ilt_step_status(int n_clips, int n, int h, const void* workspace_dev, cudaStream_t stream);

/* One Adam step at iteration it >= 1 (opc/ilt.py:582-591), in place. */
int litho_ilt_adam(const float* g_dev, long long count, float step, float b1, float b2, float eps,
                   int it, float* theta_dev, float* m1_dev, float* m2_dev, cudaStream_t stream);

/* scipy.ndimage.gaussian_filter (mode 'reflect') of n_fields N x N images:
 * the 1-D weights[2 radius + 1] along rows, then along columns
 * (opc/ilt.py:_blur, :274-289). tmp_dev: scratch of the input's size. */
int litho_gaussian_blur(const float* in_dev, float* out_dev, float* tmp_dev, int n_fields, int n,
                        const float* weights_dev, int radius, cudaStream_t stream);

/* ---- process-window helpers ----
 * The dose axis of a dose-focus sweep (analysis/process_window.py:285-290):
 * out[f][d] = raw[f] * normalisation_scale(mode, peak[f], clear[f], dose[d])
 * (expose/aerial_image.py:217-241); mode 0 none, 1 peak, 2 clear. raw:
 * [n_planes][npix] raw Abbe sums (litho_abbe with scale 1); out:
 * [n_planes][n_doses][npix]; peak/clear: device [n_planes]; doses: device. */
int litho_dose_stack(const float* raw_dev, const float* peak_dev, const float* clear_dev, int mode, int n_planes,
                     long long npix, const float* doses_dev, int n_doses, float* out_dev, cudaStream_t stream);
/* x = min(max(x, lo), hi) in place: the clip after PEB diffusion
 * (bake/peb.py:65-66). */
int litho_clamp(float* x_dev, long long count, float lo, float hi, cudaStream_t stream);
/* Depth interpolation of an exposure volume (develop/resist3d.py:176-183,
 * np.interp per pixel along depth): out[v][p] = a[p] + w[v] (b[p] - a[p])
 * with a = planes[k[2v]], b = planes[k[2v + 1]] for v < n_out. planes:
 * [n_planes][npix] optical planes; k_dev: device int32 [n_out][2] plane
 * indices (8-byte aligned); w_dev: device float [n_out]; out: [n_out][npix].
 * A plane index outside [0, n_planes) leaves that voxel plane unwritten and
 * sets LITHO_E_BAND in *status_dev (zero it before the call). */
int litho_depth_interp(const float* planes_dev, int n_planes, long long npix, const int* k_dev, const float* w_dev,
                       int n_out, float* out_dev, int* status_dev, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* LITHO_B200_H */
