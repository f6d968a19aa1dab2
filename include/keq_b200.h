/*
 * keq_b200.h -- C ABI of the B200 (sm_100a) backend for kineticEQ's BGK1D1V
 * implicit (Picard + Anderson) and HOLO time steps.
 *
 * Conventions
 *  - All array pointers are CUDA device pointers unless a comment says host.
 *  - f is (nx, nv) row-major FP64, v contiguous; W arrays are (nx).
 *  - The library never allocates device memory.  Every entry point that needs
 *    scratch space takes a caller-provided workspace whose size comes from the
 *    matching *_workspace_size query (the reference's gtsv_ws_bytes /
 *    potrf_lwork pattern).
 *  - Every call is asynchronous on the given stream and returns a keq_status
 *    for host-side validation; device-side failures (non-finite values, wait
 *    timeouts) are reported through keq_step_stats.status after the stream is
 *    synchronised.
 *  - No C++ types, no exceptions cross this boundary.
 */
#ifndef KEQ_B200_H
#define KEQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* keq_stream_t; /* == cudaStream_t */

typedef enum keq_status {
    KEQ_OK = 0,
    KEQ_ERR_INVALID = 1,      /* bad sizes, null pointers, bad parameters */
    KEQ_ERR_WORKSPACE = 2,    /* workspace too small or misaligned */
    KEQ_ERR_CUDA = 3,         /* a CUDA runtime call failed (see keq_last_cuda_error) */
    KEQ_ERR_TIMEOUT = 4,      /* a device-side wait gave up (bounded spin) */
    KEQ_ERR_NONFINITE = 5,    /* NaN/Inf detected in the new distribution */
    KEQ_ERR_NOCONV = 6,       /* iteration cap reached without convergence (informational) */
    KEQ_ERR_UNSUPPORTED = 7,  /* device or configuration not supported */
    KEQ_ERR_CAPACITY = 8      /* request exceeds a fixed capacity of the entry point */
} keq_status;

/* ---- version / diagnostics ------------------------------------------------ */
int32_t keq_abi_version(void);
const char* keq_status_string(int32_t status);
/* Last CUDA runtime error string seen by this thread (empty if none). */
const char* keq_last_cuda_error(void);

/* ---- problem description --------------------------------------------------
 * Grid of one BGK1D1V instance: core/states/state_1d.py:30-58
 * (dx = Lx/(nx-1), dv = 2 vmax/(nv-1), v = linspace(-vmax, vmax, nv)). */
typedef struct keq_grid {
    int32_t nx;
    int32_t nv;
    double dx;
    double dv;
    const double* v; /* device, nv entries, ascending */
    /* Optional host-side facts about v that save plan creation a device read
     * and a stream synchronisation: kp = number of velocities <= 0 and
     * v_max = max |v|.  kp < 0 means unknown (v is then read back). */
    int32_t kp;
    double v_max;
} keq_grid;

/* implicit.Params: params/BGK1D1V/implicit.py:5-37 (CNN warm start excluded).
 * conv_type: 0 = "f" (distribution), 1 = "w" (moments).
 * fixed_iters > 0 replays exactly that many Picard iterations per step (the
 * residual is still computed and reported).
 * tile_rows: scan positions per tile of the step kernel, 8/16/24/32 (0 = 32);
 * a tuning knob of this backend (no reference counterpart): results depend
 * on it at rounding level only. */
typedef struct keq_implicit_params {
    int32_t picard_iter;
    double picard_tol;
    double abs_tol;
    int32_t conv_type;
    int32_t aa_enable;
    int32_t aa_m;
    double aa_beta;
    int32_t aa_stride;
    int32_t aa_start_iter;
    double aa_reg;
    double aa_alpha_max;
    int32_t fixed_iters;
    int32_t tile_rows;
    /* precision: 0 = FP64 (the reference's method), 1 = mixed-precision form:
     * FP32 sweeps (Maxwellian, reciprocal and recurrence in FP32 on FP32
     * copies of f^n and of the iterate; moments, Anderson and residuals in
     * FP64) until a sweep meets mixed_tol (0 = 1e-6), then FP64 sweeps until
     * picard_tol as in the FP64 form.  keq_step_stats.lo_iters reports the
     * FP32 sweeps.  A backend knob without reference counterpart. */
    int32_t precision;
    double mixed_tol;
} keq_implicit_params;

/* holo.Params: params/BGK1D1V/holo.py:5-13 (+ the hidden SVdown flag read at
 * core/schemes/BGK1D1V/bgk1d_holo_cuda_kernel.py:443). */
typedef struct keq_holo_params {
    int32_t ho_iter;
    double ho_tol;
    double ho_abs_tol;
    int32_t lo_iter;
    double lo_tol;
    double lo_abs_tol;
    int32_t con_terms_do;
    int32_t flux_consistency_do;
    int32_t sv_down;
    int32_t fixed_ho_iters;
    int32_t fixed_lo_iters;
} keq_holo_params;

/* Per-instance result of the last step (device memory; read after sync).
 * Implicit fills iters/residual/std_residual/aa_applied (benchlog keys
 * picard_iter, picard_residual, std_picard_residual); HOLO fills
 * iters (= ho_iter), residual/std_residual (ho), lo_* and max_YI. */
typedef struct keq_step_stats {
    int32_t status;     /* keq_status of the step (0 = OK) */
    int32_t iters;      /* Picard (or HO) iterations of the last step */
    int32_t aa_applied; /* Anderson combinations applied in the last step */
    int32_t lo_iters;   /* HOLO: LO iterations of the last HO iteration */
    double residual;    /* picard_residual / ho_residual */
    double std_residual;/* std_picard_residual / std_ho_residual */
    double lo_residual;
    double std_lo_residual;
    double max_YI;
    int64_t total_iters;/* iterations summed over all steps since plan creation */
    int64_t total_steps;
} keq_step_stats;

/* One instance of a batched solve. */
typedef struct keq_instance {
    keq_grid grid;
    double dt;
    double tau_tilde;
    const double* f_in; /* device (nx, nv): f^n, read only */
    double* f_out;      /* device (nx, nv): receives f^{n+1}; may not alias f_in */
    keq_step_stats* stats; /* device, one record */
    void* workspace;    /* device, keq_*_instance_workspace_size bytes, 256-B aligned */
} keq_instance;

/* ==== implicit Picard step (replaces core/schemes/BGK1D1V/
 *      bgk1d_implicit_cuda_kernel.py:28-311 step() and its kernels
 *      K1 moments, K2 assembly, K3 cuSPARSE gtsv, K4 Anderson) ============== */

/* Bytes of per-instance workspace for one instance. */
keq_status keq_implicit_instance_workspace_size(const keq_grid* grid,
                                                const keq_implicit_params* params,
                                                size_t* bytes);

/* A batch plan binds a list of instances (host array, copied) to one shared
 * device workspace.  The plan is a host object; it holds no device memory of
 * its own. */
typedef struct keq_plan keq_plan;

/* Bytes of shared (batch-level) device workspace for n instances. */
keq_status keq_implicit_plan_workspace_size(const keq_instance* insts, int32_t n,
                                            const keq_implicit_params* params,
                                            int32_t per_instance_params, size_t* bytes);
/* params: one record applied to every instance, or an array of n records when
 * per_instance_params != 0. */
keq_status keq_implicit_plan_create(const keq_instance* insts, int32_t n,
                                    const keq_implicit_params* params,
                                    int32_t per_instance_params, void* plan_workspace,
                                    size_t plan_workspace_bytes, keq_stream_t stream,
                                    keq_plan** plan_out);
/* Replace the f_in/f_out pointers of the instances (host arrays of n device
 * pointers) without rebuilding the plan; used to ping-pong state buffers. */
keq_status keq_plan_set_buffers(keq_plan* plan, const double* const* f_in,
                                double* const* f_out, keq_stream_t stream);
/* Advance every instance of the plan by n_steps time steps.  Step k of the
 * call (k = 0..n_steps-1) reads f_in and writes f_out when (parity + k) is
 * even, and the reverse when it is odd, so the state ping-pongs between the
 * two buffers without copies; the caller tracks where the newest state is. */
keq_status keq_plan_step(keq_plan* plan, int32_t n_steps, int32_t parity, keq_stream_t stream);
/* Attach (iters > 0) or detach (iters = 0) a phase trace: a device buffer of
 * iters * 4 uint64 that the caller initialises with {UINT64_MAX, 0,
 * UINT64_MAX, 0} per row; each step then records, per Picard iteration, the
 * earliest start and latest end (%globaltimer ns) of pass 1 and pass 2 over
 * all warps.  No reference counterpart (profiling aid). */
keq_status keq_plan_set_trace(keq_plan* plan, unsigned long long* trace, int32_t iters,
                              keq_stream_t stream);
/* Implicit plans: attach a device int32 mask of n entries (or NULL to
 * detach).  While mask[b] == 0, instance b is left untouched by every step
 * (no state, stats or workspace write), so a serving loop can retire slots
 * without rebuilding the plan; the mask is read on the device at every
 * launch and may be changed by stream-ordered device writes.  Synchronises
 * the stream.  No reference counterpart. */
keq_status keq_plan_set_enable_mask(keq_plan* plan, const int32_t* mask, keq_stream_t stream);
/* Device-side error bits of the plan (1 << keq_status) accumulated over every
 * launch since plan creation or the last keq_plan_reset, synchronising the
 * stream; 0 when every device-side wait completed.  A launch whose wait gave
 * up also leaves KEQ_ERR_TIMEOUT in every instance's keq_step_stats.status. */
keq_status keq_plan_error(keq_plan* plan, keq_stream_t stream, int32_t* err_bits);
/* Clear the plan's accumulated error bits (asynchronous on the stream).  The
 * per-launch barrier state is cleared by keq_plan_step itself before every
 * launch, so a plan stays usable after a launch that timed out.  No reference
 * counterpart (device-side waits do not exist in the reference). */
keq_status keq_plan_reset(keq_plan* plan, keq_stream_t stream);
/* Polls a device-side wait makes before it gives up with KEQ_ERR_TIMEOUT
 * (default 2^25, i.e. seconds).  0 makes every wait that is not already
 * satisfied give up at once; tests use it to exercise the timeout path
 * without a hang.  Synchronises the stream.  No reference counterpart. */
keq_status keq_plan_set_spin_limit(keq_plan* plan, unsigned long long limit, keq_stream_t stream);
void keq_plan_destroy(keq_plan* plan);

/* ==== HOLO step (replaces core/schemes/BGK1D1V/bgk1d_holo_cuda_kernel.py:
 *      416-595 step() with theta = 1/2: HO moments, consistency terms,
 *      explicit term, LO Picard with the 3x3 block-tridiagonal solve of
 *      cuda_kernel/BGK1D1V/lo_blocktridiag, and the distribution solve) =====
 * A HOLO plan is a keq_plan too: it is stepped, reset, queried and destroyed
 * with the keq_plan_* functions above.  Each step fills the instance's
 * keq_step_stats with iters = ho_iter, residual = ho_residual, std_residual =
 * std_ho_residual, lo_iters, lo_residual, std_lo_residual and max_YI (the
 * reference's benchlog).  Supported sizes: nx - 2 <= 16384 interior cells
 * (512 LO chunks of 32 rows; the interface system is solved in one CTA's
 * shared memory); larger grids return KEQ_ERR_UNSUPPORTED. */
keq_status keq_holo_instance_workspace_size(const keq_grid* grid, const keq_holo_params* params,
                                            size_t* bytes);
keq_status keq_holo_plan_workspace_size(const keq_instance* insts, int32_t n,
                                        const keq_holo_params* params, int32_t per_instance_params,
                                        size_t* bytes);
keq_status keq_holo_plan_create(const keq_instance* insts, int32_t n, const keq_holo_params* params,
                                int32_t per_instance_params, void* plan_workspace,
                                size_t plan_workspace_bytes, keq_stream_t stream,
                                keq_plan** plan_out);

/* Single-instance convenience wrapper: workspace = instance workspace followed
 * by plan workspace, sized by keq_implicit_workspace_size.  It builds and
 * destroys a plan per call, which synchronises the stream (v is read back
 * to find the sign change) and restarts the stats totals; steppers that run
 * many steps use a plan. */
keq_status keq_implicit_workspace_size(const keq_grid* grid, const keq_implicit_params* params,
                                       size_t* bytes);
keq_status keq_implicit_step(const keq_grid* grid, double dt, double tau_tilde,
                             const keq_implicit_params* params, const double* f_in,
                             double* f_out, keq_step_stats* stats, void* workspace,
                             size_t workspace_bytes, keq_stream_t stream);

/* ==== kernel-level drop-ins =============================================== */

/* K1: cuda_kernel/BGK1D1V/implicit_fused/implicit_binding.cpp:38-71
 * (moments_n_nu_T): n = max(sum f dv, 1e-300), nu = sum f v dv,
 * T = sum f v^2 dv / n - (nu/n)^2 (T <= 0 -> 1e-300). */
keq_status keq_moments_n_nu_T(const double* f, const double* v, int32_t nx, int32_t nv,
                              double dv, double* n, double* nu, double* T, keq_stream_t stream);

/* K2: implicit_binding.cpp:73-142 (build_system_from_moments); all system
 * arrays (nv, nx-2) contiguous per velocity. */
keq_status keq_build_system_from_moments(const double* B0, const double* v, int32_t nx,
                                         int32_t nv, double dt, double dx, double tau_tilde,
                                         double inv_sqrt_2pi, const double* n, const double* nu,
                                         const double* T, const double* f_bc_l,
                                         const double* f_bc_r, double* dl, double* dd,
                                         double* du, double* B, keq_stream_t stream);

/* K3: cuda_kernel/BGK1D1V/gtsv/gtsv_binding.cpp:48-117 (gtsv_ws_bytes,
 * gtsv_strided_inplace): batch independent tridiagonal systems of length n,
 * rows of dl/d/du/B contiguous (stride n); solution overwrites B; d is not
 * modified. */
keq_status keq_gtsv_workspace_size(int32_t n, int32_t batch, size_t* bytes);
keq_status keq_gtsv_strided_inplace(const double* dl, const double* d, const double* du,
                                    double* B, int32_t n, int32_t batch, void* workspace,
                                    size_t workspace_bytes, keq_stream_t stream);

/* The same solve as keq_gtsv_strided_inplace, for callers that cannot
 * allocate device memory and so cannot pass a workspace (a binding that only
 * forwards the operation's own tensors, or a host that must not call
 * cudaMalloc).  It allocates nothing: its scratch is a fixed array inside the
 * library, KEQ_GTSV_NOALLOC_MAX_ELEMS doubles (16 MiB) on every GPU that
 * loads the library, held until the process exits.  n * batch above that
 * limit returns KEQ_ERR_CAPACITY.  The first call on a device looks the
 * array's device address up (with that device current) and caches it; make
 * that first call before any stream capture.  All calls share the one array,
 * so two calls that may overlap on the GPU (different streams, no ordering)
 * race on it: order them on one stream.  It keeps the last call's contents,
 * which is harmless here because the kernel writes every scratch element it
 * reads.  This entry point has no counterpart in the reference. */
#define KEQ_GTSV_NOALLOC_MAX_ELEMS (1 << 21)
keq_status keq_gtsv_strided_inplace_noalloc(const double* dl, const double* d, const double* du,
                                            double* B, int32_t n, int32_t batch,
                                            keq_stream_t stream);


/* K5: cuda_kernel/BGK1D1V/lo_blocktridiag/block_tridiag_binding.cpp:25-108
 * (block_tridiag_solve): batch 3x3-block tridiagonal systems of n block rows.
 * A, B, C: (batch, n, 3, 3) row-major blocks; D, X: (batch, n, 3).  A[0] and
 * C[n-1] are ignored.  A block with |det| < 1e-30 contributes a zero inverse. */
keq_status keq_block_tridiag_workspace_size(int32_t n, int32_t batch, size_t* bytes);
keq_status keq_block_tridiag_solve(const double* A, const double* B, const double* C,
                                   const double* D, double* X, int32_t n, int32_t batch,
                                   void* workspace, size_t workspace_bytes,
                                   keq_stream_t stream);

/* Maxwellian of per-row moments: core/schemes/BGK1D1V/bgk1d_utils/general/
 * bgk1d_maxwellian.py:7-33 (maxwellian; used by set_initial_condition,
 * bgk1d_set_initial_condition.py:9-44): f[i, j] = n_i / sqrt(2 pi T_i)
 * exp(-(v_j - u_i)^2 / (2 T_i)); n, u, T are (nx), f is (nx, nv). */
keq_status keq_maxwellian(const double* n, const double* u, const double* T, const double* v,
                          int32_t nx, int32_t nv, double* f, keq_stream_t stream);

/* Raw row moments without clamps, (nx, 3) row-major: sum f dv, sum f v dv,
 * sum f v^2/2 dv (the sums of core/schemes/BGK1D1V/bgk1d_utils/general/
 * bgk1d_compute_moments.py:7-17); the conservation totals of a state are
 * their sums over x times dx. */
keq_status keq_row_moments(const double* f, const double* v, int32_t nx, int32_t nv, double dv,
                           double* out, keq_stream_t stream);

/* Numerical self-test of the device math used by the fused kernels (no
 * reference counterpart): kind 0 evaluates the branch-free e^x for x <= 0,
 * kind 1 the Newton reciprocal 1/x for x >= 1, element-wise on device
 * arrays x -> y. */
keq_status keq_math_selftest(int32_t kind, const double* x, double* y, int32_t n,
                             keq_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* KEQ_B200_H */
