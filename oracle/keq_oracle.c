/*
 * keq_oracle.c -- CPU restatement of kineticEQ's BGK1D1V implicit (Picard +
 * Anderson) and HOLO time steps, in plain C (FP64, OpenMP over independent
 * rows / velocities).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path in kineticeq_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.  The product path never
 * links or calls it.
 *
 * Every function names the reference code it restates (paths relative to the
 * kineticEQ project root, src/kineticEQ/...).  Arithmetic follows the
 * reference's expression order, so the sequential C++ CPU kernels (moments,
 * assembly, Thomas) are reproduced bit for bit; the torch-level code
 * (convergence test, Anderson least squares, HOLO) is reproduced up to
 * floating-point summation order.
 *
 * Build without -ffast-math and with -ffp-contract=off: the reference's CPU
 * extensions are plain -O3 for x86-64 (no FMA contraction).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KEQO_TINY 1.0e-300

static inline double clamp_pos(double x) { return x > KEQO_TINY ? x : KEQO_TINY; }
static inline double dmax(double a, double b) { return a > b ? a : b; }
/* torch.clamp(x, min=lo): NaN stays NaN. */
static inline double clamp_min_t(double x, double lo) { return (isnan(x) || x >= lo) ? x : lo; }
/* torch.maximum: NaN propagates. */
static inline double max_t(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a > b ? a : b;
}

/* Running torch.max over a tensor: NaN anywhere gives NaN. */
typedef struct { double v; int nan; } tmax_t;
static inline void tmax_init(tmax_t* m) { m->v = -INFINITY; m->nan = 0; }
static inline void tmax_add(tmax_t* m, double x) {
    if (isnan(x)) m->nan = 1; else if (x > m->v) m->v = x;
}
static inline double tmax_get(const tmax_t* m) { return m->nan ? NAN : m->v; }

static void* xalloc(size_t bytes) {
    void* p = calloc(1, bytes ? bytes : 8);
    return p;
}

/* ===========================================================================
 * Implicit path building blocks
 * ======================================================================== */

/* moments_n_nu_T: cpu_kernel/BGK1D1V/implicit_fused_cpu/implicit_binding.cpp:30-90.
 * Sequential sum over v per row; n clamped at 1e-300, T <= 0 -> 1e-300. */
void keqo_moments_n_nu_T(const double* f, const double* v, int nx, int nv, double dv, double* n,
                         double* nu, double* T) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        const double* row = f + (size_t)i * nv;
        double p0 = 0.0, p1 = 0.0, p2 = 0.0;
        for (int j = 0; j < nv; ++j) {
            const double fij = row[j];
            const double vj = v[j];
            p0 += fij;
            p1 += fij * vj;
            p2 += fij * vj * vj;
        }
        const double n_raw = p0 * dv;
        const double nu_raw = p1 * dv;
        const double s2_raw = p2 * dv;
        const double n_val = clamp_pos(n_raw);
        const double u_val = nu_raw / n_val;
        double T_val = s2_raw / n_val - u_val * u_val;
        if (!(T_val > 0.0)) T_val = KEQO_TINY;
        n[i] = n_val;
        nu[i] = nu_raw;
        T[i] = T_val;
    }
}

/* maxwell_1v: implicit_binding.cpp:22-26. */
static inline double maxwell_1v(double n, double u, double Tgas, double vj, double inv_sqrt_2pi) {
    const double Tg = clamp_pos(Tgas);
    const double diff = vj - u;
    return n * inv_sqrt_2pi / sqrt(Tg) * exp(-0.5 * diff * diff / Tg);
}

/* build_system_from_moments: implicit_binding.cpp:92-187.
 * dl/dd/du/B/B0 are (nv, nx-2), contiguous per velocity. */
void keqo_build_system(const double* B0, const double* v, int nx, int nv, double dt, double dx,
                       double tau_tilde, double inv_sqrt_2pi, const double* n, const double* nu,
                       const double* T, const double* f_bc_l, const double* f_bc_r, double* dl,
                       double* dd, double* du, double* B) {
    const int n_inner = nx - 2;
    if (n_inner <= 0) return;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nv; ++j) {
        const double vj = v[j];
        const double alpha = vj > 0.0 ? (dt / dx) * vj : 0.0;
        const double beta = vj < 0.0 ? (dt / dx) * (-vj) : 0.0;
        const size_t off = (size_t)j * n_inner;
        for (int k = 0; k < n_inner; ++k) {
            const int i = k + 1;
            const double n_i = clamp_pos(n[i]);
            const double T_i = clamp_pos(T[i]);
            const double u_i = nu[i] / n_i;
            const double inv_tau = (n_i * sqrt(T_i)) / tau_tilde;
            const double fM = maxwell_1v(n_i, u_i, T_i, vj, inv_sqrt_2pi);
            dd[off + k] = 1.0 + alpha + beta + dt * inv_tau;
            dl[off + k] = k == 0 ? 0.0 : -alpha;
            du[off + k] = k == n_inner - 1 ? 0.0 : -beta;
            double rhs = B0[off + k] + dt * inv_tau * fM;
            if (k == 0) rhs += alpha * f_bc_l[j];
            if (k == n_inner - 1) rhs += beta * f_bc_r[j];
            B[off + k] = rhs;
        }
    }
}

/* Thomas without pivoting: cpu_kernel/BGK1D1V/gtsv_cpu/gtsv_binding.cpp:51-97,
 * pivots floored to +-1e-300 (:32-37).  In place on d and B. */
static inline double safe_pivot(double x) {
    if (fabs(x) >= 1.0e-300) return x;
    return x < 0.0 ? -1.0e-300 : 1.0e-300;
}

void keqo_gtsv(const double* dl, double* d, const double* du, double* B, int batch, int n) {
    if (batch <= 0 || n <= 0) return;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < batch; ++b) {
        const double* dlr = dl + (size_t)b * n;
        double* dr = d + (size_t)b * n;
        const double* dur = du + (size_t)b * n;
        double* Br = B + (size_t)b * n;
        for (int i = 1; i < n; ++i) {
            const double pivot = safe_pivot(dr[i - 1]);
            const double w = dlr[i] / pivot;
            dr[i] -= w * dur[i - 1];
            Br[i] -= w * Br[i - 1];
        }
        Br[n - 1] /= safe_pivot(dr[n - 1]);
        for (int i = n - 1; i-- > 0;) Br[i] = (Br[i] - dur[i] * Br[i + 1]) / safe_pivot(dr[i]);
    }
}

/* check_convergence: core/schemes/BGK1D1V/bgk1d_utils/implicit/bgk1d_conv_util.py:9-60.
 * Returns max(df/(abs_tol+tol*ref)); *rel = max(df/clamp(ref, min=abs_tol)). */
static double conv_max(const double* a_new, const double* a_old, size_t cnt, double abs_tol,
                       double tol, double* rel) {
    tmax_t r1, r2;
    tmax_init(&r1);
    tmax_init(&r2);
    for (size_t k = 0; k < cnt; ++k) {
        const double df = fabs(a_new[k] - a_old[k]);
        const double ref = max_t(fabs(a_new[k]), fabs(a_old[k]));
        tmax_add(&r1, df / (abs_tol + tol * ref));
        tmax_add(&r2, df / clamp_min_t(ref, abs_tol));
    }
    *rel = tmax_get(&r2);
    return tmax_get(&r1);
}

/* ---------------------------------------------------------------------------
 * Small dense symmetric solve used by Anderson acceleration: restates
 * torch.linalg.cholesky + cholesky_solve with the fall-back to a minimum-norm
 * least-squares solve (bgk1d_aa_cpu.py:93-97; torch.linalg.lstsq), here a
 * Jacobi eigen-decomposition pseudo-inverse.
 * ------------------------------------------------------------------------ */
#define KEQO_AA_MAXC 16

static int chol_solve(int m, const double* A, const double* b, double* x) {
    double L[KEQO_AA_MAXC * KEQO_AA_MAXC];
    double y[KEQO_AA_MAXC];
    memset(L, 0, sizeof(L));
    for (int j = 0; j < m; ++j) {
        double s = A[j * m + j];
        for (int k = 0; k < j; ++k) s -= L[j * m + k] * L[j * m + k];
        if (!(s > 0.0)) return -1;
        const double ljj = sqrt(s);
        L[j * m + j] = ljj;
        for (int i = j + 1; i < m; ++i) {
            double t = A[i * m + j];
            for (int k = 0; k < j; ++k) t -= L[i * m + k] * L[j * m + k];
            L[i * m + j] = t / ljj;
        }
    }
    for (int i = 0; i < m; ++i) {
        double t = b[i];
        for (int k = 0; k < i; ++k) t -= L[i * m + k] * y[k];
        y[i] = t / L[i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {
        double t = y[i];
        for (int k = i + 1; k < m; ++k) t -= L[k * m + i] * x[k];
        x[i] = t / L[i * m + i];
    }
    return 0;
}

static void pinv_solve(int m, const double* A, const double* b, double* x) {
    double a[KEQO_AA_MAXC * KEQO_AA_MAXC], V[KEQO_AA_MAXC * KEQO_AA_MAXC];
    memcpy(a, A, sizeof(double) * (size_t)m * m);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) V[i * m + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) off += a[p * m + q] * a[p * m + q];
        if (!(off > 1e-300)) break;
        for (int p = 0; p < m; ++p) {
            for (int q = p + 1; q < m; ++q) {
                const double apq = a[p * m + q];
                if (apq == 0.0) continue;
                const double theta = (a[q * m + q] - a[p * m + p]) / (2.0 * apq);
                const double t =
                    (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < m; ++k) {
                    const double akp = a[k * m + p], akq = a[k * m + q];
                    a[k * m + p] = c * akp - s * akq;
                    a[k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = a[p * m + k], aqk = a[q * m + k];
                    a[p * m + k] = c * apk - s * aqk;
                    a[q * m + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double vkp = V[k * m + p], vkq = V[k * m + q];
                    V[k * m + p] = c * vkp - s * vkq;
                    V[k * m + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    double lmax = 0.0;
    for (int i = 0; i < m; ++i) lmax = dmax(lmax, fabs(a[i * m + i]));
    const double cut = lmax * (double)m * 2.220446049250313e-16;
    for (int i = 0; i < m; ++i) x[i] = 0.0;
    for (int k = 0; k < m; ++k) {
        const double lam = a[k * m + k];
        if (!(fabs(lam) > cut)) continue;
        double proj = 0.0;
        for (int i = 0; i < m; ++i) proj += V[i * m + k] * b[i];
        proj /= lam;
        for (int i = 0; i < m; ++i) x[i] += proj * V[i * m + k];
    }
}

/* Plain W update: bgk1d_implicit_cpu_kernel.py:249-251. */
static void plain_update(int nx, double* n, double* nu, double* T, const double* n_new,
                         const double* nu_new, const double* T_new, double n_floor,
                         double T_floor) {
    for (int i = 0; i < nx; ++i) {
        n[i] = clamp_min_t(n_new[i], n_floor);
        nu[i] = nu_new[i];
        T[i] = clamp_min_t(T_new[i], T_floor);
    }
}

/* step_inplace: core/schemes/BGK1D1V/bgk1d_utils/implicit/bgk1d_aa_cpu.py:7-129.
 * G and R are (d, aa_cols) row-major rings, d = 3*(nx-2).  Returns 1 if the
 * Anderson combination was applied. */
static int aa_step_inplace(int nx, double* n, double* nu, double* T, const double* n_new,
                           const double* nu_new, const double* T_new, double* G, double* R,
                           int aa_cols, int* hist_len, int* head, int apply, double beta,
                           double reg, double alpha_max, double n_floor, double T_floor,
                           double u_max, double* wk, double* wnew, double* wtmp) {
    const int n_inner = nx - 2 > 0 ? nx - 2 : 0;
    const int d = 3 * n_inner;
    const int cols = aa_cols > 1 ? aa_cols : 1;
    const int hist_in = *hist_len > 0 ? *hist_len : 0;
    const int head_in = (*head > 0 ? *head : 0) % cols;
    const int hist_out = hist_in + 1 < aa_cols ? hist_in + 1 : aa_cols;
    const int head_out = (head_in + 1) % cols;
    *hist_len = hist_out;
    *head = head_out;
    if (n_inner <= 0 || d <= 0) {
        plain_update(nx, n, nu, T, n_new, nu_new, T_new, n_floor, T_floor);
        return 0;
    }
    for (int k = 0; k < n_inner; ++k) {
        wk[k] = n[k + 1];
        wk[n_inner + k] = nu[k + 1];
        wk[2 * n_inner + k] = T[k + 1];
        wnew[k] = n_new[k + 1];
        wnew[n_inner + k] = nu_new[k + 1];
        wnew[2 * n_inner + k] = T_new[k + 1];
    }
    for (int k = 0; k < d; ++k) {
        wtmp[k] = wnew[k] - wk[k];
        G[(size_t)k * aa_cols + head_in] = wnew[k];
        R[(size_t)k * aa_cols + head_in] = wtmp[k];
    }
    if (!(apply && hist_out >= 2)) {
        plain_update(nx, n, nu, T, n_new, nu_new, T_new, n_floor, T_floor);
        return 0;
    }
    const int m = hist_out;
    int cidx[KEQO_AA_MAXC];
    for (int j = 0; j < m; ++j) cidx[j] = (((head_out - m + j) % aa_cols) + aa_cols) % aa_cols;
    double A[KEQO_AA_MAXC * KEQO_AA_MAXC];
    for (int p = 0; p < m; ++p) {
        for (int q = 0; q < m; ++q) {
            double acc = 0.0;
            for (int k = 0; k < d; ++k)
                acc += R[(size_t)k * aa_cols + cidx[p]] * R[(size_t)k * aa_cols + cidx[q]];
            A[p * m + q] = acc;
        }
    }
    for (int p = 0; p < m; ++p) A[p * m + p] += reg;
    double rhs[KEQO_AA_MAXC], alpha[KEQO_AA_MAXC];
    for (int p = 0; p < m; ++p) rhs[p] = 1.0;
    if (chol_solve(m, A, rhs, alpha) != 0) pinv_solve(m, A, rhs, alpha);
    double asum = 0.0;
    for (int p = 0; p < m; ++p) asum += alpha[p];
    if (fabs(asum) < 1.0e-30) asum = 1.0e-30;
    for (int p = 0; p < m; ++p) {
        double a = alpha[p] / asum;
        if (alpha_max > 0.0) {
            if (a < -alpha_max) a = -alpha_max;
            if (a > alpha_max) a = alpha_max;
        }
        alpha[p] = a;
    }
    for (int k = 0; k < d; ++k) {
        double acc = 0.0;
        for (int p = 0; p < m; ++p) acc += G[(size_t)k * aa_cols + cidx[p]] * alpha[p];
        wtmp[k] = acc * beta + (1.0 - beta) * wnew[k];
    }
    n[0] = clamp_min_t(n_new[0], n_floor);
    nu[0] = nu_new[0];
    T[0] = clamp_min_t(T_new[0], T_floor);
    n[nx - 1] = clamp_min_t(n_new[nx - 1], n_floor);
    nu[nx - 1] = nu_new[nx - 1];
    T[nx - 1] = clamp_min_t(T_new[nx - 1], T_floor);
    for (int k = 0; k < n_inner; ++k) {
        const double nm = clamp_min_t(wtmp[k], n_floor);
        const double Tm = clamp_min_t(wtmp[2 * n_inner + k], T_floor);
        double um = wtmp[n_inner + k] / nm;
        if (!isfinite(um)) um = 0.0;
        if (um < -u_max) um = -u_max;
        if (um > u_max) um = u_max;
        n[k + 1] = nm;
        nu[k + 1] = nm * um;
        T[k + 1] = Tm;
    }
    return 1;
}

/* ---------------------------------------------------------------------------
 * One implicit time step: core/schemes/BGK1D1V/bgk1d_implicit_cpu_kernel.py:29-267
 * (no CNN warm start, fixed_maxwellian boundary rows).  f is (nx, nv) in/out.
 * fixed_iters > 0 replays a given Picard count (the convergence test is
 * evaluated but ignored).
 * ------------------------------------------------------------------------ */
typedef struct {
    int picard_iter;
    double picard_tol;
    double abs_tol;
    int conv_type; /* 0 = "f", 1 = "w" */
    int aa_enable;
    int aa_m;
    double aa_beta;
    int aa_stride;
    int aa_start_iter;
    double aa_reg;
    double aa_alpha_max;
    int fixed_iters;
} keqo_implicit_params;

typedef struct {
    int picard_iter;
    double picard_residual;
    double std_picard_residual;
    int aa_applied;
} keqo_implicit_log;

int keqo_implicit_step(int nx, int nv, const double* v, double dx, double dv, double dt,
                       double tau_tilde, const keqo_implicit_params* p, double* f,
                       keqo_implicit_log* log) {
    if (nx < 3 || nv < 1) return -1;
    const double n_floor = 1e-12, T_floor = 1e-12;
    const double inv_sqrt_2pi = 1.0 / sqrt(2.0 * M_PI);
    const int n_inner = nx - 2;
    const size_t N = (size_t)nx * nv, Ni = (size_t)nv * n_inner;
    const int aa_m = p->aa_m > 0 ? p->aa_m : 0;
    double aa_beta = p->aa_beta;
    aa_beta = aa_beta < 0.0 ? 0.0 : (aa_beta > 1.0 ? 1.0 : aa_beta);
    const int aa_stride = p->aa_stride > 1 ? p->aa_stride : 1;
    const int aa_start = p->aa_start_iter > 1 ? p->aa_start_iter : 1;
    const double aa_reg = p->aa_reg > 1e-14 ? p->aa_reg : 1e-14;
    const double aa_amax = p->aa_alpha_max > 0.0 ? p->aa_alpha_max : 0.0;
    const int aa_cols = (p->aa_enable && aa_m >= 1) ? aa_m + 1 : 1;
    const int aa_on = p->aa_enable && aa_m >= 1 && aa_cols >= 2 && aa_cols <= KEQO_AA_MAXC;
    double vmaxabs = 0.0;
    for (int j = 0; j < nv; ++j) vmaxabs = dmax(vmaxabs, fabs(v[j]));
    const double u_max = 0.95 * vmaxabs;

    double* fbl = xalloc(sizeof(double) * nv);
    double* fbr = xalloc(sizeof(double) * nv);
    double* B0 = xalloc(sizeof(double) * Ni);
    double* dl = xalloc(sizeof(double) * Ni);
    double* dd = xalloc(sizeof(double) * Ni);
    double* du = xalloc(sizeof(double) * Ni);
    double* B = xalloc(sizeof(double) * Ni);
    double* fz = xalloc(sizeof(double) * N);
    double* fn = xalloc(sizeof(double) * N);
    double* W = xalloc(sizeof(double) * 6 * nx);
    double* G = xalloc(sizeof(double) * 3 * n_inner * aa_cols);
    double* R = xalloc(sizeof(double) * 3 * n_inner * aa_cols);
    double* wbuf = xalloc(sizeof(double) * 9 * n_inner);
    double *n = W, *nu = W + nx, *T = W + 2 * nx;
    double *n_new = W + 3 * nx, *nu_new = W + 4 * nx, *T_new = W + 5 * nx;

    memcpy(fbl, f, sizeof(double) * nv);
    memcpy(fbr, f + (size_t)(nx - 1) * nv, sizeof(double) * nv);
    for (int j = 0; j < nv; ++j)
        for (int k = 0; k < n_inner; ++k) B0[(size_t)j * n_inner + k] = f[(size_t)(k + 1) * nv + j];
    memcpy(fz, f, sizeof(double) * N);
    keqo_moments_n_nu_T(fz, v, nx, nv, dv, n, nu, T);

    int hist_len = 0, head = 0, aa_applied = 0, z = 0;
    double residual = INFINITY, rel = INFINITY;
    double* latest = fz;
    for (z = 0; z < p->picard_iter; ++z) {
        keqo_build_system(B0, v, nx, nv, dt, dx, tau_tilde, inv_sqrt_2pi, n, nu, T, fbl, fbr, dl,
                          dd, du, B);
        keqo_gtsv(dl, dd, du, B, nv, n_inner);
        for (int k = 0; k < n_inner; ++k)
            for (int j = 0; j < nv; ++j) fn[(size_t)(k + 1) * nv + j] = B[(size_t)j * n_inner + k];
        memcpy(fn, fbl, sizeof(double) * nv);
        memcpy(fn + (size_t)(nx - 1) * nv, fbr, sizeof(double) * nv);
        keqo_moments_n_nu_T(fn, v, nx, nv, dv, n_new, nu_new, T_new);
        if (p->conv_type == 1) {
            double r1, r2, r3, q1, q2, q3;
            r1 = conv_max(n_new, n, nx, p->abs_tol, p->picard_tol, &q1);
            r2 = conv_max(nu_new, nu, nx, p->abs_tol, p->picard_tol, &q2);
            r3 = conv_max(T_new, T, nx, p->abs_tol, p->picard_tol, &q3);
            residual = max_t(r1, max_t(r2, r3));
            rel = max_t(q1, max_t(q2, q3));
        } else {
            residual = conv_max(fn, fz, N, p->abs_tol, p->picard_tol, &rel);
        }
        latest = fn;
        const int done = p->fixed_iters > 0 ? (z + 1 >= p->fixed_iters) : (residual <= 1.0);
        if (done) break;
        if (z + 1 < p->picard_iter) {
            if (aa_on) {
                const int should = (z + 1) >= aa_start && ((z + 1 - aa_start) % aa_stride == 0);
                aa_applied += aa_step_inplace(nx, n, nu, T, n_new, nu_new, T_new, G, R, aa_cols,
                                              &hist_len, &head, should, aa_beta, aa_reg, aa_amax,
                                              n_floor, T_floor, u_max, wbuf, wbuf + 3 * n_inner,
                                              wbuf + 6 * n_inner);
            } else {
                plain_update(nx, n, nu, T, n_new, nu_new, T_new, n_floor, T_floor);
            }
        }
        double* t = fz;
        fz = fn;
        fn = t;
    }
    /* state.f_tmp <- latest; apply_bc restores rows 0 and nx-1 from the old f
     * (identical values for fixed_maxwellian). */
    memcpy(f + nv, latest + nv, sizeof(double) * (size_t)nv * n_inner);
    if (log) {
        log->picard_iter = (z < p->picard_iter) ? z + 1 : p->picard_iter;
        log->picard_residual = rel;
        log->std_picard_residual = residual;
        log->aa_applied = aa_applied;
    }
    free(fbl); free(fbr); free(B0); free(dl); free(dd); free(du); free(B);
    free(fz);
    free(fn);
    free(W); free(G); free(R); free(wbuf);
    return 0;
}

/* ===========================================================================
 * HOLO path: core/schemes/BGK1D1V/bgk1d_holo_cuda_kernel.py:31-595 (torch
 * ops, device-agnostic), run here on the host.  The distribution solve uses
 * the CPU Thomas above (cuSPARSE in the reference's CUDA run); the 3x3
 * block-tridiagonal LO solve is a block Thomas sweep with the reference's
 * singular-block convention (|det| < 1e-30 -> zero inverse,
 * cuda_kernel/BGK1D1V/lo_blocktridiag/block_tridiag_kernel.cu:32-68, 248-250).
 * ======================================================================== */

/* calculate_moments: core/schemes/BGK1D1V/bgk1d_utils/general/bgk1d_compute_moments.py:7-17
 * (no clamps). */
static void holo_moments(const double* f, const double* v, int nx, int nv, double dv, double* n,
                         double* u, double* T) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        const double* row = f + (size_t)i * nv;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int j = 0; j < nv; ++j) {
            s0 += row[j];
            s1 += row[j] * v[j];
            s2 += row[j] * (v[j] * v[j]);
        }
        const double nn = s0 * dv;
        const double uu = (s1 * dv) / nn;
        n[i] = nn;
        u[i] = uu;
        T[i] = (s2 * dv) / nn - uu * uu;
    }
}

/* maxwellian: bgk1d_utils/general/bgk1d_maxwellian.py:7-33 for one cell. */
static inline double holo_maxwell(double n, double u, double T, double vj, double inv_sqrt_2pi) {
    const double coeff = (n * inv_sqrt_2pi) / sqrt(T);
    const double invT = 0.5 / T;
    const double diff = vj - u;
    return exp(diff * diff * (-invT)) * coeff;
}

/* _HO_calculate_moments_face: bgk1d_holo_cuda_kernel.py:31-77 (upwind face state). */
static void holo_face_moments(const double* f, const double* v, int nx, int nv, double dv,
                              int SVdown, double* S1, double* S2, double* S3) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx - 1; ++i) {
        double a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (int j = 0; j < nv; ++j) {
            const double fu = v[j] > 0.0 ? f[(size_t)i * nv + j] : f[(size_t)(i + 1) * nv + j];
            double w1, w2, w3;
            if (SVdown) {
                w1 = 1.0;
                w2 = v[j];
                w3 = 0.5 * v[j] * v[j];
            } else {
                w1 = v[j];
                w2 = v[j] * v[j];
                w3 = 0.5 * v[j] * v[j] * v[j];
            }
            a1 += fu * w1;
            a2 += fu * w2;
            a3 += fu * w3;
        }
        S1[i] = a1 * dv;
        S2[i] = a2 * dv;
        S3[i] = a3 * dv;
    }
}

/* _HO_calculate_fluxes_Q: bgk1d_holo_cuda_kernel.py:81-99. */
static void holo_Q(const double* f, const double* v, int nx, int nv, double dv, double* tmp3,
                   double* Q) {
    double *n = tmp3, *u = tmp3 + nx, *T = tmp3 + 2 * nx;
    holo_moments(f, v, nx, nv, dv, n, u, T);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        double acc = 0.0;
        for (int j = 0; j < nv; ++j) {
            const double d = v[j] - u[i];
            acc += d * d * d * f[(size_t)i * nv + j];
        }
        Q[i] = acc * (0.5 * dv);
    }
}

/* 3x3 helpers (row-major). */
static inline void m3_mul(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
static inline void m3_vec(const double* A, const double* x, double* y) {
    for (int i = 0; i < 3; ++i) y[i] = A[3 * i] * x[0] + A[3 * i + 1] * x[1] + A[3 * i + 2] * x[2];
}
static inline int m3_inv(const double* M, double* Mi) {
    const double a00 = M[0], a01 = M[1], a02 = M[2];
    const double a10 = M[3], a11 = M[4], a12 = M[5];
    const double a20 = M[6], a21 = M[7], a22 = M[8];
    const double c00 = (a11 * a22 - a12 * a21), c01 = -(a10 * a22 - a12 * a20),
                 c02 = (a10 * a21 - a11 * a20);
    const double c10 = -(a01 * a22 - a02 * a21), c11 = (a00 * a22 - a02 * a20),
                 c12 = -(a00 * a21 - a01 * a20);
    const double c20 = (a01 * a12 - a02 * a11), c21 = -(a00 * a12 - a02 * a10),
                 c22 = (a00 * a11 - a01 * a10);
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (!(fabs(det) >= 1e-30)) {
        for (int k = 0; k < 9; ++k) Mi[k] = 0.0;
        return 0;
    }
    const double id = 1.0 / det;
    Mi[0] = c00 * id; Mi[1] = c10 * id; Mi[2] = c20 * id;
    Mi[3] = c01 * id; Mi[4] = c11 * id; Mi[5] = c21 * id;
    Mi[6] = c02 * id; Mi[7] = c12 * id; Mi[8] = c22 * id;
    return 1;
}

/* Block Thomas for A_i X_{i-1} + B_i X_i + C_i X_{i+1} = D_i, i = 0..n-1
 * (A_0 and C_{n-1} ignored).  Blocks (n,3,3) row-major, D/X (n,3). */
void keqo_block_tridiag_solve(const double* A, const double* Bm, const double* C, const double* D,
                              double* X, int n) {
    if (n <= 0) return;
    double* Cp = xalloc(sizeof(double) * 9 * (size_t)n);
    double* Dp = xalloc(sizeof(double) * 3 * (size_t)n);
    double Mi[9], T9[9], t3[3], y3[3];
    for (int i = 0; i < n; ++i) {
        double M[9], rhs[3];
        if (i == 0) {
            memcpy(M, Bm, sizeof(M));
            memcpy(rhs, D, sizeof(rhs));
        } else {
            m3_mul(A + 9 * (size_t)i, Cp + 9 * (size_t)(i - 1), T9);
            for (int k = 0; k < 9; ++k) M[k] = Bm[9 * (size_t)i + k] - T9[k];
            m3_vec(A + 9 * (size_t)i, Dp + 3 * (size_t)(i - 1), t3);
            for (int k = 0; k < 3; ++k) rhs[k] = D[3 * (size_t)i + k] - t3[k];
        }
        m3_inv(M, Mi);
        if (i < n - 1) m3_mul(Mi, C + 9 * (size_t)i, Cp + 9 * (size_t)i);
        m3_vec(Mi, rhs, Dp + 3 * (size_t)i);
    }
    for (int k = 0; k < 3; ++k) X[3 * (size_t)(n - 1) + k] = Dp[3 * (size_t)(n - 1) + k];
    for (int i = n - 2; i >= 0; --i) {
        m3_vec(Cp + 9 * (size_t)i, X + 3 * (size_t)(i + 1), y3);
        for (int k = 0; k < 3; ++k) X[3 * (size_t)i + k] = Dp[3 * (size_t)i + k] - y3[k];
    }
    free(Cp);
    free(Dp);
}

typedef struct {
    int ho_iter;
    double ho_tol;
    double ho_abs_tol;
    int lo_iter;
    double lo_tol;
    double lo_abs_tol;
    int con_terms_do;
    int flux_consistency_do;
    int sv_down;
    int fixed_ho_iters; /* >0: replay this many HO iterations */
    int fixed_lo_iters; /* >0: replay this many LO iterations per HO iteration */
} keqo_holo_params;

typedef struct {
    int ho_iter;
    double ho_residual;
    double std_ho_residual;
    int lo_iter;
    double lo_residual;
    double std_lo_residual;
    double max_YI;
} keqo_holo_log;

/* One HOLO step: bgk1d_holo_cuda_kernel.py:416-595, theta = 1/2. */
int keqo_holo_step(int nx, int nv, const double* v, double dx, double dv, double dt,
                   double tau_tilde, const keqo_holo_params* p, double* f, keqo_holo_log* log) {
    if (nx < 3 || nv < 1) return -1;
    const double theta = 0.5;
    const double inv_sqrt_2pi = 1.0 / sqrt(2.0 * M_PI);
    const int n_inner = nx - 2;
    const size_t N = (size_t)nx * nv;
    double* fz = xalloc(sizeof(double) * N);
    double* fn = xalloc(sizeof(double) * N);
    double* E = xalloc(sizeof(double) * N);
    double* sol = xalloc(sizeof(double) * (size_t)nv * n_inner);
    double* dl = xalloc(sizeof(double) * (size_t)nv * n_inner);
    double* dd = xalloc(sizeof(double) * (size_t)nv * n_inner);
    double* du = xalloc(sizeof(double) * (size_t)nv * n_inner);
    double* vec = xalloc(sizeof(double) * 40 * (size_t)nx);
    double* blk = xalloc(sizeof(double) * 40 * (size_t)nx);
    double *nHO = vec, *uHO = vec + nx, *THO = vec + 2 * nx;
    double *S1 = vec + 3 * nx, *S2 = vec + 4 * nx, *S3 = vec + 5 * nx;
    double *Q = vec + 6 * nx, *tmp3 = vec + 7 * nx; /* 3*nx */
    double *nN = vec + 10 * nx, *uN = vec + 11 * nx, *TN = vec + 12 * nx;
    double *Y = vec + 13 * nx;          /* (nx,3) */
    double *WHO = vec + 16 * nx;        /* (nx,3) */
    double *Wm = vec + 19 * nx;         /* (nx,3) */
    double *Wf = vec + 22 * nx;         /* (nx,3) */
    double *FHO = vec + 25 * nx;        /* (nx-1,3) */
    double *nlo = vec + 28 * nx, *ulo = vec + 29 * nx, *Tlo = vec + 30 * nx, *taulo = vec + 31 * nx;
    double *AAb = blk, *BBb = blk + 9 * (size_t)nx, *CCb = blk + 18 * (size_t)nx;
    double *DD = blk + 27 * (size_t)nx, *XX = blk + 30 * (size_t)nx;
    double *fbl = blk + 33 * (size_t)nx, *fbr = fbl + nv; /* needs 2*nv <= 7*nx */
    double* fbbuf = NULL;
    if (2 * (size_t)nv > 7 * (size_t)nx) {
        fbbuf = xalloc(sizeof(double) * 2 * nv);
        fbl = fbbuf;
        fbr = fbbuf + nv;
    }

    memcpy(fz, f, sizeof(double) * N);
    memcpy(fn, f, sizeof(double) * N);
    holo_moments(f, v, nx, nv, dv, nHO, uHO, THO);
    holo_face_moments(f, v, nx, nv, dv, p->sv_down, S1, S2, S3);

    /* _compute_explicit_term: :103-131. */
    {
        const double a = (1.0 - theta) * dt;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i) {
            const double tau = tau_tilde / (nHO[i] * sqrt(THO[i]));
            for (int j = 0; j < nv; ++j) {
                const double fij = f[(size_t)i * nv + j];
                const double fM = holo_maxwell(nHO[i], uHO[i], THO[i], v[j], inv_sqrt_2pi);
                const double vc = -v[j] / dx;
                double st = 0.0;
                if (v[j] > 0.0) {
                    if (i >= 1) st = (fij - f[(size_t)(i - 1) * nv + j]) * vc;
                } else {
                    if (i <= nx - 2) st = (f[(size_t)(i + 1) * nv + j] - fij) * vc;
                }
                const double col = (fM - fij) / tau;
                E[(size_t)i * nv + j] = fij + a * (st + col);
            }
        }
    }
    memcpy(fbl, f, sizeof(double) * nv);
    memcpy(fbr, f + (size_t)(nx - 1) * nv, sizeof(double) * nv);

    double ho_res_val = INFINITY, ho_std = INFINITY, lo_res_val = INFINITY, lo_std = INFINITY;
    double max_YI = 0.0;
    int lo_done = 0, z = 0;
    double* latest = fz;
    for (z = 0; z < p->ho_iter; ++z) {
        holo_Q(fz, v, nx, nv, dv, tmp3, Q);
        memset(Y, 0, sizeof(double) * 3 * nx);
        if (p->con_terms_do) {
            /* _compute_Y_I_terms: :135-227 (face moments of the current iterate
             * overwrite the step-start ones, as in the reference). */
            holo_face_moments(fz, v, nx, nv, dv, p->sv_down, S1, S2, S3);
            holo_moments(fz, v, nx, nv, dv, nN, uN, TN);
            if (p->flux_consistency_do && nx > 2) {
                for (int i = 1; i < nx - 1; ++i) {
                    double g[2][3];
                    for (int s = 0; s < 2; ++s) {
                        const int fi = i - 1 + s; /* face index */
                        const int a0 = fi, a1 = fi + 1;
                        const double P0 = nN[a0] * TN[a0], P1 = nN[a1] * TN[a1];
                        const double nu0 = nN[a0] * uN[a0], nu1 = nN[a1] * uN[a1];
                        const double U0 = 0.5 * nN[a0] * (uN[a0] * uN[a0] + TN[a0]);
                        const double U1 = 0.5 * nN[a1] * (uN[a1] * uN[a1] + TN[a1]);
                        const double mf0 = nu0 * nu0 / (nN[a0] + 1e-30) + P0;
                        const double mf1 = nu1 * nu1 / (nN[a1] + 1e-30) + P1;
                        const double ef0 = (U0 + P0) * uN[a0] + Q[a0];
                        const double ef1 = (U1 + P1) * uN[a1] + Q[a1];
                        g[s][0] = -S1[fi] + 0.5 * (nu0 + nu1);
                        g[s][1] = -S2[fi] + 0.5 * (mf0 + mf1);
                        g[s][2] = -S3[fi] + 0.5 * (ef0 + ef1);
                    }
                    for (int c = 0; c < 3; ++c) Y[3 * i + c] += dt * ((g[1][c] - g[0][c]) / dx);
                }
            }
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nx; ++i) {
                const double tn = tau_tilde / (nN[i] * sqrt(TN[i]));
                const double to = tau_tilde / (nHO[i] * sqrt(THO[i]));
                double m0 = 0.0, m1 = 0.0, m2 = 0.0;
                for (int j = 0; j < nv; ++j) {
                    const double Mn = holo_maxwell(nN[i], uN[i], TN[i], v[j], inv_sqrt_2pi);
                    const double Mo = holo_maxwell(nHO[i], uHO[i], THO[i], v[j], inv_sqrt_2pi);
                    const double Cn = (Mn - fz[(size_t)i * nv + j]) / tn;
                    const double Co = (Mo - f[(size_t)i * nv + j]) / to;
                    const double Cm = theta * Cn + (1.0 - theta) * Co;
                    m0 += Cm;
                    m1 += Cm * v[j];
                    m2 += Cm * (0.5 * v[j] * v[j]);
                }
                Y[3 * i + 0] += dt * (m0 * dv);
                Y[3 * i + 1] += dt * (m1 * dv);
                Y[3 * i + 2] += dt * (m2 * dv);
            }
        }
        max_YI = 0.0;
        {
            tmax_t mm;
            tmax_init(&mm);
            for (int k = 0; k < 3 * nx; ++k) tmax_add(&mm, fabs(Y[k]));
            max_YI = tmax_get(&mm);
        }

        /* _LO_calculate_moments_picard: :234-409. */
        for (int i = 0; i < nx; ++i) {
            WHO[3 * i + 0] = nHO[i];
            WHO[3 * i + 1] = nHO[i] * uHO[i];
            WHO[3 * i + 2] = 0.5 * nHO[i] * (uHO[i] * uHO[i] + THO[i]);
        }
        memcpy(Wm, WHO, sizeof(double) * 3 * nx);
        for (int fi = 0; fi < nx - 1; ++fi) {
            const double Qh = 0.5 * (Q[fi] + Q[fi + 1]);
            FHO[3 * fi + 0] = S1[fi];
            FHO[3 * fi + 1] = S2[fi];
            FHO[3 * fi + 2] = S3[fi] + 2.0 * Qh;
        }
        const double c4 = dt / (4.0 * dx), c2 = dt / (2.0 * dx);
        lo_done = 0;
        for (int m = 0; m < p->lo_iter; ++m) {
            lo_done = m + 1;
            /* u*, P* at cells, then half values at faces. */
            for (int i = 0; i < nx; ++i) {
                const double den = Wm[3 * i] + 1e-30;
                const double us = Wm[3 * i + 1] / den;
                double Ts = 2.0 * (Wm[3 * i + 2] / den - 0.5 * us * us);
                Ts = clamp_min_t(Ts, 1e-30);
                tmp3[i] = us;
                tmp3[nx + i] = Wm[3 * i] * Ts;
            }
            for (int k = 0; k < n_inner; ++k) {
                /* faces L = k, R = k+1 for interior cell i = k+1 */
                double Aint[2][9], bint[2][3];
                for (int s = 0; s < 2; ++s) {
                    const int fi = k + s;
                    const double uh = 0.5 * (tmp3[fi] + tmp3[fi + 1]);
                    const double Ph = 0.5 * (tmp3[nx + fi] + tmp3[nx + fi + 1]);
                    for (int q = 0; q < 9; ++q) Aint[s][q] = 0.0;
                    Aint[s][1] = 1.0;
                    Aint[s][3] = uh * uh;
                    Aint[s][8] = uh;
                    bint[s][0] = 0.0;
                    bint[s][1] = Ph;
                    bint[s][2] = uh * Ph;
                }
                for (int q = 0; q < 9; ++q) {
                    AAb[9 * k + q] = (k >= 1) ? Aint[0][q] * (-c4) : 0.0;
                    CCb[9 * k + q] = (k <= n_inner - 2) ? Aint[1][q] * c4 : 0.0;
                    BBb[9 * k + q] = (Aint[1][q] - Aint[0][q]) * c4 + ((q % 4 == 0) ? 1.0 : 0.0);
                }
                for (int c = 0; c < 3; ++c) {
                    const double Fd = FHO[3 * (k + 1) + c] - FHO[3 * k + c];
                    const double bd = bint[1][c] - bint[0][c];
                    double dval = WHO[3 * (k + 1) + c];
                    dval = dval + (-c2) * Fd;
                    dval = dval + (-c2) * bd;
                    dval = dval + Y[3 * (k + 1) + c];
                    DD[3 * k + c] = dval;
                }
            }
            keqo_block_tridiag_solve(AAb, BBb, CCb, DD, XX, n_inner);
            memcpy(Wf, WHO, sizeof(double) * 3 * nx);
            memcpy(Wf + 3, XX, sizeof(double) * 3 * n_inner);
            tmax_t md, ms;
            tmax_init(&md);
            tmax_init(&ms);
            for (int q = 0; q < 3 * nx; ++q) {
                const double df = fabs(Wf[q] - Wm[q]);
                const double ref = max_t(fabs(Wf[q]), fabs(Wm[q]));
                tmax_add(&md, df);
                tmax_add(&ms, df / (p->lo_abs_tol + p->lo_tol * ref));
            }
            lo_res_val = tmax_get(&md);
            lo_std = tmax_get(&ms);
            memcpy(Wm, Wf, sizeof(double) * 3 * nx);
            const int lo_stop = p->fixed_lo_iters > 0 ? (m + 1 >= p->fixed_lo_iters) : (lo_std < 1.0);
            if (lo_stop) break;
        }
        for (int i = 0; i < nx; ++i) {
            const double den = Wm[3 * i] + 1e-30;
            const double ul = Wm[3 * i + 1] / den;
            double Tl = 2.0 * (Wm[3 * i + 2] / den - 0.5 * ul * ul);
            Tl = clamp_min_t(Tl, 1e-30);
            nlo[i] = Wm[3 * i];
            ulo[i] = ul;
            Tlo[i] = Tl;
            taulo[i] = tau_tilde / (Wm[3 * i] * sqrt(Tl));
        }

        /* Distribution solve: :526-555. */
        const double h = dt / (2.0 * dx);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < nv; ++j) {
            const double al = h * (v[j] > 0.0 ? v[j] : 0.0);
            const double be = h * (-v[j] > 0.0 ? -v[j] : 0.0);
            const size_t off = (size_t)j * n_inner;
            for (int k = 0; k < n_inner; ++k) {
                const int i = k + 1;
                dl[off + k] = k == 0 ? 0.0 : -al;
                du[off + k] = k == n_inner - 1 ? 0.0 : -be;
                dd[off + k] = (1.0 + al + be) + (theta * dt) / taulo[i];
                const double fM = holo_maxwell(nlo[i], ulo[i], Tlo[i], v[j], inv_sqrt_2pi);
                double b = E[(size_t)i * nv + j] + (theta * dt) * (fM / taulo[i]);
                if (k == 0) b += al * fbl[j];
                if (k == n_inner - 1) b += be * fbr[j];
                sol[off + k] = b;
            }
        }
        keqo_gtsv(dl, dd, du, sol, nv, n_inner);
        memcpy(fn, fz, sizeof(double) * N);
        for (int k = 0; k < n_inner; ++k)
            for (int j = 0; j < nv; ++j) fn[(size_t)(k + 1) * nv + j] = sol[(size_t)j * n_inner + k];
        tmax_t mres, mdf, mref;
        tmax_init(&mres);
        tmax_init(&mdf);
        tmax_init(&mref);
        for (size_t q = 0; q < N; ++q) {
            const double df = fabs(fn[q] - fz[q]);
            const double ref = max_t(fabs(fn[q]), fabs(fz[q]));
            tmax_add(&mres, df / (p->ho_abs_tol + p->ho_tol * ref));
            tmax_add(&mdf, df);
            tmax_add(&mref, ref);
        }
        const double ho_res = tmax_get(&mres);
        ho_res_val = tmax_get(&mdf) / tmax_get(&mref);
        ho_std = ho_res;
        latest = fn;
        const int ho_stop = p->fixed_ho_iters > 0 ? (z + 1 >= p->fixed_ho_iters) : (ho_res <= 1.0);
        if (ho_stop) break;
        double* t = fz;
        fz = fn;
        fn = t;
    }
    memcpy(f + nv, latest + nv, sizeof(double) * (size_t)nv * n_inner);
    if (log) {
        log->ho_iter = (z < p->ho_iter) ? z + 1 : p->ho_iter;
        log->ho_residual = ho_res_val;
        log->std_ho_residual = ho_std;
        log->lo_iter = lo_done;
        log->lo_residual = lo_res_val;
        log->std_lo_residual = lo_std;
        log->max_YI = max_YI;
    }
    free(fz);
    free(fn);
    free(E); free(sol); free(dl); free(dd); free(du); free(vec); free(blk);
    if (fbbuf) free(fbbuf);
    return 0;
}

/* set_initial_condition + maxwellian: bgk1d_set_initial_condition.py:9-44,
 * bgk1d_maxwellian.py:7-33.  Regions are (a, b, n, u, T) quintuples; the last
 * region is closed on the right. */
void keqo_initial_condition(const double* x, int nx, const double* v, int nv, const double* regions,
                            int n_regions, double* f) {
    const double inv_sqrt_2pi = 1.0 / sqrt(2.0 * M_PI);
    for (int i = 0; i < nx; ++i) {
        double n = 1.0, u = 0.0, T = 1.0;
        for (int r = 0; r < n_regions; ++r) {
            const double* q = regions + 5 * r;
            const int in = (r == n_regions - 1) ? (x[i] >= q[0] && x[i] <= q[1])
                                                : (x[i] >= q[0] && x[i] < q[1]);
            if (in) {
                n = q[2];
                u = q[3];
                T = q[4];
            }
        }
        for (int j = 0; j < nv; ++j) f[(size_t)i * nv + j] = holo_maxwell(n, u, T, v[j], inv_sqrt_2pi);
    }
}
