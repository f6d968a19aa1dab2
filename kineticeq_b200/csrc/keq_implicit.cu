// keq_implicit.cu -- BGK1D1V implicit (Picard + Anderson) time step for a
// batch of independent instances, as ONE persistent cooperative kernel per
// time step on sm_100a.
//
// Replaces core/schemes/BGK1D1V/bgk1d_implicit_cuda_kernel.py:28-311 (step)
// and the kernels it launches per Picard iteration:
//   K1 moments_n_nu_T     cuda_kernel/BGK1D1V/implicit_fused/implicit_kernels.cu:28-81
//   K2 build_system       implicit_kernels.cu:84-134
//   K3 cuSPARSE gtsv2     cuda_kernel/BGK1D1V/gtsv/gtsv_batch.cu:12-126
//   transposes / residual bgk1d_implicit_cuda_kernel.py:82,215-237, bgk1d_conv_util.py:9-60
//   K4 Anderson           cuda_kernel/BGK1D1V/implicit_AA/implicit_AA_kernel.cu:403-694
//                         (numerics of the CPU twin bgk1d_utils/implicit/bgk1d_aa_cpu.py:7-129)
//
// Structure of one launch (one time step for every instance of the plan):
//   P0  zero per-step device state, copy the fixed boundary rows to f_out
//   P1  velocity moments of f^n (tile partial sums)          -- grid barrier
//   P2  row reduction -> W^(0)=(n,nu,T), per-row coefficients -- grid barrier
//   loop over Picard iterations m while any instance is active:
//     S(m)  fused tile pass: Maxwellian + upwind implicit assembly + solve of
//           the first-order recurrence along x (decoupled look-back between
//           x-chunks), residual vs f^(m), partial moments of f^(m+1)
//                                                              -- grid barrier
//     R(m)  row reduction of the partial moments -> W_new, "w" residual,
//           Anderson history / Gram matrix (last block solves the m x m
//           system), W^(m+1) and per-row coefficients         -- grid barrier
//   E   per-instance statistics
//
// The upwind system of one velocity row is bidiagonal (alpha = dt/dx max(v,0),
// beta = dt/dx max(-v,0), one of them is zero): for v > 0
//     x_i = (b_i + alpha x_{i-1}) / d_i,   x_0 = f^n(0, v)      (forward in x)
// and for v <= 0 the mirror image backward from f^n(nx-1, v).  Velocity tiles
// are split at the sign change so that a tile scans in one direction only.
// Each tile of 32 velocities x LX scan positions composes affine maps
// x -> P x + Y per thread segment, per tile, and between tiles through a
// deterministic decoupled look-back (predecessor maps are applied in a fixed
// nested order, so the result does not depend on timing).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "keq_common.cuh"
#include "keq_internal.h"

namespace keq {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kRows = 8;                 // scan positions per thread
constexpr int kLX = kWarps * kRows;      // scan positions per tile (64)
constexpr int kRB = kThreads;            // rows per reduction block
constexpr int kMaxAACols = 8;            // Anderson ring columns (aa_m <= 7)
constexpr int kMaxPairs = kMaxAACols * (kMaxAACols + 1) / 2;
constexpr int kPartQ = 4;                // doubles per (v-tile,row) partial

struct ImpInst {
    int nx, nv, n_inner, kp;
    int nt_neg, nvt, nchunks, nrb;
    long long tile_off, rb_off;
    double dx, dv, dt, tau_tilde, dtdx, u_max;
    int picard_iter, conv_type, fixed_iters;
    double tol, abs_tol;
    int aa_on, aa_cols, aa_stride, aa_start;
    double aa_beta, aa_reg, aa_alpha_max;
    const double* v;
    const double* f_in;
    double* f_out;
    keq_step_stats* stats;
    // workspace carve
    double* W;       // 3*nx  : n | nu | T   (W^(m))
    double* Wn;      // 3*nx  : moments of the newest iterate (unfloored)
    double* Wc;      // 4*nx  : per-row (u, -1/(2T), n/sqrt(2 pi T), dt/tau)
    double* Wb;      // 8     : moments of the two boundary rows (n,nu,T) x2 + flags
    double* part;    // nvt*n_inner*kPartQ
    double* lb;      // nvt*nchunks*3*32  (P | Y | X per lane)
    unsigned* lbflag;// nvt*nchunks
    double* res;     // 2*picard_iter : std / rel residual slots
    int* st;         // picard_iter   : 1 if active in iteration m
    int* nonfin;     // picard_iter   : non-finite flag of iterate m+1
    double* aaG;     // aa_cols * 3*n_inner
    double* aaR;     // aa_cols * 3*n_inner
    double* gpart;   // nrb * kMaxPairs
    double* alpha;   // picard_iter * kMaxAACols
    unsigned* rbdone;// picard_iter
};

struct PlanDev {
    GridBarrier bar;
    int err;
    int n_inst;
    int max_iter;
    int pad;
    long long total_tiles;
    long long total_rb;
    ImpInst* inst;
    long long* tile_off;  // n_inst+1
    long long* rb_off;    // n_inst+1
    unsigned* tickets;    // max_iter+1
};

struct SMem {
    double segP[kWarps][32];
    double segY[kWarps][32];
    double carry[kWarps][32];
    double red[kWarps][4];
    double alpha[kMaxAACols];
    long long tile;
    int flags;
};

__device__ __forceinline__ int find_inst(const long long* off, int n, long long t) {
    int lo = 0, hi = n;  // off[lo] <= t < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool iter_done(const ImpInst& I, int m) {
    // Convergence test of iteration m (bgk1d_implicit_cuda_kernel.py:241).
    if (I.fixed_iters > 0) return m + 1 >= I.fixed_iters;
    const double r = ld_cg(&I.res[2 * m]);
    return r <= 1.0;
}

__device__ __forceinline__ bool inst_active(const ImpInst& I, int m) {
    if (m >= I.picard_iter) return false;
    if (m == 0) return true;
    if (__ldcg(&I.st[m - 1]) != 1) return false;
    return !iter_done(I, m - 1);
}

// Per-row solve coefficients from (n, nu, T): implicit_kernels.cu:115-125
// (n, T clamped at 1e-300; 1/tau = n sqrt(T)/tau_tilde).
__device__ __forceinline__ void row_coeffs(const ImpInst& I, double n, double nu, double T,
                                           double* c4) {
    const double ni = n > kTiny ? n : kTiny;
    const double Ti = T > kTiny ? T : kTiny;
    const double ui = nu / ni;
    const double sT = sqrt(Ti);
    const double inv_tau = (ni * sT) / I.tau_tilde;
    c4[0] = ui;
    c4[1] = -0.5 / Ti;
    c4[2] = ni * kInvSqrt2Pi / sT;
    c4[3] = I.dt * inv_tau;
}

// C1/K1 moment semantics from raw sums.
__device__ __forceinline__ void moments_from_sums(double s0, double s1, double s2, double dv,
                                                  double* n, double* nu, double* T) {
    const double n_raw = s0 * dv;
    const double nu_raw = s1 * dv;
    const double s2d = s2 * dv;
    const double nv_ = n_raw > kTiny ? n_raw : kTiny;
    const double u = nu_raw / nv_;
    double Tg = s2d / nv_ - u * u;
    if (!(Tg > 0.0)) Tg = kTiny;
    *n = nv_;
    *nu = nu_raw;
    *T = Tg;
}

__device__ __forceinline__ double clamp_min_t(double x, double lo) {
    return (x != x || x >= lo) ? x : lo;
}

// ---- tile geometry --------------------------------------------------------
struct TileGeo {
    bool pos;      // velocities > 0 -> forward scan
    int j;         // this lane's velocity index
    bool lane_ok;
    int s0;        // first scan position of the tile
};

__device__ __forceinline__ TileGeo tile_geo(const ImpInst& I, int vt, int c, int lane) {
    TileGeo g;
    g.pos = vt >= I.nt_neg;
    g.j = g.pos ? I.kp + 32 * (vt - I.nt_neg) + lane : I.kp - 32 * (vt + 1) + lane;
    g.lane_ok = g.pos ? (g.j < I.nv) : (g.j >= 0);
    g.s0 = c * kLX;
    return g;
}

__device__ __forceinline__ int scan_row(const ImpInst& I, bool pos, int s) {
    return pos ? 1 + s : I.nx - 2 - s;
}

// ---- P1: partial moments of f^n -----------------------------------------
__device__ void moments_tile(const ImpInst& I, int vt, int c, const double* __restrict__ f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const TileGeo g = tile_geo(I, vt, c, lane);
    const double vj = g.lane_ok ? I.v[g.j] : 0.0;
    double acc[kRows * 3];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const int s = g.s0 + warp * kRows + r;
        double x = 0.0;
        if (s < I.n_inner && g.lane_ok) x = f[(size_t)scan_row(I, g.pos, s) * I.nv + g.j];
        acc[3 * r + 0] = x;
        acc[3 * r + 1] = x * vj;
        acc[3 * r + 2] = x * vj * vj;
    }
    warp_reduce_scatter<kRows, 3>(acc, lane);
    if (owner_writes<kRows>(lane)) {
        const int s = g.s0 + warp * kRows + owner_row<kRows>(lane);
        if (s < I.n_inner) {
            const int k = scan_row(I, g.pos, s) - 1;
            double* p = I.part + ((size_t)vt * I.n_inner + k) * kPartQ;
            p[0] = acc[0];
            p[1] = acc[1];
            p[2] = acc[2];
        }
    }
}

// ---- S(m): fused solve tile --------------------------------------------------
__device__ void solve_tile(int* err, const ImpInst& I, int vt, int c, int m, SMem& sm,
                           const double* __restrict__ fn, double* __restrict__ fo) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const TileGeo g = tile_geo(I, vt, c, lane);
    const double vj = g.lane_ok ? I.v[g.j] : 0.0;
    const double cpl = I.dtdx * fabs(vj);     // alpha (v>0) or beta (v<0)
    const double one_plus = 1.0 + cpl;          // 1 + alpha + beta
    const size_t tile_id = (size_t)c * I.nvt + vt;
    const unsigned f_agg = 2u * (unsigned)m + 1u, f_inc = 2u * (unsigned)m + 2u;

    // Anderson-combined W^(m) for this tile's rows (iterations after an
    // applied Anderson step).  alpha was solved by the last block of R(m-1).
    // Anderson call m-1 applied iff (m >= start, (m-start) % stride == 0) and
    // its history length min(m, cols) >= 2 (bgk1d_implicit_cuda_kernel.py:248-251).
    const int mh = m < I.aa_cols ? m : I.aa_cols;
    const bool aa_apply_prev = I.aa_on && m >= 1 && m >= I.aa_start &&
                               ((m - I.aa_start) % I.aa_stride == 0) && mh >= 2;

    double y[kRows], Pm[kRows], fold[kRows];
    double Pseg = 1.0, Yseg = 0.0;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const int s = g.s0 + warp * kRows + r;
        y[r] = Yseg;
        Pm[r] = Pseg;
        fold[r] = 0.0;
        if (s < I.n_inner) {
            const int i = scan_row(I, g.pos, s);
            double c4[4];
            if (aa_apply_prev) {
                // bgk1d_aa_cpu.py:170-188 on the fly for row i.
                const int k = i - 1, d = 3 * I.n_inner;
                const int head_out = m % I.aa_cols;
                double w[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    double acc = 0.0;
                    for (int jj = 0; jj < mh; ++jj) {
                        const int col = ((head_out - mh + jj) % I.aa_cols + I.aa_cols) % I.aa_cols;
                        acc += ld_cg(&I.aaG[(size_t)col * d + q * I.n_inner + k]) * sm.alpha[jj];
                    }
                    const double wnew = ld_cg(&I.Wn[q * I.nx + i]);
                    w[q] = acc * I.aa_beta + (1.0 - I.aa_beta) * wnew;
                }
                const double nm = clamp_min_t(w[0], 1e-12);
                const double Tm = clamp_min_t(w[2], 1e-12);
                double um = w[1] / nm;
                if (!isfinite(um)) um = 0.0;
                um = um < -I.u_max ? -I.u_max : (um > I.u_max ? I.u_max : um);
                const double num = nm * um;
                row_coeffs(I, nm, num, Tm, c4);
                if (vt == 0 && lane == 0) {
                    I.W[i] = nm;
                    I.W[I.nx + i] = num;
                    I.W[2 * I.nx + i] = Tm;
                }
            } else {
                const double2 c01 = __ldcg(reinterpret_cast<const double2*>(&I.Wc[4 * (size_t)i]));
                const double2 c23 = __ldcg(reinterpret_cast<const double2*>(&I.Wc[4 * (size_t)i + 2]));
                c4[0] = c01.x; c4[1] = c01.y; c4[2] = c23.x; c4[3] = c23.y;
            }
            if (g.lane_ok) {
                const size_t idx = (size_t)i * I.nv + g.j;
                const double fin = fn[idx];
                fold[r] = (m == 0) ? fin : fo[idx];
                const double diff = vj - c4[0];
                const double M = c4[2] * exp(diff * diff * c4[1]);
                const double b = fma(c4[3], M, fin);
                const double dd = one_plus + c4[3];
                const double rr = __drcp_rn(dd);
                Yseg = fma(cpl, Yseg, b) * rr;
                Pseg = Pseg * (cpl * rr);
                y[r] = Yseg;
                Pm[r] = Pseg;
            }
        }
    }
    sm.segP[warp][lane] = Pseg;
    sm.segY[warp][lane] = Yseg;
    __syncthreads();

    if (warp == 0) {
        // tile aggregate (nested composition of the 8 segment maps)
        double Pt = 1.0, Yt = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            Yt = fma(sm.segP[w][lane], Yt, sm.segY[w][lane]);
            Pt = sm.segP[w][lane] * Pt;
        }
        double* lbt = I.lb + tile_id * 96;
        lbt[lane] = Pt;
        lbt[32 + lane] = Yt;
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(&I.lbflag[tile_id], f_agg);

        // carry into the tile
        double X;
        if (c == 0) {
            X = g.lane_ok ? fn[(size_t)(g.pos ? 0 : I.nx - 1) * I.nv + g.j] : 0.0;
        } else {
            int k0 = -1;  // nearest predecessor chunk with an inclusive value
            bool ok = true;
            for (int base = c - 1; base >= 0 && ok; base -= 32) {
                const int kk = base - lane;
                unsigned fl = f_inc;  // chunks < 0: the boundary acts as inclusive
                if (kk >= 0) {
                    const unsigned* fp = &I.lbflag[(size_t)kk * I.nvt + vt];
                    if (!wait_flag_geq(fp, f_agg, err)) ok = false;
                    fl = ld_acquire(fp);
                }
                const unsigned incl = __ballot_sync(0xffffffffu, fl >= f_inc);
                if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
                if (incl) {
                    const int l = __ffs(incl) - 1;
                    k0 = base - l;
                    break;
                }
            }
            if (!ok) {
                X = 0.0;
            } else {
                if (k0 < 0)
                    X = g.lane_ok ? fn[(size_t)(g.pos ? 0 : I.nx - 1) * I.nv + g.j] : 0.0;
                else
                    X = ld_cg(&I.lb[((size_t)k0 * I.nvt + vt) * 96 + 64 + lane]);
                for (int k = (k0 < 0 ? 0 : k0 + 1); k < c; ++k) {
                    const double* q = I.lb + ((size_t)k * I.nvt + vt) * 96;
                    X = fma(ld_cg(q + lane), X, ld_cg(q + 32 + lane));
                }
            }
        }
        lbt[64 + lane] = fma(Pt, X, Yt);
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(&I.lbflag[tile_id], f_inc);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            sm.carry[w][lane] = X;
            X = fma(sm.segP[w][lane], X, sm.segY[w][lane]);
        }
    }
    __syncthreads();

    // final values, residual, non-finite check, partial moments
    const double Xc = sm.carry[warp][lane];
    double acc[kRows * 3];
    double q1 = 0.0, q2 = 0.0;
    bool bad = false;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const int s = g.s0 + warp * kRows + r;
        double x = 0.0;
        if (s < I.n_inner && g.lane_ok) {
            const int i = scan_row(I, g.pos, s);
            x = fma(Pm[r], Xc, y[r]);
            fo[(size_t)i * I.nv + g.j] = x;
            const double df = fabs(x - fold[r]);
            const double ref = nan_max(fabs(x), fabs(fold[r]));
            q1 = nan_max(q1, df / (I.abs_tol + I.tol * ref));
            const double rc = (ref != ref || ref >= I.abs_tol) ? ref : I.abs_tol;
            q2 = nan_max(q2, df / rc);
            bad |= !isfinite(x);
        }
        acc[3 * r + 0] = x;
        acc[3 * r + 1] = x * vj;
        acc[3 * r + 2] = x * vj * vj;
    }
    warp_reduce_scatter<kRows, 3>(acc, lane);
    if (owner_writes<kRows>(lane)) {
        const int s = g.s0 + warp * kRows + owner_row<kRows>(lane);
        if (s < I.n_inner) {
            const int k = scan_row(I, g.pos, s) - 1;
            double* p = I.part + ((size_t)vt * I.n_inner + k) * kPartQ;
            p[0] = acc[0];
            p[1] = acc[1];
            p[2] = acc[2];
        }
    }
    if (I.conv_type == 0) {
        q1 = warp_max(q1);
        q2 = warp_max(q2);
        if (lane == 0) {
            atomic_max_nonneg(&I.res[2 * m], q1);
            atomic_max_nonneg(&I.res[2 * m + 1], q2);
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&I.nonfin[m], 1);
}

// ---- Anderson: small symmetric solve (Cholesky, min-norm fall-back) -------
// torch.linalg.cholesky / cholesky_solve with the lstsq fall-back of
// bgk1d_aa_cpu.py:93-97; the fall-back here is a Jacobi eigen pseudo-inverse.
__device__ __noinline__ void aa_small_solve(int m, double* A, double* x) {
    double L[kMaxAACols * kMaxAACols];
    double yv[kMaxAACols];
    bool ok = true;
    for (int i = 0; i < kMaxAACols * kMaxAACols; ++i) L[i] = 0.0;
    for (int j = 0; j < m && ok; ++j) {
        double s = A[j * m + j];
        for (int k = 0; k < j; ++k) s -= L[j * m + k] * L[j * m + k];
        if (!(s > 0.0)) { ok = false; break; }
        const double ljj = sqrt(s);
        L[j * m + j] = ljj;
        for (int i = j + 1; i < m; ++i) {
            double t = A[i * m + j];
            for (int k = 0; k < j; ++k) t -= L[i * m + k] * L[j * m + k];
            L[i * m + j] = t / ljj;
        }
    }
    if (ok) {
        for (int i = 0; i < m; ++i) {
            double t = 1.0;
            for (int k = 0; k < i; ++k) t -= L[i * m + k] * yv[k];
            yv[i] = t / L[i * m + i];
        }
        for (int i = m - 1; i >= 0; --i) {
            double t = yv[i];
            for (int k = i + 1; k < m; ++k) t -= L[k * m + i] * x[k];
            x[i] = t / L[i * m + i];
        }
        return;
    }
    double a[kMaxAACols * kMaxAACols], V[kMaxAACols * kMaxAACols];
    for (int i = 0; i < m * m; ++i) a[i] = A[i];
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) V[i * m + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) off += a[p * m + q] * a[p * m + q];
        if (!(off > 1e-300)) break;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double apq = a[p * m + q];
                if (apq == 0.0) continue;
                const double th = (a[q * m + q] - a[p * m + p]) / (2.0 * apq);
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < m; ++k) {
                    const double akp = a[k * m + p], akq = a[k * m + q];
                    a[k * m + p] = cs * akp - sn * akq;
                    a[k * m + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = a[p * m + k], aqk = a[q * m + k];
                    a[p * m + k] = cs * apk - sn * aqk;
                    a[q * m + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double vkp = V[k * m + p], vkq = V[k * m + q];
                    V[k * m + p] = cs * vkp - sn * vkq;
                    V[k * m + q] = sn * vkp + cs * vkq;
                }
            }
    }
    double lmax = 0.0;
    for (int i = 0; i < m; ++i) lmax = fmax(lmax, fabs(a[i * m + i]));
    const double cut = lmax * (double)m * 2.220446049250313e-16;
    for (int i = 0; i < m; ++i) x[i] = 0.0;
    for (int k = 0; k < m; ++k) {
        const double lam = a[k * m + k];
        if (!(fabs(lam) > cut)) continue;
        double proj = 0.0;
        for (int i = 0; i < m; ++i) proj += V[i * m + k];
        proj /= lam;
        for (int i = 0; i < m; ++i) x[i] += proj * V[i * m + k];
    }
}

// Block-wide sum of one value per thread into red[] (fixed order); result
// valid in thread 0.
__device__ __forceinline__ double block_sum(double v, SMem& sm, int slot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sm.red[warp][slot] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) t += sm.red[w][slot];
    __syncthreads();
    return t;
}

__device__ __forceinline__ double block_max(double v, SMem& sm, int slot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_max(v);
    if (lane == 0) sm.red[warp][slot] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) t = nan_max(t, sm.red[w][slot]);
    __syncthreads();
    return t;
}

// ---- R(m): row reduction / W update ---------------------------------------
__device__ void reduce_block(const ImpInst& I, int rb, int m, SMem& sm) {
    const int k = rb * kRB + threadIdx.x;
    const bool ok = k < I.n_inner;
    const int i = k + 1;
    const int d = 3 * I.n_inner;
    double wn[3] = {0.0, 0.0, 0.0}, wo[3] = {0.0, 0.0, 0.0};
    if (ok) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int vt = 0; vt < I.nvt; ++vt) {
            const double* p = I.part + ((size_t)vt * I.n_inner + k) * kPartQ;
            s0 += ld_cg(p);
            s1 += ld_cg(p + 1);
            s2 += ld_cg(p + 2);
        }
        moments_from_sums(s0, s1, s2, I.dv, &wn[0], &wn[1], &wn[2]);
        wo[0] = ld_cg(&I.W[i]);
        wo[1] = ld_cg(&I.W[I.nx + i]);
        wo[2] = ld_cg(&I.W[2 * I.nx + i]);
        I.Wn[i] = wn[0];
        I.Wn[I.nx + i] = wn[1];
        I.Wn[2 * I.nx + i] = wn[2];
    }
    // conv_type "w": bgk1d_conv_util.py:35-58 over all nx cells
    if (I.conv_type == 1) {
        double q1 = 0.0, q2 = 0.0;
        auto add = [&](double a, double o) {
            const double df = fabs(a - o);
            const double ref = nan_max(fabs(a), fabs(o));
            q1 = nan_max(q1, df / (I.abs_tol + I.tol * ref));
            const double rc = (ref != ref || ref >= I.abs_tol) ? ref : I.abs_tol;
            q2 = nan_max(q2, df / rc);
        };
        if (ok)
            for (int q = 0; q < 3; ++q) add(wn[q], wo[q]);
        if (rb == 0 && threadIdx.x < 2) {
            const int ib = threadIdx.x == 0 ? 0 : I.nx - 1;
            for (int q = 0; q < 3; ++q) add(ld_cg(&I.Wb[3 * threadIdx.x + q]), ld_cg(&I.W[q * I.nx + ib]));
        }
        q1 = block_max(q1, sm, 0);
        q2 = block_max(q2, sm, 1);
        if (threadIdx.x == 0) {
            atomic_max_nonneg(&I.res[2 * m], q1);
            atomic_max_nonneg(&I.res[2 * m + 1], q2);
        }
    }
    // boundary rows: W <- floors(moments of the fixed boundary rows)
    if (rb == 0 && threadIdx.x < 2) {
        const int ib = threadIdx.x == 0 ? 0 : I.nx - 1;
        I.W[ib] = clamp_min_t(ld_cg(&I.Wb[3 * threadIdx.x + 0]), 1e-12);
        I.W[I.nx + ib] = ld_cg(&I.Wb[3 * threadIdx.x + 1]);
        I.W[2 * I.nx + ib] = clamp_min_t(ld_cg(&I.Wb[3 * threadIdx.x + 2]), 1e-12);
    }

    bool plain = true;
    if (I.aa_on) {
        // Anderson call number m (bgk1d_aa_cpu.py:7-129): history column
        // head_in = m % cols, history length min(m+1, cols).
        const int head_in = m % I.aa_cols;
        const int mh = (m + 1) < I.aa_cols ? (m + 1) : I.aa_cols;
        const int head_out = (m + 1) % I.aa_cols;
        const bool should = (m + 1) >= I.aa_start && ((m + 1 - I.aa_start) % I.aa_stride == 0);
        const bool apply = should && mh >= 2;
        if (ok) {
            for (int q = 0; q < 3; ++q) {
                I.aaG[(size_t)head_in * d + q * I.n_inner + k] = wn[q];
                I.aaR[(size_t)head_in * d + q * I.n_inner + k] = wn[q] - wo[q];
            }
        }
        if (apply) {
            plain = false;
            __syncthreads();  // this block's history writes are its own rows only
            int cols[kMaxAACols];
            for (int jj = 0; jj < mh; ++jj)
                cols[jj] = ((head_out - mh + jj) % I.aa_cols + I.aa_cols) % I.aa_cols;
            int pi = 0;
            for (int p = 0; p < mh; ++p)
                for (int q = p; q < mh; ++q, ++pi) {
                    double v = 0.0;
                    if (ok)
                        for (int cc = 0; cc < 3; ++cc)
                            v += I.aaR[(size_t)cols[p] * d + cc * I.n_inner + k] *
                                 I.aaR[(size_t)cols[q] * d + cc * I.n_inner + k];
                    v = block_sum(v, sm, 2);
                    if (threadIdx.x == 0) I.gpart[(size_t)rb * kMaxPairs + pi] = v;
                }
            // last block of this instance assembles the Gram matrix and solves
            if (threadIdx.x == 0) {
                __threadfence();
                const unsigned prev = atomicAdd(&I.rbdone[m], 1u);
                sm.flags = (prev == (unsigned)I.nrb - 1) ? 1 : 0;
            }
            __syncthreads();
            if (sm.flags && threadIdx.x == 0) {
                __threadfence();
                double A[kMaxAACols * kMaxAACols];
                int pj = 0;
                for (int p = 0; p < mh; ++p)
                    for (int q = p; q < mh; ++q, ++pj) {
                        double s = 0.0;
                        for (int r2 = 0; r2 < I.nrb; ++r2) s += ld_cg(&I.gpart[(size_t)r2 * kMaxPairs + pj]);
                        A[p * mh + q] = s;
                        A[q * mh + p] = s;
                    }
                for (int p = 0; p < mh; ++p) A[p * mh + p] += I.aa_reg;
                double al[kMaxAACols];
                aa_small_solve(mh, A, al);
                double asum = 0.0;
                for (int p = 0; p < mh; ++p) asum += al[p];
                if (fabs(asum) < 1.0e-30) asum = 1.0e-30;
                for (int p = 0; p < mh; ++p) {
                    double a = al[p] / asum;
                    if (I.aa_alpha_max > 0.0) {
                        if (a < -I.aa_alpha_max) a = -I.aa_alpha_max;
                        if (a > I.aa_alpha_max) a = I.aa_alpha_max;
                    }
                    I.alpha[(size_t)m * kMaxAACols + p] = a;
                }
            }
        }
    }
    if (plain && ok) {
        // bgk1d_implicit_cuda_kernel.py:285-287
        const double nn = clamp_min_t(wn[0], 1e-12);
        const double TT = clamp_min_t(wn[2], 1e-12);
        I.W[i] = nn;
        I.W[I.nx + i] = wn[1];
        I.W[2 * I.nx + i] = TT;
        double c4[4];
        row_coeffs(I, nn, wn[1], TT, c4);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[0] = make_double2(c4[0], c4[1]);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[1] = make_double2(c4[2], c4[3]);
    }
    if (rb == 0 && threadIdx.x == 0) I.st[m] = 1;
}

// ---- the persistent kernel --------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2)
implicit_step_kernel(PlanDev* __restrict__ Pp, int swap_io) {
    __shared__ SMem sm;
    PlanDev& P = *Pp;
    const unsigned G = gridDim.x;
    const int n_inst = P.n_inst;

    // P0: reset per-step state, boundary rows of f_out
    for (int b = blockIdx.x; b < n_inst; b += G) {
        const ImpInst& I = P.inst[b];
        const double* fn = swap_io ? I.f_out : I.f_in;
        double* fo = swap_io ? const_cast<double*>(I.f_in) : I.f_out;
        for (int q = threadIdx.x; q < 2 * I.picard_iter; q += kThreads) I.res[q] = 0.0;
        for (int q = threadIdx.x; q < I.picard_iter; q += kThreads) {
            I.st[q] = 0;
            I.nonfin[q] = 0;
            I.rbdone[q] = 0u;
        }
        for (int q = threadIdx.x; q < I.nvt * I.nchunks; q += kThreads) I.lbflag[q] = 0u;
        for (int q = threadIdx.x; q < I.nv; q += kThreads) {
            fo[q] = fn[q];
            fo[(size_t)(I.nx - 1) * I.nv + q] = fn[(size_t)(I.nx - 1) * I.nv + q];
        }
        // boundary-row moments (sequential per row, C1 order)
        if (threadIdx.x < 2) {
            const double* row = fn + (size_t)(threadIdx.x == 0 ? 0 : I.nx - 1) * I.nv;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int jj = 0; jj < I.nv; ++jj) {
                const double x = row[jj], vv = I.v[jj];
                s0 += x;
                s1 += x * vv;
                s2 += x * vv * vv;
            }
            double n, nu, T;
            moments_from_sums(s0, s1, s2, I.dv, &n, &nu, &T);
            I.Wb[3 * threadIdx.x + 0] = n;
            I.Wb[3 * threadIdx.x + 1] = nu;
            I.Wb[3 * threadIdx.x + 2] = T;
        }
    }
    if (blockIdx.x == 0)
        for (int q = threadIdx.x; q <= P.max_iter; q += kThreads) P.tickets[q] = 0u;
    if (!grid_sync(&P.bar, G, &P.err)) return;

    // P1: moments of f^n
    for (long long t = blockIdx.x; t < P.total_tiles; t += G) {
        const int b = find_inst(P.tile_off, n_inst, t);
        const ImpInst& I = P.inst[b];
        const long long tl = t - I.tile_off;
        const int c = (int)(tl / I.nvt), vt = (int)(tl % I.nvt);
        moments_tile(I, vt, c, swap_io ? I.f_out : I.f_in);
    }
    if (!grid_sync(&P.bar, G, &P.err)) return;

    // P2: W^(0) (unfloored C1 moments) and coefficients
    for (long long t = blockIdx.x; t < P.total_rb; t += G) {
        const int b = find_inst(P.rb_off, n_inst, t);
        const ImpInst& I = P.inst[b];
        const int rb = (int)(t - I.rb_off);
        const int k = rb * kRB + threadIdx.x;
        if (k < I.n_inner) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int vt = 0; vt < I.nvt; ++vt) {
                const double* p = I.part + ((size_t)vt * I.n_inner + k) * kPartQ;
                s0 += ld_cg(p);
                s1 += ld_cg(p + 1);
                s2 += ld_cg(p + 2);
            }
            double n, nu, T;
            moments_from_sums(s0, s1, s2, I.dv, &n, &nu, &T);
            const int i = k + 1;
            I.W[i] = n;
            I.W[I.nx + i] = nu;
            I.W[2 * I.nx + i] = T;
            double c4[4];
            row_coeffs(I, n, nu, T, c4);
            reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[0] = make_double2(c4[0], c4[1]);
            reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[1] = make_double2(c4[2], c4[3]);
        }
        if (rb == 0 && threadIdx.x < 2) {
            const int ib = threadIdx.x == 0 ? 0 : I.nx - 1;
            for (int q = 0; q < 3; ++q) I.W[q * I.nx + ib] = ld_cg(&I.Wb[3 * threadIdx.x + q]);
        }
    }
    if (!grid_sync(&P.bar, G, &P.err)) return;

    // Picard iterations
    for (int m = 0; m < P.max_iter; ++m) {
        bool any = false;
        for (int b = 0; b < n_inst && !any; ++b) any = inst_active(P.inst[b], m);
        if (!any) break;
        if (__ldcg(&P.err) != 0) break;

        // S(m)
        while (true) {
            if (threadIdx.x == 0) sm.tile = (long long)atomicAdd(&P.tickets[m], 1u);
            __syncthreads();
            const long long t = sm.tile;
            __syncthreads();
            if (t >= P.total_tiles) break;
            const int b = find_inst(P.tile_off, n_inst, t);
            const ImpInst& I = P.inst[b];
            if (!inst_active(I, m)) continue;
            const long long tl = t - I.tile_off;
            const int c = (int)(tl / I.nvt), vt = (int)(tl % I.nvt);
            // Anderson weights of the previous call, if it applied
            if (I.aa_on && m >= 1 && threadIdx.x < kMaxAACols)
                sm.alpha[threadIdx.x] = ld_cg(&I.alpha[(size_t)(m - 1) * kMaxAACols + threadIdx.x]);
            __syncthreads();
            const double* fn = swap_io ? I.f_out : I.f_in;
            double* fo = swap_io ? const_cast<double*>(I.f_in) : I.f_out;
            solve_tile(&P.err, I, vt, c, m, sm, fn, fo);
            __syncthreads();
        }
        if (!grid_sync(&P.bar, G, &P.err)) return;

        // R(m)
        for (long long t = blockIdx.x; t < P.total_rb; t += G) {
            const int b = find_inst(P.rb_off, n_inst, t);
            const ImpInst& I = P.inst[b];
            if (!inst_active(I, m)) continue;
            reduce_block(I, (int)(t - I.rb_off), m, sm);
            __syncthreads();
        }
        if (!grid_sync(&P.bar, G, &P.err)) return;
    }

    // E: statistics
    for (int b = blockIdx.x; b < n_inst; b += G) {
        if (threadIdx.x != 0) continue;
        const ImpInst& I = P.inst[b];
        int last = -1;
        for (int m = 0; m < I.picard_iter; ++m) {
            if (__ldcg(&I.st[m]) == 1) last = m;
            else break;
        }
        keq_step_stats* s = I.stats;
        int aa_applied = 0;
        if (I.aa_on)
            for (int m = 0; m < last; ++m) {
                const int mh = (m + 1) < I.aa_cols ? (m + 1) : I.aa_cols;
                const bool should = (m + 1) >= I.aa_start && ((m + 1 - I.aa_start) % I.aa_stride == 0);
                if (should && mh >= 2) ++aa_applied;
            }
        int status = KEQ_OK;
        if (last >= 0 && __ldcg(&I.nonfin[last])) status = KEQ_ERR_NONFINITE;
        if (P.err & (1 << KEQ_ERR_TIMEOUT)) status = KEQ_ERR_TIMEOUT;
        s->status = status;
        s->iters = last + 1;
        s->aa_applied = aa_applied;
        s->lo_iters = 0;
        s->residual = last >= 0 ? ld_cg(&I.res[2 * last + 1]) : 0.0;
        s->std_residual = last >= 0 ? ld_cg(&I.res[2 * last]) : 0.0;
        s->lo_residual = 0.0;
        s->std_lo_residual = 0.0;
        s->max_YI = 0.0;
        s->total_iters += last + 1;
        s->total_steps += 1;
    }
}

}  // namespace keq

// ===========================================================================
// Host side: plan construction and launch
// ===========================================================================
namespace {

using keq::ImpInst;
using keq::PlanDev;

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Carve {
    char* base;
    size_t off;
    template <class T>
    T* take(size_t count) {
        off = align_up(off, 256);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += sizeof(T) * (count ? count : 1);
        return p;
    }
};

struct Derived {
    int n_inner, nt_neg, nt_pos, nvt, nchunks, nrb, aa_cols, aa_on;
};

Derived derive(int nx, int nv, int kp, const keq_implicit_params& p) {
    Derived d;
    d.n_inner = nx - 2;
    d.nt_neg = (kp + 31) / 32;
    d.nt_pos = (nv - kp + 31) / 32;
    d.nvt = d.nt_neg + d.nt_pos;
    d.nchunks = (d.n_inner + keq::kLX - 1) / keq::kLX;
    d.nrb = (d.n_inner + keq::kRB - 1) / keq::kRB;
    const int aa_m = p.aa_m > 0 ? p.aa_m : 0;
    d.aa_on = (p.aa_enable && aa_m >= 1 && aa_m + 1 >= 2) ? 1 : 0;
    d.aa_cols = d.aa_on ? aa_m + 1 : 1;
    return d;
}

// Carve the per-instance workspace; with base == nullptr only the size is
// computed.  The layout depends on (nx, nv, kp, params).
size_t carve_instance(void* base, int nx, int nv, int kp, const keq_implicit_params& p,
                      ImpInst* I) {
    const Derived d = derive(nx, nv, kp, p);
    Carve c{static_cast<char*>(base), 0};
    const int it = p.picard_iter > 0 ? p.picard_iter : 1;
    double* W = c.take<double>(3 * (size_t)nx);
    double* Wn = c.take<double>(3 * (size_t)nx);
    double* Wc = c.take<double>(4 * (size_t)nx);
    double* Wb = c.take<double>(8);
    double* part = c.take<double>((size_t)d.nvt * d.n_inner * keq::kPartQ);
    double* lb = c.take<double>((size_t)d.nvt * d.nchunks * 96);
    unsigned* lbflag = c.take<unsigned>((size_t)d.nvt * d.nchunks);
    double* res = c.take<double>(2 * (size_t)it);
    int* st = c.take<int>(it);
    int* nonfin = c.take<int>(it);
    double* aaG = c.take<double>(d.aa_on ? (size_t)d.aa_cols * 3 * d.n_inner : 1);
    double* aaR = c.take<double>(d.aa_on ? (size_t)d.aa_cols * 3 * d.n_inner : 1);
    double* gpart = c.take<double>(d.aa_on ? (size_t)d.nrb * keq::kMaxPairs : 1);
    double* alpha = c.take<double>((size_t)it * keq::kMaxAACols);
    unsigned* rbdone = c.take<unsigned>(it);
    if (I) {
        I->W = W; I->Wn = Wn; I->Wc = Wc; I->Wb = Wb; I->part = part; I->lb = lb;
        I->lbflag = lbflag; I->res = res; I->st = st; I->nonfin = nonfin; I->aaG = aaG;
        I->aaR = aaR; I->gpart = gpart; I->alpha = alpha; I->rbdone = rbdone;
    }
    return align_up(c.off, 256);
}

// Worst-case kp for sizing before v is known on the host: the tile count is
// maximal when the sign change is not 32-aligned.
int sizing_kp(int nv) { return nv / 2 + 1 <= nv ? nv / 2 + 1 : nv; }

bool valid_params(const keq_implicit_params& p) {
    if (p.picard_iter < 1 || p.picard_iter > 100000) return false;
    if (p.conv_type != 0 && p.conv_type != 1) return false;
    if (p.aa_enable && p.aa_m > keq::kMaxAACols - 1) return false;
    return true;
}

keq_implicit_params normalized(const keq_implicit_params& in) {
    // bgk1d_implicit_cuda_kernel.py:56-65
    keq_implicit_params p = in;
    p.aa_m = p.aa_m > 0 ? p.aa_m : 0;
    p.aa_beta = p.aa_beta < 0.0 ? 0.0 : (p.aa_beta > 1.0 ? 1.0 : p.aa_beta);
    p.aa_stride = p.aa_stride > 1 ? p.aa_stride : 1;
    p.aa_start_iter = p.aa_start_iter > 1 ? p.aa_start_iter : 1;
    p.aa_reg = p.aa_reg > 1e-14 ? p.aa_reg : 1e-14;
    p.aa_alpha_max = p.aa_alpha_max > 0.0 ? p.aa_alpha_max : 0.0;
    return p;
}

}  // namespace

struct keq_plan {
    std::vector<ImpInst> host_inst;
    std::vector<long long> tile_off, rb_off;
    PlanDev* dev;           // device header (inside the plan workspace)
    ImpInst* dev_inst;
    int grid;
    int n_inst;
    int device;
};

extern "C" {

keq_status keq_implicit_instance_workspace_size(const keq_grid* grid,
                                                const keq_implicit_params* params,
                                                size_t* bytes) {
    if (!grid || !params || !bytes) return KEQ_ERR_INVALID;
    if (grid->nx < 3 || grid->nv < 1) return KEQ_ERR_INVALID;
    if (!valid_params(*params)) return KEQ_ERR_INVALID;
    const keq_implicit_params p = normalized(*params);
    *bytes = carve_instance(nullptr, grid->nx, grid->nv, sizing_kp(grid->nv), p, nullptr);
    // the tile count is maximal for some kp; take the max over both extremes
    const size_t b2 = carve_instance(nullptr, grid->nx, grid->nv, 0, p, nullptr);
    const size_t b3 = carve_instance(nullptr, grid->nx, grid->nv, grid->nv, p, nullptr);
    if (b2 > *bytes) *bytes = b2;
    if (b3 > *bytes) *bytes = b3;
    // any kp: nt_neg + nt_pos <= nv/32 + 2
    const size_t worst = carve_instance(nullptr, grid->nx, grid->nv + 64, (grid->nv + 64) / 2, p, nullptr);
    if (worst > *bytes) *bytes = worst;
    return KEQ_OK;
}

static size_t plan_bytes(int n, int max_iter) {
    Carve c{nullptr, 0};
    c.take<PlanDev>(1);
    c.take<ImpInst>(n);
    c.take<long long>(n + 1);
    c.take<long long>(n + 1);
    c.take<unsigned>(max_iter + 1);
    return align_up(c.off, 256);
}

keq_status keq_implicit_plan_workspace_size(const keq_instance* insts, int32_t n,
                                            const keq_implicit_params* params,
                                            int32_t per_instance_params, size_t* bytes) {
    if (!insts || n < 1 || !params || !bytes) return KEQ_ERR_INVALID;
    int max_iter = 1;
    for (int b = 0; b < n; ++b) {
        const int pi = params[per_instance_params ? b : 0].picard_iter;
        if (pi > max_iter) max_iter = pi;
    }
    *bytes = plan_bytes(n, max_iter);
    return KEQ_OK;
}

keq_status keq_implicit_plan_create(const keq_instance* insts, int32_t n,
                                    const keq_implicit_params* params,
                                    int32_t per_instance_params, void* plan_ws,
                                    size_t plan_ws_bytes, keq_stream_t stream,
                                    keq_plan** plan_out) {
    using namespace keq;
    if (!insts || n < 1 || !params || !plan_ws || !plan_out) return KEQ_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(plan_ws) % 256) return KEQ_ERR_WORKSPACE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // Bind this thread's runtime to the device that owns the buffers.
    int dev_of_buffers = -1;
    {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, insts[0].f_in) != cudaSuccess ||
            pa.type != cudaMemoryTypeDevice) {
            cudaGetLastError();
            return KEQ_ERR_INVALID;
        }
        dev_of_buffers = pa.device;
        if (cudaSetDevice(dev_of_buffers) != cudaSuccess) {
            keq_internal_set_cuda_error(cudaGetLastError());
            return KEQ_ERR_CUDA;
        }
    }
    int max_iter = 1;
    for (int b = 0; b < n; ++b) {
        const keq_implicit_params& p = params[per_instance_params ? b : 0];
        if (!valid_params(p)) return KEQ_ERR_INVALID;
        if (p.picard_iter > max_iter) max_iter = p.picard_iter;
    }
    if (plan_ws_bytes < plan_bytes(n, max_iter)) return KEQ_ERR_WORKSPACE;

    keq_plan* plan = new keq_plan();
    plan->n_inst = n;
    plan->device = dev_of_buffers;
    plan->host_inst.resize(n);
    plan->tile_off.resize(n + 1);
    plan->rb_off.resize(n + 1);
    long long toff = 0, roff = 0;
    std::vector<double> vh;
    for (int b = 0; b < n; ++b) {
        const keq_instance& in = insts[b];
        const keq_implicit_params p = normalized(params[per_instance_params ? b : 0]);
        const int nx = in.grid.nx, nv = in.grid.nv;
        if (nx < 3 || nv < 1 || !in.grid.v || !in.f_in || !in.f_out || !in.stats ||
            !in.workspace || in.f_in == in.f_out || !(in.dt > 0.0) || !(in.tau_tilde > 0.0) ||
            !(in.grid.dx > 0.0) || !(in.grid.dv > 0.0)) {
            delete plan;
            return KEQ_ERR_INVALID;
        }
        if (reinterpret_cast<uintptr_t>(in.workspace) % 256) {
            delete plan;
            return KEQ_ERR_WORKSPACE;
        }
        vh.resize(nv);
        if (cudaMemcpyAsync(vh.data(), in.grid.v, sizeof(double) * nv, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            keq_internal_set_cuda_error(cudaGetLastError());
            delete plan;
            return KEQ_ERR_CUDA;
        }
        int kp = 0;
        double vmax = 0.0;
        for (int j = 0; j < nv; ++j) {
            if (j > 0 && !(vh[j] > vh[j - 1])) {
                delete plan;
                return KEQ_ERR_INVALID;  // v must be strictly ascending
            }
            if (!(vh[j] > 0.0)) kp = j + 1;
            vmax = fmax(vmax, fabs(vh[j]));
        }
        const Derived d = derive(nx, nv, kp, p);
        ImpInst I{};
        I.nx = nx; I.nv = nv; I.n_inner = d.n_inner; I.kp = kp;
        I.nt_neg = d.nt_neg; I.nvt = d.nvt; I.nchunks = d.nchunks; I.nrb = d.nrb;
        I.tile_off = toff; I.rb_off = roff;
        I.dx = in.grid.dx; I.dv = in.grid.dv; I.dt = in.dt; I.tau_tilde = in.tau_tilde;
        I.dtdx = in.dt / in.grid.dx;
        I.u_max = 0.95 * vmax;
        I.picard_iter = p.picard_iter; I.conv_type = p.conv_type; I.fixed_iters = p.fixed_iters;
        I.tol = p.picard_tol; I.abs_tol = p.abs_tol;
        I.aa_on = d.aa_on; I.aa_cols = d.aa_cols; I.aa_stride = p.aa_stride;
        I.aa_start = p.aa_start_iter; I.aa_beta = p.aa_beta; I.aa_reg = p.aa_reg;
        I.aa_alpha_max = p.aa_alpha_max;
        I.v = in.grid.v; I.f_in = in.f_in; I.f_out = in.f_out; I.stats = in.stats;
        carve_instance(in.workspace, nx, nv, kp, p, &I);
        plan->host_inst[b] = I;
        plan->tile_off[b] = toff;
        plan->rb_off[b] = roff;
        toff += (long long)d.nvt * d.nchunks;
        roff += d.nrb;
    }
    plan->tile_off[n] = toff;
    plan->rb_off[n] = roff;

    Carve c{static_cast<char*>(plan_ws), 0};
    PlanDev* dev = c.take<PlanDev>(1);
    ImpInst* dinst = c.take<ImpInst>(n);
    long long* dtoff = c.take<long long>(n + 1);
    long long* droff = c.take<long long>(n + 1);
    unsigned* tickets = c.take<unsigned>(max_iter + 1);
    PlanDev h{};
    h.n_inst = n;
    h.max_iter = max_iter;
    h.total_tiles = toff;
    h.total_rb = roff;
    h.inst = dinst;
    h.tile_off = dtoff;
    h.rb_off = droff;
    h.tickets = tickets;
    plan->dev = dev;
    plan->dev_inst = dinst;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dinst, plan->host_inst.data(), sizeof(ImpInst) * n,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtoff, plan->tile_off.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(droff, plan->rb_off.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, s);
    // stats start from zero totals
    if (e == cudaSuccess)
        for (int b = 0; b < n && e == cudaSuccess; ++b)
            e = cudaMemsetAsync(insts[b].stats, 0, sizeof(keq_step_stats), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host staging must outlive the copies
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        delete plan;
        return KEQ_ERR_CUDA;
    }
    int dev_id = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, keq::implicit_step_kernel, kThreads, 0);
    if (occ < 1 || sms < 1) {
        delete plan;
        return KEQ_ERR_UNSUPPORTED;
    }
    long long work = toff > roff ? toff : roff;
    long long g = (long long)sms * occ;
    if (work < g) g = work > 0 ? work : 1;
    plan->grid = (int)g;
    *plan_out = plan;
    return KEQ_OK;
}

keq_status keq_plan_set_buffers(keq_plan* plan, const double* const* f_in, double* const* f_out,
                                keq_stream_t stream) {
    if (!plan || !f_in || !f_out) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int b = 0; b < plan->n_inst; ++b) {
        if (!f_in[b] || !f_out[b] || f_in[b] == f_out[b]) return KEQ_ERR_INVALID;
        plan->host_inst[b].f_in = f_in[b];
        plan->host_inst[b].f_out = f_out[b];
    }
    cudaError_t e = cudaMemcpyAsync(plan->dev_inst, plan->host_inst.data(),
                                    sizeof(ImpInst) * plan->n_inst, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        return KEQ_ERR_CUDA;
    }
    return KEQ_OK;
}

keq_status keq_plan_step(keq_plan* plan, int32_t n_steps, int32_t parity, keq_stream_t stream) {
    if (!plan || n_steps < 0) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaSetDevice(plan->device) != cudaSuccess) {
        keq_internal_set_cuda_error(cudaGetLastError());
        return KEQ_ERR_CUDA;
    }
    for (int k = 0; k < n_steps; ++k) {
        int swap_io = ((parity + k) & 1);
        void* args[] = {&plan->dev, &swap_io};
        cudaError_t e = cudaLaunchCooperativeKernel((const void*)keq::implicit_step_kernel,
                                                    dim3(plan->grid), dim3(keq::kThreads), args,
                                                    0, s);
        if (e != cudaSuccess) {
            keq_internal_set_cuda_error(e);
            return KEQ_ERR_CUDA;
        }
    }
    return KEQ_OK;
}

void keq_plan_destroy(keq_plan* plan) { delete plan; }

keq_status keq_plan_error(keq_plan* plan, keq_stream_t stream, int32_t* err_bits) {
    if (!plan || !err_bits) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, &plan->dev->err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        return KEQ_ERR_CUDA;
    }
    *err_bits = v;
    return KEQ_OK;
}

keq_status keq_implicit_workspace_size(const keq_grid* grid, const keq_implicit_params* params,
                                       size_t* bytes) {
    size_t a = 0;
    keq_status st = keq_implicit_instance_workspace_size(grid, params, &a);
    if (st != KEQ_OK) return st;
    *bytes = a + plan_bytes(1, params->picard_iter > 0 ? params->picard_iter : 1);
    return KEQ_OK;
}

keq_status keq_implicit_step(const keq_grid* grid, double dt, double tau_tilde,
                             const keq_implicit_params* params, const double* f_in,
                             double* f_out, keq_step_stats* stats, void* workspace,
                             size_t workspace_bytes, keq_stream_t stream) {
    if (!grid || !params || !workspace) return KEQ_ERR_INVALID;
    size_t a = 0;
    keq_status st = keq_implicit_instance_workspace_size(grid, params, &a);
    if (st != KEQ_OK) return st;
    size_t need = 0;
    keq_implicit_workspace_size(grid, params, &need);
    if (workspace_bytes < need) return KEQ_ERR_WORKSPACE;
    keq_instance in{};
    in.grid = *grid;
    in.dt = dt;
    in.tau_tilde = tau_tilde;
    in.f_in = f_in;
    in.f_out = f_out;
    in.stats = stats;
    in.workspace = workspace;
    keq_plan* plan = nullptr;
    st = keq_implicit_plan_create(&in, 1, params, 0, static_cast<char*>(workspace) + a,
                                  workspace_bytes - a, stream, &plan);
    if (st != KEQ_OK) return st;
    st = keq_plan_step(plan, 1, 0, stream);
    keq_plan_destroy(plan);
    return st;
}

}  // extern "C"
