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
//   P0  per-step device state, boundary rows of f_out, boundary-row moments
//                                                           -- grid barrier
//   P1  velocity moments of f^n (tile partial sums)         -- grid barrier
//   P2  row reduction -> W^(0) = (n, nu, T), row coefficients -- grid barrier
//   per Picard iteration m while any instance is active, ONE pass over the
//   tiles (claimed in x order from a global ticket):
//     Maxwellian + upwind implicit assembly of the tile's rows, composition
//     of the tile map, decoupled look-back for the carry (keq_tile.cuh),
//     recurrence, write of f^(m+1), residual against f^(m), partial moments;
//     the warp that completes a row block reduces it: W_new, the "w"
//     residual, Anderson history and Gram partials (the last row block
//     solves the small Anderson system)              -- grid barrier
//   E   per-instance statistics
//
// Per cell and Picard iteration the pass reads f^n and f^(m) and writes
// f^(m+1): 24 bytes in FP64; the Maxwellian, the coefficients and the
// moments stay on chip.  f_out holds the newest iterate and is updated in
// place (each element is read as f^(m) and rewritten as f^(m+1) by the same
// lane).
//
// The upwind system of one velocity row is bidiagonal (alpha = dt/dx max(v,0),
// beta = dt/dx max(-v,0), one of them is zero): for v > 0
//     x_i = (b_i + alpha x_{i-1}) / d_i,   x_0 = f^n(0, v)      (forward in x)
// with d_i = 1 + alpha + dt/tau_i and b_i = f^n_i + dt/tau_i M_i(v), and for
// v <= 0 the mirror image backward from f^n(nx-1, v).
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "keq_common.cuh"
#include "keq_internal.h"
#include "keq_tile.cuh"

namespace keq {

constexpr int kWarps = 4;                // warps per CTA
constexpr int kThreads = kWarps * 32;
constexpr int kMaxAACols = 8;            // Anderson ring columns (aa_m <= 7)
constexpr int kMaxPairs = kMaxAACols * (kMaxAACols + 1) / 2;

struct ImpInst {
    int nx, nv, n_inner, kp;
    int nt_neg, nvt, nchunks, nrb;
    int rows, pad0;  // rows per tile (R)
    long long tile_off, rb_off;
    double dx, dv, dt, tau_tilde, dtdx, u_max;
    int picard_iter, conv_type, fixed_iters, pad1;
    double tol, abs_tol;
    int aa_on, aa_cols, aa_stride, aa_start;
    double aa_beta, aa_reg, aa_alpha_max;
    int mixed, pad2;  // mixed-precision form: FP32 sweeps, then FP64 sweeps
    double tol32;     // Picard tolerance that ends the FP32 sweeps
    const double* v;
    const double* f_in;
    double* f_out;
    keq_step_stats* stats;
    const int* enable;  // optional device flag: 0 = leave this instance untouched this step
    // workspace carve
    double* W;       // 3*nx  : n | nu | T   (W^(m))
    double* Wn;      // 3*nx  : moments of the newest iterate (unfloored)
    double* Wc;      // 4*nx  : per-row (u, -1/(2T), n/sqrt(2 pi T), dt/tau)
    double* Wb;      // 8     : moments of the two boundary rows
    double* part;    // nvt*n_inner*kPartQ
    double* agg;     // ntiles*64 : tile maps (P | Y per lane)
    double* inc;     // ntiles*32 : tile inclusive values (carry out)
    unsigned long long* flag;  // ntiles : (epoch << 2) | {agg, inc}
    unsigned* rbcnt; // picard_iter*nrb  : rows x v-tiles of a row block done
    double* res;     // 2*picard_iter : std / rel residual slots
    int* st;         // picard_iter   : 1 if active in iteration m
    int* nonfin;     // picard_iter   : non-finite flag of iterate m+1
    double* aaG;     // aa_cols * 3*n_inner
    double* aaR;     // aa_cols * 3*n_inner
    double* gpart;   // kMaxPairs * nrb : Gram partials of the row blocks, pair-major
    double* alpha;   // picard_iter * kMaxAACols
    unsigned* rbdone;// picard_iter
    float* fn32;     // nx*nv (mixed form): f^n in FP32, written by P1
    float* x32;      // nx*nv (mixed form): the FP32 iterate, updated in place
};

// Device header of an implicit plan (starts with the common PlanHead).
struct PlanDev {
    PlanHead head;
    int n_inst;
    int max_iter;
    long long total_tiles;
    long long total_rb;
    ImpInst* inst;
    long long* tile_off;  // n_inst+1
    long long* rb_off;    // n_inst+1
    unsigned* tickets;    // max_iter : tile claims of iteration m
};

// Per-warp shared memory.
struct WarpSmem {
    ImpInst I;
    double a[kRmax][33];   // f^n tile -> c = b/d -> x (solution), row stride 33
    double coef[kRmax][4]; // (u, -1/(2T), n/sqrt(2 pi T), dt/tau) per row
    double vv[32];         // the tile's velocities (0 where absent)
    int cur_b, cur_m, cur_active, pad;
    int done_rb[2];
};

// Mixed-precision form: iteration m is an FP32 sweep while no earlier sweep
// met the FP32-phase tolerance tol32 (all earlier iterations are then FP32
// sweeps too) and m is in the first half of the iteration cap; every later
// iteration is an FP64 sweep with the reference's tolerance.  Replays
// (fixed_iters) run in FP64 only.
__device__ __forceinline__ bool fp32_iter(const ImpInst& I, int m) {
    if (!I.mixed || I.fixed_iters > 0 || m >= I.picard_iter / 2) return false;
    for (int k = 0; k < m; ++k)
        if (ld_cg(&I.res[2 * k]) <= 1.0) return false;
    return true;
}

__device__ __forceinline__ bool iter_done(const ImpInst& I, int m) {
    // Convergence test of iteration m (bgk1d_implicit_cuda_kernel.py:241).
    if (I.fixed_iters > 0) return m + 1 >= I.fixed_iters;
    if (fp32_iter(I, m)) return false;  // an FP32 sweep never ends the step
    const double r = ld_cg(&I.res[2 * m]);
    return r <= 1.0;
}

__device__ __forceinline__ bool inst_enabled(const ImpInst& I) {
    return I.enable == nullptr || __ldcg(I.enable) != 0;
}

__device__ __forceinline__ bool inst_active(const ImpInst& I, int m) {
    // A disabled instance's st/res hold a previous launch's values (the
    // prologue skips it), so the mask is consulted at every iteration.
    if (m >= I.picard_iter || !inst_enabled(I)) return false;
    if (m == 0) return true;
    if (__ldcg(&I.st[m - 1]) != 1) return false;
    return !iter_done(I, m - 1);
}

// Anderson call z (after Picard iteration z) applies the combination iff
// z+1 >= start, (z+1-start) % stride == 0 and its history length
// min(z+1, cols) >= 2 (bgk1d_implicit_cuda_kernel.py:247-282, bgk1d_aa_cpu.py:131).
__device__ __forceinline__ bool aa_applies(const ImpInst& I, int z) {
    const int mh = (z + 1) < I.aa_cols ? (z + 1) : I.aa_cols;
    return I.aa_on && (z + 1) >= I.aa_start && ((z + 1 - I.aa_start) % I.aa_stride == 0) &&
           mh >= 2;
}

// Per-row solve coefficients from (n, nu, T): implicit_kernels.cu:115-125
// (n, T clamped at 1e-300; 1/tau = n sqrt(T)/tau_tilde).
__device__ __forceinline__ void row_coeffs(double tau_tilde, double dt, double n, double nu,
                                           double T, double* c4) {
    const double ni = n > kTiny ? n : kTiny;
    const double Ti = T > kTiny ? T : kTiny;
    const double ui = nu / ni;
    const double sT = sqrt(Ti);
    const double inv_tau = (ni * sT) / tau_tilde;
    c4[0] = ui;
    c4[1] = -0.5 / Ti;
    c4[2] = ni * kInvSqrt2Pi / sT;
    c4[3] = dt * inv_tau;
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

__device__ __forceinline__ TileGeo inst_tile(const ImpInst& I, int vt, int c, int lane) {
    return tile_geo(I.nt_neg, I.kp, I.nv, I.n_inner, I.rows, vt, c, lane);
}

// Copy an instance descriptor into the warp's shared memory.  Reads of the
// descriptor then cannot alias the warp's global stores.
__device__ __forceinline__ void stage_warp(WarpSmem& w, const ImpInst* src, int b) {
    if (w.cur_b != b) {
        __syncwarp();
        const int lane = threadIdx.x & 31;
        const int* s = reinterpret_cast<const int*>(src);
        int* d = reinterpret_cast<int*>(&w.I);
        for (int q = lane; q < (int)(sizeof(ImpInst) / sizeof(int)); q += 32) d[q] = __ldg(s + q);
        __syncwarp();
        if (lane == 0) {
            w.cur_b = b;
            w.cur_m = -1;
        }
    }
    __syncwarp();
}

// Warp-collective fp32_iter (every lane with the same I and m): the earlier
// residuals are read 32 per round instead of one dependent load at a time.
__device__ __forceinline__ bool fp32_iter_warp(const ImpInst& I, int m) {
    if (!I.mixed || I.fixed_iters > 0 || m >= I.picard_iter / 2) return false;
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < m; base += 32) {
        const int k = base + lane;
        const bool met = k < m && ld_cg(&I.res[2 * k]) <= 1.0;
        if (__any_sync(0xffffffffu, met)) return false;
    }
    return true;
}

// inst_active with fp32_iter(I, m-1) already known.
__device__ __forceinline__ bool inst_active_known(const ImpInst& I, int m, bool prev32) {
    if (m >= I.picard_iter || !inst_enabled(I)) return false;
    if (m == 0) return true;
    if (__ldcg(&I.st[m - 1]) != 1) return false;
    if (I.fixed_iters > 0) return m < I.fixed_iters;
    if (prev32) return true;
    return !(ld_cg(&I.res[2 * (m - 1)]) <= 1.0);
}

// Activity of the staged instance in iteration m and whether iterations m
// and m-1 are FP32 sweeps, cached per warp (bit 0 active, bit 1 iteration m
// is an FP32 sweep, bit 2 iteration m-1 was).  Warp-collective.
__device__ __forceinline__ bool staged_active(WarpSmem& w, int m) {
    if (w.cur_m != m) {
        const bool p32 = m > 0 && fp32_iter_warp(w.I, m - 1);
        const bool a = inst_active_known(w.I, m, p32);
        const bool c32 = a && fp32_iter_warp(w.I, m);
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            w.cur_active = (a ? 1 : 0) | (c32 ? 2 : 0) | (p32 ? 4 : 0);
            w.cur_m = m;
        }
        __syncwarp();
    }
    return (w.cur_active & 1) != 0;
}

// Asynchronous copy of a tile's rows into shared memory (one 8-byte element
// per lane and row, all rows in flight at once).
template <int STRIDE>
__device__ __forceinline__ void stage_rows(double (*dst)[STRIDE], const double* __restrict__ src,
                                           const TileGeo& g, int nx, int nv) {
    const int lane = threadIdx.x & 31;
    if (!g.lane_ok) return;
#pragma unroll 8
    for (int r = 0; r < g.nrows; ++r)
        cp_async8(&dst[r][lane], src + (size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j);
}

// Store the per-(v-tile, row) partial moments of the tile held in w.a
// (lane r sums row r over the 32 columns).
__device__ __forceinline__ void store_partials(WarpSmem& w, const TileGeo& g, int vt) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (lane < g.nrows) {
        double s[4];
        row_sums4(w.a, w.vv, lane, s);
        const int k = scan_row(I.nx, g.pos, g.s0 + lane) - 1;
        double* p = I.part + ((size_t)vt * I.n_inner + k) * kPartQ;
        reinterpret_cast<double2*>(p)[0] = make_double2(s[0], s[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(s[2], s[3]);
    }
    __syncwarp();
}

// ---- P1: partial moments of f^n (one tile) -------------------------------
__device__ void moments_tile(WarpSmem& w, int vt, int c, const double* __restrict__ f) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    stage_rows<33>(w.a, f, g, I.nx, I.nv);
    cp_async_commit();
    w.vv[lane] = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    cp_async_wait_all();
    if (!g.lane_ok)
        for (int r = 0; r < g.nrows; ++r) w.a[r][lane] = 0.0;
    else if (I.mixed)
        for (int r = 0; r < g.nrows; ++r)
            I.fn32[(size_t)scan_row(I.nx, g.pos, g.s0 + r) * I.nv + g.j] = (float)w.a[r][lane];
    store_partials(w, g, vt);
}

// Row coefficients of W^(m) for the tile's rows into w.coef (lane r handles
// row r).  After an applied Anderson call the combination
// w = beta G alpha + (1-beta) w_new with floors and |u| <= u_max
// (bgk1d_aa_cpu.py:170-188) is formed from the history ring; tiles of v-tile 0
// then publish W^(m) and its coefficients for the reduction.
__device__ __forceinline__ void stage_coeffs(WarpSmem& w, const TileGeo& g, int vt, int m) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int nx = I.nx, n_inner = I.n_inner;
    double c4[4] = {0.0, 0.0, 0.0, 0.0};
    if (lane < g.nrows) {
        const int i = scan_row(nx, g.pos, g.s0 + lane);
        if (m >= 1 && aa_applies(I, m - 1)) {
            const int k = i - 1, d = 3 * n_inner;
            const int mh = m < I.aa_cols ? m : I.aa_cols;
            const int head_out = m % I.aa_cols;
            // every load is issued unconditionally (entries past the history
            // length repeat its last column and are selected out of the sums),
            // so that each batch is in flight together
            double al[kMaxAACols];
            int col[kMaxAACols];
            const int col0 = ((head_out - mh) % I.aa_cols + I.aa_cols) % I.aa_cols;
#pragma unroll
            for (int jj = 0; jj < kMaxAACols; ++jj) {
                const int jc = jj < mh ? jj : mh - 1;
                al[jj] = ld_cg(&I.alpha[(size_t)(m - 1) * kMaxAACols + jc]);
                col[jj] = col0 + jc >= I.aa_cols ? col0 + jc - I.aa_cols : col0 + jc;
            }
            double wv[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                double gv[kMaxAACols];
#pragma unroll
                for (int jj = 0; jj < kMaxAACols; ++jj)
                    gv[jj] = ld_cg(&I.aaG[(size_t)col[jj] * d + q * n_inner + k]);
                const double wnew = ld_cg(&I.Wn[q * nx + i]);
                double acc = 0.0;
#pragma unroll
                for (int jj = 0; jj < kMaxAACols; ++jj) acc += jj < mh ? gv[jj] * al[jj] : 0.0;
                wv[q] = acc * I.aa_beta + (1.0 - I.aa_beta) * wnew;
            }
            const double nm = clamp_min_t(wv[0], 1e-12);
            const double Tm = clamp_min_t(wv[2], 1e-12);
            double um = wv[1] / nm;
            if (!isfinite(um)) um = 0.0;
            um = um < -I.u_max ? -I.u_max : (um > I.u_max ? I.u_max : um);
            const double num = nm * um;
            row_coeffs(I.tau_tilde, I.dt, nm, num, Tm, c4);
            if (vt == 0) {
                I.W[i] = nm;
                I.W[nx + i] = num;
                I.W[2 * nx + i] = Tm;
                reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[0] = make_double2(c4[0], c4[1]);
                reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[1] = make_double2(c4[2], c4[3]);
            }
        } else {
            const double2 c01 = __ldcg(reinterpret_cast<const double2*>(&I.Wc[4 * (size_t)i]));
            const double2 c23 = __ldcg(reinterpret_cast<const double2*>(&I.Wc[4 * (size_t)i + 2]));
            c4[0] = c01.x; c4[1] = c01.y; c4[2] = c23.x; c4[3] = c23.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) w.coef[lane][q] = c4[q];
}

// ---- the Picard pass over one tile ------------------------------------------
// Assembly of the tile's rows (x_s = a_s x_{s-1} + c_s with a_s = alpha/d_s,
// c_s = b_s/d_s), look-back for the carry, recurrence, residual against
// f^(m) and partial moments of f^(m+1).  Returns false if the look-back gave
// up (timeout).
__device__ bool picard_tile(WarpSmem& w, int vt, int c, int m, unsigned long long epoch,
                            unsigned long long limit, const double* __restrict__ fn,
                            double* __restrict__ fo, FracMax& q1, FracMax& q2, bool& bad) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    const int nx = I.nx, nv = I.nv;
    const int nr = g.nrows;
    // f^n rows into shared memory; the residual reference f^(m) (f^n itself
    // at m = 0; the FP32 iterate after the FP32 sweeps of the mixed form) is
    // streamed into registers 8 rows ahead of the recurrence, the first 8
    // rows before the look-back
    const bool ref32 = (w.cur_active & 4) != 0;  // iteration m-1 was an FP32 sweep
    const double* ref64 = m > 0 ? fo : fn;
    stage_rows<33>(w.a, fn, g, nx, nv);
    cp_async_commit();
    auto ld_ref = [&](int r) -> double {
        if (r >= nr || !g.lane_ok) return 0.0;
        const size_t off = (size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j;
        return ref32 ? (double)__ldcg(&I.x32[off]) : __ldcg(&ref64[off]);
    };
    double on[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) on[t] = ld_ref(t);
    const double vj = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    w.vv[lane] = vj;
    stage_coeffs(w, g, vt, m);
    cp_async_wait_all();
    __syncwarp();
    const double cpl = I.dtdx * fabs(vj);  // alpha (v>0) or beta (v<0)
    const double one_plus = 1.0 + cpl;     // 1 + alpha + beta
    // tile map: c_s into w.a, (P, Y) composed in scan order
    double P = 1.0, Y = 0.0;
#pragma unroll 1
    for (int r0 = 0; r0 < nr; r0 += 8) {
        double av[8], cv[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int r = r0 + t < nr ? r0 + t : nr - 1;
            const double diff = vj - w.coef[r][0];
            const double dti = w.coef[r][3];
            const double M = w.coef[r][2] * exp_nonpos(diff * diff * w.coef[r][1]);
            const double rr = recip_ge1(one_plus + dti);
            const double fnv = g.lane_ok ? w.a[r][lane] : 0.0;
            cv[t] = fma(dti, M, fnv) * rr;
            av[t] = cpl * rr;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            if (r0 + t < nr) {
                w.a[r0 + t][lane] = cv[t];
                Y = fma(av[t], Y, cv[t]);
                P = P * av[t];
            }
        }
    }
    // carry into the tile
    const size_t tid = (size_t)c * I.nvt + vt;
    bool ok = true;
    double X;
    if (c == 0) {
        X = g.lane_ok ? __ldg(&fn[(size_t)(g.pos ? 0 : nx - 1) * nv + g.j]) : 0.0;
    } else {
        publish_agg(I.agg, I.flag, tid, P, Y, epoch);
        ok = lookback(I.agg, I.inc, I.flag, I.nvt, vt, c, epoch, limit, X);
    }
    if (c + 1 < I.nchunks) publish_inc(I.inc, I.flag, tid, fma(P, X, Y), epoch);
    // recurrence, write, residual.  The rows of a batch are branch-free
    // (clamped row index, selects, a predicated store) so that the compiler
    // can overlap their independent work; the residual takes the select-only
    // path of FracMax, and a tile that met a non-finite or non-positive ratio
    // term redoes its residual with the full update afterwards.
    const double tol = I.tol, abs_tol = I.abs_tol;
    bool odd = false;
#pragma unroll 1
    for (int r0 = 0; r0 < nr; r0 += 8) {
        double onx[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) onx[t] = ld_ref(r0 + 8 + t);
        const int nb = nr - r0;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const bool in = t < nb;
            const int r = in ? r0 + t : r0;
            const double a = cpl * recip_ge1(one_plus + w.coef[r][3]);
            const double Xn = fma(a, X, w.a[r][lane]);
            X = in ? Xn : X;
            const double x = g.lane_ok ? X : 0.0;
            if (in) w.a[r][lane] = x;
            const bool use = in && g.lane_ok;
            const double o = on[t];
            const double df = use ? fabs(x - o) : 0.0;
            const double ref = use ? nan_max(fabs(x), fabs(o)) : 0.0;
            const double b1 = use ? abs_tol + tol * ref : 1.0;
            const double b2 = use ? ((ref != ref || ref >= abs_tol) ? ref : abs_tol) : 1.0;
            const bool n1 = q1.add_normal(df, b1);
            const bool n2 = q2.add_normal(df, b2);
            odd |= !(n1 && n2);
            bad |= use && !isfinite(x);
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) on[t] = onx[t];
    }
    if (__any_sync(0xffffffffu, odd) && g.lane_ok) {
        // rare: the full residual update over the tile's rows (f^(m) is still
        // in place; the tile's rows are written after the reduction)
        for (int r = 0; r < nr; ++r) {
            const double x = w.a[r][lane];
            const double o = ld_ref(r);
            const double df = fabs(x - o);
            const double ref = nan_max(fabs(x), fabs(o));
            q1.add(df, abs_tol + tol * ref);
            q2.add(df, (ref != ref || ref >= abs_tol) ? ref : abs_tol);
        }
    }
    store_partials(w, g, vt);
    return ok;
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}

// FP32 sweep of the mixed-precision form over one tile: the same assembly,
// look-back and recurrence with the Maxwellian, the reciprocal and the
// recurrence in FP32 on the FP32 copies of f^n and of the iterate (12 bytes
// per cell instead of 24); the residual (against tol32) and the partial
// moments are accumulated in FP64.
__device__ bool picard_tile32(WarpSmem& w, int vt, int c, int m, unsigned long long epoch,
                              unsigned long long limit, const double* __restrict__ fn,
                              FracMax& q1, FracMax& q2, bool& bad) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    const int nx = I.nx, nv = I.nv;
    const int nr = g.nrows;
    // f^n (FP32) staged in the tile buffer (read into registers by the map
    // loop before the recurrence writes the buffer); the previous FP32
    // iterate streamed into registers
    float(*fa)[32] = reinterpret_cast<float(*)[32]>(&w.a[0][0]);
    const float* ref = m > 0 ? I.x32 : I.fn32;
    if (g.lane_ok) {
#pragma unroll 8
        for (int r = 0; r < nr; ++r) {
            const size_t off = (size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j;
            cp_async4(&fa[r][lane], I.fn32 + off);
        }
    }
    cp_async_commit();
    // the previous iterate of every row, loaded unconditionally (rows past the
    // tile and absent velocities read a clamped, present cell; their values
    // are selected out) so that the 32 loads are in flight together
    float fbv[kRmax];
    const int jc = g.j < 0 ? 0 : (g.j >= nv ? nv - 1 : g.j);
#pragma unroll
    for (int r = 0; r < kRmax; ++r) {
        const int rc = r < nr ? r : nr - 1;
        fbv[r] = __ldcg(&ref[(size_t)scan_row(nx, g.pos, g.s0 + rc) * nv + jc]);
    }
    const double vjd = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    w.vv[lane] = vjd;
    stage_coeffs(w, g, vt, m);
    cp_async_wait_all();
    __syncwarp();
    const float vj = (float)vjd;
    const float cpl = (float)(I.dtdx * fabs(vjd));
    const float one_plus = 1.0f + cpl;
    float P = 1.0f, Y = 0.0f;
    float cvs[kRmax];
#pragma unroll
    for (int r = 0; r < kRmax; ++r) {
        cvs[r] = 0.0f;
        if (r < nr) {
            const float diff = vj - (float)w.coef[r][0];
            const float dti = (float)w.coef[r][3];
            const float M = (float)w.coef[r][2] * expf(diff * diff * (float)w.coef[r][1]);
            const float rr = 1.0f / (one_plus + dti);
            const float fnv = g.lane_ok ? fa[r][lane] : 0.0f;
            const float cv = fmaf(dti, M, fnv) * rr;
            const float av = cpl * rr;
            cvs[r] = cv;
            Y = fmaf(av, Y, cv);
            P = P * av;
        }
    }
    const size_t tid = (size_t)c * I.nvt + vt;
    bool ok = true;
    double Xd;
    if (c == 0) {
        Xd = g.lane_ok ? (double)__ldg(&fn[(size_t)(g.pos ? 0 : nx - 1) * nv + g.j]) : 0.0;
    } else {
        publish_agg(I.agg, I.flag, tid, (double)P, (double)Y, epoch);
        ok = lookback(I.agg, I.inc, I.flag, I.nvt, vt, c, epoch, limit, Xd);
    }
    if (c + 1 < I.nchunks) publish_inc(I.inc, I.flag, tid, fma((double)P, Xd, (double)Y), epoch);
    __syncwarp();  // every lane has read its f^n (FP32) before the buffer takes x
    float X = (float)Xd;
    const double tol = I.tol32, abs_tol = I.abs_tol;
    // branch-free rows (selects, a predicated store) with the select-only
    // residual; a tile that met a non-finite or non-positive term redoes the
    // residual with the full update
    bool odd = false;
#pragma unroll
    for (int r = 0; r < kRmax; ++r) {
        const bool in = r < nr;
        const float a = cpl / (one_plus + (float)w.coef[r][3]);
        const float Xn = fmaf(a, X, cvs[r]);
        X = in ? Xn : X;
        const float x = g.lane_ok ? X : 0.0f;
        if (in) w.a[r][lane] = (double)x;
        const bool use = in && g.lane_ok;
        const double o = (double)fbv[r];
        const double df = use ? fabs((double)x - o) : 0.0;
        const double rf = use ? nan_max(fabs((double)x), fabs(o)) : 0.0;
        const bool n1 = q1.add_normal(df, use ? abs_tol + tol * rf : 1.0);
        const bool n2 = q2.add_normal(df, use ? ((rf != rf || rf >= abs_tol) ? rf : abs_tol) : 1.0);
        odd |= !(n1 && n2);
        bad |= use && !isfinite(x);
    }
    if (__any_sync(0xffffffffu, odd) && g.lane_ok) {
        for (int r = 0; r < nr; ++r) {
            const double x = w.a[r][lane];
            const double o = (double)__ldcg(&ref[(size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j]);
            const double df = fabs(x - o);
            const double rf = nan_max(fabs(x), fabs(o));
            q1.add(df, abs_tol + tol * rf);
            q2.add(df, (rf != rf || rf >= abs_tol) ? rf : abs_tol);
        }
    }
    store_partials(w, g, vt);
    return ok;
}

// Write the tile's new iterate (held in w.a) to HBM: FP64 into fo, or FP32
// into the mixed form's iterate.  Done after the row-block arrival, so the
// fence of that arrival does not wait for these stores.
__device__ __forceinline__ void write_tile(WarpSmem& w, int vt, int c, double* __restrict__ fo,
                                           bool fp32) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    if (!g.lane_ok) return;
    if (fp32) {
#pragma unroll 8
        for (int r = 0; r < g.nrows; ++r)
            I.x32[(size_t)scan_row(I.nx, g.pos, g.s0 + r) * I.nv + g.j] = (float)w.a[r][lane];
    } else {
#pragma unroll 8
        for (int r = 0; r < g.nrows; ++r)
            fo[(size_t)scan_row(I.nx, g.pos, g.s0 + r) * I.nv + g.j] = w.a[r][lane];
    }
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

// Index of pair (p, q), p <= q, in the row-major upper triangle of an m x m
// symmetric matrix.
__host__ __device__ constexpr int aa_pair(int p, int q, int m) {
    return p * m - (p * (p - 1)) / 2 + (q - p);
}
__device__ __forceinline__ double aa_clip(double a, double alpha_max) {
    if (alpha_max > 0.0) {
        if (a < -alpha_max) a = -alpha_max;
        if (a > alpha_max) a = alpha_max;
    }
    return a;
}

// Anderson coefficients for a history of compile-time length M in one thread,
// the factor in registers: (G + reg I) x = 1 by Cholesky with the sums in the
// order of aa_small_solve, then alpha = x / sum(x), clipped
// (bgk1d_aa_cpu.py:146-168).  Each pivot is kept as its reciprocal square
// root and the divisions by it are multiplications, so the dependent chain of
// a column is one rsqrt.  False (nothing written) when a pivot is not
// positive, for the min-norm fall-back.
template <int M>
__device__ __forceinline__ bool aa_alpha_fixed(const double* gs, double reg, double alpha_max,
                                               double* alpha_out) {
    double L[M][M], rd[M];  // strict lower factor; rd[j] = 1 / L[j][j]
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) L[i][j] = gs[aa_pair(j, i, M)] + (i == j ? reg : 0.0);
#pragma unroll
    for (int j = 0; j < M; ++j) {
        double s = L[j][j];
#pragma unroll
        for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
        if (!(s > 0.0)) return false;
        rd[j] = rsqrt(s);
#pragma unroll
        for (int i = j + 1; i < M; ++i) {
            double t = L[i][j];
#pragma unroll
            for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
            L[i][j] = t * rd[j];
        }
    }
    double y[M], x[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        double t = 1.0;
#pragma unroll
        for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
        y[i] = t * rd[i];
    }
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        double t = y[i];
#pragma unroll
        for (int k = i + 1; k < M; ++k) t -= L[k][i] * x[k];
        x[i] = t * rd[i];
    }
    double asum = 0.0;
#pragma unroll
    for (int p = 0; p < M; ++p) asum += x[p];
    if (fabs(asum) < 1.0e-30) asum = 1.0e-30;
    const double rs = 1.0 / asum;
#pragma unroll
    for (int p = 0; p < M; ++p) alpha_out[p] = aa_clip(x[p] * rs, alpha_max);
    return true;
}

// Last reduction block of Anderson call m: Gram matrix from the per-block
// partials, stored pair-major (lane l sums blocks l, l+32, ... of eight pairs
// at a time, 32 loads in flight, then a butterfly over the lanes; the sums go
// through the warp's scratch `gs` in shared memory),
// regularised Cholesky solve, normalisation by the sum, clip
// (bgk1d_aa_cpu.py:146-168).
__device__ __noinline__ void aa_finalize(const double* gpart, int nrb, int mh, double reg,
                                         double alpha_max, double* alpha_out, double* gs) {
    const int lane = threadIdx.x & 31;
    const int npairs = mh * (mh + 1) / 2;
    for (int q0 = 0; q0 < npairs; q0 += 8) {
        double acc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = 0.0;
        for (int r0 = 0; r0 < nrb; r0 += 128) {
            double t[8][4];
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    // clamped indices: every load is issued, the extra ones add 0
                    const int r = r0 + 32 * c + lane;
                    const bool in = q0 + u < npairs && r < nrb;
                    const int qc = q0 + u < npairs ? q0 + u : npairs - 1;
                    const double v = ld_cg(&gpart[(size_t)qc * nrb + (r < nrb ? r : nrb - 1)]);
                    t[u][c] = in ? v : 0.0;
                }
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[u] += t[u][c];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = warp_sum(acc[u]);
        if (lane == 0)
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (q0 + u < npairs) gs[q0 + u] = acc[u];
    }
    __syncwarp();
    if (lane != 0) return;
    bool ok = false;
    switch (mh) {
        case 1: ok = aa_alpha_fixed<1>(gs, reg, alpha_max, alpha_out); break;
        case 2: ok = aa_alpha_fixed<2>(gs, reg, alpha_max, alpha_out); break;
        case 3: ok = aa_alpha_fixed<3>(gs, reg, alpha_max, alpha_out); break;
        case 4: ok = aa_alpha_fixed<4>(gs, reg, alpha_max, alpha_out); break;
        case 5: ok = aa_alpha_fixed<5>(gs, reg, alpha_max, alpha_out); break;
        case 6: ok = aa_alpha_fixed<6>(gs, reg, alpha_max, alpha_out); break;
        case 7: ok = aa_alpha_fixed<7>(gs, reg, alpha_max, alpha_out); break;
        default: ok = aa_alpha_fixed<8>(gs, reg, alpha_max, alpha_out); break;
    }
    if (ok) return;
    // not positive definite: the min-norm fall-back on the full matrix
    double A[kMaxAACols * kMaxAACols], xv[kMaxAACols];
    for (int p = 0; p < mh; ++p)
        for (int q = 0; q < mh; ++q) {
            const int a = p < q ? p : q, b = p < q ? q : p;
            A[p * mh + q] = gs[aa_pair(a, b, mh)] + (p == q ? reg : 0.0);
        }
    aa_small_solve(mh, A, xv);
    double asum = 0.0;
    for (int p = 0; p < mh; ++p) asum += xv[p];
    if (fabs(asum) < 1.0e-30) asum = 1.0e-30;
    for (int p = 0; p < mh; ++p) alpha_out[p] = aa_clip(xv[p] / asum, alpha_max);
}

// ---- row reduction / W update of one row block (lane = row) -------------
__device__ __noinline__ void reduce_block(WarpSmem& w, int ru, int m) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int k = ru * kRB + lane;
    const bool ok = k < I.n_inner;
    const int i = k + 1;
    const int nx = I.nx, n_inner = I.n_inner, d = 3 * n_inner;
    // Anderson call m: history column head_in = m % cols, length min(m+1, cols)
    const bool aa_now = aa_applies(I, m);
    const int cols = I.aa_cols > 0 ? I.aa_cols : 1;
    const int head_in = m % cols;
    const int mh = (m + 1) < cols ? (m + 1) : cols;
    const int head_out = (m + 1) % cols;
    if (aa_now) {
        // the block's older residual columns r_j (3 components per row) into
        // the warp's tile buffer (free here; row = lane, column 3 j + c),
        // copied while the moment partials are read; the newest column
        // (jj = mh - 1, slot head_in) is formed below
        int col = ((head_out - mh) % cols + cols) % cols;
        for (int jj = 0; jj < mh - 1; ++jj) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (ok)
                    cp_async8(&w.a[lane][3 * jj + q], &I.aaR[(size_t)col * d + q * n_inner + k]);
                else
                    w.a[lane][3 * jj + q] = 0.0;
            }
            col = col + 1 == cols ? 0 : col + 1;
        }
    }
    double wn[3] = {0.0, 0.0, 0.0}, wo[3] = {0.0, 0.0, 0.0};
    if (ok) {
        wo[0] = ld_cg(&I.W[i]);
        wo[1] = ld_cg(&I.W[nx + i]);
        wo[2] = ld_cg(&I.W[2 * nx + i]);
        double s[4];
        sum_partials4(I.part, 0, I.nvt, n_inner, k, s);
        moments_from_sums(s[0], s[1], s[2], I.dv, &wn[0], &wn[1], &wn[2]);
        I.Wn[i] = wn[0];
        I.Wn[nx + i] = wn[1];
        I.Wn[2 * nx + i] = wn[2];
    }
    // conv_type "w": bgk1d_conv_util.py:35-58 over all nx cells
    if (I.conv_type == 1) {
        const double at = I.abs_tol, tl = I.tol;
        FracMax q1, q2;
        if (ok) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double df = fabs(wn[q] - wo[q]);
                const double ref = nan_max(fabs(wn[q]), fabs(wo[q]));
                q1.add(df, at + tl * ref);
                q2.add(df, (ref != ref || ref >= at) ? ref : at);
            }
        }
        if (ru == 0 && lane < 2) {  // the two boundary rows
            const int ib = lane == 0 ? 0 : nx - 1;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double a = ld_cg(&I.Wb[3 * lane + q]), o = ld_cg(&I.W[q * nx + ib]);
                const double df = fabs(a - o);
                const double ref = nan_max(fabs(a), fabs(o));
                q1.add(df, at + tl * ref);
                q2.add(df, (ref != ref || ref >= at) ? ref : at);
            }
        }
        const double r1 = warp_max(q1.value()), r2 = warp_max(q2.value());
        if (lane == 0) {
            atomic_max_nonneg(&I.res[2 * m], r1);
            atomic_max_nonneg(&I.res[2 * m + 1], r2);
        }
    }
    // boundary rows: W <- floors(moments of the fixed boundary rows)
    if (ru == 0 && lane < 2) {
        const int ib = lane == 0 ? 0 : nx - 1;
        I.W[ib] = clamp_min_t(ld_cg(&I.Wb[3 * lane + 0]), 1e-12);
        I.W[nx + ib] = ld_cg(&I.Wb[3 * lane + 1]);
        I.W[2 * nx + ib] = clamp_min_t(ld_cg(&I.Wb[3 * lane + 2]), 1e-12);
    }

    bool plain = true;
    if (I.aa_on) {
        if (ok) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                I.aaG[(size_t)head_in * d + q * n_inner + k] = wn[q];
                I.aaR[(size_t)head_in * d + q * n_inner + k] = wn[q] - wo[q];
            }
        }
        if (aa_now) {
            plain = false;
#pragma unroll
            for (int q = 0; q < 3; ++q) w.a[lane][3 * (mh - 1) + q] = ok ? wn[q] - wo[q] : 0.0;
            cp_async_wait_all();
            __syncwarp();
            // Gram partials of the block: lane t sums pair t = (p, q) over the
            // block's rows in row order
            const int npairs = mh * (mh + 1) / 2;
            for (int t = lane; t < npairs; t += 32) {
                int p = 0, rem = t;
                while (rem >= mh - p) {
                    rem -= mh - p;
                    ++p;
                }
                const int q = p + rem;
                double v = 0.0;
#pragma unroll 8
                for (int r = 0; r < kRB; ++r)
                    v += w.a[r][3 * p] * w.a[r][3 * q] + w.a[r][3 * p + 1] * w.a[r][3 * q + 1] +
                         w.a[r][3 * p + 2] * w.a[r][3 * q + 2];
                I.gpart[(size_t)t * I.nrb + ru] = v;
            }
            __syncwarp();
            fence_acq_rel();
            __syncwarp();
            unsigned prev = 0;
            if (lane == 0) prev = atomicAdd(&I.rbdone[m], 1u);
            prev = __shfl_sync(0xffffffffu, prev, 0);
            if (prev == (unsigned)I.nrb - 1) {
                fence_acq_rel();
                __syncwarp();
                aa_finalize(I.gpart, I.nrb, mh, I.aa_reg, I.aa_alpha_max,
                            I.alpha + (size_t)m * kMaxAACols, &w.coef[0][0]);
            }
        }
    }
    if (plain && ok) {
        // bgk1d_implicit_cuda_kernel.py:285-287
        const double nn = clamp_min_t(wn[0], 1e-12);
        const double TT = clamp_min_t(wn[2], 1e-12);
        I.W[i] = nn;
        I.W[nx + i] = wn[1];
        I.W[2 * nx + i] = TT;
        double c4[4];
        row_coeffs(I.tau_tilde, I.dt, nn, wn[1], TT, c4);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[0] = make_double2(c4[0], c4[1]);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[1] = make_double2(c4[2], c4[3]);
    }
    if (ru == 0 && lane == 0) I.st[m] = 1;
    __syncwarp();
}

// ---- P2: W^(0) from the moment partials of f^n (lane = row) --------------
__device__ void init_block(WarpSmem& w, int ru) {
    const ImpInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int k = ru * kRB + lane;
    const int nx = I.nx, n_inner = I.n_inner;
    if (k < n_inner) {
        double s[4];
        sum_partials4(I.part, 0, I.nvt, n_inner, k, s);
        double n, nu, T;
        moments_from_sums(s[0], s[1], s[2], I.dv, &n, &nu, &T);
        const int i = k + 1;
        I.W[i] = n;
        I.W[nx + i] = nu;
        I.W[2 * nx + i] = T;
        double c4[4];
        row_coeffs(I.tau_tilde, I.dt, n, nu, T, c4);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[0] = make_double2(c4[0], c4[1]);
        reinterpret_cast<double2*>(&I.Wc[4 * (size_t)i])[1] = make_double2(c4[2], c4[3]);
    }
    if (ru == 0 && lane < 2) {
        const int ib = lane == 0 ? 0 : nx - 1;
        for (int q = 0; q < 3; ++q) I.W[q * nx + ib] = ld_cg(&I.Wb[3 * lane + q]);
    }
}

__device__ __forceinline__ void flush_residual(const ImpInst& I, int m, FracMax& q1, FracMax& q2,
                                               bool& bad) {
    const int lane = threadIdx.x & 31;
    const double r1 = warp_max(q1.value()), r2 = warp_max(q2.value());
    const bool anybad = __any_sync(0xffffffffu, bad);
    if (lane == 0 && I.conv_type == 0) {
        atomic_max_nonneg(&I.res[2 * m], r1);
        atomic_max_nonneg(&I.res[2 * m + 1], r2);
    }
    if (lane == 0 && anybad) atomicOr(&I.nonfin[m], 1);
    q1 = FracMax();
    q2 = FracMax();
    bad = false;
}

// Phase trace (off unless a buffer is attached): per Picard iteration the
// earliest start and latest end over all warps of the pass, in
// %globaltimer nanoseconds: [m][0] min start, [1] max end; [2], [3] unused.
constexpr int kTracePhases = 4;
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void trace_mark(const PlanDev& P, int m, int ph, bool is_min) {
    if (P.head.trace == nullptr || (threadIdx.x & 31) != 0 || m >= P.head.trace_iters) return;
    unsigned long long* slot = P.head.trace + (size_t)m * kTracePhases + ph;
    const unsigned long long t = gtimer();
    if (is_min) atomicMin(slot, t); else atomicMax(slot, t);
}

// Grid barrier of a launch; on a timeout the error is also recorded in the
// sticky word read by keq_plan_error.
__device__ __forceinline__ bool plan_sync(PlanDev& P, unsigned G) {
    if (grid_sync(&P.head.bar, G, &P.head.err, P.head.spin_limit)) return true;
    if (threadIdx.x == 0) atomicOr(&P.head.err_sticky, 1 << KEQ_ERR_TIMEOUT);
    return false;
}

// Next tile ticket of iteration m (lane 0 claims, broadcast to the warp).
__device__ __forceinline__ long long claim(unsigned* tickets, int m) {
    unsigned t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(&tickets[m], 1u);
    return (long long)__shfl_sync(0xffffffffu, t, 0);
}

// ---- the persistent kernel --------------------------------------------------
// P1 tiles and row blocks are statically strided over all resident warps.
// The Picard pass claims tiles from a ticket counter so tiles are started in
// x order (chunk-major), which keeps every look-back short and guarantees
// that a tile's predecessors are held by running warps.
__global__ void __launch_bounds__(kThreads, 4)
implicit_step_kernel(PlanDev* __restrict__ Pp, int swap_io) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PlanDev& P = *Pp;
    const unsigned G = gridDim.x;
    const int n_inst = P.n_inst;
    const long long total_tiles = P.total_tiles, total_rb = P.total_rb;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
    const long long gwarp = (long long)blockIdx.x * kWarps + warp, nwarps = (long long)G * kWarps;
    if (lane == 0) w.cur_b = -1;
    __syncwarp();

    // P0: reset per-step state, boundary rows of f_out, boundary-row moments
    if (blockIdx.x == 0) {
        for (int q = threadIdx.x; q < P.max_iter; q += kThreads) P.tickets[q] = 0u;
        if (threadIdx.x == 0) P.head.seq = P.head.seq + 1ull;
    }
    for (int b = blockIdx.x; b < n_inst; b += G) {
        const ImpInst& I = P.inst[b];
        if (!inst_enabled(I)) continue;
        const double* fn = swap_io ? I.f_out : I.f_in;
        double* fo = swap_io ? const_cast<double*>(I.f_in) : I.f_out;
        // pending status: stays KEQ_ERR_TIMEOUT unless stage E of this launch
        // runs, i.e. when a device-side wait gave up and the CTAs returned
        if (threadIdx.x == 0) {
            I.stats->status = KEQ_ERR_TIMEOUT;
            if (P.head.fresh) {
                I.stats->total_iters = 0;
                I.stats->total_steps = 0;
            }
        }
        // look-back flags: epoch 0 is never current
        const long long ntiles = (long long)I.nvt * I.nchunks;
        for (long long q = threadIdx.x; q < ntiles; q += kThreads) I.flag[q] = 0ull;
        for (int q = threadIdx.x; q < 2 * I.picard_iter; q += kThreads) I.res[q] = 0.0;
        for (int q = threadIdx.x; q < I.picard_iter; q += kThreads) {
            I.st[q] = 0;
            I.nonfin[q] = 0;
            I.rbdone[q] = 0u;
        }
        for (int q = threadIdx.x; q < I.picard_iter * I.nrb; q += kThreads) I.rbcnt[q] = 0u;
        for (int q = threadIdx.x; q < I.nv; q += kThreads) {
            fo[q] = fn[q];
            fo[(size_t)(I.nx - 1) * I.nv + q] = fn[(size_t)(I.nx - 1) * I.nv + q];
        }
        if (threadIdx.x < 2) {
            // sequential per row, the C1 order
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
    if (!plan_sync(P, G)) return;
    const unsigned long long seq = __ldcg(&P.head.seq);
    const unsigned long long limit = P.head.spin_limit;

    // P1: moments of f^n
    for (long long t = gwarp; t < total_tiles; t += nwarps) {
        const int b = find_inst(P.tile_off, n_inst, t);
        stage_warp(w, &P.inst[b], b);
        if (!inst_enabled(w.I)) continue;
        const long long tl = t - w.I.tile_off;
        const int c = (int)(tl / w.I.nvt), vt = (int)(tl % w.I.nvt);
        moments_tile(w, vt, c, swap_io ? w.I.f_out : w.I.f_in);
    }
    if (!plan_sync(P, G)) return;

    // P2: W^(0) (unfloored C1 moments) and coefficients
    for (long long u = gwarp; u < total_rb; u += nwarps) {
        const int b = find_inst(P.rb_off, n_inst, u);
        stage_warp(w, &P.inst[b], b);
        if (!inst_enabled(w.I)) continue;
        init_block(w, (int)(u - w.I.rb_off));
    }
    if (!plan_sync(P, G)) return;

    // Picard iterations
    for (int m = 0; m < P.max_iter; ++m) {
        // any instance active in iteration m: every thread tests a share of
        // the instances, combined over the CTA (the same answer in every CTA)
        bool mine = false;
        for (int b = threadIdx.x; b < n_inst && !mine; b += kThreads) mine = inst_active(P.inst[b], m);
        if (!__syncthreads_or(mine)) break;
        const unsigned long long epoch = seq * (unsigned long long)(P.max_iter + 1) + m + 1;

        trace_mark(P, m, 0, true);
        FracMax q1, q2;
        bool bad = false;
        int res_b = -1;
        for (;;) {
            const long long t = claim(P.tickets, m);
            if (t >= total_tiles) break;
            const int b = find_inst(P.tile_off, n_inst, t);
            if (b != res_b && res_b >= 0 && staged_active(w, m)) flush_residual(w.I, m, q1, q2, bad);
            stage_warp(w, &P.inst[b], b);
            res_b = b;
            if (!staged_active(w, m)) continue;
            const long long tl = t - w.I.tile_off;
            const int c = (int)(tl / w.I.nvt), vt = (int)(tl % w.I.nvt);
            const double* fn = swap_io ? w.I.f_out : w.I.f_in;
            double* fo = swap_io ? const_cast<double*>(w.I.f_in) : w.I.f_out;
            const bool is32 = (w.cur_active & 2) != 0;  // staged_active above
            const bool ok = is32 ? picard_tile32(w, vt, c, m, epoch, limit, fn, q1, q2, bad)
                                 : picard_tile(w, vt, c, m, epoch, limit, fn, fo, q1, q2, bad);
            if (!ok) {
                if (lane == 0) {
                    atomicOr(&P.head.err, 1 << KEQ_ERR_TIMEOUT);
                    atomicOr(&P.head.err_sticky, 1 << KEQ_ERR_TIMEOUT);
                }
            }
            // row-block arrivals; a completed block is reduced right away
            const TileGeo g = inst_tile(w.I, vt, c, lane);
            fence_acq_rel();
            __syncwarp();
            if (lane == 0)
                rowblock_arrive(w.I.rbcnt + (size_t)m * w.I.nrb, w.I.nx, w.I.n_inner, w.I.nvt, g,
                                w.done_rb);
            __syncwarp();
            const int d0 = w.done_rb[0], d1 = w.done_rb[1];
            // acquire side of a completed block, before the tile's write-back
            // so that the fence does not wait for those stores
            if (d0 >= 0 || d1 >= 0) fence_acq_rel();
            write_tile(w, vt, c, fo, is32);
            if (d0 >= 0 || d1 >= 0) {
                __syncwarp();
                if (d0 >= 0) reduce_block(w, d0, m);
                if (d1 >= 0) reduce_block(w, d1, m);
            }
        }
        if (res_b >= 0 && staged_active(w, m)) flush_residual(w.I, m, q1, q2, bad);
        trace_mark(P, m, 1, false);
        if (!plan_sync(P, G)) return;
    }

    // E: statistics
    if (blockIdx.x == 0 && threadIdx.x == 0) P.head.fresh = 0;
    for (int b = blockIdx.x; b < n_inst; b += G) {
        if (threadIdx.x >= 32) continue;
        const ImpInst& I = P.inst[b];
        if (!inst_enabled(I)) continue;
        const int last = count_leading_ones(I.st, I.picard_iter) - 1;
        if (threadIdx.x != 0) continue;
        keq_step_stats* s = I.stats;
        int aa_applied = 0;
        for (int m = 0; m < last; ++m)
            if (aa_applies(I, m)) ++aa_applied;
        int status = KEQ_OK;
        if (last >= 0 && __ldcg(&I.nonfin[last])) status = KEQ_ERR_NONFINITE;
        if (__ldcg(&P.head.err) & (1 << KEQ_ERR_TIMEOUT)) status = KEQ_ERR_TIMEOUT;
        s->status = status;
        s->iters = last + 1;
        s->aa_applied = aa_applied;
        int n32 = 0;
        while (n32 <= last && fp32_iter(I, n32)) ++n32;
        s->lo_iters = n32;  // implicit: FP32 sweeps of the mixed-precision form
        s->residual = last >= 0 ? ld_cg(&I.res[2 * last + 1]) : 0.0;
        s->std_residual = last >= 0 ? ld_cg(&I.res[2 * last]) : 0.0;
        s->lo_residual = 0.0;
        s->std_lo_residual = 0.0;
        s->max_YI = 0.0;
        s->total_iters += last + 1;
        s->total_steps += 1;
    }
}

constexpr size_t kSmemBytes = sizeof(WarpSmem) * kWarps;

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
    int n_inner, nt_neg, nt_pos, nvt, rows, nchunks, nrb, aa_cols, aa_on;
};

int tile_rows_of(const keq_implicit_params& p) {
    const int r = p.tile_rows;
    return (r == 8 || r == 16 || r == 24 || r == 32) ? r : keq::kRmax;
}

Derived derive(int nx, int nv, int kp, const keq_implicit_params& p) {
    Derived d;
    d.n_inner = nx - 2;
    d.nt_neg = (kp + 31) / 32;
    d.nt_pos = (nv - kp + 31) / 32;
    d.nvt = d.nt_neg + d.nt_pos;
    d.rows = tile_rows_of(p);
    d.nchunks = (d.n_inner + d.rows - 1) / d.rows;
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
    const size_t ntiles = (size_t)d.nvt * d.nchunks;
    double* W = c.take<double>(3 * (size_t)nx);
    double* Wn = c.take<double>(3 * (size_t)nx);
    double* Wc = c.take<double>(4 * (size_t)nx);
    double* Wb = c.take<double>(8);
    double* part = c.take<double>((size_t)d.nvt * d.n_inner * keq::kPartQ);
    double* agg = c.take<double>(ntiles * 64);
    double* inc = c.take<double>(ntiles * 32);
    unsigned long long* flag = c.take<unsigned long long>(ntiles);
    unsigned* rbcnt = c.take<unsigned>((size_t)it * d.nrb);
    double* res = c.take<double>(2 * (size_t)it);
    int* st = c.take<int>(it);
    int* nonfin = c.take<int>(it);
    double* aaG = c.take<double>(d.aa_on ? (size_t)d.aa_cols * 3 * d.n_inner : 1);
    double* aaR = c.take<double>(d.aa_on ? (size_t)d.aa_cols * 3 * d.n_inner : 1);
    double* gpart = c.take<double>(d.aa_on ? (size_t)d.nrb * keq::kMaxPairs : 1);
    double* alpha = c.take<double>((size_t)it * keq::kMaxAACols);
    unsigned* rbdone = c.take<unsigned>(it);
    const bool mixed = p.precision == 1;
    float* fn32 = c.take<float>(mixed ? (size_t)nx * nv : 1);
    float* x32 = c.take<float>(mixed ? (size_t)nx * nv : 1);
    if (I) {
        I->W = W; I->Wn = Wn; I->Wc = Wc; I->Wb = Wb; I->part = part; I->agg = agg;
        I->inc = inc; I->flag = flag; I->rbcnt = rbcnt; I->res = res; I->st = st;
        I->nonfin = nonfin; I->aaG = aaG; I->aaR = aaR; I->gpart = gpart; I->alpha = alpha;
        I->rbdone = rbdone;
        I->fn32 = fn32;
        I->x32 = x32;
    }
    return align_up(c.off, 256);
}

bool valid_params(const keq_implicit_params& p) {
    if (p.picard_iter < 1 || p.picard_iter > 100000) return false;
    if (p.conv_type != 0 && p.conv_type != 1) return false;
    if (p.aa_enable && p.aa_m > keq::kMaxAACols - 1) return false;
    if (p.tile_rows != 0 && p.tile_rows != 8 && p.tile_rows != 16 && p.tile_rows != 24 &&
        p.tile_rows != 32)
        return false;
    if (p.precision != 0 && p.precision != 1) return false;
    if (p.precision == 1 && !(p.mixed_tol >= 0.0)) return false;
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

extern "C" {

keq_status keq_implicit_instance_workspace_size(const keq_grid* grid,
                                                const keq_implicit_params* params,
                                                size_t* bytes) {
    if (!grid || !params || !bytes) return KEQ_ERR_INVALID;
    if (grid->nx < 3 || grid->nv < 1) return KEQ_ERR_INVALID;
    if (!valid_params(*params)) return KEQ_ERR_INVALID;
    const keq_implicit_params p = normalized(*params);
    // the v-tile count depends on where v changes sign (kp): at most
    // nv/32 + 2 tiles; size for the worst case so the query needs no v
    size_t best = 0;
    const int kps[3] = {0, grid->nv, grid->nv / 2 + 1 <= grid->nv ? grid->nv / 2 + 1 : grid->nv};
    for (int q = 0; q < 3; ++q) {
        const size_t b = carve_instance(nullptr, grid->nx, grid->nv, kps[q], p, nullptr);
        if (b > best) best = b;
    }
    const size_t worst =
        carve_instance(nullptr, grid->nx, grid->nv + 64, (grid->nv + 64) / 2, p, nullptr);
    *bytes = worst > best ? worst : best;
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
    plan->kind = KEQ_PLAN_IMPLICIT;
    plan->n_inst = n;
    plan->device = dev_of_buffers;
    plan->inst_bytes = sizeof(ImpInst);
    plan->off_f_in = offsetof(ImpInst, f_in);
    plan->off_f_out = offsetof(ImpInst, f_out);
    plan->kernel = (const void*)keq::implicit_step_kernel;
    plan->smem = keq::kSmemBytes;
    plan->threads = keq::kThreads;
    plan->host_inst.resize(sizeof(ImpInst) * (size_t)n);
    std::vector<ImpInst> host_inst(n);
    std::vector<long long> tile_off(n + 1), rb_off(n + 1);
    long long toff = 0, roff = 0;
    std::vector<double> vh;
    cudaError_t e = cudaSuccess;
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
        int kp = in.grid.kp;
        double vmax = in.grid.v_max;
        if (kp < 0 || kp > nv || !(vmax > 0.0)) {
            vh.resize(nv);
            if (cudaMemcpyAsync(vh.data(), in.grid.v, sizeof(double) * nv, cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                keq_internal_set_cuda_error(cudaGetLastError());
                delete plan;
                return KEQ_ERR_CUDA;
            }
            kp = 0;
            vmax = 0.0;
            for (int j = 0; j < nv; ++j) {
                if (j > 0 && !(vh[j] > vh[j - 1])) {
                    delete plan;
                    return KEQ_ERR_INVALID;  // v must be strictly ascending
                }
                if (!(vh[j] > 0.0)) kp = j + 1;
                vmax = fmax(vmax, fabs(vh[j]));
            }
        }
        const Derived d = derive(nx, nv, kp, p);
        ImpInst I{};
        I.nx = nx; I.nv = nv; I.n_inner = d.n_inner; I.kp = kp;
        I.nt_neg = d.nt_neg; I.nvt = d.nvt; I.nchunks = d.nchunks; I.nrb = d.nrb;
        I.rows = d.rows;
        I.tile_off = toff; I.rb_off = roff;
        I.dx = in.grid.dx; I.dv = in.grid.dv; I.dt = in.dt; I.tau_tilde = in.tau_tilde;
        I.dtdx = in.dt / in.grid.dx;
        I.u_max = 0.95 * vmax;
        I.picard_iter = p.picard_iter; I.conv_type = p.conv_type; I.fixed_iters = p.fixed_iters;
        I.tol = p.picard_tol; I.abs_tol = p.abs_tol;
        I.aa_on = d.aa_on; I.aa_cols = d.aa_cols; I.aa_stride = p.aa_stride;
        I.aa_start = p.aa_start_iter; I.aa_beta = p.aa_beta; I.aa_reg = p.aa_reg;
        I.aa_alpha_max = p.aa_alpha_max;
        I.mixed = p.precision == 1 ? 1 : 0;
        I.tol32 = p.mixed_tol > 0.0 ? p.mixed_tol : 1e-6;
        if (I.tol32 < p.picard_tol) I.tol32 = p.picard_tol;
        I.v = in.grid.v; I.f_in = in.f_in; I.f_out = in.f_out; I.stats = in.stats;
        carve_instance(in.workspace, nx, nv, kp, p, &I);
        host_inst[b] = I;
        tile_off[b] = toff;
        rb_off[b] = roff;
        toff += (long long)d.nvt * d.nchunks;
        roff += d.nrb;
    }
    tile_off[n] = toff;
    rb_off[n] = roff;
    memcpy(plan->host_inst.data(), host_inst.data(), sizeof(ImpInst) * (size_t)n);
    if (toff >= (long long)0xffffffffll) {
        delete plan;
        return KEQ_ERR_INVALID;  // tile tickets are 32-bit
    }

    Carve c{static_cast<char*>(plan_ws), 0};
    PlanDev* dev = c.take<PlanDev>(1);
    ImpInst* dinst = c.take<ImpInst>(n);
    long long* dtoff = c.take<long long>(n + 1);
    long long* droff = c.take<long long>(n + 1);
    unsigned* tickets = c.take<unsigned>(max_iter + 1);
    PlanDev h{};
    h.head.spin_limit = kSpinLimit;
    h.head.fresh = 1;  // the first launch zeroes the stats totals
    h.head.seq = 0ull;
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
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dinst, host_inst.data(), sizeof(ImpInst) * n,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtoff, tile_off.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(droff, rb_off.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        delete plan;
        return KEQ_ERR_CUDA;
    }
    const keq_status gs = keq_internal_plan_grid(plan);
    if (gs != KEQ_OK) {
        delete plan;
        return gs;
    }
    *plan_out = plan;
    return KEQ_OK;
}

keq_status keq_plan_set_enable_mask(keq_plan* plan, const int32_t* mask, keq_stream_t stream) {
    if (!plan || plan->kind != KEQ_PLAN_IMPLICIT) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int b = 0; b < plan->n_inst; ++b) {
        ImpInst* rec = reinterpret_cast<ImpInst*>(plan->host_inst.data()) + b;
        rec->enable = mask ? mask + b : nullptr;
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
