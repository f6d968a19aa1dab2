// keq_holo.cu -- BGK1D1V HOLO (high-order / low-order) time step for a batch
// of independent instances, as ONE persistent cooperative kernel per time
// step on sm_100a.
//
// Replaces core/schemes/BGK1D1V/bgk1d_holo_cuda_kernel.py:416-595 (step, theta
// fixed at 1/2) and its helpers
//   _HO_calculate_moments_face     :31-77
//   _HO_calculate_fluxes_Q         :81-99
//   _compute_explicit_term         :103-131
//   _compute_Y_I_terms             :135-227
//   _LO_calculate_moments_picard   :234-409 with the 3x3 block-tridiagonal
//                                  solve of cuda_kernel/BGK1D1V/lo_blocktridiag/
//                                  block_tridiag_kernel.cu:80-258
//   distribution solve             :526-555 (cuSPARSE gtsv in the reference)
//
// Phases of one launch (| = grid barrier):
//   P0  per-step state; boundary rows of f_out; raw moments of the two
//       boundary rows                                                    |
//   P1  velocity-moment partials of f^n (tiles)                           |
//   P2  row reduction: raw half-range sums R^n, HO-old moments, Maxwellian
//       coefficients; boundary-row Maxwellian sums                        |
//   P3  explicit term E = f + (1-theta) dt (upwind streaming + (M-f)/tau)
//       written for the interior rows, and Maxwellian partials of M_old    |
//   P4  row reduction: old collision moments I_old                        |
//   HO iteration z:
//     A   Maxwellian partials of M(f_z) (compute only), W_m = W_HO        |
//     LO iteration m (partitioned block-tridiagonal solve):
//       L1  per chunk of rows: (m = 0: Q, face moments, consistency terms
//           Y, constant part of the right-hand side) block rows from W_m,
//           local elimination                                             |
//       L2  per instance: reduced interface system by block PCR           |
//       L3  per chunk: recovery, W_full, LO residual                      |
//     C   distribution solve (look-back tiles, keq_tile.cuh) with E and
//         the LO Maxwellian, HO residual, moment partials of f_{z+1};
//         completed row blocks reduce R^{z+1}                              |
//   E   statistics
//
// The LO system's blocks have the structure of the flux Jacobian
// A = [[0,1,0],[u^2,0,0],[0,0,u]] (bgk1d_holo_cuda_kernel.py:317-331), so the
// 3x3 block system splits exactly into a 2x2 block system for (n, nu) and a
// scalar tridiagonal system for U; both are solved here by the partition
// method (chunks of rows eliminated in parallel, interface unknowns by PCR).
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

#include <vector>

#include "keq_common.cuh"
#include "keq_internal.h"
#include "keq_tile.cuh"

namespace keq {
namespace holo {

constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;
constexpr double kTheta = 0.5;
constexpr int kLoChunk = 32;        // rows per LO chunk (one per lane)
constexpr int kMaxLoChunks = 512;   // LO chunks per instance at most (16 groups of 32)

struct HoloInst {
    int nx, nv, n_inner, kp;
    int nt_neg, nvt, nchunks, nrb;
    int rows, lo_len, lo_k, pad0;  // tile rows; LO chunk length and count
    long long tile_off, rb_off, lo_off;
    double dx, dv, dt, tau_tilde, dtdx2;  // dtdx2 = dt / (2 dx)
    int ho_iter, lo_iter, con_terms, flux_cons;
    int sv_down, fixed_ho, fixed_lo, pad1;
    double ho_tol, ho_abs_tol, lo_tol, lo_abs_tol;
    const double* v;
    const double* f_in;
    double* f_out;
    keq_step_stats* stats;
    // workspace carve
    double* E;       // nx*nv : explicit term (interior rows)
    double* part;    // nvt*n_inner*kPartQ : moment / Maxwellian partials
    double* R;       // nx*8 : raw half-range sums of f_z (v>0: 1,v,v^2,v^3 | v<=0: same)
    double* Rn;      // nx*8 : same for f^n
    double* Mco;     // nx*4 : HO-old (u, -0.5/T, n/sqrt(2 pi T), 1/tau)
    double* Wm;      // nx*3 : LO iterate W_m = (n, nu, U)
    double* Who;     // nx*3 : W_HO
    double* Iold;    // nx*3 : old collision moments (1-theta) C_old . w dv
    double* Msum;    // nx*3 : velocity sums of M(f_z) per row: sum M, sum M v, sum M v^2 / 2
    double* Ib;      // 8    : boundary-row Maxwellian sums (2 rows x 3) + spare
    double* Y;       // nx*3 : consistency terms of the current HO iteration
    double* T1;      // nx*3 : W_HO - dt/2dx (F_HO diff) of the current HO iteration
    double* lorow;   // 2*n_inner*13 : y(3) | P(2x2) | P_U | Q(2x2) | Q_U per row, one set per
                     // LO-iteration parity (iteration m writes set m & 1)
    double* loedge;  // lo_k*18 : last-row blocks of each chunk (A,B,C 2x2, D 2 | U: a,b,c,d)
    double* xi;      // lo_k*3 : interface unknowns
    double* Wlo;     // 3*nx : n_lo | u_lo | T_lo of the last LO solve (state.n/u/T)
    double* agg;     // ntiles*64 : tile maps (distribution pass)
    double* inc;     // ntiles*32 : tile carries
    unsigned long long* flag;  // ntiles : look-back flags
    unsigned* rbcnt; // ho_iter*nrb : row-block arrivals of the distribution pass
    double* ho_red;  // ho_iter*4 : HO std residual, max |df|, max ref, max |Y|
    double* lo_hist; // ho_iter*lo_iter*2 : LO max |dW|, std residual
    int* ho_run;     // ho_iter : 1 if HO iteration z ran
    int* lo_run;     // ho_iter*lo_iter : 1 if LO iteration m of HO iteration z ran
    int* nonfin;     // ho_iter : non-finite flag of f_{z+1}
    double* misc;    // 8 : [0] max |f^n| over the boundary rows, [1] max |Y| of the boundary rows
};

struct HoloDev {
    PlanHead head;
    int n_inst;
    int max_ho, max_lo;
    int pad;
    long long total_tiles, total_rb, total_lo;
    HoloInst* inst;
    long long* tile_off;
    long long* rb_off;
    long long* lo_off;
    unsigned* tickets;  // max_ho : tile claims of the distribution pass
};

struct WarpSmem {
    HoloInst I;
    double a[kRmax][33];
    double o[kRmax][32];
    double coef[kRmax][4];
    double vv[32];
    int cur_b, pad;
    int done_rb[2];
};

// LO chunk scratch (per warp, aliasing the tile buffers of WarpSmem).
struct LoRow {
    double A[4], B[4], C[4], D[2];  // (n, nu) blocks, row-major 2x2
    double a, b, c, d;              // U
    double cu;                      // U: C' of the forward sweep
};

__device__ __forceinline__ TileGeo inst_tile(const HoloInst& I, int vt, int c, int lane) {
    return tile_geo(I.nt_neg, I.kp, I.nv, I.n_inner, I.rows, vt, c, lane);
}

__device__ __forceinline__ void stage_warp(WarpSmem& w, const HoloInst* src, int b) {
    if (w.cur_b != b) {
        __syncwarp();
        const int lane = threadIdx.x & 31;
        const int* s = reinterpret_cast<const int*>(src);
        int* d = reinterpret_cast<int*>(&w.I);
        for (int q = lane; q < (int)(sizeof(HoloInst) / sizeof(int)); q += 32) d[q] = __ldg(s + q);
        __syncwarp();
        if (lane == 0) w.cur_b = b;
    }
    __syncwarp();
}

template <int STRIDE>
__device__ __forceinline__ void stage_rows_h(double (*dst)[STRIDE], const double* __restrict__ src,
                                             const TileGeo& g, int nx, int nv) {
    const int lane = threadIdx.x & 31;
    if (!g.lane_ok) return;
#pragma unroll 8
    for (int r = 0; r < g.nrows; ++r)
        cp_async8(&dst[r][lane], src + (size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j);
}

__device__ __forceinline__ void store_partials_h(WarpSmem& w, const TileGeo& g, int vt) {
    const HoloInst& I = w.I;
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

// calculate_moments (bgk1d_utils/general/bgk1d_compute_moments.py:7-17) from
// raw half-range sums: n = sum f dv, u = (sum f v dv)/n, T = (sum f v^2 dv)/n - u^2.
struct Mom {
    double n, u, T, s1, s2, s3;  // s_k = sum f v^k dv
};
__device__ __forceinline__ Mom mom_of(const double* R8, double dv) {
    Mom m;
    m.n = (R8[0] + R8[4]) * dv;
    m.s1 = (R8[1] + R8[5]) * dv;
    m.s2 = (R8[2] + R8[6]) * dv;
    m.s3 = (R8[3] + R8[7]) * dv;
    m.u = m.s1 / m.n;
    m.T = m.s2 / m.n - m.u * m.u;
    return m;
}
// Q = 1/2 sum (v-u)^3 f dv (_HO_calculate_fluxes_Q, :81-99) by the binomial
// expansion of the raw moments.
__device__ __forceinline__ double q_of(const Mom& m) {
    const double u = m.u;
    return 0.5 * (m.s3 - 3.0 * u * m.s2 + 3.0 * u * u * m.s1 - u * u * u * m.n);
}

// ---- P1: moment partials of f^n --------------------------------------------
__device__ __noinline__ void moments_tile(WarpSmem& w, int vt, int c, const double* __restrict__ f) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    stage_rows_h<33>(w.a, f, g, I.nx, I.nv);
    cp_async_commit();
    w.vv[lane] = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    cp_async_wait_all();
    if (!g.lane_ok)
        for (int r = 0; r < g.nrows; ++r) w.a[r][lane] = 0.0;
    store_partials_h(w, g, vt);
}

// Raw half-range sums of interior row k (v <= 0 tiles, then v > 0 tiles).
__device__ __forceinline__ void half_sums(const HoloInst& I, int k, double* R8) {
    double sn[4], sp[4];
    sum_partials4(I.part, 0, I.nt_neg, I.n_inner, k, sn);
    sum_partials4(I.part, I.nt_neg, I.nvt, I.n_inner, k, sp);
    R8[0] = sp[0]; R8[1] = sp[1]; R8[2] = sp[2]; R8[3] = sp[3];
    R8[4] = sn[0]; R8[5] = sn[1]; R8[6] = sn[2]; R8[7] = sn[3];
}

// Maxwellian coefficients of (n, u, T) (bgk1d_maxwellian.py:7-33) and 1/tau.
__device__ __forceinline__ void mc_of(const Mom& m, double tau_tilde, double* c4) {
    const double sT = sqrt(m.T);
    c4[0] = m.u;
    c4[1] = -(0.5 / m.T);
    c4[2] = (m.n * kInvSqrt2Pi) / sT;
    c4[3] = (m.n * sT) / tau_tilde;  // 1/tau, tau = tau_tilde / (n sqrt(T))
}

// Sum over the velocities of a Maxwellian times (1, v, v^2/2), one warp.
__device__ __forceinline__ void maxwell_sums_row(const double* v, int nv, const double* c4,
                                                 double* s3) {
    const int lane = threadIdx.x & 31;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = lane; j < nv; j += 32) {
        const double vj = __ldg(&v[j]);
        const double d = vj - c4[0];
        const double M = c4[2] * exp_nonpos(d * d * c4[1]);
        a0 += M;
        a1 += M * vj;
        a2 += M * vj * vj;
    }
    s3[0] = warp_sum(a0);
    s3[1] = warp_sum(a1);
    s3[2] = 0.5 * warp_sum(a2);
}

// ---- P3: explicit term and old-Maxwellian partials (one tile) --------------
__device__ __noinline__ void explicit_tile(WarpSmem& w, int vt, int c, const double* __restrict__ fn) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    const int nx = I.nx, nv = I.nv;
    stage_rows_h<33>(w.a, fn, g, nx, nv);
    cp_async_commit();
    const double vj = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    w.vv[lane] = vj;
    if (lane < g.nrows) {
        const int i = scan_row(nx, g.pos, g.s0 + lane);
        const double2 q01 = __ldcg(reinterpret_cast<const double2*>(&I.Mco[4 * (size_t)i]));
        const double2 q23 = __ldcg(reinterpret_cast<const double2*>(&I.Mco[4 * (size_t)i + 2]));
        w.coef[lane][0] = q01.x; w.coef[lane][1] = q01.y; w.coef[lane][2] = q23.x;
        w.coef[lane][3] = q23.y;
    }
    // upwind neighbour of scan position s0 (scan position s0-1; the
    // boundary row for s0 = 0)
    double prev = 0.0;
    if (g.lane_ok) {
        const int ip = g.pos ? scan_row(nx, true, g.s0) - 1 : scan_row(nx, false, g.s0) + 1;
        prev = __ldg(&fn[(size_t)ip * nv + g.j]);
    }
    cp_async_wait_all();
    __syncwarp();
    const double vc = (-vj) / I.dx;
    const double a = (1.0 - kTheta) * I.dt;
    for (int r = 0; r < g.nrows; ++r) {
        const double f = g.lane_ok ? w.a[r][lane] : 0.0;
        const double d = vj - w.coef[r][0];
        const double M = w.coef[r][2] * exp_nonpos(d * d * w.coef[r][1]);
        // bgk1d_compute_streaming.py: (f_i - f_{i-1}) (-v/dx) for v > 0,
        // (f_{i+1} - f_i) (-v/dx) for v <= 0
        const double st = g.pos ? (f - prev) * vc : (prev - f) * vc;
        const double col = (M - f) * w.coef[r][3];
        const double e = f + a * (st + col);
        if (g.lane_ok) I.E[(size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j] = e;
        prev = f;
        w.a[r][lane] = g.lane_ok ? M : 0.0;  // Maxwellian partials for I_old
    }
    store_partials_h(w, g, vt);
}

// ---- A: velocity sums of M(f_z) for one interior row (one warp) -----------
// The Maxwellian of the row's moments (bgk1d_maxwellian.py:7-33) summed over
// the velocity grid against 1, v and v^2/2, lane-strided with a fixed warp
// reduction; lane 0 stores the three sums.
__device__ __noinline__ void maxwell_row(WarpSmem& w, int k) {
    const HoloInst& I = w.I;
    const int i = k + 1;
    double R8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) R8[q] = __ldcg(&I.R[8 * (size_t)i + q]);
    const Mom m = mom_of(R8, I.dv);
    double c4[4];
    mc_of(m, I.tau_tilde, c4);
    double s3[3];
    maxwell_sums_row(I.v, I.nv, c4, s3);
    if ((threadIdx.x & 31) == 0) {
        I.Msum[3 * (size_t)i + 0] = s3[0];
        I.Msum[3 * (size_t)i + 1] = s3[1];
        I.Msum[3 * (size_t)i + 2] = s3[2];
    }
}

// ---- LO: structured blocks -----------------------------------------------------
// u*, P* of a cell from W = (n, nu, U) (:293-303): den = n + 1e-30,
// u = nu/den, T = max(2 (U/den - u^2/2), 1e-30), P = n T.
__device__ __forceinline__ void star_of(const double* W3, double& us, double& Ps) {
    const double den = W3[0] + 1e-30;
    us = W3[1] / den;
    double Ts = 2.0 * (W3[2] / den - 0.5 * us * us);
    Ts = (Ts != Ts || Ts >= 1e-30) ? Ts : 1e-30;
    Ps = W3[0] * Ts;
}

__device__ __forceinline__ bool inv2(const double* M, double* Mi) {
    const double det = M[0] * M[3] - M[1] * M[2];
    if (!(fabs(det) >= 1e-30)) {
        Mi[0] = Mi[1] = Mi[2] = Mi[3] = 0.0;
        return false;
    }
    const double id = 1.0 / det;
    Mi[0] = M[3] * id;
    Mi[1] = -M[1] * id;
    Mi[2] = -M[2] * id;
    Mi[3] = M[0] * id;
    return true;
}
__device__ __forceinline__ void mm2(const double* A, const double* B, double* C) {
    C[0] = A[0] * B[0] + A[1] * B[2];
    C[1] = A[0] * B[1] + A[1] * B[3];
    C[2] = A[2] * B[0] + A[3] * B[2];
    C[3] = A[2] * B[1] + A[3] * B[3];
}
__device__ __forceinline__ void mv2(const double* A, const double* x, double* y) {
    y[0] = A[0] * x[0] + A[1] * x[1];
    y[1] = A[2] * x[0] + A[3] * x[1];
}
__device__ __forceinline__ double rcp_or0(double d) { return fabs(d) >= 1e-30 ? 1.0 / d : 0.0; }

// Block row of interior row k (cell i = k+1) from W_m: faces L (i-1, i) and
// R (i, i+1); AA = -c4 A_L (0 at k = 0), CC = c4 A_R (0 at the last row),
// BB = I + c4 (A_R - A_L), DD = ((T1 - c2 (b_R - b_L)) + Y).
__device__ __forceinline__ void lo_row_w(const HoloInst& I, int k, const double* Wl,
                                         const double* Wc, const double* Wr, LoRow& r) {
    const int i = k + 1;
    double uL, PL, uC, PC, uR, PR;
    star_of(Wl, uL, PL);
    star_of(Wc, uC, PC);
    star_of(Wr, uR, PR);
    const double uhL = 0.5 * (uL + uC), PhL = 0.5 * (PL + PC);
    const double uhR = 0.5 * (uC + uR), PhR = 0.5 * (PC + PR);
    const double c4 = I.dt / (4.0 * I.dx), c2 = I.dt / (2.0 * I.dx);
    const double aL = (k >= 1) ? 1.0 : 0.0, aR = (k <= I.n_inner - 2) ? 1.0 : 0.0;
    // A_int = [[0,1,0],[uh^2,0,0],[0,0,uh]]
    const double uL2 = uhL * uhL, uR2 = uhR * uhR;
    r.A[0] = 0.0; r.A[1] = aL * (1.0 * (-c4)); r.A[2] = aL * (uL2 * (-c4)); r.A[3] = 0.0;
    r.C[0] = 0.0; r.C[1] = aR * (1.0 * c4); r.C[2] = aR * (uR2 * c4); r.C[3] = 0.0;
    r.B[0] = (0.0 - 0.0) * c4 + 1.0;
    r.B[1] = (1.0 - 1.0) * c4;
    r.B[2] = (uR2 - uL2) * c4;
    r.B[3] = (0.0 - 0.0) * c4 + 1.0;
    r.a = aL * (uhL * (-c4));
    r.c = aR * (uhR * c4);
    r.b = (uhR - uhL) * c4 + 1.0;
    // b_int = (0, Ph, uh Ph)
    const double bd0 = 0.0 - 0.0, bd1 = PhR - PhL, bd2 = uhR * PhR - uhL * PhL;
    const double* T1 = I.T1 + 3 * (size_t)i;
    const double* Y = I.Y + 3 * (size_t)i;
    r.D[0] = __dadd_rn(__dadd_rn(__ldcg(&T1[0]), __dmul_rn(-c2, bd0)), __ldcg(&Y[0]));
    r.D[1] = __dadd_rn(__dadd_rn(__ldcg(&T1[1]), __dmul_rn(-c2, bd1)), __ldcg(&Y[1]));
    r.d = __dadd_rn(__dadd_rn(__ldcg(&T1[2]), __dmul_rn(-c2, bd2)), __ldcg(&Y[2]));
}

// The same from the LO iterate in I.Wm (rows i-1, i, i+1).
__device__ __forceinline__ void lo_row(const HoloInst& I, int k, LoRow& r) {
    const int i = k + 1;
    lo_row_w(I, k, I.Wm + 3 * (size_t)(i - 1), I.Wm + 3 * (size_t)i, I.Wm + 3 * (size_t)(i + 1),
             r);
}

// Constant part of the LO right-hand side and the consistency terms Y of row
// i for HO iteration z (m = 0), from the raw sums of f_z (rows i-1, i, i+1),
// the Maxwellian partials of M(f_z) and I_old.  Returns max |Y_i|.
__device__ __noinline__ double lo_prep_row(const HoloInst& I, int k) {
    const int i = k + 1, nx = I.nx;
    const double dv = I.dv, dt = I.dt, dx = I.dx;
    const double c2 = dt / (2.0 * dx);
    Mom m3[3];
    double Q3[3];
    double Rr[3][8];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const double* src = I.R + 8 * (size_t)(i - 1 + t);
#pragma unroll
        for (int q = 0; q < 8; ++q) Rr[t][q] = __ldcg(&src[q]);
        m3[t] = mom_of(Rr[t], dv);
        Q3[t] = q_of(m3[t]);
    }
    // face moments S(f) of faces f = i-1 (L) and i (R) (_HO_calculate_moments_face):
    // upwind state: v > 0 from the left cell, v <= 0 from the right cell.
    // With the consistency terms off the reference keeps the face moments of
    // the step's f^n (:459-462); with them on, _compute_Y_I_terms replaces
    // them by those of f_z (:163-165).
    double Rs[3][8];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const double* src = (I.con_terms ? I.R : I.Rn) + 8 * (size_t)(i - 1 + t);
#pragma unroll
        for (int q = 0; q < 8; ++q) Rs[t][q] = I.con_terms ? Rr[t][q] : __ldcg(&src[q]);
    }
    double S[2][3];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const double* Lr = Rs[s];
        const double* Rg = Rs[s + 1];
        if (I.sv_down) {
            S[s][0] = (Lr[0] + Rg[4]) * dv;
            S[s][1] = (Lr[1] + Rg[5]) * dv;
            S[s][2] = 0.5 * ((Lr[2] + Rg[6]) * dv);
        } else {
            S[s][0] = (Lr[1] + Rg[5]) * dv;
            S[s][1] = (Lr[2] + Rg[6]) * dv;
            S[s][2] = 0.5 * ((Lr[3] + Rg[7]) * dv);
        }
    }
    double y[3] = {0.0, 0.0, 0.0};
    if (I.con_terms) {
        if (I.flux_cons) {
            double g[2][3];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const Mom& a0 = m3[s];
                const Mom& a1 = m3[s + 1];
                const double P0 = a0.n * a0.T, P1 = a1.n * a1.T;
                const double nu0 = a0.n * a0.u, nu1 = a1.n * a1.u;
                const double U0 = 0.5 * a0.n * (a0.u * a0.u + a0.T);
                const double U1 = 0.5 * a1.n * (a1.u * a1.u + a1.T);
                const double mf0 = nu0 * nu0 / (a0.n + 1e-30) + P0;
                const double mf1 = nu1 * nu1 / (a1.n + 1e-30) + P1;
                const double ef0 = (U0 + P0) * a0.u + Q3[s];
                const double ef1 = (U1 + P1) * a1.u + Q3[s + 1];
                g[s][0] = -S[s][0] + 0.5 * (nu0 + nu1);
                g[s][1] = -S[s][1] + 0.5 * (mf0 + mf1);
                g[s][2] = -S[s][2] + 0.5 * (ef0 + ef1);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) y[c] = dt * ((g[1][c] - g[0][c]) / dx);
        }
        // collision consistency: theta C_new + (1-theta) C_old moments
        const Mom& mn = m3[1];
        const double inv_tau_new = (mn.n * sqrt(mn.T)) / I.tau_tilde;
        const double smw[3] = {__ldcg(&I.Msum[3 * (size_t)i]) * dv,
                               __ldcg(&I.Msum[3 * (size_t)i + 1]) * dv,
                               __ldcg(&I.Msum[3 * (size_t)i + 2]) * dv};
        const double sfw[3] = {mn.n, mn.s1, 0.5 * mn.s2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double cm = kTheta * ((smw[c] - sfw[c]) * inv_tau_new) + __ldcg(&I.Iold[3 * (size_t)i + c]);
            y[c] = y[c] + dt * cm;
        }
    }
    // constant part of DD: W_HO - dt/2dx (F_HO(R) - F_HO(L)), F_HO = [S1, S2, S3 + 2 Q_half]
    const double QhL = 0.5 * (Q3[0] + Q3[1]), QhR = 0.5 * (Q3[1] + Q3[2]);
    const double Fd[3] = {S[1][0] - S[0][0], S[1][1] - S[0][1],
                          (S[1][2] + 2.0 * QhR) - (S[0][2] + 2.0 * QhL)};
    double mx = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        I.T1[3 * (size_t)i + c] = __dadd_rn(__ldcg(&I.Who[3 * (size_t)i + c]), __dmul_rn(-c2, Fd[c]));
        I.Y[3 * (size_t)i + c] = y[c];
        mx = nan_max(mx, fabs(y[c]));
    }
    (void)nx;
    return mx;
}

// ---- LO: warp-parallel block PCR ---------------------------------------------
// One block row per lane of a block-tridiagonal system with 2x2 blocks for
// (n, nu) and a scalar system for U:
//     A x_{l-1} + B x_l + C x_{l+1} = R,   a u_{l-1} + b u_l + c u_{l+1} = r,
// R holding 5 right-hand-side columns (2 x 5, row-major) and r 3.  Parallel
// cyclic reduction over the lanes: at stride d every row eliminates its
// couplings to rows l-d and l+d with their (pre-step) blocks, fetched by
// shuffles; after log2(L) steps every row is decoupled and B^{-1} R, r / b
// are the solution columns.  Lanes >= L carry identity rows.
struct PcrRow {
    double A[4], B[4], C[4], R[10];
    double a, b, c, r[3];
};

__device__ __forceinline__ double shup(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ double shdn(double v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

__device__ __forceinline__ void identity_row(PcrRow& q) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        q.A[k] = 0.0;
        q.C[k] = 0.0;
        q.B[k] = (k == 0 || k == 3) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) q.R[k] = 0.0;
    q.a = 0.0; q.b = 1.0; q.c = 0.0;
    q.r[0] = q.r[1] = q.r[2] = 0.0;
}

__device__ __forceinline__ void warp_pcr(PcrRow& q, int L) {
    const int lane = threadIdx.x & 31;
#pragma unroll 1
    for (int d = 1; d < L; d <<= 1) {
        double Bi[4];
        inv2(q.B, Bi);
        const double bi = rcp_or0(q.b);
        // Early exit once every row is decoupled to below double rounding:
        // |B^{-1}|_inf (|A|_inf + |C|_inf) <= 2^-60 and the same for the
        // scalar rows.  The couplings of an interface system are products of
        // a chunk's 31 row couplings, so this usually holds before the first
        // step there.  The test is warp-uniform and depends on the data only.
        {
            const double nbi = fmax(fabs(Bi[0]) + fabs(Bi[1]), fabs(Bi[2]) + fabs(Bi[3]));
            const double nac = fmax(fabs(q.A[0]) + fabs(q.A[1]), fabs(q.A[2]) + fabs(q.A[3])) +
                               fmax(fabs(q.C[0]) + fabs(q.C[1]), fabs(q.C[2]) + fabs(q.C[3]));
            const double kTiny = 8.673617379884035e-19;  // 2^-60
            const bool dec = nbi * nac <= kTiny && fabs(bi) * (fabs(q.a) + fabs(q.c)) <= kTiny;
            if (__all_sync(0xffffffffu, dec || lane >= L)) break;
        }
        const bool has_lo = lane >= d && lane < L, has_hi = lane + d < L;
        double nA[4], nC[4], dB[4], nR[10];
        double na, nc, db, nr[3];
        // lower neighbour: alpha = -A B_lo^{-1}
        {
            double t[4], al[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shup(Bi[k], d);
            mm2(q.A, t, al);
#pragma unroll
            for (int k = 0; k < 4; ++k) al[k] = has_lo ? -al[k] : 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shup(q.A[k], d);
            mm2(al, t, nA);
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shup(q.C[k], d);
            mm2(al, t, dB);
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                const double r0 = shup(q.R[j], d), r1 = shup(q.R[5 + j], d);
                nR[j] = q.R[j] + (al[0] * r0 + al[1] * r1);
                nR[5 + j] = q.R[5 + j] + (al[2] * r0 + al[3] * r1);
            }
            const double bl = shup(bi, d);  // every lane shuffles; the mask is the full warp
            const double a1 = has_lo ? -q.a * bl : 0.0;
            na = a1 * shup(q.a, d);
            db = a1 * shup(q.c, d);
#pragma unroll
            for (int j = 0; j < 3; ++j) nr[j] = q.r[j] + a1 * shup(q.r[j], d);
        }
        // upper neighbour: gamma = -C B_hi^{-1}
        {
            double t[4], ga[4], u[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shdn(Bi[k], d);
            mm2(q.C, t, ga);
#pragma unroll
            for (int k = 0; k < 4; ++k) ga[k] = has_hi ? -ga[k] : 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shdn(q.C[k], d);
            mm2(ga, t, nC);
#pragma unroll
            for (int k = 0; k < 4; ++k) t[k] = shdn(q.A[k], d);
            mm2(ga, t, u);
#pragma unroll
            for (int k = 0; k < 4; ++k) dB[k] += u[k];
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                const double r0 = shdn(q.R[j], d), r1 = shdn(q.R[5 + j], d);
                nR[j] += ga[0] * r0 + ga[1] * r1;
                nR[5 + j] += ga[2] * r0 + ga[3] * r1;
            }
            const double bh = shdn(bi, d);
            const double g1 = has_hi ? -q.c * bh : 0.0;
            nc = g1 * shdn(q.c, d);
            db += g1 * shdn(q.a, d);
#pragma unroll
            for (int j = 0; j < 3; ++j) nr[j] += g1 * shdn(q.r[j], d);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            q.A[k] = nA[k];
            q.C[k] = nC[k];
            q.B[k] += dB[k];
        }
#pragma unroll
        for (int k = 0; k < 10; ++k) q.R[k] = nR[k];
        q.a = na;
        q.c = nc;
        q.b += db;
#pragma unroll
        for (int j = 0; j < 3; ++j) q.r[j] = nr[j];
    }
    double Bi[4];
    inv2(q.B, Bi);
    double nR[10];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        nR[j] = Bi[0] * q.R[j] + Bi[1] * q.R[5 + j];
        nR[5 + j] = Bi[2] * q.R[j] + Bi[3] * q.R[5 + j];
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) q.R[k] = nR[k];
    const double bi = rcp_or0(q.b);
#pragma unroll
    for (int j = 0; j < 3; ++j) q.r[j] *= bi;
}

// Solution columns [y | P | Q] of a PCR row as the 13-value representation
// y(2) y_U | P(2x2) P_U | Q(2x2) Q_U of x = y + P x_left + Q x_right.
__device__ __forceinline__ void rep_of(const PcrRow& q, double* o) {
    o[0] = q.R[0]; o[1] = q.R[5]; o[2] = q.r[0];
    o[3] = q.R[1]; o[4] = q.R[2]; o[5] = q.R[6]; o[6] = q.R[7]; o[7] = q.r[1];
    o[8] = q.R[3]; o[9] = q.R[4]; o[10] = q.R[8]; o[11] = q.R[9]; o[12] = q.r[2];
}

// Local system of L rows (lane l = row l, couplings A_l, C_l) with the
// left coupling of row 0 and the right coupling of row L-1 moved to the
// right-hand side as the P and Q columns (D, -A_0 e_0, -C_{L-1} e_{L-1}).
__device__ __forceinline__ void local_rows(PcrRow& q, const double* A, const double* B,
                                           const double* C, const double* D, double a, double b,
                                           double c, double d, int l, int L) {
    if (l >= L) {
        identity_row(q);
        return;
    }
    const bool first = l == 0, last = l == L - 1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        q.A[k] = first ? 0.0 : A[k];
        q.B[k] = B[k];
        q.C[k] = last ? 0.0 : C[k];
    }
    q.R[0] = D[0];
    q.R[5] = D[1];
    q.R[1] = first ? -A[0] : 0.0; q.R[2] = first ? -A[1] : 0.0;
    q.R[6] = first ? -A[2] : 0.0; q.R[7] = first ? -A[3] : 0.0;
    q.R[3] = last ? -C[0] : 0.0; q.R[4] = last ? -C[1] : 0.0;
    q.R[8] = last ? -C[2] : 0.0; q.R[9] = last ? -C[3] : 0.0;
    q.a = first ? 0.0 : a;
    q.b = b;
    q.c = last ? 0.0 : c;
    q.r[0] = d;
    q.r[1] = first ? -a : 0.0;
    q.r[2] = last ? -c : 0.0;
}

// L1: block rows of one LO chunk (lane = row; rows s..e, e the chunk's
// interface row), the warp-parallel solve of the local rows s..e-1 into the
// representation x_r = y_r + P_r xi_{k-1} + Q_r xi_k (row e: y = 0, P = 0,
// Q = I) in lorow, and the interface row's blocks in loedge.
__device__ __forceinline__ void lo_chunk_solve(const HoloInst& I, int kc, const LoRow& L,
                                               double* __restrict__ lorow) {
    const int lane = threadIdx.x & 31;
    const int s = kc * I.lo_len;
    const int e = (s + I.lo_len < I.n_inner ? s + I.lo_len : I.n_inner) - 1;
    const int len = e - s + 1;
    const int nloc = len - 1;  // rows s..e-1 solved locally
    if (lane == nloc) {
        double* ed = I.loedge + (size_t)kc * 18;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ed[k] = L.A[k];
            ed[4 + k] = L.B[k];
            ed[8 + k] = L.C[k];
        }
        ed[12] = L.D[0]; ed[13] = L.D[1];
        ed[14] = L.a; ed[15] = L.b; ed[16] = L.c; ed[17] = L.d;
    }
    PcrRow q;
    local_rows(q, L.A, L.B, L.C, L.D, L.a, L.b, L.c, L.d, lane, nloc);
    warp_pcr(q, nloc);
    if (lane < len) {
        double o[13];
        if (lane < nloc) {
            rep_of(q, o);
        } else {
#pragma unroll
            for (int k = 0; k < 13; ++k) o[k] = 0.0;
            o[8] = 1.0; o[11] = 1.0; o[12] = 1.0;
        }
        double* dst = lorow + 13 * (size_t)(s + lane);
#pragma unroll
        for (int k = 0; k < 13; ++k) dst[k] = o[k];
    }
}

// L1 of the first LO iteration: block rows from W_m = W_HO in I.Wm, solved
// into the representation set `lorow`.
__device__ __noinline__ void lo_chunk_eliminate(WarpSmem& w, int kc, double* __restrict__ lorow) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int s = kc * I.lo_len;
    const int e = (s + I.lo_len < I.n_inner ? s + I.lo_len : I.n_inner) - 1;
    LoRow L{};
    if (lane <= e - s) lo_row(I, s + lane, L);
    lo_chunk_solve(I, kc, L, lorow);
}

// Representation (y, P, Q) of a row: from lorow, or the identity forms
// (y = 0, P = I, Q = 0: the previous interface itself; all zero: absent).
__device__ __forceinline__ void rep_load(const double* lr, double* o13) {
#pragma unroll
    for (int q = 0; q < 13; ++q) o13[q] = __ldcg(&lr[q]);
}

// Interface row of chunk k (its last row e):
//   alpha_k xi_{k-1} + beta_k xi_k + gamma_k xi_{k+1} = delta_k,
//   alpha = A_e P_{e-1}, beta = B_e + A_e Q_{e-1} + C_e P_{s'},
//   gamma = C_e Q_{s'}, delta = D_e - A_e y_{e-1} - C_e y_{s'}
// (s' the first row of chunk k+1), the same for the U scalar.
__device__ __forceinline__ void interface_row(const HoloInst& I, const double* lorow, int k,
                                              double* al, double* be, double* ga, double* de,
                                              double* s4) {
    const int s = k * I.lo_len;
    const int e = (s + I.lo_len < I.n_inner ? s + I.lo_len : I.n_inner) - 1;
    double ed[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) ed[q] = __ldcg(&I.loedge[(size_t)k * 18 + q]);
    const double* A = ed; const double* B = ed + 4; const double* C = ed + 8;
    const double* D = ed + 12;
    double pm[13], nx_[13];
    if (e > s) {
        rep_load(lorow + 13 * (size_t)(e - 1), pm);
    } else {
#pragma unroll
        for (int q = 0; q < 13; ++q) pm[q] = 0.0;
        pm[3] = 1.0; pm[6] = 1.0; pm[7] = 1.0;
    }
    if (k + 1 < I.lo_k) {
        rep_load(lorow + 13 * (size_t)(e + 1), nx_);
    } else {
#pragma unroll
        for (int q = 0; q < 13; ++q) nx_[q] = 0.0;
    }
    double T4[4], U4[4], t2[2], u2[2];
    mm2(A, pm + 3, al);
    mm2(A, pm + 8, T4);
    mm2(C, nx_ + 3, U4);
#pragma unroll
    for (int q = 0; q < 4; ++q) be[q] = B[q] + T4[q] + U4[q];
    mm2(C, nx_ + 8, ga);
    mv2(A, pm, t2);
    mv2(C, nx_, u2);
    de[0] = D[0] - t2[0] - u2[0];
    de[1] = D[1] - t2[1] - u2[1];
    const double a = ed[14], b = ed[15], c = ed[16], d = ed[17];
    s4[0] = a * pm[7];
    s4[1] = b + a * pm[12] + c * nx_[7];
    s4[2] = c * nx_[12];
    s4[3] = d - a * pm[2] - c * nx_[2];
}

// L2: the interface system of the K = lo_k chunks, one CTA per instance.
// The interface rows are split into groups of 32; each group is solved by
// warp PCR into xi_k = y_k + P_k X_{g-1} + Q_k X_g in terms of the group
// interfaces X_g (the last interface of every group), whose own system (at
// most 32 unknowns) is solved by warp 0 the same way; then every xi_k is
// recovered into I.xi.
struct GroupRec {
    double rep_prev[13];  // representation of the group row before the last
    double rep_first[13]; // representation of the group's first row
    double al[4], be[4], ga[4], de[2], s4[4];  // the group's last interface row
};

__device__ __noinline__ void lo_reduced_solve(const HoloInst& I, const double* lorow,
                                              unsigned char* smem) {
    const int K = I.lo_k;
    const int G = (K + 31) / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    GroupRec* grec = reinterpret_cast<GroupRec*>(smem);
    double* reps = reinterpret_cast<double*>(smem + sizeof(GroupRec) * G);  // K x 13
    double* X = reps + 13 * (size_t)K;                                      // G x 3
    for (int g = warp; g < G; g += kWarps) {
        const int k0 = 32 * g;
        const int len = (K - k0) < 32 ? (K - k0) : 32;
        const int nloc = len - 1;
        const int k = k0 + lane;
        double al[4] = {0, 0, 0, 0}, be[4] = {1, 0, 0, 1}, ga[4] = {0, 0, 0, 0}, de[2] = {0, 0};
        double s4[4] = {0.0, 1.0, 0.0, 0.0};
        if (lane < len) interface_row(I, lorow, k, al, be, ga, de, s4);
        PcrRow q;
        local_rows(q, al, be, ga, de, s4[0], s4[1], s4[2], s4[3], lane, nloc);
        warp_pcr(q, nloc);
        double o[13];
        if (lane < nloc) {
            rep_of(q, o);
        } else {
#pragma unroll
            for (int t = 0; t < 13; ++t) o[t] = 0.0;
            o[8] = 1.0; o[11] = 1.0; o[12] = 1.0;
        }
        if (lane < len) {
#pragma unroll
            for (int t = 0; t < 13; ++t) reps[13 * (size_t)k + t] = o[t];
        }
        if (lane == nloc) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                grec[g].al[t] = al[t];
                grec[g].be[t] = be[t];
                grec[g].ga[t] = ga[t];
                grec[g].s4[t] = s4[t];
            }
            grec[g].de[0] = de[0];
            grec[g].de[1] = de[1];
        }
        __syncwarp();
        if (lane < 13) {
            grec[g].rep_first[lane] = reps[13 * (size_t)k0 + lane];
            grec[g].rep_prev[lane] = (nloc >= 1) ? reps[13 * (size_t)(k0 + nloc - 1) + lane]
                                                 : ((lane == 3 || lane == 6 || lane == 7) ? 1.0 : 0.0);
        }
    }
    __syncthreads();
    // group interfaces: the same interface-row construction one level up
    if (warp == 0) {
        double A[4] = {0, 0, 0, 0}, B[4] = {1, 0, 0, 1}, C[4] = {0, 0, 0, 0}, D[2] = {0, 0};
        double a = 0.0, b = 1.0, c = 0.0, d = 0.0;
        if (lane < G) {
            const GroupRec& gr = grec[lane];
            const double* pm = gr.rep_prev;
            double nx_[13];
#pragma unroll
            for (int t = 0; t < 13; ++t) nx_[t] = (lane + 1 < G) ? grec[lane + 1].rep_first[t] : 0.0;
            double T4[4], U4[4], t2[2], u2[2];
            mm2(gr.al, pm + 3, A);
            mm2(gr.al, pm + 8, T4);
            mm2(gr.ga, nx_ + 3, U4);
#pragma unroll
            for (int t = 0; t < 4; ++t) B[t] = gr.be[t] + T4[t] + U4[t];
            mm2(gr.ga, nx_ + 8, C);
            mv2(gr.al, pm, t2);
            mv2(gr.ga, nx_, u2);
            D[0] = gr.de[0] - t2[0] - u2[0];
            D[1] = gr.de[1] - t2[1] - u2[1];
            a = gr.s4[0] * pm[7];
            b = gr.s4[1] + gr.s4[0] * pm[12] + gr.s4[2] * nx_[7];
            c = gr.s4[2] * nx_[12];
            d = gr.s4[3] - gr.s4[0] * pm[2] - gr.s4[2] * nx_[2];
        }
        PcrRow q;
        if (lane < G) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                q.A[t] = A[t];
                q.B[t] = B[t];
                q.C[t] = C[t];
            }
#pragma unroll
            for (int t = 0; t < 10; ++t) q.R[t] = 0.0;
            q.R[0] = D[0];
            q.R[5] = D[1];
            q.a = a; q.b = b; q.c = c;
            q.r[0] = d; q.r[1] = 0.0; q.r[2] = 0.0;
        } else {
            identity_row(q);
        }
        warp_pcr(q, G);
        if (lane < G) {
            X[3 * lane + 0] = q.R[0];
            X[3 * lane + 1] = q.R[5];
            X[3 * lane + 2] = q.r[0];
        }
    }
    __syncthreads();
    // every interface unknown from its group representation
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int g = k >> 5;
        const double* o = reps + 13 * (size_t)k;
        double xl[3] = {0.0, 0.0, 0.0};
        if (g > 0)
#pragma unroll
            for (int t = 0; t < 3; ++t) xl[t] = X[3 * (g - 1) + t];
        const double xr[3] = {X[3 * g], X[3 * g + 1], X[3 * g + 2]};
        double x0 = o[0] + (o[3] * xl[0] + o[4] * xl[1]) + (o[8] * xr[0] + o[9] * xr[1]);
        double x1 = o[1] + (o[5] * xl[0] + o[6] * xl[1]) + (o[10] * xr[0] + o[11] * xr[1]);
        double x2 = o[2] + o[7] * xl[2] + o[12] * xr[2];
        I.xi[3 * (size_t)k + 0] = x0;
        I.xi[3 * (size_t)k + 1] = x1;
        I.xi[3 * (size_t)k + 2] = x2;
    }
    __syncthreads();
}

// x = y + P xl + Q xr for a row with representation o (13 values), in one
// fixed, non-contracted order: a chunk's warp recovers its rows with it, and
// the previous chunk's warp recomputes this chunk's first row with it, so
// both get the same value.
__device__ __forceinline__ void rep_apply(const double* o, const double* xl, const double* xr,
                                          double* x) {
    x[0] = __dadd_rn(__dadd_rn(o[0], __dadd_rn(__dmul_rn(o[3], xl[0]), __dmul_rn(o[4], xl[1]))),
                     __dadd_rn(__dmul_rn(o[8], xr[0]), __dmul_rn(o[9], xr[1])));
    x[1] = __dadd_rn(__dadd_rn(o[1], __dadd_rn(__dmul_rn(o[5], xl[0]), __dmul_rn(o[6], xl[1]))),
                     __dadd_rn(__dmul_rn(o[10], xr[0]), __dmul_rn(o[11], xr[1])));
    x[2] = __dadd_rn(__dadd_rn(o[2], __dmul_rn(o[7], xl[2])), __dmul_rn(o[12], xr[2]));
}

// L3 of LO iteration m fused with L1 of iteration m+1, by the chunk's warp
// (lane = row): recovery of the rows from the representation set `cur` and
// the interface values (W_full, the LO residual, W_m <- W_full); then, when
// `next` is given, the block rows of iteration m+1 from the recovered values
// and their solve into the set `next`.  The neighbours outside the chunk are
// the previous chunk's interface value (row s-1), the next chunk's first row
// recomputed from its representation in `cur` (row e+1), or the fixed
// boundary cells, so no barrier is needed between the two halves.  Iteration
// m+1 is prepared before it is known whether iteration m converged; if it
// did, the prepared rows are not used.
__device__ __noinline__ void lo_chunk_step(WarpSmem& w, int kc, int z, int m,
                                           const double* __restrict__ cur,
                                           double* __restrict__ next) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int s = kc * I.lo_len;
    const int e = (s + I.lo_len < I.n_inner ? s + I.lo_len : I.n_inner) - 1;
    const int len = e - s + 1;
    double xl[3] = {0.0, 0.0, 0.0}, xr[3];
    if (kc > 0)
        for (int q = 0; q < 3; ++q) xl[q] = __ldcg(&I.xi[3 * (size_t)(kc - 1) + q]);
    for (int q = 0; q < 3; ++q) xr[q] = __ldcg(&I.xi[3 * (size_t)kc + q]);
    double x[3] = {0.0, 0.0, 0.0};
    double mdf = 0.0;
    FracMax fm;
    const int r = s + lane;
    if (lane < len) {
        double o13[13];
        rep_load(cur + 13 * (size_t)r, o13);
        rep_apply(o13, xl, xr, x);
        if (r == e) { x[0] = xr[0]; x[1] = xr[1]; x[2] = xr[2]; }
        double* Wr = I.Wm + 3 * (size_t)(r + 1);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double old = __ldcg(&Wr[q]);
            const double df = fabs(x[q] - old);
            const double ref = nan_max(fabs(x[q]), fabs(old));
            mdf = nan_max(mdf, df);
            fm.add(df, I.lo_abs_tol + I.lo_tol * ref);
            Wr[q] = x[q];
        }
    }
    const double a = warp_max(mdf), b = warp_max(fm.value());
    if (lane == 0) {
        double* h = I.lo_hist + 2 * ((size_t)z * I.lo_iter + m);
        atomic_max_nonneg(&h[0], a);
        atomic_max_nonneg(&h[1], b);
        if (kc == 0) I.lo_run[(size_t)z * I.lo_iter + m] = 1;
    }
    if (next == nullptr) return;
    // neighbours of every row (all lanes shuffle; the mask is the full warp)
    double wl[3], wr[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        wl[q] = __shfl_up_sync(0xffffffffu, x[q], 1);
        wr[q] = __shfl_down_sync(0xffffffffu, x[q], 1);
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) wl[q] = kc > 0 ? xl[q] : __ldcg(&I.Wm[q]);
    }
    if (lane == len - 1) {
        if (kc + 1 < I.lo_k) {
            const int s2 = e + 1;
            const int e2 = (s2 + I.lo_len < I.n_inner ? s2 + I.lo_len : I.n_inner) - 1;
            double xr2[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) xr2[q] = __ldcg(&I.xi[3 * (size_t)(kc + 1) + q]);
            if (s2 == e2) {
#pragma unroll
                for (int q = 0; q < 3; ++q) wr[q] = xr2[q];
            } else {
                double o13[13];
                rep_load(cur + 13 * (size_t)s2, o13);
                rep_apply(o13, xr, xr2, wr);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) wr[q] = __ldcg(&I.Wm[3 * (size_t)(I.nx - 1) + q]);
        }
    }
    LoRow L{};
    if (lane < len) lo_row_w(I, r, wl, x, wr, L);
    lo_chunk_solve(I, kc, L, next);
}

// ---- C: distribution solve over one tile (theta = 1/2) ------------------------
// x_s = a_s x_{s-1} + c_s with d = 1 + alpha + beta + theta dt / tau_lo,
// a = alpha/d, c = (E + theta dt M_lo / tau_lo) / d (:526-555).
__device__ __noinline__ bool dist_tile(WarpSmem& w, int vt, int c, int z, unsigned long long epoch,
                          unsigned long long limit, const double* __restrict__ fn,
                          double* __restrict__ fo, FracMax& q1, double& mdf, double& mref,
                          bool& bad) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const TileGeo g = inst_tile(I, vt, c, lane);
    const int nx = I.nx, nv = I.nv;
    const int nr = g.nrows;
    stage_rows_h<33>(w.a, I.E, g, nx, nv);
    stage_rows_h<32>(w.o, z > 0 ? fo : fn, g, nx, nv);
    cp_async_commit();
    const double vj = g.lane_ok ? __ldg(&I.v[g.j]) : 0.0;
    w.vv[lane] = vj;
    if (lane < nr) {
        const int i = scan_row(nx, g.pos, g.s0 + lane);
        const double* W3 = I.Wm + 3 * (size_t)i;
        const double n = __ldcg(&W3[0]), nu = __ldcg(&W3[1]), U = __ldcg(&W3[2]);
        // back to (n, u, T, tau) (:393-407)
        const double den = n + 1e-30;
        const double u = nu / den;
        double T = 2.0 * (U / den - 0.5 * u * u);
        T = (T != T || T >= 1e-30) ? T : 1e-30;
        const double sT = sqrt(T);
        const double tau = I.tau_tilde / (n * sT);
        w.coef[lane][0] = u;
        w.coef[lane][1] = -(0.5 / T);
        w.coef[lane][2] = (n * kInvSqrt2Pi) / sT;
        w.coef[lane][3] = (kTheta * I.dt) / tau;
        if (vt == 0) {
            I.Wlo[i] = n;
            I.Wlo[nx + i] = u;
            I.Wlo[2 * nx + i] = T;
        }
    }
    cp_async_wait_all();
    __syncwarp();
    const double cpl = I.dtdx2 * fabs(vj);
    const double one_plus = 1.0 + cpl;
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
            const double ev = g.lane_ok ? w.a[r][lane] : 0.0;
            cv[t] = fma(dti, M, ev) * rr;
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
    // rows without branches (selects and a predicated store) so that their
    // independent work overlaps; the residual takes FracMax's select-only path
    // and a tile that met a non-finite or non-positive term redoes it in full
    const double tol = I.ho_tol, abs_tol = I.ho_abs_tol;
    bool odd = false;
#pragma unroll 4
    for (int r = 0; r < nr; ++r) {
        const double a = cpl * recip_ge1(one_plus + w.coef[r][3]);
        X = fma(a, X, w.a[r][lane]);
        const double x = g.lane_ok ? X : 0.0;
        w.a[r][lane] = x;
        if (g.lane_ok) fo[(size_t)scan_row(nx, g.pos, g.s0 + r) * nv + g.j] = x;
        const double o = w.o[r][lane];
        const double df = g.lane_ok ? fabs(x - o) : 0.0;
        const double ref = g.lane_ok ? nan_max(fabs(x), fabs(o)) : 0.0;
        odd |= !q1.add_normal(df, g.lane_ok ? abs_tol + tol * ref : 1.0);
        mdf = nan_max(mdf, df);
        mref = nan_max(mref, ref);
        bad |= g.lane_ok && !isfinite(x);
    }
    if (__any_sync(0xffffffffu, odd) && g.lane_ok) {
        for (int r = 0; r < nr; ++r) {
            const double x = w.a[r][lane], o = w.o[r][lane];
            q1.add(fabs(x - o), abs_tol + tol * nan_max(fabs(x), fabs(o)));
        }
    }
    store_partials_h(w, g, vt);
    return ok;
}


// ---- the persistent kernel ----------------------------------------------------
// Phase trace (off unless a buffer is attached): four rows of 4 stamps
// (%globaltimer ns) per HO iteration z:
//   row 4z   = [A start (min), A work end (max), LO start (min), LO end (max)]
//   row 4z+1 = [C start (min), C work end (max), LO iterations, 0]
//   row 4z+2 = LO iteration 0: [L1 start (min), L1 end (max), L2 start (min), L2 end (max)]
//   row 4z+3 = LO iteration 0: [L3 start (min), L3 end (max), after its barrier (min), 0]
__device__ __forceinline__ unsigned long long gtimer_h() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void trace_h(const HoloDev& P, int z, int slot, bool is_min) {
    if (P.head.trace == nullptr || (threadIdx.x & 31) != 0 || 4 * z + 3 >= P.head.trace_iters)
        return;
    unsigned long long* p = P.head.trace + (size_t)16 * z + slot;
    const unsigned long long t = gtimer_h();
    if (is_min) atomicMin(p, t); else atomicMax(p, t);
}

__device__ __forceinline__ bool holo_sync(HoloDev& P, unsigned G) {
    if (grid_sync(&P.head.bar, G, &P.head.err, P.head.spin_limit)) return true;
    if (threadIdx.x == 0) atomicOr(&P.head.err_sticky, 1 << KEQ_ERR_TIMEOUT);
    return false;
}

__device__ __forceinline__ bool ho_stop(const HoloInst& I, int z) {
    if (I.fixed_ho > 0) return z + 1 >= I.fixed_ho;
    return __ldcg(&I.ho_red[4 * z + 0]) <= 1.0;  // :566
}
__device__ __forceinline__ bool ho_active(const HoloInst& I, int z) {
    if (z >= I.ho_iter) return false;
    if (z == 0) return true;
    if (__ldcg(&I.ho_run[z - 1]) != 1) return false;
    return !ho_stop(I, z - 1);
}
__device__ __forceinline__ bool lo_stop(const HoloInst& I, int z, int m) {
    if (I.fixed_lo > 0) return m + 1 >= I.fixed_lo;
    return __ldcg(&I.lo_hist[2 * ((size_t)z * I.lo_iter + m) + 1]) < 1.0;  // :389
}
__device__ __forceinline__ bool lo_active(const HoloInst& I, int z, int m) {
    if (!ho_active(I, z) || m >= I.lo_iter) return false;
    if (m == 0) return true;
    if (__ldcg(&I.lo_run[(size_t)z * I.lo_iter + m - 1]) != 1) return false;
    return !lo_stop(I, z, m - 1);
}

__device__ __forceinline__ long long claim_h(unsigned* tickets, int z) {
    unsigned t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(&tickets[z], 1u);
    return (long long)__shfl_sync(0xffffffffu, t, 0);
}

// P2 row reduction (lane = interior row): raw half sums of f^n, HO-old
// moments, W_HO and the old Maxwellian's coefficients.
__device__ void init_rows(WarpSmem& w, int ru) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int k = ru * kRB + lane;
    if (k >= I.n_inner) return;
    const int i = k + 1;
    double R8[8];
    half_sums(I, k, R8);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        I.Rn[8 * (size_t)i + q] = R8[q];
        I.R[8 * (size_t)i + q] = R8[q];
    }
    const Mom m = mom_of(R8, I.dv);
    double c4[4];
    mc_of(m, I.tau_tilde, c4);
    reinterpret_cast<double2*>(I.Mco + 4 * (size_t)i)[0] = make_double2(c4[0], c4[1]);
    reinterpret_cast<double2*>(I.Mco + 4 * (size_t)i)[1] = make_double2(c4[2], c4[3]);
    // W_HO = (n, n u, n (u^2 + T) / 2) (:268-271)
    I.Who[3 * (size_t)i + 0] = m.n;
    I.Who[3 * (size_t)i + 1] = m.n * m.u;
    I.Who[3 * (size_t)i + 2] = 0.5 * m.n * (m.u * m.u + m.T);
}

// Boundary rows (warp-wide, row ib in {0, nx-1}): raw half sums from P0,
// W_HO, the Maxwellian sums and the constant consistency term
// Y_b = dt (sum M w - sum f w) dv / tau (C_new = C_old on these rows).
__device__ __noinline__ void init_boundary_row(WarpSmem& w, int side) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int ib = side == 0 ? 0 : I.nx - 1;
    double R8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) R8[q] = __ldcg(&I.Rn[8 * (size_t)ib + q]);
    const Mom m = mom_of(R8, I.dv);
    double c4[4];
    mc_of(m, I.tau_tilde, c4);
    double sm[3];
    maxwell_sums_row(I.v, I.nv, c4, sm);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) I.R[8 * (size_t)ib + q] = R8[q];
        reinterpret_cast<double2*>(I.Mco + 4 * (size_t)ib)[0] = make_double2(c4[0], c4[1]);
        reinterpret_cast<double2*>(I.Mco + 4 * (size_t)ib)[1] = make_double2(c4[2], c4[3]);
        I.Who[3 * (size_t)ib + 0] = m.n;
        I.Who[3 * (size_t)ib + 1] = m.n * m.u;
        I.Who[3 * (size_t)ib + 2] = 0.5 * m.n * (m.u * m.u + m.T);
        const double sfw[3] = {m.n, m.s1, 0.5 * m.s2};
        double mx = 0.0;
        for (int q = 0; q < 3; ++q) {
            const double y = I.con_terms ? I.dt * (((sm[q] * I.dv) - sfw[q]) * c4[3]) : 0.0;
            I.Y[3 * (size_t)ib + q] = y;
            mx = nan_max(mx, fabs(y));
        }
        atomic_max_nonneg(&I.misc[1], mx);
        // n_lo, u_lo, T_lo of the boundary rows (W_m = W_HO there)
        const double den = m.n + 1e-30;
        const double u = (m.n * m.u) / den;
        double T = 2.0 * ((0.5 * m.n * (m.u * m.u + m.T)) / den - 0.5 * u * u);
        T = (T != T || T >= 1e-30) ? T : 1e-30;
        I.Wlo[ib] = m.n;
        I.Wlo[I.nx + ib] = u;
        I.Wlo[2 * I.nx + ib] = T;
    }
}

// P4 (lane = interior row): I_old = (1-theta) (sum M_old w - sum f^n w) dv / tau_old.
__device__ void iold_rows(WarpSmem& w, int ru) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int k = ru * kRB + lane;
    if (k >= I.n_inner) return;
    const int i = k + 1;
    double sM[4], R8[8];
    sum_partials4(I.part, 0, I.nvt, I.n_inner, k, sM);
#pragma unroll
    for (int q = 0; q < 8; ++q) R8[q] = __ldcg(&I.Rn[8 * (size_t)i + q]);
    const Mom m = mom_of(R8, I.dv);
    const double inv_tau = __ldcg(&I.Mco[4 * (size_t)i + 3]);
    const double smw[3] = {sM[0] * I.dv, sM[1] * I.dv, 0.5 * (sM[2] * I.dv)};
    const double sfw[3] = {m.n, m.s1, 0.5 * m.s2};
#pragma unroll
    for (int q = 0; q < 3; ++q)
        I.Iold[3 * (size_t)i + q] = (1.0 - kTheta) * ((smw[q] - sfw[q]) * inv_tau);
}

// Row reduction after the distribution pass (lane = interior row): raw half
// sums of f_{z+1}.
__device__ void ho_rows(WarpSmem& w, int ru, int z) {
    const HoloInst& I = w.I;
    const int lane = threadIdx.x & 31;
    const int k = ru * kRB + lane;
    if (k < I.n_inner) {
        double R8[8];
        half_sums(I, k, R8);
#pragma unroll
        for (int q = 0; q < 8; ++q) I.R[8 * (size_t)(k + 1) + q] = R8[q];
    }
    if (ru == 0 && lane == 0) I.ho_run[z] = 1;
    __syncwarp();
}

__global__ void __launch_bounds__(kThreads, 3) holo_step_kernel(HoloDev* __restrict__ Pp,
                                                                int swap_io) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HoloDev& P = *Pp;
    const unsigned G = gridDim.x;
    const int n_inst = P.n_inst;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
    const long long gwarp = (long long)blockIdx.x * kWarps + warp, nwarps = (long long)G * kWarps;
    const long long total_tiles = P.total_tiles, total_rb = P.total_rb, total_lo = P.total_lo;
    if (lane == 0) w.cur_b = -1;
    __syncwarp();

    // P0
    if (blockIdx.x == 0) {
        for (int q = threadIdx.x; q < P.max_ho; q += kThreads) P.tickets[q] = 0u;
        if (threadIdx.x == 0) P.head.seq = P.head.seq + 1ull;
    }
    for (int b = blockIdx.x; b < n_inst; b += G) {
        const HoloInst& I = P.inst[b];
        const double* fn = swap_io ? I.f_out : I.f_in;
        double* fo = swap_io ? const_cast<double*>(I.f_in) : I.f_out;
        if (threadIdx.x == 0) {
            I.stats->status = KEQ_ERR_TIMEOUT;  // pending until stage E
            if (P.head.fresh) {
                I.stats->total_iters = 0;
                I.stats->total_steps = 0;
            }
        }
        const long long ntiles = (long long)I.nvt * I.nchunks;
        for (long long q = threadIdx.x; q < ntiles; q += kThreads) I.flag[q] = 0ull;
        for (int q = threadIdx.x; q < 4 * I.ho_iter; q += kThreads) I.ho_red[q] = 0.0;
        for (int q = threadIdx.x; q < 2 * I.ho_iter * I.lo_iter; q += kThreads) I.lo_hist[q] = 0.0;
        for (int q = threadIdx.x; q < I.ho_iter * I.lo_iter; q += kThreads) I.lo_run[q] = 0;
        for (int q = threadIdx.x; q < I.ho_iter; q += kThreads) {
            I.ho_run[q] = 0;
            I.nonfin[q] = 0;
        }
        for (int q = threadIdx.x; q < I.ho_iter * I.nrb; q += kThreads) I.rbcnt[q] = 0u;
        for (int q = threadIdx.x; q < 8; q += kThreads) I.misc[q] = 0.0;
        for (int q = threadIdx.x; q < I.nv; q += kThreads) {
            fo[q] = fn[q];
            fo[(size_t)(I.nx - 1) * I.nv + q] = fn[(size_t)(I.nx - 1) * I.nv + q];
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            // boundary row raw half sums (sequential) and max |f|
            const int ib = threadIdx.x == 0 ? 0 : I.nx - 1;
            const double* row = fn + (size_t)ib * I.nv;
            double R8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            double mx = 0.0;
            for (int j = 0; j < I.nv; ++j) {
                const double x = row[j], vj = I.v[j];
                const double t1 = x * vj, t2 = t1 * vj;
                const int o = vj > 0.0 ? 0 : 4;
                R8[o + 0] += x;
                R8[o + 1] += t1;
                R8[o + 2] += t2;
                R8[o + 3] = fma(t2, vj, R8[o + 3]);
                mx = nan_max(mx, fabs(x));
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) I.Rn[8 * (size_t)ib + q] = R8[q];
            atomic_max_nonneg(&I.misc[0], mx);
        }
    }
    if (!holo_sync(P, G)) return;
    const unsigned long long seq = __ldcg(&P.head.seq);
    const unsigned long long limit = P.head.spin_limit;

    // P1: moment partials of f^n
    for (long long t = gwarp; t < total_tiles; t += nwarps) {
        const int b = find_inst(P.tile_off, n_inst, t);
        stage_warp(w, &P.inst[b], b);
        const long long tl = t - w.I.tile_off;
        moments_tile(w, (int)(tl % w.I.nvt), (int)(tl / w.I.nvt), swap_io ? w.I.f_out : w.I.f_in);
    }
    if (!holo_sync(P, G)) return;

    // P2: per-row HO-old data; boundary rows
    for (long long u = gwarp; u < total_rb; u += nwarps) {
        const int b = find_inst(P.rb_off, n_inst, u);
        stage_warp(w, &P.inst[b], b);
        init_rows(w, (int)(u - w.I.rb_off));
    }
    for (long long u = gwarp; u < 2LL * n_inst; u += nwarps) {
        const int b = (int)(u >> 1);
        stage_warp(w, &P.inst[b], b);
        init_boundary_row(w, (int)(u & 1));
    }
    if (!holo_sync(P, G)) return;

    // P3: explicit term and old-Maxwellian partials
    for (long long t = gwarp; t < total_tiles; t += nwarps) {
        const int b = find_inst(P.tile_off, n_inst, t);
        stage_warp(w, &P.inst[b], b);
        const long long tl = t - w.I.tile_off;
        explicit_tile(w, (int)(tl % w.I.nvt), (int)(tl / w.I.nvt), swap_io ? w.I.f_out : w.I.f_in);
    }
    if (!holo_sync(P, G)) return;

    // P4: I_old
    for (long long u = gwarp; u < total_rb; u += nwarps) {
        const int b = find_inst(P.rb_off, n_inst, u);
        stage_warp(w, &P.inst[b], b);
        iold_rows(w, (int)(u - w.I.rb_off));
    }
    if (!holo_sync(P, G)) return;

    for (int z = 0; z < P.max_ho; ++z) {
        // any instance active in HO iteration z (a share of the instances per
        // thread, combined over the CTA)
        bool mine = false;
        for (int b = threadIdx.x; b < n_inst && !mine; b += kThreads) mine = ho_active(P.inst[b], z);
        if (!__syncthreads_or(mine)) break;

        trace_h(P, z, 0, true);
        // A: velocity sums of M(f_z) per interior row (one warp per row);
        // W_m = W_HO; boundary |Y| into max_YI
        for (long long u = gwarp; u < total_rb * kRB; u += nwarps) {
            const long long rb = u / kRB;
            const int b = find_inst(P.rb_off, n_inst, rb);
            stage_warp(w, &P.inst[b], b);
            if (!ho_active(w.I, z) || !w.I.con_terms) continue;
            const int k = (int)(rb - w.I.rb_off) * kRB + (int)(u % kRB);
            if (k < w.I.n_inner) maxwell_row(w, k);
        }
        // W_m = W_HO, spread over every thread of the grid (one element each
        // for a 4096-row instance; a single CTA would take ~100 dependent
        // load-store rounds)
        {
            const long long gt = (long long)blockIdx.x * kThreads + threadIdx.x;
            const long long gn = (long long)G * kThreads;
            for (int b = 0; b < n_inst; ++b) {
                const HoloInst& I = P.inst[b];
                if (!ho_active(I, z)) continue;
                for (long long q = gt; q < 3LL * I.nx; q += gn) I.Wm[q] = __ldcg(&I.Who[q]);
                if (gt == 0) atomic_max_nonneg(&I.ho_red[4 * z + 3], __ldcg(&I.misc[1]));
            }
        }
        trace_h(P, z, 1, false);
        if (!holo_sync(P, G)) return;

        trace_h(P, z, 2, true);
        // LO Picard iterations
        for (int m = 0; m < P.max_lo; ++m) {
            bool lmine = false;
            for (int b = threadIdx.x; b < n_inst && !lmine; b += kThreads)
                lmine = lo_active(P.inst[b], z, m);
            if (!__syncthreads_or(lmine)) break;
            // representation sets: iteration m's in lorow set (m & 1)
            const size_t set_cur = (size_t)(m & 1), set_next = (size_t)((m + 1) & 1);
            // L1 (first LO iteration only; later ones are prepared by the
            // fused recovery below)
            if (m == 0) {
                trace_h(P, z, 8, true);
                for (long long u = gwarp; u < total_lo; u += nwarps) {
                    const int b = find_inst(P.lo_off, n_inst, u);
                    stage_warp(w, &P.inst[b], b);
                    if (!lo_active(w.I, z, m)) continue;
                    const int kc = (int)(u - w.I.lo_off);
                    const int s0 = kc * w.I.lo_len;
                    const int e0 = (s0 + w.I.lo_len < w.I.n_inner ? s0 + w.I.lo_len : w.I.n_inner);
                    double mx = 0.0;
                    for (int k = s0 + lane; k < e0; k += 32) mx = nan_max(mx, lo_prep_row(w.I, k));
                    mx = warp_max(mx);
                    if (lane == 0) atomic_max_nonneg(&w.I.ho_red[4 * z + 3], mx);
                    __syncwarp();
                    lo_chunk_eliminate(w, kc, w.I.lorow);
                }
                trace_h(P, z, 9, false);
                if (!holo_sync(P, G)) return;
            }
            if (m == 0) trace_h(P, z, 10, true);
            // L2: one CTA per instance
            if (lane == 0) w.cur_b = -1;  // shared memory is reused below
            __syncthreads();
            for (int b = blockIdx.x; b < n_inst; b += G) {
                const HoloInst& I = P.inst[b];
                if (!lo_active(I, z, m)) continue;
                lo_reduced_solve(I, I.lorow + set_cur * 13 * (size_t)I.n_inner, smem_raw);
            }
            __syncthreads();
            if (lane == 0) w.cur_b = -1;
            __syncwarp();
            if (m == 0) trace_h(P, z, 11, false);
            if (!holo_sync(P, G)) return;
            if (m == 0) trace_h(P, z, 12, true);
            // L3 of iteration m fused with L1 of iteration m+1
            for (long long u = gwarp; u < total_lo; u += nwarps) {
                const int b = find_inst(P.lo_off, n_inst, u);
                stage_warp(w, &P.inst[b], b);
                if (!lo_active(w.I, z, m)) continue;
                const HoloInst& I = w.I;
                const bool more = m + 1 < I.lo_iter && (I.fixed_lo <= 0 || m + 1 < I.fixed_lo);
                lo_chunk_step(w, (int)(u - I.lo_off), z, m,
                              I.lorow + set_cur * 13 * (size_t)I.n_inner,
                              more ? I.lorow + set_next * 13 * (size_t)I.n_inner : nullptr);
            }
            if (m == 0) trace_h(P, z, 13, false);
            if (!holo_sync(P, G)) return;
            if (m == 0) trace_h(P, z, 14, true);
        }

        trace_h(P, z, 3, false);
        if (P.head.trace && blockIdx.x == 0 && threadIdx.x == 0 && 4 * z + 3 < P.head.trace_iters) {
            int nlo = 0;
            while (nlo < P.max_lo && lo_active(P.inst[0], z, nlo)) ++nlo;
            P.head.trace[(size_t)16 * z + 6] = (unsigned long long)nlo;
        }
        trace_h(P, z, 4, true);
        // C: distribution solve
        {
            const unsigned long long epoch = seq * (unsigned long long)(P.max_ho + 1) + z + 1;
            FracMax q1;
            double mdf = 0.0, mref = 0.0;
            bool bad = false;
            int res_b = -1;
            for (;;) {
                const long long t = claim_h(P.tickets, z);
                if (t >= total_tiles) break;
                const int b = find_inst(P.tile_off, n_inst, t);
                if (b != res_b && res_b >= 0 && ho_active(w.I, z)) {
                    const double r1 = warp_max(q1.value()), r2 = warp_max(mdf), r3 = warp_max(mref);
                    const bool nb = __any_sync(0xffffffffu, bad);
                    if (lane == 0) {
                        atomic_max_nonneg(&w.I.ho_red[4 * z + 0], r1);
                        atomic_max_nonneg(&w.I.ho_red[4 * z + 1], r2);
                        atomic_max_nonneg(&w.I.ho_red[4 * z + 2], r3);
                        if (nb) atomicOr(&w.I.nonfin[z], 1);
                    }
                    q1 = FracMax();
                    mdf = mref = 0.0;
                    bad = false;
                }
                stage_warp(w, &P.inst[b], b);
                res_b = b;
                if (!ho_active(w.I, z)) continue;
                const long long tl = t - w.I.tile_off;
                const int c = (int)(tl / w.I.nvt), vt = (int)(tl % w.I.nvt);
                const double* fn = swap_io ? w.I.f_out : w.I.f_in;
                double* fo = swap_io ? const_cast<double*>(w.I.f_in) : w.I.f_out;
                if (!dist_tile(w, vt, c, z, epoch, limit, fn, fo, q1, mdf, mref, bad)) {
                    if (lane == 0) {
                        atomicOr(&P.head.err, 1 << KEQ_ERR_TIMEOUT);
                        atomicOr(&P.head.err_sticky, 1 << KEQ_ERR_TIMEOUT);
                    }
                }
                const TileGeo g = inst_tile(w.I, vt, c, lane);
                fence_acq_rel();
                __syncwarp();
                if (lane == 0)
                    rowblock_arrive(w.I.rbcnt + (size_t)z * w.I.nrb, w.I.nx, w.I.n_inner, w.I.nvt,
                                    g, w.done_rb);
                __syncwarp();
                const int d0 = w.done_rb[0], d1 = w.done_rb[1];
                if (d0 >= 0 || d1 >= 0) {
                    fence_acq_rel();
                    __syncwarp();
                    if (d0 >= 0) ho_rows(w, d0, z);
                    if (d1 >= 0) ho_rows(w, d1, z);
                }
            }
            if (res_b >= 0 && ho_active(w.I, z)) {
                const double r1 = warp_max(q1.value()), r2 = warp_max(mdf), r3 = warp_max(mref);
                const bool nb = __any_sync(0xffffffffu, bad);
                if (lane == 0) {
                    atomic_max_nonneg(&w.I.ho_red[4 * z + 0], r1);
                    atomic_max_nonneg(&w.I.ho_red[4 * z + 1], r2);
                    atomic_max_nonneg(&w.I.ho_red[4 * z + 2], r3);
                    if (nb) atomicOr(&w.I.nonfin[z], 1);
                }
            }
        }
        trace_h(P, z, 5, false);
        if (!holo_sync(P, G)) return;
    }

    // E: statistics (benchlog keys of :586-594)
    if (blockIdx.x == 0 && threadIdx.x == 0) P.head.fresh = 0;
    for (int b = blockIdx.x; b < n_inst; b += G) {
        if (threadIdx.x >= 32) continue;
        const HoloInst& I = P.inst[b];
        const int last = count_leading_ones(I.ho_run, I.ho_iter) - 1;
        const int lo_last =
            last >= 0 ? count_leading_ones(I.lo_run + (size_t)last * I.lo_iter, I.lo_iter) - 1 : -1;
        if (threadIdx.x != 0) continue;
        keq_step_stats* st = I.stats;
        int status = KEQ_OK;
        double lo_df = 0.0, lo_std = 0.0, ho_std = 0.0, ho_rel = 0.0, myi = 0.0;
        if (last >= 0) {
            if (lo_last >= 0) {
                lo_df = __ldcg(&I.lo_hist[2 * ((size_t)last * I.lo_iter + lo_last)]);
                lo_std = __ldcg(&I.lo_hist[2 * ((size_t)last * I.lo_iter + lo_last) + 1]);
            }
            ho_std = __ldcg(&I.ho_red[4 * last + 0]);
            const double mref = nan_max(__ldcg(&I.ho_red[4 * last + 2]), __ldcg(&I.misc[0]));
            ho_rel = __ldcg(&I.ho_red[4 * last + 1]) / mref;
            myi = __ldcg(&I.ho_red[4 * last + 3]);
            if (__ldcg(&I.nonfin[last])) status = KEQ_ERR_NONFINITE;
        }
        if (__ldcg(&P.head.err) & (1 << KEQ_ERR_TIMEOUT)) status = KEQ_ERR_TIMEOUT;
        st->status = status;
        st->iters = last + 1;
        st->aa_applied = 0;
        st->lo_iters = lo_last + 1;
        st->residual = ho_rel;
        st->std_residual = ho_std;
        st->lo_residual = lo_df;
        st->std_lo_residual = lo_std;
        st->max_YI = myi;
        st->total_iters += last + 1;
        st->total_steps += 1;
    }
}

constexpr size_t kSmemBytes = sizeof(WarpSmem) * kWarps;
static_assert(sizeof(GroupRec) * (kMaxLoChunks / 32) + 13 * sizeof(double) * kMaxLoChunks +
                      3 * sizeof(double) * (kMaxLoChunks / 32) <=
                  kSmemBytes,
              "interface system of the LO solve must fit the CTA's shared memory");

}  // namespace holo
}  // namespace keq

// ===========================================================================
// Host side
// ===========================================================================
namespace {

using keq::holo::HoloDev;
using keq::holo::HoloInst;

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

struct HDerived {
    int n_inner, nt_neg, nvt, rows, nchunks, nrb, lo_len, lo_k;
};

HDerived hderive(int nx, int nv, int kp) {
    HDerived d;
    d.n_inner = nx - 2;
    d.nt_neg = (kp + 31) / 32;
    d.nvt = d.nt_neg + (nv - kp + 31) / 32;
    d.rows = keq::kRmax;
    d.nchunks = (d.n_inner + d.rows - 1) / d.rows;
    d.nrb = (d.n_inner + keq::kRB - 1) / keq::kRB;
    // LO chunks of 32 rows (one row per lane of the chunk's warp)
    d.lo_len = keq::holo::kLoChunk;
    d.lo_k = (d.n_inner + d.lo_len - 1) / d.lo_len;
    return d;
}

bool holo_valid(const keq_holo_params& p) {
    return p.ho_iter >= 1 && p.ho_iter <= 4096 && p.lo_iter >= 1 && p.lo_iter <= 4096 &&
           (long long)p.ho_iter * p.lo_iter <= (1LL << 22);
}

size_t carve_holo(void* base, int nx, int nv, int kp, const keq_holo_params& p, HoloInst* I) {
    const HDerived d = hderive(nx, nv, kp);
    Carve c{static_cast<char*>(base), 0};
    const size_t ntiles = (size_t)d.nvt * d.nchunks;
    const size_t ho = (size_t)p.ho_iter, lo = (size_t)p.lo_iter;
    double* Wlo = c.take<double>(3 * (size_t)nx);  // first: the host reads it as state.n/u/T
    double* E = c.take<double>((size_t)nx * nv);
    double* part = c.take<double>((size_t)d.nvt * d.n_inner * keq::kPartQ);
    double* R = c.take<double>(8 * (size_t)nx);
    double* Rn = c.take<double>(8 * (size_t)nx);
    double* Mco = c.take<double>(4 * (size_t)nx);
    double* Wm = c.take<double>(3 * (size_t)nx);
    double* Who = c.take<double>(3 * (size_t)nx);
    double* Iold = c.take<double>(3 * (size_t)nx);
    double* Msum = c.take<double>(3 * (size_t)nx);
    double* Ib = c.take<double>(8);
    double* Y = c.take<double>(3 * (size_t)nx);
    double* T1 = c.take<double>(3 * (size_t)nx);
    double* lorow = c.take<double>(2 * 13 * (size_t)d.n_inner);
    double* loedge = c.take<double>(18 * (size_t)d.lo_k);
    double* xi = c.take<double>(3 * (size_t)d.lo_k);
    double* agg = c.take<double>(ntiles * 64);
    double* inc = c.take<double>(ntiles * 32);
    unsigned long long* flag = c.take<unsigned long long>(ntiles);
    unsigned* rbcnt = c.take<unsigned>(ho * d.nrb);
    double* ho_red = c.take<double>(4 * ho);
    double* lo_hist = c.take<double>(2 * ho * lo);
    int* ho_run = c.take<int>(ho);
    int* lo_run = c.take<int>(ho * lo);
    int* nonfin = c.take<int>(ho);
    double* misc = c.take<double>(8);
    if (I) {
        I->E = E; I->part = part; I->R = R; I->Rn = Rn; I->Mco = Mco; I->Wm = Wm; I->Who = Who;
        I->Iold = Iold; I->Msum = Msum; I->Ib = Ib; I->Y = Y; I->T1 = T1; I->lorow = lorow; I->loedge = loedge;
        I->xi = xi; I->Wlo = Wlo; I->agg = agg; I->inc = inc; I->flag = flag; I->rbcnt = rbcnt;
        I->ho_red = ho_red; I->lo_hist = lo_hist; I->ho_run = ho_run; I->lo_run = lo_run;
        I->nonfin = nonfin; I->misc = misc;
    }
    return align_up(c.off, 256);
}

size_t holo_plan_bytes(int n, int max_ho) {
    Carve c{nullptr, 0};
    c.take<HoloDev>(1);
    c.take<HoloInst>(n);
    c.take<long long>(n + 1);
    c.take<long long>(n + 1);
    c.take<long long>(n + 1);
    c.take<unsigned>(max_ho + 1);
    return align_up(c.off, 256);
}

}  // namespace

extern "C" {

keq_status keq_holo_instance_workspace_size(const keq_grid* grid, const keq_holo_params* params,
                                            size_t* bytes) {
    if (!grid || !params || !bytes) return KEQ_ERR_INVALID;
    if (grid->nx < 3 || grid->nv < 1 || !holo_valid(*params)) return KEQ_ERR_INVALID;
    size_t best = 0;
    const int kps[3] = {0, grid->nv, grid->nv / 2 + 1 <= grid->nv ? grid->nv / 2 + 1 : grid->nv};
    for (int q = 0; q < 3; ++q) {
        const size_t b = carve_holo(nullptr, grid->nx, grid->nv, kps[q], *params, nullptr);
        if (b > best) best = b;
    }
    const size_t worst =
        carve_holo(nullptr, grid->nx, grid->nv + 64, (grid->nv + 64) / 2, *params, nullptr);
    *bytes = worst > best ? worst : best;
    return KEQ_OK;
}

keq_status keq_holo_plan_workspace_size(const keq_instance* insts, int32_t n,
                                        const keq_holo_params* params, int32_t per_instance_params,
                                        size_t* bytes) {
    if (!insts || n < 1 || !params || !bytes) return KEQ_ERR_INVALID;
    int max_ho = 1;
    for (int b = 0; b < n; ++b) {
        const int h = params[per_instance_params ? b : 0].ho_iter;
        if (h > max_ho) max_ho = h;
    }
    *bytes = holo_plan_bytes(n, max_ho);
    return KEQ_OK;
}

keq_status keq_holo_plan_create(const keq_instance* insts, int32_t n, const keq_holo_params* params,
                                int32_t per_instance_params, void* plan_ws, size_t plan_ws_bytes,
                                keq_stream_t stream, keq_plan** plan_out) {
    using namespace keq;
    if (!insts || n < 1 || !params || !plan_ws || !plan_out) return KEQ_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(plan_ws) % 256) return KEQ_ERR_WORKSPACE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
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
    int max_ho = 1, max_lo = 1;
    for (int b = 0; b < n; ++b) {
        const keq_holo_params& p = params[per_instance_params ? b : 0];
        if (!holo_valid(p)) return KEQ_ERR_INVALID;
        if (p.ho_iter > max_ho) max_ho = p.ho_iter;
        if (p.lo_iter > max_lo) max_lo = p.lo_iter;
    }
    if (plan_ws_bytes < holo_plan_bytes(n, max_ho)) return KEQ_ERR_WORKSPACE;

    keq_plan* plan = new keq_plan();
    plan->kind = KEQ_PLAN_HOLO;
    plan->n_inst = n;
    plan->device = dev_of_buffers;
    plan->inst_bytes = sizeof(HoloInst);
    plan->off_f_in = offsetof(HoloInst, f_in);
    plan->off_f_out = offsetof(HoloInst, f_out);
    plan->kernel = (const void*)holo::holo_step_kernel;
    plan->smem = holo::kSmemBytes;
    plan->threads = holo::kThreads;
    plan->host_inst.resize(sizeof(HoloInst) * (size_t)n);
    std::vector<HoloInst> host(n);
    std::vector<long long> toff(n + 1), roff(n + 1), loff(n + 1);
    long long t = 0, r = 0, l = 0;
    std::vector<double> vh;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < n; ++b) {
        const keq_instance& in = insts[b];
        const keq_holo_params& p = params[per_instance_params ? b : 0];
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
        if (kp < 0 || kp > nv) {
            vh.resize(nv);
            if (cudaMemcpyAsync(vh.data(), in.grid.v, sizeof(double) * nv, cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                keq_internal_set_cuda_error(cudaGetLastError());
                delete plan;
                return KEQ_ERR_CUDA;
            }
            kp = 0;
            for (int j = 0; j < nv; ++j) {
                if (j > 0 && !(vh[j] > vh[j - 1])) {
                    delete plan;
                    return KEQ_ERR_INVALID;
                }
                if (!(vh[j] > 0.0)) kp = j + 1;
            }
        }
        const HDerived d = hderive(nx, nv, kp);
        if (d.lo_k > holo::kMaxLoChunks) {
            delete plan;
            return KEQ_ERR_UNSUPPORTED;  // nx beyond the LO solver's capacity
        }
        HoloInst I{};
        I.nx = nx; I.nv = nv; I.n_inner = d.n_inner; I.kp = kp;
        I.nt_neg = d.nt_neg; I.nvt = d.nvt; I.nchunks = d.nchunks; I.nrb = d.nrb;
        I.rows = d.rows; I.lo_len = d.lo_len; I.lo_k = d.lo_k;
        I.tile_off = t; I.rb_off = r; I.lo_off = l;
        I.dx = in.grid.dx; I.dv = in.grid.dv; I.dt = in.dt; I.tau_tilde = in.tau_tilde;
        I.dtdx2 = in.dt / (2.0 * in.grid.dx);
        I.ho_iter = p.ho_iter; I.lo_iter = p.lo_iter;
        I.con_terms = p.con_terms_do ? 1 : 0; I.flux_cons = p.flux_consistency_do ? 1 : 0;
        I.sv_down = p.sv_down ? 1 : 0; I.fixed_ho = p.fixed_ho_iters; I.fixed_lo = p.fixed_lo_iters;
        I.ho_tol = p.ho_tol; I.ho_abs_tol = p.ho_abs_tol; I.lo_tol = p.lo_tol;
        I.lo_abs_tol = p.lo_abs_tol;
        I.v = in.grid.v; I.f_in = in.f_in; I.f_out = in.f_out; I.stats = in.stats;
        carve_holo(in.workspace, nx, nv, kp, p, &I);
        host[b] = I;
        toff[b] = t; roff[b] = r; loff[b] = l;
        t += (long long)d.nvt * d.nchunks;
        r += d.nrb;
        l += d.lo_k;
    }
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        delete plan;
        return KEQ_ERR_CUDA;
    }
    toff[n] = t; roff[n] = r; loff[n] = l;
    if (t >= (long long)0xffffffffll) {
        delete plan;
        return KEQ_ERR_INVALID;
    }
    memcpy(plan->host_inst.data(), host.data(), sizeof(HoloInst) * (size_t)n);
    Carve c{static_cast<char*>(plan_ws), 0};
    HoloDev* dev = c.take<HoloDev>(1);
    HoloInst* dinst = c.take<HoloInst>(n);
    long long* dt_ = c.take<long long>(n + 1);
    long long* dr_ = c.take<long long>(n + 1);
    long long* dl_ = c.take<long long>(n + 1);
    unsigned* tickets = c.take<unsigned>(max_ho + 1);
    HoloDev h{};
    h.head.spin_limit = kSpinLimit;
    h.head.fresh = 1;  // the first launch zeroes the stats totals
    h.n_inst = n;
    h.max_ho = max_ho;
    h.max_lo = max_lo;
    h.total_tiles = t;
    h.total_rb = r;
    h.total_lo = l;
    h.inst = dinst;
    h.tile_off = dt_;
    h.rb_off = dr_;
    h.lo_off = dl_;
    h.tickets = tickets;
    plan->dev = dev;
    plan->dev_inst = dinst;
    e = cudaMemcpyAsync(dev, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dinst, host.data(), sizeof(HoloInst) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dt_, toff.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dr_, roff.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dl_, loff.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
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

}  // extern "C"
