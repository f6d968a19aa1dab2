// keq_kernels.cu -- kernel-level drop-ins of the reference's extension
// modules (implicit_fused, gtsv, lo_blocktridiag) behind the C ABI.  The
// fused time-step kernels (keq_implicit.cu, keq_holo.cu) do not call these;
// they serve callers that use the reference's module-level API directly.
#include <cuda_runtime.h>
#include <math.h>

#include "keq_common.cuh"
#include "keq_internal.h"

namespace keq {

// ---- K1: velocity moments, one warp per row -------------------------------
// implicit_kernels.cu:28-81 semantics (clamps), reduction = per-lane strided
// partial sums + fixed butterfly.
__global__ void __launch_bounds__(256) moments_kernel(const double* __restrict__ f,
                                                      const double* __restrict__ v, int nx,
                                                      int nv, double dv, double* __restrict__ n,
                                                      double* __restrict__ nu,
                                                      double* __restrict__ T) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nx) return;
    const double* row = f + (size_t)warp * nv;
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;
    for (int j = lane; j < nv; j += 32) {
        const double x = row[j], vj = v[j];
        p0 += x;
        p1 += x * vj;
        p2 += x * vj * vj;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p0 += __shfl_xor_sync(0xffffffffu, p0, o);
        p1 += __shfl_xor_sync(0xffffffffu, p1, o);
        p2 += __shfl_xor_sync(0xffffffffu, p2, o);
    }
    if (lane == 0) {
        const double n_raw = p0 * dv, nu_raw = p1 * dv, s2 = p2 * dv;
        const double nn = n_raw > kTiny ? n_raw : kTiny;
        const double u = nu_raw / nn;
        double Tg = s2 / nn - u * u;
        if (!(Tg > 0.0)) Tg = kTiny;
        n[warp] = nn;
        nu[warp] = nu_raw;
        T[warp] = Tg;
    }
}

// ---- K2: Maxwellian + upwind implicit assembly ----------------------------
// implicit_kernels.cu:84-134; one thread per (v_j, k), k fastest.
__global__ void __launch_bounds__(256) build_system_kernel(
    const double* __restrict__ B0, const double* __restrict__ v, const double* __restrict__ n,
    const double* __restrict__ nu, const double* __restrict__ Tg, const double* __restrict__ fl,
    const double* __restrict__ fr, int nx, int nv, double dt, double dx, double tau_tilde,
    double inv_sqrt_2pi, double* __restrict__ dl, double* __restrict__ dd,
    double* __restrict__ du, double* __restrict__ B) {
    const int n_inner = nx - 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_inner * nv) return;
    const int j = (int)(t / n_inner), k = (int)(t % n_inner);
    const double vj = v[j];
    const double alpha = vj > 0.0 ? (dt / dx) * vj : 0.0;
    const double beta = vj < 0.0 ? (dt / dx) * (-vj) : 0.0;
    const int i = k + 1;
    const double ni = n[i] > kTiny ? n[i] : kTiny;
    const double Ti = Tg[i] > kTiny ? Tg[i] : kTiny;
    const double ui = nu[i] / ni;
    const double inv_tau = (ni * sqrt(Ti)) / tau_tilde;
    dd[t] = 1.0 + alpha + beta + dt * inv_tau;
    dl[t] = k == 0 ? 0.0 : -alpha;
    du[t] = k == n_inner - 1 ? 0.0 : -beta;
    const double diff = vj - ui;
    const double fM = ni * inv_sqrt_2pi / sqrt(Ti) * exp(-0.5 * diff * diff / Ti);
    double rhs = B0[t] + dt * inv_tau * fM;
    if (k == 0) rhs += alpha * fl[j];
    if (k == n_inner - 1) rhs += beta * fr[j];
    B[t] = rhs;
}

// ---- K3: batched general tridiagonal solve ---------------------------------
// Thomas without pivoting, pivot floor +-1e-300 (the CPU twin's semantics,
// cpu_kernel/BGK1D1V/gtsv_cpu/gtsv_binding.cpp:32-37, 51-97); one thread per
// system, modified super-diagonal kept in the workspace (d is not modified).
__global__ void __launch_bounds__(128) gtsv_kernel(const double* __restrict__ dl,
                                                   const double* __restrict__ d,
                                                   const double* __restrict__ du,
                                                   double* __restrict__ B, int n, int batch,
                                                   double* __restrict__ cp) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const size_t o = (size_t)b * n;
    auto piv = [](double x) {
        if (fabs(x) >= 1.0e-300) return x;
        return x < 0.0 ? -1.0e-300 : 1.0e-300;
    };
    // forward elimination exactly as the CPU twin: d'_i = d_i - w du_{i-1}
    double dprev = d[o];
    cp[o] = dprev;
    for (int i = 1; i < n; ++i) {
        const double w = dl[o + i] / piv(dprev);
        const double di = d[o + i] - w * du[o + i - 1];
        B[o + i] -= w * B[o + i - 1];
        cp[o + i] = di;
        dprev = di;
    }
    B[o + n - 1] /= piv(cp[o + n - 1]);
    for (int i = n - 1; i-- > 0;) B[o + i] = (B[o + i] - du[o + i] * B[o + i + 1]) / piv(cp[o + i]);
}

// ---- K5: batched 3x3 block-tridiagonal solve -------------------------------
__device__ __forceinline__ void m3mul(const double* A, const double* B, double* C) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ __forceinline__ void m3vec(const double* A, const double* x, double* y) {
#pragma unroll
    for (int i = 0; i < 3; ++i) y[i] = A[3 * i] * x[0] + A[3 * i + 1] * x[1] + A[3 * i + 2] * x[2];
}
// Adjugate inverse; |det| < 1e-30 -> zero matrix
// (lo_blocktridiag/block_tridiag_kernel.cu:32-68, 248-250 convention).
__device__ __forceinline__ void m3inv(const double* M, double* Mi) {
    const double a00 = M[0], a01 = M[1], a02 = M[2], a10 = M[3], a11 = M[4], a12 = M[5],
                 a20 = M[6], a21 = M[7], a22 = M[8];
    const double c00 = (a11 * a22 - a12 * a21), c01 = -(a10 * a22 - a12 * a20),
                 c02 = (a10 * a21 - a11 * a20);
    const double c10 = -(a01 * a22 - a02 * a21), c11 = (a00 * a22 - a02 * a20),
                 c12 = -(a00 * a21 - a01 * a20);
    const double c20 = (a01 * a12 - a02 * a11), c21 = -(a00 * a12 - a02 * a10),
                 c22 = (a00 * a11 - a01 * a10);
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (!(fabs(det) >= 1e-30)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) Mi[k] = 0.0;
        return;
    }
    const double id = 1.0 / det;
    Mi[0] = c00 * id; Mi[1] = c10 * id; Mi[2] = c20 * id;
    Mi[3] = c01 * id; Mi[4] = c11 * id; Mi[5] = c21 * id;
    Mi[6] = c02 * id; Mi[7] = c12 * id; Mi[8] = c22 * id;
}

// Partition method for batched 3x3 block-tridiagonal systems
//   A_i x_{i-1} + B_i x_i + C_i x_{i+1} = D_i,   i = 0 .. n-1 (A_0, C_{n-1} ignored).
// Rows are cut into K chunks of L rows.  Per chunk (one thread), the rows
// s..e-1 before the chunk's last row e are eliminated by block Thomas with
// the chunk's two interface unknowns xi_{k-1} = x_{s-1} and xi_k = x_e moved
// to the right-hand side, giving x_i = y_i + P_i xi_{k-1} + Q_i xi_k.  The
// chunks' last rows then form a K-row block-tridiagonal system in the xi,
// solved by parallel cyclic reduction in one CTA per system; a last pass
// recovers every x_i.  Singular 3x3 pivots (|det| < 1e-30) contribute a zero
// inverse, the convention of lo_blocktridiag/block_tridiag_kernel.cu:32-68.
struct BtGeo {
    int L, K;
};
__host__ __device__ inline BtGeo bt_geo(int n) {
    BtGeo g;
    int L = (n + 127) / 128;
    if (L < 8) L = 8;
    g.L = L;
    g.K = (n + L - 1) / L;
    return g;
}
constexpr int kBtRep = 21;  // y (3) | P (3x3) | Q (3x3) per row

__global__ void __launch_bounds__(64) bt_local_kernel(const double* __restrict__ A,
                                                      const double* __restrict__ Bm,
                                                      const double* __restrict__ C,
                                                      const double* __restrict__ D, int n,
                                                      int batch, double* __restrict__ rep,
                                                      double* __restrict__ cpw) {
    const BtGeo G = bt_geo(n);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)batch * G.K) return;
    const int b = (int)(t / G.K), k = (int)(t % G.K);
    const int s = k * G.L;
    const int e = (s + G.L < n ? s + G.L : n) - 1;
    const size_t mo = (size_t)b * n * 9, vo = (size_t)b * n * 3;
    double* R = rep + (size_t)b * n * kBtRep;
    double* Cp = cpw + (size_t)b * n * 9;
    const int nloc = e - s;  // rows s..e-1
    // forward sweep: R'_i = M_i^-1 (R_i - A_i R'_{i-1}), C'_i = M_i^-1 C_i
    for (int r = 0; r < nloc; ++r) {
        const int i = s + r;
        const double* Ai = A + mo + 9 * (size_t)i;
        double M[9], ry[3], rP[9], rQ[9];
        if (r == 0) {
            for (int q = 0; q < 9; ++q) M[q] = Bm[mo + 9 * (size_t)i + q];
            for (int q = 0; q < 3; ++q) ry[q] = D[vo + 3 * (size_t)i + q];
            for (int q = 0; q < 9; ++q) rP[q] = (k == 0) ? 0.0 : -Ai[q];
            for (int q = 0; q < 9; ++q) rQ[q] = 0.0;
        } else {
            double T9[9], t3[3];
            m3mul(Ai, Cp + 9 * (size_t)(i - 1), T9);
            for (int q = 0; q < 9; ++q) M[q] = Bm[mo + 9 * (size_t)i + q] - T9[q];
            const double* Rp = R + kBtRep * (size_t)(i - 1);
            m3vec(Ai, Rp, t3);
            for (int q = 0; q < 3; ++q) ry[q] = D[vo + 3 * (size_t)i + q] - t3[q];
            m3mul(Ai, Rp + 3, T9);
            for (int q = 0; q < 9; ++q) rP[q] = -T9[q];
            m3mul(Ai, Rp + 12, T9);
            for (int q = 0; q < 9; ++q) rQ[q] = -T9[q];
        }
        if (r == nloc - 1)
            for (int q = 0; q < 9; ++q) rQ[q] -= C[mo + 9 * (size_t)i + q];
        double Mi[9];
        m3inv(M, Mi);
        double* Ro = R + kBtRep * (size_t)i;
        m3vec(Mi, ry, Ro);
        m3mul(Mi, rP, Ro + 3);
        m3mul(Mi, rQ, Ro + 12);
        if (r < nloc - 1) m3mul(Mi, C + mo + 9 * (size_t)i, Cp + 9 * (size_t)i);
    }
    // backward sweep: x_i = R'_i - C'_i x_{i+1}
    for (int r = nloc - 2; r >= 0; --r) {
        const int i = s + r;
        double* Ro = R + kBtRep * (size_t)i;
        const double* Rn = R + kBtRep * (size_t)(i + 1);
        const double* Ci = Cp + 9 * (size_t)i;
        double t3[3], T9[9];
        m3vec(Ci, Rn, t3);
        for (int q = 0; q < 3; ++q) Ro[q] -= t3[q];
        m3mul(Ci, Rn + 3, T9);
        for (int q = 0; q < 9; ++q) Ro[3 + q] -= T9[q];
        m3mul(Ci, Rn + 12, T9);
        for (int q = 0; q < 9; ++q) Ro[12 + q] -= T9[q];
    }
    // the chunk's last row is its interface unknown: y = 0, P = 0, Q = I
    double* Re = R + kBtRep * (size_t)e;
    for (int q = 0; q < kBtRep; ++q) Re[q] = 0.0;
    Re[12] = Re[16] = Re[20] = 1.0;
}

struct BtRed {
    double al[9], be[9], ga[9], de[3];
};

__global__ void __launch_bounds__(128) bt_reduced_kernel(const double* __restrict__ A,
                                                         const double* __restrict__ Bm,
                                                         const double* __restrict__ C,
                                                         const double* __restrict__ D, int n,
                                                         const double* __restrict__ rep,
                                                         double* __restrict__ xi) {
    extern __shared__ __align__(16) unsigned char bt_smem[];
    const BtGeo G = bt_geo(n);
    const int b = blockIdx.x, K = G.K;
    BtRed* buf[2] = {reinterpret_cast<BtRed*>(bt_smem), reinterpret_cast<BtRed*>(bt_smem) + K};
    const size_t mo = (size_t)b * n * 9, vo = (size_t)b * n * 3;
    const double* R = rep + (size_t)b * n * kBtRep;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int s = k * G.L;
        const int e = (s + G.L < n ? s + G.L : n) - 1;
        const double* Ae = A + mo + 9 * (size_t)e;
        const double* Be = Bm + mo + 9 * (size_t)e;
        const double* Ce = C + mo + 9 * (size_t)e;
        double pm[kBtRep], nx_[kBtRep];
        for (int q = 0; q < kBtRep; ++q) pm[q] = 0.0;
        if (e > s) {
            for (int q = 0; q < kBtRep; ++q) pm[q] = R[kBtRep * (size_t)(e - 1) + q];
        } else {
            pm[3] = pm[7] = pm[11] = 1.0;  // x_{e-1} = xi_{k-1}
        }
        for (int q = 0; q < kBtRep; ++q) nx_[q] = 0.0;
        const bool has_next = k + 1 < K;
        if (has_next)
            for (int q = 0; q < kBtRep; ++q) nx_[q] = R[kBtRep * (size_t)(e + 1) + q];
        double Aeff[9], Ceff[9];
        for (int q = 0; q < 9; ++q) {
            Aeff[q] = (e == 0) ? 0.0 : Ae[q];
            Ceff[q] = has_next ? Ce[q] : 0.0;
        }
        BtRed r;
        double T9[9], U9[9], t3[3], u3[3];
        m3mul(Aeff, pm + 3, r.al);
        m3mul(Aeff, pm + 12, T9);
        m3mul(Ceff, nx_ + 3, U9);
        for (int q = 0; q < 9; ++q) r.be[q] = Be[q] + T9[q] + U9[q];
        m3mul(Ceff, nx_ + 12, r.ga);
        m3vec(Aeff, pm, t3);
        m3vec(Ceff, nx_, u3);
        for (int q = 0; q < 3; ++q) r.de[q] = D[vo + 3 * (size_t)e + q] - t3[q] - u3[q];
        buf[0][k] = r;
    }
    __syncthreads();
    int cur = 0;
    for (int sd = 1; sd < K; sd <<= 1) {
        for (int k = threadIdx.x; k < K; k += blockDim.x) {
            const BtRed& me = buf[cur][k];
            BtRed nw = me;
            double bi[9], e1[9], T9[9], t3[3];
            if (k - sd >= 0) {
                const BtRed& lo = buf[cur][k - sd];
                m3inv(lo.be, bi);
                m3mul(me.al, bi, e1);
                m3mul(e1, lo.al, T9);
                for (int q = 0; q < 9; ++q) nw.al[q] = -T9[q];
                m3mul(e1, lo.ga, T9);
                for (int q = 0; q < 9; ++q) nw.be[q] -= T9[q];
                m3vec(e1, lo.de, t3);
                for (int q = 0; q < 3; ++q) nw.de[q] -= t3[q];
            } else {
                for (int q = 0; q < 9; ++q) nw.al[q] = 0.0;
            }
            if (k + sd < K) {
                const BtRed& hi = buf[cur][k + sd];
                m3inv(hi.be, bi);
                m3mul(me.ga, bi, e1);
                m3mul(e1, hi.ga, T9);
                for (int q = 0; q < 9; ++q) nw.ga[q] = -T9[q];
                m3mul(e1, hi.al, T9);
                for (int q = 0; q < 9; ++q) nw.be[q] -= T9[q];
                m3vec(e1, hi.de, t3);
                for (int q = 0; q < 3; ++q) nw.de[q] -= t3[q];
            } else {
                for (int q = 0; q < 9; ++q) nw.ga[q] = 0.0;
            }
            buf[cur ^ 1][k] = nw;
        }
        __syncthreads();
        cur ^= 1;
    }
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double bi[9];
        m3inv(buf[cur][k].be, bi);
        m3vec(bi, buf[cur][k].de, xi + ((size_t)b * K + k) * 3);
    }
}

__global__ void __launch_bounds__(128) bt_recover_kernel(int n, int batch,
                                                         const double* __restrict__ rep,
                                                         const double* __restrict__ xi,
                                                         double* __restrict__ X) {
    const BtGeo G = bt_geo(n);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)batch * n) return;
    const int b = (int)(t / n), i = (int)(t % n);
    const int k = i / G.L;
    const double* R = rep + ((size_t)b * n + i) * kBtRep;
    const double* xl = xi + ((size_t)b * G.K + (k > 0 ? k - 1 : 0)) * 3;
    const double* xr = xi + ((size_t)b * G.K + k) * 3;
    double out[3], a3[3], c3[3];
    m3vec(R + 3, xl, a3);
    m3vec(R + 12, xr, c3);
    for (int q = 0; q < 3; ++q) out[q] = R[q] + (k > 0 ? a3[q] : 0.0) + c3[q];
    for (int q = 0; q < 3; ++q) X[((size_t)b * n + i) * 3 + q] = out[q];
}

// ---- Maxwellian of per-row moments -----------------------------------------
// bgk1d_utils/general/bgk1d_maxwellian.py:7-33, element for element:
// coeff = n/sqrt(2 pi T) (n * inv_sqrt_2pi / sqrt(T)), e = (v-u)^2 * (-0.5/T),
// f = exp(e) * coeff.  One thread per (i, j), j fastest (coalesced rows).
__global__ void __launch_bounds__(256) maxwellian_kernel(const double* __restrict__ n,
                                                         const double* __restrict__ u,
                                                         const double* __restrict__ T,
                                                         const double* __restrict__ v, int nx,
                                                         int nv, double* __restrict__ f) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * nv) return;
    const int i = (int)(t / nv), j = (int)(t % nv);
    const double Ti = T[i];
    const double coeff = (n[i] * kInvSqrt2Pi) / sqrt(Ti);
    const double invT = 0.5 / Ti;
    const double d = v[j] - u[i];
    f[t] = exp((d * d) * (-invT)) * coeff;
}

// ---- raw velocity moments (no clamps) ---------------------------------------
// Row densities of mass, momentum and energy: (sum f dv, sum f v dv,
// sum f v^2/2 dv), one warp per row, fixed butterfly order.  Used for the
// conservation totals of a state and as calculate_moments' raw sums
// (bgk1d_utils/general/bgk1d_compute_moments.py:7-17).
__global__ void __launch_bounds__(256) row_moments_kernel(const double* __restrict__ f,
                                                          const double* __restrict__ v, int nx,
                                                          int nv, double dv,
                                                          double* __restrict__ out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nx) return;
    const double* row = f + (size_t)warp * nv;
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;
    for (int j = lane; j < nv; j += 32) {
        const double x = row[j], vj = v[j];
        p0 += x;
        p1 += x * vj;
        p2 += x * (vj * vj);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p0 += __shfl_xor_sync(0xffffffffu, p0, o);
        p1 += __shfl_xor_sync(0xffffffffu, p1, o);
        p2 += __shfl_xor_sync(0xffffffffu, p2, o);
    }
    if (lane == 0) {
        out[3 * (size_t)warp + 0] = p0 * dv;
        out[3 * (size_t)warp + 1] = p1 * dv;
        out[3 * (size_t)warp + 2] = 0.5 * (p2 * dv);
    }
}

// Evaluates the device math helpers on an array (numerical self-test).
__global__ void math_selftest_kernel(int kind, const double* __restrict__ x, double* __restrict__ y,
                                     int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y[i] = kind == 0 ? exp_nonpos(x[i]) : recip_ge1(x[i]);
}

}  // namespace keq

namespace {
keq_status launch_status() {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        return KEQ_ERR_CUDA;
    }
    return KEQ_OK;
}
}  // namespace

extern "C" {

keq_status keq_moments_n_nu_T(const double* f, const double* v, int32_t nx, int32_t nv, double dv,
                              double* n, double* nu, double* T, keq_stream_t stream) {
    if (!f || !v || !n || !nu || !T || nx < 1 || nv < 1) return KEQ_ERR_INVALID;
    const long long threads = (long long)nx * 32;
    const int blocks = (int)((threads + 255) / 256);
    keq::moments_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(f, v, nx, nv,
                                                                                   dv, n, nu, T);
    return launch_status();
}

keq_status keq_build_system_from_moments(const double* B0, const double* v, int32_t nx,
                                         int32_t nv, double dt, double dx, double tau_tilde,
                                         double inv_sqrt_2pi, const double* n, const double* nu,
                                         const double* T, const double* f_bc_l,
                                         const double* f_bc_r, double* dl, double* dd,
                                         double* du, double* B, keq_stream_t stream) {
    if (!B0 || !v || !n || !nu || !T || !f_bc_l || !f_bc_r || !dl || !dd || !du || !B)
        return KEQ_ERR_INVALID;
    if (nx < 3 || nv < 1) return KEQ_ERR_INVALID;
    const long long total = (long long)(nx - 2) * nv;
    const int blocks = (int)((total + 255) / 256);
    keq::build_system_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        B0, v, n, nu, T, f_bc_l, f_bc_r, nx, nv, dt, dx, tau_tilde, inv_sqrt_2pi, dl, dd, du, B);
    return launch_status();
}

keq_status keq_maxwellian(const double* n, const double* u, const double* T, const double* v,
                          int32_t nx, int32_t nv, double* f, keq_stream_t stream) {
    if (!n || !u || !T || !v || !f || nx < 1 || nv < 1) return KEQ_ERR_INVALID;
    const long long total = (long long)nx * nv;
    keq::maxwellian_kernel<<<(unsigned)((total + 255) / 256), 256, 0,
                             reinterpret_cast<cudaStream_t>(stream)>>>(n, u, T, v, nx, nv, f);
    return launch_status();
}

keq_status keq_row_moments(const double* f, const double* v, int32_t nx, int32_t nv, double dv,
                           double* out, keq_stream_t stream) {
    if (!f || !v || !out || nx < 1 || nv < 1) return KEQ_ERR_INVALID;
    const long long threads = (long long)nx * 32;
    keq::row_moments_kernel<<<(unsigned)((threads + 255) / 256), 256, 0,
                              reinterpret_cast<cudaStream_t>(stream)>>>(f, v, nx, nv, dv, out);
    return launch_status();
}

keq_status keq_math_selftest(int32_t kind, const double* x, double* y, int32_t n,
                             keq_stream_t stream) {
    if (!x || !y || n < 0 || (kind != 0 && kind != 1)) return KEQ_ERR_INVALID;
    if (n == 0) return KEQ_OK;
    keq::math_selftest_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        kind, x, y, n);
    return launch_status();
}

keq_status keq_gtsv_workspace_size(int32_t n, int32_t batch, size_t* bytes) {
    if (!bytes || n < 0 || batch < 0) return KEQ_ERR_INVALID;
    *bytes = sizeof(double) * (size_t)(n > 0 ? n : 1) * (size_t)(batch > 0 ? batch : 1);
    return KEQ_OK;
}

keq_status keq_gtsv_strided_inplace(const double* dl, const double* d, const double* du,
                                    double* B, int32_t n, int32_t batch, void* workspace,
                                    size_t workspace_bytes, keq_stream_t stream) {
    if (n < 0 || batch < 0) return KEQ_ERR_INVALID;
    if (n == 0 || batch == 0) return KEQ_OK;
    if (!dl || !d || !du || !B || !workspace) return KEQ_ERR_INVALID;
    size_t need = 0;
    keq_gtsv_workspace_size(n, batch, &need);
    if (workspace_bytes < need || reinterpret_cast<uintptr_t>(workspace) % 8)
        return KEQ_ERR_WORKSPACE;
    keq::gtsv_kernel<<<(batch + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        dl, d, du, B, n, batch, static_cast<double*>(workspace));
    return launch_status();
}

keq_status keq_block_tridiag_workspace_size(int32_t n, int32_t batch, size_t* bytes) {
    if (!bytes || n < 0 || batch < 0) return KEQ_ERR_INVALID;
    const size_t nn = (size_t)(n > 0 ? n : 1), bb = (size_t)(batch > 0 ? batch : 1);
    const keq::BtGeo G = keq::bt_geo(n > 0 ? n : 1);
    *bytes = sizeof(double) * (nn * bb * (keq::kBtRep + 9) + (size_t)G.K * bb * 3) + 256;
    return KEQ_OK;
}

keq_status keq_block_tridiag_solve(const double* A, const double* B, const double* C,
                                   const double* D, double* X, int32_t n, int32_t batch,
                                   void* workspace, size_t workspace_bytes,
                                   keq_stream_t stream) {
    if (n < 0 || batch < 0) return KEQ_ERR_INVALID;
    if (n == 0 || batch == 0) return KEQ_OK;
    if (!A || !B || !C || !D || !X || !workspace) return KEQ_ERR_INVALID;
    size_t need = 0;
    keq_block_tridiag_workspace_size(n, batch, &need);
    if (workspace_bytes < need || reinterpret_cast<uintptr_t>(workspace) % 8)
        return KEQ_ERR_WORKSPACE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const keq::BtGeo G = keq::bt_geo(n);
    double* rep = static_cast<double*>(workspace);
    double* cpw = rep + (size_t)n * batch * keq::kBtRep;
    double* xi = cpw + (size_t)n * batch * 9;
    const long long nloc = (long long)batch * G.K;
    keq::bt_local_kernel<<<(unsigned)((nloc + 63) / 64), 64, 0, s>>>(A, B, C, D, n, batch, rep, cpw);
    const size_t smem = 2 * sizeof(keq::BtRed) * (size_t)G.K;
    cudaFuncSetAttribute(keq::bt_reduced_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    keq::bt_reduced_kernel<<<batch, 128, smem, s>>>(A, B, C, D, n, rep, xi);
    const long long nrow = (long long)batch * n;
    keq::bt_recover_kernel<<<(unsigned)((nrow + 127) / 128), 128, 0, s>>>(n, batch, rep, xi, X);
    return launch_status();
}

}  // extern "C"
