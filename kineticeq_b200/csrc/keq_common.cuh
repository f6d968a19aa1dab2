// keq_common.cuh -- device utilities shared by the sm_100a kernels:
// memory-ordering primitives, the bounded grid barrier of the persistent
// kernels, NaN-aware max reductions and the warp reduce-scatter used for the
// per-row velocity moments.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/keq_b200.h"

namespace keq {

constexpr int kLanes = 32;                 // velocities per tile (one warp width)
constexpr double kTiny = 1.0e-300;         // clamp of n and T in the moment kernels
constexpr double kInvSqrt2Pi = 0.39894228040143267794;  // 1/sqrt(2 pi), correctly rounded
// Default spin limit of every device-side wait (each poll sleeps ~32-256 ns):
// a few seconds at most before the wait gives up and reports KEQ_ERR_TIMEOUT.
// Plans carry their own copy (keq_plan_set_spin_limit) so that a test can make
// a wait run out without hanging anything.
constexpr unsigned long long kSpinLimit = 1ull << 25;

// Polling load without ordering; a wait that ends on it is followed by
// fence_gpu() (relaxed load + fence = acquire), so each poll costs no L1
// invalidation.
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

// Non-negative doubles (and +NaN) order like their bit patterns, so the max
// of a residual can be accumulated with an integer atomicMax.  NaN (0x7ff8..)
// sorts above +Inf, i.e. a NaN residual wins, as torch.max propagates NaN.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ double nan_max(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ll);
    return a > b ? a : b;
}

// 1/d by Newton-Raphson iteration r <- r + r (1 - d r) (quadratic
// convergence) from a single-precision seed: the seed's relative error is
// below 2^-22, two steps bring it below 2^-80, so the result is within one
// rounding of 1/d.  Valid for 2^-120 < |d| < 2^120; outside that range the
// IEEE division is used.
__device__ __forceinline__ double recip_nr(double d) {
    const double ad = fabs(d);
    if (!(ad > 7.5e-37 && ad < 1.3e36)) return 1.0 / d;
    double r = (double)__frcp_rn((float)d);
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// 1/d for d >= 1 (the implicit diagonal 1 + alpha + beta + dt/tau), branch
// and conversion free: Newton-Raphson r <- r + r (1 - d r) twice from the
// hardware reciprocal approximation rcp.approx.ftz.f64 (relative error below
// 2^-20, so two steps leave < 2^-80 before the final rounding).
__device__ __forceinline__ double recip_ge1(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// e^x for x <= 0, branch and conversion free (so that independent
// evaluations interleave at full FP64 issue rate).  Cody-Waite argument
// reduction x = k ln2 + r with ln2 split into a 32-bit head (exact products
// k*LN2_HI for |k| < 2^21) and a tail, |r| <= ln2/2; k is rounded with the
// 1.5*2^52 addition trick and read from the low word of the sum; then the
// degree-13 Taylor polynomial of e^r (truncation < 5e-18 relative) by Horner's
// rule, and the scale 2^k built in the exponent field (two factors below
// 2^-1000 so that subnormal results round once).  NaN propagates, -inf and
// x < -745.5 give 0.  Accuracy is checked against CUDA's exp in the tests.
__device__ __forceinline__ double exp_nonpos(double x) {
    constexpr double LOG2E = 1.4426950408889634;
    constexpr double LN2_HI = 0.6931471806019545;       // 0x3fe62e42ff000000
    constexpr double LN2_LO = -4.2009150726810846e-11;  // ln2 - LN2_HI
    constexpr double ROUND = 6755399441055744.0;         // 1.5 * 2^52
    const double xc = (x < -745.5) ? -745.5 : x;
    const double kr = fma(xc, LOG2E, ROUND);              // k in the low mantissa bits
    const int ki = __double2loint(kr);                    // k in [-1076, 0]
    const double k = kr - ROUND;
    double r = fma(-k, LN2_HI, xc);
    r = fma(-k, LN2_LO, r);
    double p = 1.6059043836821613e-10;   // 1/13!
    p = fma(p, r, 2.08767569878681e-09);  // 1/12!
    p = fma(p, r, 2.505210838544172e-08);
    p = fma(p, r, 2.755731922398589e-07);
    p = fma(p, r, 2.7557319223985893e-06);
    p = fma(p, r, 2.48015873015873e-05);
    p = fma(p, r, 0.0001984126984126984);
    p = fma(p, r, 0.001388888888888889);
    p = fma(p, r, 0.008333333333333333);
    p = fma(p, r, 0.041666666666666664);
    p = fma(p, r, 0.16666666666666666);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const bool sub = ki < -1000;
    const int e1 = sub ? ki + 60 : ki;
    const double s1 = __hiloint2double((e1 + 1023) << 20, 0);
    const double s2 = sub ? 8.673617379884035e-19 : 1.0;  // 2^-60
    return (p * s1) * s2;
}

// Running maximum of ratios num/den without a division per element: the
// maximum is kept as a fraction and compared by cross-multiplication
// (num_a * den_b > num_b * den_a for positive finite denominators).
// Elements with a zero, infinite or NaN denominator or numerator take an
// exact slow path (IEEE division, NaN-propagating max), so the result equals
// max_i(num_i / den_i) as torch.max computes it, up to one rounding.
struct FracMax {
    double num, den, special;
    __device__ __forceinline__ FracMax() : num(0.0), den(1.0), special(0.0) {}
    __device__ __forceinline__ void add(double a, double b) {
        if (b > 0.0 && b < 1.0e300 && a >= 0.0 && a < 1.0e300) {
            if (a * den > num * b) {
                num = a;
                den = b;
            }
        } else {
            const double q = a / b;
            special = (q != q || special != special) ? q + special : (q > special ? q : special);
        }
    }
    // The common case of add() without a branch: finite a >= 0 and a finite
    // positive b.  Returns false (and changes nothing) otherwise; the caller
    // then redoes its inputs with add(), which is idempotent for a max.
    __device__ __forceinline__ bool add_normal(double a, double b) {
        const bool normal = b > 0.0 && b < 1.0e300 && a >= 0.0 && a < 1.0e300;
        const bool take = normal && (a * den > num * b);
        num = take ? a : num;
        den = take ? b : den;
        return normal;
    }
    __device__ __forceinline__ double value() const {
        const double q = num / den;
        if (special != special) return special;
        return q > special ? q : special;
    }
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Number of leading entries equal to 1 in flags[0..n) (the iterations that
// ran), by a whole warp: 32 flags per load round, first miss by ballot.
__device__ __forceinline__ int count_leading_ones(const int* flags, int n) {
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < n; base += 32) {
        const int q = base + lane;
        const bool miss = q >= n || __ldcg(&flags[q]) != 1;
        const unsigned mm = __ballot_sync(0xffffffffu, miss);
        if (mm != 0u) return base + __ffs(mm) - 1 < n ? base + __ffs(mm) - 1 : n;
    }
    return n;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Grid barrier for a cooperative launch.  One arrival per CTA on a counter
// that only grows within a launch (the host zeroes it before each launch):
// the k-th barrier is passed once the counter reaches k * nblocks, and an
// arriving CTA learns k from the value its own arrival returns (arrivals of
// barrier k lie in [(k-1) nblocks, k nblocks) because no CTA can arrive at
// barrier k+1 before barrier k is passed).  The arrival is a release; the
// wait polls relaxed and ends with an acq_rel fence (the last arriver, which
// does not wait, fences too), so stores made by any thread of any CTA before
// the barrier are visible to every thread after it (the CTA's bar.sync
// carries the ordering to and from thread 0); the fence also invalidates
// the SM's L1 for the ordinary loads that follow.  No word is reset between
// barriers, which saves the release round trip of a generation counter.
// Every wait is bounded: on timeout the CTA records KEQ_ERR_TIMEOUT in *err
// and the caller leaves its loop.
struct GridBarrier {
    unsigned count;
    unsigned pad;
};

__device__ __forceinline__ unsigned atom_add_release(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ bool grid_sync(GridBarrier* gb, unsigned nblocks, int* err,
                                          unsigned long long limit = kSpinLimit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned old = atom_add_release(&gb->count, 1u);
        const unsigned target = (old / nblocks + 1u) * nblocks;
        if (old + 1u != target) {
            unsigned long long it = 0;
            unsigned ns = 0;
            while ((int)(ld_relaxed(&gb->count) - target) < 0) {
                if (++it > limit) {
                    atomicOr(err, 1 << KEQ_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                if (ns) __nanosleep(ns);
                ns = ns ? (ns < 128 ? 2 * ns : ns) : 16;
            }
        }
        if (ok) fence_gpu();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Common head of every persistent-kernel plan's device header.  The first
// 16 bytes ({bar, err, err_sticky}) are the launch state: keq_plan_step
// clears bar and err before every launch, so a launch that gave up on a wait
// (and left the barrier count behind) cannot poison the next one;
// err_sticky accumulates the error bits of all launches until
// keq_plan_reset.
struct PlanHead {
    GridBarrier bar;
    int err;
    int err_sticky;
    unsigned long long spin_limit;
    unsigned long long seq;     // launch sequence (epochs of look-back flags)
    unsigned long long* trace;  // optional phase trace (profiling aid)
    int trace_iters;
    int fresh;                  // 1 until the first launch completes: stats totals start at 0
};

// Warp reduce-scatter of ROWS x Q partial sums held by every lane
// (acc[r*Q + q]).  On return lanes holding row r (see owner_row()) carry the
// warp-wide sums of that row in acc[0..Q-1].  The combination order is fixed
// (butterfly on lane bits 4..0), so results are reproducible.
//   ROWS must be a power of two <= 32.
template <int ROWS, int Q>
__device__ __forceinline__ void warp_reduce_scatter(double (&acc)[ROWS * Q], int lane) {
    // Level lvl uses lane bit (16 >> lvl).  While more than one row is left
    // the row set is halved; afterwards the remaining bits all-reduce.
#pragma unroll
    for (int lvl = 0; lvl < 5; ++lvl) {
        const int bit = 16 >> lvl;
        const int nrows = (ROWS >> lvl) > 0 ? (ROWS >> lvl) : 1;
        if (nrows > 1) {
            const int half = nrows >> 1;
            const bool upper = (lane & bit) != 0;
#pragma unroll
            for (int r = 0; r < half; ++r) {
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const double lo = acc[r * Q + q];
                    const double hi = acc[(r + half) * Q + q];
                    const double mine = upper ? hi : lo;
                    const double send = upper ? lo : hi;
                    acc[r * Q + q] = mine + __shfl_xor_sync(0xffffffffu, send, bit);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], bit);
        }
    }
}

// Row owned by `lane` after warp_reduce_scatter<ROWS,Q>: lane bit 4 is the
// most significant bit of the row index, then bit 3, ...
template <int ROWS>
__device__ __forceinline__ int owner_row(int lane) {
    int row = 0;
#pragma unroll
    for (int lvl = 0; lvl < 5; ++lvl) {
        const int nrows = (ROWS >> lvl) > 0 ? (ROWS >> lvl) : 1;
        if (nrows > 1 && (lane & (16 >> lvl))) row += nrows >> 1;
    }
    return row;
}

// True for the single lane that writes row owner_row(lane): the lane bits
// not used for the row id are zero.
template <int ROWS>
__device__ __forceinline__ bool owner_writes(int lane) {
    int lvls = 0;
#pragma unroll
    for (int n = ROWS; n > 1; n >>= 1) ++lvls;
    const int low_mask = (1 << (5 - lvls)) - 1;
    return (lane & low_mask) == 0;
}

}  // namespace keq
