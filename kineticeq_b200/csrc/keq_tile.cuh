// keq_tile.cuh -- the velocity-tile machinery shared by the persistent step
// kernels (implicit Picard and HOLO distribution solve).
//
// Both steps solve, per velocity v_j, a first-order upwind recurrence along x
//     x_s = a_s x_{s-1} + c_s,   s = 0 .. n_inner-1 in scan order,
// with x_{-1} the fixed boundary value (row 0 for v > 0, row nx-1 for v <= 0;
// the scan runs forward in x for v > 0 and backward for v <= 0).  A warp
// owns a tile of 32 consecutive velocities (one per lane; tiles are split at
// the sign change of v so each scans one way) by R consecutive scan
// positions (a "chunk").  Tiles are processed in one pass with a decoupled
// look-back between the chunks of a velocity column:
//   1. the tile composes its rows into the affine map x_out = P x_in + Y and
//      publishes (P, Y) with an "aggregate" flag;
//   2. it polls up to 32 predecessor chunks at once, takes the nearest one
//      that has published its inclusive value (the carry out of that chunk),
//      pushes it through the aggregates of the chunks in between in x order,
//      and publishes its own inclusive value x_in P + Y;
//   3. it runs the recurrence from the carry.
// Every inclusive value is defined by incl(c) = fma(P_c, incl(c-1), Y_c)
// whatever path the look-back takes (maps are always applied to values,
// never composed with each other), so the result does not depend on timing.
// Flags carry an epoch (launch sequence and iteration) so no flag is reset
// between iterations.
#pragma once

#include "keq_common.cuh"

namespace keq {

constexpr int kRmax = 32;   // rows (scan positions) per tile at most
constexpr int kRB = 32;     // rows per row block (unit of the row reductions)
constexpr int kWin = 32;    // predecessor chunks polled per look-back round (one per lane)
constexpr int kWinRounds = 4;  // rounds a look-back may reach back: 128 chunks
constexpr int kPartQ = 4;   // doubles per (v-tile, row) partial: sum x, x v, x v^2, x v^3
constexpr unsigned long long kFlagAgg = 1ull, kFlagInc = 2ull;

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

struct TileGeo {
    bool pos;      // velocities > 0: forward scan
    bool lane_ok;  // this lane's velocity exists
    int j;         // this lane's velocity index
    int s0;        // first scan position of the tile
    int nrows;     // scan positions in the tile (<= R)
};

__device__ __forceinline__ TileGeo tile_geo(int nt_neg, int kp, int nv, int n_inner, int R, int vt,
                                            int c, int lane) {
    TileGeo g;
    g.pos = vt >= nt_neg;
    g.j = g.pos ? kp + 32 * (vt - nt_neg) + lane : kp - 32 * (vt + 1) + lane;
    g.lane_ok = g.pos ? (g.j < nv) : (g.j >= 0);
    // Chunks of R scan positions cut so that their interior rows start at
    // multiples of R: a forward (v > 0) chunk c holds rows k in [cR, cR + R);
    // a backward scan runs from k = n_inner - 1 down and its chunk 0 takes the
    // remainder n_inner mod R, so that every later backward chunk starts at a
    // multiple of R as well.  With R dividing the row-block size every tile
    // then lies inside one row block.  Both directions have ceil(n_inner / R)
    // chunks.
    const int pad = g.pos ? 0 : (R - n_inner % R) % R;
    g.s0 = c == 0 ? 0 : c * R - pad;
    const int end = (c + 1) * R - pad;
    g.nrows = (end < n_inner ? end : n_inner) - g.s0;
    return g;
}

__device__ __forceinline__ int scan_row(int nx, bool pos, int s) { return pos ? 1 + s : nx - 2 - s; }

// Publish the tile's aggregate map (P, Y) (one value per lane/velocity).
// The warp barrier orders every lane's stores before lane 0's flag store, and
// a release is cumulative over what precedes it, so one release by lane 0
// publishes the whole warp's values (the bar.sync + one-thread fence pattern
// of a grid barrier, at warp level); no per-lane fence is needed.
__device__ __forceinline__ void publish_agg(double* agg, unsigned long long* flag, size_t tid,
                                            double P, double Y, unsigned long long epoch) {
    const int lane = threadIdx.x & 31;
    __stcg(&agg[tid * 64 + lane], P);
    __stcg(&agg[tid * 64 + 32 + lane], Y);
    __syncwarp();
    if (lane == 0) st_release64(&flag[tid], (epoch << 2) | kFlagAgg);
}

// Publish the tile's inclusive value (the carry out of its chunk).
__device__ __forceinline__ void publish_inc(double* inc, unsigned long long* flag, size_t tid,
                                            double X, unsigned long long epoch) {
    const int lane = threadIdx.x & 31;
    __stcg(&inc[tid * 32 + lane], X);
    __syncwarp();
    if (lane == 0) st_release64(&flag[tid], (epoch << 2) | kFlagInc);
}

// Carry into chunk c >= 1 of v-tile column vt (tile index t = chunk * nvt +
// vt).  Round r polls chunks c-1-32r-lane (relaxed; the fence after the wait
// makes it an acquire); the nearest chunk with an inclusive value whose
// successors up to c-1 all have aggregates is the base.  A deeper round is
// polled only when every chunk of the rounds before it has an aggregate but
// none an inclusive value, so a chunk far from the resolved prefix can start
// from an inclusive value up to 128 chunks back instead of waiting for the
// prefix to advance 32 chunks at a time.  Bounded: on timeout returns false
// (X = 0).
__device__ __forceinline__ bool lookback(const double* agg, const double* inc,
                                         const unsigned long long* flag, int nvt, int vt, int c,
                                         unsigned long long epoch, unsigned long long limit,
                                         double& X) {
    const int lane = threadIdx.x & 31;
    const int nval = c < kWin * kWinRounds ? c : kWin * kWinRounds;
    unsigned long long it = 0;
    unsigned ns = 32;
    int q = -1;
    for (;;) {
        // every branch below is warp-uniform (ballot results)
        for (int rd = 0; rd < kWinRounds && rd * kWin < nval; ++rd) {
            const int qq = rd * kWin + lane;
            unsigned long long f = 0ull;
            if (qq < nval) f = ld_relaxed64(&flag[(size_t)(c - 1 - qq) * nvt + vt]);
            const bool cur = (f >> 2) == epoch;
            const unsigned incm = __ballot_sync(0xffffffffu, cur && (f & 3ull) == kFlagInc);
            const unsigned aggm = __ballot_sync(0xffffffffu, cur && (f & 3ull) != 0ull);
            if (incm != 0u) {
                const int qr = __ffs(incm) - 1;
                const unsigned need = (qr == 0) ? 0u : ((1u << qr) - 1u);
                if ((aggm & need) == need) q = rd * kWin + qr;
                break;
            }
            const int left = nval - rd * kWin;
            const unsigned valid = left >= 32 ? 0xffffffffu : ((1u << left) - 1u);
            if ((aggm & valid) != valid) break;  // a missing aggregate: no deeper base
        }
        if (q >= 0) break;
        if (++it > limit) {
            X = 0.0;
            return false;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    // the polling lanes' fence completes their acquire; the warp barrier then
    // orders every lane's loads below after it
    fence_acq_rel();
    __syncwarp();
    double x = __ldcg(&inc[((size_t)(c - 1 - q) * nvt + vt) * 32 + lane]);
    // eight predecessor maps per round, loaded unconditionally (an index past
    // the first is clamped to it and its map replaced by the identity) so that
    // all sixteen loads are in flight together
    for (int k0 = q - 1; k0 >= 0; k0 -= 8) {
        double Pk[8], Yk[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int k = k0 - t >= 0 ? k0 - t : 0;
            const size_t tid = (size_t)(c - 1 - k) * nvt + vt;
            Pk[t] = __ldcg(&agg[tid * 64 + lane]);
            Yk[t] = __ldcg(&agg[tid * 64 + 32 + lane]);
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const bool use = k0 - t >= 0;
            x = fma(use ? Pk[t] : 1.0, x, use ? Yk[t] : 0.0);
        }
    }
    X = x;
    return true;
}

// Sums over the 32 columns of row r of a tile held in shared memory (row
// stride 33 doubles), weighted by the columns' velocities vv (zero for
// absent velocities): s = (sum x, sum x v, sum x v^2, sum x v^3), in column
// order.
__device__ __forceinline__ void row_sums4(const double (*buf)[33], const double* vv, int r,
                                          double* s) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) {
        const double x = buf[r][j];
        const double vj = vv[j];
        const double t1 = x * vj;
        const double t2 = t1 * vj;
        a0 += x;
        a1 += t1;
        a2 += t2;
        a3 = fma(t2, vj, a3);
    }
    s[0] = a0;
    s[1] = a1;
    s[2] = a2;
    s[3] = a3;
}

// Sum of the per-v-tile partials of interior row k over the v-tiles
// [vt0, vt1), in v-tile order (loads issued in batches of B).
template <int B = 8>
__device__ __forceinline__ void sum_partials4(const double* part, int vt0, int vt1, int n_inner,
                                              int k, double* s) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (int v0 = vt0; v0 < vt1; v0 += B) {
        double2 p01[B], p23[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int v = v0 + q < vt1 ? v0 + q : vt1 - 1;  // clamped: every load is issued
            const double* p = part + ((size_t)v * n_inner + k) * kPartQ;
            p01[q] = __ldcg(reinterpret_cast<const double2*>(p));
            p23[q] = __ldcg(reinterpret_cast<const double2*>(p + 2));
        }
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const bool in = v0 + q < vt1;  // a select, not a branch, keeps the loads above
            a0 += in ? p01[q].x : 0.0;
            a1 += in ? p01[q].y : 0.0;
            a2 += in ? p23[q].x : 0.0;
            a3 += in ? p23[q].y : 0.0;
        }
    }
    s[0] = a0;
    s[1] = a1;
    s[2] = a2;
    s[3] = a3;
}

// Row blocks (kRB interior rows each) that a tile's rows complete: adds the
// tile's row count to each overlapped block's arrival counter (rows x
// v-tiles) and returns in done[0..1] the blocks this tile completed (-1 if
// none).  Lane 0 only; the caller broadcasts.
__device__ __forceinline__ void rowblock_arrive(unsigned* cnt, int nx, int n_inner, int nvt,
                                                const TileGeo& g, int* done) {
    done[0] = -1;
    done[1] = -1;
    const int s_lo = g.s0, s_hi = g.s0 + g.nrows - 1;
    const int k_a = scan_row(nx, g.pos, s_lo) - 1, k_b = scan_row(nx, g.pos, s_hi) - 1;
    const int k_lo = k_a < k_b ? k_a : k_b, k_hi = k_a < k_b ? k_b : k_a;
    int nd = 0;
    for (int rb = k_lo / kRB; rb <= k_hi / kRB; ++rb) {
        const int lo = rb * kRB > k_lo ? rb * kRB : k_lo;
        const int hi = (rb + 1) * kRB - 1 < k_hi ? (rb + 1) * kRB - 1 : k_hi;
        const unsigned add = (unsigned)(hi - lo + 1);
        const int rows_in_rb = ((rb + 1) * kRB < n_inner ? (rb + 1) * kRB : n_inner) - rb * kRB;
        const unsigned expect = (unsigned)rows_in_rb * (unsigned)nvt;
        const unsigned prev = atomicAdd(&cnt[rb], add);
        if (prev + add == expect && nd < 2) done[nd++] = rb;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int find_inst(const long long* off, int n, long long t) {
    int lo = 0, hi = n;  // off[lo] <= t < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&off[mid]) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

}  // namespace keq
