// Exact banded elastic distances (src/ElasticMeasures.cpp:24-198, dispatch
// src/fsmeld.cpp:170-183) for candidate windows, one lane per candidate.
//
// Each lane keeps one band row (offsets d = j - i + w, 2w+1 cells, updated in
// place: cell d of the previous row is the diagonal neighbour of cell d and
// the upper neighbour of cell d-1) and a power-of-two ring of its z-normalised
// candidate points, both in shared memory laid out [slot][lane] so lanes never
// share a bank word.  Candidate points are normalised once each, as
// (t - mu) / sigma (src/fsmeld.cpp:823-826, 1202-1204).
//
// Every in-band cell is computed from its three neighbours with the
// reference's formula and operand order.  The reference reads MAX_VAL = 1e18
// (0 for LCSS) for neighbours outside the band; its column 0 of ERP/EDR/MSM
// has its own formula.  Two modes reproduce that:
//
//  * fast mode (every lane, every row, one code path): the ring holds +-1e300
//    for candidate columns outside the matrix, so cells outside the band come
//    out >= 1e18 (0 for LCSS) without a per-cell test, and the column-0 cells
//    reduce to the reference's column formula because their other two terms
//    are >= 1e18.  This equals the reference bit for bit while every in-band
//    value stays below 1e17, which holds when every cost term is below
//    1e17 / (2m+2): guaranteed when |y| <= ylim for every candidate point,
//    ylim = sqrt(1e17 / (2m+2)) - max|x| - |arg| - 2 (EDR/LCSS values are
//    match counts, always in range).
//  * exact mode (a candidate with a point beyond ylim, or a query whose
//    ylim <= 0): the candidate restarts and every row clips the cells outside
//    the band to the sentinel and evaluates column 0 with the reference's
//    column formula, so sentinels are read exactly where the reference reads
//    them whatever the magnitudes.
//
// DTW/LCSS, and MSM in the fast mode, start from a virtual cell (-1,-1) of
// value 0 above a row of sentinels: cell (0,0) becomes its own point distance
// (or match), and MSM's row-0 cells j >= 1 keep only their left term,
// cost[0][j-1] + C(y_j, x_0, y_{j-1}), the reference's row-0 loop
// (src/ElasticMeasures.cpp:182-184).  A fresh candidate's band, ring padding
// and first w+1 points are written by the whole warp, one pass each.
//
// Lanes are independent: each lane advances its own candidate one row per
// step and, when its candidate finishes, takes the next one from a global
// work counter, so lanes never wait for slower neighbours.
//
// Early abandon: every path to the last cell crosses each row and costs only
// add non-negative terms, so the final cost is at least the row's minimum
// plus, for every later row, the GLB's per-point Q->T term (the cheapest way
// to align that query point with the candidate's envelope).  The GLB stage
// hands over each survivor's Q->T sum; the DP subtracts the terms of the rows
// it has done (terms computed without divisions on a slightly narrowed
// envelope, which only loosens the bound).  A candidate whose bound already
// exceeds the cutoff (with a 1e-9 relative slack for round-off) cannot be
// kept and stops.  For LCSS the
// final match count is at most the row maximum plus the matches the
// remaining rows can still reach.  Out-of-band cells can only lower a row
// minimum (raise an LCSS row maximum), which keeps the bound valid.  Results
// are unchanged: only candidates that would be discarded stop early.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

constexpr double kPad = 1e300;  // candidate points outside the matrix (fast mode)

// Cascading abandon margin: the bound and the DP carry independent round-off
// (relative ~1e-13); a 1e-9 relative slack keeps the test conservative.
__device__ __forceinline__ double slack(double cut) { return cut + 1e-9 * (1.0 + fabs(cut)); }

// src/ElasticMeasures.cpp:173-176
__device__ __forceinline__ double msm_c(double np, double x, double y, double c) {
    if ((x <= np && np <= y) || (y <= np && np <= x)) return c;
    const double a = fabs(dsub(np, x)), b = fabs(dsub(np, y));
    return dadd(c, (b < a) ? b : a);
}

// Per-row constants of the query point the row aligns.
struct RowCtx {
    double xi;   // query point of the row
    double c0;   // ERP: dist(x, g); MSM: |x_i - x_{i-1}|
    double xp;   // MSM: x_{i-1}
    bool ge, le; // MSM: x_{i-1} <= x_i, x_i <= x_{i-1}
    int i;       // row
};

// Minimum / maximum by one comparison and a select.  Every DP value here is
// a non-NaN number >= +0 (sums of non-negative terms, match counts, +inf at
// most), so they equal std::min/std::max (and fmin/fmax) on these operands;
// fmin/fmax also handle NaN operands, which costs extra instructions per call.
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// One cell.  pn/pd: the previous row's cells above and diagonally left; left:
// this row's previous cell; y: the candidate point read by the cell (y_j, or
// y[j-1] for ERP/EDR); yprev: y_{j-1} (MSM).
template <int METRIC, bool EXACT>
__device__ __forceinline__ double dp_cell(double pn, double pd, double left, double y, double yprev,
                                          const RowCtx& rc, double arg, int d, int dlo, int dhi, int d0) {
    constexpr double SENT = (METRIC == LCSS) ? 0.0 : kDpMax;
    const double xi = rc.xi;
    double v;
    // the minimum of three non-negative values does not depend on the order:
    // the left neighbour (the previous cell of this row) enters last, so the
    // chain from one cell to the next is one minimum and one add
    if (METRIC == DTW) {
        v = dadd(smin(smin(pn, pd), left), dsq(xi, y));
    } else if (METRIC == ERP) {  // y = y[j-1]
        const double match = dadd(pd, dsq(xi, y));
        const double ins = dadd(left, dsq(y, arg));
        const double del = dadd(pn, rc.c0);
        v = smin(smin(match, del), ins);
        if (EXACT && d == d0) v = del;                       // cur[0] = prev[0] + dist(x, g)
    } else if (METRIC == EDR) {  // y = y[j-1]
        const double sub = (fabs(dsub(xi, y)) <= arg) ? 0.0 : 1.0;
        v = smin(smin(dadd(pn, 1.0), dadd(pd, sub)), dadd(left, 1.0));
        if (EXACT && d == d0) v = (double)rc.i;              // cur[0] = i
    } else if (METRIC == LCSS) {
        // both sides computed, then selected: data-dependent branches here
        // would split the warp cell by cell
        const double hit1 = dadd(pd, 1.0);
        double best = (fabs(dsub(xi, y)) <= arg) ? hit1 : pd;
        best = (best < pn) ? pn : best;
        best = (best < left) ? left : best;
        v = best;
    } else {  // MSM, y = y_j, yprev = y_{j-1}; every term computed, then selected
        const double axy = fabs(dsub(xi, y));
        const double c1 = dadd(pd, axy);
        const bool xle = xi <= y, yle = y <= xi;
        // C(x_i, x_{i-1}, y_j): x_i lies between x_{i-1} and y_j
        const bool b2 = (rc.ge && xle) || (yle && rc.le);
        const double m2 = dadd(arg, smin(rc.c0, axy));
        const double c2 = dadd(pn, b2 ? arg : m2);
        // C(y_j, x_i, y_{j-1}): y_j lies between x_i and y_{j-1}
        const bool b3 = (xle && y <= yprev) || (yprev <= y && yle);
        const double m3 = dadd(arg, smin(axy, fabs(dsub(y, yprev))));
        const double c3 = dadd(left, b3 ? arg : m3);
        v = smin(smin(c1, c2), c3);
        if (EXACT && d == d0) v = dadd(pn, msm_c(xi, rc.xp, y, arg));  // column 0
    }
    if (EXACT && (d < dlo || d > dhi)) v = SENT;
    return v;
}

// One band row in place.  A: band row [d * 32], A[W2 * 32] is a permanent
// out-of-band cell; R: ring [slot * 32], RM = ring size - 1; s0: ring index
// of the candidate column read by cell d = 0 (the column itself for
// DTW/LCSS/MSM, column j-1 for ERP/EDR).  One loop of 2w+1 cells with a
// masked ring index: lanes sit at different rows, so a loop split where the
// ring wraps would differ between lanes and run both parts for all of them.
// Returns the row minimum (maximum for LCSS).  EXACT: clip cells outside
// [dlo, dhi] to the sentinel and use the reference's column-0 formula (cell
// d0 = w - i).
template <int METRIC, bool EXACT>
__device__ __forceinline__ double dp_row(double* __restrict__ A, const double* __restrict__ R, int RM, int W2,
                                         int s0, const RowCtx& rc, double arg, int dlo, int dhi, int d0) {
    constexpr double SENT = (METRIC == LCSS) ? 0.0 : kDpMax;
    double left = SENT, ext = SENT;
    double pd = A[0];
    double yprev = (METRIC == MSM) ? R[((s0 - 1) & RM) * 32] : 0.0;  // y_{j-1} for MSM
#pragma unroll 3
    for (int d = 0; d < W2; ++d) {
        const double pn = A[(d + 1) * 32];
        const double y = R[((s0 + d) & RM) * 32];
        const double v = dp_cell<METRIC, EXACT>(pn, pd, left, y, yprev, rc, arg, d, dlo, dhi, d0);
        A[d * 32] = v;
        left = v;
        pd = pn;
        yprev = y;
        ext = (METRIC == LCSS) ? smax(ext, v) : smin(ext, v);
    }
    return ext;
}

}  // namespace

template <int METRIC, bool GW>
__global__ void __launch_bounds__(kDpThreads) k_dp(Geom g, DpJob job) {
    extern __shared__ __align__(16) double dp_smem[];
    const QueryDev& q = job.q;
    const int m = q.m, w = q.w;
    const int W2 = 2 * w + 1;
    const int RING = dp_ring(w), RM = RING - 1;
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* __restrict__ X = q.qn;
    const size_t per_warp = dp_warp_doubles(w);
    // GW: band and ring in global scratch (too wide for shared memory); the
    // shared-memory form keeps the pointers provably shared, so every band and
    // ring access compiles to a shared-memory access
    double* wbase = GW ? job.gwork + ((size_t)blockIdx.x * warps + warp) * per_warp
                       : dp_smem + warp * per_warp;
    double* const A = wbase + lane;                            // band row, A[d * 32], d in [0, W2]
    double* const R = wbase + (size_t)(W2 + 1) * 32 + lane;    // ring, R[slot * 32]
    const unsigned long long n_all = job.list ? *job.n_list : (unsigned long long)job.n_windows;
    const unsigned long long n =
        (job.list && n_all > (unsigned long long)job.list_cap) ? job.list_cap : n_all;
    const double cut = job.cutoff_ptr ? *job.cutoff_ptr : job.cutoff;
    const double arg = q.arg;
    // abandon thresholds, once per kernel, each a little looser than the plain
    // test so that it can only abandon less: DTW/ERP sqrt(b) > s as b > s^2,
    // LCSS 1 - v/m > s as v < m(1 - s) (s = the slackened cutoff)
    const double cut_s = slack(cut);
    const bool neg_lim = cut_s < 0.0;
    const double cut_sq = dmul(dmul(cut_s, cut_s), 1.0 + 0x1p-50);
    const double lcss_lim = dmul(dmul((double)m, dsub(1.0, cut_s)), 1.0 - 0x1p-50);
    constexpr bool ONE_BASED = (METRIC == ERP || METRIC == EDR);  // rows 1..m, columns 0..m
    constexpr double SENT = (METRIC == LCSS) ? 0.0 : kDpMax;
    const int last = ONE_BASED ? m : m - 1;  // last row and last column

    // fast-mode limit on candidate points (see the header)
    double ylim;
    if (METRIC == EDR) {
        ylim = INFINITY;
    } else if (METRIC == LCSS) {
        ylim = (fabs(arg) < 1e299) ? INFINITY : -1.0;  // padding must never match
    } else {
        double xm = 0.0;
        for (int k = lane; k < m; k += 32) xm = fmax(xm, fabs(X[k]));
        for (int o = 16; o; o >>= 1) xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, o));
        ylim = sqrt(1e17 / (2.0 * m + 2.0)) - xm - fabs(arg) - 2.0;
    }
    const bool query_exact = job.force_exact || !(ylim > 0.0);

    // per-lane candidate state
    bool active = false;
    bool exact = query_exact;  // exact mode for the lane's candidate
    bool over = false;         // a candidate point exceeded ylim (fast mode)
    long long gi = 0;
    const double* tp = job.target;
    const double* lr = job.lraw;
    const double* ur = job.uraw;
    double mu = 0.0, sg = 1.0, inv = 1.0;
    bool rok = false;  // sg in the range of the reciprocal division (zdiv)
    int row = 0, ny = 0;
    double Ssum = 0.0, Pre = 0.0;  // GLB Q->T sum of the candidate, and its prefix over rows done
    bool has_s = false;
    // inputs of the lane's next row, loaded one row ahead so that their
    // latency overlaps the current row: query points, the next raw candidate
    // point (held for index nty) and the cascade term's forward-window reads
    double nx = 0.0, nxp = 0.0, nt = 0.0, na0 = 0.0, na1 = 0.0, nb0 = 0.0, nb1 = 0.0;
    int nty = -1;
    auto prefetch = [&](int r) {
        const int k = ONE_BASED ? r - 1 : r;
        nx = X[k];
        if (METRIC == MSM) nxp = (r > 0) ? X[r - 1] : -kPad;
        if (ny < m) { nt = tp[ny]; nty = ny; }
        if (has_s && (METRIC == LCSS || (k >= 1 && k <= m - 2))) {
            const int p0 = qt_p0(k, w), p1 = qt_p1(k, m, w);
            na0 = lr[p0]; na1 = lr[p1];
            nb0 = ur[p0]; nb1 = ur[p1];
        }
    };

    // candidate points ny..upto into the ring; columns past the window are padding
    auto fill_ring = [&](int upto) {
        for (; ny <= upto; ++ny) {
            double y = kPad;
            if (ny < m) {
                y = zdiv(dsub(ny == nty ? nt : tp[ny], mu), sg, inv, rok);
                over = over || !(fabs(y) <= ylim);
            }
            R[(ny & RM) * 32] = y;
        }
    };

    // band before the first general row (the reference's initialisation
    // loops), one lane alone: the restart of a candidate in the exact mode
    auto start = [&]() {
        ny = 0;
        over = false;
        Pre = 0.0;
        for (int d = 0; d <= W2; ++d) A[d * 32] = SENT;
        for (int c = -w - 1; c < 0; ++c) R[(c & RM) * 32] = -kPad;  // columns left of the matrix
        switch (METRIC) {
            case DTW:  // virtual (-1,-1) = 0 feeds cell (0,0)
            case LCSS:
                A[w * 32] = 0.0;
                row = 0;
                break;
            case ERP: {  // prev[0] = 0, prev[j] = prev[j-1] + dist(y[j-1], g), j <= min(m, w)
                A[w * 32] = 0.0;
                double acc = 0.0;
                for (int j = 1; j <= min(m, w); ++j) {
                    fill_ring(j - 1);
                    acc = dadd(acc, dsq(R[((j - 1) & RM) * 32], arg));
                    A[(j + w) * 32] = acc;
                }
                row = 1;
                break;
            }
            case EDR:  // prev[j] = j, j <= min(m, w)
                for (int j = 0; j <= min(m, w); ++j) A[(j + w) * 32] = (double)j;
                row = 1;
                break;
            default: {  // MSM row 0: cost[0] = |x0-y0|, cost[j] = cost[j-1] + C(y_j, x_0, y_{j-1})
                fill_ring(min(m - 1, w));
                double acc = fabs(dsub(X[0], R[0]));
                A[w * 32] = acc;
                for (int j = 1; j < m && j <= w; ++j) {
                    acc = dadd(acc, msm_c(R[(j & RM) * 32], X[0], R[((j - 1) & RM) * 32], arg));
                    A[(j + w) * 32] = acc;
                }
                row = 1;
                break;
            }
        }
    };

    unsigned long long valid_count = 0, cells = 0;
    bool drained = false;
    // Work reservoir: the warp claims 32 consecutive work items with one
    // atomic, lane j holds item rbase + j with its list entry, window
    // statistics and cascade sum already loaded, and idle lanes take items
    // rptr, rptr + 1, ... by shuffle.  The atomic's and the loads' latency is
    // paid once per 32 refills instead of once per refill (a candidate ends
    // every few rows under early abandon).  Every item is taken exactly once.
    int rptr = 32;  // next unused reservoir item (32: empty)
    long long r_gi = 0;
    double r_mu = 0.0, r_sg = 1.0, r_S = 0.0;
    int r_flags = 0;  // bit 0: a valid window, bit 1: its cascade sum is present
    for (;;) {
        // refill idle lanes from the reservoir (lanes that draw an invalid
        // window ask again)
        while (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (!need) break;
            if (rptr >= 32) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(job.next, 32ull);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= n) { drained = true; break; }
                rptr = 0;
                r_flags = 0;
                const unsigned long long c = base + (unsigned long long)lane;
                if (c < n) {
                    r_gi = job.list ? job.list[c] : (long long)c;
                    long long s;
                    int j;
                    g.locate(r_gi, &s, &j);
                    r_mu = job.MU[s * g.kml + j];
                    r_sg = job.SIG[s * g.kml + j];
                    if (!window_invalid(r_sg, g, r_gi)) {
                        r_flags = 1;
                        if (job.list_s && job.lraw) {
                            r_S = job.list_s[c];
                            if (r_S >= 0.0) r_flags |= 2;
                        }
                    }
                }
            }
            const int rank = __popc(need & ((1u << lane) - 1));
            const bool take = !active && rank < 32 - rptr;
            const int src = take ? rptr + rank : lane;
            const long long t_gi = __shfl_sync(0xffffffffu, r_gi, src);
            const double t_mu = __shfl_sync(0xffffffffu, r_mu, src);
            const double t_sg = __shfl_sync(0xffffffffu, r_sg, src);
            const double t_S = __shfl_sync(0xffffffffu, r_S, src);
            const int t_flags = __shfl_sync(0xffffffffu, r_flags, src);
            rptr = min(32, rptr + __popc(need));
            bool fresh = false;
            if (take && (t_flags & 1)) {
                gi = t_gi;
                mu = t_mu;
                sg = t_sg;
                tp = job.target + gi;
                inv = ddiv(1.0, sg);
                rok = rcp_div_in_range(sg);
                if (job.lraw) { lr = job.lraw + gi; ur = job.uraw + gi; }
                ++valid_count;
                has_s = (t_flags & 2) != 0;
                Ssum = has_s ? t_S : 0.0;
                exact = query_exact;
                fresh = true;
                active = true;
            }
            // The warp initialises each fresh lane's band, ring padding and
            // first w+1 candidate points together, one pass each, instead of
            // the fresh lane alone while the others wait.
            unsigned fm = __ballot_sync(0xffffffffu, fresh);
            while (fm) {
                const int L = __ffs(fm) - 1;
                fm &= fm - 1;
                const double* tpL = (const double*)__shfl_sync(0xffffffffu, (unsigned long long)tp, L);
                const double muL = __shfl_sync(0xffffffffu, mu, L);
                const double sgL = __shfl_sync(0xffffffffu, sg, L);
                const double invL = __shfl_sync(0xffffffffu, inv, L);
                const bool rokL = __shfl_sync(0xffffffffu, (int)rok, L) != 0;
                double* AL = wbase + L;
                double* RL = wbase + (size_t)(W2 + 1) * 32 + L;
                for (int d = lane; d <= W2; d += 32) {
                    double v = SENT;
                    if (METRIC == EDR) {  // prev[j] = j, j <= min(m, w)
                        if (d >= w && d - w <= min(m, w)) v = (double)(d - w);
                    } else if (d == w) {  // DTW/LCSS/MSM: virtual (-1,-1) = 0; ERP: prev[0] = 0
                        v = 0.0;
                    }
                    AL[d * 32] = v;
                }
                for (int c = lane; c <= w; c += 32) RL[((c - w - 1) & RM) * 32] = -kPad;  // left of the matrix
                bool bad = false;
                for (int c = lane; c <= w; c += 32) {
                    double y = kPad;
                    if (c < m) {
                        y = zdiv(dsub(tpL[c], muL), sgL, invL, rokL);
                        bad = bad || !(fabs(y) <= ylim);
                    }
                    RL[(c & RM) * 32] = y;
                }
                const bool anybad = __any_sync(0xffffffffu, bad);
                if (lane == L) over = anybad;
            }
            __syncwarp();
            if (fresh) {
                ny = w + 1;
                Pre = 0.0;
                row = ONE_BASED ? 1 : 0;
                if (METRIC == ERP) {  // prev[j] = prev[j-1] + dist(y[j-1], g), j <= min(m, w)
                    double acc = 0.0;
                    for (int j = 1; j <= min(m, w); ++j) {
                        acc = dadd(acc, dsq(R[((j - 1) & RM) * 32], arg));
                        A[(j + w) * 32] = acc;
                    }
                }
                if (METRIC == MSM && exact) {
                    // exact mode: the reference's row 0, cost[0] = |x0-y0|,
                    // cost[j] = cost[j-1] + C(y_j, x_0, y_{j-1}); the fast mode
                    // computes row 0 as a general row from the virtual cell
                    double acc = fabs(dsub(X[0], R[0]));
                    A[w * 32] = acc;
                    for (int j = 1; j < m && j <= w; ++j) {
                        acc = dadd(acc, msm_c(R[(j & RM) * 32], X[0], R[((j - 1) & RM) * 32], arg));
                        A[(j + w) * 32] = acc;
                    }
                    row = 1;
                }
                nty = -1;
                prefetch(row);
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            if (drained) break;
            continue;
        }
        if (!active) continue;

        const int i = row;
        const int s0 = ONE_BASED ? i - w - 1 : i - w;  // ring index read by cell d = 0
        fill_ring(s0 + 2 * w);                          // one new point per row in steady state
        if (over && !exact) {                           // out of the fast-mode range: restart exact
            exact = true;
            nty = -1;
            start();
            prefetch(row);
            continue;
        }
        const int k = ONE_BASED ? i - 1 : i;  // query index aligned by this row
        RowCtx rc;
        rc.xi = nx;
        rc.c0 = 0.0;
        rc.xp = rc.xi;
        rc.i = i;
        if (METRIC == ERP) rc.c0 = dsq(rc.xi, arg);
        if (METRIC == MSM) {
            // row 0 (fast mode): with x_{-1} = -1e300 a move from the row above
            // costs ~1e300 next to the left padding, so the virtual cell
            // (-1,-1) reaches cell (0,0) only, through the diagonal
            rc.xp = (i > 0) ? nxp : -kPad;
            rc.c0 = fabs(dsub(rc.xi, rc.xp));
        }
        rc.ge = rc.xp <= rc.xi;
        rc.le = rc.xi <= rc.xp;
        // cascading-bound term of this row's query point (inputs loaded a row ahead)
        const bool use_term = has_s && (METRIC == LCSS || (k >= 1 && k <= m - 2));
        const double ta = fmin(na0, na1), tb = fmax(nb0, nb1);
        if (i < last) prefetch(i + 1);  // next row's loads overlap this row's cells
        const double term = use_term ? qt_term_bound(METRIC, rc.xi, ta, tb, mu, inv, arg) : 0.0;
        double ext;
        if (!exact) {
            ext = dp_row<METRIC, false>(A, R, RM, W2, s0, rc, arg, 0, 0, -1);
        } else {
            const int dlo = max(0, w - i), dhi = min(2 * w, last - i + w);
            const int d0 = (METRIC == ERP || METRIC == EDR || METRIC == MSM) ? w - i : -1;
            ext = dp_row<METRIC, true>(A, R, RM, W2, s0, rc, arg, dlo, dhi, d0);
        }
        if (use_term) Pre = dadd(Pre, term);
        cells += (unsigned long long)W2;

        bool done = false, keep = false;
        double dist = 0.0;
        if (i == last) {
            const double fin = A[w * 32];
            if (METRIC == DTW || METRIC == ERP) dist = isfinite(fin) ? dsqrt(dmax0(fin)) : kDpMax;
            else if (METRIC == LCSS) dist = dsub(1.0, ddiv(fin, (double)m));
            else dist = fin;
            done = true;
            keep = dist <= cut && isfinite(dist);
        } else if (METRIC == LCSS) {
            // remaining rows can add at most one match each, and only where the
            // query point meets the candidate envelope
            double rest = (double)(m - 1 - i);
            if (has_s) rest = fmin(rest, fmax(0.0, dsub(Ssum, Pre)));
            if (dadd(ext, rest) < lcss_lim) done = true;
        } else {
            const double bnd = dadd(ext, fmax(0.0, dsub(Ssum, Pre)));
            if (METRIC == DTW || METRIC == ERP) {
                if (neg_lim || bnd > cut_sq) done = true;
            } else if (bnd > cut_s) {
                done = true;
            }
        }
        if (done) {
            active = false;
            if (keep) {
                const unsigned long long o = atomicAdd(job.n_out, 1ull);
                if (o < (unsigned long long)job.out_cap) {
                    job.out_idx[o] = gi;
                    job.out_dist[o] = dist;
                }
            }
        } else {
            ++row;
        }
    }
    if (job.n_valid) {
        for (int o = 16; o; o >>= 1) valid_count += __shfl_xor_sync(0xffffffffu, valid_count, o);
        if (lane == 0 && valid_count) atomicAdd(job.n_valid, valid_count);
    }
    if (job.n_cells) {
        for (int o = 16; o; o >>= 1) cells += __shfl_xor_sync(0xffffffffu, cells, o);
        if (lane == 0 && cells) atomicAdd(job.n_cells, cells);
    }
}

__host__ __device__ int dp_ring(int w) {
    int r = 1;
    while (r < 2 * w + 2) r <<= 1;
    return r;
}

__host__ __device__ size_t dp_warp_doubles(int w) { return (size_t)((2 * w + 2) + dp_ring(w)) * 32; }

#define FSM_DP_INST(M)                                   \
    template __global__ void k_dp<M, false>(Geom, DpJob); \
    template __global__ void k_dp<M, true>(Geom, DpJob);
FSM_DP_INST(DTW)
FSM_DP_INST(ERP)
FSM_DP_INST(EDR)
FSM_DP_INST(LCSS)
FSM_DP_INST(MSM)

const void* dp_kernel(int metric, bool gw) {
    switch (metric) {
        case DTW: return gw ? (const void*)k_dp<DTW, true> : (const void*)k_dp<DTW, false>;
        case ERP: return gw ? (const void*)k_dp<ERP, true> : (const void*)k_dp<ERP, false>;
        case EDR: return gw ? (const void*)k_dp<EDR, true> : (const void*)k_dp<EDR, false>;
        case LCSS: return gw ? (const void*)k_dp<LCSS, true> : (const void*)k_dp<LCSS, false>;
        default: return gw ? (const void*)k_dp<MSM, true> : (const void*)k_dp<MSM, false>;
    }
}

}  // namespace fsm
