// Exact banded elastic distances (src/ElasticMeasures.cpp:24-198, dispatch
// src/fsmeld.cpp:170-183) for candidate windows, one lane per candidate.
//
// Each lane keeps the previous and current band rows (offsets d = j - i + w,
// 2w+1 cells) and a ring of its z-normalised candidate points in shared
// memory laid out [slot][lane].  Every cell is computed from its three
// neighbours with the reference's formula and operand order; out-of-band
// neighbours read the reference's sentinels (1e18 for DTW/ERP/EDR/MSM, 0 for
// LCSS) and the row-0 / column-0 boundary cells follow the reference's
// initialisation loops.  A cell depends only on its neighbours, so the rows
// give the reference's bits.  Candidate points are normalised once each, as
// (t - mu) / sigma (src/fsmeld.cpp:823-826, 1202-1204).
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
// it has done.  A candidate whose bound already exceeds the cutoff (with a
// 1e-9 relative slack for round-off) cannot be kept and stops.  For LCSS the
// final match count is at most the row maximum plus the matches the
// remaining rows can still reach.  Results are unchanged: only candidates
// that would be discarded stop early.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

__device__ __forceinline__ double fmin3(double a, double b, double c) { return fmin(fmin(a, b), c); }

// src/ElasticMeasures.cpp:173-176
__device__ __forceinline__ double msm_c(double np, double x, double y, double c) {
    if ((x <= np && np <= y) || (y <= np && np <= x)) return c;
    const double a = fabs(dsub(np, x)), b = fabs(dsub(np, y));
    return dadd(c, (b < a) ? b : a);
}

// Cascading abandon margin: the bound and the DP carry independent round-off
// (relative ~1e-13); a 1e-9 relative slack keeps the test conservative.
__device__ __forceinline__ double slack(double cut) { return cut + 1e-9 * (1.0 + fabs(cut)); }

struct Lane {
    double* P;   // previous row [W2][32]
    double* Cu;  // current row  [W2][32]
    double* R;   // candidate ring [RING][32]
    int lane;
    __device__ double& p(int d) const { return P[d * 32 + lane]; }
    __device__ double& cu(int d) const { return Cu[d * 32 + lane]; }
    __device__ double& r(int s) const { return R[s * 32 + lane]; }
};

}  // namespace

template <int METRIC>
__global__ void __launch_bounds__(128) k_dp(Geom g, DpJob job) {
    extern __shared__ __align__(16) double dp_smem[];
    const QueryDev& q = job.q;
    const int m = q.m, w = q.w;
    const int W2 = 2 * w + 1, RING = 2 * w + 2;
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* X = dp_smem;
    for (int i = threadIdx.x; i < m; i += blockDim.x) X[i] = q.qn[i];
    const size_t per_warp = (size_t)(2 * W2 + RING) * 32;
    double* wbase = job.gwork ? job.gwork + ((size_t)blockIdx.x * warps + warp) * per_warp
                              : dp_smem + ((m + 1) & ~1) + warp * per_warp;
    __syncthreads();
    Lane B{wbase, wbase + (size_t)W2 * 32, wbase + (size_t)2 * W2 * 32, lane};
    const unsigned long long n_all = job.list ? *job.n_list : (unsigned long long)job.n_windows;
    const unsigned long long n =
        (job.list && n_all > (unsigned long long)job.list_cap) ? job.list_cap : n_all;
    const double cut = job.cutoff;
    const double arg = q.arg;

    // per-lane candidate state
    bool active = false;
    long long gi = 0;
    const double* tp = job.target;
    const double* lr = job.lraw;
    const double* ur = job.uraw;
    double mu = 0.0, sg = 1.0;
    int row = 0, ny = 0;
    double col = 0.0;  // ERP/EDR: previous row's column 0; MSM: running column 0
    double Ssum = 0.0, Pre = 0.0;  // GLB Q->T sum of the candidate, and its prefix over rows done
    bool has_s = false;            // the candidate came with a GLB Q->T sum

    auto y_at = [&](int j) { return ddiv(dsub(tp[j], mu), sg); };
    auto ring_slot = [&](int j) { int s = j % RING; return s < 0 ? s + RING : s; };
    auto fill_ring = [&](int upto) {  // candidate points 0..upto into the ring
        for (; ny <= upto; ++ny) B.r(ring_slot(ny)) = y_at(ny);
    };

    // row-0 set-up per metric (the reference's initialisation loops)
    auto start = [&]() {
        ny = 0;
        switch (METRIC) {
            case DTW:
                for (int d = 0; d < W2; ++d) B.p(d) = kDpMax;
                row = 0;
                break;
            case ERP: {  // prev[0] = 0, prev[j] = prev[j-1] + dist(y[j-1], g), j <= min(m, w)
                for (int d = 0; d < W2; ++d) B.p(d) = kDpMax;
                double acc = 0.0;
                for (int j = 1; j <= min(m, w); ++j) {
                    fill_ring(j - 1);
                    acc = dadd(acc, dsq(B.r(ring_slot(j - 1)), arg));
                    B.p(j + w) = acc;
                }
                col = 0.0;
                row = 1;
                break;
            }
            case EDR:
                for (int d = 0; d < W2; ++d) B.p(d) = kDpMax;
                for (int j = 1; j <= min(m, w); ++j) B.p(j + w) = (double)j;
                col = 0.0;
                row = 1;
                break;
            case LCSS:
                for (int d = 0; d < W2; ++d) B.p(d) = 0.0;
                row = 0;
                break;
            default: {  // MSM row 0: cost[0] = |x0-y0|, cost[j] = cost[j-1] + C(y_j, x_0, y_{j-1})
                for (int d = 0; d < W2; ++d) B.p(d) = kDpMax;
                fill_ring(min(m - 1, w));
                double acc = fabs(dsub(X[0], B.r(0)));
                col = acc;
                B.p(w) = acc;
                for (int j = 1; j < m && j <= w; ++j) {
                    acc = dadd(acc, msm_c(B.r(ring_slot(j)), X[0], B.r(ring_slot(j - 1)), arg));
                    B.p(j + w) = acc;
                }
                row = 1;
                break;
            }
        }
    };

    unsigned long long valid_count = 0;
    bool drained = false;
    for (;;) {
        // refill idle lanes from the work counter (lanes that draw an invalid
        // window ask again)
        while (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (!need) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(job.next, (unsigned long long)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= n) { drained = true; break; }
            if (!active) {
                const unsigned long long c = base + __popc(need & ((1u << lane) - 1));
                if (c < n) {
                    gi = job.list ? job.list[c] : (long long)c;
                    long long s;
                    int j;
                    g.locate(gi, &s, &j);
                    mu = job.MU[s * g.kml + j];
                    sg = job.SIG[s * g.kml + j];
                    if (!window_invalid(sg, g, gi)) {
                        tp = job.target + gi;
                        if (job.lraw) { lr = job.lraw + gi; ur = job.uraw + gi; }
                        ++valid_count;
                        has_s = job.list_s && job.lraw && job.list_s[c] >= 0.0;
                        Ssum = has_s ? job.list_s[c] : 0.0;
                        Pre = 0.0;
                        start();
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            if (drained) break;
            continue;
        }
        if (active) {
            bool done = false, keep = false;
            double dist = 0.0;
            const int i = row;
            switch (METRIC) {
                case DTW: {
                    fill_ring(min(m - 1, i + w));
                    const double xi = X[i];
                    double left = kDpMax, rmin = kDpMax;
                    int sl = ring_slot(i - w);
                    for (int d = 0; d < W2; ++d, sl = (sl + 1 == RING) ? 0 : sl + 1) {
                        const int j = i - w + d;
                        double v = kDpMax;
                        if (j >= 0 && j < m) {
                            const double yv0 = B.r(sl);
                            const double dd = dsq(xi, yv0);
                            if (i == 0 && j == 0) {
                                v = dd;
                            } else {
                                const double yv = (j == 0 || d == 0) ? kDpMax : left;
                                const double xv = (i == 0 || d + 1 > 2 * w) ? kDpMax : B.p(d + 1);
                                const double zv = (i == 0 || j == 0) ? kDpMax : B.p(d);
                                v = dadd(fmin3(xv, yv, zv), dd);
                            }
                            rmin = fmin(rmin, v);
                        }
                        B.cu(d) = v;
                        left = v;
                    }
                    if (has_s && i >= 1 && i <= m - 2) Pre = dadd(Pre, qt_term(DTW, xi, i, m, w, tp, lr, ur, mu, sg, arg));
                    if (i == m - 1) {
                        const double fin = B.cu(w);
                        dist = isfinite(fin) ? dsqrt(dmax0(fin)) : kDpMax;
                        done = true;
                        keep = dist <= cut;
                    } else if (dsqrt(dmax0(dadd(rmin, fmax(0.0, dsub(Ssum, Pre))))) > slack(cut)) {
                        done = true;
                    }
                    break;
                }
                case ERP:
                case EDR: {
                    fill_ring(min(m, i + w) - 1);
                    const double xi = X[i - 1];
                    const double dxg = (METRIC == ERP) ? dsq(xi, arg) : 1.0;
                    const double cur_col0 = (i <= w) ? ((METRIC == ERP) ? dadd(col, dxg) : (double)i) : kDpMax;
                    double rmin = cur_col0;
                    const int lo = max(1, i - w);
                    double left = kDpMax;
                    int sl = ring_slot(i - w - 1);
                    for (int d = 0; d < W2; ++d, sl = (sl + 1 == RING) ? 0 : sl + 1) {
                        const int j = i - w + d;
                        double v = kDpMax;
                        if (j >= lo && j <= m) {
                            if (j == lo) left = (j - 1 == 0) ? cur_col0 : kDpMax;
                            const double yj1 = B.r(sl);
                            const double up = (d + 1 <= 2 * w) ? B.p(d + 1) : kDpMax;
                            const double dg = (j - 1 == 0) ? col : B.p(d);
                            if (METRIC == ERP) {
                                const double match = dadd(dg, dsq(xi, yj1));
                                const double ins = dadd(left, dsq(yj1, arg));
                                const double del = dadd(up, dxg);
                                v = fmin3(match, ins, del);
                            } else {
                                const double sub = (fabs(dsub(xi, yj1)) <= arg) ? 0.0 : 1.0;
                                v = fmin3(dadd(up, 1.0), dadd(left, 1.0), dadd(dg, sub));
                            }
                            rmin = fmin(rmin, v);
                        }
                        B.cu(d) = v;
                        left = v;
                    }
                    col = cur_col0;
                    if (has_s && i - 1 >= 1 && i - 1 <= m - 2) Pre = dadd(Pre, qt_term(METRIC, xi, i - 1, m, w, tp, lr, ur, mu, sg, arg));
                    if (i == m) {
                        const double res = B.cu(w);
                        if (METRIC == ERP) dist = isfinite(res) ? dsqrt(dmax0(res)) : kDpMax;
                        else dist = res;
                        done = true;
                        keep = dist <= cut;
                    } else {
                        const double bnd = dadd(rmin, fmax(0.0, dsub(Ssum, Pre)));
                        if ((METRIC == ERP ? dsqrt(dmax0(bnd)) : bnd) > slack(cut)) done = true;
                    }
                    break;
                }
                case LCSS: {
                    fill_ring(min(m - 1, i + w));
                    const double xi = X[i];
                    const int wmin = max(0, i - w), wmax = min(m - 1, i + w);
                    double left = 0.0, rmax = 0.0;
                    int sl = ring_slot(i - w);
                    for (int d = 0; d < W2; ++d, sl = (sl + 1 == RING) ? 0 : sl + 1) {
                        const int j = i - w + d;
                        double v = 0.0;
                        if (j >= wmin && j <= wmax) {
                            const double yv0 = B.r(sl);
                            const bool hit = fabs(dsub(xi, yv0)) <= arg;
                            if (i + j == 0) {
                                v = hit ? 1.0 : 0.0;
                            } else if (i == 0) {
                                v = hit ? 1.0 : ((j > wmin) ? left : 0.0);
                            } else if (j == 0) {
                                v = hit ? 1.0 : B.p(d + 1);
                            } else {
                                const double v1 = B.p(d);
                                const double v2 = (d + 1 <= 2 * w) ? B.p(d + 1) : 0.0;
                                const double v3 = (j > wmin) ? left : 0.0;
                                double best = hit ? dadd(v1, 1.0) : v1;
                                if (best < v2) best = v2;
                                if (best < v3) best = v3;
                                v = best;
                            }
                            rmax = fmax(rmax, v);
                        }
                        B.cu(d) = v;
                        left = v;
                    }
                    if (has_s) Pre = dadd(Pre, qt_term(LCSS, xi, i, m, w, tp, lr, ur, mu, sg, arg));
                    if (i == m - 1) {
                        dist = dsub(1.0, ddiv(B.cu(w), (double)m));
                        done = true;
                        keep = dist <= cut;
                    } else {
                        // remaining rows can add at most one match each, and only where the
                        // query point meets the candidate envelope
                        double rest = (double)(m - 1 - i);
                        if (has_s) rest = fmin(rest, fmax(0.0, dsub(Ssum, Pre)));
                        if (dsub(1.0, ddiv(dadd(rmax, rest), (double)m)) > slack(cut)) done = true;
                    }
                    break;
                }
                default: {  // MSM
                    fill_ring(min(m - 1, i + w));
                    const double xi = X[i], xi1 = X[i - 1];
                    double colv = kDpMax;
                    if (i <= w) {
                        col = dadd(col, msm_c(xi, xi1, B.r(0), arg));
                        colv = col;
                    }
                    const int js = max(1, i - w), je = min(m - 1, i + w);
                    double left = kDpMax, rmin = colv;
                    int sl = ring_slot(i - w);
                    for (int d = 0; d < W2; ++d, sl = (sl + 1 == RING) ? 0 : sl + 1) {
                        const int j = i - w + d;
                        double v = kDpMax;
                        if (j == 0) {
                            v = colv;  // column 0 (in band only while i <= w)
                        } else if (j >= js && j <= je) {
                            if (j == js) left = (j - 1 == 0) ? colv : kDpMax;
                            const double yj = B.r(sl);
                            const double yj1 = B.r(sl == 0 ? RING - 1 : sl - 1);
                            const double c1 = dadd(B.p(d), fabs(dsub(xi, yj)));
                            const double c2 = dadd((d + 1 <= 2 * w) ? B.p(d + 1) : kDpMax, msm_c(xi, xi1, yj, arg));
                            const double c3 = dadd(left, msm_c(yj, xi, yj1, arg));
                            v = fmin3(c1, c2, c3);
                            rmin = fmin(rmin, v);
                        }
                        B.cu(d) = v;
                        left = v;
                    }
                    if (has_s && i >= 1 && i <= m - 2) Pre = dadd(Pre, qt_term(MSM, xi, i, m, w, tp, lr, ur, mu, sg, arg));
                    if (i == m - 1) {
                        dist = B.cu(w);
                        done = true;
                        keep = dist <= cut;
                    } else if (dadd(rmin, fmax(0.0, dsub(Ssum, Pre))) > slack(cut)) {
                        done = true;
                    }
                    break;
                }
            }
            if (done) {
                active = false;
                keep = keep && isfinite(dist);
                if (keep) {
                    const unsigned long long o = atomicAdd(job.n_out, 1ull);
                    if (o < (unsigned long long)job.out_cap) {
                        job.out_idx[o] = gi;
                        job.out_dist[o] = dist;
                    }
                }
            } else {
                double* t = B.P; B.P = B.Cu; B.Cu = t;
                ++row;
            }
        }
    }
    if (job.n_valid) {
        for (int o = 16; o; o >>= 1) valid_count += __shfl_xor_sync(0xffffffffu, valid_count, o);
        if (lane == 0 && valid_count) atomicAdd(job.n_valid, valid_count);
    }
}

size_t dp_warp_doubles(int w) { return (size_t)(2 * (2 * w + 1) + (2 * w + 2)) * 32; }

template __global__ void k_dp<DTW>(Geom, DpJob);
template __global__ void k_dp<ERP>(Geom, DpJob);
template __global__ void k_dp<EDR>(Geom, DpJob);
template __global__ void k_dp<LCSS>(Geom, DpJob);
template __global__ void k_dp<MSM>(Geom, DpJob);

}  // namespace fsm
