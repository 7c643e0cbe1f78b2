// Exact banded elastic distances (src/ElasticMeasures.cpp:24-198, dispatch
// src/fsmeld.cpp:170-183) for candidate windows, one lane per candidate.
//
// Each lane keeps the previous and current band rows (offsets d = j - i + w,
// 2w+1 cells) and a ring of its z-normalised candidate points in shared
// memory laid out [slot][lane], so lanes never share a bank word.  Every
// cell is computed from its three neighbours with the reference's formula
// and operand order; out-of-band neighbours read the reference's sentinels
// (1e18 for DTW/ERP/EDR/MSM, 0 for LCSS), and the row-0 / column-0 boundary
// cells follow the reference's initialisation loops.  The value of a cell
// depends only on its neighbours, so evaluating rows band by band gives the
// reference's bits.  Candidate points are normalised once each, as
// (t - mu) / sigma (src/fsmeld.cpp:823-826, 1202-1204).
//
// When 3 band-width arrays per lane do not fit in shared memory (very wide
// bands), the same code runs on a global-memory scratch with the same
// lane-interleaved layout.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

struct LaneBand {
    double* prev;  // [W2][32]
    double* cur;   // [W2][32]
    double* ring;  // [RING][32]
    int lane, RING;
    __device__ double& P(int d) const { return prev[d * 32 + lane]; }
    __device__ double& Cc(int d) const { return cur[d * 32 + lane]; }
    __device__ double& Y(int j) const { return ring[(j % RING) * 32 + lane]; }
    __device__ void swap() { double* t = prev; prev = cur; cur = t; }
};

struct Cand {
    const double* tp;
    double mu, sg;
    __device__ double y(int j) const { return ddiv(dsub(tp[j], mu), sg); }
};

__device__ __forceinline__ double fmin3(double a, double b, double c) { return fmin(fmin(a, b), c); }

// src/ElasticMeasures.cpp:24-61
__device__ double dp_dtw(const double* X, int m, int r, const Cand& cd, LaneBand& B) {
    const int W2 = 2 * r + 1;
    for (int k = 0; k < W2; ++k) { B.P(k) = kDpMax; B.Cc(k) = kDpMax; }
    int ny = 0;
    for (int i = 0; i < m; ++i) {
        const int need = min(m - 1, i + r);
        for (; ny <= need; ++ny) B.Y(ny) = cd.y(ny);
        const int jlo = max(0, i - r), jhi = min(m - 1, i + r);
        const double xi = X[i];
        double left = kDpMax;
        int k = jlo - i + r;
        for (int j = jlo; j <= jhi; ++j, ++k) {
            const double d = dsq(xi, B.Y(j));
            double v;
            if (i == 0 && j == 0) {
                v = d;
            } else {
                const double yv = (j == jlo) ? kDpMax : left;
                const double xv = (i == 0 || k + 1 > 2 * r) ? kDpMax : B.P(k + 1);
                const double zv = (i == 0 || j == 0) ? kDpMax : B.P(k);
                v = dadd(fmin3(xv, yv, zv), d);
            }
            B.Cc(k) = v;
            left = v;
        }
        B.swap();
    }
    const double fin = B.P(r);
    if (!isfinite(fin)) return kDpMax;
    return dsqrt(dmax0(fin));
}

// src/ElasticMeasures.cpp:95-130 (rows i = 1..m, band j in [max(1,i-w), min(m,i+w)])
__device__ double dp_erp(const double* X, int m, int w, double gv, const Cand& cd, LaneBand& B) {
    const int W2 = 2 * w + 1;
    for (int d = 0; d < W2; ++d) B.P(d) = kDpMax;
    int ny = 0;
    // row 0: prev[0] = 0, prev[j] = prev[j-1] + dist(y[j-1], g) for j <= min(m, w)
    double acc = 0.0;
    for (int j = 1; j <= min(m, w); ++j) {
        for (; ny <= j - 1; ++ny) B.Y(ny) = cd.y(ny);
        acc = dadd(acc, dsq(B.Y(j - 1), gv));
        B.P(j + w) = acc;
    }
    double prev_col0 = 0.0;
    for (int i = 1; i <= m; ++i) {
        const int need = min(m, i + w) - 1;
        for (; ny <= need; ++ny) B.Y(ny) = cd.y(ny);
        const double xi = X[i - 1];
        const double dxg = dsq(xi, gv);
        const double cur_col0 = (i <= w) ? dadd(prev_col0, dxg) : kDpMax;
        const int lo = max(1, i - w), hi = min(m, i + w);
        double left = (lo - 1 == 0) ? cur_col0 : kDpMax;
        for (int j = lo; j <= hi; ++j) {
            const int d = j - i + w;
            const double yj1 = B.Y(j - 1);
            const double mb = (j - 1 == 0) ? prev_col0 : B.P(d);
            const double match = dadd(mb, dsq(xi, yj1));
            const double ins = dadd(left, dsq(yj1, gv));
            const double del = dadd((d + 1 <= 2 * w) ? B.P(d + 1) : kDpMax, dxg);
            const double v = fmin3(match, ins, del);
            B.Cc(d) = v;
            left = v;
        }
        B.swap();
        prev_col0 = cur_col0;
    }
    const double res = B.P(w);
    if (!isfinite(res)) return kDpMax;
    return dsqrt(dmax0(res));
}

// src/ElasticMeasures.cpp:132-165
__device__ double dp_edr(const double* X, int m, int w, double eps, const Cand& cd, LaneBand& B) {
    const int W2 = 2 * w + 1;
    for (int d = 0; d < W2; ++d) B.P(d) = kDpMax;
    for (int j = 1; j <= min(m, w); ++j) B.P(j + w) = (double)j;
    int ny = 0;
    double prev_col0 = 0.0;
    for (int i = 1; i <= m; ++i) {
        const int need = min(m, i + w) - 1;
        for (; ny <= need; ++ny) B.Y(ny) = cd.y(ny);
        const double xi = X[i - 1];
        const double cur_col0 = (i <= w) ? (double)i : kDpMax;
        const int lo = max(1, i - w), hi = min(m, i + w);
        double left = (lo - 1 == 0) ? cur_col0 : kDpMax;
        for (int j = lo; j <= hi; ++j) {
            const int d = j - i + w;
            const double yj1 = B.Y(j - 1);
            const double sub = (fabs(dsub(xi, yj1)) <= eps) ? 0.0 : 1.0;
            const double up = dadd((d + 1 <= 2 * w) ? B.P(d + 1) : kDpMax, 1.0);
            const double lf = dadd(left, 1.0);
            const double dg = dadd((j - 1 == 0) ? prev_col0 : B.P(d), sub);
            const double v = fmin3(up, lf, dg);
            B.Cc(d) = v;
            left = v;
        }
        B.swap();
        prev_col0 = cur_col0;
    }
    return B.P(w);
}

// src/ElasticMeasures.cpp:63-93 (0-based rows; out-of-band cells read 0)
__device__ double dp_lcss(const double* X, int m, int w, double eps, const Cand& cd, LaneBand& B) {
    const int W2 = 2 * w + 1;
    for (int d = 0; d < W2; ++d) { B.P(d) = 0.0; B.Cc(d) = 0.0; }
    int ny = 0;
    for (int i = 0; i < m; ++i) {
        const int need = min(m - 1, i + w);
        for (; ny <= need; ++ny) B.Y(ny) = cd.y(ny);
        const int wmin = max(0, i - w), wmax = min(m, i + w + 1);
        const double xi = X[i];
        double left = 0.0;
        for (int j = wmin; j < wmax; ++j) {
            const int d = j - i + w;
            const bool hit = fabs(dsub(xi, B.Y(j))) <= eps;
            double v;
            if (i + j == 0) {
                v = hit ? 1.0 : 0.0;
            } else if (i == 0) {
                v = hit ? 1.0 : ((j > wmin) ? left : 0.0);
            } else if (j == 0) {
                v = hit ? 1.0 : B.P(d + 1);
            } else {
                const double v1 = B.P(d);
                const double v2 = (d + 1 <= 2 * w) ? B.P(d + 1) : 0.0;
                const double v3 = (j > wmin) ? left : 0.0;
                double best = hit ? dadd(v1, 1.0) : v1;
                if (best < v2) best = v2;
                if (best < v3) best = v3;
                v = best;
            }
            B.Cc(d) = v;
            left = v;
        }
        // cells of this row outside its band stay 0 for the next row's reads
        for (int d = 0; d < W2; ++d) {
            const int j = d + i - w;
            if (j < wmin || j >= wmax) B.Cc(d) = 0.0;
        }
        B.swap();
    }
    const double res = B.P(w);
    return dsub(1.0, ddiv(res, (double)m));
}

// src/ElasticMeasures.cpp:173-176
__device__ __forceinline__ double msm_c(double np, double x, double y, double c) {
    if ((x <= np && np <= y) || (y <= np && np <= x)) return c;
    const double a = fabs(dsub(np, x)), b = fabs(dsub(np, y));
    return dadd(c, (b < a) ? b : a);
}

// src/ElasticMeasures.cpp:167-198
__device__ double dp_msm(const double* X, int m, int w, double c, const Cand& cd, LaneBand& B) {
    const int W2 = 2 * w + 1;
    for (int d = 0; d < W2; ++d) { B.P(d) = kDpMax; B.Cc(d) = kDpMax; }
    int ny = 0;
    for (; ny <= min(m - 1, w); ++ny) B.Y(ny) = cd.y(ny);
    // row 0: cost[0] = |x0 - y0|, cost[j] = cost[j-1] + C(y_j, x_0, y_{j-1}) for j <= w
    double acc = fabs(dsub(X[0], B.Y(0)));
    B.P(w) = acc;
    for (int j = 1; j < m && j <= w; ++j) {
        acc = dadd(acc, msm_c(B.Y(j), X[0], B.Y(j - 1), c));
        B.P(j + w) = acc;
    }
    double col = fabs(dsub(X[0], B.Y(0)));  // column 0 running value
    const double y0 = B.Y(0);
    for (int i = 1; i < m; ++i) {
        const int need = min(m - 1, i + w);
        for (; ny <= need; ++ny) B.Y(ny) = cd.y(ny);
        const double xi = X[i], xi1 = X[i - 1];
        for (int d = 0; d < W2; ++d) B.Cc(d) = kDpMax;
        double colv = kDpMax;
        if (i <= w) {
            col = dadd(col, msm_c(xi, xi1, y0, c));
            colv = col;
            B.Cc(w - i) = colv;
        }
        const int js = max(1, i - w), je = min(m - 1, i + w);
        double left = (js - 1 == 0) ? colv : kDpMax;
        for (int j = js; j <= je; ++j) {
            const int d = j - i + w;
            const double yj = B.Y(j), yj1 = B.Y(j - 1);
            const double c1 = dadd(B.P(d), fabs(dsub(xi, yj)));
            const double c2 = dadd((d + 1 <= 2 * w) ? B.P(d + 1) : kDpMax, msm_c(xi, xi1, yj, c));
            const double c3 = dadd(left, msm_c(yj, xi, yj1, c));
            const double v = fmin3(c1, c2, c3);
            B.Cc(d) = v;
            left = v;
        }
        B.swap();
    }
    return B.P(w);
}

}  // namespace

// mode 0: keep finite distances <= cutoff (search / exact); mode 1: keep all
// finite distances (cutoff command).  Candidates come from `list` or, when
// list is null, are the windows [0, n).
template <int METRIC>
__global__ void __launch_bounds__(128) k_dp(Geom g, DpJob job) {
    extern __shared__ __align__(16) double dp_smem[];
    const QueryDev& q = job.q;
    const int m = q.m, w = q.w;
    const int W2 = 2 * w + 1, RING = 2 * w + 3;
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* X = dp_smem;
    for (int i = threadIdx.x; i < m; i += blockDim.x) X[i] = q.qn[i];
    const size_t per_warp = (size_t)(2 * W2 + RING) * 32;
    double* wbase = job.gwork ? job.gwork + ((size_t)blockIdx.x * warps + warp) * per_warp
                              : dp_smem + ((m + 1) & ~1) + warp * per_warp;
    __syncthreads();
    LaneBand B{wbase, wbase + (size_t)W2 * 32, wbase + (size_t)2 * W2 * 32, lane, RING};
    const unsigned long long n_all = job.list ? *job.n_list : (unsigned long long)job.n_windows;
    const unsigned long long n = (job.list && n_all > (unsigned long long)job.list_cap) ? job.list_cap : n_all;
    for (unsigned long long base = ((unsigned long long)blockIdx.x * warps + warp) * 32; base < n;
         base += (unsigned long long)gridDim.x * warps * 32) {
        const unsigned long long c = base + lane;
        const bool active = c < n;
        long long gi = 0;
        bool valid = false;
        Cand cd{job.target, 0.0, 1.0};
        if (active) {
            gi = job.list ? job.list[c] : (long long)c;
            long long s;
            int j;
            g.locate(gi, &s, &j);
            cd.mu = job.MU[s * g.kml + j];
            cd.sg = job.SIG[s * g.kml + j];
            valid = !window_invalid(cd.sg, g, gi);
            cd.tp = job.target + gi;
        }
        if (!valid) { cd.tp = job.target; cd.mu = 0.0; cd.sg = 1.0; }  // harmless work for idle lanes
        double dist;
        switch (METRIC) {
            case DTW: dist = dp_dtw(X, m, w, cd, B); break;
            case ERP: dist = dp_erp(X, m, w, q.arg, cd, B); break;
            case EDR: dist = dp_edr(X, m, w, q.arg, cd, B); break;
            case LCSS: dist = dp_lcss(X, m, w, q.arg, cd, B); break;
            default: dist = dp_msm(X, m, w, q.arg, cd, B); break;
        }
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        if (lane == 0 && job.n_valid && vmask) atomicAdd(job.n_valid, (unsigned long long)__popc(vmask));
        const bool keep = valid && isfinite(dist) && (job.mode == 1 || dist <= job.cutoff);
        const unsigned kmask = __ballot_sync(0xffffffffu, keep);
        if (kmask) {
            unsigned long long o = 0;
            if (lane == 0) o = atomicAdd(job.n_out, (unsigned long long)__popc(kmask));
            o = __shfl_sync(0xffffffffu, o, 0) + __popc(kmask & ((1u << lane) - 1));
            if (keep && o < (unsigned long long)job.out_cap) {
                job.out_idx[o] = gi;
                job.out_dist[o] = dist;
            }
        }
    }
}

size_t dp_warp_doubles(int w) { return (size_t)(2 * (2 * w + 1) + (2 * w + 3)) * 32; }

template __global__ void k_dp<DTW>(Geom, DpJob);
template __global__ void k_dp<ERP>(Geom, DpJob);
template __global__ void k_dp<EDR>(Geom, DpJob);
template __global__ void k_dp<LCSS>(Geom, DpJob);
template __global__ void k_dp<MSM>(Geom, DpJob);

}  // namespace fsm
