// Exact banded elastic distances (src/ElasticMeasures.cpp:24-198, dispatch
// src/fsmeld.cpp:170-183) for wide bands: one warp per candidate, one
// anti-diagonal of the band per step.
//
// The lane-per-candidate DP (k_dp.cu) keeps a band row and a candidate ring
// per lane in shared memory, (2w+2 + ring) x 32 doubles per warp, which no
// longer fits once w reaches about a hundred.  Here the band lives in the
// warp's registers: band offset d = j - i + w (0 <= d <= 2w) belongs to lane
// (d mod 64) / 2 of chunk d / 64, in register E[chunk] when d is even and
// O[chunk] when d is odd.  Cell (i, j) lies on anti-diagonal a = i + j, and
// the cells of one anti-diagonal all have the parity of a + w, so a step
// updates either every E or every O register:
//
//   even d:  up (i-1, j)   = band d+1, anti-diagonal a-1 = own O
//            left (i, j-1) = band d-1, anti-diagonal a-1 = O of lane l-1
//                            (lane 0: O of lane 31, previous chunk)
//            diag (i-1,j-1)= band d,   anti-diagonal a-2 = own E (old value)
//   odd d:   left          = own E;  up = E of lane l+1 (lane 31: lane 0 of
//            the next chunk);  diag = own O (old value)
//
// so one shuffle per chunk and step carries the only cross-lane operand.
// Cells outside the band or outside the matrix hold the reference's
// out-of-band value (MAX_VAL = 1e18, 0 for LCSS), which is exactly what the
// reference reads for such neighbours; row 0 and column 0 of ERP, EDR and
// MSM take the reference's own initialisation formulas.  Every in-band cell
// is computed with the reference's formula in its operation order (explicit
// round-to-nearest intrinsics), so distances are bit-identical whatever the
// magnitudes (no fast mode is needed here).
//
// Grids: DTW, LCSS, MSM use rows/columns 0..m-1 over (query, candidate);
// ERP and EDR use 0..m with row/column 0 the empty prefix (x[i-1], y[j-1]).
//
// Early abandon: every monotone path from (0,0) to (R,R) visits anti-diagonal
// a-1 or a, and costs only grow along a path, so the final cost is at least
// the minimum over those two anti-diagonals (the warp minimum of all band
// registers after step a) plus a lower bound for the rows the path still has
// to enter: rows after the largest row of the pair.  Each such row costs at
// least its GLB Q->T term (the query point against the candidate's window
// envelope), computed here on an envelope widened by a relative 2^-49, which
// contains the exact envelope, so each term is at most the exact one (LCSS:
// the match indicator at least the exact one).  Suffix sums of those terms
// are kept per block of four rows and read at the next block boundary, which
// drops a few rows and only loosens the bound.  For LCSS the final match
// count is at most the maximum over the pair plus one possible match per
// remaining row after the pair's smallest row.  A candidate whose bound
// exceeds the cutoff (1e-9 relative slack) cannot be a match and stops.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

__device__ __forceinline__ double wslack(double cut) { return cut + 1e-9 * (1.0 + fabs(cut)); }
__device__ __forceinline__ double wmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double wmax(double a, double b) { return (a < b) ? b : a; }

// src/ElasticMeasures.cpp:173-176
__device__ __forceinline__ double wmsm_c(double np, double x, double y, double c) {
    if ((x <= np && np <= y) || (y <= np && np <= x)) return c;
    const double a = fabs(dsub(np, x)), b = fabs(dsub(np, y));
    return dadd(c, (b < a) ? b : a);
}

// Q->T term of query point x against the candidate envelope, on the raw
// window extremes [a, b] normalised with inv = fl(1/sigma) and widened by a
// relative 2^-49, so the envelope contains the exact normalised envelope:
// distance terms are at most the exact ones, the LCSS match indicator at
// least the exact one.
__device__ __forceinline__ double qt_term_wide(int metric, double x, double a, double b, double mu, double inv,
                                               double arg) {
    double lo = dmul(dsub(a, mu), inv);
    double up = dmul(dsub(b, mu), inv);
    lo = dsub(lo, dadd(dmul(fabs(lo), 0x1p-49), 0x1p-1000));
    up = dadd(up, dadd(dmul(fabs(up), 0x1p-49), 0x1p-1000));
    return qt_term_norm(metric, x, lo, up, arg);
}

// One cell at grid position (i, j) from its three neighbours.  X: query,
// Y: z-normalised candidate (both in shared memory); R: last grid index.
template <int METRIC>
__device__ __forceinline__ double wave_cell(int i, int j, double up, double left, double diag,
                                            const double* __restrict__ X, const double* __restrict__ Y,
                                            double arg) {
    if (METRIC == DTW) {
        // cost[k] = min({x, y, z}) + dist(A[i], B[j]); (0,0) reads diag = 0
        return dadd(wmin(wmin(up, diag), left), dsq(X[i], Y[j]));
    } else if (METRIC == LCSS) {
        const double hit = (fabs(dsub(X[i], Y[j])) <= arg) ? 1.0 : 0.0;
        double best = (hit != 0.0) ? dadd(diag, 1.0) : diag;
        best = wmax(best, up);
        return wmax(best, left);
    } else if (METRIC == ERP) {
        if (i == 0) return (j == 0) ? 0.0 : dadd(left, dsq(Y[j - 1], arg));   // prev[j] = prev[j-1] + dist(y, g)
        const double xd = dsq(X[i - 1], arg);
        if (j == 0) return dadd(up, xd);                                        // cur[0] = prev[0] + dist(x, g)
        const double match = dadd(diag, dsq(X[i - 1], Y[j - 1]));
        const double ins = dadd(left, dsq(Y[j - 1], arg));
        const double del = dadd(up, xd);
        return wmin(wmin(match, ins), del);
    } else if (METRIC == EDR) {
        if (i == 0) return (double)j;
        if (j == 0) return (double)i;
        const double sub = (fabs(dsub(X[i - 1], Y[j - 1])) <= arg) ? 0.0 : 1.0;
        return wmin(wmin(dadd(up, 1.0), dadd(left, 1.0)), dadd(diag, sub));
    } else {  // MSM
        if (i == 0 && j == 0) return fabs(dsub(X[0], Y[0]));
        if (j == 0) return dadd(up, wmsm_c(X[i], X[i - 1], Y[0], arg));
        if (i == 0) return dadd(left, wmsm_c(Y[j], X[0], Y[j - 1], arg));
        const double c1 = dadd(diag, fabs(dsub(X[i], Y[j])));
        const double c2 = dadd(up, wmsm_c(X[i], X[i - 1], Y[j], arg));
        const double c3 = dadd(left, wmsm_c(Y[j], X[i], Y[j - 1], arg));
        return wmin(wmin(c1, c2), c3);
    }
}

}  // namespace

size_t dpw_smem_bytes(int m, int warps) {
    const size_t xq = ((size_t)m + 1) & ~(size_t)1;
    return sizeof(double) * (xq + (size_t)warps * dpw_warp_doubles(m));
}

template <int METRIC, int K>
__global__ void __launch_bounds__(kDpwThreads) k_dpw(Geom g, DpJob job) {
    extern __shared__ __align__(16) double dpw_smem[];
    const QueryDev& q = job.q;
    const int m = q.m, w = q.w;
    constexpr bool ONE_BASED = (METRIC == ERP || METRIC == EDR);
    constexpr double SENT = (METRIC == LCSS) ? 0.0 : kDpMax;
    const int R = ONE_BASED ? m : m - 1;  // last grid row and column
    const int W2 = 2 * w + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* X = dpw_smem;
    double* Y = dpw_smem + ((m + 1) & ~1) + (size_t)warp * dpw_warp_doubles(m);
    double* S4 = Y + (((m + 1) & ~1));  // suffix sums of the row terms, per block of 4 rows
    const int nblk = (R + 4) >> 2;      // row blocks covering rows 0..R
    for (int k = threadIdx.x; k < m; k += blockDim.x) X[k] = q.qn[k];
    __syncthreads();

    const unsigned long long n_all = job.list ? *job.n_list : (unsigned long long)job.n_windows;
    const unsigned long long n =
        (job.list && n_all > (unsigned long long)job.list_cap) ? job.list_cap : n_all;
    const double cut = job.cutoff_ptr ? *job.cutoff_ptr : job.cutoff;
    const double arg = q.arg;
    const double cut_s = wslack(cut);
    const bool neg_lim = cut_s < 0.0;
    const double cut_sq = dmul(dmul(cut_s, cut_s), 1.0 + 0x1p-50);
    const double lcss_lim = dmul(dmul((double)m, dsub(1.0, cut_s)), 1.0 - 0x1p-50);
    const bool cascade = job.lraw != nullptr;
    // owner of the final cell (R, R): band offset w
    const int fin_lane = (w & 63) >> 1, fin_chunk = w >> 6;
    const bool fin_odd = (w & 1) != 0;

    unsigned long long valid_count = 0, cells = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(job.next, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n) break;
        const long long gi = job.list ? job.list[item] : (long long)item;
        long long s;
        int jj;
        g.locate(gi, &s, &jj);
        const double mu = job.MU[s * g.kml + jj];
        const double sg = job.SIG[s * g.kml + jj];
        if (window_invalid(sg, g, gi)) continue;
        ++valid_count;
        const double inv = ddiv(1.0, sg);
        const bool rok = rcp_div_in_range(sg) != 0;
        const double* tp = job.target + gi;
        for (int k = lane; k < m; k += 32) Y[k] = zdiv(dsub(tp[k], mu), sg, inv, rok);
        if (cascade) {
            // per-row terms, summed per block of 4 grid rows, then suffix sums
            const double* lr = job.lraw + gi;
            const double* ur = job.uraw + gi;
            const int per = (nblk + 31) >> 5;
            const int b0 = lane * per, b1 = min(nblk, b0 + per);
            double part = 0.0;
            for (int b = b1 - 1; b >= b0; --b) {
                double blk = 0.0;
                for (int r = 4 * b; r < 4 * b + 4 && r <= R; ++r) {
                    const int k = ONE_BASED ? r - 1 : r;
                    if (k < 0 || !(METRIC == LCSS || (k >= 1 && k <= m - 2))) continue;
                    const int p0 = qt_p0(k, w), p1 = qt_p1(k, m, w);
                    const double a0 = lr[p0], a1 = lr[p1], c0 = ur[p0], c1 = ur[p1];
                    blk = dadd(blk, qt_term_wide(METRIC, X[k], (a1 < a0) ? a1 : a0, (c0 < c1) ? c1 : c0, mu, inv,
                                                 arg));
                }
                part = dadd(part, blk);
                S4[b] = part;  // suffix within this lane's range, completed below
            }
            // add the suffix of the lanes to the right
            double after = 0.0, tot = part;
            for (int o = 1; o < 32; o <<= 1) {
                const double v = __shfl_down_sync(0xffffffffu, tot, o);
                if (lane + o < 32) tot = dadd(tot, v);
            }
            after = __shfl_down_sync(0xffffffffu, tot, 1);
            if (lane == 31) after = 0.0;
            for (int b = b0; b < b1; ++b) S4[b] = dadd(S4[b], after);
            if (lane == 0) S4[nblk] = 0.0;
        }
        __syncwarp();

        double E[K], O[K];
#pragma unroll
        for (int c = 0; c < K; ++c) { E[c] = SENT; O[c] = SENT; }
        if (METRIC == DTW) {  // virtual cell (-1,-1) = 0: the diagonal of (0,0)
#pragma unroll
            for (int c = 0; c < K; ++c)
                if (c == fin_chunk && lane == fin_lane) {
                    if (fin_odd) O[c] = 0.0;
                    else E[c] = 0.0;
                }
        }
        bool stop = false;
        int a = 0;
        for (; a <= 2 * R; ++a) {
            if (((a + w) & 1) == 0) {
                double rot[K];
#pragma unroll
                for (int c = 0; c < K; ++c) rot[c] = __shfl_sync(0xffffffffu, O[c], (lane + 31) & 31);
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    const int d = 64 * c + 2 * lane;
                    const double left = (lane == 0) ? (c == 0 ? SENT : rot[c > 0 ? c - 1 : 0]) : rot[c];
                    const int i = (a - d + w) >> 1, j = i + d - w;
                    const bool ok = d < W2 && i >= 0 && j >= 0 && i <= R && j <= R;
                    const int ic = ok ? i : 0, jc = ok ? j : 0;
                    const double v = wave_cell<METRIC>(ic, jc, O[c], left, E[c], X, Y, arg);
                    E[c] = ok ? v : SENT;
                }
            } else {
                double rot[K];
#pragma unroll
                for (int c = 0; c < K; ++c) rot[c] = __shfl_sync(0xffffffffu, E[c], (lane + 1) & 31);
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    const int d = 64 * c + 2 * lane + 1;
                    const double up = (lane == 31) ? (c == K - 1 ? SENT : rot[c < K - 1 ? c + 1 : c]) : rot[c];
                    const int i = (a - d + w) >> 1, j = i + d - w;
                    const bool ok = d < W2 && i >= 0 && j >= 0 && i <= R && j <= R;
                    const int ic = ok ? i : 0, jc = ok ? j : 0;
                    const double v = wave_cell<METRIC>(ic, jc, up, E[c], O[c], X, Y, arg);
                    O[c] = ok ? v : SENT;
                }
            }
            if ((a & 7) == 7 && a < 2 * R) {
                // bound over anti-diagonals a-1 and a
                double ext = SENT;
                if (METRIC == LCSS) {
#pragma unroll
                    for (int c = 0; c < K; ++c) ext = wmax(ext, wmax(E[c], O[c]));
                    for (int o = 16; o; o >>= 1) ext = wmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
                    const int imin = max(0, (a - 1 - w) >> 1);  // no row of the pair lies above imin
                    double rest = (double)(R - imin);
                    if (cascade) rest = fmin(rest, S4[(imin + 1) >> 2]);
                    if (dadd(ext, rest) < lcss_lim) stop = true;
                } else {
#pragma unroll
                    for (int c = 0; c < K; ++c) ext = wmin(ext, wmin(E[c], O[c]));
                    for (int o = 16; o; o >>= 1) ext = wmin(ext, __shfl_xor_sync(0xffffffffu, ext, o));
                    const int imax = min(R, (a + w) >> 1);  // no row of the pair lies below imax
                    const double rest = cascade ? S4[min(nblk, (imax + 4) >> 2)] : 0.0;
                    const double bnd = dadd(ext, rest);
                    if (METRIC == DTW || METRIC == ERP) stop = neg_lim || bnd > cut_sq;
                    else stop = bnd > cut_s;
                }
                if (stop) break;
            }
        }
        if (stop) {
            cells += (unsigned long long)((a + 2) >> 1) * (unsigned long long)W2;
            __syncwarp();
            continue;
        }
        cells += (unsigned long long)(R + 1 - (ONE_BASED ? 1 : 0)) * (unsigned long long)W2;
        double fin = SENT;
#pragma unroll
        for (int c = 0; c < K; ++c)
            if (c == fin_chunk) fin = fin_odd ? O[c] : E[c];
        fin = __shfl_sync(0xffffffffu, fin, fin_lane);
        double dist;
        if (METRIC == DTW || METRIC == ERP) dist = isfinite(fin) ? dsqrt(dmax0(fin)) : kDpMax;
        else if (METRIC == LCSS) dist = dsub(1.0, ddiv(fin, (double)m));
        else dist = fin;
        if (lane == 0 && dist <= cut && isfinite(dist)) {
            const unsigned long long o = atomicAdd(job.n_out, 1ull);
            if (o < (unsigned long long)job.out_cap) {
                job.out_idx[o] = gi;
                job.out_dist[o] = dist;
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        if (job.n_valid && valid_count) atomicAdd(job.n_valid, valid_count);
        if (job.n_cells && cells) atomicAdd(job.n_cells, cells);
    }
}

__host__ __device__ size_t dpw_warp_doubles(int m) {
    // candidate [m] (rounded to even) + suffix sums [ceil((m+1)/4) + 1], rounded to even
    const size_t y = ((size_t)m + 1) & ~(size_t)1;
    const size_t s4 = ((size_t)(m + 4) / 4 + 2) & ~(size_t)1;
    return y + s4;
}

#define FSM_DPW_INST(M)                                     \
    template __global__ void k_dpw<M, 1>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 2>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 3>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 4>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 5>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 6>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 7>(Geom, DpJob);      \
    template __global__ void k_dpw<M, 8>(Geom, DpJob);
FSM_DPW_INST(DTW)
FSM_DPW_INST(ERP)
FSM_DPW_INST(EDR)
FSM_DPW_INST(LCSS)
FSM_DPW_INST(MSM)

template <int M>
static const void* dpw_for(int k) {
    switch (k) {
        case 1: return (const void*)k_dpw<M, 1>;
        case 2: return (const void*)k_dpw<M, 2>;
        case 3: return (const void*)k_dpw<M, 3>;
        case 4: return (const void*)k_dpw<M, 4>;
        case 5: return (const void*)k_dpw<M, 5>;
        case 6: return (const void*)k_dpw<M, 6>;
        case 7: return (const void*)k_dpw<M, 7>;
        case 8: return (const void*)k_dpw<M, 8>;
        default: return nullptr;
    }
}

const void* dpw_kernel(int metric, int w) {
    const int k = (2 * w + 1 + 63) / 64;
    if (k < 1 || k > kDpwMaxChunks) return nullptr;
    switch (metric) {
        case DTW: return dpw_for<DTW>(k);
        case ERP: return dpw_for<ERP>(k);
        case EDR: return dpw_for<EDR>(k);
        case LCSS: return dpw_for<LCSS>(k);
        default: return dpw_for<MSM>(k);
    }
}

}  // namespace fsm
