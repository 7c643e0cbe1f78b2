// GLB second filter (src/glb.cpp:200-373), split in the reference's own two
// directions:
//  * k_glb_tq: one lane per LB_IP survivor computes the boundary term and the
//    T->Q sum with early abandon, z-normalising candidate points lazily
//    (t - mu) / sigma exactly as src/fsmeld.cpp:823-826 does (one correctly
//    rounded division, taken from the window's reciprocal by FMA corrections),
//    so abandoned candidates never pay for the whole window;
//  * k_glb_qt: one lane per T->Q survivor adds the Q->T terms in the
//    reference's order.  The candidate envelope (lower_upper_lemire of the
//    z-normalised window, src/glb.cpp:302-304) is never materialised:
//    z-normalisation x -> (x - mu) / sigma is monotone even after rounding,
//    so the minimum of the normalised points equals the normalised minimum of
//    the raw points, bit for bit; every envelope point, edge or interior, is
//    the min/max of two forward windows of the target (k_fwd_env).
// Early abandon compares a running sum of non-negative terms with the
// cutoff; running sums never decrease, so testing the final sum once is the
// same decision as testing after every term.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

__device__ __forceinline__ double edr_sub(double a, double b, double eps) {
    return (fabs(dsub(a, b)) <= eps) ? 0.0 : 1.0;
}
__device__ __forceinline__ double dminv(double a, double b) { return (a < b) ? a : b; }  // MIN macro
__device__ __forceinline__ double dmaxv(double a, double b) { return (a > b) ? a : b; }  // MAX macro

// warp-aggregated append; returns nothing, writes entry via functor
template <typename F>
__device__ __forceinline__ void warp_append(bool pred, unsigned long long* counter, F write) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) write(base + __popc(mask & ((1u << lane) - 1)));
}

// N quotients dividend(u) / sg (zdiv) with one range test for the group: a
// group with any estimate outside the reciprocal method's range (zero
// dividends, extreme scales) is divided directly -- the same bits either way,
// one branch per group instead of one per point.  The rare direct path
// evaluates the dividends again rather than keeping them live.
template <int N, typename F>
__device__ __forceinline__ void zdiv_group(F dividend, double sg, double inv, bool ok, double (&z)[N]) {
    bool good = ok;
#pragma unroll
    for (int u = 0; u < N; ++u) {
        const double a = dividend(u);
        const double q0 = rcp_div_estimate(a, inv);
        good = good & (rcp_div_in_range_bits(q0) != 0);
        z[u] = rcp_div_finish(a, sg, inv, q0);
    }
    if (!good) {
#pragma unroll
        for (int u = 0; u < N; ++u) z[u] = ddiv(dividend(u), sg);
    }
}

}  // namespace

// T->Q term of normalised candidate point t against the query envelope
// [lo, hi] at the same index (src/glb.cpp:230-300), written with selects so
// lanes never split on the data.  lo <= hi, so at most one of t < lo, t > hi
// holds: the side is selected first and one distance computed to it.
template <int METRIC>
__device__ __forceinline__ double tq_term(double t, double lo, double hi, double arg) {
    const bool below = t < lo, above = t > hi;
    const double e = above ? hi : lo;  // the nearer side when outside
    if (METRIC == DTW) {
        const double a = dsq(t, e);
        return (below || above) ? a : 0.0;
    } else if (METRIC == ERP) {
        const double a = dminv(dsq(t, e), dsq(t, arg));
        return (below || above) ? a : 0.0;
    } else if (METRIC == EDR) {
        const double a = edr_sub(t, e, arg);
        return (below || above) ? a : 0.0;
    } else if (METRIC == LCSS) {  // match indicator: lo - t or t - hi within eps
        const bool a = dsub(below ? lo : t, below ? t : hi) <= arg;
        return ((below || above) ? a : true) ? 1.0 : 0.0;
    } else {  // MSM
        const double a = dminv(fabs(dsub(t, e)), arg);
        return (below || above) ? a : 0.0;
    }
}

template <int METRIC>
__global__ void __launch_bounds__(256, 4) k_glb_tq(Geom g, GlbJob job) {
    extern __shared__ double gq_smem[];
    const QueryDev& q = job.q;
    const int m = q.m;
    double* Q = gq_smem;
    double* LQ = Q + m;
    double* UQ = LQ + m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) { Q[i] = q.qn[i]; LQ[i] = q.LQ[i]; UQ[i] = q.UQ[i]; }
    __syncthreads();
    const double bsf = job.cutoff_ptr ? *job.cutoff_ptr : q.cutoff;
    const double sq = dmul(bsf, bsf);  // glb_exceeds_squared_bsf, src/glb.cpp:28-31
    const double lim = (METRIC == DTW || METRIC == ERP) ? sq : bsf;
    const double arg = q.arg;
    const unsigned long long n_in = *job.n_in;
    const unsigned long long n_lim = n_in < (unsigned long long)job.in_cap ? n_in : job.in_cap;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < n_lim;
         base += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long idx = base + threadIdx.x;
        const bool active = idx < n_lim;
        long long gi = 0;
        double mu = 0.0, sg = 1.0, inv = 1.0;
        if (active) {
            gi = job.in[idx];
            long long s;
            int j;
            g.locate(gi, &s, &j);
            mu = job.MU[s * g.kml + j];
            sg = job.SIG[s * g.kml + j];
            inv = __drcp_rn(sg);
        }
        const bool rok = rcp_div_in_range(sg);
        const double* tp = job.target + gi;
        bool alive = active;
        double boundary = 0.0, tq = 0.0;
        if (active) {
#define TN(k) zdiv_i(dsub(tp[(k)], mu), sg, inv, rok)
            const double T0 = TN(0), TL = TN(m - 1);
            if (METRIC == DTW) {
                boundary = dadd(dsq(T0, Q[0]), dsq(TL, Q[m - 1]));
            } else if (METRIC == ERP) {
                boundary = dmin3(dsq(Q[m - 1], TL), dsq(Q[m - 1], arg), dsq(TL, arg));
            } else if (METRIC == EDR) {
                boundary = dminv(edr_sub(Q[m - 1], TL, arg), 1.0);
            } else if (METRIC == MSM) {
                const double T2 = TN(m - 2);
                const double q0 = Q[0], ql = Q[m - 1], ql2 = Q[m - 2];
                if ((T2 >= TL && TL >= ql) || (T2 <= TL && TL <= ql) || (ql2 <= ql && ql <= TL) ||
                    (ql2 >= ql && ql >= TL)) {
                    boundary = dadd(fabs(dsub(q0, T0)), dminv(fabs(dsub(ql, TL)), arg));
                } else {
                    boundary = dadd(fabs(dsub(q0, T0)),
                                    dmin3(fabs(dsub(ql, TL)), dadd(arg, fabs(dsub(TL, T2))),
                                          dadd(arg, fabs(dsub(ql, ql2)))));
                }
            }
            if (METRIC == LCSS) {
                // every point, no abandon (src/glb.cpp:238-252)
                const double min_len = (double)m;
                int k = 0;
                for (; k + 4 <= m; k += 4) {
                    double z4[4], t4[4];
                    zdiv_group([&](int u) { return dsub(tp[k + u], mu); }, sg, inv, rok, z4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) t4[u] = tq_term<LCSS>(z4[u], LQ[k + u], UQ[k + u], arg);
#pragma unroll
                    for (int u = 0; u < 4; ++u) tq = dadd(tq, t4[u]);
                }
                for (; k < m; ++k) tq = dadd(tq, tq_term<LCSS>(TN(k), LQ[k], UQ[k], arg));
                if (dmax0(dsub(1.0, ddiv(tq, min_len))) > bsf) alive = false;
            } else {
                // points 1..m-2 four at a time: the four normalisations are
                // independent, the sum takes them in the reference's order, and
                // the abandon test runs once per group -- the sum never
                // decreases, so a sum past the limit anywhere in the group is
                // past it at the group's end (the same decision)
                int k = 1;
                for (; k + 4 <= m - 1; k += 4) {
                    double z4[4], t4[4];
                    zdiv_group([&](int u) { return dsub(tp[k + u], mu); }, sg, inv, rok, z4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) t4[u] = tq_term<METRIC>(z4[u], LQ[k + u], UQ[k + u], arg);
#pragma unroll
                    for (int u = 0; u < 4; ++u) tq = dadd(tq, t4[u]);
                    if (dadd(boundary, tq) > lim) { alive = false; break; }
                }
                if (alive) {
                    for (; k < m - 1; ++k) tq = dadd(tq, tq_term<METRIC>(TN(k), LQ[k], UQ[k], arg));
                    if (dadd(boundary, tq) > lim) alive = false;
                }
            }
#undef TN
        }
        if (active && !alive) {
            // abandoned: GLB returns MAX_VAL (src/glb.cpp:221 etc.); it survives only if
            // MAX_VAL <= cutoff
            if (kGlbMax <= bsf) alive = true, boundary = -1.0;  // marker: keep as MAX_VAL
        }
        warp_append(alive, job.n_out, [&](unsigned long long o) {
            if (o < (unsigned long long)job.out_cap) {
                job.out[o] = gi;
                job.out_b[o] = boundary;
                job.out_t[o] = tq;
            }
        });
    }
}

// Forward windows of the raw target: lo/up[p] = min/max(t[p .. min(n-1, p+w)])
// with fmin/fmax (NaN ignored unless the whole window is NaN; only windows
// inside valid candidate windows, which hold no NaN, are ever read).
//
// Doubling in shared memory: after pass k, M[i] = min(t[i .. i + 2^k - 1]);
// a window of length L = w+1 is the union of the two length-2^K runs at its
// ends (2^K <= L < 2^(K+1)), min(M[p], M[p + L - 2^K]) -- the same set, so
// the same value as a direct scan.  log2(L) passes of one min per element
// replace the L reads per output of a direct scan, so the cost no longer
// grows with the radius.  A CTA produces kFwdTile outputs per tile from the
// tile plus its w-point halo, ping-ponging between two shared buffers.
__global__ void __launch_bounds__(kFwdThreads) k_fwd_env(const double* __restrict__ t, long long n, int w,
                                                        double* __restrict__ lo, double* __restrict__ up) {
    extern __shared__ double fw_smem[];
    const int ext = kFwdTile + w;  // tile plus halo
    double* An = fw_smem;
    double* Ax = An + ext;
    double* Bn = Ax + ext;
    double* Bx = Bn + ext;
    const int L = w + 1;
    int K = 0;
    while ((2 << K) <= L) ++K;  // 2^K <= L < 2^(K+1)
    const int off = L - (1 << K);
    for (long long p0 = (long long)blockIdx.x * kFwdTile; p0 < n; p0 += (long long)gridDim.x * kFwdTile) {
        const int cnt = (int)((n - p0) < ext ? (n - p0) : ext);
        for (int i = threadIdx.x; i < ext; i += kFwdThreads) {
            const double v = i < cnt ? t[p0 + i] : NAN;
            An[i] = v;
            Ax[i] = v;
        }
        __syncthreads();
        for (int k = 0; k < K; ++k) {
            const int s = 1 << k;
            for (int i = threadIdx.x; i < ext; i += kFwdThreads) {
                const bool in = i + s < ext;
                Bn[i] = in ? fmin(An[i], An[i + s]) : An[i];
                Bx[i] = in ? fmax(Ax[i], Ax[i + s]) : Ax[i];
            }
            __syncthreads();
            double* tn = An; An = Bn; Bn = tn;
            double* tx = Ax; Ax = Bx; Bx = tx;
        }
        for (int i = threadIdx.x; i < kFwdTile; i += kFwdThreads) {
            const long long p = p0 + i;
            if (p >= n) break;
            double mn, mx;
            if (p + w <= n - 1) {
                mn = fmin(An[i], An[i + off]);
                mx = fmax(Ax[i], Ax[i + off]);
            } else {  // the last w points: the window is clipped at the end of the target
                mn = t[p];
                mx = t[p];
                for (long long j = p + 1; j < n; ++j) {
                    mn = fmin(mn, t[j]);
                    mx = fmax(mx, t[j]);
                }
            }
            lo[p] = mn;
            up[p] = mx;
        }
        __syncthreads();
    }
}

size_t fwd_env_smem_bytes(int w) { return sizeof(double) * 4 * (size_t)(kFwdTile + w); }

// one lane per T->Q survivor: Q->T terms added in the reference's order
template <int METRIC>
__global__ void __launch_bounds__(128) k_glb_qt(Geom g, GlbJob job) {
    extern __shared__ double gqt_smem[];
    const QueryDev& q = job.q;
    const int m = q.m, w = q.w;
    double* Q = gqt_smem;
    for (int i = threadIdx.x; i < m; i += blockDim.x) Q[i] = q.qn[i];
    __syncthreads();
    const double bsf = job.cutoff_ptr ? *job.cutoff_ptr : q.cutoff;
    const double sq = dmul(bsf, bsf);
    const double arg = q.arg;
    const unsigned long long n_in = *job.n_in;
    const unsigned long long n_lim = n_in < (unsigned long long)job.in_cap ? n_in : job.in_cap;
    for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < n_lim;
         c += (unsigned long long)gridDim.x * blockDim.x) {
        const long long gi = job.in[c];
        const double boundary = job.in_b[c];
        const double tq = job.in_t[c];
        long long s;
        int j;
        g.locate(gi, &s, &j);
        double glb, qt = 0.0;
        if (boundary == -1.0) {
            glb = kGlbMax;  // abandoned in T->Q but MAX_VAL <= cutoff
        } else {
            const double mu = job.MU[s * g.kml + j], sg = job.SIG[s * g.kml + j];
            const double inv = __drcp_rn(sg);
            const bool rok = rcp_div_in_range(sg);
            const double* lf = job.lraw + gi;
            const double* uf = job.uraw + gi;
            const int k0 = (METRIC == LCSS) ? 0 : 1, k1 = (METRIC == LCSS) ? m - 1 : m - 2;
            // the terms are independent (unrolled so their loads and divisions
            // overlap); only the sum is sequential, in the reference's order.
            // Interior points (w <= k <= m-1-w) read the windows at k-w and k
            // directly; the edges take the clamped indices.
            const int i0 = max(k0, w), i1 = min(k1, m - 1 - w);
            int k = k0;
            for (; k <= k1 && k < i0; ++k) qt = dadd(qt, qt_term(METRIC, Q[k], k, m, w, lf, uf, mu, sg, inv, rok, arg));
            for (; k + 1 <= i1; k += 2) {  // two points, four quotients, one range test
                double z4[4];
                zdiv_group(
                    [&](int u) {
                        const int kk = k + (u & 1);
                        if (u < 2) { const double a0 = lf[kk - w], a1 = lf[kk]; return dsub((a1 < a0) ? a1 : a0, mu); }
                        const double b0 = uf[kk - w], b1 = uf[kk];
                        return dsub((b0 < b1) ? b1 : b0, mu);
                    },
                    sg, inv, rok, z4);
                qt = dadd(qt, qt_term_norm(METRIC, Q[k], z4[0], z4[2], arg));
                qt = dadd(qt, qt_term_norm(METRIC, Q[k + 1], z4[1], z4[3], arg));
            }
            for (; k <= i1; ++k) {
                const double a0 = lf[k - w], a1 = lf[k], b0 = uf[k - w], b1 = uf[k];
                qt = dadd(qt, qt_term_env(METRIC, Q[k], (a1 < a0) ? a1 : a0, (b0 < b1) ? b1 : b0, mu, sg, inv, rok,
                                          arg));
            }
            for (; k <= k1; ++k) qt = dadd(qt, qt_term(METRIC, Q[k], k, m, w, lf, uf, mu, sg, inv, rok, arg));
            if (METRIC == LCSS) {
                glb = dmax0(dsub(1.0, ddiv(dminv(tq, qt), (double)m)));
            } else {
                const double tot = dadd(boundary, qt);
                if (METRIC == DTW || METRIC == ERP)
                    glb = (tot > sq) ? kGlbMax : dsqrt(dmax0(dadd(boundary, dmaxv(tq, qt))));
                else
                    glb = (tot > bsf) ? kGlbMax : dadd(boundary, dmaxv(tq, qt));
            }
        }
        if (glb <= bsf) {
            const unsigned long long o = atomicAdd(job.n_out, 1ull);
            if (o < (unsigned long long)job.out_cap) {
                job.out[o] = gi;
                if (job.out_t) job.out_t[o] = (boundary == -1.0) ? -1.0 : qt;
            }
            if (job.segc && s < g.forsize) atomicAdd((unsigned long long*)&job.segc[3 * s + 2], 1ull);
        }
    }
}

#define FSM_GLB_INST(M)                                       \
    template __global__ void k_glb_tq<M>(Geom, GlbJob);       \
    template __global__ void k_glb_qt<M>(Geom, GlbJob);
FSM_GLB_INST(DTW)
FSM_GLB_INST(ERP)
FSM_GLB_INST(EDR)
FSM_GLB_INST(LCSS)
FSM_GLB_INST(MSM)

}  // namespace fsm
