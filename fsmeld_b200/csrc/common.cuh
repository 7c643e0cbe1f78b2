// Shared definitions for the FSMELD sm_100a kernels.
//
// Bit-exactness: every stage whose bits decide a match (window statistics,
// candidate z-normalisation, GLB, the elastic DPs, the threshold sweep) uses
// explicit round-to-nearest intrinsics (__dadd_rn, __dmul_rn, ...), which the
// compiler never contracts into fused multiply-adds, so each operation rounds
// exactly as the reference's scalar C++ does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rcpdiv.h"

namespace fsm {

constexpr double kDpMax = 1e18;                     // src/ElasticMeasures.cpp:7
constexpr double kGlbMax = (double)1008610086;      // include/def.h:7
constexpr double kSigmaFloor = 1e-12;               // src/fsmeld.cpp:126,129
constexpr double kLbTol = 1e-9;                     // include/fsmeld_internal.h:10

enum Metric : int { DTW = 1, EDR = 2, ERP = 3, LCSS = 4, MSM = 5 };

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000LL); }
__device__ __forceinline__ double dsq(double a, double b) { double d = dsub(a, b); return dmul(d, d); }
// a / sg correctly rounded, from inv = RN(1/sg): the reciprocal and two FMA
// corrections of rcpdiv.h when sg (ok) and the quotient estimate are in that
// method's range, a division otherwise -- the same bits either way
__device__ __forceinline__ double zdiv(double a, double sg, double inv, bool ok) {
    const double q0 = rcp_div_estimate(a, inv);
    if (ok && rcp_div_in_range(q0)) return rcp_div_finish(a, sg, inv, q0);
    return ddiv(a, sg);
}
// zdiv with the estimate's range tested on the integer pipe
__device__ __forceinline__ double zdiv_i(double a, double sg, double inv, bool ok) {
    const double q0 = rcp_div_estimate(a, inv);
    if (ok && rcp_div_in_range_bits(q0)) return rcp_div_finish(a, sg, inv, q0);
    return ddiv(a, sg);
}
// std::max(0.0, x): (0.0 < x) ? x : 0.0 (a NaN x gives 0.0)
__device__ __forceinline__ double dmax0(double x) { return (0.0 < x) ? x : 0.0; }
// std::min({a, b, c}) for non-NaN operands
__device__ __forceinline__ double dmin3(double a, double b, double c) {
    double r = a;
    if (b < r) r = b;
    if (c < r) r = c;
    return r;
}

// Macro-segment geometry of one (target, m) pair (src/fsmeld.cpp:28-37,
// 647-661): segment s < forsize starts at s*kml; the last segment (when
// tail > 0) is the EOF-aligned tail whose processed windows are
// [tail_lo, kml).  Window j of segment s has global index s*kml + j - lo(s),
// which is also its start position in the target.
struct Geom {
    long long n;
    int m, m_k, kml;
    int tail_lo;           // kml - tail (== kml when there is no tail)
    long long forsize, S;  // full segments; total segments including the tail
    long long tsn;         // n - m + 1 windows
    long long excl_b, excl_e;
    double inv_kml;        // fl(1 / kml), for the quotient estimate in locate()
    // raw (non-normalised) mode: every window whose points are all finite gets
    // mean 0 and sigma 1, so the z-normalisation (t - 0) / 1 leaves it as is
    int raw = 0;
    __host__ __device__ long long off(long long s) const { return s < forsize ? s * kml : n - m_k; }
    __host__ __device__ int lo(long long s) const { return s < forsize ? 0 : tail_lo; }
    __host__ __device__ long long gidx(long long s, int j) const { return s * kml + (j - lo(s)); }
    // statistics row/column of global window g
    __host__ __device__ void locate(long long g, long long* s, int* j) const {
        // g / kml without a 64-bit integer division: the double estimate is
        // within one of the quotient for g < 2^52; one step corrects it
        long long q = (long long)((double)g * inv_kml);
        long long r = g - q * kml;
        if (r < 0) { --q; r += kml; }
        else if (r >= kml) { ++q; r -= kml; }
        if (q < forsize) { *s = q; *j = (int)r; }
        else { *s = forsize; *j = tail_lo + (int)(g - forsize * kml); }
    }
    __host__ __device__ bool excluded(long long g) const {
        return excl_b >= 0 && excl_e > excl_b && g >= excl_b && g < excl_e;
    }
};

// src/fsmeld.cpp:126 (with mvmean's NaN for non-finite windows) and the
// exclusion interval of src/fsmeld.cpp:139-152.
__device__ __forceinline__ bool window_invalid(double sigma, const Geom& g, long long gi) {
    return !(isfinite(sigma) && sigma > kSigmaFloor) || g.excluded(gi);
}

// include/fsmeld_internal.h:9-19: prune only bounds that exceed the cutoff by
// more than the FFT round-off guard.
__device__ __forceinline__ bool lbip_exceeds(double bound, double cutoff, int metric) {
    if (!isfinite(bound) || !(bound > dadd(cutoff, kLbTol))) return false;
    if (metric == DTW || metric == ERP) {
        const double limit = dadd(cutoff, kLbTol);
        return bound > dsqrt(dadd(dmul(limit, limit), kLbTol));
    }
    return true;
}

// Q->T term of query point x (index k) against the candidate envelope: the
// per-point term of src/glb.cpp:306-372; LCSS returns the match indicator.
// The candidate envelope at k is the min/max of the z-normalised window over
// [max(0, k-w), min(m-1, k+w)] (lower_upper_lemire, src/glb.cpp:302-304).
// x -> (x - mu) / sigma is monotone, so min/max commute with it exactly and
// the raw min/max suffice.  lf/uf hold the target's forward windows
// min/max(t[p .. p+w]) from the candidate start: the two windows starting at
// p0 = max(0, k-w) and p1 = min(k, m-1-w) lie inside the candidate window and
// their union is exactly [max(0, k-w), min(m-1, k+w)], so every point, edge
// or interior, costs the same two reads per side.
__device__ __forceinline__ int qt_p0(int k, int w) { return k - w < 0 ? 0 : k - w; }
__device__ __forceinline__ int qt_p1(int k, int m, int w) { return k < m - 1 - w ? k : m - 1 - w; }

// The term from the raw window minimum a and maximum b of the candidate at k.
// The term from the normalised envelope [lo, up] of the candidate at k.
__device__ __forceinline__ double qt_term_norm(int metric, double x, double lo, double up, double arg) {
    switch (metric) {
        case DTW:
            if (x < lo) return dsq(x, lo);
            if (x > up) return dsq(x, up);
            return 0.0;
        case ERP:
            if (x > up) { const double p = dsq(x, up), r = dsq(x, arg); return (p < r) ? p : r; }
            if (x < lo) { const double p = dsq(x, lo), r = dsq(x, arg); return (p < r) ? p : r; }
            return 0.0;
        case EDR:
            if (x > up) return (fabs(dsub(x, up)) <= arg) ? 0.0 : 1.0;
            if (x < lo) return (fabs(dsub(x, lo)) <= arg) ? 0.0 : 1.0;
            return 0.0;
        case LCSS:
            if (x < lo) return (dsub(lo, x) <= arg) ? 1.0 : 0.0;
            if (x > up) return (dsub(x, up) <= arg) ? 1.0 : 0.0;
            return 1.0;
        default:
            if (x > up) { const double p = fabs(dsub(x, up)); return (p < arg) ? p : arg; }
            if (x < lo) { const double p = fabs(dsub(x, lo)); return (p < arg) ? p : arg; }
            return 0.0;
    }
}

__device__ __forceinline__ double qt_term_env(int metric, double x, double a, double b, double mu, double sg,
                                              double inv, bool ok, double arg) {
    return qt_term_norm(metric, x, zdiv(dsub(a, mu), sg, inv, ok), zdiv(dsub(b, mu), sg, inv, ok), arg);
}

// The same term for the DP's cascading abandon test, without divisions: the
// window bounds are scaled by inv = fl(1/sigma) (relative error ~2^-52) and
// the envelope is then narrowed by a relative 2^-49 (lo raised, up lowered),
// so it lies inside the exact envelope.  Every term is then at least the
// exact term (DTW/ERP/EDR/MSM: distances to a narrower envelope) and LCSS's
// match indicator at most the exact one; the abandon bound built from these
// terms can only be looser than the exact one, never tighter.
__device__ __forceinline__ double qt_term_bound(int metric, double x, double a, double b, double mu, double inv,
                                                double arg) {
    double lo = dmul(dsub(a, mu), inv);
    double up = dmul(dsub(b, mu), inv);
    lo = dadd(lo, dadd(dmul(fabs(lo), 0x1p-49), 0x1p-1000));
    up = dsub(up, dadd(dmul(fabs(up), 0x1p-49), 0x1p-1000));
    switch (metric) {
        case DTW:
            if (x < lo) return dsq(x, lo);
            if (x > up) return dsq(x, up);
            return 0.0;
        case ERP:
            if (x > up) { const double p = dsq(x, up), r = dsq(x, arg); return (p < r) ? p : r; }
            if (x < lo) { const double p = dsq(x, lo), r = dsq(x, arg); return (p < r) ? p : r; }
            return 0.0;
        case EDR:
            if (x > up) return (fabs(dsub(x, up)) <= arg) ? 0.0 : 1.0;
            if (x < lo) return (fabs(dsub(x, lo)) <= arg) ? 0.0 : 1.0;
            return 0.0;
        case LCSS:
            if (x < lo) return (dsub(lo, x) <= arg) ? 1.0 : 0.0;
            if (x > up) return (dsub(x, up) <= arg) ? 1.0 : 0.0;
            return 1.0;
        default:
            if (x > up) { const double p = fabs(dsub(x, up)); return (p < arg) ? p : arg; }
            if (x < lo) { const double p = fabs(dsub(x, lo)); return (p < arg) ? p : arg; }
            return 0.0;
    }
}

__device__ __forceinline__ double qt_term(int metric, double x, int k, int m, int w, const double* lf,
                                          const double* uf, double mu, double sg, double inv, bool ok,
                                          double arg) {
    const int p0 = qt_p0(k, w), p1 = qt_p1(k, m, w);
    // valid windows hold no NaN: a comparison and a select give the min / max
    const double a0 = lf[p0], a1 = lf[p1], b0 = uf[p0], b1 = uf[p1];
    return qt_term_env(metric, x, (a1 < a0) ? a1 : a0, (b0 < b1) ? b1 : b0, mu, sg, inv, ok, arg);
}

// Per-query tables prepared on the host (query z-normalisation as
// src/fsmeld.cpp:622-643, powers with the C library's pow as
// src/find_t_lp.cpp:253 etc.).
struct QueryDev {
    int m, w, metric, p;
    double arg;
    double cutoff;
    const double* qn;      // normalised query, original order [m]
    const double* LQ;      // query envelope (radius w) [m]
    const double* UQ;
    const double* qs;      // sorted ascending [m]
    const double* pw;      // pow(qs[j], a) for a = 0,1,2: [3][m]
    const double* Dq;      // D(qs[j]) [m]   (src/find_t_lp.cpp:148-159)
    const double* tlq;     // t_l(qs[j]) [m] (src/find_t_lp.cpp:177-186)
    const double* tuq;     // t_u(qs[j]) [m] (src/find_t_lp.cpp:167-176)
    // ERP (src/find_t_lp.cpp:510-654): tables by original query index
    const double* opw;     // pow(qn[i], a): [3][m]
    const double* oD;      // D(qn[i]) [m]
    const double* otl;     // t_l(qn[i]) [m]
    const double* otu;     // t_u(qn[i]) [m]
    const int* ordA_l;     // H2 pop order, lower side: t_l desc, index asc
    const int* ordB_l;     // H1 pop order, lower side: q desc
    const int* ordA_u;     // H2 pop order, upper side: t_u asc, index asc
    const int* ordB_u;     // H1 pop order, upper side: q asc
};

}  // namespace fsm

#define FSM_CUDA_TRY(expr)                                                        \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) return ::fsm::cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

namespace fsm {
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);
}
