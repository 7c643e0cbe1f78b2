// C-callable wrappers around the reference's own hot-path functions, compiled
// together with the reference sources (unmodified, read in place) into
// oracle/_ref/libfsmeld_ref.so.  Test infrastructure only: the tests use these
// entry points to pin the C restatement (fsmeld_oracle.c) function by function
// against the reference's bits.  Each wrapper names the reference function it
// forwards to (file:line in the reference tree).
#include "funcs.h"
#include "fsmeld_internal.h"

#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>

namespace {
char* tag_of(int metric) {
    static char names[6][8] = {"", "dtw", "edr", "erp", "lcss", "msm"};
    return names[metric];
}
}

extern "C" {

// src/mvmean.cpp:9-46
void ref_mvmean(double* a, int len_a, int l, double* miu, double* si) {
    mvmean(a, len_a, l, miu, si);
}

// src/fsmeld.cpp:110-153 (no exclusion interval active)
void ref_invalid_mask(const double* t, const double* si, int seg, int m, uint8_t* out) {
    std::vector<char> mask(seg > 0 ? seg : 1, 0);
    precompute_invalid_mask_fast(t, si, seg, m, reinterpret_cast<bool*>(mask.data()));
    for (int j = 0; j < seg - m + 1; ++j) out[j] = mask[j] ? 1 : 0;
}

// src/lower_upper_lemire.cpp:94-126
void ref_min_max_window(double* a, int n, int m, double* mn, double* mx) {
    min_max_window(a, n, m, mn, mx);
}

// src/lower_upper_lemire.cpp:8-44
void ref_lemire(double* a, int n, int r, double* l, double* u) {
    lower_upper_lemire(a, n, r, l, u);
}

// src/lb_normalize.cpp:9-32
void ref_normalized(const double* U, const double* L, double* Un, double* Ln, int len,
                    double* max_mean, double* min_mean, double* max_std, double* min_std) {
    compute_normalized_arrays(U, L, Un, Ln, len, max_mean, min_mean, max_std, min_std);
}

// src/find_t_lp.cpp:218-398,510-825, selected per metric as src/fsmeld.cpp:778-790
double ref_find_t(int upper, int metric, double* env, int l, double* q, int m, double arg) {
    int p = (metric == METRIC_DTW || metric == METRIC_ERP) ? 2 : (metric == METRIC_MSM ? 1 : 0);
    std::vector<double> LB(l - 2 * m + 2 > 0 ? l - 2 * m + 2 : 1);
    std::vector<double> m_p(p + 1);
    std::vector<double> qs(q, q + m);
    std::sort(qs.begin(), qs.end());
    char* tag = tag_of(metric);
    if (metric == METRIC_DTW) {
        return upper ? find_tu_lp_dtw(env, l, q, m, p, LB.data(), m_p.data(), tag, qs.data())
                     : find_tl_lp_dtw(env, l, q, m, p, LB.data(), m_p.data(), tag, qs.data());
    }
    if (metric == METRIC_ERP) {
        return upper ? find_tu_lp_erp(env, l, q, m, p, arg, LB.data(), m_p.data())
                     : find_tl_lp_erp(env, l, q, m, p, arg, LB.data(), m_p.data());
    }
    return upper ? find_tu_lp(env, l, q, m, p, arg, LB.data(), m_p.data(), tag, qs.data())
                 : find_tl_lp(env, l, q, m, p, arg, LB.data(), m_p.data(), tag, qs.data());
}

// src/q_to_h.cpp:11-64 (lower) and 84-134 (upper)
void ref_q_to_h(int upper, int metric, const double* q, int m, double t, double arg, double* h) {
    if (upper) q_to_h_u(q, m, t, arg, h, m, tag_of(metric));
    else q_to_h_l(q, m, t, arg, h, m, tag_of(metric));
}

// src/lb.cpp:18-34
void ref_s_to_g(int upper, const double* env, int n, double t, double* g) {
    if (upper) s_to_g_u(env, n, t, g, n);
    else s_to_g_l(env, n, t, g, n);
}

// src/sip.cpp:16-52 as sequenced at src/fsmeld.cpp:798-806
void ref_sip(int n, int m, double* h, double* g, double* z) {
    double* Z = (double*)fftw_alloc_real(n);
    fftw_complex* XX = fftw_alloc_complex(n / 2 + 1);
    fftw_complex* YY = fftw_alloc_complex(n / 2 + 1);
    fftw_complex* ZZ = fftw_alloc_complex(n / 2 + 1);
    fftw_plan r2c = fftw_plan_dft_r2c_1d(n, Z, ZZ, FFTW_ESTIMATE);
    fftw_plan c2r = fftw_plan_dft_c2r_1d(n, ZZ, Z, FFTW_ESTIMATE);
    inv_and_padding_y(n, m, h, YY, r2c);
    FFT_x(g, XX, r2c);
    cov_IFFT(XX, YY, ZZ, n, z, c2r);
    fftw_destroy_plan(r2c); fftw_destroy_plan(c2r);
    fftw_free(XX); fftw_free(YY); fftw_free(ZZ); fftw_free(Z);
}

// src/fsmeld.cpp:84-106
void ref_trans(double* zl, double* zu, double* z, int m, int count, int metric) {
    trans(zl, zu, z, m, count, tag_of(metric));
}

// include/fsmeld_internal.h:9-19
int ref_lbip_exceeds(double bound, double cutoff, int metric) {
    return fsmeld_lbip_exceeds_cutoff(bound, cutoff, static_cast<MetricType>(metric)) ? 1 : 0;
}

// src/glb.cpp:200-373
double ref_glb(int metric, double* Q, double* T, int m, double arg, double* LQ, double* UQ,
               int w, double bsf) {
    return glb_elastic(static_cast<MetricType>(metric), Q, m, T, m, arg, LQ, UQ, w, bsf);
}

// src/fsmeld.cpp:170-183 -> src/ElasticMeasures.cpp:24-198
double ref_distance(int metric, double* q, double* t, int m, int w, double arg) {
    return exact_elastic_distance(static_cast<MetricType>(metric), q, t, m, w, arg);
}

}  // extern "C"
