/*
 * fsmeld_oracle.c -- plain-C restatement of the FSMELD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke()) and the "port" CPU baseline in bench.py.
 * The product never links, loads or calls it.
 *
 * Each function follows the cited reference function (file:line in the
 * reference tree) operation by operation, with the same floating-point
 * operation order and no fused multiply-adds (built with -ffp-contract=off),
 * so that its outputs can be compared bit for bit with the reference's own
 * sources built in oracle/_ref.  Parity of this restatement is pinned by
 * tests/test_oracle_pins.py against oracle/_ref and tests/golden/.
 *
 * One documented deviation: the reference sorts threshold candidates with
 * std::sort, whose order is unspecified for equal keys and undefined when the
 * keys contain NaN.  Here candidates sort by value with NaN placed last and
 * ties broken by position, a total order the CUDA path reproduces.  The
 * selected threshold value is the same whenever the envelope core holds no
 * NaN (equal values give equal thresholds); match sets never depend on it.
 */
#include "fsmeld_oracle.h"
#include "fftw_shim/fftw3.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_DP_MAX 1e18                  /* src/ElasticMeasures.cpp:7 */
#define ORC_GLB_MAX ((double)1008610086) /* include/def.h:7 */
#define ORC_MIN(x, y) ((x) < (y) ? (x) : (y))
#define ORC_MAX(x, y) ((x) > (y) ? (x) : (y))

static double dmax0(double x) { return (0.0 < x) ? x : 0.0; } /* std::max(0.0, x) */

/* ------------------------------------------------------------------ geometry */

/* src/fsmeld.cpp:28-37 */
int orc_macro_length(int m, long long available_points) {
    long long selected = 1;
    while (selected < 8LL * m) selected *= 2;
    if (available_points < 2LL * m - 1) return -1;
    if (available_points < selected) selected = available_points;
    if (selected > 2147483647LL) return -1;
    return (int)selected;
}

/* ------------------------------------------------------------- window stats */

/* src/mvmean.cpp:9-46 */
void orc_mvmean(const double* a, int len_a, int l, double* miu, double* si) {
    double sum1 = 0, sum2 = 0;
    int nonfinite = 0;
    for (int i = 0; i < l; i++) {
        if (isfinite(a[i])) {
            sum1 += a[i];
            sum2 += a[i] * a[i];
        } else {
            ++nonfinite;
        }
    }
    const int ll = len_a - l + 1;
    miu[0] = nonfinite ? NAN : sum1 / l;
    si[0] = nonfinite ? NAN : sqrt(sum2 / l - miu[0] * miu[0]);
    for (int i = 1; i < ll; i++) {
        const int of = isfinite(a[i - 1]), inf = isfinite(a[i + l - 1]);
        const double outgoing = of ? a[i - 1] : 0.0;
        const double incoming = inf ? a[i + l - 1] : 0.0;
        nonfinite += !inf - !of;
        sum1 = sum1 - outgoing + incoming;
        sum2 = sum2 - outgoing * outgoing + incoming * incoming;
        miu[i] = nonfinite ? NAN : sum1 / l;
        si[i] = nonfinite ? NAN : sqrt(sum2 / l - miu[i] * miu[i]);
    }
}

/* src/fsmeld.cpp:110-130 (the exclusion part, 131-152, is applied by the drivers) */
void orc_invalid_mask(const double* t, const double* si, int seg, int m, uint8_t* out) {
    const int count = seg - m + 1;
    if (count <= 0) return;
    int bad = 0;
    for (int k = 0; k < m; k++)
        if (!isfinite(t[k])) bad++;
    out[0] = bad > 0;
    for (int j = 1; j < count; j++) {
        if (!isfinite(t[j - 1])) bad--;
        if (!isfinite(t[j + m - 1])) bad++;
        out[j] = bad > 0 || !isfinite(si[j]) || si[j] <= 1e-12;
    }
    out[0] = out[0] || !isfinite(si[0]) || si[0] <= 1e-12;
}

/* src/lower_upper_lemire.cpp:94-126 (trailing window of length m, deque) */
void orc_min_max_window(const double* a, int n, int m, double* mn, double* mx) {
    const int kml = n - m + 1;
    int* ql = (int*)malloc(sizeof(int) * (kml > 0 ? kml : 1));
    int* qu = (int*)malloc(sizeof(int) * (kml > 0 ? kml : 1));
    int hl = 0, tl = -1, hu = 0, tu = -1;
    for (int i = 0; i < kml; i++) {
        while (hl <= tl && a[ql[tl]] >= a[i]) tl--;
        ql[++tl] = i;
        if (ql[hl] <= i - m) hl++;
        mn[i] = a[ql[hl]];
        while (hu <= tu && a[qu[tu]] <= a[i]) tu--;
        qu[++tu] = i;
        if (qu[hu] <= i - m) hu++;
        mx[i] = a[qu[hu]];
    }
    for (int i = kml; i < n; i++) {
        if (ql[hl] <= i - m) hl++;
        mn[i] = a[ql[hl]];
        if (qu[hu] <= i - m) hu++;
        mx[i] = a[qu[hu]];
    }
    free(ql);
    free(qu);
}

/* src/lower_upper_lemire.cpp:8-44 (centred radius-r envelope, deque) */
void orc_lemire(const double* a, int n, int r, double* l, double* u) {
    int li = 0, ui = 0;
    const int k = 2 * r + 1;
    int* qu = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    int* ql = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    int hl = 0, tl = -1, hu = 0, tu = -1;
    for (int i = 0; i < k - 1 - r; i++) {
        while (hl <= tl && a[ql[tl]] >= a[i]) tl--;
        ql[++tl] = i;
        while (hu <= tu && a[qu[tu]] <= a[i]) tu--;
        qu[++tu] = i;
    }
    for (int i = k - 1 - r; i < n; i++) {
        while (hl <= tl && a[ql[tl]] >= a[i]) tl--;
        ql[++tl] = i;
        while (ql[hl] <= i - k) hl++;
        l[li++] = a[ql[hl]];
        while (hu <= tu && a[qu[tu]] <= a[i]) tu--;
        qu[++tu] = i;
        while (qu[hu] <= i - k) hu++;
        u[ui++] = a[qu[hu]];
    }
    for (int i = n; i < n + r; i++) {
        while (qu[hu] <= i - k) hu++;
        u[ui++] = a[qu[hu]];
        while (ql[hl] <= i - k) hl++;
        l[li++] = a[ql[hl]];
    }
    free(qu);
    free(ql);
}

/* src/lb_normalize.cpp:9-32 */
void orc_normalized(const double* U, const double* L, double* Un, double* Ln, int len,
                    const double* max_mean, const double* min_mean,
                    const double* max_std, const double* min_std) {
    for (int i = 0; i < len; i++) {
        const double nu = U[i] - min_mean[i];
        Un[i] = (nu >= 0) ? nu / min_std[i] : nu / max_std[i];
        const double nl = L[i] - max_mean[i];
        Ln[i] = (nl <= 0) ? nl / min_std[i] : nl / max_std[i];
    }
}

/* ------------------------------------------------------ threshold selection */

typedef struct { double value; int count; int pos; } orc_run;

/* src/find_t_lp.cpp:53-67: runs of consecutive equal values of env[m-1 .. m-1+n) */
static int unique_runs(const double* T, orc_run* out, int m, int n) {
    if (n <= 0) return 0;
    int j = 0;
    for (int i = 0; i < n; i++) {
        if (i == 0 || T[m - 1 + i] != T[m + i - 2]) {
            out[j].value = T[m - 1 + i];
            out[j].count = 1;
            out[j].pos = j;
            j++;
        } else {
            out[j - 1].count++;
        }
    }
    return j;
}

/* src/find_t_lp.cpp:68-81 with a total order: NaN last, ties by position */
static int cmp_run_asc(const void* pa, const void* pb) {
    const orc_run* a = (const orc_run*)pa;
    const orc_run* b = (const orc_run*)pb;
    const int na = isnan(a->value), nb = isnan(b->value);
    if (na != nb) return na ? 1 : -1;
    if (!na) {
        if (a->value < b->value) return -1;
        if (a->value > b->value) return 1;
    }
    return (a->pos > b->pos) - (a->pos < b->pos);
}
static int cmp_run_desc(const void* pa, const void* pb) {
    const orc_run* a = (const orc_run*)pa;
    const orc_run* b = (const orc_run*)pb;
    const int na = isnan(a->value), nb = isnan(b->value);
    if (na != nb) return na ? 1 : -1;
    if (!na) {
        if (a->value > b->value) return -1;
        if (a->value < b->value) return 1;
    }
    return (a->pos > b->pos) - (a->pos < b->pos);
}

static int metric_p(int metric) {  /* src/fsmeld.cpp:586-598 */
    return (metric == ORC_DTW || metric == ORC_ERP) ? 2 : (metric == ORC_MSM ? 1 : 0);
}

/* src/find_t_lp.cpp:148-159 */
static double fn_D(double q, double C, int metric) {
    if (metric == ORC_MSM) return C;
    if (metric == ORC_ERP) return (q - C) * (q - C);
    if (metric == ORC_EDR || metric == ORC_LCSS) return 1;
    if (metric == ORC_DTW) return (q - C) * (q - C);
    return 0.0;
}
/* src/find_t_lp.cpp:167-176 */
static double fn_tu(double q, double C, int metric) {
    if (metric == ORC_MSM) return q - C;
    if (metric == ORC_ERP) return q - fabs(q - C);
    if (metric == ORC_EDR || metric == ORC_LCSS) return q - C;
    return q;
}
/* src/find_t_lp.cpp:177-186 */
static double fn_tl(double q, double C, int metric) {
    if (metric == ORC_MSM) return q + C;
    if (metric == ORC_ERP) return q + fabs(q - C);
    if (metric == ORC_EDR || metric == ORC_LCSS) return q + C;
    return q;
}
/* src/find_t_lp.cpp:187-199 */
static double fn_fp(const double* mp, int p, int metric, double t) {
    if (p == 0) return (metric == ORC_LCSS || metric == ORC_EDR) ? 0 : mp[0];
    if (p == 1) return mp[1] - mp[0] * t;
    if (p == 2) return mp[2] - mp[1] * t * 2 + mp[0] * (t * t);
    return 0.0;
}
/* src/find_t_lp.cpp:206-216 */
static int first_max(const double* arr, int size) {
    if (size <= 0) return -1;
    int best = 0;
    for (int i = 0; i < size; ++i)
        if (arr[i] > arr[best]) best = i;
    return best;
}

static void mp_add(double* mp, int p, double v) {
    for (int a = 0; a < p + 1; a++) mp[a] += pow(v, a);
}
static void mp_sub(double* mp, int p, double v) {
    for (int a = 0; a < p + 1; a++) mp[a] -= pow(v, a);
}

/* Binary heap with the sift order of the C++ standard library's
 * push_heap/pop_heap (GNU libstdc++), which std::priority_queue uses in
 * src/find_t_lp.cpp:525-571,597-643.  Pop order among equal keys follows that
 * sift order, which the ERP threshold sweep depends on bit for bit. */
typedef struct { double value; int index; } orc_hitem;
static int h_less(const orc_hitem* a, const orc_hitem* b, int minheap) {
    return minheap ? (a->value > b->value) : (a->value < b->value);
}
static void h_push_hole(orc_hitem* h, long hole, long top, orc_hitem v, int mh) {
    long parent = (hole - 1) / 2;
    while (hole > top && h_less(&h[parent], &v, mh)) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = v;
}
static void h_push(orc_hitem* h, long* len, orc_hitem v, int mh) {
    h[*len] = v;
    (*len)++;
    h_push_hole(h, *len - 1, 0, v, mh);
}
static void h_pop(orc_hitem* h, long* len, int mh) {
    if (*len > 1) {
        const long n = *len - 1;
        const orc_hitem v = h[n];
        h[n] = h[0];
        long hole = 0, second = 0;
        while (second < (n - 1) / 2) {
            second = 2 * (second + 1);
            if (h_less(&h[second], &h[second - 1], mh)) second--;
            h[hole] = h[second];
            hole = second;
        }
        if ((n & 1) == 0 && second == (n - 2) / 2) {
            second = 2 * (second + 1);
            h[hole] = h[second - 1];
            hole = second - 1;
        }
        h_push_hole(h, hole, 0, v, mh);
    }
    (*len)--;
}

/* src/find_t_lp.cpp:218-287 (lower, DTW) and 655-724 (upper, DTW) */
static double find_t_dtw(int upper, const orc_run* R, int nr, const double* qs, int m, int metric,
                         double* LB) {
    const int p = 2;
    double mp[3] = {0, 0, 0};
    long long g = 0;
    const double t0 = R[0].value;
    if (!upper) {
        int idx1 = m - 1;
        while (idx1 >= 0 && qs[idx1] >= t0) idx1--;
        for (int i = 0; i <= idx1; i++) mp_add(mp, p, qs[i]);
        for (int i = 0; i < nr; i++) {
            const double t = R[i].value;
            g += R[i].count;
            while (idx1 >= 0) {
                const double v = qs[idx1];
                if (v >= t) { mp_sub(mp, p, v); idx1--; } else break;
            }
            LB[i] = fabs(fn_fp(mp, p, metric, t)) * (int)g;
        }
    } else {
        int idx1 = 0;
        while (idx1 < m && qs[idx1] <= t0) idx1++;
        for (int i = idx1; i < m; i++) mp_add(mp, p, qs[i]);
        for (int i = 0; i < nr; i++) {
            const double t = R[i].value;
            g += R[i].count;
            while (idx1 < m) {
                const double v = qs[idx1];
                if (v < t) { mp_sub(mp, p, v); idx1++; } else break;
            }
            LB[i] = fn_fp(mp, p, metric, t) * (int)g;
        }
    }
    return R[first_max(LB, nr)].value;
}

/* src/find_t_lp.cpp:288-398 (lower) and 726-825 (upper): MSM, EDR, LCSS */
static double find_t_gen(int upper, const orc_run* R, int nr, const double* qs, int m, int metric,
                         double Cq, double* LB) {
    const int p = metric_p(metric);
    double mp[3] = {0, 0, 0};
    double C = 0;
    long long g = 0;
    const double t0 = R[0].value;
    if (!upper) {
        int idx1 = m - 1;
        while (idx1 >= 0 && qs[idx1] >= t0) idx1--;
        int idx2 = idx1;
        while (idx2 >= 0) {
            if (fn_tl(qs[idx2], Cq, metric) >= t0) { mp_add(mp, p, qs[idx2]); idx2--; } else break;
        }
        for (int j = 0; j <= idx2; j++) C += fn_D(qs[j], Cq, metric);
        for (int i = 0; i < nr; i++) {
            const double t = R[i].value;
            g += R[i].count;
            while (idx2 >= 0) {
                if (fn_tl(qs[idx2], Cq, metric) >= t) {
                    C = C - fn_D(qs[idx2], Cq, metric);
                    mp_add(mp, p, qs[idx2]);
                    idx2--;
                } else break;
            }
            while (idx1 > idx2) {
                const double v = qs[idx1];
                if (v > t) { mp_sub(mp, p, v); idx1--; } else break;
            }
            LB[i] = (C + fabs(fn_fp(mp, p, metric, t))) * (int)g;
        }
    } else {
        int idx1 = 0;
        while (idx1 < m && qs[idx1] <= t0) idx1++;
        int idx2 = idx1;
        while (idx2 < m) {
            if (fn_tu(qs[idx2], Cq, metric) <= t0) { mp_add(mp, p, qs[idx2]); idx2++; } else break;
        }
        for (int j = idx2; j < m; j++) C += fn_D(qs[j], Cq, metric);
        for (int i = 0; i < nr; i++) {
            const double t = R[i].value;
            g += R[i].count;
            while (idx2 < m) {
                if (fn_tu(qs[idx2], Cq, metric) <= t) {
                    C = C - fn_D(qs[idx2], Cq, metric);
                    mp_add(mp, p, qs[idx2]);
                    idx2++;
                } else break;
            }
            while (idx1 < idx2) {
                const double v = qs[idx1];
                if (v < t) { mp_sub(mp, p, v); idx1++; } else break;
            }
            LB[i] = (C + fn_fp(mp, p, metric, t)) * (int)g;
        }
    }
    return R[first_max(LB, nr)].value;
}

/* src/find_t_lp.cpp:510-582 (lower) and 583-654 (upper): ERP, heaps over the
 * unsorted query */
static double find_t_erp(int upper, const orc_run* R, int nr, const double* q, int m,
                         double Cq, double* LB) {
    const int p = 2;
    double mp[3] = {0, 0, 0};
    double C = 0;
    long long g = 0;
    const double t0 = R[0].value;
    orc_hitem* H1 = (orc_hitem*)malloc(sizeof(orc_hitem) * (2 * m + 1));
    orc_hitem* H2 = (orc_hitem*)malloc(sizeof(orc_hitem) * (m + 1));
    long n1 = 0, n2 = 0;
    const int mh = upper;  /* upper: HeapItem (min-heap); lower: maxHeapItem */
    for (int i = 0; i < m; i++) {
        const double tau = upper ? fn_tu(q[i], Cq, ORC_ERP) : fn_tl(q[i], Cq, ORC_ERP);
        const int ignore = upper ? (q[i] <= t0) : (q[i] >= t0);
        const int heap1 = upper ? (tau <= t0) : (tau >= t0);
        if (ignore) {
        } else if (heap1) {
            orc_hitem it = {q[i], i};
            h_push(H1, &n1, it, mh);
            mp_add(mp, p, q[i]);
        } else {
            orc_hitem it = {tau, i};
            h_push(H2, &n2, it, mh);
            C += fn_D(q[i], Cq, ORC_ERP);
        }
    }
    for (int i = 0; i < nr; i++) {
        const double t = R[i].value;
        g += R[i].count;
        while (n2 > 0 && (upper ? (H2[0].value <= t) : (H2[0].value >= t))) {
            const int oi = H2[0].index;
            const double oq = q[oi];
            h_pop(H2, &n2, mh);
            C -= fn_D(oq, Cq, ORC_ERP);
            orc_hitem it = {oq, oi};
            h_push(H1, &n1, it, mh);
            mp_add(mp, p, oq);
        }
        while (n1 > 0 && (upper ? (H1[0].value <= t) : (H1[0].value >= t))) {
            const double oq = q[H1[0].index];
            h_pop(H1, &n1, mh);
            mp_sub(mp, p, oq);
        }
        const double f = fn_fp(mp, p, ORC_ERP, t);
        LB[i] = (C + (upper ? f : fabs(f))) * (int)g;
    }
    free(H1);
    free(H2);
    return R[first_max(LB, nr)].value;
}

static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* dispatch as src/fsmeld.cpp:778-790 */
double orc_find_t(int upper, int metric, const double* env, int l, const double* q,
                  const double* q_sorted, int m, double arg) {
    const int n = l - 2 * m + 2;
    orc_run* R = (orc_run*)malloc(sizeof(orc_run) * (n > 0 ? n : 1));
    double* LB = (double*)calloc(n > 0 ? n : 1, sizeof(double));
    double* own = NULL;
    if (!q_sorted) {
        own = (double*)malloc(sizeof(double) * m);
        memcpy(own, q, sizeof(double) * m);
        qsort(own, m, sizeof(double), cmp_double);
        q_sorted = own;
    }
    const int nr = unique_runs(env, R, m, n);
    qsort(R, nr, sizeof(orc_run), upper ? cmp_run_asc : cmp_run_desc);
    double t;
    if (metric == ORC_DTW) t = find_t_dtw(upper, R, nr, q_sorted, m, metric, LB);
    else if (metric == ORC_ERP) t = find_t_erp(upper, R, nr, q, m, arg, LB);
    else t = find_t_gen(upper, R, nr, q_sorted, m, metric, arg, LB);
    free(R);
    free(LB);
    free(own);
    return t;
}

/* ------------------------------------------------- penalties, masks, SIP */

/* src/q_to_h.cpp:11-64 (lower) and 84-134 (upper) */
void orc_q_to_h(int upper, int metric, const double* q, int m, double t, double C, double* h) {
    for (int i = 0; i < m; i++) {
        const double x = q[i];
        double v = 0.0;
        if (!upper) {
            if (metric == ORC_MSM) v = (x < t) ? ORC_MIN(C, t - x) : 0.0;
            else if (metric == ORC_DTW) v = (x < t) ? (t - x) * (t - x) : 0.0;
            else if (metric == ORC_ERP)
                v = (x < t) ? (((x - t) * (x - t) > (x - C) * (x - C)) ? (x - C) * (x - C)
                                                                       : (x - t) * (x - t))
                            : 0.0;
            else v = (x < t - C) ? 1 : 0.0;
        } else {
            if (metric == ORC_MSM) v = (x > t) ? ORC_MIN(C, x - t) : 0.0;
            else if (metric == ORC_DTW) v = (x > t) ? (x - t) * (x - t) : 0.0;
            else if (metric == ORC_ERP)
                v = (x > t) ? (((x - t) * (x - t) > (x - C) * (x - C)) ? (x - C) * (x - C)
                                                                       : (x - t) * (x - t))
                            : 0.0;
            else v = (x > t + C) ? 1 : 0.0;
        }
        h[i] = v;
    }
}

/* src/lb.cpp:18-34 */
void orc_s_to_g(int upper, const double* env, int n, double t, double* g) {
    for (int i = 0; i < n; i++) g[i] = upper ? ((env[i] <= t) ? 1.0 : 0.0) : ((env[i] >= t) ? 1.0 : 0.0);
}

typedef struct {
    int n;
    double* Z;
    fftw_complex *XX, *YY, *ZZ;
    fftw_plan r2c, c2r;
    double* ytmp;
} orc_fft;

static void fft_init(orc_fft* f, int n) {
    f->n = n;
    f->Z = fftw_alloc_real(n);
    f->XX = fftw_alloc_complex(n / 2 + 1);
    f->YY = fftw_alloc_complex(n / 2 + 1);
    f->ZZ = fftw_alloc_complex(n / 2 + 1);
    f->r2c = fftw_plan_dft_r2c_1d(n, f->Z, f->ZZ, FFTW_ESTIMATE);
    f->c2r = fftw_plan_dft_c2r_1d(n, f->ZZ, f->Z, FFTW_ESTIMATE);
    f->ytmp = (double*)malloc(sizeof(double) * n);
}
static void fft_free(orc_fft* f) {
    fftw_destroy_plan(f->r2c);
    fftw_destroy_plan(f->c2r);
    fftw_free(f->XX); fftw_free(f->YY); fftw_free(f->ZZ); fftw_free(f->Z);
    free(f->ytmp);
}

/* src/sip.cpp:16-52, sequenced as src/fsmeld.cpp:798-806 */
static void sip_with(orc_fft* f, int m, const double* h, const double* g, double* z) {
    const int n = f->n;
    for (int i = 0; i < n; i++) f->ytmp[i] = (i < m) ? h[m - i - 1] : 0;
    fftw_execute_dft_r2c(f->r2c, f->ytmp, f->YY);
    fftw_execute_dft_r2c(f->r2c, (double*)g, f->XX);
    const double inv_n = 1.0 / n;
    for (int i = 0; i <= n / 2; i++) {
        f->ZZ[i][0] = (f->XX[i][0] * f->YY[i][0] - f->XX[i][1] * f->YY[i][1]) * inv_n;
        f->ZZ[i][1] = (f->XX[i][1] * f->YY[i][0] + f->XX[i][0] * f->YY[i][1]) * inv_n;
    }
    fftw_execute_dft_c2r(f->c2r, f->ZZ, z);
}

void orc_sip(int n, int m, const double* h, const double* g, double* z) {
    orc_fft f;
    fft_init(&f, n);
    sip_with(&f, m, h, g, z);
    fft_free(&f);
}

/* src/fsmeld.cpp:84-106 (and the tail variant at 912-921) */
double orc_trans_one(double zl, double zu, int m, int metric) {
    if (metric == ORC_ERP || metric == ORC_DTW) return sqrt(dmax0(zl + zu));
    if (metric == ORC_LCSS) return dmax0((zl + zu) / m);
    return zl + zu;
}

/* include/fsmeld_internal.h:9-19 */
int orc_lbip_exceeds(double bound, double cutoff, int metric) {
    const double tol = 1e-9;
    if (!isfinite(bound) || !(bound > cutoff + tol)) return 0;
    if (metric == ORC_DTW || metric == ORC_ERP) {
        const double limit = cutoff + tol;
        return bound > sqrt(limit * limit + tol);
    }
    return 1;
}

/* ------------------------------------------------------------------- GLB */

#define GLB_DIST(x, y) (((x) - (y)) * ((x) - (y)))
static double edr_subcost(double a, double b, double eps) { return (fabs(a - b) <= eps) ? 0.0 : 1.0; }
static int env_match(double v, double lo, double hi, double eps) {
    if (v < lo) return lo - v <= eps;
    if (v > hi) return v - hi <= eps;
    return 1;
}
static double min3(double a, double b, double c) {  /* std::min({a,b,c}) */
    double r = a;
    if (b < r) r = b;
    if (c < r) r = c;
    return r;
}

/* src/glb.cpp:200-373 */
double orc_glb(int metric, const double* Q, const double* T, int m, double arg,
               const double* LQ, const double* UQ, int w, double bsf) {
    const int lenQ = m, lenT = m;
    if (lenQ < 2 || lenT < 2) return 0.0;
    double boundary = 0.0, t_to_q = 0.0, lcss_t = 0.0;
    const double sq = bsf * bsf;
    switch (metric) {
    case ORC_DTW:
        boundary = GLB_DIST(T[0], Q[0]) + GLB_DIST(T[lenT - 1], Q[lenQ - 1]);
        for (int i = 1; i < lenT - 1; ++i) {
            if (T[i] < LQ[i]) t_to_q += GLB_DIST(T[i], LQ[i]);
            else if (T[i] > UQ[i]) t_to_q += GLB_DIST(T[i], UQ[i]);
            if (boundary + t_to_q > sq) return ORC_GLB_MAX;
        }
        break;
    case ORC_ERP:
        boundary = min3(GLB_DIST(Q[lenQ - 1], T[lenT - 1]), GLB_DIST(Q[lenQ - 1], arg),
                        GLB_DIST(T[lenT - 1], arg));
        for (int i = 1; i < lenT - 1; ++i) {
            if (T[i] > UQ[i]) t_to_q += ORC_MIN(GLB_DIST(T[i], UQ[i]), GLB_DIST(T[i], arg));
            else if (T[i] < LQ[i]) t_to_q += ORC_MIN(GLB_DIST(T[i], LQ[i]), GLB_DIST(T[i], arg));
            if (boundary + t_to_q > sq) return ORC_GLB_MAX;
        }
        break;
    case ORC_EDR:
        boundary = ORC_MIN(edr_subcost(Q[lenQ - 1], T[lenT - 1], arg), 1.0);
        for (int i = 1; i < lenT - 1; ++i) {
            if (T[i] > UQ[i]) t_to_q += edr_subcost(T[i], UQ[i], arg);
            else if (T[i] < LQ[i]) t_to_q += edr_subcost(T[i], LQ[i], arg);
            if (boundary + t_to_q > bsf) return ORC_GLB_MAX;
        }
        break;
    case ORC_LCSS: {
        const double min_len = ORC_MIN(lenQ, lenT);
        for (int i = 0; i < lenT; ++i)
            if (env_match(T[i], LQ[i], UQ[i], arg)) lcss_t += 1.0;
        if (dmax0(1.0 - lcss_t / min_len) > bsf) return ORC_GLB_MAX;
        break;
    }
    case ORC_MSM:
        if ((T[lenT - 2] >= T[lenT - 1] && T[lenT - 1] >= Q[lenQ - 1]) ||
            (T[lenT - 2] <= T[lenT - 1] && T[lenT - 1] <= Q[lenQ - 1]) ||
            (Q[lenQ - 2] <= Q[lenQ - 1] && Q[lenQ - 1] <= T[lenT - 1]) ||
            (Q[lenQ - 2] >= Q[lenQ - 1] && Q[lenQ - 1] >= T[lenT - 1])) {
            boundary = fabs(Q[0] - T[0]) + ORC_MIN(fabs(Q[lenQ - 1] - T[lenT - 1]), arg);
        } else {
            boundary = fabs(Q[0] - T[0]) + min3(fabs(Q[lenQ - 1] - T[lenT - 1]),
                                                arg + fabs(T[lenT - 1] - T[lenT - 2]),
                                                arg + fabs(Q[lenQ - 1] - Q[lenQ - 2]));
        }
        for (int i = 1; i < lenT - 1; ++i) {
            if (T[i] > UQ[i]) t_to_q += ORC_MIN(fabs(T[i] - UQ[i]), arg);
            else if (T[i] < LQ[i]) t_to_q += ORC_MIN(fabs(T[i] - LQ[i]), arg);
            if (boundary + t_to_q > bsf) return ORC_GLB_MAX;
        }
        break;
    default:
        return ORC_GLB_MAX;
    }

    double* LT = (double*)malloc(sizeof(double) * lenT);
    double* UT = (double*)malloc(sizeof(double) * lenT);
    orc_lemire(T, lenT, w, LT, UT);
    double res = ORC_GLB_MAX, q_to_t = 0.0;
    switch (metric) {
    case ORC_DTW:
        for (int i = 1; i < lenQ - 1; ++i) {
            if (Q[i] < LT[i]) q_to_t += GLB_DIST(Q[i], LT[i]);
            else if (Q[i] > UT[i]) q_to_t += GLB_DIST(Q[i], UT[i]);
            if (boundary + q_to_t > sq) goto done;
        }
        res = sqrt(dmax0(boundary + ORC_MAX(t_to_q, q_to_t)));
        break;
    case ORC_ERP:
        for (int i = 1; i < lenQ - 1; ++i) {
            if (Q[i] > UT[i]) q_to_t += ORC_MIN(GLB_DIST(Q[i], UT[i]), GLB_DIST(Q[i], arg));
            else if (Q[i] < LT[i]) q_to_t += ORC_MIN(GLB_DIST(Q[i], LT[i]), GLB_DIST(Q[i], arg));
            if (boundary + q_to_t > sq) goto done;
        }
        res = sqrt(dmax0(boundary + ORC_MAX(t_to_q, q_to_t)));
        break;
    case ORC_EDR:
        for (int i = 1; i < lenQ - 1; ++i) {
            if (Q[i] > UT[i]) q_to_t += edr_subcost(Q[i], UT[i], arg);
            else if (Q[i] < LT[i]) q_to_t += edr_subcost(Q[i], LT[i], arg);
            if (boundary + q_to_t > bsf) goto done;
        }
        res = boundary + ORC_MAX(t_to_q, q_to_t);
        break;
    case ORC_LCSS: {
        double qr = 0.0;
        for (int i = 0; i < lenQ; ++i)
            if (env_match(Q[i], LT[i], UT[i], arg)) qr += 1.0;
        const double min_len = ORC_MIN(lenQ, lenT);
        res = dmax0(1.0 - ORC_MIN(lcss_t, qr) / min_len);
        break;
    }
    case ORC_MSM:
        for (int i = 1; i < lenQ - 1; ++i) {
            if (Q[i] > UT[i]) q_to_t += ORC_MIN(fabs(Q[i] - UT[i]), arg);
            else if (Q[i] < LT[i]) q_to_t += ORC_MIN(fabs(Q[i] - LT[i]), arg);
            if (boundary + q_to_t > bsf) goto done;
        }
        res = boundary + ORC_MAX(t_to_q, q_to_t);
        break;
    }
done:
    free(LT);
    free(UT);
    return res;
}

/* ------------------------------------------------------ exact distances */

static double* dp_buf(size_t need) {
    static double* buf = NULL;
    static size_t cap = 0;
    if (cap < need) {
        free(buf);
        buf = (double*)malloc(sizeof(double) * need);
        cap = need;
    }
    return buf;
}

/* src/ElasticMeasures.cpp:24-61 */
static double dp_dtw(const double* A, int m, const double* B, int n, int r) {
    const int row = 2 * r + 1;
    double* base = dp_buf((size_t)2 * row);
    double* cost = base;
    double* prev = base + row;
    for (int i = 0; i < row; i++) { cost[i] = ORC_DP_MAX; prev[i] = ORC_DP_MAX; }
    for (int i = 0; i < m; i++) {
        int k = ORC_MAX(0, r - i);
        const int jlo = ORC_MAX(0, i - r), jhi = ORC_MIN(n - 1, i + r);
        for (int j = jlo; j <= jhi; j++, k++) {
            if (i == 0 && j == 0) { cost[k] = (A[0] - B[0]) * (A[0] - B[0]); continue; }
            const double y = (j - 1 < 0 || k - 1 < 0) ? ORC_DP_MAX : cost[k - 1];
            const double x = (i - 1 < 0 || k + 1 > 2 * r) ? ORC_DP_MAX : prev[k + 1];
            const double z = (i - 1 < 0 || j - 1 < 0) ? ORC_DP_MAX : prev[k];
            cost[k] = min3(x, y, z) + (A[i] - B[j]) * (A[i] - B[j]);
        }
        double* tmp = cost; cost = prev; prev = tmp;
    }
    const double fin = prev[r + (n - 1) - (m - 1)];
    if (!isfinite(fin)) return ORC_DP_MAX;
    return sqrt(dmax0(fin));
}

/* src/ElasticMeasures.cpp:63-93 */
static double dp_lcss(const double* Q, int n, const double* A, int m, int w, double eps) {
    double* arr = dp_buf((size_t)n * m);
    for (int i = 0; i < n * m; i++) arr[i] = 0.0;
    for (int i = 0; i < n; ++i) {
        const int wmin = ORC_MAX(0, i - w), wmax = ORC_MIN(m, i + w + 1);
        for (int j = wmin; j < wmax; ++j) {
            const int idx = i * m + j;
            const int hit = fabs(Q[i] - A[j]) <= eps;
            if (i + j == 0) {
                if (hit) arr[idx] = 1;
            } else if (i == 0) {
                if (hit) arr[idx] = 1;
                else arr[idx] = (j > wmin) ? arr[i * m + (j - 1)] : 0;
            } else if (j == 0) {
                if (hit) arr[idx] = 1;
                else arr[idx] = arr[(i - 1) * m + j];
            } else {
                const double v1 = arr[(i - 1) * m + (j - 1)];
                const double v2 = arr[(i - 1) * m + j];
                const double v3 = (j > wmin) ? arr[idx - 1] : 0;
                double best = hit ? v1 + 1 : v1;  /* std::max({a,b,c}) */
                if (best < v2) best = v2;
                if (best < v3) best = v3;
                arr[idx] = best;
            }
        }
    }
    const double result = arr[(n - 1) * m + (m - 1)];
    return 1 - result / ORC_MIN(n, m);
}

/* src/ElasticMeasures.cpp:95-130 */
static double dp_erp(const double* x, int lenx, const double* y, int leny, double g, int w) {
    const size_t row = (size_t)leny + 1;
    double* base = dp_buf(2 * row);
    double* cur = base;
    double* prev = base + row;
    for (size_t j = 0; j < row; j++) prev[j] = ORC_DP_MAX;
    prev[0] = 0.0;
    for (int j = 1; j <= ORC_MIN(leny, w); ++j) prev[j] = prev[j - 1] + (y[j - 1] - g) * (y[j - 1] - g);
    for (int i = 1; i <= lenx; ++i) {
        for (size_t j = 0; j < row; j++) cur[j] = ORC_DP_MAX;
        if (i <= w) cur[0] = prev[0] + (x[i - 1] - g) * (x[i - 1] - g);
        const int lo = ORC_MAX(1, i - w), hi = ORC_MIN(leny, i + w);
        for (int j = lo; j <= hi; ++j) {
            const double match = prev[j - 1] + (x[i - 1] - y[j - 1]) * (x[i - 1] - y[j - 1]);
            const double ins = cur[j - 1] + (y[j - 1] - g) * (y[j - 1] - g);
            const double del = prev[j] + (x[i - 1] - g) * (x[i - 1] - g);
            cur[j] = min3(match, ins, del);
        }
        double* tmp = cur; cur = prev; prev = tmp;
    }
    const double res = prev[leny];
    if (!isfinite(res)) return ORC_DP_MAX;
    return sqrt(dmax0(res));
}

/* src/ElasticMeasures.cpp:132-165 */
static double dp_edr(const double* x, int n, const double* y, int msz, double eps, int w) {
    const size_t row = (size_t)msz + 1;
    double* base = dp_buf(2 * row);
    double* cur = base;
    double* prev = base + row;
    for (size_t j = 0; j < row; j++) prev[j] = ORC_DP_MAX;
    prev[0] = 0.0;
    for (int j = 1; j <= ORC_MIN(msz, w); ++j) prev[j] = (double)j;
    for (int i = 1; i <= n; ++i) {
        for (size_t j = 0; j < row; j++) cur[j] = ORC_DP_MAX;
        if (i <= w) cur[0] = (double)i;
        const int lo = ORC_MAX(1, i - w), hi = ORC_MIN(msz, i + w);
        for (int j = lo; j <= hi; ++j) {
            const double sub = (fabs(x[i - 1] - y[j - 1]) <= eps) ? 0.0 : 1.0;
            cur[j] = min3(prev[j] + 1.0, cur[j - 1] + 1.0, prev[j - 1] + sub);
        }
        double* tmp = cur; cur = prev; prev = tmp;
    }
    return prev[msz];
}

/* src/ElasticMeasures.cpp:173-176 */
static double msm_c(double np, double x, double y, double c) {
    if ((x <= np && np <= y) || (y <= np && np <= x)) return c;
    return c + ORC_MIN(fabs(np - x), fabs(np - y));
}

/* src/ElasticMeasures.cpp:167-198 */
static double dp_msm(const double* x, int xl, const double* y, int yl, double c, int w) {
    double* cost = dp_buf((size_t)xl * yl);
    for (int i = 0; i < xl * yl; i++) cost[i] = ORC_DP_MAX;
    cost[0] = fabs(x[0] - y[0]);
    for (int i = 1; i < xl && i <= w; ++i)
        cost[i * yl] = cost[(i - 1) * yl] + msm_c(x[i], x[i - 1], y[0], c);
    for (int j = 1; j < yl && j <= w; ++j)
        cost[j] = cost[j - 1] + msm_c(y[j], x[0], y[j - 1], c);
    for (int i = 1; i < xl; ++i) {
        const int js = ORC_MAX(1, i - w), je = ORC_MIN(yl, i + w + 1);
        for (int j = js; j < je; ++j) {
            const double c1 = cost[(i - 1) * yl + (j - 1)] + fabs(x[i] - y[j]);
            const double c2 = cost[(i - 1) * yl + j] + msm_c(x[i], x[i - 1], y[j], c);
            const double c3 = cost[i * yl + (j - 1)] + msm_c(y[j], x[i], y[j - 1], c);
            cost[i * yl + j] = min3(c1, c2, c3);
        }
    }
    return cost[xl * yl - 1];
}

/* src/fsmeld.cpp:170-183 */
double orc_distance(int metric, const double* q, const double* t, int m, int w, double arg) {
    switch (metric) {
    case ORC_MSM: return dp_msm(q, m, t, m, arg, w);
    case ORC_ERP: return dp_erp(q, m, t, m, arg, w);
    case ORC_LCSS: return dp_lcss(q, m, t, m, w, arg);
    case ORC_EDR: return dp_edr(q, m, t, m, arg, w);
    case ORC_DTW: return dp_dtw(q, m, t, m, w);
    default: return NAN;
    }
}

/* --------------------------------------------------------------- drivers */

/* Normalisation mode (include/funcs.h:20-28, src/normalization_mode.cpp):
 * 0 z-score, the reference command line's only mode; 1 raw.  The reference
 * declares the raw mode but never consults it, so its raw behaviour is this
 * restatement's own definition (parity unpinned): the query is used as
 * given, a window is valid iff its points are all finite, and its
 * statistics are mean 0 and sigma 1, so (t - 0) / 1 leaves candidates and
 * envelopes as they are and the cascade runs unchanged on raw values. */
static int g_orc_raw = 0;
void orc_set_normalization(int raw) { g_orc_raw = raw != 0; }

/* src/fsmeld.cpp:622-639 */
void orc_normalize_query(const double* q, int m, double* qn) {
    if (g_orc_raw) {
        memcpy(qn, q, sizeof(double) * (size_t)m);
        return;
    }
    double ex = 0, ex2 = 0;
    for (int i = 0; i < m; i++) { ex += q[i]; ex2 += q[i] * q[i]; }
    const double mean = ex / m;
    double sd = ex2 / m;
    sd = sqrt(sd - mean * mean);
    for (int i = 0; i < m; i++) qn[i] = (q[i] - mean) / sd;
}

typedef struct {
    int m, m_k, w, metric;
    double arg;
    long long excl_b, excl_e;
    double *qn, *qs, *LQ, *UQ;
    double *miu, *si, *mumin, *mumax, *simin, *simax, *U, *L, *Un, *Ln;
    double *hl, *hu, *gl, *gu, *zl, *zu, *z, *ttmp;
    uint8_t* invalid;
    orc_fft fft;
} orc_seg;

static int seg_init(orc_seg* s, const double* query, int m, int m_k, int w, int metric,
                    double arg, long long eb, long long ee, int with_lb) {
    memset(s, 0, sizeof(*s));
    s->m = m; s->m_k = m_k; s->w = w; s->metric = metric; s->arg = arg;
    s->excl_b = eb; s->excl_e = ee;
    s->qn = (double*)malloc(sizeof(double) * m);
    s->qs = (double*)malloc(sizeof(double) * m);
    s->LQ = (double*)malloc(sizeof(double) * m);
    s->UQ = (double*)malloc(sizeof(double) * m);
    orc_normalize_query(query, m, s->qn);
    memcpy(s->qs, s->qn, sizeof(double) * m);
    qsort(s->qs, m, sizeof(double), cmp_double);
    orc_lemire(s->qn, m, w, s->LQ, s->UQ);
    double** bufs[] = {&s->miu, &s->si, &s->mumin, &s->mumax, &s->simin, &s->simax, &s->U, &s->L,
                       &s->Un, &s->Ln, &s->gl, &s->gu, &s->zl, &s->zu, &s->z};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        *bufs[i] = (double*)calloc(m_k, sizeof(double));
    s->hl = (double*)calloc(m, sizeof(double));
    s->hu = (double*)calloc(m, sizeof(double));
    s->ttmp = (double*)calloc(m, sizeof(double));
    s->invalid = (uint8_t*)calloc(m_k, 1);
    if (with_lb) fft_init(&s->fft, m_k);
    else s->fft.n = 0;
    return 0;
}

static void seg_free(orc_seg* s) {
    free(s->qn); free(s->qs); free(s->LQ); free(s->UQ);
    double* bufs[] = {s->miu, s->si, s->mumin, s->mumax, s->simin, s->simax, s->U, s->L,
                      s->Un, s->Ln, s->gl, s->gu, s->zl, s->zu, s->z, s->hl, s->hu, s->ttmp};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++) free(bufs[i]);
    free(s->invalid);
    if (s->fft.n) fft_free(&s->fft);
}

/* Statistics + invalid mask for one macro segment t[0..m_k) whose windows
 * [first, first+count) are processed with global indices gstart + (j-first):
 * src/fsmeld.cpp:753-755 / 861-864 and the exclusion at 131-152. */
static void seg_stats(orc_seg* s, const double* t, int first, int count, long long gstart) {
    orc_mvmean(t, s->m_k, s->m, s->miu, s->si);
    if (g_orc_raw) {  /* raw mode: (0, 1) for windows of finite points, NaN otherwise */
        int bad = 0;
        for (int k = 0; k < s->m; k++) bad += !isfinite(t[k]);
        for (int j = 0; j + s->m <= s->m_k; j++) {
            if (j > 0) bad += !isfinite(t[j + s->m - 1]) - !isfinite(t[j - 1]);
            s->miu[j] = bad ? NAN : 0.0;
            s->si[j] = bad ? NAN : 1.0;
        }
    }
    memset(s->invalid, 0, s->m_k);
    orc_invalid_mask(t, s->si, s->m_k, s->m, s->invalid);
    if (s->excl_b >= 0 && s->excl_e > s->excl_b) {
        for (int j = first; j < first + count; j++) {
            const long long gi = gstart + (j - first);
            if (gi >= s->excl_b && gi < s->excl_e) s->invalid[j] = 1;
        }
    }
}

/* LB_IP for every window of the segment: src/fsmeld.cpp:756-808 */
static void seg_lbip(orc_seg* s, const double* t) {
    const int m = s->m, mk = s->m_k, metric = s->metric;
    const int kml = mk - m + 1;
    orc_min_max_window(s->miu, mk, m, s->mumin, s->mumax);
    orc_min_max_window(s->si, mk, m, s->simin, s->simax);
    orc_lemire(t, mk, s->w, s->L, s->U);
    orc_normalized(s->U, s->L, s->Un, s->Ln, mk, s->mumax, s->mumin, s->simax, s->simin);
    const double tu = orc_find_t(1, metric, s->Un, mk, s->qn, s->qs, m, s->arg);
    const double tl = orc_find_t(0, metric, s->Ln, mk, s->qn, s->qs, m, s->arg);
    orc_q_to_h(0, metric, s->qn, m, tl, s->arg, s->hl);
    orc_q_to_h(1, metric, s->qn, m, tu, s->arg, s->hu);
    orc_s_to_g(0, s->Ln, mk, tl, s->gl);
    orc_s_to_g(1, s->Un, mk, tu, s->gu);
    sip_with(&s->fft, m, s->hl, s->gl, s->zl);
    sip_with(&s->fft, m, s->hu, s->gu, s->zu);
    for (int j = 0; j < kml; j++) s->z[j] = orc_trans_one(s->zl[m - 1 + j], s->zu[m - 1 + j], m, metric);
}

static void seg_candidate(orc_seg* s, const double* t, int j) {
    for (int k = 0; k < s->m; k++) s->ttmp[k] = (t[k + j] - s->miu[j]) / s->si[j];
}

typedef struct { long long idx; double* vals; } orc_surv;

/* src/fsmeld.cpp:570-1074 (search) */
long long orc_search(const double* target, long long n, const double* query, int m,
                     double cutoff, int metric, int w, double arg,
                     long long eb, long long ee, long long* out_idx, long long cap,
                     orc_counters* cnt, long long* seg_counts) {
    const int mk = orc_macro_length(m, n);
    if (mk < 0) return -1;
    orc_seg s;
    seg_init(&s, query, m, mk, w, metric, arg, eb, ee, 1);
    const long long kml = mk - m + 1, tsn = n - m + 1;
    const long long forsize = tsn / kml, tail = tsn % kml;
    const int tfirst = (int)(kml - tail), tend = tfirst + (int)tail;
    long long kk1 = 0, kk2 = 0, kk3 = 0, invalid = 0, nmatch = 0;
    orc_surv* sv = (orc_surv*)malloc(sizeof(orc_surv) * (size_t)kml);
    for (long long seg = 0; seg <= forsize; seg++) {
        const int is_tail = (seg == forsize);
        if (is_tail && tail == 0) break;
        const double* t = is_tail ? target + (n - mk) : target + seg * kml;
        const int first = is_tail ? tfirst : 0;
        const int end = is_tail ? tend : (int)kml;
        const long long gstart = seg * kml;
        seg_stats(&s, t, first, end - first, gstart);
        seg_lbip(&s, t);
        long long a1 = 0, a2 = 0, a3 = 0;
        int ns = 0;
        for (int j = first; j < end; j++) {
            if (s.invalid[j]) { invalid++; continue; }
            a1++;
            if (!orc_lbip_exceeds(s.z[j], cutoff, metric)) {
                a2++;
                seg_candidate(&s, t, j);
                const double glb = orc_glb(metric, s.qn, s.ttmp, m, arg, s.LQ, s.UQ, w, cutoff);
                if (glb <= cutoff) {
                    a3++;
                    sv[ns].idx = gstart + (j - first);
                    sv[ns].vals = (double*)malloc(sizeof(double) * m);
                    memcpy(sv[ns].vals, s.ttmp, sizeof(double) * m);
                    ns++;
                }
            }
        }
        for (int i = 0; i < ns; i++) {
            const double d = orc_distance(metric, s.qn, sv[i].vals, m, w, arg);
            if (isfinite(d) && d <= cutoff) {
                if (nmatch < cap) out_idx[nmatch] = sv[i].idx;
                nmatch++;
            }
            free(sv[i].vals);
        }
        if (seg_counts && !is_tail) {
            seg_counts[3 * seg] = a1; seg_counts[3 * seg + 1] = a2; seg_counts[3 * seg + 2] = a3;
        }
        kk1 += a1; kk2 += a2; kk3 += a3;
    }
    free(sv);
    if (cnt) {
        memset(cnt, 0, sizeof(*cnt));
        cnt->valid = kk1; cnt->invalid = invalid; cnt->after_lb = kk2; cnt->after_glb = kk3;
        cnt->exact_evals = kk3; cnt->matches = nmatch; cnt->threshold = cutoff;
        cnt->m_k = mk; cnt->segments = forsize; cnt->tail = tail;
    }
    seg_free(&s);
    return nmatch;
}

/* src/fsmeld.cpp:1075-1344 (exact, with exact_top_k = 0 as the CLI passes) */
long long orc_exact(const double* target, long long n, const double* query, int m,
                    double cutoff, int metric, int w, double arg,
                    long long eb, long long ee, long long* out_idx, double* out_dist,
                    long long cap, orc_counters* cnt) {
    const int mk = orc_macro_length(m, n);
    if (mk < 0) return -1;
    orc_seg s;
    seg_init(&s, query, m, mk, w, metric, arg, eb, ee, 0);
    const long long kml = mk - m + 1, tsn = n - m + 1;
    const long long forsize = tsn / kml, tail = tsn % kml;
    const int tfirst = (int)(kml - tail), tend = tfirst + (int)tail;
    long long kk1 = 0, invalid = 0, nmatch = 0;
    for (long long seg = 0; seg <= forsize; seg++) {
        const int is_tail = (seg == forsize);
        if (is_tail && tail == 0) break;
        const double* t = is_tail ? target + (n - mk) : target + seg * kml;
        const int first = is_tail ? tfirst : 0;
        const int end = is_tail ? tend : (int)kml;
        const long long gstart = seg * kml;
        seg_stats(&s, t, first, end - first, gstart);
        for (int j = first; j < end; j++) {
            if (s.invalid[j]) { invalid++; continue; }
            kk1++;
            seg_candidate(&s, t, j);
            const double d = orc_distance(metric, s.qn, s.ttmp, m, w, arg);
            if (!isfinite(d)) continue;
            if (d <= cutoff) {
                if (nmatch < cap) {
                    out_idx[nmatch] = gstart + (j - first);
                    if (out_dist) out_dist[nmatch] = d;
                }
                nmatch++;
            }
        }
    }
    if (cnt) {
        memset(cnt, 0, sizeof(*cnt));
        cnt->valid = kk1; cnt->invalid = invalid; cnt->after_lb = kk1; cnt->after_glb = kk1;
        cnt->exact_evals = kk1; cnt->matches = nmatch; cnt->threshold = cutoff;
        cnt->m_k = mk; cnt->segments = forsize; cnt->tail = tail;
    }
    seg_free(&s);
    return nmatch;
}

/* max-heap of (distance, index) pairs ordered lexicographically, as
 * std::priority_queue<pair<double,long long>> in src/fsmeld.cpp:190 */
typedef struct { double d; long long i; } orc_pair;
static int pair_less(orc_pair a, orc_pair b) { return a.d < b.d || (!(b.d < a.d) && a.i < b.i); }
static void pq_push(orc_pair* h, int* n, orc_pair v) {
    int k = (*n)++;
    while (k > 0) {
        const int p = (k - 1) / 2;
        if (!pair_less(h[p], v)) break;
        h[k] = h[p];
        k = p;
    }
    h[k] = v;
}
static orc_pair pq_pop(orc_pair* h, int* n) {
    const orc_pair top = h[0];
    const orc_pair v = h[--(*n)];
    int k = 0;
    for (;;) {
        int c = 2 * k + 1;
        if (c >= *n) break;
        if (c + 1 < *n && pair_less(h[c], h[c + 1])) c++;
        if (!pair_less(v, h[c])) break;
        h[k] = h[c];
        k = c;
    }
    if (*n > 0) h[k] = v;
    return top;
}

/* src/fsmeld.cpp:185-569 (cutoff, filter_by_initial_epsilon = false) */
long long orc_cutoff(const double* target, long long n, const double* query, int m,
                     int k, int metric, int w, double arg, long long eb, long long ee,
                     long long* out_idx, double* out_dist, orc_counters* cnt) {
    const int mk = orc_macro_length(m, n);
    if (mk < 0 || k < 1) return -1;
    orc_seg s;
    seg_init(&s, query, m, mk, w, metric, arg, eb, ee, 1);
    const long long kml = mk - m + 1, tsn = n - m + 1;
    const long long forsize = tsn / kml, tail = tsn % kml;
    const int tfirst = (int)(kml - tail), tend = tfirst + (int)tail;
    long long kk1 = 0, exact = 0, lbp = 0, glbp = 0;
    double threshold = DBL_MAX;
    orc_pair* heap = (orc_pair*)malloc(sizeof(orc_pair) * (size_t)(k + 1));
    int hn = 0;
    for (long long seg = 0; seg <= forsize; seg++) {
        const int is_tail = (seg == forsize);
        if (is_tail && tail == 0) break;
        const double* t = is_tail ? target + (n - mk) : target + seg * kml;
        const int first = is_tail ? tfirst : 0;
        const int end = is_tail ? tend : (int)kml;
        const long long gstart = seg * kml;
        seg_stats(&s, t, first, end - first, gstart);
        seg_lbip(&s, t);
        for (int j = first; j < end; j++) {
            if (s.invalid[j]) continue;
            kk1++;
            const int full = hn >= k;
            const double active = full ? threshold : DBL_MAX;
            if (orc_lbip_exceeds(s.z[j], active, metric)) { lbp++; continue; }
            seg_candidate(&s, t, j);
            if (full) {
                const double glb = orc_glb(metric, s.qn, s.ttmp, m, arg, s.LQ, s.UQ, w, threshold);
                if (glb > threshold) { glbp++; continue; }
            }
            const double d = orc_distance(metric, s.qn, s.ttmp, m, w, arg);
            exact++;
            if (!isfinite(d)) continue;
            const orc_pair pr = {d, gstart + (j - first)};
            if (hn < k) {
                pq_push(heap, &hn, pr);
                if (hn == k) threshold = heap[0].d;
            } else if (d < heap[0].d) {
                pq_pop(heap, &hn);
                pq_push(heap, &hn, pr);
                threshold = heap[0].d;
            }
        }
    }
    long long res = hn;
    if (hn < k) {
        res = -2;  /* fewer valid, non-excluded candidates than k (src/fsmeld.cpp:519-520) */
    } else {
        for (int i = hn - 1; i >= 0; i--) {
            const orc_pair p = pq_pop(heap, &hn);
            out_idx[i] = p.i;
            if (out_dist) out_dist[i] = p.d;
        }
    }
    if (cnt) {
        memset(cnt, 0, sizeof(*cnt));
        cnt->valid = kk1; cnt->after_lb = kk1 - lbp; cnt->after_glb = kk1 - lbp - glbp;
        cnt->exact_evals = exact; cnt->matches = res > 0 ? res : 0; cnt->threshold = threshold;
        cnt->m_k = mk; cnt->segments = forsize; cnt->tail = tail;
    }
    free(heap);
    seg_free(&s);
    return res;
}
