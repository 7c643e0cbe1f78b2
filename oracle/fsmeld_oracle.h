/*
 * fsmeld_oracle.h -- CPU restatement of the FSMELD hot path (test
 * infrastructure only: the checker for the CUDA path and the "port" CPU
 * baseline; never linked into the product).
 *
 * Every function restates one reference function in plain C, with the
 * reference's operation order (no fused multiply-adds; build with
 * -ffp-contract=off) so its bits can be pinned against the reference built
 * from its own sources (oracle/_ref).  Citations are file:line in the
 * reference tree.
 *
 * Metric ids are the reference's MetricType values (include/funcs.h:10-18).
 */
#ifndef FSMELD_ORACLE_H
#define FSMELD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_DTW = 1, ORC_EDR = 2, ORC_ERP = 3, ORC_LCSS = 4, ORC_MSM = 5 };

/* src/fsmeld.cpp:28-37; returns the macro-segment length or -1 if too short */
int orc_macro_length(int m, long long available_points);

void orc_mvmean(const double* a, int len_a, int l, double* miu, double* si);
void orc_invalid_mask(const double* t, const double* si, int seg, int m, uint8_t* out);
void orc_min_max_window(const double* a, int n, int m, double* mn, double* mx);
void orc_lemire(const double* a, int n, int r, double* l, double* u);
void orc_normalized(const double* U, const double* L, double* Un, double* Ln, int len,
                    const double* max_mean, const double* min_mean,
                    const double* max_std, const double* min_std);
/* threshold selection; q_sorted may be NULL (sorted internally) */
double orc_find_t(int upper, int metric, const double* env, int l, const double* q,
                  const double* q_sorted, int m, double arg);
void orc_q_to_h(int upper, int metric, const double* q, int m, double t, double arg, double* h);
void orc_s_to_g(int upper, const double* env, int n, double t, double* g);
/* z[0..n) = cyclic correlation as src/sip.cpp computes it (FFT via the shim) */
void orc_sip(int n, int m, const double* h, const double* g, double* z);
double orc_trans_one(double zl, double zu, int m, int metric);
int orc_lbip_exceeds(double bound, double cutoff, int metric);
double orc_glb(int metric, const double* Q, const double* T, int m, double arg,
               const double* LQ, const double* UQ, int w, double bsf);
double orc_distance(int metric, const double* q, const double* t, int m, int w, double arg);

/* normalisation mode: 0 z-score (default), 1 raw (see fsmeld_oracle.c) */
void orc_set_normalization(int raw);

/* query z-normalisation as src/fsmeld.cpp:622-639 (sum, sum of squares);
 * a copy in raw mode */
void orc_normalize_query(const double* q, int m, double* q_normal);

typedef struct {
    long long valid;        /* kk1 */
    long long invalid;      /* invalid_candidates */
    long long after_lb;     /* kk2 (search) / candidates not pruned by LB_IP (cutoff) */
    long long after_glb;    /* kk3 (search) / candidates not pruned by GLB (cutoff) */
    long long exact_evals;  /* exact ELD evaluations */
    long long matches;      /* |A| (search / exact); k (cutoff) */
    double threshold;       /* final threshold (cutoff) */
    int m_k;                /* macro-segment length */
    long long segments;     /* full macro segments (forsize) */
    long long tail;         /* tail window count */
} orc_counters;

/*
 * Drivers over an in-memory target (the reference reads the same bytes from a
 * file).  Results go to caller buffers of capacity `cap`; the return value is
 * the number of results (may exceed cap: only cap are written), or a negative
 * error code.  seg_counts, when non-NULL, receives per-segment
 * (valid, after_lb, after_glb) triples for the forsize full segments (search).
 */
long long orc_search(const double* target, long long n, const double* query, int m,
                     double cutoff, int metric, int w, double arg,
                     long long excl_begin, long long excl_end,
                     long long* out_idx, long long cap, orc_counters* cnt,
                     long long* seg_counts);
long long orc_exact(const double* target, long long n, const double* query, int m,
                    double cutoff, int metric, int w, double arg,
                    long long excl_begin, long long excl_end,
                    long long* out_idx, double* out_dist, long long cap, orc_counters* cnt);
long long orc_cutoff(const double* target, long long n, const double* query, int m,
                     int k, int metric, int w, double arg,
                     long long excl_begin, long long excl_end,
                     long long* out_idx, double* out_dist, orc_counters* cnt);

#ifdef __cplusplus
}
#endif
#endif
