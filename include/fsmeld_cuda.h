/*
 * fsmeld_cuda.h -- C ABI of the B200 (sm_100a) implementation of FSMELD's
 * exact z-normalised subsequence range search (LB_IP -> GLB -> ELD).
 *
 * The reference exposes no library interface: its boundary is the
 * `fsmeld search|cutoff|exact` command (src/main.cpp:40-110) and three C++
 * entry points that take file paths and print to stdout
 * (include/funcs.h:64-72):
 *
 *   FSMELD(...)                 -> fsmeld_search, fsmeld_search_file
 *   FSMELD_find_threshold(...)  -> fsmeld_cutoff, fsmeld_cutoff_file
 *   FSMELD_exact(...)           -> fsmeld_exact,  fsmeld_exact_file
 *
 * The *_file entry points are drop-ins for those three functions: same
 * arguments (paths, m, cutoff or k, metric tag, w, arg, optional exclusion
 * interval), same stdout and CSV output.  The in-memory entry points below
 * them are what an FFI binding calls: plain pointers and sizes, caller-owned
 * host buffers, integer status codes (no exception crosses the ABI).
 *
 * Threading: a context owns one CUDA stream and its device buffers; calls on
 * one context are serialised by the caller; different contexts are
 * independent.
 */
#ifndef FSMELD_CUDA_H
#define FSMELD_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FSMELD_OK 0
#define FSMELD_E_ARG (-1)        /* invalid argument (message in fsmeld_last_error) */
#define FSMELD_E_CUDA (-2)       /* CUDA runtime error */
#define FSMELD_E_NOMEM (-3)      /* device allocation failed or budget exceeded */
#define FSMELD_E_SHORT (-4)      /* target shorter than 2*m-1 points */
#define FSMELD_E_FEWER_K (-5)    /* fewer valid, non-excluded candidates than k */
#define FSMELD_E_UNSUPPORTED (-6)
#define FSMELD_E_IO (-7)         /* file could not be read */

/* metric ids: the reference's MetricType values (include/funcs.h:10-18) */
#define FSMELD_DTW 1
#define FSMELD_EDR 2
#define FSMELD_ERP 3
#define FSMELD_LCSS 4
#define FSMELD_MSM 5

typedef struct fsmeld_ctx fsmeld_ctx;

/* Counters of one query; names follow the reference's printed counters
 * (src/fsmeld.cpp:981-996, 521-528, 1295-1306). */
typedef struct {
    int64_t valid;        /* kk1: valid, non-excluded candidates */
    int64_t invalid;      /* invalid or excluded candidates */
    int64_t after_lb;     /* kk2: candidates not pruned by LB_IP */
    int64_t after_glb;    /* kk3: candidates not pruned by GLB */
    int64_t exact_evals;  /* exact elastic distances computed */
    int64_t matches;      /* matches (search/exact) or k (cutoff) */
    double threshold;     /* cutoff used (search/exact) or final top-k threshold */
    int32_t m_k;          /* macro-segment length 2^ceil(log2(8m)), clipped to n */
    int32_t reserved;
    int64_t segments;     /* full macro segments */
    int64_t tail;         /* windows in the EOF-aligned tail segment */
    double device_ms;     /* device time of the call (CUDA events) */
    int64_t dp_cells;     /* band cells the exact DP computed (rows done x (2w+1)) */
} fsmeld_counters;

/* one query of a batched call */
typedef struct {
    const double* query;  /* host, m raw (unnormalised) values */
    int32_t m;
    int32_t metric;       /* FSMELD_DTW .. FSMELD_MSM */
    int32_t w;            /* Sakoe-Chiba radius, 0 <= w < m */
    int32_t k;            /* cutoff mode: k; otherwise ignored */
    double arg;           /* ERP gap g, EDR/LCSS epsilon, MSM cost c; 0 for DTW */
    double cutoff;        /* search/exact: distance cutoff */
    int64_t exclude_begin;/* optional half-open exclusion [begin,end) of */
    int64_t exclude_end;  /* candidate starts; -1,-1 for none */
} fsmeld_query;

/* results of one query of a batched call (caller-owned buffers) */
typedef struct {
    int64_t* idx;         /* match / rank indices, ascending index (search,
                             exact) or ascending (distance, index) (cutoff) */
    double* dist;         /* optional: distances for idx (exact, cutoff) */
    int64_t capacity;     /* entries available in idx (and dist) */
    int64_t count;        /* out: entries produced (may exceed capacity) */
    int32_t status;       /* out: FSMELD_OK or an error code */
    int32_t reserved;
    fsmeld_counters counters;  /* out */
    int64_t* seg_counts;  /* optional (search): 3 * segments int64 entries,
                             per full segment (valid, after_lb, after_glb) */
} fsmeld_result;

/* ---- context -------------------------------------------------------- */

/* Copy a host target (n native-endian doubles) to device `device`. */
int fsmeld_open(int device, const double* host_target, int64_t n, fsmeld_ctx** out);
/* Read a target file (headerless doubles) into a new context. */
int fsmeld_open_file(int device, const char* path, fsmeld_ctx** out);
/* Replace the context's target with a host series (copied; the device buffer
 * is reused when large enough). */
int fsmeld_load(fsmeld_ctx* ctx, const double* host_target, int64_t n);
/* Use a target already resident in device memory (not copied, not freed). */
int fsmeld_open_device(int device, const double* device_target, int64_t n, fsmeld_ctx** out);
int fsmeld_close(fsmeld_ctx* ctx);
int64_t fsmeld_target_length(const fsmeld_ctx* ctx);
/* Device address of the context's resident target (owned or borrowed), for
 * opening further contexts over the same series with fsmeld_open_device
 * (they must be closed before the owner).  No counterpart in the reference. */
const double* fsmeld_target_device(const fsmeld_ctx* ctx);
const char* fsmeld_last_error(const fsmeld_ctx* ctx);
const char* fsmeld_strerror(int status);
/* Batched calls (fsmeld_batch): the queries of one (m, w) group run
 * concurrently on this many worker streams of the context (1..16, default 4;
 * 1 runs them one after another).  Each worker holds its own query buffers,
 * so the device workspace grows with the concurrency.  No reference
 * counterpart (the reference runs one query per process). */
int fsmeld_set_concurrency(fsmeld_ctx* ctx, int queries);

/* Normalisation mode of the context's queries (include/funcs.h:20-28,
 * src/normalization_mode.cpp:7-21: set_normalization_mode /
 * normalization_mode).  FSMELD_NORM_ZSCORE (default; the only mode the
 * reference's command line sets, src/main.cpp:89) z-normalises the query and
 * every candidate window.  FSMELD_NORM_RAW compares raw values: the query is
 * used as given (a flat query is allowed) and every window whose points are
 * all finite is a candidate, flat windows included.  The reference declares
 * the raw mode but never consults it; here it runs the same cascade on raw
 * values (window mean 0, sigma 1). */
#define FSMELD_NORM_ZSCORE 0
#define FSMELD_NORM_RAW 1
int fsmeld_set_normalization(fsmeld_ctx* ctx, int mode);
int fsmeld_normalization(const fsmeld_ctx* ctx);

/* LB_IP form of batched searches and top-k queries (fsmeld_batch, modes 0
 * and 1) whose queries share (m, w) and metric (no reference counterpart; the reference computes LB_IP
 * per query with FFTs, src/sip.cpp:16-52).  FSMELD_LB_FFT: per query and
 * segment, the reference's threshold selection and an FP64 FFT.
 * FSMELD_LB_GEMM: one threshold pair for the group and the sliding inner
 * products of all its queries as one tensor-core product (BF16x3 split, FP32
 * accumulation, each bound lowered by its rounding-error margin).  Match
 * sets and rankings are the same either way; the LB_IP survivor counters
 * differ.
 * FSMELD_LB_AUTO (default): the tuner's choice for the group's shape. */
#define FSMELD_LB_AUTO 0
#define FSMELD_LB_FFT 1
#define FSMELD_LB_GEMM 2
int fsmeld_set_lb_form(fsmeld_ctx* ctx, int form);

/* Tuning table for the automatic choices (no reference counterpart): one rule
 * per line, "kind metric m_k limit choice", first match wins, '#' comments.
 *   dp <metric> <m_k> <w_max>  lane|wave   exact DP kernel over a candidate list
 *                                          (search, top-k) for w <= w_max
 *   dpx <metric> <m_k> <w_max> lane|wave   the same for the exact scan
 *   lb <metric> <m_k> <q_min>  fft|gemm    LB_IP form for groups of >= q_min searches
 *   lbk <metric> <m_k> <q_min> fft|gemm    the same for groups of top-k queries
 * Shapes no rule covers keep the built-in choice (the lane DP while its band
 * fits shared memory; the FFT LB_IP).  fsmeld_b200/tune.py measures the
 * rules on the GPU and writes fsmeld_b200/tune_table.txt, which the Python
 * binding loads into every context. */
int fsmeld_set_tuning(fsmeld_ctx* ctx, const char* table);

/* Cap on device workspace bytes (0 = no cap); exceeding it -> FSMELD_E_NOMEM.
 * The cap covers the context and the worker contexts of its batches together.
 * A batch query refused for workspace while the other queries of its batch
 * held theirs is run again alone, after the workers' buffers are released;
 * only a query that does not fit alone fails with FSMELD_E_NOMEM. */
int fsmeld_set_workspace_limit(fsmeld_ctx* ctx, int64_t bytes);
/* Device workspace bytes the context and its workers hold now (buffers grow
 * to the largest query served and are kept for the next call). */
int64_t fsmeld_workspace_bytes(fsmeld_ctx* ctx);
/* Frees the workspace of the context and its workers (the target stays
 * resident); the next call allocates what it needs again.  Waits for the
 * context's work in flight. */
int fsmeld_release_workspace(fsmeld_ctx* ctx);
/* Number of CUDA kernel launches issued by this context so far. */
int64_t fsmeld_kernel_launches(const fsmeld_ctx* ctx);
/* Per-stage device timing (no counterpart in the reference): when on, each
 * kernel launch is bracketed by CUDA events on the context's stream and its
 * time is added to its stage; fsmeld_stage_times copies per-stage totals (ms)
 * and launch counts and returns the number of stages; fsmeld_stage_name names
 * stage i (the kernel). */
int fsmeld_set_profiling(fsmeld_ctx* ctx, int on);
int fsmeld_stage_times(fsmeld_ctx* ctx, double* ms, int64_t* launches, int cap);
const char* fsmeld_stage_name(int stage);
/* Device time (ms, CUDA events on the context's stream) of the last query call. */
double fsmeld_last_call_ms(const fsmeld_ctx* ctx);

/* ---- single queries (src/fsmeld.cpp:570-1074, 185-569, 1075-1344) --- */

int fsmeld_search(fsmeld_ctx* ctx, const double* query, int m, double cutoff, int metric, int w,
                  double arg, int64_t exclude_begin, int64_t exclude_end, int64_t* out_idx,
                  int64_t capacity, int64_t* out_count, fsmeld_counters* counters,
                  int64_t* seg_counts);
int fsmeld_cutoff(fsmeld_ctx* ctx, const double* query, int m, int k, int metric, int w,
                  double arg, int64_t exclude_begin, int64_t exclude_end, int64_t* out_idx,
                  double* out_dist, fsmeld_counters* counters);
int fsmeld_exact(fsmeld_ctx* ctx, const double* query, int m, double cutoff, int metric, int w,
                 double arg, int64_t exclude_begin, int64_t exclude_end, int64_t* out_idx,
                 double* out_dist, int64_t capacity, int64_t* out_count,
                 fsmeld_counters* counters);

/* ---- batched queries: one call, many queries of mixed m, metric, w ---- */
/* mode: 0 = search, 1 = cutoff (k from each query), 2 = exact */
int fsmeld_batch(fsmeld_ctx* ctx, int mode, const fsmeld_query* queries, int nq,
                 fsmeld_result* results);

/* ---- diagnostics (no counterpart in the reference): per-stage device
 * arrays of one query, for stage-by-stage comparison with a CPU model.
 * what: 0 window means [S*kml], 1 window sigmas [S*kml], 2 U_normal
 * [S*m_k], 3 L_normal [S*m_k], 4 thresholds (t_l, t_u) [2*S], 5 LB_IP per
 * window [S*kml] (NaN for invalid windows), 6 LB_IP per window through the
 * tensor-core form (fsmeld_set_lb_form) with this query as the group, 7 the
 * (t_l, t_u, margin_l, margin_u) that form used; S counts the tail segment.
 * Returns the number of doubles available (copies at most cap). ---- */
int64_t fsmeld_inspect(fsmeld_ctx* ctx, const double* query, int m, int metric, int w, double arg,
                       int what, double* out, int64_t cap);

/* ---- exact scan that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- a serving loop
 * whose device memory belongs to another allocator (a framework's caching
 * pool, a memory-capped tenant) or code that must not allocate while a
 * request is in flight.  Same results as fsmeld_exact without an exclusion
 * interval: every valid window of device_target[0..n) through the banded
 * elastic DP; matches (distance <= cutoff) written in ascending window order
 * to the caller's device buffers device_out_idx / device_out_dist (at most
 * capacity entries; *host_out_count gets the total); runs on `stream` (a
 * cudaStream_t, NULL for the default stream) and returns after it finishes.
 * Scratch is one static device array of 12 MiB per GPU, held until exit.
 * Limits: n - m + 1 <= FSMELD_NOALLOC_MAX_WINDOWS, m <= FSMELD_NOALLOC_MAX_M,
 * and the DP band (2w+1) must fit shared memory (w <= 94 on a 227 KB opt-in
 * device); larger requests return FSMELD_E_ARG with a message.  The first
 * call on a device looks up the scratch array's device address and keeps it
 * for the process: make it before any stream capture, and do not use the
 * entry point on a device after cudaDeviceReset.  The call is synchronous and
 * must never be made while its stream is capturing.  It restores the caller's
 * current device.  Calls share the array: calls that overlap on the GPU race,
 * so serialise them. */
#define FSMELD_NOALLOC_MAX_WINDOWS 262144
#define FSMELD_NOALLOC_MAX_M 2048
int fsmeld_exact_noalloc(int device, const double* device_target, int64_t n, const double* host_query, int m,
                         int metric, int w, double arg, double cutoff, int64_t* device_out_idx,
                         double* device_out_dist, int64_t capacity, int64_t* host_out_count, void* stream);

/* ---- drop-ins for the reference's entry points (include/funcs.h:64-72):
 *      read TARGET.bin / QUERY.txt, print the reference's stdout lines and
 *      append the experiment CSV.  tag is "dtw", "erp", "edr", "lcss" or
 *      "msm".  Return FSMELD_OK or an error code (message on stderr). ---- */
int fsmeld_search_file(const char* target_path, const char* query_path, int m, double cutoff,
                       const char* tag, int w, double arg, int64_t exclude_begin,
                       int64_t exclude_end);
int fsmeld_cutoff_file(const char* target_path, const char* query_path, int m, int k,
                       const char* tag, int w, double arg, int64_t exclude_begin,
                       int64_t exclude_end);
int fsmeld_exact_file(const char* target_path, const char* query_path, int m, double cutoff,
                      const char* tag, int w, double arg, int64_t exclude_begin,
                      int64_t exclude_end);

#ifdef __cplusplus
}
#endif
#endif
