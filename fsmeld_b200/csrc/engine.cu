// Host orchestration of the FSMELD pipeline on one GPU, behind the C ABI in
// include/fsmeld_cuda.h.
//
// Per query: window statistics (k_mvmean) -> envelopes (k_envelope) ->
// thresholds (k_threshold) -> LB_IP + compaction (k_lbip) -> GLB
// (k_glb_tq, k_glb_qt) -> exact DP (k_dp) -> ordered results.  Statistics
// and envelopes depend only on (target, m, w), so a batch computes them once
// per distinct (m, w).  All candidate lists stay on the device; the host
// reads back counters and the final (small) result lists.
//
// The host prepares each query exactly as the reference does
// (src/fsmeld.cpp:622-643: sequential sums, mean, sigma, (q - mean) / sigma;
// sorted copy; pow(q, a) from the C library as src/find_t_lp.cpp:253) and
// uploads the tables the kernels read.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fsmeld_cuda.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.cuh"

namespace fsm {

// The dynamic shared-memory limit of a kernel is a process-wide attribute
// (per device), so every context raises it through this one record and no
// context ever lowers it under another's launches.
cudaError_t raise_smem_limit(const void* kernel, int device, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = set[{device, kernel}];
    if (cur >= bytes) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

thread_local std::string g_last_error;

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(e),
             cudaGetErrorString(e), file, line, what);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? FSMELD_E_NOMEM : FSMELD_E_CUDA;
}

static int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// ------------------------------------------------------------------ geometry

// src/fsmeld.cpp:28-37
int macro_length(int m, long long available) {
    long long sel = 1;
    while (sel < 8LL * m) sel *= 2;
    if (available < 2LL * m - 1) return -1;
    if (available < sel) sel = available;
    if (sel > 2147483647LL) return -1;
    return (int)sel;
}

int make_geom(long long n, int m, long long eb, long long ee, Geom* g) {
    const int mk = macro_length(m, n);
    if (mk < 0) return fail(FSMELD_E_SHORT, "Target is too short for this query length.");
    g->n = n;
    g->m = m;
    g->m_k = mk;
    g->kml = mk - m + 1;
    g->inv_kml = 1.0 / (double)g->kml;
    g->tsn = n - m + 1;
    g->forsize = g->tsn / g->kml;
    const long long tail = g->tsn % g->kml;
    g->tail_lo = (int)(g->kml - tail);
    g->S = g->forsize + (tail > 0 ? 1 : 0);
    g->excl_b = (eb >= 0 && ee > eb) ? eb : -1;
    g->excl_e = (eb >= 0 && ee > eb) ? ee : -1;
    return FSMELD_OK;
}

// ----------------------------------------------------------------- queries

static int metric_p(int metric) { return (metric == DTW || metric == ERP) ? 2 : (metric == MSM ? 1 : 0); }

// src/find_t_lp.cpp:148-186
static double fn_D(double q, double C, int metric) {
    if (metric == MSM) return C;
    if (metric == ERP || metric == DTW) return (q - C) * (q - C);
    return 1;
}
static double fn_tu(double q, double C, int metric) {
    if (metric == MSM) return q - C;
    if (metric == ERP) return q - std::fabs(q - C);
    if (metric == EDR || metric == LCSS) return q - C;
    return q;
}
static double fn_tl(double q, double C, int metric) {
    if (metric == MSM) return q + C;
    if (metric == ERP) return q + std::fabs(q - C);
    if (metric == EDR || metric == LCSS) return q + C;
    return q;
}

int prepare_query(const double* q, int m, int metric, int w, double arg, HostQuery* hq, bool raw) {
    if (m < 2) return fail(FSMELD_E_ARG, "m must be at least 2.");
    if (w < 0 || w >= m) return fail(FSMELD_E_ARG, "w must satisfy 0 <= w < m.");
    if (metric < DTW || metric > MSM) return fail(FSMELD_E_ARG, "Unsupported metric.");
    if ((metric == EDR || metric == LCSS || metric == MSM) && !(arg >= 0))
        return fail(FSMELD_E_ARG, "Matching tolerance and MSM cost must be non-negative.");
    if (!std::isfinite(arg)) return fail(FSMELD_E_ARG, "Invalid finite metric parameter.");
    double ex = 0, ex2 = 0;
    for (int i = 0; i < m; ++i) {
        if (!std::isfinite(q[i])) return fail(FSMELD_E_ARG, "Query must begin with m finite numeric values.");
        ex += q[i];
        ex2 += q[i] * q[i];
    }
    const double mean = ex / m;
    double sd = ex2 / m;
    sd = std::sqrt(sd - mean * mean);
    if (!raw && (!std::isfinite(sd) || sd <= 1e-12))
        return fail(FSMELD_E_ARG,
                    "Query cannot be z-normalized: non-finite or near-zero standard deviation.");
    hq->m = m; hq->w = w; hq->metric = metric; hq->arg = arg; hq->p = metric_p(metric);
    hq->qn.resize(m);
    for (int i = 0; i < m; ++i) hq->qn[i] = raw ? q[i] : (q[i] - mean) / sd;
    const std::vector<double>& qn = hq->qn;
    // query envelope (src/fsmeld.cpp:721): window extremes, most recent on ties
    hq->LQ.resize(m); hq->UQ.resize(m);
    for (int o = 0; o < m; ++o) {
        const int a = std::max(0, o - w), b = std::min(m - 1, o + w);
        double lo = qn[a], hi = qn[a];
        for (int i = a + 1; i <= b; ++i) {
            lo = (qn[i] <= lo) ? qn[i] : lo;
            hi = (qn[i] >= hi) ? qn[i] : hi;
        }
        hq->LQ[o] = lo; hq->UQ[o] = hi;
    }
    hq->qs = qn;
    std::sort(hq->qs.begin(), hq->qs.end());
    hq->pw.resize(3 * m); hq->opw.resize(3 * m);
    hq->Dq.resize(m); hq->tlq.resize(m); hq->tuq.resize(m);
    hq->oD.resize(m); hq->otl.resize(m); hq->otu.resize(m);
    for (int j = 0; j < m; ++j) {
        for (int a = 0; a < 3; ++a) {
            hq->pw[a * m + j] = std::pow(hq->qs[j], a);
            hq->opw[a * m + j] = std::pow(qn[j], a);
        }
        hq->Dq[j] = fn_D(hq->qs[j], arg, metric);
        hq->tlq[j] = fn_tl(hq->qs[j], arg, metric);
        hq->tuq[j] = fn_tu(hq->qs[j], arg, metric);
        hq->oD[j] = fn_D(qn[j], arg, metric);
        hq->otl[j] = fn_tl(qn[j], arg, metric);
        hq->otu[j] = fn_tu(qn[j], arg, metric);
    }
    auto order = [&](const std::vector<double>& key, bool desc) {
        std::vector<int> o(m);
        for (int i = 0; i < m; ++i) o[i] = i;
        std::stable_sort(o.begin(), o.end(), [&](int a, int b) {
            return desc ? key[a] > key[b] : key[a] < key[b];
        });
        return o;
    };
    hq->ordA_l = order(hq->otl, true);
    hq->ordB_l = order(qn, true);
    hq->ordA_u = order(hq->otu, false);
    hq->ordB_u = order(qn, false);
    return FSMELD_OK;
}

}  // namespace fsm

// ------------------------------------------------------------------ context

using namespace fsm;

struct fsmeld_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double* d_target = nullptr;
    long long n = 0;
    bool own_target = false;
    int sm_count = 148;
    int smem_optin = 227 * 1024;
    long long ws_limit = 0;
    // worker contexts point at the context that created them; workspace
    // bytes are counted and capped over the whole family (the context and
    // its workers) under the root's mutex
    fsmeld_ctx* parent = nullptr;
    std::mutex ws_mu;
    long long launches = 0;
    // queries of one batch group run concurrently on this many worker
    // contexts (own stream and buffers, shared target, statistics, envelopes)
    int concurrency = 4;
    std::vector<fsmeld_ctx*> workers;
    cudaEvent_t ev_ready = nullptr;  // shared statistics/envelopes of a group are on the device
    // FSMELD_DP_EXACT=1: run every DP candidate in the exact boundary mode
    // (same results; a diagnostic switch for the mode that in-range data never needs)
    bool dp_exact = false;
    // FSMELD_DP_FORM: which exact-DP kernel runs -- 0 auto (the lane-per-candidate
    // DP while its band and ring fit shared memory, else the wavefront), 1 the
    // lane DP only (global band scratch for wide bands), 2 the wavefront
    // wherever it applies (w <= 255).  Same results; a switch for tests and
    // measurements.
    int dp_form = 0;
    // LB_IP form for batched searches of equal (m, w) and metric: 0 auto (the
    // tuner's choice), 1 the per-query FFT form, 2 the tensor-core product
    int lb_form = 0;
    // tuning table (fsmeld_set_tuning): rules for the automatic choices
    struct TuneRule { int kind, metric, m_k, lim, choice; };  // 0 dp, 1 lb (search), 2 lbk (top-k), 3 dpx (scan)
    std::vector<TuneRule> tune;
    // normalisation mode (the reference's set_normalization_mode, include/funcs.h:20-28):
    // false z-score (the reference CLI's only mode), true raw
    bool raw = false;
    double last_ms = 0.0;
    std::string err;
    struct Buf { void* p = nullptr; size_t bytes = 0; };
    std::map<std::string, Buf> bufs;
    std::map<int, double2*> twiddles;
    // opt-in per-stage device timing (CUDA events around each launch)
    bool prof = false;
    struct ProfRec { int stage; cudaEvent_t a, b; };
    std::vector<ProfRec> pending;
    std::vector<cudaEvent_t> pool;
    double stage_ms[16] = {0};
    long long stage_n[16] = {0};
};

namespace fsm {

static size_t ws_total(const fsmeld_ctx* c) {
    size_t t = 0;
    for (auto& kv : c->bufs) t += kv.second.bytes;
    return t;
}

static fsmeld_ctx* ws_root(fsmeld_ctx* c) {
    while (c->parent) c = c->parent;
    return c;
}

// workspace bytes of a context and its workers (and theirs); the caller
// holds the root's ws_mu
static size_t ws_family_total(const fsmeld_ctx* c) {
    size_t t = ws_total(c);
    for (const fsmeld_ctx* w : c->workers) t += ws_family_total(w);
    return t;
}

// frees every workspace buffer of c (after its stream's work is done)
static void release_bufs(fsmeld_ctx* c) {
    if (c->stream) cudaStreamSynchronize(c->stream);
    std::lock_guard<std::mutex> lk(ws_root(c)->ws_mu);
    for (auto& kv : c->bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    c->bufs.clear();
}

static int buf(fsmeld_ctx* c, const std::string& name, size_t bytes, void** out) {
    if (bytes == 0) bytes = 16;
    fsmeld_ctx* root = ws_root(c);
    std::lock_guard<std::mutex> lk(root->ws_mu);
    auto& b = c->bufs[name];
    if (b.bytes < bytes) {
        if (b.p) { cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
        const size_t want = bytes + bytes / 8;
        const size_t held = ws_family_total(root);
        if (root->ws_limit > 0 && (long long)(held + want) > root->ws_limit) {
            char msg[256];
            snprintf(msg, sizeof(msg),
                     "Device workspace budget exceeded: %.2f GB held, %.2f GB more for '%s', limit %.2f GB.",
                     held / 1e9, want / 1e9, name.c_str(), root->ws_limit / 1e9);
            return fail(FSMELD_E_NOMEM, msg);
        }
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) { b.p = nullptr; return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__); }
        b.bytes = want;
    }
    *out = b.p;
    return FSMELD_OK;
}

template <typename T>
static int bufT(fsmeld_ctx* c, const std::string& name, size_t count, T** out) {
    void* p;
    int r = buf(c, name, count * sizeof(T), &p);
    *out = (T*)p;
    return r;
}

template <typename K>
static int allow_smem(fsmeld_ctx* c, K kernel, size_t bytes) {
    if (bytes > (size_t)c->smem_optin) return fail(FSMELD_E_UNSUPPORTED, "shared memory request too large");
    const cudaError_t e = fsm::raise_smem_limit((const void*)kernel, c->device, bytes);
    if (e != cudaSuccess) return fsm::cuda_fail(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    return FSMELD_OK;
}

enum Stage { ST_STATS, ST_ENV, ST_THR, ST_LBIP, ST_GLB1, ST_GLB2, ST_DP, ST_SELECT, ST_FWD, ST_DPW, ST_GEMM, ST_N };
static const char* kStageNames[ST_N] = {"k_mvmean", "k_envelope", "k_threshold", "k_lbip",
                                        "k_glb_tq", "k_glb_qt", "k_dp", "k_select",
                                        "k_fwd_env", "k_dpw", "k_lbgemm"};

static cudaEvent_t prof_event(fsmeld_ctx* c) {
    if (!c->pool.empty()) { cudaEvent_t e = c->pool.back(); c->pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
static void prof_begin(fsmeld_ctx* c, int stage) {
    if (!c->prof) return;
    fsmeld_ctx::ProfRec r{stage, prof_event(c), prof_event(c)};
    cudaEventRecord(r.a, c->stream);
    c->pending.push_back(r);
}
static void prof_end(fsmeld_ctx* c) {
    if (!c->prof || c->pending.empty()) return;
    cudaEventRecord(c->pending.back().b, c->stream);
}
static void prof_collect(fsmeld_ctx* c) {
    if (c->pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto& r : c->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            c->stage_ms[r.stage] += ms;
            c->stage_n[r.stage] += 1;
        }
        c->pool.push_back(r.a);
        c->pool.push_back(r.b);
    }
    c->pending.clear();
}

#define LAUNCH_CHECK(c)                                                  \
    do {                                                                 \
        prof_end(c);                                                     \
        (c)->launches++;                                                 \
        cudaError_t _le = cudaGetLastError();                            \
        if (_le != cudaSuccess) return cuda_fail(_le, "kernel launch", __FILE__, __LINE__); \
    } while (0)

static int twiddle_table(fsmeld_ctx* c, int P, const double2** out) {
    auto it = c->twiddles.find(P);
    if (it != c->twiddles.end()) { *out = it->second; return FSMELD_OK; }
    std::vector<double2> w(P);
    for (int k = 0; k < P; ++k) {
        const double ang = 6.283185307179586476925286766559 * (double)k / (double)P;
        w[k] = make_double2(std::cos(ang), -std::sin(ang));
    }
    double2* d;
    FSM_CUDA_TRY(cudaMalloc(&d, sizeof(double2) * P));
    FSM_CUDA_TRY(cudaMemcpy(d, w.data(), sizeof(double2) * P, cudaMemcpyHostToDevice));
    c->twiddles[P] = d;
    *out = d;
    return FSMELD_OK;
}

// upload a prepared query into a named device slot
static int upload_query(fsmeld_ctx* c, const HostQuery& hq, const std::string& slot, QueryDev* qd) {
    const int m = hq.m;
    const size_t nd = (size_t)m * (3 + 4 + 3 + 3 + 3 + 3), ni = (size_t)m * 4;
    std::vector<unsigned char> host(nd * 8 + ni * 4);
    double* d = (double*)host.data();
    size_t o = 0;
    auto put = [&](const std::vector<double>& v) { memcpy(d + o, v.data(), v.size() * 8); size_t at = o; o += v.size(); return at; };
    const size_t o_qn = put(hq.qn), o_LQ = put(hq.LQ), o_UQ = put(hq.UQ), o_qs = put(hq.qs);
    const size_t o_pw = put(hq.pw), o_Dq = put(hq.Dq), o_tlq = put(hq.tlq), o_tuq = put(hq.tuq);
    const size_t o_opw = put(hq.opw), o_oD = put(hq.oD), o_otl = put(hq.otl), o_otu = put(hq.otu);
    int* ip = (int*)(d + nd);
    memcpy(ip, hq.ordA_l.data(), m * 4);
    memcpy(ip + m, hq.ordB_l.data(), m * 4);
    memcpy(ip + 2 * m, hq.ordA_u.data(), m * 4);
    memcpy(ip + 3 * m, hq.ordB_u.data(), m * 4);
    void* dev;
    int r = buf(c, slot, host.size(), &dev);
    if (r) return r;
    FSM_CUDA_TRY(cudaMemcpyAsync(dev, host.data(), host.size(), cudaMemcpyHostToDevice, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));  // host staging buffer is released on return
    const double* D = (const double*)dev;
    const int* I = (const int*)(D + nd);
    qd->m = m; qd->w = hq.w; qd->metric = hq.metric; qd->p = hq.p; qd->arg = hq.arg;
    qd->cutoff = 0.0;
    qd->qn = D + o_qn; qd->LQ = D + o_LQ; qd->UQ = D + o_UQ; qd->qs = D + o_qs;
    qd->pw = D + o_pw; qd->Dq = D + o_Dq; qd->tlq = D + o_tlq; qd->tuq = D + o_tuq;
    qd->opw = D + o_opw; qd->oD = D + o_oD; qd->otl = D + o_otl; qd->otu = D + o_otu;
    qd->ordA_l = I; qd->ordB_l = I + m; qd->ordA_u = I + 2 * m; qd->ordB_u = I + 3 * m;
    return FSMELD_OK;
}

// ------------------------------------------------------------- pipeline

struct Stats {
    double* MU = nullptr;
    double* SIG = nullptr;
    double* Un = nullptr;
    double* Ln = nullptr;
    double* Lraw = nullptr;  // forward windows min / max(t[p .. p+w]) of the raw target
    double* Uraw = nullptr;
};

static int run_stats(fsmeld_ctx* c, const Geom& g, Stats* st, const std::string& tag) {
    int r;
    if ((r = bufT(c, "mu" + tag, (size_t)g.S * g.kml, &st->MU))) return r;
    if ((r = bufT(c, "sig" + tag, (size_t)g.S * g.kml, &st->SIG))) return r;
    const size_t smem = mvmean_smem_bytes();
    if ((r = allow_smem(c, k_mvmean, smem))) return r;
    const unsigned blocks = (unsigned)((g.S + 31) / 32);
    prof_begin(c, ST_STATS);
    k_mvmean<<<blocks, kMvmeanThreads, smem, c->stream>>>(c->d_target, g, st->MU, st->SIG);
    LAUNCH_CHECK(c);
    return FSMELD_OK;
}

// Per-block scratch areas in global memory start on 256-byte boundaries (the
// kernels' layouts align their arrays relative to the area's start).
static inline size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

template <int T, int OPT>
static int launch_env(fsmeld_ctx* c, const Geom& g, int w, Stats* st) {
    const size_t work = round256(envelope_work_bytes(g.m_k));
    double* gwork = nullptr;
    size_t smem = work;
    unsigned grid;
    int r;
    const bool gw_path = work + 8192 > (size_t)c->smem_optin;
    if (!gw_path) {
        if ((r = allow_smem(c, k_envelope<T, OPT, false>, smem))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_envelope<T, OPT, false>, T, smem));
        grid = (unsigned)std::min<long long>(g.S, (long long)std::max(1, per_sm) * c->sm_count);
    } else {
        smem = 0;
        grid = (unsigned)std::min<long long>(g.S, (long long)c->sm_count * 2);
        if ((r = bufT(c, "envwork", (work / 8) * grid, &gwork))) return r;
    }
    prof_begin(c, ST_ENV);
    if (gw_path)
        k_envelope<T, OPT, true><<<grid, T, smem, c->stream>>>(c->d_target, st->MU, st->SIG, g, w, st->Un, st->Ln,
                                                               gwork, (long long)(work / 8));
    else
        k_envelope<T, OPT, false><<<grid, T, smem, c->stream>>>(c->d_target, st->MU, st->SIG, g, w, st->Un, st->Ln,
                                                                gwork, (long long)(work / 8));
    LAUNCH_CHECK(c);
    return FSMELD_OK;
}

static int run_env(fsmeld_ctx* c, const Geom& g, int w, Stats* st, const std::string& tag) {
    int r;
    if ((r = bufT(c, "un" + tag, (size_t)g.S * g.m_k, &st->Un))) return r;
    if ((r = bufT(c, "ln" + tag, (size_t)g.S * g.m_k, &st->Ln))) return r;
    if ((r = bufT(c, "lraw" + tag, (size_t)g.n, &st->Lraw))) return r;
    if ((r = bufT(c, "uraw" + tag, (size_t)g.n, &st->Uraw))) return r;
    {
        const size_t fsm = fwd_env_smem_bytes(w);
        if ((r = allow_smem(c, k_fwd_env, fsm))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fwd_env, kFwdThreads, fsm));
        const unsigned fgrid = (unsigned)std::max<long long>(
            1, std::min<long long>((g.n + kFwdTile - 1) / kFwdTile, (long long)std::max(1, per_sm) * c->sm_count));
        prof_begin(c, ST_FWD);
        k_fwd_env<<<fgrid, kFwdThreads, fsm, c->stream>>>(c->d_target, g.n, w, st->Lraw, st->Uraw);
        LAUNCH_CHECK(c);
    }
    const int mk = g.m_k;
    if (mk <= 1024) return launch_env<256, 4>(c, g, w, st);
    if (mk <= 2048) return launch_env<512, 4>(c, g, w, st);
    if (mk <= 4096) return launch_env<1024, 4>(c, g, w, st);
    if (mk <= 8192) return launch_env<1024, 8>(c, g, w, st);
    if (mk <= 16384) return launch_env<1024, 16>(c, g, w, st);
    return fail(FSMELD_E_UNSUPPORTED, "macro segments longer than 16384 points are not supported");
}

template <int T, int IPT>
static int launch_thr(fsmeld_ctx* c, const Geom& g, const ThrJob* djobs, int njobs, int m) {
    const size_t work = round256(threshold_work_bytes(T * IPT, threshold_sort_tmp_bytes<T, IPT>(), m));
    unsigned char* gwork = nullptr;
    size_t smem = work;
    unsigned gx;
    int r;
    const bool gw_path = work + 16384 > (size_t)c->smem_optin;
    if (!gw_path) {
        if ((r = allow_smem(c, k_threshold<T, IPT, false>, smem))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_threshold<T, IPT, false>, T, smem));
        gx = (unsigned)std::min<long long>(2 * g.S, (long long)std::max(1, per_sm) * c->sm_count * 4);
    } else {
        // global scratch for the runs, sorted values and sweep; the sort's temp
        // storage in shared memory
        smem = threshold_sort_tmp_bytes<T, IPT>();
        if (smem + 8192 > (size_t)c->smem_optin)
            return fail(FSMELD_E_UNSUPPORTED, "threshold sort does not fit in shared memory");
        if ((r = allow_smem(c, k_threshold<T, IPT, true>, smem))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_threshold<T, IPT, true>, T, smem));
        gx = (unsigned)std::min<long long>(2 * g.S, (long long)std::max(1, per_sm) * c->sm_count * 2);
        const size_t gstride = round256(threshold_work_bytes(T * IPT, 0, m));
        if ((r = bufT(c, "thrwork", gstride * gx * (size_t)njobs, &gwork))) return r;
        dim3 grid(gx, njobs);
        prof_begin(c, ST_THR);
        k_threshold<T, IPT, true><<<grid, T, smem, c->stream>>>(g, djobs, gwork, (long long)gstride);
        LAUNCH_CHECK(c);
        return FSMELD_OK;
    }
    dim3 grid(gx, njobs);
    prof_begin(c, ST_THR);
    k_threshold<T, IPT, false><<<grid, T, smem, c->stream>>>(g, djobs, gwork, (long long)work);
    LAUNCH_CHECK(c);
    return FSMELD_OK;
}

static int run_thr(fsmeld_ctx* c, const Geom& g, const std::vector<ThrJob>& jobs) {
    if (jobs.empty()) return FSMELD_OK;
    ThrJob* dj;
    int r;
    if ((r = bufT(c, "thrjobs", jobs.size(), &dj))) return r;
    FSM_CUDA_TRY(cudaMemcpyAsync(dj, jobs.data(), sizeof(ThrJob) * jobs.size(), cudaMemcpyHostToDevice, c->stream));
    const int m = g.m;
    const int cnt = g.m_k - 2 * m + 2;
    const int nj = (int)jobs.size();
    if (cnt <= 512) r = launch_thr<128, 4>(c, g, dj, nj, m);
    else if (cnt <= 1024) r = launch_thr<256, 4>(c, g, dj, nj, m);
    else if (cnt <= 2048) r = launch_thr<256, 8>(c, g, dj, nj, m);
    else if (cnt <= 4096) r = launch_thr<512, 8>(c, g, dj, nj, m);
    else if (cnt <= 8192) r = launch_thr<1024, 8>(c, g, dj, nj, m);
    else if (cnt <= 16384) r = launch_thr<1024, 16>(c, g, dj, nj, m);
    else r = fail(FSMELD_E_UNSUPPORTED, "envelope core longer than 16384 points is not supported");
    if (r) return r;
    // the job array is read by the kernel: keep it alive until it finishes
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return FSMELD_OK;
}

static int run_lbip(fsmeld_ctx* c, const Geom& g, LbJob job) {
    int P = 1, logP = 0;
    while (P < g.m_k) { P <<= 1; ++logP; }
    const double2* W;
    int r;
    if ((r = twiddle_table(c, P, &W))) return r;
    size_t smem = lbip_smem_bytes(P, g.m_k, g.m, job.q.metric);
    unsigned grid;
    if (smem + 8192 <= (size_t)c->smem_optin) {
        job.gwork = nullptr;
        if ((r = allow_smem(c, k_lbip<256, false>, smem))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lbip<256, false>, 256, smem));
        grid = (unsigned)std::min<long long>(g.S, (long long)std::max(1, per_sm) * c->sm_count);
    } else {
        grid = (unsigned)std::min<long long>(g.S, (long long)c->sm_count * 2);
        unsigned char* gw;
        smem = round256(smem);
        if ((r = bufT(c, "lbwork", smem * grid, &gw))) return r;
        job.gwork = gw;
        job.slot_stride = (long long)smem;
        smem = 0;
    }
    prof_begin(c, ST_LBIP);
    if (job.gwork)
        k_lbip<256, true><<<grid, 256, smem, c->stream>>>(g, job, W, P, logP);
    else
        k_lbip<256, false><<<grid, 256, smem, c->stream>>>(g, job, W, P, logP);
    LAUNCH_CHECK(c);
    return FSMELD_OK;
}

// counters slot layout
enum { C_SURV, C_G1, C_G2, C_OUT, C_VALID, C_SEED, C_SEEDOUT, C_DPNEXT, C_CELLS, C_N };

static int run_glb(fsmeld_ctx* c, const Geom& g, const QueryDev& qd, const Stats& st, const long long* in,
                   unsigned long long* cnt, long long cap, long long* segc, long long** out_list,
                   double** out_qt = nullptr, const double* cutoff_ptr = nullptr) {
    long long *g1, *g2;
    double *g1b, *g1t;
    int r;
    if ((r = bufT(c, "g1", (size_t)cap, &g1))) return r;
    if ((r = bufT(c, "g1b", (size_t)cap, &g1b))) return r;
    if ((r = bufT(c, "g1t", (size_t)cap, &g1t))) return r;
    if ((r = bufT(c, "g2", (size_t)cap, &g2))) return r;
    GlbJob j1{};
    j1.q = qd; j1.target = c->d_target; j1.MU = st.MU; j1.SIG = st.SIG;
    j1.lraw = st.Lraw; j1.uraw = st.Uraw;
    j1.in = in; j1.n_in = cnt + C_SURV; j1.in_cap = cap;
    j1.out = g1; j1.out_b = g1b; j1.out_t = g1t; j1.n_out = cnt + C_G1; j1.out_cap = cap;
    j1.segc = segc;
    j1.cutoff_ptr = cutoff_ptr;
    const size_t sm1 = sizeof(double) * 3 * qd.m;
    const void* tqf = qd.metric == DTW ? (const void*)k_glb_tq<DTW>
                    : qd.metric == ERP ? (const void*)k_glb_tq<ERP>
                    : qd.metric == EDR ? (const void*)k_glb_tq<EDR>
                    : qd.metric == LCSS ? (const void*)k_glb_tq<LCSS> : (const void*)k_glb_tq<MSM>;
    if ((r = allow_smem(c, tqf, sm1))) return r;
    prof_begin(c, ST_GLB1);
    switch (qd.metric) {
        case DTW: k_glb_tq<DTW><<<c->sm_count * 8, 256, sm1, c->stream>>>(g, j1); break;
        case ERP: k_glb_tq<ERP><<<c->sm_count * 8, 256, sm1, c->stream>>>(g, j1); break;
        case EDR: k_glb_tq<EDR><<<c->sm_count * 8, 256, sm1, c->stream>>>(g, j1); break;
        case LCSS: k_glb_tq<LCSS><<<c->sm_count * 8, 256, sm1, c->stream>>>(g, j1); break;
        default: k_glb_tq<MSM><<<c->sm_count * 8, 256, sm1, c->stream>>>(g, j1); break;
    }
    LAUNCH_CHECK(c);
    GlbJob j2 = j1;
    double* g2t;
    if ((r = bufT(c, "g2t", (size_t)cap, &g2t))) return r;
    j2.in = g1; j2.in_b = g1b; j2.in_t = g1t; j2.n_in = cnt + C_G1;
    j2.out = g2; j2.out_b = nullptr; j2.out_t = g2t; j2.n_out = cnt + C_G2;
    const size_t sm2 = sizeof(double) * (((size_t)qd.m + 1) & ~(size_t)1);
    const void* qtf = qd.metric == DTW ? (const void*)k_glb_qt<DTW>
                    : qd.metric == ERP ? (const void*)k_glb_qt<ERP>
                    : qd.metric == EDR ? (const void*)k_glb_qt<EDR>
                    : qd.metric == LCSS ? (const void*)k_glb_qt<LCSS> : (const void*)k_glb_qt<MSM>;
    if ((r = allow_smem(c, qtf, sm2))) return r;
    int per_sm = 0;
    FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qtf, 128, sm2));
    const unsigned g2grid = (unsigned)(std::max(1, per_sm) * c->sm_count);
    prof_begin(c, ST_GLB2);
    switch (qd.metric) {
        case DTW: k_glb_qt<DTW><<<g2grid, 128, sm2, c->stream>>>(g, j2); break;
        case ERP: k_glb_qt<ERP><<<g2grid, 128, sm2, c->stream>>>(g, j2); break;
        case EDR: k_glb_qt<EDR><<<g2grid, 128, sm2, c->stream>>>(g, j2); break;
        case LCSS: k_glb_qt<LCSS><<<g2grid, 128, sm2, c->stream>>>(g, j2); break;
        default: k_glb_qt<MSM><<<g2grid, 128, sm2, c->stream>>>(g, j2); break;
    }
    LAUNCH_CHECK(c);
    if (out_qt) *out_qt = g2t;
    *out_list = g2;
    return FSMELD_OK;
}

// The tuning table's choice for a shape: the first rule of `kind` for the
// metric and macro-segment length whose limit matches v (dp, dpx: v = w <=
// limit, choice 1 lane / 2 wave; lb, lbk: v = the group's query count >=
// limit, choice 1 fft / 2 gemm).  0 when no rule matches.
static int tuned(const fsmeld_ctx* c, int kind, int metric, int m_k, int v) {
    for (const auto& t : c->tune) {
        if (t.kind != kind || t.metric != metric || t.m_k != m_k) continue;
        if ((kind == 0 || kind == 3) ? v <= t.lim : v >= t.lim) return t.choice;
    }
    return 0;
}

static int run_dp(fsmeld_ctx* c, const Geom& g, DpJob job, long long expected) {
    const int w = job.q.w;
    const int warps = kDpThreads / 32;
    const size_t per_warp = dp_warp_doubles(w);
    size_t smem = sizeof(double) * per_warp * warps;
    int r;
    unsigned long long* next;
    if ((r = bufT(c, "dpnext", 1, &next))) return r;
    FSM_CUDA_TRY(cudaMemsetAsync(next, 0, sizeof(unsigned long long), c->stream));
    job.next = next;
    job.gwork = nullptr;
    job.force_exact = c->dp_exact ? 1 : 0;
    unsigned grid;
    const bool gw_path = smem > (size_t)c->smem_optin - 4096;
    // wide bands (and FSMELD_DP_FORM=wave): one warp per candidate, band in registers
    int form = c->dp_form;
    if (form == 0) form = tuned(c, job.list ? 0 : 3, job.q.metric, g.m_k, w);
    const void* wk = form == 1 ? nullptr : dpw_kernel(job.q.metric, w);
    const size_t wsm = dpw_smem_bytes(job.q.m, kDpwThreads / 32);
    if (wk && wsm + 1024 <= (size_t)c->smem_optin && (form == 2 || gw_path)) {
        if ((r = allow_smem(c, wk, wsm))) return r;
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wk, kDpwThreads, wsm));
        const long long want = (expected + kDpwThreads / 32 - 1) / (kDpwThreads / 32);
        grid = (unsigned)std::max<long long>(1, std::min<long long>(want, (long long)std::max(1, per_sm) * c->sm_count));
        prof_begin(c, ST_DPW);
        Geom ga = g;
        void* args[] = {&ga, &job};
        const cudaError_t le = cudaLaunchKernel(wk, dim3(grid), dim3(kDpwThreads), args, wsm, c->stream);
        if (le != cudaSuccess) return cuda_fail(le, "k_dpw launch", __FILE__, __LINE__);
        LAUNCH_CHECK(c);
        return FSMELD_OK;
    }
    if (gw_path) {
        // band scratch in global memory (L2-resident per warp): 16 warps per SM
        const long long want = (expected + warps * 32 - 1) / (warps * 32);
        grid = (unsigned)std::max<long long>(1, std::min<long long>(want, (long long)c->sm_count * (16 / warps)));
        double* gw;
        if ((r = bufT(c, "dpwork", per_warp * warps * grid, &gw))) return r;
        job.gwork = gw;
        smem = 0;
    }
    const void* kf = dp_kernel(job.q.metric, gw_path);
    if ((r = allow_smem(c, kf, smem))) return r;
    if (!gw_path) {
        int per_sm = 0;
        FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, warps * 32, smem));
        const long long want = (expected + warps * 32 - 1) / (warps * 32);
        grid = (unsigned)std::max<long long>(1, std::min<long long>(want, (long long)std::max(1, per_sm) * c->sm_count));
    }
    prof_begin(c, ST_DP);
    Geom ga = g;
    void* args[] = {&ga, &job};
    const cudaError_t le = cudaLaunchKernel(kf, dim3(grid), dim3(warps * 32), args, smem, c->stream);
    if (le != cudaSuccess) return cuda_fail(le, "k_dp launch", __FILE__, __LINE__);
    LAUNCH_CHECK(c);
    return FSMELD_OK;
}

// sort int64 keys (optionally with double values) in place through a scratch copy
static int sort_pairs_i64(fsmeld_ctx* c, long long* keys, double* vals, long long n) {
    if (n <= 1) return FSMELD_OK;
    long long* k2;
    double* v2 = nullptr;
    int r;
    if ((r = bufT(c, "sortk", (size_t)n, &k2))) return r;
    if (vals && (r = bufT(c, "sortv", (size_t)n, &v2))) return r;
    size_t tmp = 0;
    if (vals) FSM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, k2, vals, v2, (int)n, 0, 64, c->stream));
    else FSM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp, keys, k2, (int)n, 0, 64, c->stream));
    void* t;
    if ((r = buf(c, "sorttmp", tmp, &t))) return r;
    if (vals) FSM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, keys, k2, vals, v2, (int)n, 0, 64, c->stream));
    else FSM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(t, tmp, keys, k2, (int)n, 0, 64, c->stream));
    FSM_CUDA_TRY(cudaMemcpyAsync(keys, k2, sizeof(long long) * n, cudaMemcpyDeviceToDevice, c->stream));
    if (vals) FSM_CUDA_TRY(cudaMemcpyAsync(vals, v2, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    return FSMELD_OK;
}

// lexicographic (distance, index) order: index sort, then stable distance sort
static int sort_lex(fsmeld_ctx* c, long long* idx, double* dist, long long n) {
    int r;
    if ((r = sort_pairs_i64(c, idx, dist, n))) return r;
    if (n <= 1) return FSMELD_OK;
    long long* k2;
    double* d2;
    if ((r = bufT(c, "sortk", (size_t)n, &k2))) return r;
    if ((r = bufT(c, "sortv", (size_t)n, &d2))) return r;
    size_t tmp = 0;
    FSM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dist, d2, idx, k2, (int)n, 0, 64, c->stream));
    void* t;
    if ((r = buf(c, "sorttmp", tmp, &t))) return r;
    FSM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, dist, d2, idx, k2, (int)n, 0, 64, c->stream));
    FSM_CUDA_TRY(cudaMemcpyAsync(idx, k2, sizeof(long long) * n, cudaMemcpyDeviceToDevice, c->stream));
    FSM_CUDA_TRY(cudaMemcpyAsync(dist, d2, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    return FSMELD_OK;
}

struct QueryRun {
    const HostQuery* hq;
    int mode;  // 0 search, 1 cutoff, 2 exact
    double cutoff;
    int k;
    long long eb, ee;
    int64_t* out_idx;
    double* out_dist;
    int64_t cap;
    int64_t* out_count;
    fsmeld_counters* cnt;
    int64_t* seg_counts;
};

// The search after LB_IP: GLB on the survivor list `surv` (count at
// cnt[C_SURV]), the exact DP, ordered matches and counters.
static int search_tail(fsmeld_ctx* c, const Geom& g, const QueryDev& qd, const Stats& st, long long* surv,
                       unsigned long long* cnt, long long cap, long long* segc, const QueryRun& qr) {
    int r;
    unsigned long long h[C_N] = {0};
    fsmeld_counters out{};
    out.m_k = g.m_k;
    out.segments = g.forsize;
    out.tail = g.tsn % g.kml;
    long long* g2;
    double* g2t;
    if ((r = run_glb(c, g, qd, st, surv, cnt, cap, segc, &g2, &g2t))) return r;
    long long* oi;
    double* od;
    if ((r = bufT(c, "outi", (size_t)cap, &oi))) return r;
    if ((r = bufT(c, "outd", (size_t)cap, &od))) return r;
    DpJob dj{};
    dj.q = qd; dj.target = c->d_target; dj.MU = st.MU; dj.SIG = st.SIG;
    dj.lraw = st.Lraw; dj.uraw = st.Uraw;
    dj.list = g2; dj.list_s = g2t; dj.n_list = cnt + C_G2; dj.list_cap = cap; dj.mode = 0; dj.cutoff = qr.cutoff;
    dj.out_idx = oi; dj.out_dist = od; dj.n_out = cnt + C_OUT; dj.n_cells = cnt + C_CELLS; dj.out_cap = cap; dj.n_valid = nullptr;
    if ((r = run_dp(c, g, dj, (long long)c->sm_count * 16 * 128))) return r;
    FSM_CUDA_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const long long nout = (long long)h[C_OUT];
    if ((r = sort_pairs_i64(c, oi, nullptr, nout))) return r;
    const long long ncopy = std::min<long long>(nout, qr.cap);
    if (ncopy > 0)
        FSM_CUDA_TRY(cudaMemcpyAsync(qr.out_idx, oi, sizeof(long long) * ncopy, cudaMemcpyDeviceToHost, c->stream));
    if (qr.seg_counts && segc && g.forsize > 0)
        FSM_CUDA_TRY(cudaMemcpyAsync(qr.seg_counts, segc, sizeof(long long) * 3 * g.forsize,
                                     cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    out.valid = (long long)h[C_VALID];
    out.invalid = g.tsn - out.valid;
    out.after_lb = (long long)h[C_SURV];
    out.after_glb = (long long)h[C_G2];
    out.exact_evals = out.after_glb;
    out.matches = nout;
    out.dp_cells = (long long)h[C_CELLS];
    out.threshold = qr.cutoff;
    if (qr.out_count) *qr.out_count = nout;
    if (qr.cnt) *qr.cnt = out;
    return FSMELD_OK;
}

// The top-k after LB_IP: per-segment seeds by bound z (NaN: invalid), the
// k-th seed distance tau selected on the device, the LB filter, GLB and the
// exact DP at tau, ordered (distance, index) results and counters.
static int cutoff_tail(fsmeld_ctx* c, const Geom& g, const QueryDev& qd, const Stats& st, double* z,
                       unsigned long long* cnt, const QueryRun& qr) {
    int r;
    const long long cap = g.tsn;
    unsigned long long h[C_N] = {0};
    fsmeld_counters out{};
    out.m_k = g.m_k;
    out.segments = g.forsize;
    out.tail = g.tsn % g.kml;
    // seeds
    // seeds per segment: enough for k of them (2k over all segments), at most 32
    const int per_seg = (int)std::min<long long>(32, std::max<long long>(1, (2 * qr.k + g.S - 1) / g.S));
    const long long nslot = g.S * per_seg;
    long long* seeds;
    if ((r = bufT(c, "seeds", (size_t)nslot, &seeds))) return r;
    prof_begin(c, ST_SELECT);
    k_seed<<<(unsigned)std::min<long long>(g.S, (long long)c->sm_count * 8), 256, 0, c->stream>>>(
        g, z, st.SIG, per_seg, seeds, cnt + C_SEED, nslot);
    LAUNCH_CHECK(c);
    long long* si;
    double* sd;
    if ((r = bufT(c, "seedi", (size_t)nslot, &si))) return r;
    if ((r = bufT(c, "seedd", (size_t)nslot, &sd))) return r;
    // unused seed slots hold all-ones bit patterns, which sort after every distance
    FSM_CUDA_TRY(cudaMemsetAsync(sd, 0xff, sizeof(double) * (size_t)nslot, c->stream));
    DpJob sj{};
    sj.q = qd; sj.target = c->d_target; sj.MU = st.MU; sj.SIG = st.SIG;
    sj.list = seeds; sj.n_list = cnt + C_SEED; sj.list_cap = nslot; sj.mode = 1; sj.cutoff = DBL_MAX;
    sj.out_idx = si; sj.out_dist = sd; sj.n_out = cnt + C_SEEDOUT; sj.n_cells = cnt + C_CELLS; sj.out_cap = nslot;
    if ((r = run_dp(c, g, sj, nslot))) return r;
    // tau = k-th smallest seed distance, selected on the device: the rest of
    // the query reads it from device memory, so the host waits only once
    unsigned long long* sdk;
    double* tau_dev;
    if ((r = bufT(c, "seedsort", (size_t)nslot, &sdk))) return r;
    if ((r = bufT(c, "tau", 1, &tau_dev))) return r;
    {
        size_t tmp = 0;
        FSM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp, (const unsigned long long*)sd, sdk, (int)nslot, 0,
                                                    64, c->stream));
        void* tp;
        if ((r = buf(c, "seedsorttmp", tmp, &tp))) return r;
        FSM_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tp, tmp, (const unsigned long long*)sd, sdk, (int)nslot, 0, 64,
                                                    c->stream));
        k_tau<<<1, 32, 0, c->stream>>>(sdk, qr.k, nslot, tau_dev);
        LAUNCH_CHECK(c);
    }
    // filter, GLB and DP at tau
    long long* f1;
    if ((r = bufT(c, "surv", (size_t)cap, &f1))) return r;
    prof_begin(c, ST_SELECT);
    k_lb_filter<<<(unsigned)std::min<long long>((g.tsn + 255) / 256, (long long)c->sm_count * 16), 256, 0, c->stream>>>(
        g, z, st.SIG, tau_dev, qd.metric, f1, cnt + C_SURV, cap);
    LAUNCH_CHECK(c);
    QueryDev qt = qd;
    qt.cutoff = DBL_MAX;  // the GLB kernels read tau from device memory
    long long* g2;
    double* g2t;
    if ((r = run_glb(c, g, qt, st, f1, cnt, cap, nullptr, &g2, &g2t, tau_dev))) return r;
    long long* oi;
    double* od;
    if ((r = bufT(c, "outi", (size_t)cap, &oi))) return r;
    if ((r = bufT(c, "outd", (size_t)cap, &od))) return r;
    DpJob dj{};
    dj.q = qt; dj.target = c->d_target; dj.MU = st.MU; dj.SIG = st.SIG;
    dj.lraw = st.Lraw; dj.uraw = st.Uraw;
    dj.list = g2; dj.list_s = g2t; dj.n_list = cnt + C_G2; dj.list_cap = cap; dj.mode = 1; dj.cutoff = DBL_MAX;
    dj.cutoff_ptr = tau_dev;
    dj.out_idx = oi; dj.out_dist = od; dj.n_out = cnt + C_OUT; dj.n_cells = cnt + C_CELLS; dj.out_cap = cap;
    if ((r = run_dp(c, g, dj, (long long)c->sm_count * 16 * 128))) return r;
    FSM_CUDA_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const long long nvalid = (long long)h[C_VALID];
    const long long nseed = (long long)h[C_SEEDOUT];
    if (nvalid < qr.k) return fail(FSMELD_E_FEWER_K, "Fewer valid, non-excluded candidates than requested k.");
    const long long nout = (long long)h[C_OUT];
    if (nout < qr.k) return fail(FSMELD_E_FEWER_K, "Fewer valid, non-excluded candidates than requested k.");
    if ((r = sort_lex(c, oi, od, nout))) return r;
    FSM_CUDA_TRY(cudaMemcpyAsync(qr.out_idx, oi, sizeof(long long) * qr.k, cudaMemcpyDeviceToHost, c->stream));
    std::vector<double> kd(qr.k);
    FSM_CUDA_TRY(cudaMemcpyAsync(kd.data(), od, sizeof(double) * qr.k, cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (qr.out_dist) memcpy(qr.out_dist, kd.data(), sizeof(double) * qr.k);
    out.valid = nvalid;
    out.invalid = g.tsn - nvalid;
    out.after_lb = (long long)h[C_SURV];
    out.after_glb = (long long)h[C_G2];
    out.exact_evals = (long long)h[C_G2] + nseed;
    out.matches = qr.k;
    out.dp_cells = (long long)h[C_CELLS];
    out.threshold = kd[qr.k - 1];
    if (qr.out_count) *qr.out_count = qr.k;
    if (qr.cnt) *qr.cnt = out;
    return FSMELD_OK;
}

static int run_query(fsmeld_ctx* c, const QueryRun& qr, const Geom& g0, Stats& st, bool have_env) {
    int r;
    Geom g = g0;
    g.excl_b = (qr.eb >= 0 && qr.ee > qr.eb) ? qr.eb : -1;
    g.excl_e = (qr.eb >= 0 && qr.ee > qr.eb) ? qr.ee : -1;
    const HostQuery& hq = *qr.hq;
    QueryDev qd;
    if ((r = upload_query(c, hq, "query", &qd))) return r;
    unsigned long long* cnt;
    if ((r = bufT(c, "counters", C_N, &cnt))) return r;
    FSM_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, c->stream));
    const long long cap = g.tsn;
    unsigned long long h[C_N] = {0};
    fsmeld_counters out{};
    out.m_k = g.m_k;
    out.segments = g.forsize;
    out.tail = g.tsn % g.kml;

    if (qr.mode == 2) {  // exact: every valid window through the DP
        long long *oi;
        double* od;
        if ((r = bufT(c, "outi", (size_t)cap, &oi))) return r;
        if ((r = bufT(c, "outd", (size_t)cap, &od))) return r;
        qd.cutoff = qr.cutoff;
        DpJob dj{};
        dj.q = qd; dj.target = c->d_target; dj.MU = st.MU; dj.SIG = st.SIG;
        dj.list = nullptr; dj.n_windows = g.tsn; dj.mode = 0; dj.cutoff = qr.cutoff;
        dj.out_idx = oi; dj.out_dist = od; dj.n_out = cnt + C_OUT; dj.n_cells = cnt + C_CELLS; dj.out_cap = cap; dj.n_valid = cnt + C_VALID;
        if ((r = run_dp(c, g, dj, g.tsn))) return r;
        FSM_CUDA_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        const long long nout = (long long)h[C_OUT];
        if ((r = sort_pairs_i64(c, oi, od, nout))) return r;
        const long long ncopy = std::min<long long>(nout, qr.cap);
        if (ncopy > 0) {
            FSM_CUDA_TRY(cudaMemcpyAsync(qr.out_idx, oi, sizeof(long long) * ncopy, cudaMemcpyDeviceToHost, c->stream));
            if (qr.out_dist) FSM_CUDA_TRY(cudaMemcpyAsync(qr.out_dist, od, sizeof(double) * ncopy, cudaMemcpyDeviceToHost, c->stream));
        }
        FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        out.valid = (long long)h[C_VALID];
        out.invalid = g.tsn - out.valid;
        out.after_lb = out.after_glb = out.exact_evals = out.valid;
        out.matches = nout;
        out.dp_cells = (long long)h[C_CELLS];
        out.threshold = qr.cutoff;
        if (qr.out_count) *qr.out_count = nout;
        if (qr.cnt) *qr.cnt = out;
        return FSMELD_OK;
    }

    // thresholds
    double* thr;
    if ((r = bufT(c, "thr", (size_t)2 * g.S, &thr))) return r;
    std::vector<ThrJob> jobs(1);
    jobs[0].q = qd; jobs[0].Un = st.Un; jobs[0].Ln = st.Ln; jobs[0].thr = thr;
    if ((r = run_thr(c, g, jobs))) return r;
    (void)have_env;

    long long* segc = nullptr;
    if ((r = bufT(c, "segc", (size_t)3 * g.S, &segc))) return r;

    if (qr.mode == 0) {  // search
        long long* surv;
        if ((r = bufT(c, "surv", (size_t)cap, &surv))) return r;
        qd.cutoff = qr.cutoff;
        LbJob lj{};
        lj.q = qd; lj.Un = st.Un; lj.Ln = st.Ln; lj.thr = thr; lj.SIG = st.SIG;
        lj.zout = nullptr; lj.surv = surv; lj.surv_cap = cap; lj.nsurv = cnt + C_SURV;
        lj.nvalid = cnt + C_VALID; lj.segc = segc;
        if ((r = run_lbip(c, g, lj))) return r;
        return search_tail(c, g, qd, st, surv, cnt, cap, segc, qr);
    }

    // cutoff (top-k)
    double* z;
    if ((r = bufT(c, "zbuf", (size_t)g.S * g.kml, &z))) return r;
    LbJob lj{};
    lj.q = qd; lj.Un = st.Un; lj.Ln = st.Ln; lj.thr = thr; lj.SIG = st.SIG;
    lj.zout = z; lj.surv = nullptr; lj.nsurv = cnt + C_SURV; lj.nvalid = cnt + C_VALID; lj.segc = nullptr;
    if ((r = run_lbip(c, g, lj))) return r;
    return cutoff_tail(c, g, qd, st, z, cnt, qr);
}

// ------------------------------------------------ tensor-core LB_IP (groups)

// src/q_to_h.cpp:11-64 (lower) / 84-134 (upper), the penalties of k_lbip
static double host_q_to_h(int metric, bool upper, double x, double t, double C) {
    auto sq = [](double a, double b) { const double d = a - b; return d * d; };
    if (!upper) {
        switch (metric) {
            case MSM: return (x < t) ? ((t - x < C) ? t - x : C) : 0.0;
            case DTW: return (x < t) ? sq(t, x) : 0.0;
            case ERP: return (x < t) ? ((sq(x, t) > sq(x, C)) ? sq(x, C) : sq(x, t)) : 0.0;
            default: return (x < t - C) ? 1.0 : 0.0;
        }
    }
    switch (metric) {
        case MSM: return (x > t) ? ((x - t < C) ? x - t : C) : 0.0;
        case DTW: return (x > t) ? sq(x, t) : 0.0;
        case ERP: return (x > t) ? ((sq(x, t) > sq(x, C)) ? sq(x, C) : sq(x, t)) : 0.0;
        default: return (x > t + C) ? 1.0 : 0.0;
    }
}

// round a double to BF16 (through float); the split below measures the
// residual exactly, so the rounding direction does not matter
static uint16_t to_bf16(double v) {
    const float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan: truncate
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static double from_bf16(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

struct GemmChoice {
    double t_l = 0.0, t_u = 0.0;
    bool ok = false;
};

// The group's thresholds: the medians over the segments of the thresholds
// the reference's selection (k_threshold) picks for the group's first query.
static int gemm_thresholds(fsmeld_ctx* c, const Geom& g, const Stats& st, const HostQuery& rep, GemmChoice* out) {
    QueryDev qd;
    int r;
    if ((r = upload_query(c, rep, "query", &qd))) return r;
    double* thr;
    if ((r = bufT(c, "thr", (size_t)2 * g.S, &thr))) return r;
    std::vector<ThrJob> jobs(1);
    jobs[0].q = qd; jobs[0].Un = st.Un; jobs[0].Ln = st.Ln; jobs[0].thr = thr;
    if ((r = run_thr(c, g, jobs))) return r;
    std::vector<double> h(2 * (size_t)g.S);
    FSM_CUDA_TRY(cudaMemcpyAsync(h.data(), thr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::vector<double> tl, tu;
    for (long long s = 0; s < g.S; ++s) {
        if (std::isfinite(h[2 * s])) tl.push_back(h[2 * s]);
        if (std::isfinite(h[2 * s + 1])) tu.push_back(h[2 * s + 1]);
    }
    out->ok = !tl.empty() && !tu.empty();
    if (!out->ok) return FSMELD_OK;
    std::nth_element(tl.begin(), tl.begin() + tl.size() / 2, tl.end());
    std::nth_element(tu.begin(), tu.begin() + tu.size() / 2, tu.end());
    out->t_l = tl[tl.size() / 2];
    out->t_u = tu[tu.size() / 2];
    return FSMELD_OK;
}

// Searches (top-k queries) of equal (m, w), mode and metric with LB_IP as one
// tensor-core product per chunk of up to 128 (16) queries (k_lbgemm), then
// per query GLB and the exact DP (the top-k selection) as in run_query.
// Match sets and rankings are those of the per-query path (every bound is a
// lower bound); the LB_IP survivor counters differ (one shared threshold
// pair instead of one per segment and query).
static int get_worker(fsmeld_ctx* c, int i, fsmeld_ctx** out);
static void absorb_worker(fsmeld_ctx* c, fsmeld_ctx* wk);

static int run_search_gemm(fsmeld_ctx* c, const Geom& g0, Stats& st, const std::vector<const QueryRun*>& qs,
                           std::vector<int>* qstatus, double* zout_dev = nullptr, double* diag = nullptr,
                           bool parallel_tails = false) {
    int r;
    const int m = qs[0]->hq->m, w = qs[0]->hq->w, metric = qs[0]->hq->metric;
    GemmChoice th;
    if ((r = gemm_thresholds(c, g0, st, *qs[0]->hq, &th))) return r;
    if (!th.ok) return FSMELD_E_UNSUPPORTED;  // no finite threshold: the caller runs the per-query path
    const int kchunks = (m + kLbGemmKChunk - 1) / kLbGemmKChunk;
    const int kpad = kchunks * kLbGemmKChunk;
    const long long cap = g0.tsn;
    const long long words = (g0.tsn + 31) / 32 + 1;
    for (size_t q0 = 0; q0 < qs.size(); q0 += (qs[0]->mode == 1 ? 16 : 128)) {
        const bool topk = qs[0]->mode == 1;
        const int nq = (int)std::min<size_t>(topk ? 16 : 128, qs.size() - q0);
        const int NQ = nq <= 16 ? 16 : nq <= 32 ? 32 : nq <= 64 ? 64 : 128;
        // B operand and margins
        std::vector<uint16_t> B((size_t)kchunks * 6 * NQ * kLbGemmKChunk, 0);
        std::vector<double> marg(2 * (size_t)nq), cut(nq);
        std::vector<int> met(nq);
        std::vector<long long> eb(nq), ee(nq);
        const double nadd = 3.0 * kpad + 16.0;
        for (int i = 0; i < nq; ++i) {
            const QueryRun& qr = *qs[q0 + i];
            const HostQuery& hq = *qr.hq;
            for (int side = 0; side < 2; ++side) {
                const double t = side ? th.t_u : th.t_l;
                double S = 0.0, R = 0.0;
                for (int k = 0; k < m; ++k) {
                    const double hv = host_q_to_h(hq.metric, side == 1, hq.qn[k], t, hq.arg);
                    const uint16_t b0 = to_bf16(hv);
                    const double r1 = hv - from_bf16(b0);
                    const uint16_t b1 = to_bf16(r1);
                    const double r2 = r1 - from_bf16(b1);
                    const uint16_t b2 = to_bf16(r2);
                    const double r3 = r2 - from_bf16(b2);
                    S += std::fabs(from_bf16(b0)) + std::fabs(from_bf16(b1)) + std::fabs(from_bf16(b2));
                    R += std::fabs(r3);
                    const int ch = k / kLbGemmKChunk, kk = k % kLbGemmKChunk, kg = kk / 8, e = kk % 8;
                    const uint16_t bs[3] = {b0, b1, b2};
                    for (int sp = 0; sp < 3; ++sp) {
                        const size_t off = (size_t)ch * 6 * NQ * kLbGemmKChunk +   // chunk
                                           (size_t)(side * 3 + sp) * NQ * kLbGemmKChunk +  // sub-operand
                                           (size_t)kg * NQ * 8 + (size_t)(i / 8) * 64 + (size_t)(i % 8) * 8 + e;
                        B[off] = bs[sp];
                    }
                }
                // FP32 accumulation of nadd terms (truncating adds bound each error by
                // 2^-23 of the running magnitude <= S), times 4 for safety, plus the
                // split's residual and a relative 2^-40 for these host sums
                marg[2 * i + side] = (R + 4.0 * nadd * std::ldexp(S, -23)) * (1.0 + std::ldexp(1.0, -40)) + 1e-300;
            }
            cut[i] = topk ? DBL_MAX : qr.cutoff;
            met[i] = hq.metric;
            const bool ex = qr.eb >= 0 && qr.ee > qr.eb;
            eb[i] = ex ? qr.eb : -1;
            ee[i] = ex ? qr.ee : -1;
        }
        // upload
        uint16_t* dB;
        double *dM, *dC;
        int* dMet;
        long long *dE;
        unsigned* dbits;
        unsigned long long* dcnt;
        if ((r = bufT(c, "gemmB", B.size(), &dB))) return r;
        if ((r = bufT(c, "gemmM", 2 * (size_t)nq, &dM))) return r;
        if ((r = bufT(c, "gemmC", (size_t)nq, &dC))) return r;
        if ((r = bufT(c, "gemmMet", (size_t)nq, &dMet))) return r;
        if ((r = bufT(c, "gemmE", 2 * (size_t)nq, &dE))) return r;
        if ((r = bufT(c, "gemmBits", (size_t)nq * words, &dbits))) return r;
        if ((r = bufT(c, "gemmCnt", 2 * (size_t)nq + 2, &dcnt))) return r;
        std::vector<double> ml(nq), mu_(nq);
        for (int i = 0; i < nq; ++i) { ml[i] = marg[2 * i]; mu_[i] = marg[2 * i + 1]; }
        std::vector<long long> ebe(2 * (size_t)nq);
        for (int i = 0; i < nq; ++i) { ebe[i] = eb[i]; ebe[nq + i] = ee[i]; }
        FSM_CUDA_TRY(cudaMemcpyAsync(dB, B.data(), B.size() * 2, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemcpyAsync(dM, ml.data(), 8 * (size_t)nq, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemcpyAsync(dM + nq, mu_.data(), 8 * (size_t)nq, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemcpyAsync(dC, cut.data(), 8 * (size_t)nq, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemcpyAsync(dMet, met.data(), 4 * (size_t)nq, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemcpyAsync(dE, ebe.data(), 16 * (size_t)nq, cudaMemcpyHostToDevice, c->stream));
        FSM_CUDA_TRY(cudaMemsetAsync(dbits, 0, 4 * (size_t)nq * words, c->stream));
        FSM_CUDA_TRY(cudaMemsetAsync(dcnt, 0, 8 * (2 * (size_t)nq + 2), c->stream));
        GemmJob gj{};
        gj.Un = st.Un; gj.Ln = st.Ln; gj.SIG = st.SIG; gj.t_l = th.t_l; gj.t_u = th.t_u;
        gj.B = (const uint4*)dB; gj.m = m; gj.nq = nq; gj.kchunks = kchunks;
        gj.margin_l = dM; gj.margin_u = dM + nq; gj.metric = dMet; gj.cutoff = dC;
        gj.excl_b = dE; gj.excl_e = dE + nq;
        double* zq = zout_dev;
        if (topk && !zq && (r = bufT(c, "gemmZ", (size_t)nq * g0.S * g0.kml, &zq))) return r;
        gj.zout = zq; gj.zstride = g0.S * g0.kml;
        gj.bits = topk ? nullptr : dbits; gj.bit_words = words;
        gj.nsurv = dcnt; gj.nvalid = dcnt + nq; gj.err = (unsigned*)(dcnt + 2 * nq);
        // the group's window masks, once for all tiles
        {
            const int mw = gemm_mask_words(g0.m_k, g0.kml, m);
            unsigned* dmask;
            if ((r = bufT(c, "gemmMask", 2 * (size_t)g0.S * mw, &dmask))) return r;
            gj.mask_l = dmask;
            gj.mask_u = dmask + (size_t)g0.S * mw;
            gj.mask_words = mw;
            const long long warps = g0.S * (long long)mw;
            const unsigned mgrid = (unsigned)std::max<long long>(1, std::min<long long>((warps + 7) / 8,
                                                                                         (long long)c->sm_count * 16));
            prof_begin(c, ST_GEMM);
            k_gemm_masks<<<mgrid, 256, 0, c->stream>>>(g0, st.Ln, st.Un, th.t_l, th.t_u, dmask,
                                                       dmask + (size_t)g0.S * mw, mw);
            LAUNCH_CHECK(c);
        }
        const void* kf = lbgemm_kernel(NQ);
        const size_t smem = lbgemm_smem_bytes(NQ, m);
        if ((r = allow_smem(c, kf, smem))) return r;
        // resident CTAs per SM from the kernel's own resources: shared memory
        // (dynamic + static + the 1 KB the SM reserves per block), registers,
        // threads, and TMEM (512 columns per SM, 2 NQ (>= 32) per CTA)
        int per_sm = 0;
        {
            cudaFuncAttributes fa;
            FSM_CUDA_TRY(cudaFuncGetAttributes(&fa, kf));
            int smem_sm = 0, regs_sm = 0, thr_sm = 0;
            FSM_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device));
            FSM_CUDA_TRY(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, c->device));
            FSM_CUDA_TRY(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, c->device));
            const size_t per_block = smem + fa.sharedSizeBytes + 1024;
            per_sm = (int)std::min<size_t>((size_t)smem_sm / per_block, (size_t)thr_sm / kLbGemmThreads);
            if (fa.numRegs > 0) per_sm = std::min(per_sm, regs_sm / (fa.numRegs * kLbGemmThreads));
        }
        const int cols = std::max(32, 2 * NQ);
        per_sm = std::max(1, std::min(per_sm, 512 / cols));  // TMEM: 512 columns per SM
        const long long items = g0.S * ((g0.kml + 127) / 128);
        const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(items, (long long)per_sm * c->sm_count));
        Geom ga = g0;
        void* args[] = {&ga, &gj};
        prof_begin(c, ST_GEMM);
        const cudaError_t le = cudaLaunchKernel(kf, dim3(grid), dim3(kLbGemmThreads), args, smem, c->stream);
        if (le != cudaSuccess) return cuda_fail(le, "k_lbgemm launch", __FILE__, __LINE__);
        LAUNCH_CHECK(c);
        std::vector<unsigned long long> hc(2 * (size_t)nq + 2);
        FSM_CUDA_TRY(cudaMemcpyAsync(hc.data(), dcnt, 8 * hc.size(), cudaMemcpyDeviceToHost, c->stream));
        FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (hc[2 * nq] & 0xffffffffull) return fail(FSMELD_E_CUDA, "k_lbgemm: a bounded wait for the tensor cores gave up");
        if (zout_dev) {  // diagnostics: the bounds, thresholds and margins of the first query only
            if (diag) { diag[0] = th.t_l; diag[1] = th.t_u; diag[2] = marg[0]; diag[3] = marg[1]; }
            return FSMELD_OK;
        }
        // per query: survivor list from its bits (top-k: its bounds), then GLB +
        // DP, on the worker streams of a top-level context (the device work of
        // one query's tail is independent of the others')
        auto tail = [&](fsmeld_ctx* x, int i) -> int {
            const QueryRun& qr = *qs[q0 + i];
            Geom g = g0;
            g.excl_b = eb[i];
            g.excl_e = ee[i];
            QueryDev qd;
            int rr;
            if ((rr = upload_query(x, *qr.hq, "query", &qd))) return rr;
            qd.cutoff = qr.cutoff;
            unsigned long long* cnt;
            if ((rr = bufT(x, "counters", C_N, &cnt))) return rr;
            FSM_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, x->stream));
            FSM_CUDA_TRY(cudaMemcpyAsync(cnt + C_VALID, dcnt + nq + i, 8, cudaMemcpyDeviceToDevice, x->stream));
            if (topk) {
                if ((long long)hc[nq + i] < qr.k)
                    return fail(FSMELD_E_FEWER_K, "Fewer valid, non-excluded candidates than requested k.");
                return cutoff_tail(x, g, qd, st, zq + (size_t)i * g0.S * g0.kml, cnt, qr);
            }
            long long* surv;
            if ((rr = bufT(x, "surv", (size_t)cap, &surv))) return rr;
            prof_begin(x, ST_LBIP);
            k_bits_to_list<<<(unsigned)std::min<long long>((words + 255) / 256, (long long)x->sm_count * 8), 256, 0,
                             x->stream>>>(dbits + (size_t)i * words, words, surv, cap, cnt + C_SURV);
            LAUNCH_CHECK(x);
            return search_tail(x, g, qd, st, surv, cnt, cap, nullptr, qr);
        };
        const int conc = parallel_tails ? std::min(std::max(1, c->concurrency), nq) : 1;
        if (conc <= 1) {
            for (int i = 0; i < nq; ++i) {
                const int q = tail(c, i);
                (*qstatus)[q0 + i] = q;
                if (q == FSMELD_E_CUDA) return q;
            }
        } else {
            std::vector<fsmeld_ctx*> ws(conc);
            for (int t = 0; t < conc; ++t)
                if ((r = get_worker(c, t, &ws[t]))) return r;
            std::vector<std::string> errs(conc);
            std::vector<std::thread> th;
            for (int t = 0; t < conc; ++t) {
                th.emplace_back([&, t] {
                    cudaSetDevice(c->device);
                    for (int i = t; i < nq; i += conc) {
                        const int q = tail(ws[t], i);
                        (*qstatus)[q0 + i] = q;
                        if (q && errs[t].empty()) errs[t] = g_last_error;
                        if (q == FSMELD_E_CUDA) break;
                    }
                });
            }
            for (auto& x : th) x.join();
            for (int t = 0; t < conc; ++t) absorb_worker(c, ws[t]);
            for (int i = 0; i < nq; ++i)
                if ((*qstatus)[q0 + i]) {
                    for (auto& e : errs) if (!e.empty()) { g_last_error = e; break; }
                    if ((*qstatus)[q0 + i] == FSMELD_E_CUDA) return FSMELD_E_CUDA;
                }
        }
    }
    (void)w;
    (void)metric;
    return FSMELD_OK;
}

// One call over many queries: statistics per distinct m, envelopes per distinct (m, w).
// worker context i of c (created on first use): same device and target, its
// own stream and grow-only buffers
static int get_worker(fsmeld_ctx* c, int i, fsmeld_ctx** out) {
    while ((int)c->workers.size() <= i) {
        fsmeld_ctx* w = new fsmeld_ctx();
        w->parent = c;
        w->device = c->device;
        w->sm_count = c->sm_count;
        w->smem_optin = c->smem_optin;
        w->dp_exact = c->dp_exact;
        w->dp_form = c->dp_form;
        w->raw = c->raw;
        w->lb_form = c->lb_form;
        if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&w->ev0) != cudaSuccess || cudaEventCreate(&w->ev1) != cudaSuccess) {
            delete w;
            return fail(FSMELD_E_CUDA, "stream/event creation failed");
        }
        std::lock_guard<std::mutex> lk(ws_root(c)->ws_mu);
        c->workers.push_back(w);
    }
    fsmeld_ctx* w = c->workers[i];
    w->d_target = c->d_target;  // borrowed: the target may have been reloaded
    w->own_target = false;
    w->n = c->n;
    w->ws_limit = c->ws_limit;
    w->prof = c->prof;
    w->raw = c->raw;
    w->lb_form = c->lb_form;
    w->tune = c->tune;
    *out = w;
    return FSMELD_OK;
}


// Searches and top-k queries of one (m, w) group (order[gi..gj)) through the
// tensor-core LB_IP when it is selected: one product per mode and metric with
// at least two queries.  Marks the queries it ran in `done`.
static int group_gemm(fsmeld_ctx* c, const Geom& g, Stats& st, std::vector<QueryRun>& runs,
                      const std::vector<size_t>& order, size_t gi, size_t gj, std::vector<int>* status,
                      std::vector<char>* done, bool parallel_tails) {
    if (c->lb_form == 1) return FSMELD_OK;
    for (int mode = 0; mode <= 1; ++mode)
    for (int metric = DTW; metric <= MSM; ++metric) {
        std::vector<const QueryRun*> qs;
        std::vector<size_t> idx;
        for (size_t k = gi; k < gj; ++k) {
            const QueryRun& qr = runs[order[k]];
            if ((*done)[k]) continue;  // already answered
            if (qr.mode == mode && qr.hq->metric == metric) { qs.push_back(&qr); idx.push_back(k); }
        }
        if (qs.size() < 2) continue;
        if (c->lb_form == 0 && tuned(c, mode == 0 ? 1 : 2, metric, g.m_k, (int)qs.size()) != 2) continue;
        std::vector<int> qst(qs.size(), FSMELD_OK);
        const int r = run_search_gemm(c, g, st, qs, &qst, nullptr, nullptr, parallel_tails);
        if (r == FSMELD_E_UNSUPPORTED) continue;  // no usable threshold: per-query path
        for (size_t t = 0; t < idx.size(); ++t) {
            (*status)[order[idx[t]]] = r ? r : qst[t];
            (*done)[idx[t]] = 1;
        }
        if (r == FSMELD_E_CUDA) return r;
    }
    return FSMELD_OK;
}

// fold a worker's profile and launch counts into its parent context
static void absorb_worker(fsmeld_ctx* c, fsmeld_ctx* wk) {
    cudaStreamSynchronize(wk->stream);
    prof_collect(wk);
    for (int k = 0; k < ST_N; ++k) {
        c->stage_ms[k] += wk->stage_ms[k];
        c->stage_n[k] += wk->stage_n[k];
        wk->stage_ms[k] = 0.0;
        wk->stage_n[k] = 0;
    }
    c->launches += wk->launches;
    wk->launches = 0;
}

// Batches of many distinct query lengths: every distinct m is a task (its
// window statistics, then for each of its radii the envelopes, then the
// queries of each (m, w) group one after another), and the tasks run
// concurrently on the worker streams, each worker with its own statistics,
// envelopes and query buffers over the shared target.  Independent pipelines
// on several streams keep the GPU busy through the latency-bound phases of
// each (the running-sum statistics, the threshold replay, DP tails).
static int run_tasks_parallel(fsmeld_ctx* c, std::vector<QueryRun>& runs, const std::vector<size_t>& order,
                              const std::vector<std::pair<size_t, size_t>>& tasks, std::vector<int>* status) {
    const int conc = std::min<int>(std::max(1, c->concurrency), (int)tasks.size());
    std::vector<fsmeld_ctx*> ws(conc);
    int r;
    for (int t = 0; t < conc; ++t)
        if ((r = get_worker(c, t, &ws[t]))) return r;
    std::atomic<size_t> next{0};
    std::atomic<bool> cuda_dead{false};
    std::vector<std::string> errs(conc);
    // task ti on worker wk; retry: only the task's queries whose status is
    // FSMELD_E_NOMEM (the statistics and envelopes are computed again)
    auto run_task = [&](fsmeld_ctx* wk, size_t ti, bool retry, std::string& err) {
        const size_t lo = tasks[ti].first, hi = tasks[ti].second;
        auto wanted = [&](size_t k) { return !retry || (*status)[order[k]] == FSMELD_E_NOMEM; };
        auto mark = [&](size_t a, size_t b, int code) {
            for (size_t k = a; k < b; ++k)
                if (wanted(k)) (*status)[order[k]] = code;
            if (err.empty()) err = g_last_error;
            if (code == FSMELD_E_CUDA) cuda_dead = true;
        };
        Geom g{};
        Stats st;
        int q = make_geom(c->n, runs[order[lo]].hq->m, -1, -1, &g);
        g.raw = c->raw ? 1 : 0;
        if (!q) q = run_stats(wk, g, &st, "");
        if (q) { mark(lo, hi, q); return; }
        size_t gi = lo;
        while (gi < hi) {
            const int w = runs[order[gi]].hq->w;
            size_t gj = gi + 1;
            while (gj < hi && runs[order[gj]].hq->w == w) ++gj;
            bool need_env = false, any = false;
            for (size_t k = gi; k < gj; ++k) {
                need_env = need_env || runs[order[k]].mode != 2;
                any = any || wanted(k);
            }
            if (!any) { gi = gj; continue; }
            if (need_env && (q = run_env(wk, g, w, &st, ""))) { mark(gi, gj, q); gi = gj; continue; }
            std::vector<char> done(hi, 0);
            for (size_t k = gi; k < gj; ++k) done[k] = !wanted(k);
            if ((q = group_gemm(wk, g, st, runs, order, gi, gj, status, &done, false)) == FSMELD_E_CUDA) {
                mark(gi, gj, q);
                break;
            }
            for (size_t k = gi; k < gj; ++k) {
                if (done[k]) continue;
                q = run_query(wk, runs[order[k]], g, st, need_env);
                (*status)[order[k]] = q;
                if (q && err.empty()) err = g_last_error;
                if (q == FSMELD_E_CUDA) { cuda_dead = true; break; }
            }
            if (cuda_dead.load()) break;
            gi = gj;
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < conc; ++t) {
        th.emplace_back([&, t] {
            cudaSetDevice(c->device);
            for (;;) {
                const size_t ti = next.fetch_add(1);
                if (ti >= tasks.size() || cuda_dead.load()) break;
                run_task(ws[t], ti, false, errs[t]);
            }
        });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < conc; ++t) absorb_worker(c, ws[t]);
    // Queries refused for workspace while other tasks held theirs run again
    // one task at a time on the first worker, after every worker's buffers
    // are released; a query that still does not fit keeps FSMELD_E_NOMEM.
    bool nomem = false;
    for (size_t k = 0; k < order.size(); ++k) nomem = nomem || (*status)[order[k]] == FSMELD_E_NOMEM;
    if (nomem && !cuda_dead.load()) {
        // every task computes its own statistics on its worker, so nothing the
        // context itself holds is needed here either
        release_bufs(c);
        for (fsmeld_ctx* w : c->workers) release_bufs(w);
        for (size_t ti = 0; ti < tasks.size() && !cuda_dead.load(); ++ti) {
            bool any = false;
            for (size_t k = tasks[ti].first; k < tasks[ti].second; ++k)
                any = any || (*status)[order[k]] == FSMELD_E_NOMEM;
            if (!any) continue;
            errs[0].clear();
            run_task(ws[0], ti, true, errs[0]);
        }
        absorb_worker(c, ws[0]);
    }
    int first_err = FSMELD_OK;
    for (size_t k = 0; k < order.size() && !first_err; ++k) first_err = (*status)[order[k]];
    if (first_err)
        for (auto& e : errs) if (!e.empty()) { g_last_error = e; break; }
    return first_err;
}

// One call over many queries: statistics per distinct m, envelopes per distinct
// (m, w).  Several distinct lengths: the lengths run concurrently on worker
// streams (run_tasks_parallel).  One length: the queries of each (m, w) group
// run concurrently on worker streams (each query's pipeline is independent;
// its last step waits for its own stream, so the group is done on the device
// when its threads return).
int run_batch(fsmeld_ctx* c, std::vector<QueryRun>& runs, std::vector<int>* status) {
    status->assign(runs.size(), FSMELD_OK);
    std::vector<size_t> order(runs.size());
    for (size_t i = 0; i < runs.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (runs[a].hq->m != runs[b].hq->m) return runs[a].hq->m < runs[b].hq->m;
        return runs[a].hq->w < runs[b].hq->w;
    });
    {
        std::vector<std::pair<size_t, size_t>> tasks;  // [lo, hi) of order per distinct m
        for (size_t i = 0; i < order.size();) {
            size_t j = i + 1;
            while (j < order.size() && runs[order[j]].hq->m == runs[order[i]].hq->m) ++j;
            tasks.emplace_back(i, j);
            i = j;
        }
        if (tasks.size() > 1 && c->concurrency > 1) return run_tasks_parallel(c, runs, order, tasks, status);
    }
    if (!c->ev_ready) FSM_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_ready, cudaEventDisableTiming));
    int cur_m = -1, cur_w = -1;
    Stats st;
    Geom g{};
    bool have_env = false;
    int first_err = FSMELD_OK;
    size_t oi = 0;
    while (oi < order.size()) {
        const int m = runs[order[oi]].hq->m, w = runs[order[oi]].hq->w;
        size_t oj = oi + 1;
        while (oj < order.size() && runs[order[oj]].hq->m == m && runs[order[oj]].hq->w == w) ++oj;
        int r = FSMELD_OK;
        if (m != cur_m) {
            have_env = false;
            cur_w = -1;
            r = make_geom(c->n, m, -1, -1, &g);
            g.raw = c->raw ? 1 : 0;
            if (!r) r = run_stats(c, g, &st, "");
            cur_m = r ? -1 : m;
        }
        bool need_env = false;
        for (size_t k = oi; k < oj; ++k) need_env = need_env || runs[order[k]].mode != 2;
        if (!r && need_env && w != cur_w) {
            r = run_env(c, g, w, &st, "");
            cur_w = r ? -1 : w;
            have_env = !r;
        }
        if (r) {
            for (size_t k = oi; k < oj; ++k) (*status)[order[k]] = r;
            if (!first_err) first_err = r;
            if (r == FSMELD_E_CUDA) break;
            oi = oj;
            continue;
        }
        // searches through the tensor-core LB_IP (when selected), then the rest
        std::vector<char> done(oj, 0);
        if ((r = group_gemm(c, g, st, runs, order, oi, oj, status, &done, true)) == FSMELD_E_CUDA) return r;
        std::vector<size_t> rest;
        for (size_t k = oi; k < oj; ++k)
            if (!done[k]) rest.push_back(order[k]);
        for (size_t k = oi; k < oj; ++k)
            if (done[k] && (*status)[order[k]] && !first_err) first_err = (*status)[order[k]];
        const int nq = (int)rest.size();
        const int conc = std::min(std::max(1, c->concurrency), std::max(1, nq));
        if (conc <= 1) {
            for (size_t k : rest) {
                int q = run_query(c, runs[k], g, st, have_env);
                if (q == FSMELD_E_NOMEM && !c->workers.empty()) {
                    // the buffers an earlier batch's workers kept may be what is
                    // missing: release them and run the query again
                    for (fsmeld_ctx* w : c->workers) release_bufs(w);
                    q = run_query(c, runs[k], g, st, have_env);
                }
                (*status)[k] = q;
                if (q && !first_err) first_err = q;
                if (q == FSMELD_E_CUDA) break;
            }
        } else {
            FSM_CUDA_TRY(cudaEventRecord(c->ev_ready, c->stream));
            std::vector<fsmeld_ctx*> ws(conc);
            for (int t = 0; t < conc; ++t)
                if ((r = get_worker(c, t, &ws[t]))) return r;
            std::vector<std::string> errs(conc);
            std::vector<std::thread> th;
            for (int t = 0; t < conc; ++t) {
                th.emplace_back([&, t] {
                    cudaSetDevice(c->device);
                    fsmeld_ctx* wk = ws[t];
                    if (cudaStreamWaitEvent(wk->stream, c->ev_ready, 0) != cudaSuccess) {
                        for (int k = t; k < nq; k += conc) (*status)[rest[k]] = FSMELD_E_CUDA;
                        return;
                    }
                    for (int k = t; k < nq; k += conc) {
                        const int q = run_query(wk, runs[rest[k]], g, st, have_env);
                        (*status)[rest[k]] = q;
                        if (q && errs[t].empty()) errs[t] = g_last_error;
                        if (q == FSMELD_E_CUDA) break;
                    }
                });
            }
            for (auto& x : th) x.join();
            // a query that failed part-way may have left kernels queued: the next
            // group rewrites the shared statistics only after they are done
            for (int t = 0; t < conc; ++t) absorb_worker(c, ws[t]);
            // queries refused for workspace while the others held theirs run
            // again one after another on this context, the workers' buffers
            // released first; one that still does not fit keeps FSMELD_E_NOMEM
            bool nomem = false, dead = false;
            for (size_t k : rest) {
                nomem = nomem || (*status)[k] == FSMELD_E_NOMEM;
                dead = dead || (*status)[k] == FSMELD_E_CUDA;
            }
            if (nomem && !dead) {
                for (fsmeld_ctx* w : c->workers) release_bufs(w);
                for (size_t k : rest) {
                    if ((*status)[k] != FSMELD_E_NOMEM) continue;
                    const int q = run_query(c, runs[k], g, st, have_env);
                    (*status)[k] = q;
                    if (q) errs[0] = g_last_error;
                    if (q == FSMELD_E_CUDA) break;
                }
            }
            for (size_t k = oi; k < oj; ++k) {
                const int q = (*status)[order[k]];
                if (q && !first_err) {
                    first_err = q;
                    for (auto& e : errs) if (!e.empty()) { g_last_error = e; break; }
                }
            }
            if (first_err == FSMELD_E_CUDA) break;
        }
        if (first_err == FSMELD_E_CUDA) break;
        oi = oj;
    }
    return first_err;
}

}  // namespace fsm

// ====================================================================== C ABI

extern "C" {

static int open_common(int device, fsmeld_ctx** out) {
    fsmeld_ctx* c = new fsmeld_ctx();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaSetDevice", __FILE__, __LINE__); }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaGetDeviceProperties", __FILE__, __LINE__); }
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = (int)prop.sharedMemPerBlockOptin;
    if (const char* ex = getenv("FSMELD_DP_EXACT")) c->dp_exact = ex[0] == '1';
    if (const char* f = getenv("FSMELD_DP_FORM")) c->dp_form = !strcmp(f, "lane") ? 1 : !strcmp(f, "wave") ? 2 : 0;
    if (const char* f = getenv("FSMELD_LB_FORM")) c->lb_form = !strcmp(f, "fft") ? 1 : !strcmp(f, "gemm") ? 2 : 0;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        delete c;
        return fail(FSMELD_E_CUDA, "stream/event creation failed");
    }
    static std::once_flag w16;
    static int w16_status = 0;
    std::call_once(w16, [] { w16_status = lbip_set_w16(); });
    if (w16_status) { delete c; return w16_status; }
    *out = c;
    return FSMELD_OK;
}

int fsmeld_open(int device, const double* host_target, int64_t n, fsmeld_ctx** out) {
    if (!out || !host_target || n <= 0) return fail(FSMELD_E_ARG, "invalid target");
    fsmeld_ctx* c;
    int r = open_common(device, &c);
    if (r) return r;
    cudaError_t e = cudaMalloc(&c->d_target, sizeof(double) * n);
    if (e != cudaSuccess) { fsmeld_close(c); return cuda_fail(e, "cudaMalloc(target)", __FILE__, __LINE__); }
    e = cudaMemcpy(c->d_target, host_target, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { fsmeld_close(c); return cuda_fail(e, "cudaMemcpy(target)", __FILE__, __LINE__); }
    c->n = n;
    c->own_target = true;
    *out = c;
    return FSMELD_OK;
}

int fsmeld_load(fsmeld_ctx* c, const double* host_target, int64_t n) {
    if (!c || !host_target || n <= 0) return fail(FSMELD_E_ARG, "invalid target");
    FSM_CUDA_TRY(cudaSetDevice(c->device));
    if (!c->own_target || c->n < n) {
        if (c->own_target && c->d_target) cudaFree(c->d_target);
        c->d_target = nullptr;
        c->own_target = false;
        FSM_CUDA_TRY(cudaMalloc(&c->d_target, sizeof(double) * n));
        c->own_target = true;
    }
    FSM_CUDA_TRY(cudaMemcpyAsync(c->d_target, host_target, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->n = n;
    return FSMELD_OK;
}

int fsmeld_open_device(int device, const double* device_target, int64_t n, fsmeld_ctx** out) {
    if (!out || !device_target || n <= 0) return fail(FSMELD_E_ARG, "invalid target");
    fsmeld_ctx* c;
    int r = open_common(device, &c);
    if (r) return r;
    c->d_target = const_cast<double*>(device_target);
    c->n = n;
    c->own_target = false;
    *out = c;
    return FSMELD_OK;
}

int fsmeld_open_file(int device, const char* path, fsmeld_ctx** out) {
    FILE* f = path ? fopen(path, "rb") : nullptr;
    if (!f) return fail(FSMELD_E_IO, "Cannot open target file.");
    fseek(f, 0, SEEK_END);
    const long long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (bytes <= 0 || bytes % 8) { fclose(f); return fail(FSMELD_E_IO, "Target file size is not a multiple of 8 bytes."); }
    std::vector<double> t(bytes / 8);
    const size_t got = fread(t.data(), 8, t.size(), f);
    fclose(f);
    if (got != t.size()) return fail(FSMELD_E_IO, "Short read of target file.");
    return fsmeld_open(device, t.data(), (int64_t)t.size(), out);
}

int fsmeld_close(fsmeld_ctx* c) {
    if (!c) return FSMELD_OK;
    cudaSetDevice(c->device);
    for (auto* w : c->workers) fsmeld_close(w);  // borrowed target: not freed there
    c->workers.clear();
    if (c->ev_ready) cudaEventDestroy(c->ev_ready);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& kv : c->bufs) if (kv.second.p) cudaFree(kv.second.p);
    for (auto& kv : c->twiddles) cudaFree(kv.second);
    for (auto& r : c->pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : c->pool) cudaEventDestroy(e);
    if (c->own_target && c->d_target) cudaFree(c->d_target);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return FSMELD_OK;
}

int64_t fsmeld_target_length(const fsmeld_ctx* c) { return c ? c->n : 0; }

const double* fsmeld_target_device(const fsmeld_ctx* c) { return c ? c->d_target : nullptr; }

int fsmeld_set_normalization(fsmeld_ctx* c, int mode) {
    if (!c || (mode != FSMELD_NORM_ZSCORE && mode != FSMELD_NORM_RAW))
        return fail(FSMELD_E_ARG, "normalization mode must be FSMELD_NORM_ZSCORE or FSMELD_NORM_RAW");
    c->raw = mode == FSMELD_NORM_RAW;
    return FSMELD_OK;
}

int fsmeld_normalization(const fsmeld_ctx* c) { return (c && c->raw) ? FSMELD_NORM_RAW : FSMELD_NORM_ZSCORE; }

int fsmeld_set_tuning(fsmeld_ctx* c, const char* table) {
    if (!c) return fail(FSMELD_E_ARG, "null context");
    std::vector<fsmeld_ctx::TuneRule> rules;
    const char* p = table ? table : "";
    while (*p) {
        const char* e = strchr(p, '\n');
        std::string line(p, e ? (size_t)(e - p) : strlen(p));
        p = e ? e + 1 : p + strlen(p);
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        char kind[8], metric[8], choice[8];
        int mk = 0, lim = 0;
        if (sscanf(line.c_str(), "%7s %7s %d %d %7s", kind, metric, &mk, &lim, choice) != 5) {
            bool blank = true;
            for (char ch : line) blank = blank && (ch == ' ' || ch == '\t' || ch == '\r');
            if (blank) continue;
            return fail(FSMELD_E_ARG, "tuning table: a line is not 'kind metric m_k limit choice'");
        }
        fsmeld_ctx::TuneRule t{};
        t.kind = !strcmp(kind, "dp") ? 0 : !strcmp(kind, "lb") ? 1 : !strcmp(kind, "lbk") ? 2
               : !strcmp(kind, "dpx") ? 3 : -1;
        t.metric = !strcmp(metric, "dtw") ? DTW : !strcmp(metric, "erp") ? ERP : !strcmp(metric, "edr") ? EDR
                 : !strcmp(metric, "lcss") ? LCSS : !strcmp(metric, "msm") ? MSM : -1;
        t.m_k = mk;
        t.lim = lim;
        t.choice = (!strcmp(choice, "lane") || !strcmp(choice, "fft")) ? 1
                 : (!strcmp(choice, "wave") || !strcmp(choice, "gemm")) ? 2 : -1;
        if (t.kind < 0 || t.metric < 0 || t.choice < 0)
            return fail(FSMELD_E_ARG, "tuning table: unknown kind, metric or choice");
        rules.push_back(t);
    }
    c->tune = rules;
    return FSMELD_OK;
}

int fsmeld_set_lb_form(fsmeld_ctx* c, int form) {
    if (!c || form < FSMELD_LB_AUTO || form > FSMELD_LB_GEMM)
        return fail(FSMELD_E_ARG, "LB_IP form must be FSMELD_LB_AUTO, FSMELD_LB_FFT or FSMELD_LB_GEMM");
    c->lb_form = form;
    return FSMELD_OK;
}

int64_t fsmeld_workspace_bytes(fsmeld_ctx* c) {
    if (!c) return 0;
    fsmeld_ctx* root = ws_root(c);
    std::lock_guard<std::mutex> lk(root->ws_mu);
    return (int64_t)ws_family_total(c);
}

static void release_family(fsmeld_ctx* c) {
    for (fsmeld_ctx* w : c->workers) release_family(w);
    release_bufs(c);
}

int fsmeld_release_workspace(fsmeld_ctx* c) {
    if (!c) return fail(FSMELD_E_ARG, "null context");
    cudaSetDevice(c->device);
    release_family(c);
    return FSMELD_OK;
}

int fsmeld_set_concurrency(fsmeld_ctx* c, int queries) {
    if (!c || queries < 1 || queries > 16) return fail(FSMELD_E_ARG, "concurrency must be in [1, 16]");
    c->concurrency = queries;
    return FSMELD_OK;
}

const char* fsmeld_last_error(const fsmeld_ctx* c) {
    (void)c;
    return g_last_error.c_str();
}

const char* fsmeld_strerror(int s) {
    switch (s) {
        case FSMELD_OK: return "ok";
        case FSMELD_E_ARG: return "invalid argument";
        case FSMELD_E_CUDA: return "CUDA error";
        case FSMELD_E_NOMEM: return "out of device memory or workspace budget";
        case FSMELD_E_SHORT: return "target shorter than 2*m-1 points";
        case FSMELD_E_FEWER_K: return "fewer valid candidates than k";
        case FSMELD_E_UNSUPPORTED: return "unsupported configuration";
        case FSMELD_E_IO: return "I/O error";
        default: return "unknown error";
    }
}

int fsmeld_set_workspace_limit(fsmeld_ctx* c, int64_t bytes) {
    if (!c) return FSMELD_E_ARG;
    c->ws_limit = bytes;
    return FSMELD_OK;
}

int64_t fsmeld_kernel_launches(const fsmeld_ctx* c) { return c ? c->launches : 0; }

double fsmeld_last_call_ms(const fsmeld_ctx* c) { return c ? c->last_ms : 0.0; }

int fsmeld_set_profiling(fsmeld_ctx* c, int on) {
    if (!c) return FSMELD_E_ARG;
    prof_collect(c);
    c->prof = on != 0;
    for (int i = 0; i < ST_N; ++i) { c->stage_ms[i] = 0; c->stage_n[i] = 0; }
    return FSMELD_OK;
}

int fsmeld_stage_times(fsmeld_ctx* c, double* ms, int64_t* launches, int cap) {
    if (!c) return FSMELD_E_ARG;
    prof_collect(c);
    for (int i = 0; i < ST_N && i < cap; ++i) {
        if (ms) ms[i] = c->stage_ms[i];
        if (launches) launches[i] = c->stage_n[i];
    }
    return ST_N;
}

const char* fsmeld_stage_name(int i) { return (i >= 0 && i < ST_N) ? kStageNames[i] : ""; }

static int single(fsmeld_ctx* c, int mode, const double* query, int m, double cutoff, int k, int metric,
                  int w, double arg, int64_t eb, int64_t ee, int64_t* out_idx, double* out_dist,
                  int64_t cap, int64_t* out_count, fsmeld_counters* counters, int64_t* seg_counts) {
    if (!c || !query) return fail(FSMELD_E_ARG, "null context or query");
    if (mode != 1 && !(std::isfinite(cutoff) && cutoff >= 0))
        return fail(FSMELD_E_ARG, "cutoff must be finite and non-negative.");
    if (mode == 1 && (k < 1 || (long long)k > c->n - m + 1))
        return fail(FSMELD_E_ARG, "k exceeds the candidate count or supported integer range.");
    if (eb >= 0 || ee >= 0) {
        if (eb < 0 || ee <= eb) return fail(FSMELD_E_ARG, "Exclusion requires 0 <= start < end.");
    }
    FSM_CUDA_TRY(cudaSetDevice(c->device));
    HostQuery hq;
    int r = prepare_query(query, m, metric, w, arg, &hq, c->raw);
    if (r) return r;
    QueryRun qr{&hq, mode, cutoff, k, eb, ee, out_idx, out_dist, cap, out_count, counters, seg_counts};
    std::vector<QueryRun> runs{qr};
    std::vector<int> st;
    cudaEventRecord(c->ev0, c->stream);
    r = run_batch(c, runs, &st);
    cudaEventRecord(c->ev1, c->stream);
    cudaEventSynchronize(c->ev1);
    prof_collect(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    if (counters) counters->device_ms = ms;
    return r;
}

int fsmeld_search(fsmeld_ctx* c, const double* query, int m, double cutoff, int metric, int w, double arg,
                  int64_t eb, int64_t ee, int64_t* out_idx, int64_t cap, int64_t* out_count,
                  fsmeld_counters* counters, int64_t* seg_counts) {
    return single(c, 0, query, m, cutoff, 0, metric, w, arg, eb, ee, out_idx, nullptr, cap, out_count,
                  counters, seg_counts);
}

int fsmeld_cutoff(fsmeld_ctx* c, const double* query, int m, int k, int metric, int w, double arg,
                  int64_t eb, int64_t ee, int64_t* out_idx, double* out_dist, fsmeld_counters* counters) {
    int64_t cnt = 0;
    return single(c, 1, query, m, 0.0, k, metric, w, arg, eb, ee, out_idx, out_dist, k, &cnt, counters,
                  nullptr);
}

int fsmeld_exact(fsmeld_ctx* c, const double* query, int m, double cutoff, int metric, int w, double arg,
                 int64_t eb, int64_t ee, int64_t* out_idx, double* out_dist, int64_t cap,
                 int64_t* out_count, fsmeld_counters* counters) {
    return single(c, 2, query, m, cutoff, 0, metric, w, arg, eb, ee, out_idx, out_dist, cap, out_count,
                  counters, nullptr);
}

int fsmeld_batch(fsmeld_ctx* c, int mode, const fsmeld_query* qs, int nq, fsmeld_result* res) {
    if (!c || !qs || !res || nq < 0 || mode < 0 || mode > 2) return fail(FSMELD_E_ARG, "invalid batch");
    FSM_CUDA_TRY(cudaSetDevice(c->device));
    std::vector<HostQuery> hqs(nq);
    std::vector<QueryRun> runs;
    std::vector<int> map;
    for (int i = 0; i < nq; ++i) {
        res[i].count = 0;
        res[i].status = prepare_query(qs[i].query, qs[i].m, qs[i].metric, qs[i].w, qs[i].arg, &hqs[i], c->raw);
        if (res[i].status) continue;
        if (mode == 1 && (qs[i].k < 1 || (long long)qs[i].k > c->n - qs[i].m + 1)) { res[i].status = FSMELD_E_ARG; continue; }
        if (mode != 1 && !(std::isfinite(qs[i].cutoff) && qs[i].cutoff >= 0)) { res[i].status = FSMELD_E_ARG; continue; }
        if (mode == 1 && res[i].capacity < qs[i].k) { res[i].status = FSMELD_E_ARG; continue; }
        QueryRun qr{&hqs[i], mode, qs[i].cutoff, qs[i].k, qs[i].exclude_begin, qs[i].exclude_end,
                    res[i].idx, res[i].dist, res[i].capacity, &res[i].count, &res[i].counters,
                    res[i].seg_counts};
        runs.push_back(qr);
        map.push_back(i);
    }
    std::vector<int> st;
    cudaEventRecord(c->ev0, c->stream);
    int r = run_batch(c, runs, &st);
    cudaEventRecord(c->ev1, c->stream);
    cudaEventSynchronize(c->ev1);
    prof_collect(c);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    for (size_t j = 0; j < map.size(); ++j) {
        res[map[j]].status = st[j];
        res[map[j]].counters.device_ms = ms;
    }
    int first = r;
    for (int i = 0; i < nq && !first; ++i) first = res[i].status;
    return first;
}

int64_t fsmeld_inspect(fsmeld_ctx* c, const double* query, int m, int metric, int w, double arg, int what,
                       double* out, int64_t cap) {
    if (!c || !query || what < 0 || what > 7) return fail(FSMELD_E_ARG, "invalid inspect request");
    FSM_CUDA_TRY(cudaSetDevice(c->device));
    HostQuery hq;
    int r = prepare_query(query, m, metric, w, arg, &hq, c->raw);
    if (r) return r;
    Geom g;
    if ((r = make_geom(c->n, m, -1, -1, &g))) return r;
    g.raw = c->raw ? 1 : 0;
    Stats st;
    if ((r = run_stats(c, g, &st, ""))) return r;
    const double* src = nullptr;
    long long count = 0;
    if (what <= 1) {
        src = what == 0 ? st.MU : st.SIG;
        count = g.S * g.kml;
    } else {
        if ((r = run_env(c, g, w, &st, ""))) return r;
        if (what <= 3) {
            src = what == 2 ? st.Un : st.Ln;
            count = g.S * g.m_k;
        } else {
            QueryDev qd;
            if ((r = upload_query(c, hq, "query", &qd))) return r;
            double* thr;
            if ((r = bufT(c, "thr", (size_t)2 * g.S, &thr))) return r;
            std::vector<ThrJob> jobs(1);
            jobs[0].q = qd; jobs[0].Un = st.Un; jobs[0].Ln = st.Ln; jobs[0].thr = thr;
            if ((r = run_thr(c, g, jobs))) return r;
            if (what == 4) {
                src = thr;
                count = 2 * g.S;
            } else if (what >= 6) {
                // the tensor-core LB_IP of this query alone (its thresholds' medians)
                double* z;
                if ((r = bufT(c, "zbuf", (size_t)g.S * g.kml, &z))) return r;
                QueryRun qr{&hq, 0, 0.0, 0, -1, -1, nullptr, nullptr, 0, nullptr, nullptr, nullptr};
                std::vector<const QueryRun*> qs{&qr};
                std::vector<int> qst(1);
                double diag[4] = {0, 0, 0, 0};
                qr.cutoff = 1e300;
                if ((r = run_search_gemm(c, g, st, qs, &qst, z, diag))) return r;
                if (what == 6) {
                    src = z;
                    count = g.S * g.kml;
                } else {
                    const long long nd = std::min<long long>(4, cap);
                    if (out && nd > 0) memcpy(out, diag, sizeof(double) * nd);
                    return 4;
                }
            } else {
                unsigned long long* cnt;
                if ((r = bufT(c, "counters", C_N, &cnt))) return r;
                FSM_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * C_N, c->stream));
                double* z;
                if ((r = bufT(c, "zbuf", (size_t)g.S * g.kml, &z))) return r;
                LbJob lj{};
                lj.q = qd; lj.Un = st.Un; lj.Ln = st.Ln; lj.thr = thr; lj.SIG = st.SIG;
                lj.zout = z; lj.nsurv = cnt + C_SURV; lj.nvalid = cnt + C_VALID;
                if ((r = run_lbip(c, g, lj))) return r;
                src = z;
                count = g.S * g.kml;
            }
        }
    }
    const long long ncopy = std::min<long long>(count, cap);
    if (out && ncopy > 0)
        FSM_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * ncopy, cudaMemcpyDeviceToHost, c->stream));
    FSM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return count;
}

}  // extern "C"
