// Exact scan that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a serving loop
// whose device memory is owned by another allocator (a framework's caching
// pool, a memory-capped tenant), or code that must never allocate while a
// request is in flight.  fsmeld_exact_noalloc gives them the `exact` scan
// (every valid window through the banded elastic DP, matches at or below the
// cutoff) with caller-owned device inputs and outputs and a caller stream.
// Its scratch -- window statistics, the DP's work and match counters and
// match list, and an ordering buffer -- lives in one file-scope
// `static __device__` array of kScratchBytes (12 MiB), which every GPU that
// loads the library holds until the process exits.
//
// Limits: at most FSMELD_NOALLOC_MAX_WINDOWS windows (n - m + 1) and
// m <= FSMELD_NOALLOC_MAX_M per call; the DP band and candidate ring of the
// lane-per-candidate DP must fit shared memory with the same 4 KB margin the
// allocating path keeps, which on a 227 KB opt-in device means w <= 94.
// Larger requests are rejected with FSMELD_E_ARG and a message.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current (a host-side reference to
// the array is only a stand-in, not a device address) and keeps it for the
// life of the process, so the entry point must not be used on a device after
// cudaDeviceReset in the same process.  Make that first call before any stream
// capture.  The call is synchronous (it reads the match count back and waits
// for its stream), so it must never be made while its stream is capturing.
// The caller's current device is restored on return.  Every call shares the
// one array and leaves its contents behind; each call clears what must start
// at zero.  Calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on the array: serialise them.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/fsmeld_cuda.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.cuh"

namespace fsm {

namespace {

constexpr long long kMaxWin = FSMELD_NOALLOC_MAX_WINDOWS;
constexpr int kMaxM = FSMELD_NOALLOC_MAX_M;
constexpr long long kMaxKml = 8LL * kMaxM;  // kml < m_k <= 2^ceil(log2 8m) <= 8 * kMaxM
// scratch layout (bytes, 256-aligned pieces)
constexpr size_t kOffQuery = 0;                                        // qn [kMaxM]
constexpr size_t kOffCnt = kOffQuery + sizeof(double) * kMaxM;         // counters [8]
constexpr size_t kOffMu = kOffCnt + 256;                               // window means
constexpr size_t kStatN = (size_t)(kMaxWin + kMaxKml);                 // [S][kml] covers tail padding
constexpr size_t kOffSig = kOffMu + sizeof(double) * kStatN;           // window sigmas
constexpr size_t kOffLi = kOffSig + sizeof(double) * kStatN;           // DP match indices
constexpr size_t kOffLd = kOffLi + sizeof(long long) * kMaxWin;        // DP match distances
constexpr size_t kOffWin = kOffLd + sizeof(double) * kMaxWin;          // distance per window
constexpr size_t kNeed = kOffWin + sizeof(double) * kMaxWin;
constexpr size_t kScratchBytes = 12u << 20;
static_assert(kNeed <= kScratchBytes, "scratch layout exceeds the static array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[256] = {nullptr};

thread_local double t_qn[kMaxM];

int fail(int code, const char* msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

// mark each match's distance at its window (NaN elsewhere)
__global__ void k_noalloc_scatter(const long long* __restrict__ idx, const double* __restrict__ dist,
                                  const unsigned long long* __restrict__ n_out, double* __restrict__ win) {
    const unsigned long long n = *n_out;
    for (unsigned long long o = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; o < n;
         o += (unsigned long long)gridDim.x * blockDim.x)
        win[idx[o]] = dist[o];
}

// one block: the marked windows in index order into the caller's buffers
__global__ void __launch_bounds__(1024) k_noalloc_compact(const double* __restrict__ win, long long nwin,
                                                          long long* __restrict__ out_idx,
                                                          double* __restrict__ out_dist, long long cap,
                                                          unsigned long long* __restrict__ total) {
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const long long c = (nwin + 1023) / 1024;
    const long long lo = t * c, hi = lo + c < nwin ? lo + c : nwin;
    long long cnt = 0;
    for (long long i = lo; i < hi; ++i) cnt += isnan(win[i]) ? 0 : 1;
    part[t] = cnt;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const long long v = (t >= d) ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long o = part[t] - cnt;
    for (long long i = lo; i < hi; ++i) {
        const double d = win[i];
        if (isnan(d)) continue;
        if (o < cap) {
            out_idx[o] = i;
            out_dist[o] = d;
        }
        ++o;
    }
    if (t == 1023) *total = (unsigned long long)part[1023];
}

}  // namespace fsm

using namespace fsm;

static int exact_noalloc(int device, const double* device_target, int64_t n, const double* host_query, int m,
                         int metric, int w, double arg, double cutoff, int64_t* device_out_idx,
                         double* device_out_dist, int64_t capacity, int64_t* host_out_count, void* stream) {
    if (!device_target || !host_query || !device_out_idx || !device_out_dist || !host_out_count || capacity < 0)
        return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: null pointer or negative capacity");
    if (device < 0 || device >= 256) return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: bad device index");
    if (m < 2 || m > kMaxM) return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: m must be in [2, FSMELD_NOALLOC_MAX_M]");
    if (w < 0 || w >= m) return fail(FSMELD_E_ARG, "w must satisfy 0 <= w < m.");
    if (metric < DTW || metric > MSM) return fail(FSMELD_E_ARG, "Unsupported metric.");
    if (!std::isfinite(arg) || ((metric == EDR || metric == LCSS || metric == MSM) && arg < 0))
        return fail(FSMELD_E_ARG, "Matching tolerance and MSM cost must be non-negative.");
    if (!(std::isfinite(cutoff) && cutoff >= 0)) return fail(FSMELD_E_ARG, "cutoff must be finite and non-negative.");
    if (n < 2LL * m - 1) return fail(FSMELD_E_SHORT, "Target must contain at least 2*m-1 values.");
    if (n - m + 1 > kMaxWin)
        return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: more windows than FSMELD_NOALLOC_MAX_WINDOWS");
    // query z-normalisation as src/fsmeld.cpp:622-639, into a fixed per-thread buffer
    double ex = 0, ex2 = 0;
    for (int i = 0; i < m; ++i) {
        if (!std::isfinite(host_query[i])) return fail(FSMELD_E_ARG, "Query must begin with m finite numeric values.");
        ex += host_query[i];
        ex2 += host_query[i] * host_query[i];
    }
    const double mean = ex / m;
    double sd = ex2 / m;
    sd = std::sqrt(sd - mean * mean);
    if (!std::isfinite(sd) || sd <= 1e-12)
        return fail(FSMELD_E_ARG, "Query cannot be z-normalized: non-finite or near-zero standard deviation.");
    for (int i = 0; i < m; ++i) t_qn[i] = (host_query[i] - mean) / sd;

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice", __FILE__, __LINE__);
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_ptr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
            g_scratch_ptr[device] = (unsigned char*)p;
        }
        base = g_scratch_ptr[device];
    }
    Geom g;
    g.n = n;
    g.m = m;
    g.m_k = macro_length(m, n);
    g.kml = g.m_k - m + 1;
    g.inv_kml = 1.0 / (double)g.kml;
    g.tsn = n - m + 1;
    g.forsize = g.tsn / g.kml;
    const long long tail = g.tsn % g.kml;
    g.tail_lo = (int)(g.kml - tail);
    g.S = g.forsize + (tail > 0 ? 1 : 0);
    g.excl_b = g.excl_e = -1;
    if ((size_t)(g.S * g.kml) > kStatN) return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: statistics exceed scratch");

    cudaStream_t st = (cudaStream_t)stream;
    double* qn = (double*)(base + kOffQuery);
    unsigned long long* cnt = (unsigned long long*)(base + kOffCnt);
    double* MU = (double*)(base + kOffMu);
    double* SIG = (double*)(base + kOffSig);
    long long* li = (long long*)(base + kOffLi);
    double* ld = (double*)(base + kOffLd);
    double* win = (double*)(base + kOffWin);

    // band rows in shared memory only (no global spill buffer on this path)
    const int warps = kDpThreads / 32;
    const size_t smem = sizeof(double) * dp_warp_doubles(w) * warps;
    int dev_optin = 0;
    if ((e = cudaDeviceGetAttribute(&dev_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    if (smem > (size_t)dev_optin - 4096)
        return fail(FSMELD_E_ARG, "fsmeld_exact_noalloc: band 2w+1 too wide for shared memory on this path");
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);

    if ((e = cudaMemcpyAsync(qn, t_qn, sizeof(double) * m, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(query)", __FILE__, __LINE__);
    if ((e = cudaMemsetAsync(cnt, 0, 256, st)) != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync", __FILE__, __LINE__);
    if ((e = cudaMemsetAsync(win, 0xff, sizeof(double) * g.tsn, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync", __FILE__, __LINE__);

    const size_t sm_stats = mvmean_smem_bytes();
    if ((e = raise_smem_limit((const void*)k_mvmean, device, sm_stats)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    k_mvmean<<<(unsigned)((g.S + 31) / 32), kMvmeanThreads, sm_stats, st>>>(device_target, g, MU, SIG);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_mvmean", __FILE__, __LINE__);

    QueryDev qd{};
    qd.m = m; qd.w = w; qd.metric = metric; qd.arg = arg; qd.cutoff = cutoff; qd.qn = qn;
    DpJob dj{};
    dj.q = qd; dj.target = device_target; dj.MU = MU; dj.SIG = SIG;
    dj.list = nullptr; dj.n_windows = g.tsn; dj.mode = 0; dj.cutoff = cutoff;
    dj.out_idx = li; dj.out_dist = ld; dj.n_out = cnt + 0; dj.out_cap = kMaxWin;
    dj.n_valid = cnt + 1; dj.next = cnt + 2; dj.gwork = nullptr;
    const void* kf = dp_kernel(metric, false);
    if ((e = raise_smem_limit(kf, device, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, warps * 32, smem)) != cudaSuccess)
        return cuda_fail(e, "occupancy", __FILE__, __LINE__);
    const unsigned grid = (unsigned)std::max(1, per_sm) * (unsigned)sms;
    {
        void* args[] = {&g, &dj};
        if ((e = cudaLaunchKernel(kf, dim3(grid), dim3(warps * 32), args, smem, st)) != cudaSuccess)
            return cuda_fail(e, "k_dp", __FILE__, __LINE__);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_dp", __FILE__, __LINE__);
    k_noalloc_scatter<<<(unsigned)sms * 4, 256, 0, st>>>(li, ld, cnt + 0, win);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_noalloc_scatter", __FILE__, __LINE__);
    k_noalloc_compact<<<1, 1024, 0, st>>>(win, g.tsn, (long long*)device_out_idx, device_out_dist, capacity, cnt + 3);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_noalloc_compact", __FILE__, __LINE__);
    unsigned long long total = 0;
    if ((e = cudaMemcpyAsync(&total, cnt + 3, sizeof(total), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(count)", __FILE__, __LINE__);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    *host_out_count = (int64_t)total;
    return FSMELD_OK;
}

extern "C" int fsmeld_exact_noalloc(int device, const double* device_target, int64_t n, const double* host_query,
                                    int m, int metric, int w, double arg, double cutoff, int64_t* device_out_idx,
                                    double* device_out_dist, int64_t capacity, int64_t* host_out_count,
                                    void* stream) {
    int prev = -1;
    const cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
    const int r = exact_noalloc(device, device_target, n, host_query, m, metric, w, arg, cutoff, device_out_idx,
                                device_out_dist, capacity, host_out_count, stream);
    if (prev != device) cudaSetDevice(prev);
    return r;
}
