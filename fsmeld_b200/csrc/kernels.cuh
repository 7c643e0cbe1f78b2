// Kernel entry points and their job descriptors.
#pragma once

#include "common.cuh"

namespace fsm {

struct ThrJob {
    QueryDev q;
    const double* Un;  // [S][m_k]
    const double* Ln;
    double* thr;       // [S][2]: (t_l, t_u) per segment
};

struct LbJob {
    QueryDev q;
    const double* Un;
    const double* Ln;
    const double* thr;
    const double* SIG;          // window sigmas [S][kml] (validity)
    double* zout;               // optional: LB per window [S][kml] (NaN if invalid)
    long long* surv;            // optional: LB survivors (global window index)
    long long surv_cap;
    unsigned long long* nsurv;
    unsigned long long* nvalid; // valid, non-excluded windows
    long long* segc;            // optional: per segment (valid, after LB, after GLB)
    unsigned char* gwork;       // global scratch when the FFT buffers exceed shared memory
    long long slot_stride;
};

struct GlbJob {
    QueryDev q;
    const double* target;
    const double* lraw;         // forward windows min / max(t[p .. p+w]) of the raw target
    const double* uraw;
    const double* MU;
    const double* SIG;
    const long long* in;
    const double* in_b;         // stage 2 input: boundary terms
    const double* in_t;         // stage 2 input: T->Q sums (LCSS: T->Q reward)
    const unsigned long long* n_in;
    long long in_cap;
    long long* out;
    double* out_b;
    double* out_t;
    unsigned long long* n_out;
    long long out_cap;
    long long* segc;
    const double* cutoff_ptr;   // when set: the cutoff in device memory (read at kernel start)
};

struct DpJob {
    QueryDev q;
    const double* target;
    const double* lraw;         // forward windows of the raw target (cascading abandon terms)
    const double* uraw;
    const double* MU;
    const double* SIG;
    const long long* list;      // candidates, or null for windows [0, n_windows)
    const double* list_s;       // optional: GLB Q->T sum per candidate (cascading abandon)
    const unsigned long long* n_list;
    long long list_cap;
    long long n_windows;
    int mode;                   // 0: keep dist <= cutoff; 1: keep every finite dist
    double cutoff;
    long long* out_idx;
    double* out_dist;
    unsigned long long* n_out;
    long long out_cap;
    unsigned long long* n_valid;
    unsigned long long* next;   // work counter (zeroed before the launch)
    double* gwork;              // global band scratch when shared memory is too small
    int force_exact;            // every candidate in the DP's exact boundary mode
    unsigned long long* n_cells;  // band cells computed (optional)
    const double* cutoff_ptr;   // when set: the cutoff in device memory (read at kernel start)
};

// LB_IP of a group of queries of equal (m, w) with shared thresholds as one
// tensor-core product (k_lbgemm); per-query arrays are indexed by query
struct GemmJob {
    const double* Un;           // [S][m_k]
    const double* Ln;
    const double* SIG;          // [S][kml]
    double t_l, t_u;            // the group's thresholds
    const uint4* B;             // BF16 penalty operand, per K chunk [side][split][NQ x 64] (operand layout)
    int m, nq, kchunks;
    const double* margin_l;     // rounding-error margins of the lower / upper inner products
    const double* margin_u;
    const int* metric;
    const double* cutoff;
    const long long* excl_b;    // exclusion interval per query (-1: none)
    const long long* excl_e;
    double* zout;               // optional: bound per window, [q][zstride]
    long long zstride;
    unsigned* bits;             // survivors per query: bit g of bits[q * bit_words ...] (zeroed by the caller)
    long long bit_words;
    unsigned long long* nsurv;  // [nq]
    unsigned long long* nvalid; // [nq]
    unsigned int* err;          // set when a bounded wait gave up
    const unsigned* mask_l;     // window masks g of the group (k_gemm_masks): [S][mask_words] 32-bit words,
    const unsigned* mask_u;     // bit p of a segment = position p (0 at and past m_k)
    int mask_words;
};
template <int NQ>
__global__ void k_lbgemm(Geom g, GemmJob job);
// bit p of segment s: Ln[s][p] >= t_l (mask_l), Un[s][p] <= t_u (mask_u); 0 for p >= m_k
__global__ void k_gemm_masks(Geom g, const double* __restrict__ Ln, const double* __restrict__ Un, double t_l,
                             double t_u, unsigned* __restrict__ mask_l, unsigned* __restrict__ mask_u, int words);
// 32-bit mask words per segment: the positions every tile of the segment reads
int gemm_mask_words(int m_k, int kml, int m);
const void* lbgemm_kernel(int nq_pad);  // NQ in {16, 32, 64, 128}
__global__ void k_bits_to_list(const unsigned* __restrict__ bits, long long words, long long* __restrict__ out,
                               long long cap, unsigned long long* __restrict__ n);
size_t lbgemm_smem_bytes(int nq_pad, int m);
constexpr int kLbGemmThreads = 128;
constexpr int kLbGemmKChunk = 64;

// window statistics: one block per 32 segments, warp 0 runs the running sums
// and warps 1-3 derive mean and sigma
constexpr int kMvmeanThreads = 128;
__global__ void k_mvmean(const double* __restrict__ target, Geom g, double* __restrict__ mu,
                         double* __restrict__ sig);
template <int T, int OPT, bool GW>
__global__ void k_envelope(const double* __restrict__ target, const double* __restrict__ MU,
                           const double* __restrict__ SIG, Geom g, int w, double* __restrict__ Un,
                           double* __restrict__ Ln, double* gwork, long long slot_stride);
template <int T, int IPT, bool GW>
__global__ void k_threshold(Geom g, const ThrJob* __restrict__ jobs, unsigned char* gwork,
                            long long slot_stride);
template <int T, bool GW>
__global__ void k_lbip(Geom g, LbJob job, const double2* __restrict__ W, int P, int logP);
template <int METRIC>
__global__ void k_glb_tq(Geom g, GlbJob job);
template <int METRIC>
__global__ void k_glb_qt(Geom g, GlbJob job);
// forward windows min/max(t[p .. p+w]) by doubling in shared memory, kFwdTile
// outputs per CTA and tile
constexpr int kFwdThreads = 256;
constexpr int kFwdTile = 2048;
__global__ void k_fwd_env(const double* __restrict__ t, long long n, int w, double* __restrict__ lo,
                          double* __restrict__ up);
size_t fwd_env_smem_bytes(int w);
template <int METRIC, bool GW>
__global__ void k_dp(Geom g, DpJob job);
// the DP kernel for a metric, with its band in shared memory or in job.gwork
const void* dp_kernel(int metric, bool gw);
// wide-band DP: one warp per candidate, one anti-diagonal per step, the band
// in registers (K chunks of 64 band offsets per warp, 2w+1 <= 64 K)
template <int METRIC, int K>
__global__ void k_dpw(Geom g, DpJob job);
constexpr int kDpwThreads = 128;
constexpr int kDpwMaxChunks = 8;  // w <= 255
// the wavefront kernel for (metric, w), or null when the band is too wide
const void* dpw_kernel(int metric, int w);
// shared memory: the query plus, per warp, its candidate and the row-block
// suffix sums of the abandon bound
__host__ __device__ size_t dpw_warp_doubles(int m);
size_t dpw_smem_bytes(int m, int warps);
__global__ void k_lb_filter(Geom g, const double* __restrict__ z, const double* __restrict__ SIG,
                            const double* __restrict__ cutoff, int metric, long long* out,
                            unsigned long long* n_out, long long cap);
__global__ void k_tau(const unsigned long long* __restrict__ sorted, long long k, long long n, double* tau);
__global__ void k_seed(Geom g, const double* __restrict__ z, const double* __restrict__ SIG, int per_seg,
                       long long* out, unsigned long long* n_out, long long cap);

// raise a kernel's dynamic shared-memory limit on a device to at least `bytes`
// (process-wide, never lowered; the device must be current)
cudaError_t raise_smem_limit(const void* kernel, int device, size_t bytes);

size_t mvmean_smem_bytes();
size_t envelope_work_bytes(int m_k);
size_t threshold_work_bytes(int cap_items, size_t sort_tmp, int m);
template <int T, int IPT>
size_t threshold_sort_tmp_bytes();
size_t lbip_smem_bytes(int P, int m_k, int m, int metric);
int lbip_set_w16();
// DP block size (2 warps: the per-warp band scratch sets the occupancy)
constexpr int kDpThreads = 64;
// DP per-warp scratch: band row (2w+1 cells + one out-of-band cell) and the
// candidate ring (power of two >= 2w+2 points), 32 lanes each
__host__ __device__ int dp_ring(int w);
__host__ __device__ size_t dp_warp_doubles(int w);

}  // namespace fsm
