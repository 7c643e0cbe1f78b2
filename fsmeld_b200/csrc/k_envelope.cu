// Per-segment envelopes: min/max of window means and sigmas over trailing
// windows (src/lower_upper_lemire.cpp:94-126), the centred radius-w envelope
// of the segment (src/lower_upper_lemire.cpp:8-44), and the conservative
// z-normalised envelopes U_normal, L_normal (src/lb_normalize.cpp:9-32).
//
// The reference uses monotone deques.  Their outputs have a closed form that
// this kernel computes in parallel:
//  * with no NaN in the window: the window minimum (maximum); among equal
//    values the deque keeps the most recent one, which only matters for the
//    sign of a zero (window means and sigmas are never -0; a target's -0 and
//    +0 give the same U_normal / L_normal comparisons and penalties);
//  * with a NaN in the window: a NaN blocks every pop behind it, so the
//    front is the extremum of the points before the first NaN, or NaN when
//    the window starts with NaN.
// NaN-free windows by doubling: after pass k, M[i] = min(x[i .. i+2^k-1]);
// a window [a, b] of length L with 2^k <= L < 2^(k+1) is the union of the
// runs of length 2^k at its two ends, min(M[a], M[b-2^k+1]), so each output
// is taken right after the pass of its own level (full windows, and the
// shorter windows at the segment's edges alike).  Every pass is one min and
// one max per element with a block barrier, no scans.  Windows that contain
// a NaN (detected with a NaN prefix count) are evaluated directly from their
// start.
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

// Padded index of the per-segment arrays: one spare slot after every 8
// elements, so the blocked walks of the scans (thread t on elements
// [8t, 8t+8)) fall on distinct banks.
__device__ __forceinline__ int px(int i) { return i + (i >> 3); }
// slots for indices 0..n (the NaN prefix count reads index n)
__host__ __device__ inline int env_pad_len(int n) { return n + (n >> 3) + 2; }

template <int T>
struct EnvTemp {
    typename cub::BlockScan<int, T>::TempStorage ic;
};

struct EnvWork {
    double *raw, *Pmn, *Pmx, *Smn, *Smx;
    int* ncnt;  // NaN prefix counts [n + 1]
};

// Sliding min/max of src[0..n) for nout windows; CENTRED selects
// [o-w, o+w] (lemire) versus the trailing [o-m+1, o] (min_max_window), both
// clipped to [0, n-1].  Work arrays: raw copy, two ping-pong pairs (Pmn/Pmx,
// Smn/Smx) for the doubling passes, NaN prefix counts.
template <int T, int OPT, bool CENTRED>
__device__ void minmax_phase(const double* __restrict__ src, int n, int par, int nout,
                             const EnvWork& wk, EnvTemp<T>& tmp, double (&omn)[OPT],
                             double (&omx)[OPT]) {
    const int t = threadIdx.x;
    int local_nan = 0;
    for (int i = t; i < n; i += T) {
        const double v = src[i];
        wk.raw[px(i)] = v;
        wk.Pmn[px(i)] = v;
        wk.Pmx[px(i)] = v;
        local_nan |= isnan(v) ? 1 : 0;
    }
    const int any_nan = __syncthreads_or(local_nan);
    if (any_nan) {
        const int c = (n + T - 1) / T;
        const int lo = t * c, hi = min(n, lo + c);
        int cnt = 0;
        for (int i = lo; i < hi; ++i) cnt += isnan(wk.raw[px(i)]) ? 1 : 0;
        int off;
        cub::BlockScan<int, T>(tmp.ic).ExclusiveSum(cnt, off);
        for (int i = lo; i < hi; ++i) {
            wk.ncnt[px(i)] = off;
            off += isnan(wk.raw[px(i)]) ? 1 : 0;
        }
        if (hi == n && lo < hi) wk.ncnt[px(n)] = off;  // the chunk holding n-1 closes the count
        __syncthreads();
    }
    // each output's window [ws, we] (recomputed where needed, to keep the
    // per-thread state to the outputs themselves)
    auto window = [&](int o, int& ws, int& we) {
        if (CENTRED) { ws = max(0, o - par); we = min(n - 1, o + par); }
        else { ws = max(0, o - par + 1); we = min(o, n - 1); }
    };
    auto has_nan = [&](int ws, int we) {
        return any_nan && (wk.ncnt[px(we + 1)] - wk.ncnt[px(ws)] > 0);
    };
#pragma unroll
    for (int k = 0; k < OPT; ++k) { omn[k] = 0.0; omx[k] = 0.0; }
    // the deepest level any window needs: the full window length, clipped to n
    const int maxlen = CENTRED ? min(n, 2 * par + 1) : min(n, par);
    const int levels = 31 - __clz(max(1, maxlen));
    double* An = wk.Pmn;
    double* Ax = wk.Pmx;
    double* Bn = wk.Smn;
    double* Bx = wk.Smx;
    for (int lv = 0; lv <= levels; ++lv) {
        if (lv > 0) {
            const int s = 1 << (lv - 1);
            for (int i = t; i < n; i += T) {
                const bool in = i + s < n;
                const double a0 = An[px(i)], x0 = Ax[px(i)];
                const double a1 = in ? An[px(i + s)] : a0, x1 = in ? Ax[px(i + s)] : x0;
                Bn[px(i)] = (a1 < a0) ? a1 : a0;
                Bx[px(i)] = (x1 > x0) ? x1 : x0;
            }
            __syncthreads();
            double* tn = An; An = Bn; Bn = tn;
            double* tx = Ax; Ax = Bx; Bx = tx;
        }
        // outputs whose window length has this level: the two end runs
#pragma unroll
        for (int k = 0; k < OPT; ++k) {
            const int o = t + k * T;
            if (o >= nout) continue;
            int ws, we;
            window(o, ws, we);
            if (31 - __clz(we - ws + 1) != lv || has_nan(ws, we)) continue;
            const int b2 = we - (1 << lv) + 1;
            const double a0 = An[px(ws)], a1 = An[px(b2)];
            const double x0 = Ax[px(ws)], x1 = Ax[px(b2)];
            omn[k] = (a1 < a0) ? a1 : a0;
            omx[k] = (x1 > x0) ? x1 : x0;
        }
    }
    // windows holding a NaN: the deque's front from the window's start
#pragma unroll
    for (int k = 0; k < OPT; ++k) {
        const int o = t + k * T;
        if (!any_nan || o >= nout) continue;
        int ws, we;
        window(o, ws, we);
        if (!has_nan(ws, we)) continue;
        double a = wk.raw[px(ws)];
        double vmn = a, vmx = a;
        if (!isnan(a)) {
            for (int i = ws + 1; i <= we; ++i) {
                const double v = wk.raw[px(i)];
                if (isnan(v)) break;
                vmn = (v <= vmn) ? v : vmn;
                vmx = (v >= vmx) ? v : vmx;
            }
        }
        omn[k] = vmn;
        omx[k] = vmx;
    }
    __syncthreads();
}

}  // namespace

template <int T, int OPT, bool GW>
__global__ void __launch_bounds__(T) k_envelope(const double* __restrict__ target,
                                                const double* __restrict__ MU,
                                                const double* __restrict__ SIG, Geom g, int w,
                                                double* __restrict__ Un, double* __restrict__ Ln,
                                                double* gwork, long long slot_stride) {
    extern __shared__ __align__(16) unsigned char env_smem[];
    __shared__ EnvTemp<T> tmp;
    const int mk = g.m_k, kml = g.kml, m = g.m;
    double* base = GW ? gwork + (long long)blockIdx.x * slot_stride : (double*)env_smem;
    EnvWork wk;
    const int pk = env_pad_len(mk);  // padded length of each array
    wk.raw = base;
    wk.Pmn = base + pk;
    wk.Pmx = base + 2 * pk;
    wk.Smn = base + 3 * pk;
    wk.Smx = base + 4 * pk;
    wk.ncnt = (int*)(base + 5 * pk);
    for (long long s = blockIdx.x; s < g.S; s += gridDim.x) {
        double simn[OPT], simx[OPT], mumn[OPT], mumx[OPT], lmn[OPT], lmx[OPT];
        minmax_phase<T, OPT, false>(SIG + s * kml, kml, m, mk, wk, tmp, simn, simx);
        minmax_phase<T, OPT, false>(MU + s * kml, kml, m, mk, wk, tmp, mumn, mumx);
        minmax_phase<T, OPT, true>(target + g.off(s), mk, w, mk, wk, tmp, lmn, lmx);
#pragma unroll
        for (int k = 0; k < OPT; ++k) {
            const int o = threadIdx.x + k * T;
            if (o < mk) {
                const double nu = dsub(lmx[k], mumn[k]);
                const double un = (nu >= 0) ? ddiv(nu, simn[k]) : ddiv(nu, simx[k]);
                const double nl = dsub(lmn[k], mumx[k]);
                const double ln = (nl <= 0) ? ddiv(nl, simn[k]) : ddiv(nl, simx[k]);
                Un[s * mk + o] = un;
                Ln[s * mk + o] = ln;
            }
        }
    }
}

size_t envelope_work_bytes(int m_k) { return (size_t)env_pad_len(m_k) * (5 * sizeof(double) + sizeof(int)) + 16; }

#define FSM_ENV_INST(T, OPT)                                                                          \
    template __global__ void k_envelope<T, OPT, false>(const double*, const double*, const double*,  \
                                                       Geom, int, double*, double*, double*, long long); \
    template __global__ void k_envelope<T, OPT, true>(const double*, const double*, const double*,   \
                                                      Geom, int, double*, double*, double*, long long);
FSM_ENV_INST(256, 4)
FSM_ENV_INST(512, 4)
FSM_ENV_INST(1024, 4)
FSM_ENV_INST(1024, 8)
FSM_ENV_INST(1024, 16)

}  // namespace fsm
