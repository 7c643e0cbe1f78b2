// Per-segment envelopes: min/max of window means and sigmas over trailing
// windows (src/lower_upper_lemire.cpp:94-126), the centred radius-w envelope
// of the segment (src/lower_upper_lemire.cpp:8-44), and the conservative
// z-normalised envelopes U_normal, L_normal (src/lb_normalize.cpp:9-32).
//
// The reference uses monotone deques.  Their outputs have a closed form that
// this kernel computes in parallel:
//  * with no NaN in the window: the window minimum (maximum); among equal
//    values the most recent one (the deque pops older elements that compare
//    >= / <= the newcomer), which only matters for the sign of a zero;
//  * with a NaN in the window: a NaN blocks every pop behind it, so the
//    front is the extremum of the points before the first NaN, or NaN when
//    the window starts with NaN.
// NaN-free windows use van Herk / Gil-Werman: block-local prefix and suffix
// extrema (blocks of the window length B) computed by a block-segmented scan,
// then one combine per output.  Windows that contain a NaN (detected with a
// NaN prefix count) are evaluated directly from their start.
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

struct MMCarry {
    double mn, mx;
    int fl;  // bit 0: chunk contains a block start; bit 1: chunk non-empty
};

// combine(a = earlier in scan order, b = later); FWD scans run old -> new,
// REV scans run new -> old; ties keep the newer element.
template <bool REV>
struct MMComb {
    __device__ MMCarry operator()(const MMCarry& a, const MMCarry& b) const {
        MMCarry r;
        r.fl = a.fl | b.fl;
        if (b.fl & 1) { r.mn = b.mn; r.mx = b.mx; return r; }
        if (!(b.fl & 2)) { r.mn = a.mn; r.mx = a.mx; return r; }
        if (!(a.fl & 2)) { r.mn = b.mn; r.mx = b.mx; return r; }
        if (!REV) {  // a older, b newer
            r.mn = (b.mn <= a.mn) ? b.mn : a.mn;
            r.mx = (b.mx >= a.mx) ? b.mx : a.mx;
        } else {     // a newer, b older
            r.mn = (a.mn <= b.mn) ? a.mn : b.mn;
            r.mx = (a.mx >= b.mx) ? a.mx : b.mx;
        }
        return r;
    }
};

// Padded index of the per-segment arrays: one spare slot after every 8
// elements, so the blocked walks of the scans (thread t on elements
// [8t, 8t+8)) fall on distinct banks.
__device__ __forceinline__ int px(int i) { return i + (i >> 3); }
// slots for indices 0..n (the NaN prefix count reads index n)
__host__ __device__ inline int env_pad_len(int n) { return n + (n >> 3) + 2; }

template <int T>
struct EnvTemp {
    union {
        typename cub::BlockScan<MMCarry, T>::TempStorage mm;
        typename cub::BlockScan<int, T>::TempStorage ic;
    };
};

// Block-segmented inclusive min/max scan, in place, blocks [kB, (k+1)B).
// REV = false: prefix within blocks; REV = true: suffix within blocks.
template <int T, bool REV>
__device__ void seg_scan(double* mn, double* mx, int n, int B, EnvTemp<T>& tmp) {
    const int t = threadIdx.x;
    const int c = (n + T - 1) / T;
    const int lo = t * c, hi = min(n, lo + c);
    double rmn = 0.0, rmx = 0.0;
    int fl = 0, first_start = hi;
    for (int u = lo; u < hi; ++u) {
        const int i = REV ? n - 1 - u : u;
        const bool start = REV ? (u == 0 || (i % B) == B - 1) : ((i % B) == 0);
        const double xmn = mn[px(i)], xmx = mx[px(i)];
        if (start || !(fl & 2)) {
            rmn = xmn;
            rmx = xmx;
            if (start && !(fl & 1)) first_start = u;
            fl |= 2 | (start ? 1 : 0);
        } else if (!REV) {
            rmn = (xmn <= rmn) ? xmn : rmn;
            rmx = (xmx >= rmx) ? xmx : rmx;
        } else {
            rmn = (rmn <= xmn) ? rmn : xmn;
            rmx = (rmx >= xmx) ? rmx : xmx;
        }
        mn[px(i)] = rmn;
        mx[px(i)] = rmx;
    }
    MMCarry mine{rmn, rmx, fl}, cin;
    cub::BlockScan<MMCarry, T>(tmp.mm).ExclusiveScan(mine, cin, MMComb<REV>());
    __syncthreads();
    if (t > 0 && (cin.fl & 2)) {
        const int e = min(hi, first_start);
        for (int u = lo; u < e; ++u) {
            const int i = REV ? n - 1 - u : u;
            if (!REV) {
                mn[px(i)] = (mn[px(i)] <= cin.mn) ? mn[px(i)] : cin.mn;
                mx[px(i)] = (mx[px(i)] >= cin.mx) ? mx[px(i)] : cin.mx;
            } else {
                mn[px(i)] = (cin.mn <= mn[px(i)]) ? cin.mn : mn[px(i)];
                mx[px(i)] = (cin.mx >= mx[px(i)]) ? cin.mx : mx[px(i)];
            }
        }
    }
    __syncthreads();
}

struct EnvWork {
    double *raw, *Pmn, *Pmx, *Smn, *Smx;
    int* ncnt;  // NaN prefix counts [n + 1]
};

// Sliding min/max of src[0..n) for nout windows; CENTRED selects
// [o-w, o+w] (lemire) versus the trailing [o-m+1, o] (min_max_window).
template <int T, int OPT, bool CENTRED>
__device__ void minmax_phase(const double* __restrict__ src, int n, int par, int nout,
                             const EnvWork& wk, EnvTemp<T>& tmp, double (&omn)[OPT],
                             double (&omx)[OPT]) {
    const int t = threadIdx.x;
    const int B = CENTRED ? 2 * par + 1 : par;
    int local_nan = 0;
    for (int i = t; i < n; i += T) {
        const double v = src[i];
        wk.raw[px(i)] = v;
        wk.Pmn[px(i)] = v; wk.Pmx[px(i)] = v; wk.Smn[px(i)] = v; wk.Smx[px(i)] = v;
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
    }
    __syncthreads();
    seg_scan<T, false>(wk.Pmn, wk.Pmx, n, B, tmp);
    seg_scan<T, true>(wk.Smn, wk.Smx, n, B, tmp);
#pragma unroll
    for (int k = 0; k < OPT; ++k) {
        const int o = t + k * T;
        double vmn = 0.0, vmx = 0.0;
        if (o < nout) {
            int ws, we;
            if (CENTRED) { ws = max(0, o - par); we = min(n - 1, o + par); }
            else { ws = max(0, o - par + 1); we = min(o, n - 1); }
            const bool nanwin = any_nan && (wk.ncnt[px(we + 1)] - wk.ncnt[px(ws)] > 0);
            if (nanwin) {
                double a = wk.raw[px(ws)];
                if (isnan(a)) {
                    vmn = a; vmx = a;
                } else {
                    vmn = a; vmx = a;
                    for (int i = ws + 1; i <= we; ++i) {
                        const double v = wk.raw[px(i)];
                        if (isnan(v)) break;
                        vmn = (v <= vmn) ? v : vmn;
                        vmx = (v >= vmx) ? v : vmx;
                    }
                }
            } else if (ws % B == 0) {
                vmn = wk.Pmn[px(we)]; vmx = wk.Pmx[px(we)];
            } else if (ws / B == we / B) {
                vmn = wk.Smn[px(ws)]; vmx = wk.Smx[px(ws)];
            } else {
                const double pm = wk.Pmn[px(we)], sm = wk.Smn[px(ws)];
                const double pxv = wk.Pmx[px(we)], sx = wk.Smx[px(ws)];
                vmn = (pm <= sm) ? pm : sm;
                vmx = (pxv >= sx) ? pxv : sx;
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
FSM_ENV_INST(128, 8)
FSM_ENV_INST(256, 8)
FSM_ENV_INST(512, 8)
FSM_ENV_INST(1024, 8)
FSM_ENV_INST(1024, 16)

}  // namespace fsm
