// LB_IP threshold selection per macro segment and side
// (src/find_t_lp.cpp: find_tl_lp_dtw 218-287, find_tl_lp 288-398,
//  find_tl_lp_erp 510-582, find_tu_lp_erp 583-654, find_tu_lp_dtw 655-724,
//  find_tu_lp 726-825; dispatch src/fsmeld.cpp:778-790).
//
// The reference: run-length dedup of the envelope core U/L_normal[m-1 ..
// m_k-m] (consecutive equal values only), sort, then one sequential sweep
// that moves pointers over the sorted query, updates running power sums m_p
// and a penalty sum C, and scores LB[i] = h(t_i) * g_i; the argmax gives t.
//
// Here one CTA handles one (segment, side):
//  1. dedup with a block scan, sort runs with a stable block merge sort on
//     an order-preserving 64-bit key (total order: value, NaN last, ties by
//     position through the sort's stability);
//  2. every pointer move of the sweep becomes an op with the sweep step at
//     which it fires (a binary search over the sorted values); ops are
//     ordered by (step, stream, rank) -- the order the reference's loops
//     perform them in;
//  3. the ops are replayed in that order, so m_p and C carry the reference's
//     rounding bit for bit: lane j of warp 0 owns accumulator j (m_0..m_2, C)
//     and adds each op's operand, pre-signed for it, recording the state
//     after each op;
//  4. every candidate reads its state, scores LB in parallel, and a block
//     reduction takes the first maximum (NaN at index 0 wins, as in
//     findMaxIndex, src/find_t_lp.cpp:206-216).
// ERP's priority queues pop equal keys in an order the C++ library leaves
// to its heap layout; here equal keys pop by query index.  The threshold is
// the same unless two candidates' scores tie to the last bit.
#include <climits>
#include <cub/block/block_merge_sort.cuh>
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

constexpr int kNever = INT_MAX;

// Order-preserving key of a double: ascending values map to ascending keys,
// -0 and +0 to one key (they compare equal), NaN to the largest key (sorted
// last); desc reverses the order of the non-NaN values.
__device__ __forceinline__ unsigned long long order_key(double x, int desc) {
    if (isnan(x)) return ~0ull;
    const unsigned long long u = (unsigned long long)__double_as_longlong(x == 0.0 ? 0.0 : x);
    const unsigned long long k = (u >> 63) ? ~u : (u | 0x8000000000000000ull);
    return desc ? ~k : k;
}

struct KeyLess {
    __device__ __forceinline__ bool operator()(const unsigned long long& a, const unsigned long long& b) const {
        return a < b;
    }
};

struct ArgMax {
    double v;
    int i;
    int ok;  // 0 for NaN scores (never selected unless at index 0)
};
struct ArgMaxOp {
    __device__ ArgMax operator()(const ArgMax& a, const ArgMax& b) const {
        if (!a.ok) return b;
        if (!b.ok) return a;
        if (a.v > b.v) return a;
        if (b.v > a.v) return b;
        return (a.i <= b.i) ? a : b;
    }
};

enum Cmp { LE, LT, GE, GT };

// first i in [0, n) with tv[i] (cmp) x, or kNever; tv is monotone so the
// predicate is false..false true..true
__device__ __forceinline__ int first_step(const double* tv, int n, Cmp c, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const double t = tv[mid];
        bool p;
        switch (c) {
            case LE: p = t <= x; break;
            case LT: p = t < x; break;
            case GE: p = t >= x; break;
            default: p = t > x; break;
        }
        if (p) hi = mid; else lo = mid + 1;
    }
    return lo < n ? lo : kNever;
}

// prefix length of an index-ordered table whose keys satisfy pred (monotone)
template <typename F>
__device__ __forceinline__ int prefix_count(int n, F pred) {
    int lo = 0, hi = n;
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (pred(mid)) lo = mid + 1; else hi = mid; }
    return lo;
}

__device__ __forceinline__ double f_p(double mp0, double mp1, double mp2, int p, double t) {
    // src/find_t_lp.cpp:187-199 (p == 0 only occurs for EDR/LCSS, which return 0)
    if (p == 0) return 0.0;
    if (p == 1) return dsub(mp1, dmul(mp0, t));
    return dadd(dsub(mp2, dmul(dmul(mp1, t), 2.0)), dmul(mp0, dmul(t, t)));
}

// Stream plan of one (metric, side): op element, step, payload kind.
struct Plan {
    int kind;      // 0 DTW, 1 general (MSM, EDR, LCSS), 2 ERP
    int upper;
    int idx1, idx2, kA0, kB0;
    int nA, nB;
    int p;
};

}  // namespace

// Block working set: the runs (values and starts), region X (the sort's temp
// storage, then the sorted values and counts) and region Z (the sweep: op
// steps, op order, operand/state slots).  Z is used only after the runs are
// dead, so it lives in the runs region whenever it fits there (segments of at
// least 8m points, the usual case).
__host__ __device__ inline size_t thr_runs_bytes(int cap) { return ((size_t)cap * 12 + 4 + 15) & ~size_t(15); }
__host__ __device__ inline size_t thr_z_bytes(int m) { return (size_t)m * 24 + 16 + (size_t)(2 * m + 1) * 32; }
__host__ __device__ inline bool thr_z_in_runs(int cap, int m) { return thr_z_bytes(m) <= thr_runs_bytes(cap); }

// 1024 / T blocks per SM: at most 64 registers a thread, so that several
// blocks hide each other's serial phases
template <int T, int IPT, bool GW>
__global__ void __launch_bounds__(T, 1024 / T) k_threshold(Geom g, const ThrJob* __restrict__ jobs,
                                                 unsigned char* gwork, long long slot_stride) {
    using Sort = cub::BlockMergeSort<unsigned long long, T, IPT, int>;
    using IScan = cub::BlockScan<int, T>;
    using AReduce = cub::BlockReduce<ArgMax, T>;
    constexpr int CAP = T * IPT;

    extern __shared__ __align__(16) unsigned char thr_smem[];
    __shared__ typename IScan::TempStorage iscan_tmp;
    __shared__ typename AReduce::TempStorage red_tmp;
    __shared__ int s_nr, s_nfin, s_best, s_nops;
    __shared__ int s_cnt[2];

    const ThrJob& job = jobs[blockIdx.y];
    const QueryDev& q = job.q;
    const int m = q.m, mk = g.m_k;
    const int cnt = mk - 2 * m + 2;
    const int t = threadIdx.x;

    // GW: working set in global scratch; otherwise provably shared memory
    unsigned char* base = GW ? gwork + (long long)(blockIdx.y * gridDim.x + blockIdx.x) * slot_stride
                                : thr_smem;
    // runs (phases 1-3), then region X: sort temp (phase 2) / sorted values + g (phase 3)
    double* rval = (double*)base;                                          // [CAP]
    int* rstart = (int*)(base + (size_t)CAP * 8);                          // [CAP + 1]
    unsigned char* xb = base + thr_runs_bytes(CAP);
    // the sort's temp storage is always in shared memory (cub's block primitives
    // work on shared memory): in the shared-memory form it shares region X with
    // the sorted values, in the global-scratch form (GW) it is the block's whole
    // dynamic shared memory and region X in global memory holds the values only
    const size_t xbytes = GW ? (((size_t)CAP * 12 + 16 + 15) & ~size_t(15))
                             : ((sizeof(typename Sort::TempStorage) > (size_t)CAP * 12 + 16
                                     ? sizeof(typename Sort::TempStorage)
                                     : (size_t)CAP * 12 + 16) + 15) & ~size_t(15);
    typename Sort::TempStorage& sort_tmp =
        *reinterpret_cast<typename Sort::TempStorage*>(GW ? thr_smem : xb);
    double* tv = (double*)xb;                           // [CAP] sorted values
    int* gp = (int*)(xb + (size_t)CAP * 8);             // [CAP] inclusive count sums
    unsigned char* zb = thr_z_in_runs(CAP, m) ? base : xb + xbytes;
    int* sA = (int*)zb;                                 // [m]
    int* sB = sA + m;                                   // [m]
    int* opdesc = sB + m;                               // [2m]
    int* opstep = opdesc + 2 * m;                       // [2m]
    double* st = (double*)(((uintptr_t)(opstep + 2 * m) + 15) & ~uintptr_t(15));  // [(2m+1)*4]

    const int p = q.p;
    const int kind = (q.metric == DTW) ? 0 : (q.metric == ERP ? 2 : 1);

    for (long long bid = blockIdx.x; bid < 2 * g.S; bid += gridDim.x) {
        const long long s = bid >> 1;
        const int upper = (int)(bid & 1);
        const double* env = (upper ? job.Un : job.Ln) + s * mk + (m - 1);

        // ---- 1. run-length dedup (src/find_t_lp.cpp:53-67)
        double v[IPT];
        int nflag = 0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = t * IPT + k;
            v[k] = (i < cnt) ? env[i] : 0.0;
        }
        bool flag[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = t * IPT + k;
            bool f = false;
            if (i < cnt) {
                const double prev = (k > 0) ? v[k - 1] : (i > 0 ? env[i - 1] : 0.0);
                f = (i == 0) || (v[k] != prev);
            }
            flag[k] = f;
            nflag += f ? 1 : 0;
        }
        int roff, nr;
        IScan(iscan_tmp).ExclusiveSum(nflag, roff, nr);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (flag[k]) {
                rstart[roff] = t * IPT + k;
                rval[roff] = v[k];
                ++roff;
            }
        }
        if (t == 0) { rstart[nr] = cnt; s_nr = nr; }
        __syncthreads();

        // ---- 2. sort runs (src/find_t_lp.cpp:68-81)
        unsigned long long keys[IPT];
        int rid[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int r = t * IPT + k;
            keys[k] = (r < nr) ? order_key(rval[r], upper ? 0 : 1) : ~0ull;  // padding after every run
            rid[k] = r;
        }
        Sort(sort_tmp).StableSort(keys, rid, KeyLess());
        __syncthreads();

        // ---- 3. sorted values, cumulative counts g_i, finite prefix length
        int csum = 0, nf = 0;
        double sv_[IPT];
        int sc_[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = t * IPT + k;
            sv_[k] = 0.0;
            sc_[k] = 0;
            if (i < nr) {
                const int r = rid[k];
                sv_[k] = rval[r];
                sc_[k] = rstart[r + 1] - rstart[r];
                csum += sc_[k];
                nf += isnan(sv_[k]) ? 0 : 1;
            }
        }
        int cbase;
        IScan(iscan_tmp).ExclusiveSum(csum, cbase);
        __syncthreads();
        int nfin_total;
        IScan(iscan_tmp).ExclusiveSum(nf, nf, nfin_total);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = t * IPT + k;
            if (i < nr) {
                tv[i] = sv_[k];
                cbase += sc_[k];
                gp[i] = cbase;
            }
        }
        if (t == 0) { s_nfin = nfin_total; s_cnt[0] = 0; s_cnt[1] = 0; }
        __syncthreads();
        const int nfin = s_nfin;
        double* out = job.thr + s * 2 + upper;
        if (nfin == 0) {  // every score is NaN: index 0 wins
            if (t == 0) *out = tv[0];
            __syncthreads();
            continue;
        }

        // ---- 4. stream plan, src/find_t_lp.cpp init loops: the pointer
        // scans stop at the partition point of a monotone table (sorted
        // query, t_l/t_u of the sorted query, the ERP pop orders), found here
        // as a block-wide count
        const double t0 = tv[0];
        {
            int c0 = 0, c1 = 0;
            for (int j = t; j < m; j += T) {
                if (kind == 0) {
                    c0 += upper ? (q.qs[j] <= t0) : (q.qs[j] < t0);
                } else if (kind == 1) {
                    if (!upper) { c0 += q.qs[j] < t0; c1 += q.tlq[j] < t0; }
                    else { c0 += q.qs[j] <= t0; c1 += q.tuq[j] <= t0; }
                } else {
                    if (!upper) { c0 += q.otl[q.ordA_l[j]] >= t0; c1 += q.qn[q.ordB_l[j]] >= t0; }
                    else { c0 += q.otu[q.ordA_u[j]] <= t0; c1 += q.qn[q.ordB_u[j]] <= t0; }
                }
            }
            for (int o = 16; o; o >>= 1) {
                c0 += __shfl_xor_sync(0xffffffffu, c0, o);
                c1 += __shfl_xor_sync(0xffffffffu, c1, o);
            }
            if ((t & 31) == 0) { atomicAdd(&s_cnt[0], c0); atomicAdd(&s_cnt[1], c1); }
        }
        __syncthreads();
        Plan pl;
        pl.kind = kind; pl.upper = upper; pl.p = p;
        pl.idx1 = pl.idx2 = pl.kA0 = pl.kB0 = 0;
        pl.nA = pl.nB = 0;
        {
            const int c0 = s_cnt[0], c1 = s_cnt[1];
            if (kind == 0) {
                if (!upper) { pl.idx1 = c0 - 1; pl.nB = pl.idx1 + 1; }
                else { pl.idx1 = c0; pl.nB = m - pl.idx1; }
            } else if (kind == 1) {
                if (!upper) {
                    pl.idx1 = c0 - 1;
                    pl.idx2 = min(pl.idx1, c1 - 1);
                    pl.nA = pl.idx2 + 1;
                    pl.nB = pl.idx1 + 1;
                } else {
                    pl.idx1 = c0;
                    pl.idx2 = max(pl.idx1, c1);
                    pl.nA = m - pl.idx2;
                    pl.nB = m - pl.idx1;
                }
            } else {
                pl.kA0 = c0;
                pl.kB0 = c1;
                pl.nA = m - pl.kA0;
                pl.nB = m - pl.kB0;
            }
        }

        // ---- 5. firing step of every op
        for (int r = t; r < pl.nA; r += T) {
            int st_ = kNever;
            if (kind == 1) {
                if (!upper) { const int j = pl.idx2 - r; st_ = first_step(tv, nfin, LE, q.tlq[j]); }
                else { const int j = pl.idx2 + r; st_ = first_step(tv, nfin, GE, q.tuq[j]); }
            } else if (kind == 2) {
                if (!upper) { const int e = q.ordA_l[pl.kA0 + r]; st_ = first_step(tv, nfin, LE, q.otl[e]); }
                else { const int e = q.ordA_u[pl.kA0 + r]; st_ = first_step(tv, nfin, GE, q.otu[e]); }
            }
            sA[r] = st_;
        }
        for (int r = t; r < pl.nB; r += T) {
            int st_ = kNever;
            if (kind == 0) {
                if (!upper) st_ = first_step(tv, nfin, LE, q.qs[pl.idx1 - r]);
                else st_ = first_step(tv, nfin, GT, q.qs[pl.idx1 + r]);
            } else if (kind == 1) {
                if (!upper) {
                    const int j = pl.idx1 - r;
                    st_ = first_step(tv, nfin, LT, q.qs[j]);
                    if (j <= pl.idx2 && st_ != kNever) st_ = max(st_, first_step(tv, nfin, LE, q.tlq[j]));
                } else {
                    const int j = pl.idx1 + r;
                    st_ = first_step(tv, nfin, GT, q.qs[j]);
                    if (j >= pl.idx2 && st_ != kNever) st_ = max(st_, first_step(tv, nfin, GE, q.tuq[j]));
                }
            } else {
                if (!upper) {
                    const int e = q.ordB_l[pl.kB0 + r];
                    st_ = first_step(tv, nfin, LE, q.qn[e]);
                    if (q.otl[e] < t0 && st_ != kNever) st_ = max(st_, first_step(tv, nfin, LE, q.otl[e]));
                } else {
                    const int e = q.ordB_u[pl.kB0 + r];
                    st_ = first_step(tv, nfin, GE, q.qn[e]);
                    if (q.otu[e] > t0 && st_ != kNever) st_ = max(st_, first_step(tv, nfin, GE, q.otu[e]));
                }
            }
            sB[r] = st_;
        }
        __syncthreads();

        // ---- 6. op order: (step, stream A before B, rank)
        // valid ops form a prefix of each stream (steps never go from finite to kNever and back)
        const int nAv = prefix_count(pl.nA, [&](int r) { return sA[r] != kNever; });
        const int nBv = prefix_count(pl.nB, [&](int r) { return sB[r] != kNever; });
        const bool b_sorted = (kind != 2);
        for (int k = t; k < nAv + nBv; k += T) opdesc[k] = -1;
        __syncthreads();
        for (int r = t; r < nAv; r += T) {
            const int sa = sA[r];
            int blt;  // valid B ops with step < sa
            if (b_sorted) {
                blt = prefix_count(nBv, [&](int k) { return sB[k] < sa; });
            } else {
                blt = 0;
                for (int k = 0; k < nBv; ++k) blt += (sB[k] < sa) ? 1 : 0;
            }
            const int pos = r + blt;
            opdesc[pos] = r;
            opstep[pos] = sa;
        }
        for (int r = t; r < nBv; r += T) {
            const int sb = sB[r];
            int bbefore;
            if (b_sorted) {
                bbefore = r;
            } else {
                bbefore = 0;
                for (int k = 0; k < nBv; ++k) {
                    const int sk = sB[k];
                    bbefore += (sk < sb || (sk == sb && k < r)) ? 1 : 0;
                }
            }
            const int ale = prefix_count(nAv, [&](int k) { return sA[k] <= sb; });
            const int pos = bbefore + ale;
            opdesc[pos] = 0x40000000 | r;
            opstep[pos] = sb;
        }
        if (t == 0) s_nops = nAv + nBv;
        __syncthreads();
        const int nops = s_nops;

        // ---- 7. replay: initial sums then every op, in the reference's order.
        // Every thread first gathers the operands into shared memory, already
        // signed for the accumulator they go to, so that the replaying lanes
        // only add: x - y is x + (-y) in IEEE arithmetic, and an element or op
        // that leaves an accumulator unchanged contributes -0.0 (x + -0.0 == x
        // for every x, signed zeros included).
        const double* pw0 = (kind == 2) ? q.opw : q.pw;
        const double* Dt = (kind == 2) ? q.oD : q.Dq;
        for (int j = t; j < m; j += T) {
            double o0 = pw0[j], o1 = pw0[m + j], o2 = pw0[2 * m + j], o3 = Dt[j];
            if (kind == 2) {  // which initial sum the element enters, if any
                const double qv = q.qn[j];
                int cd;
                if (!upper) cd = (qv >= t0) ? 0 : (q.otl[j] >= t0 ? 1 : 2);
                else cd = (qv <= t0) ? 0 : (q.otu[j] <= t0 ? 1 : 2);
                if (cd != 1) o0 = o1 = o2 = -0.0;
                if (cd != 2) o3 = -0.0;
            }
            double* o = st + 4 * j;
            o[0] = o0; o[1] = o1; o[2] = o2; o[3] = o3;
        }
        __syncthreads();
        // initial sums: lane j of warp 0 owns accumulator j (the power sums
        // m_0..m_2 for j < 3, the penalty sum C for j = 3) and adds its
        // elements in the reference's order
        double acc = 0.0;
        if (t < 4) {
            const int jc = t;
            // elements e0, e0+dir, ... (len of them); eight operands are loaded
            // ahead of their adds
            auto chain = [&](int e0, int dir, int len) {
                for (int i0 = 0; i0 < len; i0 += 8) {
                    double v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int i = i0 + u;
                        v[u] = (i < len) ? st[4 * (e0 + dir * i) + jc] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (i0 + u < len) acc = dadd(acc, v[u]);
                }
            };
            if (jc < 3) {
                if (kind == 0) {
                    if (!upper) chain(0, 1, pl.idx1 + 1);
                    else chain(pl.idx1, 1, m - pl.idx1);
                } else if (kind == 1) {
                    if (!upper) chain(pl.idx1, -1, pl.idx1 - pl.idx2);
                    else chain(pl.idx1, 1, pl.idx2 - pl.idx1);
                } else {
                    chain(0, 1, m);
                }
            } else {
                if (kind == 1) {
                    if (!upper) chain(0, 1, pl.idx2 + 1);
                    else chain(pl.idx2, 1, m - pl.idx2);
                } else if (kind == 2) {
                    chain(0, 1, m);
                }
            }
        }
        __syncthreads();
        // op payloads into the state slots the replay overwrites: op B
        // subtracts the element's powers, op A adds them and subtracts its
        // penalty
        for (int k = t; k < nops; k += T) {
            const int d = opdesc[k];
            double* o = st + 4 * (k + 1);
            if (d < 0) {  // unreachable when the op order is a permutation; keeps reads in bounds
                o[0] = o[1] = o[2] = o[3] = -0.0;
                continue;
            }
            const int r = d & 0x3fffffff;
            const bool op_b = (d & 0x40000000) != 0;
            int x;  // table index of the op's query element
            if (kind == 2) x = op_b ? (upper ? q.ordB_u : q.ordB_l)[pl.kB0 + r]
                                    : (upper ? q.ordA_u : q.ordA_l)[pl.kA0 + r];
            else if (op_b) x = upper ? pl.idx1 + r : pl.idx1 - r;
            else x = upper ? pl.idx2 + r : pl.idx2 - r;
            x = min(max(x, 0), m - 1);
            const double a0 = pw0[x], a1 = pw0[m + x], a2 = pw0[2 * m + x], a3 = Dt[x];
            o[0] = op_b ? -a0 : a0;
            o[1] = op_b ? -a1 : a1;
            o[2] = op_b ? -a2 : a2;
            o[3] = op_b ? -0.0 : -a3;
        }
        __syncthreads();
        // replay: lane j adds every op's operand to its accumulator j and
        // stores the state after each op, in chunks of eight (the next chunk's
        // operands are loaded before this chunk's states overwrite its slots)
        if (t < 4) {
            const int jc = t;
            st[jc] = acc;
            constexpr int RC = 8;
            double a[RC];
#pragma unroll
            for (int u = 0; u < RC; ++u) a[u] = (u < nops) ? st[4 * (u + 1) + jc] : 0.0;
            for (int k0 = 0; k0 < nops; k0 += RC) {
                double na[RC];
#pragma unroll
                for (int u = 0; u < RC; ++u) {
                    const int k = k0 + RC + u;
                    na[u] = (k < nops) ? st[4 * (k + 1) + jc] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < RC; ++u) {
                    const int k = k0 + u;
                    if (k < nops) {
                        acc = dadd(acc, a[u]);
                        st[4 * (k + 1) + jc] = acc;
                    }
                }
#pragma unroll
                for (int u = 0; u < RC; ++u) a[u] = na[u];
            }
        }
        __syncthreads();

        // ---- 8. scores and first maximum
        ArgMax best{0.0, INT_MAX, 0};
        int nan0 = 0;
        // each thread scores a contiguous range of steps, so the number of ops
        // with step <= i is one binary search followed by a forward walk
        const int per = (nr + T - 1) / T;
        const int i_beg = t * per, i_end = min(i_beg + per, nr);
        int lo = 0;
        if (i_beg < i_end) {
            int hi = nops;
            while (lo < hi) { const int mid = (lo + hi) >> 1; if (opstep[mid] <= i_beg) lo = mid + 1; else hi = mid; }
        }
        for (int i = i_beg; i < i_end; ++i) {
            while (lo < nops && opstep[lo] <= i) ++lo;
            const double* sv = st + 4 * lo;
            const double tt = tv[i];
            const double f = f_p(sv[0], sv[1], sv[2], p, tt);
            double h;
            if (kind == 0) h = upper ? f : fabs(f);
            else h = dadd(sv[3], upper ? f : fabs(f));
            const double lb = dmul(h, (double)gp[i]);
            if (isnan(lb)) {
                if (i == 0) nan0 = 1;  // findMaxIndex never leaves a NaN at index 0
            } else {
                best = ArgMaxOp()(best, ArgMax{lb, i, 1});
            }
        }
        const int any_nan0 = __syncthreads_or(nan0);
        const ArgMax r = AReduce(red_tmp).Reduce(best, ArgMaxOp());
        if (t == 0) s_best = any_nan0 ? 0 : (r.ok ? r.i : 0);
        __syncthreads();
        if (t == 0) *out = tv[s_best];
        __syncthreads();
    }
}

size_t threshold_work_bytes(int cap_items, size_t sort_tmp, int m) {
    const size_t cap = (size_t)cap_items;
    const size_t runs = thr_runs_bytes(cap_items);
    const size_t x = ((sort_tmp > cap * 12 + 16 ? sort_tmp : cap * 12 + 16) + 15) & ~size_t(15);
    const size_t z = thr_z_in_runs(cap_items, m) ? 0 : thr_z_bytes(m);
    return runs + x + z + 64;
}

template <int T, int IPT>
size_t threshold_sort_tmp_bytes() {
    return sizeof(typename cub::BlockMergeSort<unsigned long long, T, IPT, int>::TempStorage);
}

#define FSM_THR_INST(T, IPT)                                                                 \
    template __global__ void k_threshold<T, IPT, false>(Geom, const ThrJob*, unsigned char*,  \
                                                        long long);                          \
    template __global__ void k_threshold<T, IPT, true>(Geom, const ThrJob*, unsigned char*,   \
                                                       long long);                           \
    template size_t threshold_sort_tmp_bytes<T, IPT>();
FSM_THR_INST(128, 4)
FSM_THR_INST(256, 4)
FSM_THR_INST(256, 8)
FSM_THR_INST(512, 8)
FSM_THR_INST(1024, 8)
FSM_THR_INST(1024, 16)

}  // namespace fsm
