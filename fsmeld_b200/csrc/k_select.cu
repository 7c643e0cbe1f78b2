// Candidate selection for the top-k `cutoff` command (src/fsmeld.cpp:185-569).
//
// The reference scans candidates in index order with a k-element max-heap of
// (distance, index) pairs and a threshold that tightens as the heap fills;
// since replacement needs a strictly smaller distance and indices arrive in
// increasing order, its result is exactly the k lexicographically smallest
// (distance, index) pairs among valid candidates.  The device form reaches
// the same set without the serial scan:
//  1. LB_IP per window (k_lbip with z output);
//  2. seeds: the windows with the smallest LB of each segment (k_seed,
//     ceil(2k/S) per segment, at most 32, so that there are at least k seeds
//     unless k > 32 S); the k-th smallest exact distance among the seeds is
//     an upper bound tau on the k-th smallest distance overall (with fewer
//     than k seeds there is no bound and every candidate is evaluated);
//  3. every valid window whose LB does not exceed tau (k_lb_filter) goes
//     through GLB at tau and then the exact DP; any window whose distance is
//     at most the true k-th distance survives both admissible bounds;
//  4. a lexicographic sort of the surviving (distance, index) pairs gives the
//     ranking and the threshold.
#include <cfloat>

#include <cub/block/block_reduce.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

__global__ void __launch_bounds__(256) k_lb_filter(Geom g, const double* __restrict__ z,
                                                   const double* __restrict__ SIG,
                                                   const double* __restrict__ cutoff_dev, int metric,
                                                   long long* out, unsigned long long* n_out, long long cap) {
    const double cutoff = *cutoff_dev;
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < g.tsn;
         base += (long long)gridDim.x * blockDim.x) {
        const long long gi = base + threadIdx.x;
        bool keep = false;
        if (gi < g.tsn) {
            long long s;
            int j;
            g.locate(gi, &s, &j);
            const double sg = SIG[s * g.kml + j];
            keep = !window_invalid(sg, g, gi) && !lbip_exceeds(z[s * g.kml + j], cutoff, metric);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (mask) {
            unsigned long long o = 0;
            const int leader = __ffs(mask) - 1;
            if (lane == leader) o = atomicAdd(n_out, (unsigned long long)__popc(mask));
            o = __shfl_sync(0xffffffffu, o, leader) + __popc(mask & ((1u << lane) - 1));
            if (keep && o < (unsigned long long)cap) out[o] = gi;
        }
    }
}

struct MinZ {
    double z;
    long long gi;
};
struct MinZOp {
    __device__ MinZ operator()(const MinZ& a, const MinZ& b) const {
        if (a.z < b.z) return a;
        if (b.z < a.z) return b;
        return (a.gi <= b.gi) ? a : b;
    }
};

// one block per segment: its per_seg valid windows with the smallest LB
// (ties: lowest index), by repeated block-wide argmin strictly after the
// previous pick in (LB, index) order
__global__ void __launch_bounds__(256) k_seed(Geom g, const double* __restrict__ z,
                                              const double* __restrict__ SIG, int per_seg,
                                              long long* out, unsigned long long* n_out, long long cap) {
    using Red = cub::BlockReduce<MinZ, 256>;
    __shared__ typename Red::TempStorage tmp;
    __shared__ MinZ s_last;
    for (long long s = blockIdx.x; s < g.S; s += gridDim.x) {
        MinZ last{-INFINITY, -1};
        for (int p = 0; p < per_seg; ++p) {
            MinZ best{INFINITY, -1};
            for (int j = g.lo(s) + threadIdx.x; j < g.kml; j += blockDim.x) {
                const long long gi = g.gidx(s, j);
                if (window_invalid(SIG[s * g.kml + j], g, gi)) continue;
                double zz = z[s * g.kml + j];
                if (isnan(zz)) zz = INFINITY;
                if (zz < last.z || (zz == last.z && gi <= last.gi)) continue;  // picked already
                best = MinZOp()(best, MinZ{zz, gi});
            }
            const MinZ r = Red(tmp).Reduce(best, MinZOp());
            if (threadIdx.x == 0) {
                s_last = r;
                if (r.gi >= 0) {
                    const unsigned long long o = atomicAdd(n_out, 1ull);
                    if (o < (unsigned long long)cap) out[o] = r.gi;
                }
            }
            __syncthreads();
            last = s_last;
            __syncthreads();
            if (last.gi < 0) break;
        }
    }
}

// The k-th smallest seed distance, as the search bound tau: the seed
// distances (non-negative, so their bit patterns order like the values) were
// sorted as 64-bit keys over all n slots, the unused slots pre-filled with
// all-ones (a NaN pattern, sorted last).  Fewer than k seeds: no bound.
__global__ void k_tau(const unsigned long long* __restrict__ sorted, long long k, long long n, double* tau) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double v = DBL_MAX;
        if (k >= 1 && k <= n) {
            const double s = __longlong_as_double((long long)sorted[k - 1]);
            if (!isnan(s)) v = s;
        }
        *tau = v;
    }
}

}  // namespace fsm
