// Rolling window mean / standard deviation per macro segment.
//
// Follows src/mvmean.cpp:9-46 operation for operation: the running sums are
// restarted at every macro segment (src/fsmeld.cpp:753, 861) and updated by
// `sum = sum - outgoing + incoming` with non-finite points replaced by 0.0;
// a window containing a non-finite point gets NaN statistics.  The sums are
// a serial recurrence whose rounding decides validity (sigma <= 1e-12) and
// every z-normalised candidate, so each segment is one sequential chain: one
// lane per segment, 32 segments per warp.
//
// Memory: lanes of a warp walk 32 different segments in lock step.  The raw
// stream is staged through shared memory in tiles of kTile points (32
// coalesced 256-byte loads per tile and stream) and the outputs are staged
// the same way, so global traffic is one read of the target (plus the
// m-1 halo per segment) and one coalesced write of mu and sigma.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {
constexpr int kTile = 32;
constexpr int kPitch = kTile + 1;  // padded rows: lane-strided smem reads hit distinct banks
}

__global__ void __launch_bounds__(32) k_mvmean(const double* __restrict__ target, Geom g,
                                               double* __restrict__ mu, double* __restrict__ sig) {
    extern __shared__ double sm[];
    double* tin = sm;                  // [32][kPitch] incoming points t[k]
    double* tout = sm + 32 * kPitch;   // [32][kPitch] outgoing points t[k-m]
    double* smu = sm + 64 * kPitch;    // [32][kPitch] staged means
    double* ssg = sm + 96 * kPitch;    // [32][kPitch] staged sigmas
    const int lane = threadIdx.x;
    const long long s0 = (long long)blockIdx.x * 32;
    const int m = g.m, mk = g.m_k, kml = g.kml;
    const double dm = (double)m;
    const double qnan = dnan();

    double s1 = 0.0, s2 = 0.0;
    int nonfinite = 0;
    for (int k0 = 0; k0 < mk; k0 += kTile) {
        const int cnt = min(kTile, mk - k0);
        for (int r = 0; r < 32; ++r) {
            const long long sr = s0 + r;
            if (sr < g.S && lane < cnt) {
                const double* tp = target + g.off(sr);
                tin[r * kPitch + lane] = tp[k0 + lane];
                const int ko = k0 + lane - m;
                tout[r * kPitch + lane] = (ko >= 0) ? tp[ko] : 0.0;
            }
        }
        __syncwarp();
        for (int x = 0; x < cnt; ++x) {
            const int k = k0 + x;
            const double incoming_raw = tin[lane * kPitch + x];
            double mean = 0.0, sd = 0.0;
            bool emit = false;
            if (k < m) {
                // initial window (src/mvmean.cpp:16-27)
                if (isfinite(incoming_raw)) {
                    s1 = dadd(s1, incoming_raw);
                    s2 = dadd(s2, dmul(incoming_raw, incoming_raw));
                } else {
                    ++nonfinite;
                }
                emit = (k == m - 1);
            } else {
                // slide by one (src/mvmean.cpp:32-44)
                const double outgoing_raw = tout[lane * kPitch + x];
                const bool of = isfinite(outgoing_raw), inf = isfinite(incoming_raw);
                const double outgoing = of ? outgoing_raw : 0.0;
                const double incoming = inf ? incoming_raw : 0.0;
                nonfinite += (int)!inf - (int)!of;
                s1 = dadd(dsub(s1, outgoing), incoming);
                s2 = dadd(dsub(s2, dmul(outgoing, outgoing)), dmul(incoming, incoming));
                emit = true;
            }
            if (emit) {
                mean = nonfinite ? qnan : ddiv(s1, dm);
                sd = nonfinite ? qnan : dsqrt(dsub(ddiv(s2, dm), dmul(mean, mean)));
                smu[lane * kPitch + x] = mean;
                ssg[lane * kPitch + x] = sd;
            }
        }
        __syncwarp();
        // events x >= xs of this tile emitted windows k0 + x - m + 1
        const int xs = max(0, m - 1 - k0);
        if (xs < cnt) {
            for (int r = 0; r < 32; ++r) {
                const long long sr = s0 + r;
                if (sr < g.S && lane >= xs && lane < cnt) {
                    const long long o = sr * kml + (k0 + lane - m + 1);
                    mu[o] = smu[r * kPitch + lane];
                    sig[o] = ssg[r * kPitch + lane];
                }
            }
        }
        __syncwarp();
    }
}

size_t mvmean_smem_bytes() { return sizeof(double) * 4 * 32 * kPitch; }

}  // namespace fsm
