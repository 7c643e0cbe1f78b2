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
// coalesced 256-byte loads per tile and stream, prefetched into registers a
// tile ahead) and the outputs are staged the same way, so global traffic is
// one read of the target (plus the m-1 halo per segment) and one coalesced
// write of mu and sigma.
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
    // the next tile's raw points are loaded into registers while the current
    // tile is processed: every load of a tile is in flight at once, behind
    // the previous tile's work (row r = segment s0 + r, column = lane)
    double pin[32], pout[32];
    auto load_tile = [&](int k0) {
        const int cnt = min(kTile, mk - k0);
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            const long long sr = s0 + r;
            double vi = 0.0, vo = 0.0;
            if (sr < g.S && lane < cnt) {
                const double* tp = target + g.off(sr);
                vi = tp[k0 + lane];
                const int ko = k0 + lane - m;
                if (ko >= 0) vo = tp[ko];
            }
            pin[r] = vi;
            pout[r] = vo;
        }
    };
    load_tile(0);
    for (int k0 = 0; k0 < mk; k0 += kTile) {
        const int cnt = min(kTile, mk - k0);
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            tin[r * kPitch + lane] = pin[r];
            tout[r * kPitch + lane] = pout[r];
        }
        __syncwarp();
        if (k0 + kTile < mk) load_tile(k0 + kTile);
        // the running sums, point by point (the serial part); each emitted
        // window's sums and non-finite flag are staged for the second pass
        for (int x = 0; x < cnt; ++x) {
            const int k = k0 + x;
            const double incoming_raw = tin[lane * kPitch + x];
            if (k < m) {
                // initial window (src/mvmean.cpp:16-27)
                if (isfinite(incoming_raw)) {
                    s1 = dadd(s1, incoming_raw);
                    s2 = dadd(s2, dmul(incoming_raw, incoming_raw));
                } else {
                    ++nonfinite;
                }
            } else {
                // slide by one (src/mvmean.cpp:32-44)
                const double outgoing_raw = tout[lane * kPitch + x];
                const bool of = isfinite(outgoing_raw), inf = isfinite(incoming_raw);
                const double outgoing = of ? outgoing_raw : 0.0;
                const double incoming = inf ? incoming_raw : 0.0;
                nonfinite += (int)!inf - (int)!of;
                s1 = dadd(dsub(s1, outgoing), incoming);
                s2 = dadd(dsub(s2, dmul(outgoing, outgoing)), dmul(incoming, incoming));
            }
            if (k >= m - 1) {  // a window ends here
                smu[lane * kPitch + x] = s1;
                ssg[lane * kPitch + x] = s2;
                tin[lane * kPitch + x] = nonfinite ? 1.0 : 0.0;
            }
        }
        // mean and sigma of every emitted window: independent of each other,
        // so consecutive windows' divisions and square roots overlap
#pragma unroll 4
        for (int x = 0; x < cnt; ++x) {
            if (k0 + x >= m - 1) {
                const double a1 = smu[lane * kPitch + x], a2 = ssg[lane * kPitch + x];
                const bool bad = tin[lane * kPitch + x] != 0.0;
                const double mean = bad ? qnan : ddiv(a1, dm);
                const double sd = bad ? qnan : dsqrt(dsub(ddiv(a2, dm), dmul(mean, mean)));
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
