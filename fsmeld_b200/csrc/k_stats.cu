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
// tile ahead), so global traffic is one read of the target (plus the m-1 halo
// per segment) and one coalesced write of mu and sigma.
//
// Raw (non-normalised) mode (g.raw): a window is valid iff its points are all
// finite, and its statistics are mean 0 and sigma 1, so every later stage
// sees the raw values ((t - 0) / 1 = t exactly) with the same code.
//
// Work split: warp 0 of the block runs the 32 running-sum chains (the serial
// part) and stages each emitted window's sums and non-finite flag in a
// double-buffered tile; warps 1-3 turn the previous tile's sums into mean
// and sigma (two divisions by m, each a multiply by RN(1/m) and FMA
// corrections that give the correctly rounded quotient, and a square root
// per window) and write them out, so the chains never wait for them.
#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {
constexpr int kTile = 32;
constexpr int kPitch = kTile + 1;  // padded rows: lane-strided smem reads hit distinct banks
constexpr int kTileDoubles = 32 * kPitch;
}

__global__ void __launch_bounds__(kMvmeanThreads) k_mvmean(const double* __restrict__ target, Geom g,
                                                           double* __restrict__ mu, double* __restrict__ sig) {
    extern __shared__ double sm[];
    double* tin = sm;                        // [32][kPitch] incoming points t[k] (warp 0)
    double* tout = sm + kTileDoubles;        // [32][kPitch] outgoing points t[k-m] (warp 0)
    double* S1 = sm + 2 * kTileDoubles;      // [2][32][kPitch] staged sums, by tile parity
    double* S2 = sm + 4 * kTileDoubles;      // [2][32][kPitch] staged sums of squares
    int* FL = (int*)(sm + 6 * kTileDoubles); // [2][32][kPitch] staged non-finite flags
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const long long s0 = (long long)blockIdx.x * 32;
    const int m = g.m, mk = g.m_k, kml = g.kml;
    const int ntiles = (mk + kTile - 1) / kTile;

    // consumers (warps 1-3): mean and sigma of the emitted windows of tile t
    auto finish_tile = [&](int t) {
        const int k0 = t * kTile, cnt = min(kTile, mk - k0);
        const int b = t & 1;
        const double dm = (double)m;
        const double invm = ddiv(1.0, dm);  // S / m by the reciprocal method (correctly rounded)
        const double qnan = dnan();
        for (int idx = tid - 32; idx < 32 * kTile; idx += kMvmeanThreads - 32) {
            const int r = idx / kTile, x = idx % kTile;  // segment s0 + r, point k0 + x
            const long long sr = s0 + r;
            if (x < cnt && k0 + x >= m - 1 && sr < g.S) {
                const int o = b * kTileDoubles + r * kPitch + x;
                const bool bad = FL[o] != 0;
                double mean, sd;
                if (g.raw) {  // raw mode: valid iff every point is finite
                    mean = bad ? qnan : 0.0;
                    sd = bad ? qnan : 1.0;
                } else {
                    mean = bad ? qnan : zdiv_i(S1[o], dm, invm, true);
                    sd = bad ? qnan : dsqrt(dsub(zdiv_i(S2[o], dm, invm, true), dmul(mean, mean)));
                }
                const long long w = sr * kml + (k0 + x - m + 1);
                mu[w] = mean;
                sig[w] = sd;
            }
        }
    };

    // producer (warp 0): the running sums of segment s0 + lane
    double s1 = 0.0, s2 = 0.0;
    int nonfinite = 0;
    double pin[32], pout[32];  // the next tile (row r = segment s0 + r, column = lane)
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
    if (tid < 32) load_tile(0);
    for (int t = 0; t <= ntiles; ++t) {
        if (tid < 32) {
            if (t < ntiles) {
                const int k0 = t * kTile, cnt = min(kTile, mk - k0);
                const int b = t & 1;
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    tin[r * kPitch + lane] = pin[r];
                    tout[r * kPitch + lane] = pout[r];
                }
                __syncwarp();
                if (k0 + kTile < mk) load_tile(k0 + kTile);
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
                        const int o = b * kTileDoubles + lane * kPitch + x;
                        S1[o] = s1;
                        S2[o] = s2;
                        FL[o] = nonfinite;
                    }
                }
                __syncwarp();
            }
        } else if (t > 0) {
            finish_tile(t - 1);
        }
        // tile t is staged and tile t-1 consumed: the producer may overwrite
        // buffer (t-1) & 1 with tile t+1
        __syncthreads();
    }
}

size_t mvmean_smem_bytes() { return sizeof(double) * 6 * kTileDoubles + sizeof(int) * 2 * kTileDoubles; }

}  // namespace fsm
