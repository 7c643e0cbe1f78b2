// LB_IP for every window of a macro segment, fused with the prune test and
// survivor compaction.
//
// Reference: penalties q_to_h_{l,u} (src/q_to_h.cpp:11-134), masks
// s_to_g_{l,u} (src/lb.cpp:18-34), sliding inner products through real FFTs
// of length m_k (src/sip.cpp:16-52 as sequenced at src/fsmeld.cpp:792-806),
// trans (src/fsmeld.cpp:84-106 and the tail variant 912-921), and the prune
// test fsmeld_lbip_exceeds_cutoff (include/fsmeld_internal.h:9-19).
//
// z_l[m-1+j] + z_u[m-1+j] = sum_k h_l[k] g_l[j+k] + h_u[k] g_u[j+k] for the
// kml windows j.  Two paths:
//  * DTW, ERP, MSM: one complex FFT packs (g_l + i g_u), one packs the
//    reversed penalties, the two real spectra of each are separated, the
//    products are summed, and one inverse FFT gives z_l + z_u directly
//    (3 complex FFTs of length P >= m_k instead of the reference's 6 real
//    FFTs).  FP64 Stockham autosort FFT in shared memory, radix 16/8/4/2
//    passes with a padded layout (one pad every 16 points) so strided
//    stores are bank-conflict free.  Rounding differs from FFTW's at the
//    1e-13 level; the prune test's 1e-9 guard makes the decision the same.
//  * EDR, LCSS: h and g are 0/1, so the products are popcounts of bit
//    masks: exact integers, no FFT.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

__constant__ double2 c_w16[16];  // exp(-2*pi*i*k/16)

namespace {

__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}
template <int R> struct Log2;
template <> struct Log2<2> { static constexpr int v = 1; };
template <> struct Log2<4> { static constexpr int v = 2; };
template <> struct Log2<8> { static constexpr int v = 3; };
template <> struct Log2<16> { static constexpr int v = 4; };

// in-register DFT of size R (radix-2 decimation in time, natural order out)
template <int R>
__device__ __forceinline__ void dft_reg(double2 (&v)[R], bool inv) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = bitrev(i, Log2<R>::v);
        if (i < j) { const double2 tmp = v[i]; v[i] = v[j]; v[j] = tmp; }
    }
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
        for (int s = 0; s < R; s += len) {
#pragma unroll
            for (int k = 0; k < len / 2; ++k) {
                double2 w = c_w16[k * (16 / len)];
                if (inv) w.y = -w.y;
                const double2 a = v[s + k];
                const double2 b = cmul(v[s + k + len / 2], w);
                v[s + k] = cadd(a, b);
                v[s + k + len / 2] = csub(a, b);
            }
        }
    }
}

// one Stockham radix-R pass: a -> b (both padded layout)
template <int R, int T>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ a, double2* __restrict__ b, int P,
                                         int Ns, const double2* __restrict__ W, bool inv) {
    const int nb = P / R;
    for (int j = threadIdx.x; j < nb; j += T) {
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = a[padi(j + r * nb)];
        const int jm = j & (Ns - 1);
        if (Ns > 1) {
            const int stride = P / (Ns * R);
#pragma unroll
            for (int r = 1; r < R; ++r) {
                double2 w = __ldg(&W[jm * r * stride]);
                if (inv) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        dft_reg<R>(v, inv);
        const int idxD = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) b[padi(idxD + r * Ns)] = v[r];
    }
}

// Full FFT of length P = 2^logP; returns the buffer holding the result.
template <int T>
__device__ double2* fft_run(double2* a, double2* b, int P, int logP, const double2* W, bool inv) {
    const int passes = (logP + 3) / 4;
    int rem = logP, Ns = 1;
    for (int ps = 0; ps < passes; ++ps) {
        const int left = passes - ps;
        const int bits = (rem + left - 1) / left;  // spread bits evenly, larger radices first
        switch (bits) {
            case 4: fft_pass<16, T>(a, b, P, Ns, W, inv); break;
            case 3: fft_pass<8, T>(a, b, P, Ns, W, inv); break;
            case 2: fft_pass<4, T>(a, b, P, Ns, W, inv); break;
            default: fft_pass<2, T>(a, b, P, Ns, W, inv); break;
        }
        __syncthreads();
        double2* tmp = a; a = b; b = tmp;
        Ns <<= bits;
        rem -= bits;
    }
    return a;
}

// src/q_to_h.cpp:11-64 (lower) / 84-134 (upper)
__device__ __forceinline__ double q_to_h(int metric, bool upper, double x, double t, double C) {
    if (!upper) {
        switch (metric) {
            case MSM: return (x < t) ? ((dsub(t, x) < C) ? dsub(t, x) : C) : 0.0;
            case DTW: return (x < t) ? dsq(t, x) : 0.0;
            case ERP: return (x < t) ? ((dsq(x, t) > dsq(x, C)) ? dsq(x, C) : dsq(x, t)) : 0.0;
            default: return (x < dsub(t, C)) ? 1.0 : 0.0;
        }
    }
    switch (metric) {
        case MSM: return (x > t) ? ((dsub(x, t) < C) ? dsub(x, t) : C) : 0.0;
        case DTW: return (x > t) ? dsq(x, t) : 0.0;
        case ERP: return (x > t) ? ((dsq(x, t) > dsq(x, C)) ? dsq(x, C) : dsq(x, t)) : 0.0;
        default: return (x > dadd(t, C)) ? 1.0 : 0.0;
    }
}

__device__ __forceinline__ unsigned long long bits64(const unsigned long long* w, int b) {
    const int q = b >> 6, r = b & 63;
    return r ? ((w[q] >> r) | (w[q + 1] << (64 - r))) : w[q];
}

}  // namespace

template <int T, bool GW>
__global__ void __launch_bounds__(T) k_lbip(Geom g, LbJob job, const double2* __restrict__ W, int P,
                                            int logP) {
    using IScan = cub::BlockScan<int, T>;
    using IReduce = cub::BlockReduce<int, T>;
    extern __shared__ __align__(16) unsigned char lb_smem[];
    __shared__ typename IScan::TempStorage scan_tmp;
    __shared__ typename IReduce::TempStorage red_tmp;
    __shared__ unsigned long long s_base;
    __shared__ double s_tl, s_tu;

    const QueryDev& q = job.q;
    const int m = q.m, mk = g.m_k, kml = g.kml, metric = q.metric;
    const int tid = threadIdx.x;
    const bool popc_path = (metric == EDR || metric == LCSS);
    const int Pp = P + (P >> 4) + 1;
    unsigned char* lbase = GW ? job.gwork + (long long)blockIdx.x * job.slot_stride : lb_smem;
    double2* bufA = (double2*)lbase;
    double2* bufB = bufA + Pp;
    double2* bufC = bufB + Pp;
    // popcount path: words of g_l, g_u, h_l, h_u
    const int gw = (mk + 63) / 64 + 2, hw = (m + 63) / 64;
    unsigned long long* GL = (unsigned long long*)lbase;
    unsigned long long* GU = GL + gw;
    unsigned long long* HL = GU + gw;
    unsigned long long* HU = HL + hw;
    double* zpop = (double*)(HU + hw);

    for (long long s = blockIdx.x; s < g.S; s += gridDim.x) {
        if (tid == 0) { s_tl = job.thr[2 * s]; s_tu = job.thr[2 * s + 1]; }
        __syncthreads();
        const double tl = s_tl, tu = s_tu;
        const double* Ln = job.Ln + s * mk;
        const double* Un = job.Un + s * mk;
        const double* zsrc;
        if (!popc_path) {
            // X = g_l + i g_u, Y = reversed h_l + i reversed h_u (src/sip.cpp:16-29)
            for (int i = tid; i < P; i += T) {
                double2 x = make_double2(0.0, 0.0), y = make_double2(0.0, 0.0);
                if (i < mk) x = make_double2(Ln[i] >= tl ? 1.0 : 0.0, Un[i] <= tu ? 1.0 : 0.0);
                if (i < m) {
                    const double qv = q.qn[m - 1 - i];
                    y = make_double2(q_to_h(metric, false, qv, tl, q.arg), q_to_h(metric, true, qv, tu, q.arg));
                }
                bufA[padi(i)] = x;
                bufC[padi(i)] = y;
            }
            __syncthreads();
            double2* X = fft_run<T>(bufA, bufB, P, logP, W, false);
            double2* freeb = (X == bufA) ? bufB : bufA;
            double2* Y = fft_run<T>(bufC, freeb, P, logP, W, false);
            double2* Zb = (Y == bufC) ? freeb : bufC;  // the buffer holding neither X nor Y
            const double half = 0.5;
            for (int k = tid; k < P; k += T) {
                const int kn = (P - k) & (P - 1);
                const double2 xk = X[padi(k)], xn = X[padi(kn)];
                const double2 yk = Y[padi(k)], yn = Y[padi(kn)];
                // split two real spectra packed in one complex FFT
                const double2 gl = make_double2(half * (xk.x + xn.x), half * (xk.y - xn.y));
                const double2 gu = make_double2(half * (xk.y + xn.y), -half * (xk.x - xn.x));
                const double2 hl = make_double2(half * (yk.x + yn.x), half * (yk.y - yn.y));
                const double2 hu = make_double2(half * (yk.y + yn.y), -half * (yk.x - yn.x));
                Zb[padi(k)] = cadd(cmul(gl, hl), cmul(gu, hu));
            }
            __syncthreads();
            double2* Z = fft_run<T>(Zb, X, P, logP, W, true);
            const double invP = 1.0 / (double)P;
            // z_l + z_u for window j sits at m-1+j; stash it in the free buffer as doubles
            double* zs = (double*)((Z == Zb) ? X : Zb);
            for (int j = tid; j < kml; j += T) zs[j] = Z[padi(m - 1 + j)].x * invP;
            __syncthreads();
            zsrc = zs;
        } else {
            // bit masks (src/lb.cpp:18-34, src/q_to_h.cpp EDR/LCSS branches)
            const int lane = tid & 31, warp = tid >> 5;
            for (int base = warp * 32; base < gw * 64; base += T) {
                const int i = base + lane;
                const unsigned bl = __ballot_sync(0xffffffffu, i < mk && Ln[min(i, mk - 1)] >= tl);
                const unsigned bu = __ballot_sync(0xffffffffu, i < mk && Un[min(i, mk - 1)] <= tu);
                if (lane == 0) {
                    unsigned* gl32 = (unsigned*)GL;
                    unsigned* gu32 = (unsigned*)GU;
                    gl32[base >> 5] = bl;
                    gu32[base >> 5] = bu;
                }
            }
            for (int base = warp * 32; base < hw * 64; base += T) {
                const int k = base + lane;
                const double qv = (k < m) ? q.qn[k] : 0.0;
                const unsigned bl = __ballot_sync(0xffffffffu, k < m && q_to_h(metric, false, qv, tl, q.arg) != 0.0);
                const unsigned bu = __ballot_sync(0xffffffffu, k < m && q_to_h(metric, true, qv, tu, q.arg) != 0.0);
                if (lane == 0) {
                    ((unsigned*)HL)[base >> 5] = bl;
                    ((unsigned*)HU)[base >> 5] = bu;
                }
            }
            __syncthreads();
            for (int j = tid; j < kml; j += T) {
                int cnt = 0;
                for (int wd = 0; wd < hw; ++wd) {
                    cnt += __popcll(HL[wd] & bits64(GL, j + 64 * wd));
                    cnt += __popcll(HU[wd] & bits64(GU, j + 64 * wd));
                }
                zpop[j] = (double)cnt;
            }
            __syncthreads();
            zsrc = zpop;
        }

        // trans + validity + prune, in window order
        const int lo = g.lo(s);
        const int nwin = kml - lo;
        const int c = (nwin + T - 1) / T;
        const int wlo = lo + tid * c, whi = min(kml, wlo + c);
        int nvalid = 0, nsurv = 0;
        for (int j = wlo; j < whi; ++j) {
            const long long gi = g.gidx(s, j);
            const double sg = job.SIG[s * kml + j];
            if (window_invalid(sg, g, gi)) {
                if (job.zout) job.zout[s * kml + j] = dnan();
                continue;
            }
            ++nvalid;
            const double zz = zsrc[j];
            double z;
            if (metric == DTW || metric == ERP) z = dsqrt(dmax0(zz));
            else if (metric == LCSS) z = dmax0(ddiv(zz, (double)m));
            else z = zz;
            if (job.zout) job.zout[s * kml + j] = z;
            if (job.surv && !lbip_exceeds(z, q.cutoff, metric)) ++nsurv;
        }
        if (!job.surv) {
            const int tv = IReduce(red_tmp).Sum(nvalid);
            if (tid == 0 && tv) atomicAdd(job.nvalid, (unsigned long long)tv);
        } else {
            int off, total;
            IScan(scan_tmp).ExclusiveSum(nsurv, off, total);
            if (tid == 0) s_base = total ? atomicAdd(job.nsurv, (unsigned long long)total) : 0ull;
            __syncthreads();
            unsigned long long o = s_base + off;
            if (nsurv) {
                for (int j = wlo; j < whi; ++j) {
                    const long long gi = g.gidx(s, j);
                    const double sg = job.SIG[s * kml + j];
                    if (window_invalid(sg, g, gi)) continue;
                    const double zz = zsrc[j];
                    double z;
                    if (metric == DTW || metric == ERP) z = dsqrt(dmax0(zz));
                    else if (metric == LCSS) z = dmax0(ddiv(zz, (double)m));
                    else z = zz;
                    if (!lbip_exceeds(z, q.cutoff, metric)) {
                        if (o < (unsigned long long)job.surv_cap) job.surv[o] = gi;
                        ++o;
                    }
                }
            }
            const int tv = IReduce(red_tmp).Sum(nvalid);
            if (tid == 0 && tv) atomicAdd(job.nvalid, (unsigned long long)tv);
            if (tid == 0 && job.segc) {
                job.segc[3 * s] = tv;
                job.segc[3 * s + 1] = total;
                job.segc[3 * s + 2] = 0;
            }
        }
        __syncthreads();
    }
}

size_t lbip_smem_bytes(int P, int m_k, int m, int metric) {
    if (metric == EDR || metric == LCSS) {
        const int gw = (m_k + 63) / 64 + 2, hw = (m + 63) / 64;
        return (size_t)(2 * gw + 2 * hw) * 8 + (size_t)(m_k + 1) * 8 + 64;
    }
    const size_t Pp = (size_t)P + (P >> 4) + 1;
    return 3 * Pp * sizeof(double2) + 64;
}

int lbip_set_w16() {
    double2 w[16];
    for (int k = 0; k < 16; ++k) {
        const double ang = 6.283185307179586476925286766559 * k / 16.0;
        w[k] = make_double2(cos(ang), -sin(ang));
    }
    FSM_CUDA_TRY(cudaMemcpyToSymbol(c_w16, w, sizeof(w)));
    return 0;
}

template __global__ void k_lbip<256, false>(Geom, LbJob, const double2*, int, int);
template __global__ void k_lbip<256, true>(Geom, LbJob, const double2*, int, int);
template __global__ void k_lbip<512, false>(Geom, LbJob, const double2*, int, int);
template __global__ void k_lbip<512, true>(Geom, LbJob, const double2*, int, int);

}  // namespace fsm
