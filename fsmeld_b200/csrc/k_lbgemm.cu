// LB_IP for a group of queries of equal (m, w) as one tensor-core
// contraction (tcgen05.mma, BF16 operands, FP32 accumulation in TMEM).
//
// LB_IP's sliding inner products (src/sip.cpp:16-52; z[m-1+j] = sum_k
// h[k] g[j+k], src/fsmeld.cpp:792-806) have a product form: the window masks
// g depend on the target envelopes and a threshold t, the penalties h on the
// query and t (src/lb.cpp:18-34, src/q_to_h.cpp:11-134).  When every query
// of a group uses the same thresholds (t_l, t_u), the masks are shared and
// the inner products of all windows with all queries are one matrix product
//
//     Z[j][q] = sum_k A[j][k] B[q][k],   A[j][k] = g[j+k] (Hankel, 0/1),
//                                        B[q][k] = h_q[k],
//
// per side (lower, upper).  A is exact in BF16 (0 or 1).  Each h_q is split
// on the host into three BF16 terms h0 + h1 + h2 (h0 = bf16(h), h1 =
// bf16(h - h0), h2 = bf16(h - h0 - h1)); the three products accumulate into
// one FP32 accumulator, so Z carries the FP32 accumulation error and the
// split's residual.  The host bounds both per query and side (margin =
// residual + 4 n 2^-23 sum_k(|h0|+|h1|+|h2|), n = the accumulated terms)
// and the epilogue lowers each Z by its margin before the bound is formed,
// so the bound stays a true lower bound of the exact FP64 inner product and
// the pruning is admissible (the exact DP decides every match).  Any
// threshold gives a valid bound (the reference picks one per segment and
// query to make it tight; here one pair serves the whole group).
//
// Tiles: a CTA of 128 threads takes one (segment, 128-window tile) at a
// time.  The group's window masks g (one bit per segment position and side)
// are computed once before the product (k_gemm_masks, one ballot per 32
// positions).  Per 64-wide K chunk, the threads write the A tiles of both
// sides from the mask words of the tile's span (positions j0 .. j0+127+m) and
// copy the chunk of B (pre-arranged on the host in the operand layout), in
// the canonical no-swizzle K-major layout (8-row x 16-byte core matrices:
// rows 16 B apart, row groups SBO = 128 B apart, 8-element K groups LBO
// apart); one thread issues 4 K-steps x 2 sides x 3 splits of
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = NQ, K = 16) into two
// TMEM accumulators (columns [0, NQ) lower, [NQ, 2 NQ) upper) and commits
// them to an mbarrier; the next chunk's operands are written once that
// mbarrier says the MMAs have read the current ones.  The epilogue: thread r
// reads TMEM lane r (window j0 + r) with tcgen05.ld, forms each query's
// bound (src/fsmeld.cpp:84-106) and prune test (include/fsmeld_internal.h:
// 9-19) in FP64, and sets the survivors' bits in the query's window bit mask
// (one atomic OR per warp, query and word); k_bits_to_list turns a mask into
// the survivor list the GLB stage reads.
//
// Waits are bounded (about a second of clock cycles): on a timeout the
// kernel records an error flag, waits once more for its MMAs, frees its
// TMEM and returns; the host reports FSMELD_E_CUDA.
#include <cute/arch/mma_sm100_desc.hpp>

#include "common.cuh"
#include "kernels.cuh"

namespace fsm {

namespace {

constexpr int kGemmThreads = 128;
constexpr int kKChunk = 64;                         // K elements per chunk
constexpr int kAChunkBytes = 128 * kKChunk * 2;     // one side's A chunk (16 KB)
constexpr int kALbo = 16 * 128;                     // A: bytes between K groups (16 row groups x 128 B)
constexpr long long kWaitCycles = 2000000000LL;     // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    cute::UMMA::SmemDescriptor d;
    d.start_address_ = static_cast<uint16_t>(saddr >> 4);
    d.leading_byte_offset_ = static_cast<uint16_t>(lbo >> 4);
    d.stride_byte_offset_ = static_cast<uint16_t>(sbo >> 4);
    d.version_ = 1;  // Blackwell descriptor
    d.lbo_mode_ = 0;
    d.base_offset_ = 0;
    d.layout_type_ = static_cast<uint8_t>(cute::UMMA::LayoutType::SWIZZLE_NONE);
    return d.desc_;
}

template <int NQ>
__host__ __device__ constexpr uint32_t gemm_idesc() {
    // kind::f16: D F32, A and B BF16, both K-major, M = 128, N = NQ
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NQ >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// bounded wait for phase `parity` of the mbarrier; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// eight 0/1 mask bits -> eight BF16 values (1.0 = 0x3F80) packed in 16 bytes
__device__ __forceinline__ uint4 bits_to_bf16x8(uint32_t b) {
    uint4 v;
    v.x = ((b & 1u) ? 0x3F80u : 0u) | ((b & 2u) ? 0x3F800000u : 0u);
    v.y = ((b & 4u) ? 0x3F80u : 0u) | ((b & 8u) ? 0x3F800000u : 0u);
    v.z = ((b & 16u) ? 0x3F80u : 0u) | ((b & 32u) ? 0x3F800000u : 0u);
    v.w = ((b & 64u) ? 0x3F80u : 0u) | ((b & 128u) ? 0x3F800000u : 0u);
    return v;
}

__device__ __forceinline__ unsigned long long bits_at(const unsigned long long* w, int p) {
    const int q = p >> 6, r = p & 63;
    return r ? ((w[q] >> r) | (w[q + 1] << (64 - r))) : w[q];
}

}  // namespace

size_t lbgemm_smem_bytes(int nq_pad, int m) {
    const int kpad = (m + kKChunk - 1) / kKChunk * kKChunk;
    const int words = (128 + kpad + 63) / 64 + 2;
    return 2 * (size_t)kAChunkBytes + 6 * (size_t)nq_pad * kKChunk * 2 + 2 * (size_t)words * 8 + 64;
}

template <int NQ>
__global__ void __launch_bounds__(kGemmThreads) k_lbgemm(Geom g, GemmJob job) {
    extern __shared__ __align__(1024) unsigned char gm_smem[];
    unsigned char* As = gm_smem;                             // [2 sides] A chunk (canonical layout)
    unsigned char* Bs = As + 2 * kAChunkBytes;              // [2 sides][3 splits] B chunk
    const int kpad = job.kchunks * kKChunk;
    const int words = (128 + kpad + 63) / 64 + 2;
    unsigned long long* GLb = (unsigned long long*)(Bs + 6 * NQ * kKChunk * 2);
    unsigned long long* GUb = GLb + words;
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_cnt[16], s_valid[16];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = job.m, mk = g.m_k, kml = g.kml;
    const int tiles = (kml + 127) / 128;
    const long long items = g.S * tiles;
    constexpr uint32_t kCols = (2 * NQ < 32) ? 32 : 2 * NQ;
    const uint32_t idesc = gemm_idesc<NQ>();
    const uint32_t bar = smem_u32(&s_bar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    uint32_t phase = 0;
    bool failed = false;

    for (long long it = blockIdx.x; it < items && !failed; it += gridDim.x) {
        const long long s = it / tiles;
        const int j0 = (int)(it - s * tiles) * 128;
        // masks of the tile's span: positions j0 .. j0 + 128 + kpad (0 past the
        // segment), copied from the group's precomputed mask words
        {
            const unsigned* ml = job.mask_l + s * (long long)job.mask_words + (j0 >> 5);
            const unsigned* mu = job.mask_u + s * (long long)job.mask_words + (j0 >> 5);
            for (int i = tid; i < 2 * words; i += kGemmThreads) {
                ((unsigned*)GLb)[i] = ml[i];
                ((unsigned*)GUb)[i] = mu[i];
            }
        }
        __syncthreads();
        for (int c = 0; c < job.kchunks; ++c) {
            // A chunk: row r = tid, K groups kg = 0..7 (elements j0 + r + 64c + 8kg .. +7)
            const unsigned long long wl = bits_at(GLb, tid + c * kKChunk);
            const unsigned long long wu = bits_at(GUb, tid + c * kKChunk);
            const int rowoff = (tid >> 3) * 128 + (tid & 7) * 16;
#pragma unroll
            for (int kg = 0; kg < 8; ++kg) {
                *(uint4*)(As + kg * kALbo + rowoff) = bits_to_bf16x8((uint32_t)(wl >> (8 * kg)) & 0xFFu);
                *(uint4*)(As + kAChunkBytes + kg * kALbo + rowoff) = bits_to_bf16x8((uint32_t)(wu >> (8 * kg)) & 0xFFu);
            }
            // B chunk: pre-arranged, 6 NQ x 64 BF16
            const uint4* src = job.B + (size_t)c * (6 * NQ * kKChunk * 2 / 16);
            for (int i = tid; i < 6 * NQ * kKChunk * 2 / 16; i += kGemmThreads) ((uint4*)Bs)[i] = src[i];
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
                for (int ks = 0; ks < kKChunk / 16; ++ks) {
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        const uint64_t ad = umma_desc(smem_u32(As + side * kAChunkBytes + 2 * ks * kALbo), kALbo, 128);
#pragma unroll
                        for (int sp = 0; sp < 3; ++sp) {
                            const unsigned char* bsub = Bs + (side * 3 + sp) * NQ * kKChunk * 2;
                            const uint64_t bd = umma_desc(smem_u32(bsub + 2 * ks * (NQ * 16)), NQ * 16, 128);
                            mma_bf16(tmem + side * NQ, ad, bd, idesc, (c > 0 || ks > 0 || sp > 0) ? 1u : 0u);
                        }
                    }
                }
                mma_commit(bar);
            }
            const bool done = mbar_wait(bar, phase);
            phase ^= 1;
            failed = __syncthreads_or(!done) != 0;  // block-uniform
            if (failed) {
                if (tid == 0) atomicExch(job.err, 1u);
                break;
            }
        }
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // epilogue: thread tid <-> TMEM lane tid <-> window j0 + tid, 16 queries at a time
        const int j = j0 + tid;
        const bool inwin = j < kml && j >= g.lo(s);
        const long long gi = inwin ? g.gidx(s, j) : 0;
        const double sg = inwin ? job.SIG[s * kml + j] : 0.0;
        const bool sig_ok = inwin && isfinite(sg) && sg > kSigmaFloor;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        for (int q0 = 0; q0 < NQ && q0 < job.nq; q0 += 16) {
            uint32_t rl[16], ru[16];
            tmem_ld16(trow + q0, rl);
            tmem_ld16(trow + NQ + q0, ru);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (tid < 16) { s_cnt[tid] = 0; s_valid[tid] = 0; }
            __syncthreads();
            // survivor bits of this warp's 32 consecutive windows: positions p0 .. p0+31
            const long long p0 = s * (long long)kml + (j0 + 32 * warp) - g.lo(s);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int q = q0 + i;
                double z = dnan();
                bool keep = false;
                if (q < job.nq && sig_ok && !(job.excl_b[q] >= 0 && gi >= job.excl_b[q] && gi < job.excl_e[q])) {
                    const double zl = dmax0(dsub((double)__uint_as_float(rl[i]), job.margin_l[q]));
                    const double zu = dmax0(dsub((double)__uint_as_float(ru[i]), job.margin_u[q]));
                    const double zz = dadd(zl, zu);
                    const int metric = job.metric[q];
                    if (metric == DTW || metric == ERP) z = dsqrt(zz);
                    else if (metric == LCSS) z = ddiv(zz, (double)m);
                    else z = zz;
                    keep = !lbip_exceeds(z, job.cutoff[q], metric);
                }
                if (job.zout && j < kml && q < job.nq) job.zout[(size_t)q * job.zstride + s * kml + j] = z;
                const unsigned bv = __ballot_sync(0xffffffffu, !isnan(z));
                const unsigned bk = __ballot_sync(0xffffffffu, keep);
                if (lane == 0 && q < job.nq) {
                    if (bv) atomicAdd(&s_valid[i], __popc(bv));
                    if (bk && job.bits) {
                        atomicAdd(&s_cnt[i], __popc(bk));
                        unsigned* bq = job.bits + (size_t)q * job.bit_words;
                        const long long w0 = p0 >> 5;  // floor for negative p0 (short targets' tail)
                        const int sh = (int)(p0 & 31);
                        const unsigned lo_bits = bk << sh;
                        if (w0 >= 0 && lo_bits) atomicOr(bq + w0, lo_bits);
                        if (sh && (bk >> (32 - sh))) atomicOr(bq + w0 + 1, bk >> (32 - sh));
                    }
                }
            }
            __syncthreads();
            if (tid < 16 && q0 + tid < job.nq) {
                const int q = q0 + tid;
                if (s_cnt[tid]) atomicAdd(job.nsurv + q, (unsigned long long)s_cnt[tid]);
                if (s_valid[tid]) atomicAdd(job.nvalid + q, (unsigned long long)s_valid[tid]);
            }
            __syncthreads();
        }
        // the accumulators are read: the next tile may overwrite them
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    if (failed) mbar_wait(bar, phase ^ 1);  // let issued MMAs drain (bounded) before freeing TMEM
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

int gemm_mask_words(int m_k, int kml, int m) {
    const int kpad = (m + kKChunk - 1) / kKChunk * kKChunk;
    const int words = (128 + kpad + 63) / 64 + 2;  // 64-bit words a tile reads (k_lbgemm)
    const int tiles = (kml + 127) / 128;
    const int need = (tiles - 1) * 4 + 2 * words;   // 32-bit words up to the last tile's span
    const int cover = (m_k + 31) / 32;
    return (need > cover ? need : cover) + 1;
}

// One warp per 32 positions: the ballot of the threshold tests is the word.
__global__ void __launch_bounds__(256) k_gemm_masks(Geom g, const double* __restrict__ Ln,
                                                    const double* __restrict__ Un, double t_l, double t_u,
                                                    unsigned* __restrict__ mask_l, unsigned* __restrict__ mask_u,
                                                    int words) {
    const int lane = threadIdx.x & 31;
    const long long total = g.S * (long long)words;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long it = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < total; it += nwarps) {
        const long long s = it / words;
        const int p = (int)(it - s * words) * 32 + lane;
        const bool in = p < g.m_k;
        const long long o = s * (long long)g.m_k + (in ? p : 0);
        const unsigned bl = __ballot_sync(0xffffffffu, in && Ln[o] >= t_l);
        const unsigned bu = __ballot_sync(0xffffffffu, in && Un[o] <= t_u);
        if (lane == 0) {
            mask_l[it] = bl;
            mask_u[it] = bu;
        }
    }
}

// survivor bit mask -> list of window indices (ascending within a block of
// 8192 windows; blocks append in any order)
__global__ void __launch_bounds__(256) k_bits_to_list(const unsigned* __restrict__ bits, long long words,
                                                      long long* __restrict__ out, long long cap,
                                                      unsigned long long* __restrict__ n) {
    __shared__ int s_pre[256];
    __shared__ unsigned long long s_off;
    const int tid = threadIdx.x;
    for (long long b0 = (long long)blockIdx.x * 256; b0 < words; b0 += (long long)gridDim.x * 256) {
        const long long wi = b0 + tid;
        const unsigned v = wi < words ? bits[wi] : 0u;
        const int c = __popc(v);
        s_pre[tid] = c;
        __syncthreads();
        for (int d = 1; d < 256; d <<= 1) {
            const int x = tid >= d ? s_pre[tid - d] : 0;
            __syncthreads();
            s_pre[tid] += x;
            __syncthreads();
        }
        if (tid == 255) s_off = s_pre[255] ? atomicAdd(n, (unsigned long long)s_pre[255]) : 0ull;
        __syncthreads();
        unsigned long long o = s_off + s_pre[tid] - c;
        unsigned r = v;
        while (r) {
            const int bit = __ffs(r) - 1;
            r &= r - 1;
            if (o < (unsigned long long)cap) out[o] = wi * 32 + bit;
            ++o;
        }
        __syncthreads();
    }
}

template __global__ void k_lbgemm<16>(Geom, GemmJob);
template __global__ void k_lbgemm<32>(Geom, GemmJob);
template __global__ void k_lbgemm<64>(Geom, GemmJob);
template __global__ void k_lbgemm<128>(Geom, GemmJob);

const void* lbgemm_kernel(int nq_pad) {
    switch (nq_pad) {
        case 16: return (const void*)k_lbgemm<16>;
        case 32: return (const void*)k_lbgemm<32>;
        case 64: return (const void*)k_lbgemm<64>;
        case 128: return (const void*)k_lbgemm<128>;
        default: return nullptr;
    }
}

}  // namespace fsm
