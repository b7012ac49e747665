// SELL-32x4 row sums with the matrix streamed by TMA bulk copies (sm_90+ /
// sm_100a): every warp owns a ring of STAGES shared-memory buffers; lane 0 keeps
// the next chunks (kTmaChunk groups of four entries for the 32 rows of a slice:
// values and column offsets, contiguous in the SELL layout of sell.cuh) in flight
// with cp.async.bulk against one mbarrier per stage, while the 32 lanes (one row
// each) wait for the current stage, gather x and accumulate.  Streaming the
// matrix no longer waits on the gather/FMA chain of the rows.
//
// Every wait is bounded: a stage that does not complete within kMbarWaitNs
// nanoseconds of the global timer sets *errorFlag, the warp waits (bounded again) for its copies still in flight
// and leaves; the caller reports the flag.  No multicast: each CTA reads only the
// slices it processes.
#pragma once

#include "sell.cuh"

namespace ciecu {

constexpr int kTmaWarps = 16;   // warps per CTA (one CTA per SM: shared memory bound)
constexpr int kTmaChunk = 4;    // groups of four entries per row per stage
constexpr unsigned long long kMbarWaitNs = 2000000000ULL;  // 2 s

template <typename V, typename CI>
struct TmaShape {
    static constexpr int STAGES = sizeof(CI) == 2 ? 4 : 3;
    static constexpr int VBYTES = 32 * kTmaChunk * 4 * static_cast<int>(sizeof(V));
    static constexpr int CBYTES = 32 * kTmaChunk * 4 * static_cast<int>(sizeof(CI));
    static constexpr int SBYTES = VBYTES + CBYTES;
    static constexpr int SMEM = kTmaWarps * STAGES * SBYTES + kTmaWarps * STAGES * 8;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    const unsigned long long t0 = global_ns();
    for (unsigned spins = 1;; ++spins) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((spins & 255u) == 0u && global_ns() - t0 > kMbarWaitNs) return false;
    }
}

// Global -> shared bulk copy completing on `bar` (16-byte aligned addresses, size
// a multiple of 16).  The CTA's own shared memory is its shared::cluster window.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

template <typename CI>
__device__ __forceinline__ void smem_cols4(const CI* sc, int idx, int row, int (&c)[4]);
template <>
__device__ __forceinline__ void smem_cols4<short>(const short* sc, int idx, int row, int (&c)[4]) {
    const uint2 a = reinterpret_cast<const uint2*>(sc)[idx];
    c[0] = row + static_cast<short>(a.x & 0xffffu);
    c[1] = row + static_cast<short>(a.x >> 16);
    c[2] = row + static_cast<short>(a.y & 0xffffu);
    c[3] = row + static_cast<short>(a.y >> 16);
}
template <>
__device__ __forceinline__ void smem_cols4<int>(const int* sc, int idx, int, int (&c)[4]) {
    const int4 a = reinterpret_cast<const int4*>(sc)[idx];
    c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
}

// Row sums of every slice assigned to this warp (slices warp, warp + nwarps, ...),
// the operand entry of column c given by gather(c), calling op.pre at a slice's
// first chunk and op.post after its last.  `smem` is the CTA's dynamic shared
// memory of TmaShape<float, CI>::SMEM bytes.
template <typename CI, typename Op, typename TGather>
__device__ __forceinline__ void sell_rows_tma_gather(const SellArgs<float, CI>& A, const TGather& gather, Op& op,
                                                     unsigned char* smem, unsigned* errorFlag) {
    using Shape = TmaShape<float, CI>;
    constexpr int S = Shape::STAGES;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* ring = smem + warp * (S * Shape::SBYTES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTmaWarps * S * Shape::SBYTES) + warp * S;
    const long nslices = (A.nrows + 31) >> 5;
    const long nwarps = static_cast<long>(gridDim.x) * kTmaWarps;
    const long first = static_cast<long>(blockIdx.x) * kTmaWarps + warp;
    // bulk copies need 16-byte aligned shared destinations: refuse (flag, no copy)
    // rather than issue one from a misplaced window
    if (smem_u32(smem) & 127u) {
        if (threadIdx.x == 0) atomicOr(errorFlag, 2u);
        return;
    }

    if (lane == 0) {
        for (int i = 0; i < S; ++i) mbar_init(&bars[i], 1);
        fence_mbarrier_init();
    }
    __syncwarp();

    auto groupsOf = [&](long s) {
        int len = __ldg(A.sliceLen + s);
        len = len < 0 ? -len : len;
        return (len + 3) >> 2;
    };
    // producer cursor (lane 0)
    long ps = first;
    int pc = 0;
    long issued = 0;
    auto issue = [&]() {
        const int stage = static_cast<int>(issued % S);
        const int G = groupsOf(ps);
        const int g0 = pc * kTmaChunk;
        const int cnt = G - g0 < kTmaChunk ? G - g0 : kTmaChunk;
        if (cnt > 0) {
            const long long e0 = __ldg(A.sliceStart + ps) + 128LL * g0;
            unsigned char* buf = ring + stage * Shape::SBYTES;
            const unsigned vb = 128u * cnt * sizeof(float), cb = 128u * cnt * sizeof(CI);
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[stage], vb + cb);
            bulk_copy_g2s(buf, A.val + e0, vb, &bars[stage]);
            bulk_copy_g2s(buf + Shape::VBYTES, A.col + e0, cb, &bars[stage]);
        } else {
            mbar_arrive(&bars[stage]);  // empty slice: complete the phase without data
        }
        ++issued;
        if ((++pc) * kTmaChunk >= G) {
            pc = 0;
            ps += nwarps;
        }
    };
    if (lane == 0)
        for (int i = 0; i < S && ps < nslices; ++i) issue();

    long consumed = 0;
    int cc = 0;
    typename Op::Pre pre{};
    float sum = 0.0f;
    int len = 0;
    bool failed = false;
    for (long cs = first; cs < nslices;) {
        const int G = groupsOf(cs);
        const int row = static_cast<int>(cs * 32 + lane);
        const bool valid = row < A.nrows;
        if (cc == 0) {
            sum = 0.0f;
            if (valid) {
                pre = op.pre(row);
                int l = __ldg(A.sliceLen + cs);
                len = l < 0 ? __ldg(A.rowLen + row) : l;
            } else {
                len = 0;
            }
        }
        const int stage = static_cast<int>(consumed % S);
        const unsigned parity = static_cast<unsigned>((consumed / S) & 1);
        // every lane observes the phase; the outcome is made warp-uniform so that
        // the lanes leave the loop together
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bars[stage], parity));
        if (!ok) {
            failed = true;
            break;
        }
        const int g0 = cc * kTmaChunk;
        const int cnt = G - g0 < kTmaChunk ? G - g0 : kTmaChunk;
        const float* sv = reinterpret_cast<const float*>(ring + stage * Shape::SBYTES);
        const CI* sc = reinterpret_cast<const CI*>(ring + stage * Shape::SBYTES + Shape::VBYTES);
#pragma unroll
        for (int gl = 0; gl < kTmaChunk; ++gl) {
            if (gl < cnt) {
                const float4 v = reinterpret_cast<const float4*>(sv)[gl * 32 + lane];
                int c[4];
                smem_cols4<CI>(sc, gl * 32 + lane, row, c);
                const int base = 4 * (g0 + gl);
                const float xv0 = base + 0 < len ? gather(c[0]) : 0.0f;
                const float xv1 = base + 1 < len ? gather(c[1]) : 0.0f;
                const float xv2 = base + 2 < len ? gather(c[2]) : 0.0f;
                const float xv3 = base + 3 < len ? gather(c[3]) : 0.0f;
                sum = fmaf(v.x, xv0, sum);
                sum = fmaf(v.y, xv1, sum);
                sum = fmaf(v.z, xv2, sum);
                sum = fmaf(v.w, xv3, sum);
            }
        }
        __syncwarp();  // every lane is done with this stage before it is refilled
        ++consumed;
        if (lane == 0 && ps < nslices) issue();
        if (G == 0 || (++cc) * kTmaChunk >= G) {
            if (valid) op.post(row, pre, sum);
            cc = 0;
            cs += nwarps;
        }
    }
    if (failed) {
        if (lane == 0) {
            atomicOr(errorFlag, 1u);
            // bounded wait for this warp's copies still in flight before leaving
            for (long k = consumed; k < issued; ++k)
                mbar_wait_bounded(&bars[k % S], static_cast<unsigned>((k / S) & 1));
        }
        __syncwarp();
    }
}

template <typename CI, typename Op>
__device__ __forceinline__ void sell_rows_tma(const SellArgs<float, CI>& A, const float* __restrict__ x, Op& op,
                                              unsigned char* smem, unsigned* errorFlag) {
    sell_rows_tma_gather<CI>(A, LoadGather<float>{x}, op, smem, errorFlag);
}

}  // namespace ciecu
