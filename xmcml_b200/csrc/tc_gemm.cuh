// BF16 GEMM on the sm_100a tensor cores (tcgen05) with fused epilogues, for the surrogate MLP.
//
//   D[M x N] = A[M x K] . B[N x K]^T      A, B bf16 row-major (K contiguous), D accumulated in FP32
//
// One CTA of 256 threads computes a 128 x BN tile of D over a range of K (split-K when the grid's
// z extent is > 1). Operand tiles of 128 (A) and BN (B) rows x 64 bf16 (128 B) are brought into
// shared memory by TMA (cp.async.bulk.tensor.2d, 128-byte swizzle) through a 2-stage ring of
// mbarrier-tracked buffers; one thread issues the tcgen05.mma instructions (M = 128, N = BN,
// K = 16 each, both operands K-major, read from shared memory through matrix descriptors) into a
// TMEM accumulator of BN columns, and tcgen05.commit signals the ring's "empty" barriers and the
// final "done" barrier. The eight warps then read the accumulator back with tcgen05.ld (warp w reads
// TMEM lanes 32 (w % 4)..+31, i.e. tile rows, and every other 32-column chunk starting at 32 (w / 4))
// and run the epilogue functor on 32 columns at a time.
//
// Every wait on an mbarrier is bounded: after kWaitNs of polling the kernel records an error in
// *err, stops issuing work, and still releases its TMEM before returning.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace xmc {
namespace tc {

constexpr int kBM = 128;          // tile rows (MMA M)
constexpr int kThreads = 256;     // 8 warps: warp w reads TMEM lanes 32 (w % 4).., column half w / 4
constexpr int kBK = 64;           // K per stage: 64 bf16 = one 128-byte swizzle row
constexpr int kStages = 2;  // small enough that two CTAs (BN = 256) share an SM: one's epilogue
                              // overlaps the other's loads and MMAs
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of any single pipeline wait: 2 s

__host__ __device__ constexpr int stage_bytes(int bn) { return (kBM + bn) * kBK * 2; }
__host__ __device__ constexpr int smem_bytes(int bn) { return kStages * stage_bytes(bn) + 1024 + 256; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase with the given parity to complete; false (and *err |= 1) after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > kWaitNs) {
            atomicOr(err, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D(tmem) (+)= A(smem desc) . B(smem desc)^T, kind::f16 (bf16 inputs, FP32 accumulate)
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
// Arrive on an mbarrier once all previously issued tcgen05.mma of this thread have completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand tile in the 128-byte swizzled layout that
// TMA writes (rows of 128 B, 8-row groups 1024 B apart): start address, leading-byte offset 16 B
// (unused for this layout), stride-byte offset 1024 B, descriptor version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor of kind::f16: FP32 accumulator, bf16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Epilogue interface: Epi::apply(row, col0, acc[32], lane, scratch) for tile row `row` (global) and
// the 32 consecutive global columns starting at col0; `lane` for warp-level work; `scratch` is the
// warp's 32 x 33 FP32 shared-memory tile (rows of the warp's 32 tile rows, padded).
template <int BN, class Epi>
__global__ void __launch_bounds__(kThreads, 2)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int k_blocks_per_split,
                int* err, const Epi epi) {
    static_assert(BN == 64 || BN == 128 || BN == 256, "BN");
    static_assert(kStages * stage_bytes(BN) >= (kThreads / 32) * 32 * 33 * 4, "epilogue staging tiles fit the ring");
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-byte aligned stage ring
    unsigned char* aligned = smem_raw + (base - raw);
    const uint32_t bars = base + kStages * stage_bytes(BN);  // full[S], empty[S], done: 8 B each
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(aligned + kStages * stage_bytes(BN) + 8 * (2 * kStages + 1));
    const uint32_t full0 = bars, empty0 = bars + 8 * kStages, done = bars + 16 * kStages;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * kBM;
    const int kb0 = blockIdx.z * k_blocks_per_split;
    const int nk = k_blocks_per_split;

    if (warp == 0) {
        tmem_alloc(smem_u32(s_tmem), BN);
        tmem_relinquish();
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *s_tmem;

    if (threadIdx.x == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
        constexpr uint32_t idesc = idesc_bf16(kBM, BN);
        const int pre = nk < kStages ? nk : kStages;
        for (int i = 0; i < pre; ++i) {
            const uint32_t sa = base + i * stage_bytes(BN), sb = sa + kBM * kBK * 2;
            mbar_expect_tx(full0 + 8 * i, stage_bytes(BN));
            tma_load_2d(sa, &tmA, full0 + 8 * i, (kb0 + i) * kBK, m0);
            tma_load_2d(sb, &tmB, full0 + 8 * i, (kb0 + i) * kBK, n0);
        }
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            if (!mbar_wait(full0 + 8 * s, (kb / kStages) & 1, err)) break;
            tc_fence_after();
            const uint32_t sa = base + s * stage_bytes(BN), sb = sa + kBM * kBK * 2;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk)
                umma_bf16(taddr, sw128_desc(sa + 32 * kk), sw128_desc(sb + 32 * kk), idesc, (kb | kk) != 0);
            umma_commit(empty0 + 8 * s);
            // refill the stage of the previous k-block once its MMAs are done
            if (kb >= 1 && kb - 1 + kStages < nk) {
                const int pk = kb - 1, ps = pk % kStages;
                if (!mbar_wait(empty0 + 8 * ps, (pk / kStages) & 1, err)) break;
                const uint32_t pa = base + ps * stage_bytes(BN), pb = pa + kBM * kBK * 2;
                mbar_expect_tx(full0 + 8 * ps, stage_bytes(BN));
                tma_load_2d(pa, &tmA, full0 + 8 * ps, (kb0 + pk + kStages) * kBK, m0);
                tma_load_2d(pb, &tmB, full0 + 8 * ps, (kb0 + pk + kStages) * kBK, n0);
            }
        }
        umma_commit(done);
    }
    __syncwarp();

    const bool ok = mbar_wait(done, 0, err);
    tc_fence_after();
    // warp-uniform: tcgen05.ld is a .sync.aligned instruction
    if (__all_sync(0xffffffffu, ok && *((volatile int*)err) == 0)) {
        const int quarter = warp & 3;  // TMEM lanes (tile rows) this warp may read
        const int row = m0 + quarter * 32 + lane;
        // the operand ring is idle once `done` has fired: its first 33 KB serve as per-warp
        // 32 x 33 FP32 staging tiles for row-coalesced stores
        float* scratch = reinterpret_cast<float*>(aligned) + warp * (32 * 33);
#pragma unroll 1
        for (int c = (warp >> 2) * 32; c < BN; c += 64) {
            uint32_t r[32];
            tmem_ld32(taddr + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, r);
            tmem_ld_wait();
            epi.apply(row, n0 + c, r, lane, scratch);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, BN);
}

}  // namespace tc
}  // namespace xmc
