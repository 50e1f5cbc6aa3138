// Fused forward pass (inference) of the surrogate MLP on the sm_100a tensor cores.
//
// One persistent CTA per SM walks 128-row tiles of the input. For each tile every layer runs in
// turn with the tile's activations kept in shared memory, so nothing but the inputs, the weights
// (L2-resident, streamed by TMA) and the FP32 outputs touches global memory:
//
//   layer 0        A = X tile [128 x 64]  (TMA)            B = W_0 [hidden x 64]
//   hidden 1..L-2  A = H [128 x hidden]   (shared memory)  B = W_l [hidden x hidden]
//   output L-1     A = H                                   B = W_out, 256 output columns per chunk
//
// Roles (576 threads): warp 16 lane 0 issues the TMA loads (the X tile and the weights, 64
// K-columns per stage through a 2-stage ring); warp 17 lane 0 issues tcgen05.mma (M = 128, N =
// hidden or 256, K = 16) into one of two 256-column TMEM accumulators, alternating, and commits to
// mbarriers; warps 0-15 drain an accumulator with tcgen05.ld (warp w: TMEM lanes 32 (w % 4).., a
// quarter of the columns chosen by w / 4). A hidden layer's epilogue adds the bias, applies SiLU and writes the BF16 activations
// back into H in the 128-byte-swizzled K-major layout the next layer's MMAs read (then
// fence.proxy.async and an mbarrier arrive); the output epilogue adds the bias and stores 32 x 32
// FP32 boxes through a swizzled staging buffer with TMA (cp.async.bulk.tensor store), so the
// stores of one 256-column chunk overlap the MMAs of the next in the other accumulator.
//
// Every mbarrier wait is bounded (tc::kWaitNs); after a failed wait the role sets *err, stops
// issuing work and the CTA still drains its copies and MMAs and releases TMEM.
#pragma once

#include "tc_gemm.cuh"

namespace xmc {
namespace fused {

constexpr int kMaxL = 9;
constexpr int kEpiWarps = 16;  // warp w reads TMEM lanes 32 (w % 4).. and column group w / 4
constexpr int kColGroups = kEpiWarps / 4;
constexpr int kThreads = 32 * (kEpiWarps + 2);
constexpr int kWStages = 2;  // weight ring depth (stages of 64 K-columns)
constexpr int kXBytes = 128 * 64 * 2;      // input tile, one 64-column k-block
constexpr int kKBlockBytes = 128 * 128;    // one 64-column k-block of a 128-row operand
constexpr int kHBytes = 4 * kKBlockBytes;  // activations, hidden <= 256
constexpr int kWBytes = 256 * 64 * 2;      // weight stage: up to 256 rows x 64 columns
constexpr int kOutBox = 32 * 32 * 4;       // one warp's 32 x 32 FP32 output box
constexpr int kOutBufs = 1;  // output staging box per epilogue warp
constexpr int kOffX = 0;
constexpr int kOffH = kOffX + kXBytes;
constexpr int kOffW = kOffH + kHBytes;
constexpr int kOffO = kOffW + kWStages * kWBytes;
constexpr int kOffBar = kOffO + kEpiWarps * kOutBufs * kOutBox;
constexpr int kSmemBytes = kOffBar + 256 + 1024;  // barriers, TMEM slot, abort flag; alignment slack
static_assert(kSmemBytes <= 232448, "fused forward exceeds the shared memory of one CTA");

struct Params {
    CUtensorMap x;             // bf16 [rows x 64], box 64 x 128, 128-byte swizzle
    CUtensorMap w[kMaxL];      // bf16 [out_l x in_l], box 64 x (hidden or 256), 128-byte swizzle
    CUtensorMap y;             // fp32 [rows x n_out], box 32 x 32, 128-byte swizzle
    const float* bias[kMaxL];  // [out_l] (padded)
    int L;                     // layers (hidden layers + 1)
    int hidden;                // 128 or 256
    int out_chunks;            // padded output columns / 256
    int n_tiles;               // rows / 128
    int n_out;                 // output columns (boxes past them are not stored)
    int* err;
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(src), "r"(x), "r"(y)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until at most N committed bulk groups of this thread still read their shared-memory source
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// SiLU(z) = z sigmoid(z) = z/2 (1 + tanh(z/2)): one MUFU operation per element
__device__ __forceinline__ float silu_tanh(float z) {
    const float h = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// layer geometry: MMA N of one chunk, chunks, 64-column k-blocks
__device__ __forceinline__ int layer_n(const Params& p, int l) { return l < p.L - 1 ? p.hidden : 256; }
__device__ __forceinline__ int layer_chunks(const Params& p, int l) { return l < p.L - 1 ? 1 : p.out_chunks; }
__device__ __forceinline__ int layer_kblocks(const Params& p, int l) { return l == 0 ? 1 : p.hidden / 64; }

__global__ void __launch_bounds__(kThreads, 1) mlp_forward_kernel(const __grid_constant__ Params p) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = tc::smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t sX = base + kOffX, sH = base + kOffH, sW = base + kOffW, sO = base + kOffO;
    const uint32_t bar = base + kOffBar;
    const uint32_t w_full = bar, w_empty = bar + 8 * kWStages;
    const uint32_t x_full = bar + 16 * kWStages, x_empty = x_full + 8;
    const uint32_t acc_full = x_empty + 8, acc_empty = acc_full + 16;  // two each
    const uint32_t h_full = acc_empty + 16, drain = h_full + 8;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + kOffBar + 192);
    volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + kOffBar + 196);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_u32(s_tmem), 512);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 32 * kEpiWarps) {
        for (int s = 0; s < kWStages; ++s) {
            tc::mbar_init(w_full + 8 * s, 1);
            tc::mbar_init(w_empty + 8 * s, 1);
        }
        tc::mbar_init(x_full, 1);
        tc::mbar_init(x_empty, 1);
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(acc_full + 8 * b, 1);
            tc::mbar_init(acc_empty + 8 * b, kEpiWarps);
        }
        tc::mbar_init(h_full, kEpiWarps);
        tc::mbar_init(drain, 1);
        *s_abort = 0;
        tc::mbar_fence_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *s_tmem;

    if (warp == kEpiWarps && lane == 0) {
        // ---------------- TMA producer ----------------
        tc::tma_prefetch_desc(&p.x);
        uint32_t it = 0;
        int tc_count = 0;
        bool ok = true;
        for (int t = blockIdx.x; ok && t < p.n_tiles; t += gridDim.x, ++tc_count) {
            if (!(ok = tc::mbar_wait(x_empty, (tc_count & 1) ^ 1, p.err))) break;
            tc::mbar_expect_tx(x_full, kXBytes);
            tc::tma_load_2d(sX, &p.x, x_full, 0, t * 128);
            for (int l = 0; ok && l < p.L; ++l) {
                const int n = layer_n(p, l), nk = layer_kblocks(p, l);
                for (int c = 0; ok && c < layer_chunks(p, l); ++c)
                    for (int kb = 0; kb < nk; ++kb, ++it) {
                        const int s = it % kWStages;
                        if (!(ok = tc::mbar_wait(w_empty + 8 * s, ((it / kWStages) & 1) ^ 1, p.err))) break;
                        tc::mbar_expect_tx(w_full + 8 * s, (uint32_t)n * 128u);
                        tc::tma_load_2d(sW + s * kWBytes, &p.w[l], w_full + 8 * s, kb * 64, c * 256);
                    }
            }
        }
        if (!ok) *s_abort = 1;
        // every issued load has landed before the CTA exits
        for (uint32_t i = it > kWStages ? it - kWStages : 0; i < it; ++i)
            tc::mbar_wait(w_full + 8 * (i % kWStages), (i / kWStages) & 1, p.err);
        if (tc_count > 0) tc::mbar_wait(x_full, (tc_count - 1) & 1, p.err);
    } else if (warp == kEpiWarps + 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        uint32_t it = 0, j = 0, hw = 0;
        int tc_count = 0;
        bool ok = true;
        const uint32_t idesc_h = tc::idesc_bf16(128, p.hidden), idesc_o = tc::idesc_bf16(128, 256);
        for (int t = blockIdx.x; ok && t < p.n_tiles; t += gridDim.x, ++tc_count) {
            for (int l = 0; ok && l < p.L; ++l) {
                const int nk = layer_kblocks(p, l);
                const uint32_t idesc = l < p.L - 1 ? idesc_h : idesc_o;
                const uint32_t a0 = l == 0 ? sX : sH;
                for (int c = 0; ok && c < layer_chunks(p, l); ++c, ++j) {
                    const uint32_t b = j & 1;
                    if (!(ok = tc::mbar_wait(acc_empty + 8 * b, ((j >> 1) & 1) ^ 1, p.err))) break;
                    if (l == 0) ok = tc::mbar_wait(x_full, tc_count & 1, p.err);
                    else if (c == 0) ok = tc::mbar_wait(h_full, (hw++) & 1, p.err);
                    if (!ok || *s_abort) { ok = false; break; }
                    tc::tc_fence_after();
                    const uint32_t d = taddr + 256u * b;
                    for (int kb = 0; kb < nk; ++kb, ++it) {
                        const int s = it % kWStages;
                        if (!(ok = tc::mbar_wait(w_full + 8 * s, (it / kWStages) & 1, p.err))) break;
                        tc::tc_fence_after();
                        const uint32_t sa = a0 + kb * kKBlockBytes, sb = sW + s * kWBytes;
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            tc::umma_bf16(d, tc::sw128_desc(sa + 32 * kk), tc::sw128_desc(sb + 32 * kk), idesc,
                                          (kb | kk) != 0);
                        tc::umma_commit(w_empty + 8 * s);
                    }
                    if (!ok) break;
                    if (l == 0) tc::umma_commit(x_empty);
                    tc::umma_commit(acc_full + 8 * b);
                }
            }
        }
        if (!ok) *s_abort = 1;
        // every issued MMA has completed before TMEM is released
        tc::umma_commit(drain);
        tc::mbar_wait(drain, 0, p.err);
    } else if (warp < kEpiWarps) {
        // ---------------- epilogue ----------------
        const int quarter = warp & 3, group = warp >> 2;
        const int trow = quarter * 32 + lane;  // tile row of this thread (TMEM lane)
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        unsigned char* h_gen = gbase + kOffH;
        unsigned char* o_gen = gbase + kOffO + (size_t)warp * kOutBufs * kOutBox;
        uint32_t j = 0;
        int obuf = 0;
        bool ok = true;
        for (int t = blockIdx.x; ok && t < p.n_tiles; t += gridDim.x) {
            for (int l = 0; ok && l < p.L; ++l) {
                const bool hidden_l = l < p.L - 1;
                const int cw = layer_n(p, l) / kColGroups;  // this warp's columns of the chunk
                const float* bias = p.bias[l];
                for (int c = 0; ok && c < layer_chunks(p, l); ++c, ++j) {
                    const uint32_t b = j & 1;
                    const bool got = tc::mbar_wait(acc_full + 8 * b, (j >> 1) & 1, p.err);
                    if (!__all_sync(0xffffffffu, got && !*s_abort)) { ok = false; break; }
                    tc::tc_fence_after();
#pragma unroll 1
                    for (int cc = 0; cc < cw; cc += 32) {
                        const int col = group * cw + cc;  // column within the chunk
                        // an output box wholly past n_out is neither staged nor stored, so that every
                        // staged buffer has its store committed (the buffer alternation relies on it)
                        if (!hidden_l && c * 256 + col >= p.n_out) continue;
                        uint32_t r[32];
                        tc::tmem_ld32(taddr + lane_base + 256u * b + (uint32_t)col, r);
                        tc::tmem_ld_wait();
                        const float4* b4 = reinterpret_cast<const float4*>(bias + c * 256 + col);
                        if (hidden_l) {
                            // 32 activations = 4 chunks of 16 B in k-block col / 64 of H
                            unsigned char* rowp = h_gen + (col >> 6) * kKBlockBytes + trow * 128;
                            const int q0 = (col & 63) >> 3;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float4 b0 = __ldg(&b4[2 * q]), b1 = __ldg(&b4[2 * q + 1]);
                                const float* v = reinterpret_cast<const float*>(r) + 8 * q;
                                uint4 o;
                                o.x = pack_bf16(silu_tanh(v[0] + b0.x), silu_tanh(v[1] + b0.y));
                                o.y = pack_bf16(silu_tanh(v[2] + b0.z), silu_tanh(v[3] + b0.w));
                                o.z = pack_bf16(silu_tanh(v[4] + b1.x), silu_tanh(v[5] + b1.y));
                                o.w = pack_bf16(silu_tanh(v[6] + b1.z), silu_tanh(v[7] + b1.w));
                                *reinterpret_cast<uint4*>(rowp + (((q0 + q) ^ (trow & 7)) << 4)) = o;
                            }
                        } else {
                            // the staging buffer's previous store has finished reading it
                            if (lane == 0) bulk_wait_read<kOutBufs - 1>();
                            __syncwarp();
                            unsigned char* rowp = o_gen + obuf * kOutBox + lane * 128;
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const float4 bb = __ldg(&b4[q]);
                                float4 o;
                                o.x = __uint_as_float(r[4 * q]) + bb.x;
                                o.y = __uint_as_float(r[4 * q + 1]) + bb.y;
                                o.z = __uint_as_float(r[4 * q + 2]) + bb.z;
                                o.w = __uint_as_float(r[4 * q + 3]) + bb.w;
                                *reinterpret_cast<float4*>(rowp + ((q ^ (lane & 7)) << 4)) = o;
                            }
                            fence_proxy_async();
                            __syncwarp();
                            if (lane == 0) {
                                tma_store_2d(&p.y, sO + (uint32_t)(warp * kOutBufs + obuf) * kOutBox, c * 256 + col,
                                             t * 128 + quarter * 32);
                                bulk_commit();
                            }
                            obuf = obuf + 1 == kOutBufs ? 0 : obuf + 1;
                        }
                    }
                    tc::tc_fence_before();
                    if (hidden_l) fence_proxy_async();  // H writes before the next layer's MMAs read them
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(acc_empty + 8 * b);
                        if (hidden_l) mbar_arrive(h_full);
                    }
                }
            }
        }
        if (!ok) *s_abort = 1;
        if (lane == 0) bulk_wait_all();
        __syncwarp();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(taddr, 512);
    }
}

}  // namespace fused
}  // namespace xmc
