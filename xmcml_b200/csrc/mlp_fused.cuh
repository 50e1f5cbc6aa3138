// Fused forward pass (inference) of the surrogate MLP on the sm_100a tensor cores.
//
// One persistent CTA per SM walks its 128-row tiles of the input two at a time, in two slots. For each
// tile every layer runs in turn with the tile's activations kept in the slot's shared-memory buffer H,
// so nothing but the inputs, the weights (L2-resident, streamed by TMA) and the FP32 outputs touches
// global memory:
//
//   layer 0        A = X tile [128 x 64]  (TMA, into k-block 0 of H)  B = W_0 [hidden x 64]
//   hidden 1..L-2  A = H [128 x hidden]   (shared memory)             B = W_l [hidden x hidden]
//   output L-1     A = H                                              B = W_out, 256 output columns per chunk
//
// The two slots alternate job by job (one layer, or one 256-column output chunk, of a tile): while
// the epilogue drains one slot's accumulator the tensor cores compute the other slot's, so a hidden
// layer's MMAs of one tile overlap the bias + SiLU epilogue of the other, and the output stores of one
// overlap the MMAs of the other.
//
// Roles (576 threads): warp 16 lane 0 issues the TMA loads (the X tiles and the weights, 64 K-columns
// per stage through a 2-stage ring); warp 17 lane 0 issues tcgen05.mma (M = 128, N = hidden or 256,
// K = 16) into its slot's 256-column TMEM accumulator and commits to mbarriers; warps 0-15 drain an
// accumulator with tcgen05.ld (warp w: TMEM lanes 32 (w % 4).., the column quarter w / 4). A hidden
// layer's epilogue adds the bias, applies SiLU and writes the BF16 activations back into the slot's H
// in the 128-byte-swizzled K-major layout the next layer's MMAs read (then fence.proxy.async and an
// mbarrier arrive); the output epilogue adds the bias and stores 32-row x 16-column FP32 boxes
// through a 64-byte-swizzled staging buffer per warp with TMA
// (cp.async.bulk.tensor store). The X tile of a slot's next tile lands in H once the MMAs of the
// slot's last output chunk have read it.
//
// Every mbarrier wait is bounded (tc::kWaitNs); after a failed wait the role sets *err, stops
// issuing work and the CTA still drains its copies and MMAs and releases TMEM.
#pragma once

#include "tc_gemm.cuh"

namespace xmc {
namespace fused {

constexpr int kMaxL = 9;
constexpr int kSlots = 2;     // tiles in flight per CTA
constexpr int kEpiWarps = 16;  // warp w reads TMEM lanes 32 (w % 4).. and column quarter w / 4
constexpr int kColGroups = kEpiWarps / 4;
constexpr int kThreads = 32 * (kEpiWarps + 2);
constexpr int kWStages = 2;                // weight ring depth (stages of 64 K-columns)
constexpr int kXBytes = 128 * 64 * 2;      // input tile, one 64-column k-block
constexpr int kKBlockBytes = 128 * 128;    // one 64-column k-block of a 128-row operand
constexpr int kHBytes = 4 * kKBlockBytes;  // activations of one slot, hidden <= 256
constexpr int kWBytes = 256 * 64 * 2;      // weight stage: up to 256 rows x 64 columns
constexpr int kOutCols = 16;               // columns of one output box (64 bytes of FP32)
constexpr int kOutBox = 32 * kOutCols * 4; // one warp's 32 x 16 FP32 output box
constexpr int kOutBufs = 1;                // output staging boxes per epilogue warp
constexpr int kOffH = 0;
constexpr int kOffW = kOffH + kSlots * kHBytes;
constexpr int kOffO = kOffW + kWStages * kWBytes;
constexpr int kOffBar = kOffO + kEpiWarps * kOutBufs * kOutBox;
constexpr int kSmemBytes = kOffBar + 256 + 1024;  // barriers, TMEM slot, abort flag; alignment slack
static_assert(kSmemBytes <= 232448, "fused forward exceeds the shared memory of one CTA");
static_assert(kXBytes == kKBlockBytes, "the X tile is k-block 0 of a slot's activations");

struct Params {
    CUtensorMap x;             // bf16 [rows x 64], box 64 x 128, 128-byte swizzle
    CUtensorMap w[kMaxL];      // bf16 [out_l x in_l], box 64 x (hidden or 256), 128-byte swizzle
    CUtensorMap y;             // fp32 [rows x n_out], box 16 x 32, 64-byte swizzle
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

// Epilogue of 32 accumulator columns of a hidden layer: bias + SiLU, written as BF16 (4 chunks of 16 B)
// into k-block col / 64 of the slot's activations, in the 128-byte-swizzled K-major layout.
__device__ __forceinline__ void epi_hidden(unsigned char* h_gen, int col, int trow, const uint32_t (&r)[32],
                                           const float4 (&b)[8]) {
    unsigned char* rowp = h_gen + (col >> 6) * kKBlockBytes + trow * 128;
    const int q0 = (col & 63) >> 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 b0 = b[2 * q], b1 = b[2 * q + 1];
        const float* v = reinterpret_cast<const float*>(r) + 8 * q;
        uint4 o;
        o.x = pack_bf16(silu_tanh(v[0] + b0.x), silu_tanh(v[1] + b0.y));
        o.y = pack_bf16(silu_tanh(v[2] + b0.z), silu_tanh(v[3] + b0.w));
        o.z = pack_bf16(silu_tanh(v[4] + b1.x), silu_tanh(v[5] + b1.y));
        o.w = pack_bf16(silu_tanh(v[6] + b1.z), silu_tanh(v[7] + b1.w));
        *reinterpret_cast<uint4*>(rowp + (((q0 + q) ^ (trow & 7)) << 4)) = o;
    }
}

// Epilogue of 32 accumulator columns of the output layer (output columns gcol..): bias added, stored as
// two 32-row x 16-column FP32 boxes through the warp's staging buffers (o_gen / o_sm, generic and
// shared addresses; kOutBufs of them, in turn). Boxes wholly past n_out are neither staged nor
// stored, so that every staged buffer has its store committed (the rotation relies on it).
// Returns the next buffer.
__device__ __forceinline__ int epi_output(const Params& p, unsigned char* o_gen, uint32_t o_sm, int obuf, int gcol,
                                           int row0, int lane, const uint32_t (&r)[32], const float4 (&b)[8]) {
#pragma unroll
    for (int hb = 0; hb < 2; ++hb) {
        const int bcol = gcol + hb * kOutCols;
        if (bcol >= p.n_out) break;
        // the staging buffer's previous store (kOutBufs boxes back) has read it
        if (lane == 0) bulk_wait_read<kOutBufs - 1>();
        __syncwarp();
        // 64-byte rows, 16-byte chunk q of row `lane` at chunk q ^ ((lane >> 1) & 3)
        unsigned char* rowp = o_gen + obuf * kOutBox + lane * 64;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 bb = b[hb * 4 + q];
            const int e = hb * 16 + 4 * q;
            float4 o;
            o.x = __uint_as_float(r[e]) + bb.x;
            o.y = __uint_as_float(r[e + 1]) + bb.y;
            o.z = __uint_as_float(r[e + 2]) + bb.z;
            o.w = __uint_as_float(r[e + 3]) + bb.w;
            *reinterpret_cast<float4*>(rowp + ((q ^ ((lane >> 1) & 3)) << 4)) = o;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            tma_store_2d(&p.y, o_sm + (uint32_t)obuf * kOutBox, bcol, row0);
            bulk_commit();
        }
        obuf = obuf + 1 == kOutBufs ? 0 : obuf + 1;
    }
    return obuf;
}

// a per-slot counter pair kept in registers (indexing a local array by the slot would put it in
// local memory)
struct SlotCount {
    uint32_t v0 = 0, v1 = 0;
    __device__ uint32_t get(int s) const { return s ? v1 : v0; }
    __device__ uint32_t take(int s) {  // the value, then +1
        const uint32_t v = get(s);
        if (s) v1 = v + 1;
        else v0 = v + 1;
        return v;
    }
};

// The CTA's jobs in the order every role takes them. A job is one layer (or one 256-column output
// chunk) of one tile; a tile has L - 1 + out_chunks jobs. Slot s takes this CTA's tiles s, s + 2,
// s + 4, ... (tile blockIdx.x + i gridDim.x for the CTA's i-th tile); the slots alternate job by job
// while both have tiles left, and each moves on to its next tile on its own.
struct JobOrder {
    int i0, l0, c0, i1, l1, c1;  // per slot: the CTA's tile ordinal, layer and chunk of its next job
    int my_tiles, turn;
    __device__ explicit JobOrder(int my_tiles_) : i0(0), l0(0), c0(0), i1(1), l1(0), c1(0), my_tiles(my_tiles_), turn(0) {}
    // the next job (slot, tile, layer, chunk); false when both slots are done
    __device__ bool next(const Params& p, int& s, int& tile, int& layer, int& chunk) {
        const bool a0 = i0 < my_tiles, a1 = i1 < my_tiles;
        if (!a0 && !a1) return false;
        s = a0 && a1 ? turn : (a0 ? 0 : 1);
        turn = s ^ 1;
        int i = s ? i1 : i0, l = s ? l1 : l0, c = s ? c1 : c0;
        tile = (int)blockIdx.x + i * (int)gridDim.x;
        layer = l;
        chunk = c;
        if (++c == layer_chunks(p, l)) {
            c = 0;
            if (++l == p.L) l = 0, i += 2;
        }
        if (s) i1 = i, l1 = l, c1 = c;
        else i0 = i, l0 = l, c0 = c;
        return true;
    }
};

__global__ void __launch_bounds__(kThreads, 1) mlp_forward_kernel(const __grid_constant__ Params p) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = tc::smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t sH = base + kOffH, sW = base + kOffW, sO = base + kOffO;
    const uint32_t bar = base + kOffBar;
    // two of each per slot (or per ring stage), 8 bytes apart
    const uint32_t w_full = bar, w_empty = bar + 16, x_full = bar + 32, x_empty = bar + 48;
    const uint32_t acc_full = bar + 64, acc_empty = bar + 80, h_full = bar + 96, drain = bar + 112;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(gbase + kOffBar + 192);
    volatile int* s_abort = reinterpret_cast<volatile int*>(gbase + kOffBar + 196);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_u32(s_tmem), 512);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 32 * kEpiWarps) {
        for (int s = 0; s < 2; ++s) {
            tc::mbar_init(w_full + 8 * s, 1);
            tc::mbar_init(w_empty + 8 * s, 1);
            tc::mbar_init(x_full + 8 * s, 1);
            tc::mbar_init(x_empty + 8 * s, 1);
            tc::mbar_init(acc_full + 8 * s, 1);
            tc::mbar_init(acc_empty + 8 * s, kEpiWarps);
            tc::mbar_init(h_full + 8 * s, kEpiWarps);
        }
        tc::mbar_init(drain, 1);
        *s_abort = 0;
        tc::mbar_fence_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *s_tmem;
    // this CTA's tiles are blockIdx.x + i gridDim.x, i < my_tiles (JobOrder deals them to the slots)
    const int my_tiles = (p.n_tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;

    if (warp == kEpiWarps && lane == 0) {
        // ---------------- TMA producer ----------------
        tc::tma_prefetch_desc(&p.x);
        uint32_t it = 0;
        SlotCount xc;
        bool ok = true;
        JobOrder jobs(my_tiles);
        int s, t, l, c;
        while (ok && jobs.next(p, s, t, l, c)) {
            const int n = layer_n(p, l), nk = layer_kblocks(p, l);
            if (l == 0) {
                // the slot's activations are free once its previous tile's last MMAs ran
                if (!(ok = tc::mbar_wait(x_empty + 8 * s, (xc.get(s) & 1) ^ 1, p.err))) break;
                tc::mbar_expect_tx(x_full + 8 * s, kXBytes);
                tc::tma_load_2d(sH + s * kHBytes, &p.x, x_full + 8 * s, 0, t * 128);
                xc.take(s);
            }
            for (int kb = 0; kb < nk; ++kb, ++it) {
                const int st = it % kWStages;
                if (!(ok = tc::mbar_wait(w_empty + 8 * st, ((it / kWStages) & 1) ^ 1, p.err))) break;
                tc::mbar_expect_tx(w_full + 8 * st, (uint32_t)n * 128u);
                tc::tma_load_2d(sW + st * kWBytes, &p.w[l], w_full + 8 * st, kb * 64, c * 256);
            }
        }
        if (!ok) *s_abort = 1;
        // every issued load has landed before the CTA exits
        for (uint32_t i = it > kWStages ? it - kWStages : 0; i < it; ++i)
            tc::mbar_wait(w_full + 8 * (i % kWStages), (i / kWStages) & 1, p.err);
        for (int s = 0; s < kSlots; ++s)
            if (xc.get(s) > 0) tc::mbar_wait(x_full + 8 * s, (xc.get(s) - 1) & 1, p.err);
    } else if (warp == kEpiWarps + 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        uint32_t it = 0;
        SlotCount ja, xm, hw;
        bool ok = true;
        const uint32_t idesc_h = tc::idesc_bf16(128, p.hidden), idesc_o = tc::idesc_bf16(128, 256);
        JobOrder jobs(my_tiles);
        int s, t, l, c;
        while (ok && jobs.next(p, s, t, l, c)) {
            const int nk = layer_kblocks(p, l), nc = layer_chunks(p, l);
            const uint32_t idesc = l < p.L - 1 ? idesc_h : idesc_o;
            if (!(ok = tc::mbar_wait(acc_empty + 8 * s, (ja.get(s) & 1) ^ 1, p.err))) break;
            if (l == 0) ok = tc::mbar_wait(x_full + 8 * s, xm.take(s) & 1, p.err);
            else if (c == 0) ok = tc::mbar_wait(h_full + 8 * s, hw.take(s) & 1, p.err);
            if (!ok || *s_abort) { ok = false; break; }
            tc::tc_fence_after();
            const uint32_t d = taddr + 256u * s, a0 = sH + s * kHBytes;
            for (int kb = 0; kb < nk; ++kb, ++it) {
                const int st = it % kWStages;
                if (!(ok = tc::mbar_wait(w_full + 8 * st, (it / kWStages) & 1, p.err))) break;
                tc::tc_fence_after();
                const uint32_t sa = a0 + kb * kKBlockBytes, sb = sW + st * kWBytes;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    tc::umma_bf16(d, tc::sw128_desc(sa + 32 * kk), tc::sw128_desc(sb + 32 * kk), idesc, (kb | kk) != 0);
                tc::umma_commit(w_empty + 8 * st);
            }
            if (!ok) break;
            // the slot's last MMAs of this tile: its activations may take the next X tile
            if (l == p.L - 1 && c == nc - 1) tc::umma_commit(x_empty + 8 * s);
            tc::umma_commit(acc_full + 8 * s);
            ja.take(s);
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
        unsigned char* o_gen = gbase + kOffO + (size_t)warp * kOutBufs * kOutBox;
        const uint32_t o_sm = sO + (uint32_t)(warp * kOutBufs * kOutBox);
        SlotCount je;
        int obuf = 0;
        bool ok = true;
        JobOrder jobs(my_tiles);
        int s, t, l, c;
        while (ok && jobs.next(p, s, t, l, c)) {
            const bool hidden_l = l < p.L - 1;
            const int cw = layer_n(p, l) / kColGroups;  // this warp's columns of the chunk
            const float* bias = p.bias[l];
            const bool got = tc::mbar_wait(acc_full + 8 * s, je.take(s) & 1, p.err);
            if (!__all_sync(0xffffffffu, got && !*s_abort)) { ok = false; break; }
            tc::tc_fence_after();
            unsigned char* h_gen = gbase + kOffH + (size_t)s * kHBytes;
            // 32 columns per round; the bias loads are issued with the TMEM load, before the wait
#pragma unroll 1
            for (int cc = 0; cc < cw; cc += 32) {
                const int col = group * cw + cc;  // column within the chunk
                const int gcol = c * 256 + col;
                if (!hidden_l && gcol >= p.n_out) continue;
                uint32_t r[32];
                tc::tmem_ld32(taddr + lane_base + 256u * s + (uint32_t)col, r);
                const float4* b4 = reinterpret_cast<const float4*>(bias + gcol);
                float4 bv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) bv[q] = __ldg(&b4[q]);
                tc::tmem_ld_wait();
                if (hidden_l) epi_hidden(h_gen, col, trow, r, bv);
                else obuf = epi_output(p, o_gen, o_sm, obuf, gcol, t * 128 + quarter * 32, lane, r, bv);
            }
            tc::tc_fence_before();
            if (hidden_l) fence_proxy_async();  // H writes before the next layer's MMAs read them
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(acc_empty + 8 * s);
                if (hidden_l) mbar_arrive(h_full + 8 * s);
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
