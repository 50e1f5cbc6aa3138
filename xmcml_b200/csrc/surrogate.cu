// Surrogate MLP on the tensor cores: training (forward, backward, Adam) and inference of a fully
// connected network with SiLU hidden layers, BF16 weights and activations and FP32 accumulation,
// built on the tcgen05 GEMM of tc_gemm.cuh. No counterpart in the reference; the network maps the
// optical properties of a layered model to its ring- and time-resolved reflectance and is
// trained on tallies of the batched Monte Carlo (batch.cu).
//
// Layer l computes Z_l = A_{l-1} W_l^T + b_l with A_{-1} = X (inputs zero-padded to 64 columns)
// and A_l = SiLU(Z_l) for hidden layers; the last layer is linear (outputs padded to a multiple of
// 256 with zero weights). Every GEMM is D = A . B^T with both operands K-major:
//   forward            A = A_{l-1} [rows x in]     B = W_l   [out x in]
//   backward (data)    A = dZ_l    [rows x out]    B = W_l^T [in x out]      -> dA_{l-1}, x SiLU'(Z_{l-1})
//   backward (weights) A = dZ_l^T  [out x rows]    B = A_{l-1}^T [in x rows] -> dW_l (split over rows)
// so the forward epilogues also write A_l^T and the backward epilogues dZ^T (coalesced: the 32
// lanes of a warp hold 32 consecutive rows), and each Adam step refreshes W_l and W_l^T in BF16
// from the FP32 master weights. Loss: mean squared error over rows x n_out.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cudaTypedefs.h>

#include "mlp_fused.cuh"
#include "photon.cuh"
#include "tc_gemm.cuh"
#include "xmc_internal.h"

using bf16 = __nv_bfloat16;

namespace xmc {
namespace {

constexpr int kInPad = 64;
constexpr int kMaxLayers = 9;

__device__ __forceinline__ float f32(uint32_t r) { return __uint_as_float(r); }

__device__ __forceinline__ void load_bf16x32(const bf16* p, float (&v)[32]) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint4 u = q[j];
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
            const float2 f = __bfloat1622float2(h);
            v[8 * j + 2 * i] = f.x;
            v[8 * j + 2 * i + 1] = f.y;
        }
    }
}

// The warp's 32 rows x 32 columns (lane t holds row row0 + t) to a row-major matrix through the
// warp's shared-memory tile: 32 stores, each one row segment of 32 consecutive elements.
__device__ __forceinline__ void warp_rows_f32(float* sw, const float (&v)[32], float* dst, size_t ld, int row0, int col0,
                                              int ncols, int lane) {
#pragma unroll
    for (int j = 0; j < 32; ++j) sw[lane * 33 + j] = v[j];
    __syncwarp();
    if (col0 + lane < ncols) {
#pragma unroll 4
        for (int k = 0; k < 32; ++k) dst[(size_t)(row0 + k) * ld + col0 + lane] = sw[k * 33 + lane];
    }
    __syncwarp();
}
__device__ __forceinline__ void warp_rows_bf16(float* sw, const float (&v)[32], bf16* dst, size_t ld, int row0, int col0,
                                               int lane) {
#pragma unroll
    for (int j = 0; j < 32; ++j) sw[lane * 33 + j] = v[j];
    __syncwarp();
#pragma unroll 4
    for (int k = 0; k < 32; ++k) dst[(size_t)(row0 + k) * ld + col0 + lane] = __float2bfloat16_rn(sw[k * 33 + lane]);
    __syncwarp();
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------- epilogues

// Plain FP32 store of the accumulator (split-K partials at blockIdx.z * split_stride).
struct EpiF32 {
    float* d;
    int ld;
    size_t split_stride;
    __device__ void apply(int row, int col0, const uint32_t (&r)[32], int lane, float* sw) const {
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = f32(r[j]);
        warp_rows_f32(sw, v, d + blockIdx.z * split_stride, (size_t)ld, row - lane, col0, col0 + 32, lane);
    }
};

// Hidden layer: Z = acc + b, A = SiLU(Z); A row-major always, Z and A^T when training.
struct EpiHidden {
    const float* bias;
    bf16* a;
    int lda;
    bf16* z;    // nullable
    bf16* at;   // nullable, [cols x ldt]
    int ldt;
    __device__ void apply(int row, int col0, const uint32_t (&r)[32], int lane, float* sw) const {
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = f32(r[j]) + __ldg(&bias[col0 + j]);
        if (z) warp_rows_bf16(sw, v, z, (size_t)lda, row - lane, col0, lane);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = silu(v[j]);
        warp_rows_bf16(sw, v, a, (size_t)lda, row - lane, col0, lane);
        if (at) {
#pragma unroll
            for (int j = 0; j < 32; ++j) at[(size_t)(col0 + j) * ldt + row] = __float2bfloat16_rn(v[j]);
        }
    }
};

// Output layer: Y = acc + b for the first n_out columns. Training (t != nullptr): the gradient of
// the (optionally per-output weighted) mean squared error dY = scale w (Y - T) (0 in the padding
// columns), row-major and transposed, and the sum of w (Y - T)^2 added to loss[*step].
struct EpiOut {
    const float* bias;
    float* y;  // nullable, [rows x ldy]
    int ldy;
    int n_out;
    const float* t;  // nullable, [rows x ldtg]
    int ldtg;
    bf16* dy;
    int lddy;
    bf16* dyt;
    int lddyt;
    float scale;
    const float* colw;  // nullable: per-output weight of the squared error
    float* loss;
    const int* step;
    __device__ void apply(int row, int col0, const uint32_t (&r)[32], int lane, float* sw) const {
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = f32(r[j]) + __ldg(&bias[col0 + j]);
        if (y && col0 < n_out) warp_rows_f32(sw, v, y, (size_t)ldy, row - lane, col0, n_out, lane);
        if (t) {
            float se = 0.0f;
            const float* tp = t + (size_t)row * ldtg;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int c = col0 + j;
                const float d = c < n_out ? v[j] - __ldg(&tp[c]) : 0.0f;
                const float wd = (colw && c < n_out) ? d * __ldg(&colw[c]) : d;
                se = fmaf(wd, d, se);
                v[j] = wd * scale;
            }
            warp_rows_bf16(sw, v, dy, (size_t)lddy, row - lane, col0, lane);
#pragma unroll
            for (int j = 0; j < 32; ++j) dyt[(size_t)(col0 + j) * lddyt + row] = __float2bfloat16_rn(v[j]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
            if (lane == 0) atomicAdd(loss + *step, se);
        }
    }
};

// Backward through SiLU: dZ = acc * SiLU'(Z), row-major and transposed.
struct EpiBwd {
    const bf16* z;
    int ldz;
    bf16* dz;
    bf16* dzt;
    int ldt;
    __device__ void apply(int row, int col0, const uint32_t (&r)[32], int lane, float* sw) const {
        float zv[32], v[32];
        load_bf16x32(z + (size_t)row * ldz + col0, zv);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = f32(r[j]) * dsilu(zv[j]);
        warp_rows_bf16(sw, v, dz, (size_t)ldz, row - lane, col0, lane);
#pragma unroll
        for (int j = 0; j < 32; ++j) dzt[(size_t)(col0 + j) * ldt + row] = __float2bfloat16_rn(v[j]);
    }
};

// ---------------------------------------------------------------- small kernels

// FP32 host inputs [rows x n_in] -> bf16 [rows x 64] (zero padded), and optionally transposed.
__global__ void pack_inputs_kernel(const float* __restrict__ x, int rows, int n_in, bf16* __restrict__ xb,
                                   bf16* __restrict__ xt, int ldt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * kInPad) return;
    const int r = i / kInPad, c = i % kInPad;
    const bf16 v = __float2bfloat16_rn(c < n_in ? x[(size_t)r * n_in + c] : 0.0f);
    xb[i] = v;
    if (xt) xt[(size_t)c * ldt + r] = v;
}

// Minibatch of `rows` rows drawn with replacement from the device data set (Philox keyed by seed,
// counter (step, row)): inputs (bf16, padded, and transposed) and FP32 targets.
__global__ void gather_kernel(const bf16* __restrict__ ds_x, const float* __restrict__ ds_t, int ds_rows, int n_out,
                              int rows, uint32_t k0, uint32_t k1, const int* __restrict__ step, bf16* __restrict__ xb,
                              bf16* __restrict__ xt, float* __restrict__ tb) {
    const int r = blockIdx.x;
    __shared__ int src;
    if (threadIdx.x == 0) {
        const uint4 u = philox4x32_10(make_uint4((uint32_t)r, (uint32_t)*step, 0x6d6c70u, 0u), k0, k1);
        src = (int)(((unsigned long long)u.x * (unsigned long long)ds_rows) >> 32);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kInPad; c += blockDim.x) {
        const bf16 v = ds_x[(size_t)src * kInPad + c];
        xb[(size_t)r * kInPad + c] = v;
        xt[(size_t)c * rows + r] = v;
    }
    for (int c = threadIdx.x; c < n_out; c += blockDim.x) tb[(size_t)r * n_out + c] = ds_t[(size_t)src * n_out + c];
}

__global__ void step_kernel(int* step, float* loss) {
    *step += 1;
    loss[*step] = 0.0f;
}

// db[n] = sum over rows of dZ^T[n][row] (fixed order: deterministic)
__global__ void bias_grad_kernel(const bf16* __restrict__ dzt, int rows, float* __restrict__ db) {
    const int n = blockIdx.x;
    float s = 0.0f;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) s += __bfloat162float(dzt[(size_t)n * rows + i]);
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = red[0];
}

// g[i] = sum over splits of part[s][i] (fixed order)
__global__ void split_sum_kernel(const float* __restrict__ part, int splits, size_t n, float* __restrict__ g) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < splits; ++k) s += part[(size_t)k * n + i];
        g[i] = s;
    }
}

// Adam (Kingma & Ba, 2015) on FP32 master parameters p[rows x cols] with bias correction from the
// step counter; refreshes the bf16 copy (row-major) and its transpose when given.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            int rows, int cols, int valid_rows, float lr, float b1, float b2, float eps,
                            const int* __restrict__ step, bf16* __restrict__ w16, bf16* __restrict__ w16t) {
    const size_t n = (size_t)rows * cols;
    const int t = *step;
    const float c1 = 1.0f - __powf(b1, (float)t), c2 = 1.0f - __powf(b2, (float)t);
    const float alpha = lr * sqrtf(c2) / c1;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        float w = p[i];
        if (r < valid_rows) {
            const float gi = g[i];
            const float mi = b1 * m[i] + (1.0f - b1) * gi;
            const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            w -= alpha * mi / (sqrtf(vi) + eps);
            p[i] = w;
        }
        if (w16) {
            const bf16 h = __float2bfloat16_rn(w);
            w16[i] = h;
            w16t[(size_t)c * rows + r] = h;
        }
    }
}

// FP32 master -> bf16 copy and transpose (after set_params)
__global__ void refresh_kernel(const float* __restrict__ p, int rows, int cols, bf16* __restrict__ w16, bf16* __restrict__ w16t) {
    const size_t n = (size_t)rows * cols;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        const bf16 h = __float2bfloat16_rn(p[i]);
        w16[i] = h;
        w16t[(size_t)c * rows + r] = h;
    }
}

// ---------------------------------------------------------------- host helpers

int mfail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}

#define XM_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return mfail(XMC_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

std::mutex g_encode_mutex;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder() {
    std::lock_guard<std::mutex> lock(g_encode_mutex);
    if (g_encode) return XMC_OK;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess)
        return mfail(XMC_ERR_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return XMC_OK;
}

// Tensor map of a row-major bf16 matrix [rows x cols] read in boxes of box_rows x 64 with the
// 128-byte swizzle (the layout the GEMM's shared-memory descriptors describe).
int make_map(CUtensorMap* map, const void* ptr, uint64_t rows, uint64_t cols, uint32_t box_rows) {
    int st = get_encoder();
    if (st) return st;
    if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (cols * 2) % 16 || cols % tc::kBK || box_rows > 256)
        return mfail(XMC_ERR_INVALID_INPUT, "tensor map: misaligned operand");
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)tc::kBK, box_rows};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mfail(XMC_ERR_DEVICE, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return XMC_OK;
}

// Tensor map of the FP32 output [rows x n_out] stored in boxes of 32 rows x 16 columns with the
// 64-byte swizzle (the fused forward's staging layout); columns past n_out are clipped by the store.
int make_out_map(CUtensorMap* map, float* y, uint64_t rows, uint64_t n_out) {
    int st = get_encoder();
    if (st) return st;
    if ((reinterpret_cast<uintptr_t>(y) & 15) || (n_out * 4) % 16)
        return mfail(XMC_ERR_INVALID_INPUT, "tensor map: misaligned output");
    const cuuint64_t dims[2] = {n_out, rows};
    const cuuint64_t strides[1] = {n_out * 4};
    const cuuint32_t box[2] = {(cuuint32_t)fused::kOutCols, 32};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, y, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mfail(XMC_ERR_DEVICE, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return XMC_OK;
}

template <int BN, class Epi>
int set_smem_attr() {
    static bool done = false;  // per template instance; set once per process (attribute is per function)
    if (done) return XMC_OK;
    XM_CUDA(cudaFuncSetAttribute(tc::gemm_kernel<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::smem_bytes(BN)));
    done = true;
    return XMC_OK;
}

// D = A[rows_a x k] . B[n x k]^T with A, B device bf16 row-major; grid (n / BN, rows_a / 128, splits).
template <int BN, class Epi>
int launch_gemm(const void* a, int rows_a, const void* b, int n, int k, int splits, const Epi& epi, int* err,
                cudaStream_t stream) {
    if (rows_a % tc::kBM || n % BN || k % (tc::kBK * splits) || splits < 1)
        return mfail(XMC_ERR_INVALID_INPUT, "gemm: shape not a multiple of the tile");
    int st = set_smem_attr<BN, Epi>();
    if (st) return st;
    CUtensorMap ma, mb;
    st = make_map(&ma, a, (uint64_t)rows_a, (uint64_t)k, tc::kBM);
    if (st) return st;
    st = make_map(&mb, b, (uint64_t)n, (uint64_t)k, BN);
    if (st) return st;
    const dim3 grid(n / BN, rows_a / tc::kBM, splits);
    tc::gemm_kernel<BN, Epi><<<grid, tc::kThreads, tc::smem_bytes(BN), stream>>>(ma, mb, k / tc::kBK / splits, err, epi);
    XM_CUDA(cudaGetLastError());
    return XMC_OK;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace
}  // namespace xmc

using namespace xmc;

// ---------------------------------------------------------------- model

struct xmc_mlp {
    xmc_mlp_spec spec{};
    int L = 0;                      // layers (hidden + 1)
    int in[kMaxLayers], out[kMaxLayers];   // padded dimensions
    int valid_out[kMaxLayers];             // rows of W that are real (n_out for the last layer)
    int cap = 0;                    // row capacity
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int* d_err = nullptr;
    int* d_step = nullptr;
    float* d_loss = nullptr;        // [max_steps + 1]
    int loss_cap = 0;
    float *w32[kMaxLayers] = {}, *b32[kMaxLayers] = {};
    float *mw[kMaxLayers] = {}, *vw[kMaxLayers] = {}, *mb[kMaxLayers] = {}, *vb[kMaxLayers] = {};
    float *gw[kMaxLayers] = {}, *gb[kMaxLayers] = {};
    bf16 *w16[kMaxLayers] = {}, *w16t[kMaxLayers] = {};
    // activations [cap x width] (and transposes [width x cap])
    bf16 *x = nullptr, *xt = nullptr;
    bf16 *a[kMaxLayers] = {}, *at[kMaxLayers] = {}, *z[kMaxLayers] = {};
    bf16 *dz[kMaxLayers] = {}, *dzt[kMaxLayers] = {};
    float *y = nullptr, *t = nullptr, *xin = nullptr;
    float* colw = nullptr;          // per-output loss weights, or null
    float* part = nullptr;
    size_t part_floats = 0;
    // data set
    bf16* ds_x = nullptr;
    float* ds_t = nullptr;
    int ds_rows = 0;
    std::map<int, cudaGraphExec_t> train_graphs;  // by batch rows (hyper-parameters in key below)
    std::map<int, cudaGraphExec_t> fwd_graphs;
    float g_lr = 0, g_b1 = 0, g_b2 = 0, g_eps = 0;
    uint64_t g_seed = 0;
    float* h_y = nullptr;           // pinned staging of the outputs read back by xmc_mlp_forward (lazy)
    size_t h_y_floats = 0;
    cudaEvent_t ev_chunk[8] = {};   // completion of each chunk of that read-back (lazy)
};

namespace xmc {
namespace {

void free_mlp(xmc_mlp* m) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m) return;
    cudaSetDevice(m->spec.device);
    for (auto& kv : m->train_graphs) cudaGraphExecDestroy(kv.second);
    for (auto& kv : m->fwd_graphs) cudaGraphExecDestroy(kv.second);
    std::vector<void*> d = {m->d_err, m->d_step, m->d_loss, m->x, m->xt, m->y, m->t, m->xin, m->part, m->ds_x, m->ds_t,
                            m->colw};
    for (int l = 0; l < kMaxLayers; ++l)
        for (void* p : {(void*)m->w32[l], (void*)m->b32[l], (void*)m->mw[l], (void*)m->vw[l], (void*)m->mb[l],
                        (void*)m->vb[l], (void*)m->gw[l], (void*)m->gb[l], (void*)m->w16[l], (void*)m->w16t[l],
                        (void*)m->a[l], (void*)m->at[l], (void*)m->z[l], (void*)m->dz[l], (void*)m->dzt[l]})
            d.push_back(p);
    for (void* p : d)
        if (p) cudaFree(p);
    for (cudaEvent_t e : m->ev)
        if (e) cudaEventDestroy(e);
    if (m->h_y) cudaFreeHost(m->h_y);
    for (cudaEvent_t e : m->ev_chunk)
        if (e) cudaEventDestroy(e);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

// split-K factor of the weight-gradient GEMM of layer l for `rows` rows: about 128 CTAs
int wgrad_splits(const xmc_mlp* m, int l, int rows) {
    const int tiles = m->out[l] / tc::kBM;
    const int kblocks = rows / tc::kBK;
    int s = std::max(1, 128 / tiles);
    while (s > 1 && (kblocks % s)) --s;
    return std::min(s, kblocks);
}

bool fused_forward_ok(const xmc_mlp* m) {
    return m->spec.forward_kernel == 0 && m->spec.n_out % 4 == 0 && m->L <= fused::kMaxL && m->in[0] == kInPad;
}

// Inference forward over `rows` rows of m->x into m->y with the fused kernel (mlp_fused.cuh).
int enqueue_fused_forward(xmc_mlp* m, int rows) {
    static bool attr = false;
    if (!attr) {
        XM_CUDA(cudaFuncSetAttribute(fused::mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     fused::kSmemBytes));
        attr = true;
    }
    fused::Params p;
    std::memset(&p, 0, sizeof(p));
    int st = make_map(&p.x, m->x, (uint64_t)rows, (uint64_t)kInPad, tc::kBM);
    for (int l = 0; !st && l < m->L; ++l) {
        st = make_map(&p.w[l], m->w16[l], (uint64_t)m->out[l], (uint64_t)m->in[l], l < m->L - 1 ? m->spec.hidden : 256);
        p.bias[l] = m->b32[l];
    }
    if (!st) st = make_out_map(&p.y, m->y, (uint64_t)rows, (uint64_t)m->spec.n_out);
    if (st) return st;
    p.L = m->L;
    p.hidden = m->spec.hidden;
    p.out_chunks = m->out[m->L - 1] / 256;
    p.n_tiles = rows / tc::kBM;
    p.n_out = m->spec.n_out;
    p.err = m->d_err;
    int sms = 0;
    XM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->spec.device));
    const int grid = std::min(p.n_tiles, sms);
    fused::mlp_forward_kernel<<<grid, fused::kThreads, fused::kSmemBytes, m->stream>>>(p);
    XM_CUDA(cudaGetLastError());
    return XMC_OK;
}

// Forward pass over `rows` rows of m->x (bf16, padded). Training: also Z, A^T, dY, loss.
int enqueue_forward(xmc_mlp* m, int rows, bool train) {
    if (!train && fused_forward_ok(m)) return enqueue_fused_forward(m, rows);
    const cudaStream_t st = m->stream;
    for (int l = 0; l < m->L; ++l) {
        const bf16* a_in = l == 0 ? m->x : m->a[l - 1];
        const int k = m->in[l];
        int s;
        if (l < m->L - 1) {
            EpiHidden e{m->b32[l], m->a[l], m->out[l], train ? m->z[l] : nullptr, train ? m->at[l] : nullptr, rows};
            s = m->out[l] == 256 ? launch_gemm<256>(a_in, rows, m->w16[l], m->out[l], k, 1, e, m->d_err, st)
                                 : launch_gemm<128>(a_in, rows, m->w16[l], m->out[l], k, 1, e, m->d_err, st);
        } else {
            EpiOut e{};
            e.bias = m->b32[l];
            e.n_out = m->spec.n_out;
            if (train) {
                e.y = nullptr;
                e.t = m->t;
                e.ldtg = m->spec.n_out;
                e.dy = m->dz[l];
                e.lddy = m->out[l];
                e.dyt = m->dzt[l];
                e.lddyt = rows;
                e.scale = 2.0f / ((float)rows * (float)m->spec.n_out);
                e.colw = m->colw;
                e.loss = m->d_loss;
                e.step = m->d_step;
            } else {
                e.y = m->y;
                e.ldy = m->spec.n_out;
            }
            s = launch_gemm<256>(a_in, rows, m->w16[l], m->out[l], k, 1, e, m->d_err, st);
        }
        if (s) return s;
    }
    return XMC_OK;
}

// Backward pass after enqueue_forward(train): gradients into gw / gb.
int enqueue_backward(xmc_mlp* m, int rows) {
    const cudaStream_t st = m->stream;
    for (int l = m->L - 1; l >= 0; --l) {
        // data gradient to the previous layer
        if (l > 0) {
            EpiBwd e{m->z[l - 1], m->out[l - 1], m->dz[l - 1], m->dzt[l - 1], rows};
            int s = m->in[l] == 256 ? launch_gemm<256>(m->dz[l], rows, m->w16t[l], m->in[l], m->out[l], 1, e, m->d_err, st)
                                    : launch_gemm<128>(m->dz[l], rows, m->w16t[l], m->in[l], m->out[l], 1, e, m->d_err, st);
            if (s) return s;
        }
        // weight gradient: dW = dZ^T . A_{l-1}, split over rows
        const int splits = wgrad_splits(m, l, rows);
        const bf16* bt = l == 0 ? m->xt : m->at[l - 1];
        const size_t n = (size_t)m->out[l] * m->in[l];
        EpiF32 e{m->part, m->in[l], n};
        int s;
        if (m->in[l] == 256) s = launch_gemm<256>(m->dzt[l], m->out[l], bt, m->in[l], rows, splits, e, m->d_err, st);
        else if (m->in[l] == 128) s = launch_gemm<128>(m->dzt[l], m->out[l], bt, m->in[l], rows, splits, e, m->d_err, st);
        else s = launch_gemm<64>(m->dzt[l], m->out[l], bt, m->in[l], rows, splits, e, m->d_err, st);
        if (s) return s;
        split_sum_kernel<<<296, 256, 0, st>>>(m->part, splits, n, m->gw[l]);
        bias_grad_kernel<<<m->out[l], 256, 0, st>>>(m->dzt[l], rows, m->gb[l]);
        XM_CUDA(cudaGetLastError());
    }
    return XMC_OK;
}

int enqueue_adam(xmc_mlp* m, float lr, float b1, float b2, float eps) {
    const cudaStream_t st = m->stream;
    for (int l = 0; l < m->L; ++l) {
        adam_kernel<<<296, 256, 0, st>>>(m->w32[l], m->gw[l], m->mw[l], m->vw[l], m->out[l], m->in[l], m->valid_out[l], lr, b1,
                                         b2, eps, m->d_step, m->w16[l], m->w16t[l]);
        adam_kernel<<<8, 256, 0, st>>>(m->b32[l], m->gb[l], m->mb[l], m->vb[l], m->out[l], 1, m->valid_out[l], lr, b1, b2,
                                       eps, m->d_step, nullptr, nullptr);
    }
    XM_CUDA(cudaGetLastError());
    return XMC_OK;
}

int check_err(xmc_mlp* m) {
    int e = 0;
    XM_CUDA(cudaMemcpy(&e, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(m->d_err, 0, sizeof(int));
        return mfail(XMC_ERR_DEVICE, "tensor-core GEMM: a pipeline wait timed out");
    }
    return XMC_OK;
}

int upload_inputs(xmc_mlp* m, const float* x, int rows, bool transposed) {
    XM_CUDA(cudaMemcpyAsync(m->xin, x, sizeof(float) * (size_t)rows * m->spec.n_in, cudaMemcpyHostToDevice, m->stream));
    pack_inputs_kernel<<<(rows * kInPad + 255) / 256, 256, 0, m->stream>>>(m->xin, rows, m->spec.n_in, m->x,
                                                                           transposed ? m->xt : nullptr, rows);
    XM_CUDA(cudaGetLastError());
    return XMC_OK;
}

int check_rows(const xmc_mlp* m, int rows) {
    if (rows <= 0 || rows % tc::kBM || rows > m->cap)
        return mfail(XMC_ERR_RANGE, "rows must be a positive multiple of 128 up to max_rows");
    return XMC_OK;
}

}  // namespace
}  // namespace xmc

extern "C" int xmc_mlp_create(const xmc_mlp_spec* spec, xmc_mlp** out) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!spec || !out) return mfail(XMC_ERR_INVALID_INPUT, "spec or out is NULL");
    *out = nullptr;
    xmc_mlp_spec s{};
    std::memcpy(&s, spec, std::min((size_t)spec->struct_size, sizeof(s)));
    s.struct_size = sizeof(s);
    if (s.n_in < 1 || s.n_in > kInPad) return mfail(XMC_ERR_RANGE, "n_in must be in [1, 64]");
    if (s.hidden != 128 && s.hidden != 256) return mfail(XMC_ERR_RANGE, "hidden must be 128 or 256");
    if (s.n_hidden < 1 || s.n_hidden > kMaxLayers - 1) return mfail(XMC_ERR_RANGE, "n_hidden must be in [1, 8]");
    if (s.n_out < 1 || s.n_out > 4096) return mfail(XMC_ERR_RANGE, "n_out must be in [1, 4096]");
    if (s.max_rows < tc::kBM || s.max_rows % tc::kBM || s.max_rows > (1 << 20))
        return mfail(XMC_ERR_RANGE, "max_rows must be a multiple of 128 in [128, 2^20]");
    xmc_mlp* m = new (std::nothrow) xmc_mlp;
    if (!m) return mfail(XMC_ERR_DEVICE, "out of host memory");
    m->spec = s;
    m->L = s.n_hidden + 1;
    m->cap = s.max_rows;
    for (int l = 0; l < m->L; ++l) {
        m->in[l] = l == 0 ? kInPad : s.hidden;
        m->out[l] = l == m->L - 1 ? round_up(s.n_out, 256) : s.hidden;
        m->valid_out[l] = l == m->L - 1 ? s.n_out : s.hidden;
    }
#define XM_TRY(call)                                                                             \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                      \
            free_mlp(m);                                                                         \
            return XMC_ERR_DEVICE;                                                               \
        }                                                                                        \
    } while (0)
    XM_TRY(cudaSetDevice(s.device));
    XM_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    XM_TRY(cudaEventCreate(&m->ev[0]));
    XM_TRY(cudaEventCreate(&m->ev[1]));
    XM_TRY(cudaMalloc(&m->d_err, sizeof(int)));
    XM_TRY(cudaMalloc(&m->d_step, sizeof(int)));
    m->loss_cap = 1 << 20;
    XM_TRY(cudaMalloc(&m->d_loss, sizeof(float) * (m->loss_cap + 1)));
    XM_TRY(cudaMemset(m->d_err, 0, sizeof(int)));
    XM_TRY(cudaMemset(m->d_step, 0, sizeof(int)));
    const size_t R = (size_t)m->cap;
    size_t part = 0;
    for (int l = 0; l < m->L; ++l) {
        const size_t n = (size_t)m->out[l] * m->in[l];
        XM_TRY(cudaMalloc(&m->w32[l], sizeof(float) * n));
        XM_TRY(cudaMalloc(&m->mw[l], sizeof(float) * n));
        XM_TRY(cudaMalloc(&m->vw[l], sizeof(float) * n));
        XM_TRY(cudaMalloc(&m->gw[l], sizeof(float) * n));
        XM_TRY(cudaMalloc(&m->w16[l], sizeof(bf16) * n));
        XM_TRY(cudaMalloc(&m->w16t[l], sizeof(bf16) * n));
        XM_TRY(cudaMalloc(&m->b32[l], sizeof(float) * m->out[l]));
        XM_TRY(cudaMalloc(&m->mb[l], sizeof(float) * m->out[l]));
        XM_TRY(cudaMalloc(&m->vb[l], sizeof(float) * m->out[l]));
        XM_TRY(cudaMalloc(&m->gb[l], sizeof(float) * m->out[l]));
        for (float* p : {m->w32[l], m->mw[l], m->vw[l], m->gw[l]}) XM_TRY(cudaMemset(p, 0, sizeof(float) * n));
        for (float* p : {m->b32[l], m->mb[l], m->vb[l], m->gb[l]}) XM_TRY(cudaMemset(p, 0, sizeof(float) * m->out[l]));
        XM_TRY(cudaMemset(m->w16[l], 0, sizeof(bf16) * n));
        XM_TRY(cudaMemset(m->w16t[l], 0, sizeof(bf16) * n));
        XM_TRY(cudaMalloc(&m->a[l], sizeof(bf16) * R * m->out[l]));
        XM_TRY(cudaMalloc(&m->at[l], sizeof(bf16) * R * m->out[l]));
        XM_TRY(cudaMalloc(&m->z[l], sizeof(bf16) * R * m->out[l]));
        XM_TRY(cudaMalloc(&m->dz[l], sizeof(bf16) * R * m->out[l]));
        XM_TRY(cudaMalloc(&m->dzt[l], sizeof(bf16) * R * m->out[l]));
        // largest split-K partial buffer over the batch sizes this model can take
        const int tiles = m->out[l] / tc::kBM;
        part = std::max(part, (size_t)std::max(1, 128 / tiles) * n);
    }
    m->part_floats = part;
    XM_TRY(cudaMalloc(&m->part, sizeof(float) * part));
    XM_TRY(cudaMalloc(&m->x, sizeof(bf16) * R * kInPad));
    XM_TRY(cudaMalloc(&m->xt, sizeof(bf16) * R * kInPad));
    XM_TRY(cudaMalloc(&m->xin, sizeof(float) * R * s.n_in));
    XM_TRY(cudaMalloc(&m->y, sizeof(float) * R * s.n_out));
    XM_TRY(cudaMalloc(&m->t, sizeof(float) * R * s.n_out));
#undef XM_TRY
    *out = m;
    return XMC_OK;
}

extern "C" int64_t xmc_mlp_param_count(const xmc_mlp* m) {
    if (!m) return -1;
    int64_t n = 0;
    int in = m->spec.n_in;
    for (int l = 0; l < m->L; ++l) {
        n += (int64_t)m->valid_out[l] * in + m->valid_out[l];
        in = m->valid_out[l];
    }
    return n;
}

// Flat parameter layout: for each layer W_l [out_l][in_l] row-major, then b_l [out_l], with
// in_0 = n_in, out_{L-1} = n_out (no padding).
extern "C" int xmc_mlp_set_params(xmc_mlp* m, const float* p) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || !p) return mfail(XMC_ERR_INVALID_INPUT, "model or params is NULL");
    XM_CUDA(cudaSetDevice(m->spec.device));
    int in = m->spec.n_in;
    const float* q = p;
    for (int l = 0; l < m->L; ++l) {
        const int vo = m->valid_out[l];
        std::vector<float> w((size_t)m->out[l] * m->in[l], 0.0f), b(m->out[l], 0.0f);
        for (int r = 0; r < vo; ++r)
            for (int c = 0; c < in; ++c) w[(size_t)r * m->in[l] + c] = q[(size_t)r * in + c];
        q += (size_t)vo * in;
        for (int r = 0; r < vo; ++r) b[r] = q[r];
        q += vo;
        XM_CUDA(cudaMemcpy(m->w32[l], w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice));
        XM_CUDA(cudaMemcpy(m->b32[l], b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice));
        XM_CUDA(cudaMemset(m->mw[l], 0, sizeof(float) * w.size()));
        XM_CUDA(cudaMemset(m->vw[l], 0, sizeof(float) * w.size()));
        XM_CUDA(cudaMemset(m->mb[l], 0, sizeof(float) * b.size()));
        XM_CUDA(cudaMemset(m->vb[l], 0, sizeof(float) * b.size()));
        refresh_kernel<<<148, 256, 0, m->stream>>>(m->w32[l], m->out[l], m->in[l], m->w16[l], m->w16t[l]);
        XM_CUDA(cudaGetLastError());
        in = vo;
    }
    XM_CUDA(cudaMemsetAsync(m->d_step, 0, sizeof(int), m->stream));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    return XMC_OK;
}

static int copy_layers_out(const xmc_mlp* m, float* const* wsrc, float* const* bsrc, float* p) {
    int in = m->spec.n_in;
    float* q = p;
    for (int l = 0; l < m->L; ++l) {
        const int vo = m->valid_out[l];
        std::vector<float> w((size_t)m->out[l] * m->in[l]), b(m->out[l]);
        XM_CUDA(cudaMemcpy(w.data(), wsrc[l], sizeof(float) * w.size(), cudaMemcpyDeviceToHost));
        XM_CUDA(cudaMemcpy(b.data(), bsrc[l], sizeof(float) * b.size(), cudaMemcpyDeviceToHost));
        for (int r = 0; r < vo; ++r)
            for (int c = 0; c < in; ++c) q[(size_t)r * in + c] = w[(size_t)r * m->in[l] + c];
        q += (size_t)vo * in;
        for (int r = 0; r < vo; ++r) q[r] = b[r];
        q += vo;
        in = vo;
    }
    return XMC_OK;
}

extern "C" int xmc_mlp_get_params(const xmc_mlp* m, float* p) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || !p) return mfail(XMC_ERR_INVALID_INPUT, "model or params is NULL");
    XM_CUDA(cudaSetDevice(m->spec.device));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    return copy_layers_out(m, m->w32, m->b32, p);
}

extern "C" int xmc_mlp_forward(xmc_mlp* m, const float* x, int rows, float* y, double* ms) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || !x || !y) return mfail(XMC_ERR_INVALID_INPUT, "model, x or y is NULL");
    int st = check_rows(m, rows);
    if (st) return st;
    XM_CUDA(cudaSetDevice(m->spec.device));
    st = upload_inputs(m, x, rows, false);
    if (st) return st;
    XM_CUDA(cudaEventRecord(m->ev[0], m->stream));
    st = enqueue_forward(m, rows, false);
    if (st) return st;
    XM_CUDA(cudaEventRecord(m->ev[1], m->stream));
    // outputs through pinned staging (kept by the model, sized for its row capacity), then into the
    // caller's array on up to 8 host threads. Large outputs go back in 8 chunks of rows, each with
    // its own event, and every thread copies its share of a chunk as soon as that chunk has landed,
    // so the host copies overlap the device-to-host transfer of the later chunks.
    const size_t nf = (size_t)rows * m->spec.n_out;
    if (m->h_y_floats < nf) {
        if (m->h_y) cudaFreeHost(m->h_y);
        m->h_y = nullptr;
        m->h_y_floats = 0;
        XM_CUDA(cudaHostAlloc((void**)&m->h_y, sizeof(float) * (size_t)m->cap * m->spec.n_out, cudaHostAllocDefault));
        m->h_y_floats = (size_t)m->cap * m->spec.n_out;
    }
    const int chunks = nf < ((size_t)1 << 22) ? 1 : 8;
    const size_t cf = ((size_t)(rows + chunks - 1) / chunks) * m->spec.n_out;  // floats per chunk (whole rows)
    for (int k = 0; k < chunks; ++k) {
        if (!m->ev_chunk[k]) XM_CUDA(cudaEventCreateWithFlags(&m->ev_chunk[k], cudaEventDisableTiming));
        const size_t a = std::min(nf, k * cf), b = std::min(nf, a + cf);
        if (a < b)
            XM_CUDA(cudaMemcpyAsync(m->h_y + a, m->y + a, sizeof(float) * (b - a), cudaMemcpyDeviceToHost, m->stream));
        XM_CUDA(cudaEventRecord(m->ev_chunk[k], m->stream));
    }
    const unsigned parts = nf < ((size_t)1 << 20) ? 1u : std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    std::atomic<int> copy_err{0};
    auto copy_part = [&](unsigned p) {
        for (int k = 0; k < chunks; ++k) {
            if (cudaEventSynchronize(m->ev_chunk[k]) != cudaSuccess) {
                copy_err = 1;
                return;
            }
            const size_t a = std::min(nf, k * cf), b = std::min(nf, a + cf);
            const size_t per = (b - a + parts - 1) / parts;
            const size_t pa = std::min(b, a + p * per), pb = std::min(b, pa + per);
            if (pa < pb) std::memcpy(y + pa, m->h_y + pa, sizeof(float) * (pb - pa));
        }
    };
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
        for (; started < parts; ++started) pool.emplace_back(copy_part, started);
    } catch (...) {
    }
    copy_part(0);
    for (unsigned p = started; p < parts; ++p) copy_part(p);
    for (auto& th : pool) th.join();
    if (copy_err) {
        const cudaError_t e = cudaStreamSynchronize(m->stream);
        return mfail(XMC_ERR_DEVICE, std::string("reading the outputs back failed: ") +
                                         cudaGetErrorString(e != cudaSuccess ? e : cudaErrorUnknown));
    }
    float t = 0.0f;
    XM_CUDA(cudaEventElapsedTime(&t, m->ev[0], m->ev[1]));
    if (ms) *ms = t;
    return check_err(m);
}

// Times `reps` forward passes of the inputs already on the device (the last xmc_mlp_forward's),
// replayed from a CUDA graph; *ms gets the mean device time of one pass.
extern "C" int xmc_mlp_forward_timed(xmc_mlp* m, int rows, int reps, double* ms) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || reps < 1) return mfail(XMC_ERR_INVALID_INPUT, "model is NULL or reps < 1");
    int st = check_rows(m, rows);
    if (st) return st;
    XM_CUDA(cudaSetDevice(m->spec.device));
    cudaGraphExec_t ex = nullptr;
    auto it = m->fwd_graphs.find(rows);
    if (it != m->fwd_graphs.end()) {
        ex = it->second;
    } else {
        XM_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        st = enqueue_forward(m, rows, false);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(m->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return mfail(XMC_ERR_DEVICE, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return mfail(XMC_ERR_DEVICE, std::string("instantiate: ") + cudaGetErrorString(e));
        m->fwd_graphs[rows] = ex;
    }
    XM_CUDA(cudaGraphLaunch(ex, m->stream));  // warm
    XM_CUDA(cudaEventRecord(m->ev[0], m->stream));
    for (int i = 0; i < reps; ++i) XM_CUDA(cudaGraphLaunch(ex, m->stream));
    XM_CUDA(cudaEventRecord(m->ev[1], m->stream));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    float t = 0.0f;
    XM_CUDA(cudaEventElapsedTime(&t, m->ev[0], m->ev[1]));
    if (ms) *ms = t / reps;
    return check_err(m);
}

// Gradients of the mean squared error over `rows` rows at the current parameters (no update), in
// the flat parameter layout; *loss gets the mean squared error.
extern "C" int xmc_mlp_gradients(xmc_mlp* m, const float* x, const float* t, int rows, float* grads, float* loss) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || !x || !t || !grads) return mfail(XMC_ERR_INVALID_INPUT, "NULL argument");
    int st = check_rows(m, rows);
    if (st) return st;
    XM_CUDA(cudaSetDevice(m->spec.device));
    st = upload_inputs(m, x, rows, true);
    if (st) return st;
    XM_CUDA(cudaMemcpyAsync(m->t, t, sizeof(float) * (size_t)rows * m->spec.n_out, cudaMemcpyHostToDevice, m->stream));
    // loss slot: loss[step + ... ] uses *d_step; use slot (current step) after zeroing it
    int step = 0;
    XM_CUDA(cudaMemcpyAsync(&step, m->d_step, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    XM_CUDA(cudaMemsetAsync(m->d_loss + step, 0, sizeof(float), m->stream));
    st = enqueue_forward(m, rows, true);
    if (st) return st;
    st = enqueue_backward(m, rows);
    if (st) return st;
    float l = 0.0f;
    XM_CUDA(cudaMemcpyAsync(&l, m->d_loss + step, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    if (loss) *loss = l / ((float)rows * (float)m->spec.n_out);
    st = check_err(m);
    if (st) return st;
    return copy_layers_out(m, m->gw, m->gb, grads);
}

extern "C" int xmc_mlp_set_dataset(xmc_mlp* m, const float* x, const float* t, int rows) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || !x || !t || rows < 1) return mfail(XMC_ERR_INVALID_INPUT, "NULL argument or empty data set");
    XM_CUDA(cudaSetDevice(m->spec.device));
    if (m->ds_x) cudaFree(m->ds_x);
    if (m->ds_t) cudaFree(m->ds_t);
    m->ds_x = nullptr;
    m->ds_t = nullptr;
    m->ds_rows = 0;
    XM_CUDA(cudaMalloc(&m->ds_x, sizeof(bf16) * (size_t)rows * kInPad));
    XM_CUDA(cudaMalloc(&m->ds_t, sizeof(float) * (size_t)rows * m->spec.n_out));
    float* xin = nullptr;
    XM_CUDA(cudaMalloc(&xin, sizeof(float) * (size_t)rows * m->spec.n_in));
    cudaError_t e = cudaMemcpy(xin, x, sizeof(float) * (size_t)rows * m->spec.n_in, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        pack_inputs_kernel<<<(int)(((size_t)rows * kInPad + 255) / 256), 256>>>(xin, rows, m->spec.n_in, m->ds_x, nullptr, 0);
        e = cudaDeviceSynchronize();
    }
    cudaFree(xin);
    if (e != cudaSuccess) return mfail(XMC_ERR_DEVICE, std::string("set_dataset: ") + cudaGetErrorString(e));
    XM_CUDA(cudaMemcpy(m->ds_t, t, sizeof(float) * (size_t)rows * m->spec.n_out, cudaMemcpyHostToDevice));
    m->ds_rows = rows;
    return XMC_OK;
}

// `steps` Adam steps on minibatches of `batch` rows drawn (with replacement, Philox keyed by seed)
// from the device data set; each step is one replay of a CUDA graph (gather, forward, backward,
// Adam). losses[i] (may be NULL) gets the mean squared error of step i's minibatch.
extern "C" int xmc_mlp_train(xmc_mlp* m, int steps, int batch, float lr, float beta1, float beta2, float eps,
                             uint64_t seed, float* losses, double* ms) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m || steps < 0) return mfail(XMC_ERR_INVALID_INPUT, "model is NULL or steps < 0");
    if (!m->ds_rows) return mfail(XMC_ERR_INVALID_INPUT, "no data set (xmc_mlp_set_dataset)");
    int st = check_rows(m, batch);
    if (st) return st;
    XM_CUDA(cudaSetDevice(m->spec.device));
    int step0 = 0;
    XM_CUDA(cudaMemcpy(&step0, m->d_step, sizeof(int), cudaMemcpyDeviceToHost));
    if (step0 + steps >= m->loss_cap) return mfail(XMC_ERR_RANGE, "too many training steps for the loss log");
    if (lr != m->g_lr || beta1 != m->g_b1 || beta2 != m->g_b2 || eps != m->g_eps || seed != m->g_seed) {
        for (auto& kv : m->train_graphs) cudaGraphExecDestroy(kv.second);
        m->train_graphs.clear();
        m->g_lr = lr; m->g_b1 = beta1; m->g_b2 = beta2; m->g_eps = eps; m->g_seed = seed;
    }
    cudaGraphExec_t ex = nullptr;
    auto it = m->train_graphs.find(batch);
    if (it != m->train_graphs.end()) {
        ex = it->second;
    } else {
        XM_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        step_kernel<<<1, 1, 0, m->stream>>>(m->d_step, m->d_loss);
        gather_kernel<<<batch, 128, 0, m->stream>>>(m->ds_x, m->ds_t, m->ds_rows, m->spec.n_out, batch, (uint32_t)seed,
                                                    (uint32_t)(seed >> 32), m->d_step, m->x, m->xt, m->t);
        st = enqueue_forward(m, batch, true);
        if (!st) st = enqueue_backward(m, batch);
        if (!st) st = enqueue_adam(m, lr, beta1, beta2, eps);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(m->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return mfail(XMC_ERR_DEVICE, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return mfail(XMC_ERR_DEVICE, std::string("instantiate: ") + cudaGetErrorString(e));
        m->train_graphs[batch] = ex;
    }
    XM_CUDA(cudaEventRecord(m->ev[0], m->stream));
    for (int i = 0; i < steps; ++i) XM_CUDA(cudaGraphLaunch(ex, m->stream));
    XM_CUDA(cudaEventRecord(m->ev[1], m->stream));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    float t = 0.0f;
    XM_CUDA(cudaEventElapsedTime(&t, m->ev[0], m->ev[1]));
    if (ms) *ms = t;
    st = check_err(m);
    if (st) return st;
    if (losses && steps > 0) {
        XM_CUDA(cudaMemcpy(losses, m->d_loss + step0 + 1, sizeof(float) * steps, cudaMemcpyDeviceToHost));
        const float inv = 1.0f / ((float)batch * (float)m->spec.n_out);
        for (int i = 0; i < steps; ++i) losses[i] *= inv;
    }
    return XMC_OK;
}

// Per-output weights of the squared error in training and in xmc_mlp_gradients (NULL: all 1).
extern "C" int xmc_mlp_set_output_weights(xmc_mlp* m, const float* w) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!m) return mfail(XMC_ERR_INVALID_INPUT, "model is NULL");
    XM_CUDA(cudaSetDevice(m->spec.device));
    XM_CUDA(cudaStreamSynchronize(m->stream));
    if (!w) {
        if (m->colw) cudaFree(m->colw);
        m->colw = nullptr;
    } else {
        for (int j = 0; j < m->spec.n_out; ++j)
            if (!(w[j] >= 0.0f) || !std::isfinite(w[j])) return mfail(XMC_ERR_INVALID_INPUT, "weights must be finite and >= 0");
        if (!m->colw) XM_CUDA(cudaMalloc(&m->colw, sizeof(float) * m->spec.n_out));
        XM_CUDA(cudaMemcpy(m->colw, w, sizeof(float) * m->spec.n_out, cudaMemcpyHostToDevice));
    }
    // the training graphs hold the old pointer
    for (auto& kv : m->train_graphs) cudaGraphExecDestroy(kv.second);
    m->train_graphs.clear();
    return XMC_OK;
}

extern "C" int xmc_mlp_destroy(xmc_mlp* m) {
    free_mlp(m);
    return XMC_OK;
}

// Plain GEMM through the same kernel, for tests: D[M x N] = A[M x K] . B[N x K]^T with bf16 inputs
// given as raw 16-bit patterns; split-K partials are summed on the host in split order.
extern "C" int xmc_gemm_bf16(const uint16_t* a, const uint16_t* b, int M, int N, int K, int bn, int splits, float* d) {
    if (!a || !b || !d) return mfail(XMC_ERR_INVALID_INPUT, "NULL argument");
    if (M <= 0 || N <= 0 || K <= 0 || splits < 1 || (bn != 64 && bn != 128 && bn != 256) || M % tc::kBM || N % bn ||
        K % (tc::kBK * splits))
        return mfail(XMC_ERR_INVALID_INPUT, "gemm: M % 128, N % bn, K % (64 splits) must be 0");
    void *da = nullptr, *db = nullptr;
    float* dd = nullptr;
    int* derr = nullptr;
    int st = XMC_OK;
    const size_t nd = (size_t)splits * M * N;
    cudaError_t e = cudaMalloc(&da, sizeof(uint16_t) * (size_t)M * K);
    if (e == cudaSuccess) e = cudaMalloc(&db, sizeof(uint16_t) * (size_t)N * K);
    if (e == cudaSuccess) e = cudaMalloc(&dd, sizeof(float) * nd);
    if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(da, a, sizeof(uint16_t) * (size_t)M * K, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(db, b, sizeof(uint16_t) * (size_t)N * K, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = mfail(XMC_ERR_DEVICE, std::string("gemm setup: ") + cudaGetErrorString(e));
    if (!st) {
        EpiF32 epi{dd, N, (size_t)M * N};
        if (bn == 256) st = launch_gemm<256>(da, M, db, N, K, splits, epi, derr, 0);
        else if (bn == 128) st = launch_gemm<128>(da, M, db, N, K, splits, epi, derr, 0);
        else st = launch_gemm<64>(da, M, db, N, K, splits, epi, derr, 0);
    }
    if (!st) {
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) st = mfail(XMC_ERR_DEVICE, std::string("gemm: ") + cudaGetErrorString(e));
    }
    int herr = 0;
    if (!st && cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && herr)
        st = mfail(XMC_ERR_DEVICE, "gemm: a pipeline wait timed out");
    if (!st) {
        std::vector<float> part(nd);
        e = cudaMemcpy(part.data(), dd, sizeof(float) * nd, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            st = mfail(XMC_ERR_DEVICE, std::string("gemm read-back: ") + cudaGetErrorString(e));
        } else {
            for (size_t i = 0; i < (size_t)M * N; ++i) {
                float s = 0.0f;
                for (int k = 0; k < splits; ++k) s += part[(size_t)k * M * N + i];
                d[i] = s;
            }
        }
    }
    cudaFree(da);
    cudaFree(db);
    cudaFree(dd);
    cudaFree(derr);
    return st;
}
