// xmc_run_noalloc: a transport run that allocates no GPU memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a host framework which owns all
// device memory through its own pool, or a process that must not grow its device footprint after
// start-up (allocation there fails, stalls on a device-wide synchronisation, or fragments the
// pool). Such a caller brings the output buffers from its own memory. Everything else the kernel
// needs beyond its inputs and outputs (the device copy of the tissue model: BVH nodes, triangle
// records, layer-transition table, detector records and the xy cell grid, plus the photon-id
// dispenser and the status word) is scratch, and it lives here in one file-scope __device__ array of fixed size,
// which every GPU that loads the library holds until the process exits.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "xmc_internal.h"

namespace xmc {
namespace {

constexpr size_t kNoAllocScratchBytes = XMC_NOALLOC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;

// The scratch array. In host code `g_noalloc_scratch` is only a host-side stand-in for the symbol;
// its device address comes from cudaGetSymbolAddress (noalloc_scratch_address below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// Once per device, with that device current: the device address of the scratch array.
int noalloc_scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) {
        set_error("xmc_run_noalloc: device ordinal out of range");
        return XMC_ERR_INVALID_INPUT;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("xmc_run_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return XMC_ERR_DEVICE;
        }
        g_scratch_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
    return XMC_OK;
}

}  // namespace
}  // namespace xmc

using namespace xmc;

extern "C" int xmc_run_noalloc(const InputInfo* input, const xmc_options* opt, uint64_t seed,
                               uint64_t first_photon_id, uint64_t n_photons, unsigned long long* d_absorption,
                               unsigned long long* d_detectors, unsigned long long* d_time_bins,
                               unsigned long long* d_ledger, void* stream) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (!d_absorption || !d_detectors || !d_time_bins || !d_ledger) {
        set_error("xmc_run_noalloc: output buffers must not be NULL");
        return XMC_ERR_INVALID_INPUT;
    }
    HostImage img;
    xmc_options o;  // the BVH is built on the host here: a GPU build would allocate device memory
    xmc_default_options(&o);
    if (opt && opt->struct_size) std::memcpy(&o, opt, std::min((size_t)opt->struct_size, sizeof(o)));
    o.flags &= ~XMC_GPU_BVH;
    o.flags |= XMC_LANE_QUERIES;  // the cooperative query's entry records would need more scratch
    int st = prepare_image(input, &o, &img);
    if (st) return st;
    if (img.kp.use_bias) {
        set_error("xmc_run_noalloc: biasing needs weight tables this entry point does not stage");
        return XMC_ERR_UNSUPPORTED;
    }
    if (img.opt.flags & (XMC_SCATTERING_MAP | XMC_DETECTOR_TRAJ)) {
        set_error("xmc_run_noalloc: scattering and trajectory maps need buffers this entry point does not take");
        return XMC_ERR_UNSUPPORTED;
    }
    const GeomImage& geom = img.geom;

    // scratch layout: [dispenser u64 | status int | cancel int] [nodes] [triangles] [transition table]
    // [detectors] [grid cells] [cell z-intervals] [grid entries] [big triangles]
    const size_t b_nodes = sizeof(float4) * geom.nodes.size();
    const size_t b_tris = sizeof(float4) * geom.tris.size();
    const size_t b_next = img.next.size();
    const size_t b_dets = sizeof(DevDetector) * img.dets.size();
    const size_t b_cells = sizeof(uint2) * img.grid.cells.size();
    const size_t b_cell_z = sizeof(float4) * img.grid.cell_z.size();
    const size_t b_entries = sizeof(float4) * img.grid.entries.size();
    const size_t b_big = sizeof(float4) * img.grid.big.size();
    const size_t o_nodes = kAlign;
    const size_t o_tris = o_nodes + align_up(b_nodes);
    const size_t o_next = o_tris + align_up(b_tris);
    const size_t o_dets = o_next + align_up(b_next);
    const size_t o_cells = o_dets + align_up(b_dets);
    const size_t o_cell_z = o_cells + align_up(b_cells);
    const size_t o_entries = o_cell_z + align_up(b_cell_z);
    const size_t o_big = o_entries + align_up(b_entries);
    const size_t need = o_big + align_up(b_big);
    if (need > kNoAllocScratchBytes) {
        set_error("xmc_run_noalloc: the model needs " + std::to_string(need) + " bytes of device scratch; this entry "
                  "point holds at most " + std::to_string(kNoAllocScratchBytes) + " (use xmc_create/xmc_run)");
        return XMC_ERR_RANGE;
    }

    const int device = img.opt.device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        set_error(std::string("xmc_run_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));
        return XMC_ERR_DEVICE;
    }
    unsigned char* scratch = nullptr;
    st = noalloc_scratch_address(device, &scratch);
    if (st) return st;

    Context c;  // host-side launch record only; owns no device memory
    c.device = device;
    c.opt = img.opt;
    c.kp = img.kp;
    c.smem_bytes = img.smem_bytes;
    c.stream = static_cast<cudaStream_t>(stream);
    KParams& kp = c.kp;
    kp.nodes = reinterpret_cast<const float4*>(scratch + o_nodes);
    kp.tris = reinterpret_cast<const float4*>(scratch + o_tris);
    kp.next_layer = reinterpret_cast<const int8_t*>(scratch + o_next);
    kp.dets = reinterpret_cast<const DevDetector*>(scratch + o_dets);
    kp.cells = reinterpret_cast<const uint2*>(scratch + o_cells);
    kp.cell_z = reinterpret_cast<const float4*>(scratch + o_cell_z);
    kp.cell_entries = reinterpret_cast<const float4*>(scratch + o_entries);
    kp.big = reinterpret_cast<const float4*>(scratch + o_big);
    kp.counter = reinterpret_cast<unsigned long long*>(scratch);
    kp.status = reinterpret_cast<int*>(scratch + sizeof(unsigned long long));
    kp.cancel = nullptr;
    kp.absorb = d_absorption;
    kp.det = d_detectors;
    kp.tbin = d_time_bins;
    kp.ledger = d_ledger;
    kp.key0 = (uint32_t)seed;
    kp.key1 = (uint32_t)(seed >> 32);
    kp.first_id = first_photon_id;
    kp.n_photons = n_photons;

#define NA_CK(call)                                                                                         \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) {                                                                            \
            set_error(std::string("xmc_run_noalloc: ") + #call + ": " + cudaGetErrorString(e_));             \
            return XMC_ERR_DEVICE;                                                                          \
        }                                                                                                   \
    } while (0)

    int sms = 0, occ = 0;
    NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    c.block = img.opt.block_size > 0 ? img.opt.block_size : 256;
    if (c.block % 32 != 0 || c.block > 1024) {
        set_error("xmc_run_noalloc: block_size must be a multiple of 32 <= 1024");
        return XMC_ERR_INVALID_INPUT;
    }
    NA_CK(transport_occupancy(c.block, c.smem_bytes, &occ));
    if (occ <= 0) {
        set_error("xmc_run_noalloc: transport kernel cannot be resident with this block size");
        return XMC_ERR_DEVICE;
    }
    c.blocks_per_sm = img.opt.blocks_per_sm > 0 ? std::min(img.opt.blocks_per_sm, occ) : occ;
    c.grid = sms * c.blocks_per_sm;

    // the scratch keeps the previous call's contents: the dispenser and status start at zero
    NA_CK(cudaMemsetAsync(scratch, 0, kAlign, c.stream));
    if (b_nodes) NA_CK(cudaMemcpyAsync(scratch + o_nodes, geom.nodes.data(), b_nodes, cudaMemcpyHostToDevice, c.stream));
    if (b_tris) NA_CK(cudaMemcpyAsync(scratch + o_tris, geom.tris.data(), b_tris, cudaMemcpyHostToDevice, c.stream));
    NA_CK(cudaMemcpyAsync(scratch + o_next, img.next.data(), b_next, cudaMemcpyHostToDevice, c.stream));
    NA_CK(cudaMemcpyAsync(scratch + o_dets, img.dets.data(), b_dets, cudaMemcpyHostToDevice, c.stream));
    if (b_cells) NA_CK(cudaMemcpyAsync(scratch + o_cells, img.grid.cells.data(), b_cells, cudaMemcpyHostToDevice, c.stream));
    if (b_cell_z) NA_CK(cudaMemcpyAsync(scratch + o_cell_z, img.grid.cell_z.data(), b_cell_z, cudaMemcpyHostToDevice, c.stream));
    if (b_entries)
        NA_CK(cudaMemcpyAsync(scratch + o_entries, img.grid.entries.data(), b_entries, cudaMemcpyHostToDevice, c.stream));
    if (b_big) NA_CK(cudaMemcpyAsync(scratch + o_big, img.grid.big.data(), b_big, cudaMemcpyHostToDevice, c.stream));
    const size_t nd = (size_t)std::max(1, img.n_dets);
    NA_CK(cudaMemsetAsync(d_absorption, 0, sizeof(unsigned long long) * (size_t)img.grid_size, c.stream));
    NA_CK(cudaMemsetAsync(d_detectors, 0, sizeof(unsigned long long) * 4 * nd, c.stream));
    NA_CK(cudaMemsetAsync(d_time_bins, 0, sizeof(unsigned long long) * 4 * nd * img.n_time, c.stream));
    NA_CK(cudaMemsetAsync(d_ledger, 0, sizeof(unsigned long long) * kLedgerSlots, c.stream));
    if (n_photons > 0) NA_CK(enqueue_transport(&c));
    int status = 0;
    NA_CK(cudaMemcpyAsync(&status, kp.status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    NA_CK(cudaStreamSynchronize(c.stream));
#undef NA_CK
    if (status & 1) {
        set_error("a photon reached the step budget and was terminated");
        return XMC_ERR_BUDGET;
    }
    return XMC_OK;
}
