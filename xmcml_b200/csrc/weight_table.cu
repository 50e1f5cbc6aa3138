// Weight-integral tables of the biased walk, computed on the GPU in FP64.
//
// The reference computes, before the walk and for each distinct anisotropy g of the tissue layers,
// W(d) for tablePrecision + 1 cosines d in [-1, 1] (weight_integral.cpp:34-104): the integral over
// the unit sphere of the Henyey-Greenstein phase function about a direction at cosine d to the
// attractive direction, times the acceptance (0.1 + 0.45 (1 + cos))^factor, divided by 2 pi, by a
// product two-point Gauss-Legendre rule on n x n cells of (theta, phi) (mcml_integration.cpp:7-83).
// With the default precisions that is 262,145 values x 65,536 integrand evaluations per table.
//
// On the GPU the integrand is split into the part that depends on the node only (sin theta,
// the cosine to the attractive direction, the acceptance factor and the quadrature weight: one
// pass over the 4 n^2 nodes) and the part that depends on d (the HG value of the cosine to the
// photon direction). One thread computes one table value, summing over the nodes staged through
// shared memory in a fixed order, so the tables are deterministic.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "xmc_internal.h"

namespace xmc {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kTile = 1024;

// per node: {cosine to the attractive direction, sin(theta) sin(phi), quadrature weight x acceptance x sin(theta)}
__global__ void wt_nodes_kernel(unsigned n, double eps, double4* __restrict__ nodes) {
    const size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= (size_t)n * n) return;
    const unsigned i = (unsigned)(cell / n), j = (unsigned)(cell % n);
    const double coeff = 2.0 * sqrt(3.0);
    const double hx = kPi / n, hy = 2 * kPi / n;
    const double x0 = hx * i, x1 = x0 + hx, y0 = hy * j, y1 = y0 + hy;
    const double xs[2] = {0.5 * (x0 + x1) + (x1 - x0) / coeff, 0.5 * (x0 + x1) - (x1 - x0) / coeff};
    const double ys[2] = {0.5 * (y0 + y1) + (y1 - y0) / coeff, 0.5 * (y0 + y1) - (y1 - y0) / coeff};
    const double area = 0.25 * (x1 - x0) * (y1 - y0);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double st = sin(xs[a]);
            const double along = st * cos(ys[b]);
            const double q = st * sin(ys[b]);
            const double w = area * pow(0.1 + 0.9 * 0.5 * (1 + along), eps) * st;
            nodes[4 * cell + 2 * a + b] = make_double4(along, q, w, 0.0);
        }
}

__global__ void wt_table_kernel(const double4* __restrict__ nodes, size_t n_nodes, double g, int n_elem,
                                double* __restrict__ out) {
    __shared__ double4 tile[kTile];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const double step = 2.0 / (n_elem - 1);
    const double dot = e < n_elem ? -1.0 + e * step : 0.0;
    const double s = sqrt(fmax(0.0, 1 - dot * dot));
    const double g2 = g * g, num = 1 - g2;
    double sum = 0.0;
    for (size_t base = 0; base < n_nodes; base += kTile) {
        const int cnt = (int)min((size_t)kTile, n_nodes - base);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) tile[k] = nodes[base + k];
        __syncthreads();
        for (int k = 0; k < cnt; ++k) {
            const double4 nd = tile[k];
            const double c = dot * nd.x + s * nd.y;
            const double q = 1 + g2 - 2 * g * c;
            sum += nd.z * num / (2 * q * sqrt(q));
        }
    }
    if (e < n_elem) out[e] = sum / (2.0 * kPi);
}

int wfail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}

}  // namespace

// weight_integral.cpp:95-104: integral precision raised for strongly forward-peaked layers
unsigned weight_integral_precision(double g, unsigned base) {
    if (g > 0.98) return base * 16;
    if (g > 0.97) return base * 8;
    if (g > 0.95) return base * 4;
    if (g > 0.90) return base * 2;
    return base;
}

// weight_integral.cpp:67-93: distinct anisotropies of layers 1..L-1, in first-seen order
std::vector<double> distinct_anisotropies(const InputInfo* in) {
    std::vector<double> gs;
    for (int l = 1; l < in->numberOfLayers; ++l) {
        const double g = in->layerInfo[l].anisotropy;
        bool seen = false;
        for (double h : gs) seen |= (h == g);
        if (!seen) gs.push_back(g);
    }
    return gs;
}

int compute_weight_tables(const InputInfo* in, int device, std::vector<double>* gs, std::vector<double>* tables,
                          int* n_elem) {
    xmc::DeviceGuard device_guard;  // the caller's current device is restored on return
    if (in->weightTablePrecision < 1 || in->weightTablePrecision > (1u << 24))
        return wfail(XMC_ERR_RANGE, "weightTablePrecision must be in [1, 2^24]");
    if (in->weightIntegralPrecision < 1 || in->weightIntegralPrecision > 4096)
        return wfail(XMC_ERR_RANGE, "weightIntegralPrecision must be in [1, 4096]");
    if (!std::isfinite(in->attractiveFactor) || in->attractiveFactor < 0)
        return wfail(XMC_ERR_INVALID_INPUT, "attractiveFactor must be finite and >= 0");
    *gs = distinct_anisotropies(in);
    *n_elem = (int)in->weightTablePrecision + 1;
    tables->assign(gs->size() * (size_t)*n_elem, 0.0);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return wfail(XMC_ERR_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    double4* nodes = nullptr;
    double* out = nullptr;
    size_t cap = 0;
    int st = XMC_OK;
    for (size_t k = 0; k < gs->size() && !st; ++k) {
        const unsigned n = weight_integral_precision((*gs)[k], in->weightIntegralPrecision);
        const size_t nn = 4 * (size_t)n * n;
        if (nn > cap) {
            if (nodes) cudaFree(nodes);
            nodes = nullptr;
            e = cudaMalloc(&nodes, sizeof(double4) * nn);
            if (e != cudaSuccess) { st = wfail(XMC_ERR_DEVICE, std::string("weight table nodes: ") + cudaGetErrorString(e)); break; }
            cap = nn;
        }
        if (!out) {
            e = cudaMalloc(&out, sizeof(double) * (size_t)*n_elem);
            if (e != cudaSuccess) { st = wfail(XMC_ERR_DEVICE, std::string("weight table: ") + cudaGetErrorString(e)); break; }
        }
        const size_t cells = (size_t)n * n;
        wt_nodes_kernel<<<(unsigned)((cells + 255) / 256), 256>>>(n, in->attractiveFactor, nodes);
        wt_table_kernel<<<(*n_elem + 255) / 256, 256>>>(nodes, nn, (*gs)[k], *n_elem, out);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpy(tables->data() + k * (size_t)*n_elem, out, sizeof(double) * (size_t)*n_elem,
                           cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = wfail(XMC_ERR_DEVICE, std::string("weight table kernels: ") + cudaGetErrorString(e));
    }
    if (nodes) cudaFree(nodes);
    if (out) cudaFree(out);
    return st;
}

}  // namespace xmc

using namespace xmc;

// Replaces the computing branch of GetWeightIntegralTable (base/xmcml/xmcmlLauncher/weight_integral.cpp:17-65):
// fills input->weightTable / numberOfWeightTables (new[]-allocated, freed by xmc_free_input).
extern "C" int xmc_weight_integral_table(InputInfo* input, int device) {
    if (!input || !input->layerInfo) return wfail(XMC_ERR_INVALID_INPUT, "input or its layers are NULL");
    std::vector<double> gs, tables;
    int n_elem = 0;
    int st = compute_weight_tables(input, device, &gs, &tables, &n_elem);
    if (st) return st;
    WeightIntegralTable* t = new WeightIntegralTable[gs.empty() ? 1 : gs.size()];
    for (size_t k = 0; k < gs.size(); ++k) {
        t[k].anisotropy = gs[k];
        t[k].numberOfElements = n_elem;
        t[k].elements = new double[n_elem];
        std::memcpy(t[k].elements, tables.data() + k * (size_t)n_elem, sizeof(double) * n_elem);
    }
    input->weightTable = t;
    input->numberOfWeightTables = (int)gs.size();
    return XMC_OK;
}
