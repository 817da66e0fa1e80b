// Energy diagnostic over caller-owned device arrays, with no device
// allocation: the reduction's scratch is a fixed file-scope __device__ array.
//
// Who needs it: a caller that holds the ocean state in device buffers of its
// own (for example a driver whose arrays come from another framework's
// memory pool) and wants the domain energy (energy, fv_average_dynamic.F90:
// 476-554) without creating a fesomc_model, whose init allocates the whole
// prognostic state; or a caller that has reserved all device memory up front
// and must not make further allocations.  This entry point makes none: no
// cudaMalloc, no cudaFree, no allocating library call.
//
// Scratch: g_energy_scratch holds kEsParts x 3 compensated partial sums (one
// triple per block) and the 3 totals: 1,779 doubles, 14,232 bytes.  The grid
// is fixed at kEsParts blocks that stride over the mesh, so any mesh size
// fits (a static_assert ties the grid to the array size); node and element
// counts below 1 are rejected with FESOMC_EINVAL.  Every call writes all the partials and totals
// it later reads, so nothing in the array has to start at zero.  All calls on
// a device share the one array: calls that overlap in time (different
// streams or host threads) race on it and must be serialised by the caller.
//
// Set-up: the first call on a device (that device current) looks up the
// array's device address once with cudaGetSymbolAddress and keeps it for the
// life of the process; make that first call before any stream capture
// begins.  The kept address belongs to the device's primary context: after
// cudaDeviceReset on that device the next context may place the array
// elsewhere, so a process that resets a device must not call this entry
// point on it again.
#include <mutex>

#include "device_common.cuh"
#include "fesomc_gpu.h"

namespace fesomc {
namespace {
using namespace fesomc::f64;

constexpr int kEsBlock = 256;
constexpr int kEsParts = 592;                    // 4 blocks per SM on 148 SMs
constexpr int kEsDoubles = kEsParts * 3 + 3;     // partial triples + totals
constexpr int kEsMaxDevices = 64;
static_assert(kEsDoubles * sizeof(double) == 14232, "documented scratch size");

static __device__ __align__(256) double g_energy_scratch[kEsDoubles];

// compensated (Neumaier) running sum
struct NSum {
    double s, c;
    __device__ void add(double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ double value() const { return s + c; }
};

// Per-block partial sums of potential energy, kinetic energy and area;
// element nodes are 1-based (4 per element, triangles repeat node 1).
__global__ void k_energy_dev_part(int N, int E, double Dmin, const double *eta, const double *depth,
                                  const double *area, const int32_t *en4, const double *w4, const double *u2,
                                  const double *earea, double *scratch) {
    __shared__ double sh[3][kEsBlock];
    NSum pe{0.0, 0.0}, ke{0.0, 0.0}, ar{0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double e = eta[i];
        pe.add(0.5 * kG * area[i] * (e * e));
        ar.add(area[i]);
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (long long)gridDim.x * blockDim.x) {
        const int n0 = en4[4 * i] - 1, n1 = en4[4 * i + 1] - 1, n2 = en4[4 * i + 2] - 1, n3 = en4[4 * i + 3] - 1;
        const double4 w = make_double4(w4[4 * i], w4[4 * i + 1], w4[4 * i + 2], w4[4 * i + 3]);
        const double s = wsum(w, dmax(Dmin, depth[n0] + eta[n0]), dmax(Dmin, depth[n1] + eta[n1]),
                              dmax(Dmin, depth[n2] + eta[n2]), dmax(Dmin, depth[n3] + eta[n3]));
        const double ux = u2[2 * i], uy = u2[2 * i + 1];
        ke.add(0.5 * s * earea[i] * (ux * ux + uy * uy));
    }
    sh[0][threadIdx.x] = pe.value();
    sh[1][threadIdx.x] = ke.value();
    sh[2][threadIdx.x] = ar.value();
    __syncthreads();
    if (threadIdx.x < 3) {
        NSum t{0.0, 0.0};
        for (int k = 0; k < kEsBlock; ++k) t.add(sh[threadIdx.x][k]);
        scratch[(size_t)blockIdx.x * 3 + threadIdx.x] = t.value();
    }
}

__global__ void k_energy_dev_final(double *scratch, int nparts) {
    if (threadIdx.x < 3 && blockIdx.x == 0) {
        NSum t{0.0, 0.0};
        for (int b = 0; b < nparts; ++b) t.add(scratch[(size_t)b * 3 + threadIdx.x]);
        scratch[(size_t)kEsParts * 3 + threadIdx.x] = t.value();
    }
}

std::mutex g_setup_mu;
double *g_scratch_addr[kEsMaxDevices] = {};

}  // namespace
}  // namespace fesomc

extern "C" int fesomc_energy_device(int32_t nod2D, int32_t elem2D, double Dmin, const double *eta_n,
                                    const double *depth, const double *area, const int32_t *elem2D_nodes,
                                    const double *w_cv, const double *U_n_2D, const double *elem_area,
                                    void *stream, double *eout) {
    using namespace fesomc;
    if (nod2D < 1 || elem2D < 1 || !eta_n || !depth || !area || !elem2D_nodes || !w_cv || !U_n_2D || !elem_area ||
        !eout)
        return FESOMC_EINVAL;
    const int nparts = kEsParts;
    static_assert(kEsParts * 3 + 3 <= kEsDoubles, "one partial triple per block and the totals fit the scratch");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return FESOMC_ECUDA;
    if (dev < 0 || dev >= kEsMaxDevices) return FESOMC_EINVAL;
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_energy_scratch) != cudaSuccess || !p) return FESOMC_ECUDA;
            g_scratch_addr[dev] = static_cast<double *>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_energy_dev_part<<<nparts, kEsBlock, 0, s>>>(nod2D, elem2D, Dmin, eta_n, depth, area, elem2D_nodes, w_cv,
                                                  U_n_2D, elem_area, scratch);
    k_energy_dev_final<<<1, 32, 0, s>>>(scratch, nparts);
    if (cudaGetLastError() != cudaSuccess) return FESOMC_ECUDA;
    double h[3];
    if (cudaMemcpyAsync(h, scratch + (size_t)kEsParts * 3, 3 * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return FESOMC_ECUDA;
    *eout = (h[0] + h[1]) / h[2];
    return FESOMC_OK;
}
