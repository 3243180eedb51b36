// noalloc.cu -- CELL_SORT for callers that cannot allocate device memory.
//
// Some host programs cannot let a library call cudaMalloc: their device
// memory is owned by another allocator (a framework's caching pool, or a
// Fortran code that reserves one arena at start-up and expects no foreign
// allocations), or they bin atoms inside a tight per-step loop where a
// cudaMalloc/cudaFree pair would synchronise the whole device.  For them,
// simox_cell_sort_noalloc() bins atoms exactly like simox_cell_sort() but keeps
// its only scratch -- the per-cell atom counters and a status word -- in the
// fixed array below, which every GPU that loads this library holds until the
// process exits.  The caller passes the positions and the npt/link outputs as
// device pointers.
#include "simox_internal.cuh"

#include <mutex>

namespace sx {

// Capacity of the fixed scratch: cell counters for up to this many cells.
constexpr int kNoallocMaxCells = 65536;
constexpr int kNoallocMaxPerCell = 4096;   // shared-memory row for the in-cell order

struct NoallocScratch {
    int count[kNoallocMaxCells];
    int status;
};

static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// One address per device, looked up with that device current on the first call.
static void* g_scratch_addr[128];
static std::mutex g_scratch_mutex;

static int scratch_for_current_device(NoallocScratch** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= 128) return SIMOX_E_ARG;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return e != cudaSuccess ? cuda_status(e) : SIMOX_E_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<NoallocScratch*>(g_scratch_addr[dev]);
    return SIMOX_OK;
}

// Bin and append: the same FP64 arithmetic as CELL_SORT (cellsort.f90:69-71);
// the atom is appended to its cell's row of the caller's link array.
__global__ void noalloc_bin_kernel(int n, const double* __restrict__ x, double3 hbox, double3 lc, int3 nc,
                                   int stride, NoallocScratch* __restrict__ S, int* __restrict__ link) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double hb[3] = {hbox.x, hbox.y, hbox.z};
    const double l[3] = {lc.x, lc.y, lc.z};
    const int m[3] = {nc.x, nc.y, nc.z};
    int id[3];
    for (int d = 0; d < 3; d++) {
        const double t = __ddiv_rn(__dadd_rn(x[3 * i + d], hb[d]), l[d]);
        if (!(fabs(t) < 1.0e9)) { atomicOr(&S->status, ST_POSITION); return; }
        int v = (__double2int_rz(t) + m[d]) % m[d];
        if (v < 0) { atomicOr(&S->status, ST_POSITION); return; }
        id[d] = v;
    }
    const int c = id[0] + id[1] * m[0] + id[2] * m[0] * m[1];
    const int slot = atomicAdd(&S->count[c], 1);
    if (slot < stride) link[(size_t)c * stride + slot] = i + 1;
    else atomicOr(&S->status, ST_CELL_OVERFLOW);
}

// Per cell: ascending atom order (the order CELL_SORT appends in) and Npt.
__global__ void noalloc_order_kernel(int stride, const NoallocScratch* __restrict__ S, int* __restrict__ npt,
                                     int* __restrict__ link) {
    __shared__ int buf[kNoallocMaxPerCell];
    const int c = blockIdx.x;
    const int cnt = S->count[c];
    if (threadIdx.x == 0) npt[c] = cnt;
    const int m = cnt < stride ? cnt : stride;   // stride <= kNoallocMaxPerCell (checked on the host)
    if (m <= 1) return;
    int* row = link + (size_t)c * stride;
    for (int k = threadIdx.x; k < m; k += blockDim.x) buf[k] = row[k];
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int v = buf[k];
        int rank = 0;
        for (int j = 0; j < m; j++) rank += buf[j] < v;
        row[rank] = v;
    }
}

}  // namespace sx

using namespace sx;

extern "C" int simox_cell_sort_noalloc(const double* x_dev, int n, const double* box, double rcut, int* npt_dev,
                                       int* link_dev, int link_stride, void* stream) {
    if (!x_dev && n > 0) return SIMOX_E_ARG;
    if (!box || !npt_dev || !link_dev || n < 0 || link_stride < 1 || !(rcut > 0.0)) return SIMOX_E_ARG;
    if (link_stride > kNoallocMaxPerCell) return SIMOX_E_SCRATCH_LIMIT;
    int nc[3];
    double lc[3], hbox[3];
    for (int d = 0; d < 3; d++) {
        if (!(box[d] > 0.0)) return SIMOX_E_ARG;
        nc[d] = (int)(box[d] / rcut);                  // main.f90:269-270
        // simox_create's rule: a dimension below 2 cells pairs an atom with
        // itself at r = 0 in FORCE, so neither entry point accepts it
        if (nc[d] < 2) return SIMOX_E_CELL_TOO_SMALL;
        lc[d] = box[d] / (double)nc[d];
        hbox[d] = 0.5 * box[d];
    }
    if (nc[0] < 3 && nc[1] < 3 && nc[2] < 3) return SIMOX_E_CELL_TOO_SMALL;   // main.f90:271
    const long long ncell = (long long)nc[0] * nc[1] * nc[2];
    if (ncell > kNoallocMaxCells) return SIMOX_E_SCRATCH_LIMIT;
    NoallocScratch* S = nullptr;
    int st = scratch_for_current_device(&S);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the counters and the status word must start at zero on every call
    cudaError_t e = cudaMemsetAsync(S, 0, sizeof(int) * ncell, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&S->status, 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_status(e);
    if (n > 0)
        noalloc_bin_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, x_dev, make_double3(hbox[0], hbox[1], hbox[2]),
                                                           make_double3(lc[0], lc[1], lc[2]),
                                                           make_int3(nc[0], nc[1], nc[2]), link_stride, S, link_dev);
    noalloc_order_kernel<<<(unsigned)ncell, 128, 0, s>>>(link_stride, S, npt_dev, link_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    int h_status = 0;
    e = cudaMemcpyAsync(&h_status, &S->status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    if (h_status & ST_POSITION) return SIMOX_E_POSITION;
    if (h_status & ST_CELL_OVERFLOW) return SIMOX_E_CELL_OVERFLOW;
    return SIMOX_OK;
}
