// Neighbour-list build that allocates no device memory (dmffb_build_neighbors_noalloc).
//
// Some callers cannot allocate device memory on demand: an MD engine or plugin host whose
// platform owns the whole device heap (OpenMM-style contexts that hand out only their own
// buffers), a process that runs under a fixed memory budget with the allocator locked after
// start-up, or code that must not fragment or grow the caching allocator of a framework sharing
// the GPU.  For them this entry point runs the same cell-list kernels as dmffb_build_neighbors
// with every scratch buffer (cell bins, per-atom counts and offsets, the scan's temporary
// storage) carved out of one file-scope device array of fixed size, so a call performs no
// cudaMalloc / cudaFree and calls no allocating library routine.
//
// Limits: at most DMFFB_NOALLOC_MAX_ATOMS atoms and DMFFB_NOALLOC_MAX_CELLS cells (the cell grid
// is coarsened to fit; cells only need to be at least rc wide).  Every GPU that loads the
// library holds the array (about 2.6 MB) until the process exits.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cmath>
#include <mutex>

#include "../../include/dmffb200.h"
#include "nblist.cuh"

using namespace dmffb;

namespace {

constexpr size_t kAtoms = DMFFB_NOALLOC_MAX_ATOMS;
constexpr size_t kCells = DMFFB_NOALLOC_MAX_CELLS;
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
// scratch regions, in order
constexpr size_t kOffAtomCell = 0;
constexpr size_t kOffCellAtoms = kOffAtomCell + align256(kAtoms * 4);
constexpr size_t kOffCount = kOffCellAtoms + align256(kAtoms * 4);
constexpr size_t kOffOffsets = kOffCount + align256(kAtoms * 4);
constexpr size_t kOffCellCount = kOffOffsets + align256((kAtoms + 1) * 8);
constexpr size_t kOffCellStart = kOffCellCount + align256((kCells + 1) * 4);
constexpr size_t kOffCellCursor = kOffCellStart + align256((kCells + 1) * 4);
constexpr size_t kOffEmptyCov = kOffCellCursor + align256((kCells + 1) * 4);
constexpr size_t kOffScanTemp = kOffEmptyCov + align256((kAtoms + 1) * 4);
constexpr size_t kScanTempBytes = 512 * 1024;
constexpr size_t kScratchBytes = kOffScanTemp + kScanTempBytes;

// The scratch itself.  Host code must not use this name as a device address: it is a host-side
// stand-in; kernels get the address returned by cudaGetSymbolAddress for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// one-time set-up per device, with that device current: look up the array's device address
int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DMFFB_CUDA_ERROR;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DMFFB_CUDA_ERROR;
        g_scratch_ptr[dev] = p;
    }
    *out = (unsigned char*)g_scratch_ptr[dev];
    return DMFFB_OK;
}

void make_box_host(const double* m, Box& bx) {
    for (int k = 0; k < 9; ++k) bx.h[k] = m[k];
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    double inv[9] = {(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det,
                     (m[1] * m[5] - m[2] * m[4]) / det, (m[5] * m[6] - m[3] * m[8]) / det,
                     (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                     (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det,
                     (m[0] * m[4] - m[1] * m[3]) / det};
    if (m[1] == 0 && m[2] == 0 && m[3] == 0 && m[5] == 0 && m[6] == 0 && m[7] == 0) {
        for (int k = 0; k < 9; ++k) inv[k] = 0.0;
        inv[0] = 1.0 / m[0];
        inv[4] = 1.0 / m[4];
        inv[8] = 1.0 / m[8];
    }
    for (int k = 0; k < 9; ++k) bx.hinv[k] = inv[k];
}

inline unsigned nb(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" int dmffb_build_neighbors_noalloc(void* stream, const double* pos, int32_t n_atoms, const double* box,
                                             double rc, const int32_t* cov_ptr, const int32_t* cov_j,
                                             const int32_t* cov_nb, int32_t* pairs_out, int64_t capacity,
                                             int64_t* npairs_out) {
    if (!pos || !box || !npairs_out || n_atoms <= 0 || !(rc > 0)) return DMFFB_BAD_ARG;
    if ((size_t)n_atoms > kAtoms) return DMFFB_SCRATCH_TOO_SMALL;
    if ((cov_ptr == nullptr) != (cov_j == nullptr) || (cov_ptr == nullptr) != (cov_nb == nullptr)) return DMFFB_BAD_ARG;
    unsigned char* scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = n_atoms;
    Box bx;
    make_box_host(box, bx);
    // cells per axis from the perpendicular widths, coarsened until the grid fits the scratch
    const double* m = bx.h;
    const double V = fabs(m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                          m[2] * (m[3] * m[7] - m[4] * m[6]));
    int nc[3];
    bool cells = true;
    for (int k = 0; k < 3; ++k) {
        const double* u = m + 3 * ((k + 1) % 3);
        const double* w = m + 3 * ((k + 2) % 3);
        const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        nc[k] = (int)floor(V / sqrt(cx * cx + cy * cy + cz * cz) / rc);
        if (nc[k] > 64) nc[k] = 64;
        if (nc[k] < 3) cells = false;
    }
    while (cells && (size_t)nc[0] * nc[1] * nc[2] > kCells) {
        int kmax = nc[0] >= nc[1] && nc[0] >= nc[2] ? 0 : (nc[1] >= nc[2] ? 1 : 2);
        nc[kmax] -= 1;
        if (nc[kmax] < 3) cells = false;
    }
    const int ncell = cells ? nc[0] * nc[1] * nc[2] : 1;
    int32_t* atom_cell = (int32_t*)(scratch + kOffAtomCell);
    int32_t* cell_atoms = (int32_t*)(scratch + kOffCellAtoms);
    int32_t* count = (int32_t*)(scratch + kOffCount);
    int64_t* offsets = (int64_t*)(scratch + kOffOffsets);
    int32_t* cell_count = (int32_t*)(scratch + kOffCellCount);
    int32_t* cell_start = (int32_t*)(scratch + kOffCellStart);
    int32_t* cell_cursor = (int32_t*)(scratch + kOffCellCursor);
    void* temp = (void*)(scratch + kOffScanTemp);
    size_t need1 = 0, need2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need1, (int32_t*)nullptr, (int32_t*)nullptr, ncell + 1);
    cub::DeviceScan::InclusiveSum(nullptr, need2, (int32_t*)nullptr, (int64_t*)nullptr, n);
    if (need1 > kScanTempBytes || need2 > kScanTempBytes) return DMFFB_SCRATCH_TOO_SMALL;

    NbArgs a;
    a.n = n;
    a.pos = pos;
    a.box = bx;
    a.rc = rc;
    for (int k = 0; k < 3; ++k) a.nc[k] = cells ? nc[k] : 1;
    a.cov_ptr = cov_ptr;
    a.cov_j = cov_j;
    a.cov_nb = cov_nb;
    if (!cov_ptr) {  // no covalent map: every atom gets an empty row list, so every nbond is 0
        int32_t* empty = (int32_t*)(scratch + kOffEmptyCov);
        if (cudaMemsetAsync(empty, 0, (size_t)(n + 1) * 4, s) != cudaSuccess) return DMFFB_CUDA_ERROR;
        a.cov_ptr = empty;
        a.cov_j = empty;
        a.cov_nb = empty;
    }
    a.count = count;
    a.offset = offsets;
    a.pairs = pairs_out;
    a.cap = pairs_out ? capacity : 0;
    // the array keeps the previous call's contents: zero every counter this call accumulates into
    if (cudaMemsetAsync(offsets, 0, sizeof(int64_t), s) != cudaSuccess) return DMFFB_CUDA_ERROR;
    if (cells) {
        if (cudaMemsetAsync(cell_count, 0, (size_t)(ncell + 1) * 4, s) != cudaSuccess) return DMFFB_CUDA_ERROR;
        if (cudaMemsetAsync(cell_cursor, 0, (size_t)(ncell + 1) * 4, s) != cudaSuccess) return DMFFB_CUDA_ERROR;
        k_cell_count<<<nb(n, 256), 256, 0, s>>>(n, pos, bx, nc[0], nc[1], nc[2], atom_cell, cell_count);
        if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
        size_t tb = kScanTempBytes;
        if (cub::DeviceScan::ExclusiveSum(temp, tb, cell_count, cell_start, ncell + 1, s) != cudaSuccess)
            return DMFFB_CUDA_ERROR;
        k_cell_fill<<<nb(n, 256), 256, 0, s>>>(n, atom_cell, cell_start, cell_cursor, cell_atoms);
        if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
        a.cell_start = cell_start;
        a.cell_atoms = cell_atoms;
        k_pairs_warp<0><<<nb((int64_t)n * 32, 256), 256, 0, s>>>(a);
    } else {
        k_pairs_all<0><<<nb(n, 128), 128, 0, s>>>(a);
    }
    // a failed launch here would leave the count pass undone and the total below stale (the
    // array keeps the previous call's offsets), so check before reading it
    if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
    size_t tb = kScanTempBytes;
    if (cub::DeviceScan::InclusiveSum(temp, tb, count, offsets + 1, n, s) != cudaSuccess) return DMFFB_CUDA_ERROR;
    int64_t total = 0;
    if (cudaMemcpyAsync(&total, offsets + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return DMFFB_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DMFFB_CUDA_ERROR;
    *npairs_out = total;
    if (total > capacity || !pairs_out) return DMFFB_NEIGHBOR_OVERFLOW;
    if (cells) k_pairs_warp<1><<<nb((int64_t)n * 32, 256), 256, 0, s>>>(a);
    else k_pairs_all<1><<<nb(n, 128), 128, 0, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DMFFB_CUDA_ERROR;
    return DMFFB_OK;
}
