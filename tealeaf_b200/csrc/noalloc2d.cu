// noalloc2d.cu -- an allocation-free variant of the 2D 2-norm reduction.
//
// Why it exists: the regular entry point run_calculate_2norm reduces through
// scratch memory that run_kernel_initialise obtained with cudaMalloc (one
// partial sum per block, a ticket counter, a mapped host result slot). Some
// callers cannot make that allocation, or cannot afford it: a host that has
// handed (nearly) all device memory to its own pool allocator and must not
// fail with out-of-memory in the middle of a solve, or latency-sensitive code
// that must not take the device-wide synchronisation cudaFree implies. For
// them tl2d_calculate_2norm_noalloc computes the same sum (equal to
// run_calculate_2norm's up to rounding: its blocks cover 8 rows where the
// regular sweep's cover a per-mesh row count, so the partials are added in
// another tree) with its scratch in a fixed static device array.
//
// When the array is reserved: under CUDA's lazy module loading (the default
// since CUDA 12.2) the driver loads this file's module, and with it the
// array, the first time its address is looked up. run_kernel_initialise does
// that look-up (tl_noalloc_prepare below), so a host that calls it, as every
// TeaLeaf host does, has the array in place before it hands the rest of the
// device memory to its pool. A caller that uses this entry point without
// run_kernel_initialise should make its first call before that hand-over, or
// run with CUDA_MODULE_LOADING=EAGER, which loads the array with the library.
//
// The limit: the array holds kMaxBlocks block partials, one per block of the
// interior sweep (128 columns x 8 rows per block), which covers interior
// grids of up to 65536 blocks, e.g. 8192 x 8192 cells. Larger grids are
// rejected with an error; nothing is launched for them.
//
// Every call on a device shares the one array, and it keeps the previous
// call's contents. Each call therefore clears the ticket counter before its
// launch. Calls that overlap on the GPU (for example on two streams at once)
// race on the array and give wrong results: serialise them.
#include "common.cuh"
#include "tealeaf_b200_2d.h"

#include <cuda_runtime.h>
#include <atomic>

namespace {

// Launch shape: 128 columns x 8 rows per block (one partial per block).
constexpr int kBX = 128;
constexpr int kRows = 8;
constexpr long kMaxBlocks = 65536;
constexpr int kMaxDevices = 64;

// Scratch: [0, kMaxBlocks) block partials; then the ticket word and a result
// slot, each on its own 256-byte line. Reserved for every GPU that loads the
// library, until the process exits (about 512 KiB).
constexpr long kTicketOffset = kMaxBlocks;
constexpr long kResultOffset = kMaxBlocks + 32;
static __device__ __align__(256) double g_norm_scratch[kMaxBlocks + 64];

// Host-side cache of the scratch array's device address, per device. Two
// host threads making their first call at once both store the same address.
std::atomic<double*> g_scratch_addr[kMaxDevices];

struct AccumulateInto {
    double* out;
    __device__ void operator()(const double* total) const { *out += total[0]; }
};

__global__ void __launch_bounds__(kBX) k_norm2_noalloc(int x, int y, int hd, const double* __restrict__ b,
                                                      tl::ReduceSlots rs, double* __restrict__ norm_dev)
{
    const int k = hd + blockIdx.x * kBX + threadIdx.x;
    const int j0 = hd + blockIdx.y * kRows;
    const int j1 = min(j0 + kRows, y - hd);
    double acc[1] = {0.0};
    if (k < x - hd) {
        long i = k + (long)j0 * x;
#pragma unroll 4
        for (int j = j0; j < j1; ++j, i += x) acc[0] += b[i] * b[i];
    }
    tl::grid_sum<1, kBX>(acc, rs, blockIdx.x + blockIdx.y * gridDim.x, gridDim.x * gridDim.y,
                         AccumulateInto{norm_dev});
}

// The scratch array's device address on the current device (looked up once,
// which loads the module under lazy loading); nullptr after a recorded error.
double* scratch_on_current_device(int code)
{
    int dev = 0;
    if (!TL_CUDA(cudaGetDevice(&dev))) return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        tl::fail(code, "tl2d_calculate_2norm_noalloc: device %d out of range", dev);
        return nullptr;
    }
    double* addr = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!addr) {
        if (!TL_CUDA(cudaGetSymbolAddress((void**)&addr, g_norm_scratch))) return nullptr;
        g_scratch_addr[dev].store(addr, std::memory_order_release);
    }
    return addr;
}

}  // namespace

// Called by run_kernel_initialise with the chunk's device current, so the
// static scratch is in place before the host's solve starts.
bool tl_noalloc_prepare()
{
    return scratch_on_current_device(24) != nullptr;
}

extern "C" int tl2d_calculate_2norm_noalloc(const double* field, int x, int y, int halo_depth, double* norm_dev,
                                            void* stream)
{
    // 1. Validate before touching the device.
    if (!field || !norm_dev) {
        tl::fail(20, "tl2d_calculate_2norm_noalloc: field and norm_dev must be device pointers");
        return 20;
    }
    if (halo_depth < 1 || x < 2 * halo_depth + 1 || y < 2 * halo_depth + 1) {
        tl::fail(21, "tl2d_calculate_2norm_noalloc: invalid extents x=%d y=%d halo_depth=%d", x, y, halo_depth);
        return 21;
    }
    const long gx = tl::ceil_div(x - 2 * halo_depth, kBX);
    const long gy = tl::ceil_div(y - 2 * halo_depth, kRows);
    if (gx * gy > kMaxBlocks || gy > 65535) {
        tl::fail(22,
                 "tl2d_calculate_2norm_noalloc: interior %d x %d needs %ld reduction blocks; the static "
                 "scratch holds %ld (about 8192 x 8192 cells). Use run_calculate_2norm for larger grids.",
                 x - 2 * halo_depth, y - 2 * halo_depth, gx * gy, kMaxBlocks);
        return 22;
    }
    // 2. Once per device, with that device current: the scratch array's address.
    double* scratch = scratch_on_current_device(24);
    if (!scratch) return 25;
    cudaStream_t st = (cudaStream_t)stream;
    tl::ReduceSlots rs;
    rs.partials = scratch;
    rs.ticket = (unsigned int*)(scratch + kTicketOffset);
    rs.out_dev = scratch + kResultOffset;
    rs.out_host = nullptr;
    // 3. The ticket must start at zero; the array keeps the last call's contents.
    if (!TL_CUDA(cudaMemsetAsync(rs.ticket, 0, sizeof(unsigned int), st))) return 26;
    k_norm2_noalloc<<<dim3((unsigned)gx, (unsigned)gy), kBX, 0, st>>>(x, y, halo_depth, field, rs, norm_dev);
    if (!TL_LAUNCHED("k_norm2_noalloc")) return 27;
    return 0;
}
