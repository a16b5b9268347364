// noalloc.cu -- compaction order of a point set without any device allocation.
//
// icempm_cell_order_noalloc computes the order icempm_sort_compact applies
// (remove disabled points, sort the rest by cell index x*GridY + y, ties in
// index order) for callers that must not allocate device memory: code running
// under a host framework that owns every device byte (a fixed memory pool, a
// caching allocator they may not bypass), or callers that issue work into a
// stream they do not control and cannot synchronise for cudaMalloc/cudaFree.
// The caller passes device inputs and outputs; every intermediate buffer --
// sort keys, values and the radix sort's temporary storage -- lives in one
// file-scope static device array of fixed size (36 MiB), which every GPU that loads
// this library keeps until the process exits.
#include <cstdint>
#include <mutex>
#include <string>

#include <cub/device/device_radix_sort.cuh>

#include "engine_iface.h"

namespace {

constexpr uint32_t kMaxPoints = ICEMPM_NOALLOC_MAX_POINTS;
constexpr size_t kKeyBytes = (size_t)kMaxPoints * sizeof(uint64_t);
constexpr size_t kValBytes = (size_t)kMaxPoints * sizeof(uint32_t);
constexpr size_t kTempBytes = (size_t)16 << 20;  // radix sort temporary storage, checked at set-up
constexpr size_t kScratchBytes = 2 * kKeyBytes + kValBytes + kTempBytes;   // 36 MiB
constexpr int kMaxDevices = 64;

}  // namespace

// Static scratch: [keys | alternate keys | alternate values | radix sort temp].  Host
// code must not use this name as an address: it is a host-side stand-in; the
// device address comes from cudaGetSymbolAddress, with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mutex;
bool g_temp_checked[kMaxDevices] = {};

// With the device current: the scratch array's device address (looked up on
// every call, which allocates nothing; a cached address would go stale after
// cudaDeviceReset), and once per device the check that the radix sort fits
// its reserved temporary storage.
int scratch_for_current_device(unsigned char **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return icempm::fail(ICEMPM_E_UNSUPPORTED, "device ordinal out of range");
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return icempm::fail(ICEMPM_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_temp_checked[dev]) {
        size_t need = 0;
        cub::DoubleBuffer<uint64_t> kb(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
        e = cub::DeviceRadixSort::SortPairs(nullptr, need, kb, vb, (int)kMaxPoints, 0, 64);
        if (e != cudaSuccess)
            return icempm::fail(ICEMPM_E_CUDA, std::string("radix sort size query: ") + cudaGetErrorString(e));
        if (need > kTempBytes)
            return icempm::fail(ICEMPM_E_UNSUPPORTED, "radix sort needs " + std::to_string(need) +
                                                          " bytes of temporary storage, more than the " +
                                                          std::to_string(kTempBytes) + " reserved");
        g_temp_checked[dev] = true;
    }
    *out = static_cast<unsigned char *>(p);
    return ICEMPM_OK;
}

// Bits that hold every value below v (at least 1).
int bits_below(uint64_t v)
{
    int b = 1;
    while (b < 64 && (v >> b) != 0) b++;
    return b;
}

// Key = cell index x*GridY + y shifted above the point index (ties in index
// order): (cell << ib) | i, below `sentinel` = 1 << (ib + cb); disabled points
// get the sentinel.  Only the low ib + cb + 1 bits take part in the sort.
__global__ void k_noalloc_keys(const uint32_t *__restrict__ cell, const uint32_t *__restrict__ util, uint32_t n,
                               uint32_t gy, int ib, uint64_t sentinel, uint64_t *keys, uint32_t *vals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t key = sentinel;
    if (!(util[i] & ICEMPM_STATUS_DISABLED)) {
        const uint64_t c = cell[i];
        key = (((c & 0xffffu) * (uint64_t)gy + (c >> 16)) << ib) | i;
    }
    keys[i] = key;
    vals[i] = i;
}

// Number of enabled points = length of the leading run of keys below the sentinel.
__global__ void k_noalloc_count(const uint64_t *__restrict__ keys, uint32_t n, uint64_t sentinel, uint32_t *count)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool act = keys[i] != sentinel;
    const bool next_inact = (i == n - 1) || keys[i + 1] == sentinel;
    if (act && next_inact) *count = i + 1;
    if (i == 0 && !act) *count = 0;
}

}  // namespace

extern "C" int icempm_cell_order_noalloc(const uint32_t *d_cell, const uint32_t *d_utility, uint32_t n,
                                         int32_t grid_y, uint32_t *d_order, uint32_t *d_count, void *stream)
{
    if (n > kMaxPoints)
        return icempm::fail(ICEMPM_E_CAPACITY, "n = " + std::to_string(n) + " exceeds ICEMPM_NOALLOC_MAX_POINTS (" +
                                                   std::to_string(kMaxPoints) + ")");
    if (!d_count || (n > 0 && (!d_cell || !d_utility || !d_order)))
        return icempm::fail(ICEMPM_E_ARG, "null device pointer");
    if (grid_y <= 0) return icempm::fail(ICEMPM_E_ARG, "grid_y must be > 0");
    unsigned char *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (n == 0) {
        e = cudaMemsetAsync(d_count, 0, sizeof(uint32_t), s);
        if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
        return ICEMPM_OK;
    }
    uint64_t *keys_a = reinterpret_cast<uint64_t *>(scratch);
    uint64_t *keys_b = reinterpret_cast<uint64_t *>(scratch + kKeyBytes);
    uint32_t *vals_b = reinterpret_cast<uint32_t *>(scratch + 2 * kKeyBytes);
    void *temp = scratch + 2 * kKeyBytes + kValBytes;
    const unsigned nb = (n + 255) / 256;
    // cell indices stay below 65536 * grid_y (x and y are 16-bit fields)
    const int ib = bits_below((uint64_t)n - 1);
    const int cb = bits_below((uint64_t)65535 * (uint64_t)grid_y + 65535);
    const int end_bit = ib + cb + 1;
    const uint64_t sentinel = 1ull << (ib + cb);
    // keys and indices are generated into keys_a and the caller's d_order; the
    // double-buffered radix sort ping-pongs with keys_b / vals_b
    k_noalloc_keys<<<nb, 256, 0, s>>>(d_cell, d_utility, n, (uint32_t)grid_y, ib, sentinel, keys_a, d_order);
    e = cudaGetLastError();
    if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("key kernel: ") + cudaGetErrorString(e));
    cub::DoubleBuffer<uint64_t> kb(keys_a, keys_b);
    cub::DoubleBuffer<uint32_t> vb(d_order, vals_b);
    size_t temp_bytes = kTempBytes;
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, kb, vb, (int)n, 0, end_bit, s);
    if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("radix sort: ") + cudaGetErrorString(e));
    if (vb.Current() != d_order) {
        e = cudaMemcpyAsync(d_order, vb.Current(), (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("order copy: ") + cudaGetErrorString(e));
    }
    k_noalloc_count<<<nb, 256, 0, s>>>(kb.Current(), n, sentinel, d_count);
    e = cudaGetLastError();
    if (e != cudaSuccess) return icempm::fail(ICEMPM_E_CUDA, std::string("count kernel: ") + cudaGetErrorString(e));
    return ICEMPM_OK;
}
