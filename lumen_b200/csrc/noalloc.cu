/*
 * noalloc.cu - lumen_gpu_sort_pairs_noalloc: the stable pair sort of
 * lumen_gpu_sort_pairs for callers that cannot allocate device memory.
 *
 * Who needs it: code embedded in a host application that owns every byte of
 * device memory (an engine plugin or an FFI host with its own allocator and
 * budget), and frame loops that must not call cudaMalloc/cudaFree because
 * those calls can synchronise the whole device. Such a caller passes only
 * its keys and values; the sort's control block, look-back descriptors and
 * alternate key/value buffers live in one file-scope device array,
 * g_noalloc_scratch, sized for LUMEN_GPU_NOALLOC_MAX_PAIRS pairs
 * (about 3.6 MB, held by every GPU that loads the library until the process
 * exits).
 *
 * Host code cannot use g_noalloc_scratch's name as a device address, so the
 * first call on each device (with that device current) looks the address up
 * with cudaGetSymbolAddress and caches it, and raises the digit passes'
 * shared memory limit on that device; that first call should come before
 * any stream capture. Every call shares the array and finds the previous
 * call's contents in it: the control block is cleared on each call, and calls
 * whose work overlaps on the GPU (different streams, or different host
 * threads on one device) race on the array and must be serialised by the
 * caller.
 */
#include <cstring>
#include <mutex>

#include "splat_common.cuh"

namespace lumen {

void launch_sort64(unsigned long long* k0, unsigned int* v0, unsigned long long* k1, unsigned int* v1,
                   long long capacity, SortControl* sc, unsigned int* lb, long long lb_tiles_cap, unsigned int* err,
                   int num_sms, cudaStream_t st);
void launch_key_stats64(const unsigned long long* keys, long long n, SortControl* sc, int num_sms, cudaStream_t st);
int device_sm_count();
LumenStatus map_cuda(cudaError_t e);
LumenStatus status_from_flags(unsigned int flags);
void configure_sort_kernels();

namespace {

constexpr long long kMaxPairs = LUMEN_GPU_NOALLOC_MAX_PAIRS;
/* look-back descriptors are addressed by the 64-bit sort's tile, which the
 * standalone scratch layout (ScratchLayout) also sizes by */
constexpr long long kTiles = (kMaxPairs + kSort64Tile - 1) / kSort64Tile;
static_assert(kSort64Tile == kSortTile, "the 64-bit sort's tile must be the tile the scratch layout counts");
constexpr size_t kControlBytes = align_up(sizeof(Control), 256) + align_up(view_table_bytes(1), 256);
/* control block and a one-view table, then 8 digit passes x tiles x 256
 * look-back descriptors */
constexpr size_t kScratchBytes = kControlBytes + (size_t)8 * (size_t)kTiles * 256 * sizeof(unsigned int);
constexpr size_t kAltKeysBytes = (size_t)kMaxPairs * sizeof(unsigned long long);
constexpr size_t kAltValsBytes = (size_t)kMaxPairs * sizeof(unsigned int);

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes + kAltKeysBytes + kAltValsBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_address[kMaxDevices] = {};
bool g_configured[kMaxDevices] = {};

/* Set-up on the current device, once per device: the device address of
 * g_noalloc_scratch, and the digit passes' dynamic shared memory limit
 * above 48 KB (a kernel attribute that applies to the device current when
 * it is set; this may be the first call into the library on the device). */
cudaError_t device_setup(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_address[dev] = p;
    }
    if (!g_configured[dev]) {
        configure_sort_kernels();
        g_configured[dev] = true;
    }
    *out = g_address[dev];
    return cudaSuccess;
}

/* Copy the sorted pairs back when the last digit pass left them in the
 * alternate buffers (decided on the device). */
__global__ void copy_back_kernel(const Control* ctrl, unsigned long long* keys, unsigned int* vals,
                                 const unsigned long long* alt_keys, const unsigned int* alt_vals, long long n) {
    if (ctrl->tile_sort.sorted_buffer == 0) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        keys[i] = alt_keys[i];
        vals[i] = alt_vals[i];
    }
}

}  // namespace
}  // namespace lumen

using namespace lumen;

extern "C" LumenStatus lumen_gpu_sort_pairs_noalloc(uint64_t* keys, uint32_t* vals, int64_t n, void* stream) {
    if (n < 0 || n > kMaxPairs) return LUMEN_ERROR_INVALID_ARGUMENT;   /* beyond the static array */
    if (n > 0 && (!keys || !vals)) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n == 0) return LUMEN_SUCCESS;
    /* the regular layout of a standalone sort must fit the static array */
    const ScratchLayout L = ScratchLayout::make(0, kMaxPairs);
    if (L.tile_lb_off != kControlBytes || L.total > kScratchBytes) return LUMEN_ERROR_INVALID_ARGUMENT;
    void* addr = nullptr;
    cudaError_t e = device_setup(&addr);
    if (e != cudaSuccess) return map_cuda(e);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)addr;
    Control* ctrl = (Control*)base;
    unsigned int* lb = (unsigned int*)(base + kControlBytes);
    unsigned long long* alt_keys = (unsigned long long*)(base + kScratchBytes);
    unsigned int* alt_vals = (unsigned int*)(base + kScratchBytes + kAltKeysBytes);
    unsigned long long* k = reinterpret_cast<unsigned long long*>(keys);
    /* the previous call's control block is still there: start from zero */
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Control), s)) != cudaSuccess) return map_cuda(e);
    const int sms = device_sm_count();
    launch_key_stats64(k, n, &ctrl->tile_sort, sms, s);
    launch_sort64(k, vals, alt_keys, alt_vals, n, &ctrl->tile_sort, lb, kTiles, &ctrl->error_flags, sms, s);
    copy_back_kernel<<<sms * 4, 256, 0, s>>>(ctrl, k, vals, alt_keys, alt_vals, n);
    if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(e);
    unsigned int flags = 0;
    e = cudaMemcpyAsync(&flags, &ctrl->error_flags, sizeof(flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    return status_from_flags(flags);
}
