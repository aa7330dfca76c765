// io.cu -- array transfers between device arrays and page-locked, device-mapped host
// buffers, as kernels a captured CUDA graph can hold.  AGO keeps an array's item count in
// its device buffer header (DATA_GPU_ARRAY_OFFSET, ago_internal.h:171) and reads it back
// with a blocking copy before the items (ago_util_hip.cpp:321-608); here the count word
// and the items cross PCIe inside the graph, so a graph's array inputs and outputs cost no
// host round trip per array.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

constexpr int kIoThreads = 256;
constexpr int kIoBlocks = 16;

__device__ __forceinline__ void copy_bytes(uint8_t *dst, const uint8_t *src, size_t bytes)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x, n = (size_t)gridDim.x * blockDim.x;
    if ((((uintptr_t)dst | (uintptr_t)src | bytes) & 3) == 0) {
        const uint32_t *s = (const uint32_t *)src;
        uint32_t *d = (uint32_t *)dst;
        for (size_t i = t; i < bytes / 4; i += n) d[i] = s[i];
    } else {
        for (size_t i = t; i < bytes; i += n) dst[i] = src[i];
    }
}

// count slot: kArraySkip leaves the device array as it is
__global__ void __launch_bounds__(kIoThreads)
k_array_upload(uint8_t *dev, uint32_t *devCount, const uint8_t *host, const volatile uint32_t *slot,
               uint32_t itemSize, uint32_t capacity)
{
    __shared__ uint32_t n;
    if (threadIdx.x == 0) n = *slot;
    __syncthreads();
    if (n == AGOCUDA_ARRAY_SKIP) return;
    const uint32_t m = min(n, capacity);
    copy_bytes(dev, host, (size_t)m * itemSize);
    if (blockIdx.x == 0 && threadIdx.x == 0) *devCount = m;
}

// blockIdx.y: the transfer
__global__ void __launch_bounds__(kIoThreads) k_array_upload_batch(const agocuda_array_xfer *xfers)
{
    const agocuda_array_xfer X = xfers[blockIdx.y];
    __shared__ uint32_t n;
    if (threadIdx.x == 0) n = *(const volatile uint32_t *)X.countSlotMapped;
    __syncthreads();
    if (n == AGOCUDA_ARRAY_SKIP) return;
    const uint32_t m = min(n, X.capacity);
    copy_bytes((uint8_t *)X.devItems, (const uint8_t *)X.hostItemsMapped, (size_t)m * X.itemSize);
    if (blockIdx.x == 0 && threadIdx.x == 0) *X.devCount = m;
}

__global__ void __launch_bounds__(kIoThreads)
k_array_download(uint8_t *host, volatile uint32_t *slot, const uint8_t *dev, const uint32_t *devCount,
                 uint32_t itemSize, uint32_t capacity)
{
    const uint32_t m = min(*devCount, capacity);
    copy_bytes(host, dev, (size_t)m * itemSize);
    if (blockIdx.x == 0 && threadIdx.x == 0) *slot = m;
}

}  // namespace

extern "C" int agocuda_array_upload(void *stream, void *devItems, uint32_t *devCount, const void *hostItemsMapped,
                                    const uint32_t *countSlotMapped, uint32_t itemSize, uint32_t capacity)
{
    if (!devItems || !devCount || !hostItemsMapped || !countSlotMapped || !itemSize || !capacity)
        return AGOCUDA_INVALID_PARAMS;
    k_array_upload<<<kIoBlocks, kIoThreads, 0, as_stream(stream)>>>((uint8_t *)devItems, devCount,
                                                                    (const uint8_t *)hostItemsMapped, countSlotMapped,
                                                                    itemSize, capacity);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_array_upload_batch(void *stream, const agocuda_array_xfer *xfers, uint32_t count)
{
    if (!xfers || !count || count > 65535) return AGOCUDA_INVALID_PARAMS;
    k_array_upload_batch<<<dim3(kIoBlocks, count), kIoThreads, 0, as_stream(stream)>>>(xfers);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_array_download(void *stream, void *hostItemsMapped, uint32_t *countSlotMapped,
                                      const void *devItems, const uint32_t *devCount, uint32_t itemSize,
                                      uint32_t capacity)
{
    if (!devItems || !devCount || !hostItemsMapped || !countSlotMapped || !itemSize || !capacity)
        return AGOCUDA_INVALID_PARAMS;
    k_array_download<<<kIoBlocks, kIoThreads, 0, as_stream(stream)>>>((uint8_t *)hostItemsMapped, countSlotMapped,
                                                                      (const uint8_t *)devItems, devCount, itemSize,
                                                                      capacity);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
