// Puts a re-trace list into sample order. The speculative passes append the
// samples they hand to the FP64 re-trace in the order they find them, which
// leaves the longest rays (found last) at the end of the list and makes them
// the re-trace's tail. Sorted by sample index, the list is traced in the
// order the FP64 form traces the frame.
//
// The list holds distinct indices in [0, n): they are marked in a bitmap, and
// a stream compaction of the bitmap (per-block popcounts, one scan of the
// block sums, then an ordered write) rewrites the list. The count does not
// change.
#include <cuda_runtime.h>

#include <cstdint>

#include "render_launch.h"

namespace grrt_b200 {

namespace {

constexpr int kOrdThreads = 256;
constexpr int kWordsPerThread = 8;
constexpr unsigned kWordsPerBlock = kOrdThreads * kWordsPerThread;  // 65536 samples

__global__ void __launch_bounds__(kOrdThreads) mark_kernel(const unsigned* __restrict__ list,
                                                           const unsigned* __restrict__ count, unsigned n,
                                                           unsigned* __restrict__ bitmap) {
    const unsigned c = *count;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const unsigned q = list[i];
        if (q < n) atomicOr(bitmap + (q >> 5), 1u << (q & 31u));
    }
}

// Exclusive scan of one value per thread over the block (warp shuffles, then
// the warp totals); returns the block total in *total.
__device__ unsigned block_exclusive_scan(unsigned v, unsigned* total) {
    __shared__ unsigned warp_sums[kOrdThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned s = (lane < kOrdThreads / 32) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kOrdThreads / 32) warp_sums[lane] = s;  // inclusive warp prefix
    }
    __syncthreads();
    const unsigned before = (w > 0) ? warp_sums[w - 1] : 0u;
    *total = warp_sums[kOrdThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

__device__ unsigned thread_popcount(const unsigned* __restrict__ bitmap, unsigned words, unsigned w0) {
    unsigned c = 0;
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) {
        const unsigned w = w0 + k;
        if (w < words) c += __popc(bitmap[w]);
    }
    return c;
}

__global__ void __launch_bounds__(kOrdThreads) count_kernel(const unsigned* __restrict__ bitmap, unsigned words,
                                                            unsigned* __restrict__ block_sums) {
    const unsigned w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
    unsigned total;
    block_exclusive_scan(thread_popcount(bitmap, words, w0), &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the block sums in place (any number of blocks).
__global__ void __launch_bounds__(kOrdThreads) scan_sums_kernel(unsigned* __restrict__ block_sums, unsigned nblocks) {
    unsigned carry = 0;
    for (unsigned base = 0; base < nblocks; base += kOrdThreads) {
        const unsigned i = base + threadIdx.x;
        const unsigned v = (i < nblocks) ? block_sums[i] : 0u;
        unsigned total;
        const unsigned ex = block_exclusive_scan(v, &total);
        if (i < nblocks) block_sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kOrdThreads) write_kernel(const unsigned* __restrict__ bitmap, unsigned words,
                                                            const unsigned* __restrict__ block_offsets,
                                                            unsigned* __restrict__ list) {
    const unsigned w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
    unsigned total;
    unsigned pos = block_offsets[blockIdx.x] + block_exclusive_scan(thread_popcount(bitmap, words, w0), &total);
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) {
        const unsigned w = w0 + k;
        if (w >= words) break;
        unsigned bits = bitmap[w];
        while (bits) {
            const int b = __ffs(bits) - 1;
            list[pos++] = w * 32u + static_cast<unsigned>(b);
            bits &= bits - 1u;
        }
    }
}

}  // namespace

size_t order_list_scratch_bytes(size_t n) {
    const size_t words = (n + 31) / 32;
    const size_t blocks = (words + kWordsPerBlock - 1) / kWordsPerBlock;
    return ((words * sizeof(unsigned) + 255) / 256) * 256 + ((blocks * sizeof(unsigned) + 255) / 256) * 256;
}

cudaError_t order_sample_list(unsigned* list, const unsigned* count, size_t n, void* scratch, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (n > 0xffffffffull || !list || !count || !scratch) return cudaErrorInvalidValue;
    const unsigned words = static_cast<unsigned>((n + 31) / 32);
    const unsigned blocks = (words + kWordsPerBlock - 1) / kWordsPerBlock;
    auto* bitmap = static_cast<unsigned*>(scratch);
    auto* block_sums =
        reinterpret_cast<unsigned*>(static_cast<unsigned char*>(scratch) + ((words * sizeof(unsigned) + 255) / 256) * 256);
    cudaError_t e = cudaMemsetAsync(bitmap, 0, words * sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    mark_kernel<<<(sms > 0 ? sms : 1) * 4, kOrdThreads, 0, stream>>>(list, count, static_cast<unsigned>(n), bitmap);
    count_kernel<<<blocks, kOrdThreads, 0, stream>>>(bitmap, words, block_sums);
    scan_sums_kernel<<<1, kOrdThreads, 0, stream>>>(block_sums, blocks);
    write_kernel<<<blocks, kOrdThreads, 0, stream>>>(bitmap, words, block_sums, list);
    return cudaGetLastError();
}

}  // namespace grrt_b200
