// Device-side FITS plane packing: plane k of a [pixel][bin] double cube to
// big-endian doubles in FITS row order (the byte swap and row flip of
// FITSStreamWriter::write_row, src/fits_writer.cpp:356-395, done on the GPU so
// the host only streams bytes to the file).
#include <cuda_runtime.h>

#include "../fits.h"

namespace grrt_b200 {

__global__ void pack_fits_plane_kernel(const double* __restrict__ cube, int width, int height, int nb, int k,
                                       unsigned long long* __restrict__ out) {
    const size_t n = static_cast<size_t>(width) * height;
    for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
         q += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int fits_row = static_cast<int>(q / width);
        const int i = static_cast<int>(q % width);
        const int j = height - 1 - fits_row;
        const double v = cube[(static_cast<size_t>(j) * width + i) * nb + k];
        unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(v));
        // byte swap: big-endian on disk
        const unsigned lo = static_cast<unsigned>(bits), hi = static_cast<unsigned>(bits >> 32);
        const unsigned long long be = (static_cast<unsigned long long>(__byte_perm(lo, 0, 0x0123)) << 32) |
                                      __byte_perm(hi, 0, 0x0123);
        out[q] = be;
    }
}

cudaError_t pack_fits_plane(const double* cube, int width, int height, int nb, int k, unsigned char* out_be,
                            cudaStream_t stream) {
    const size_t n = static_cast<size_t>(width) * height;
    if (n == 0) return cudaSuccess;
    const int threads = 256;
    int blocks = static_cast<int>((n + threads - 1) / threads);
    if (blocks > 148 * 16) blocks = 148 * 16;
    pack_fits_plane_kernel<<<blocks, threads, 0, stream>>>(cube, width, height, nb, k,
                                                           reinterpret_cast<unsigned long long*>(out_be));
    return cudaGetLastError();
}

}  // namespace grrt_b200
