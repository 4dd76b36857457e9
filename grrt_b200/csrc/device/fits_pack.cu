// Device-side FITS packing: planes [k0, k1) of a [pixel][bin] double cube to
// big-endian doubles in FITS order (the byte swap and row flip of
// FITSStreamWriter::write_row, src/fits_writer.cpp:356-395, done on the GPU so
// the host only streams bytes to the file).
//
// A tiled transpose: each block takes 32 consecutive pixels x 32 bins of the
// cube through shared memory, so both the cube reads (consecutive bins of a
// pixel) and the plane writes (consecutive pixels of a FITS row) are
// coalesced. HBM-bound: 8 bytes read and 8 written per value.
#include <cuda_runtime.h>

#include <algorithm>

#include "../fits.h"

namespace grrt_b200 {

namespace {

constexpr int kTile = 32;   // pixels and bins per tile
constexpr int kRows = 8;    // warps per block; each walks kTile / kRows tile rows

__device__ __forceinline__ unsigned long long to_big_endian(double v) {
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(v));
    const unsigned lo = static_cast<unsigned>(bits), hi = static_cast<unsigned>(bits >> 32);
    return (static_cast<unsigned long long>(__byte_perm(lo, 0, 0x0123)) << 32) | __byte_perm(hi, 0, 0x0123);
}

// grid.x: pixel tiles (grid-stride), grid.y: bin tiles of [k0, k1)
__global__ void __launch_bounds__(kTile * kRows) pack_fits_planes_kernel(
    const double* __restrict__ cube, int width, int height, int nb, int k0, int k1,
    unsigned long long* __restrict__ out) {
    __shared__ unsigned long long tile[kTile][kTile + 1];
    const long long npix = static_cast<long long>(width) * height;
    const long long ntiles = (npix + kTile - 1) / kTile;
    const int kb = k0 + static_cast<int>(blockIdx.y) * kTile;
    const int lane = threadIdx.x, row = threadIdx.y;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long p0 = t * kTile;
        // load: warp row r reads pixel p0 + r's bins kb..kb+31 (contiguous)
        for (int r = row; r < kTile; r += kRows) {
            const long long p = p0 + r;
            const int k = kb + lane;
            if (p < npix && k < k1) tile[r][lane] = to_big_endian(cube[p * nb + k]);
        }
        __syncthreads();
        // store: warp row r writes bin kb + r of pixels p0..p0+31; pixel p
        // (image row j, column i) goes to FITS row height-1-j of its plane
        for (int r = row; r < kTile; r += kRows) {
            const int k = kb + r;
            const long long p = p0 + lane;
            if (p < npix && k < k1) {
                const long long j = p / width, i = p - j * width;
                out[static_cast<long long>(k - k0) * npix + (height - 1 - j) * width + i] = tile[lane][r];
            }
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t pack_fits_planes(const double* cube, int width, int height, int nb, int k0, int k1,
                             unsigned char* out_be, cudaStream_t stream) {
    const long long npix = static_cast<long long>(width) * height;
    if (npix <= 0 || k1 <= k0) return cudaSuccess;
    const long long ntiles = (npix + kTile - 1) / kTile;
    const int bin_tiles = (k1 - k0 + kTile - 1) / kTile;
    // about 8 resident 256-thread blocks per SM over the 148 SMs
    const long long want = (148LL * 8 + bin_tiles - 1) / bin_tiles;
    const unsigned gx = static_cast<unsigned>(std::max(1LL, std::min(ntiles, want)));
    pack_fits_planes_kernel<<<dim3(gx, static_cast<unsigned>(bin_tiles)), dim3(kTile, kRows), 0, stream>>>(
        cube, width, height, nb, k0, k1, reinterpret_cast<unsigned long long*>(out_be));
    return cudaGetLastError();
}

}  // namespace grrt_b200
