// FITS spectral-cube output (BITPIX -64, big-endian, NAXIS1 = width,
// NAXIS2 = height, NAXIS3 = bins, image rows flipped so FITS row 1 is the
// bottom). Header cards and data layout follow src/fits_writer.cpp:148-406 so
// the files are byte-identical to the reference's.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

namespace grrt_b200 {

struct FitsMetadata {
    double spin = 0.0, mass = 1.0, observer_r = 50.0, observer_theta = 1.396, fov = 1.047;
    int samples_per_pixel = 1;
};

// All header cards up to and including END, each exactly 80 characters.
std::vector<std::string> fits_header_cards(int width, int height, int num_bins,
                                           const std::vector<double>& freqs, const FitsMetadata& meta);

// Writes the header on construction, then whole frequency planes in order
// (the data section is contiguous: plane k starts k * width * height * 8
// bytes after the header).
class FitsCubeWriter {
public:
    FitsCubeWriter(const std::string& path, int width, int height, int num_bins,
                   const std::vector<double>& freqs, const FitsMetadata& meta);
    ~FitsCubeWriter();
    FitsCubeWriter(const FitsCubeWriter&) = delete;
    FitsCubeWriter& operator=(const FitsCubeWriter&) = delete;
    // planes_be: planes [k0, k1), each width*height big-endian doubles in
    // FITS row order, back to back; k0 must be the next unwritten plane.
    void write_planes(int k0, int k1, const void* planes_be);
    void finalize();

private:
    std::FILE* f_ = nullptr;
    std::string path_;
    int width_, height_, bins_;
    int next_plane_ = 0;
};

// Device: converts planes [k0, k1) of a [pixel][bin] double cube into
// big-endian doubles in FITS order (row j of the image becomes FITS row
// height-1-j), plane after plane into out_be.
cudaError_t pack_fits_planes(const double* cube, int width, int height, int num_bins, int k0, int k1,
                             unsigned char* out_be, cudaStream_t stream);

}  // namespace grrt_b200
