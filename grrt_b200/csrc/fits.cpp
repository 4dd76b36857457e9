// FITS header cards and the plane writer (format of src/fits_writer.cpp).
#include "fits.h"

#include <cmath>
#include <cstring>
#include <stdexcept>

namespace grrt_b200 {
namespace {

constexpr int kCard = 80;
constexpr int kBlock = 2880;

std::string fit_width(std::string s, size_t n) {
    if (s.size() >= n) return s.substr(0, n);
    s.append(n - s.size(), ' ');
    return s;
}

// keyword in columns 1-8, "= " in 9-10, value right-justified in 11-30,
// optional " / comment", padded or cut to 80 characters.
std::string card(const std::string& key, const std::string& value, const std::string& comment = "") {
    std::string v = value;
    if (v.size() < 20) v = std::string(20 - v.size(), ' ') + v;
    std::string c = fit_width(key, 8) + "= " + v;
    if (!comment.empty()) c += " / " + comment;
    return fit_width(c, kCard);
}

std::string card_int(const std::string& key, long long v, const std::string& comment) {
    return card(key, std::to_string(v), comment);
}

std::string card_real(const std::string& key, double v, const std::string& comment) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.12E", v);
    return card(key, buf, comment);
}

std::string card_text(const std::string& key, const std::string& v, const std::string& comment) {
    std::string inner = v;
    if (inner.size() < 8) inner.append(8 - inner.size(), ' ');
    if (inner.size() > 18) inner = inner.substr(0, 18);
    return card(key, "'" + inner + "'", comment);
}

bool uniform_linear(const std::vector<double>& f) {
    if (f.size() < 2) return true;
    const double step = f[1] - f[0];
    if (step == 0.0) return false;
    for (size_t i = 2; i < f.size(); ++i)
        if (std::abs(((f[i] - f[i - 1]) - step) / step) > 1e-4) return false;
    return true;
}

bool uniform_log(const std::vector<double>& f) {
    if (f.size() < 2) return true;
    if (f[0] <= 0.0 || f[1] <= 0.0) return false;
    const double step = std::log10(f[1]) - std::log10(f[0]);
    if (step == 0.0) return false;
    for (size_t i = 2; i < f.size(); ++i) {
        if (f[i] <= 0.0) return false;
        if (std::abs(((std::log10(f[i]) - std::log10(f[i - 1])) - step) / step) > 1e-4) return false;
    }
    return true;
}

std::string bin_key(int k) {
    char buf[16];
    std::snprintf(buf, sizeof buf, "FREQ%04d", k + 1);
    return buf;
}

std::string bin_comment(int k) { return "freq bin " + std::to_string(k + 1) + " (Hz)"; }

}  // namespace

std::vector<std::string> fits_header_cards(int width, int height, int num_bins, const std::vector<double>& f,
                                           const FitsMetadata& m) {
    std::vector<std::string> c;
    c.push_back(card("SIMPLE", "T", "conforms to FITS standard"));
    c.push_back(card_int("BITPIX", -64, "IEEE 754 double precision"));
    c.push_back(card_int("NAXIS", 3, "number of array dimensions"));
    c.push_back(card_int("NAXIS1", width, "pixels along RA axis"));
    c.push_back(card_int("NAXIS2", height, "pixels along Dec axis"));
    c.push_back(card_int("NAXIS3", num_bins, "number of frequency bins"));
    c.push_back(card_text("BUNIT", "erg/s/cm2/Hz/sr", "specific intensity"));
    if (!f.empty()) {
        const int nk = std::min<int>(num_bins, static_cast<int>(f.size()));
        if (uniform_linear(f) && f.size() >= 2) {
            c.push_back(card_text("CTYPE3", "FREQ", "frequency"));
            c.push_back(card_text("CUNIT3", "Hz", "frequency unit"));
            c.push_back(card_real("CRPIX3", 1.0, "reference pixel"));
            c.push_back(card_real("CRVAL3", f.front(), "frequency at ref pixel (Hz)"));
            c.push_back(card_real("CDELT3", f[1] - f[0], "frequency step (Hz)"));
        } else if (uniform_log(f) && f.size() >= 2) {
            c.push_back(card_text("CTYPE3", "FREQ-LOG", "log10(frequency/Hz)"));
            c.push_back(card_text("CUNIT3", "log(Hz)", "log10 of frequency in Hz"));
            c.push_back(card_real("CRPIX3", 1.0, "reference pixel"));
            c.push_back(card_real("CRVAL3", std::log10(f.front()), "log10(freq) at ref pixel"));
            c.push_back(card_real("CDELT3", std::log10(f[1]) - std::log10(f[0]), "log10(freq) step per pixel"));
            for (int k = 0; k < nk; ++k) c.push_back(card_real(bin_key(k), f[k], bin_comment(k)));
        } else {
            c.push_back(card_text("CTYPE3", "FREQ-TAB", "frequency (see FREQnnnn keys)"));
            c.push_back(card_text("CUNIT3", "Hz", "frequency unit"));
            c.push_back(card_real("CRPIX3", 1.0, "reference pixel"));
            c.push_back(card_real("CRVAL3", 1.0, "slice index"));
            c.push_back(card_real("CDELT3", 1.0, "slice index step"));
            for (int k = 0; k < nk; ++k) c.push_back(card_real(bin_key(k), f[k], bin_comment(k)));
        }
    }
    c.push_back(card_real("SPIN", m.spin, "Kerr spin parameter a/M"));
    c.push_back(card_real("MASS", m.mass, "black hole mass (geometrized units)"));
    c.push_back(card_real("OBS_R", m.observer_r, "observer radial coordinate (M)"));
    c.push_back(card_real("OBS_TH", m.observer_theta, "observer polar angle (rad)"));
    c.push_back(card_real("FOV", m.fov, "camera field of view (rad)"));
    c.push_back(card_int("SPP", m.samples_per_pixel, "samples per pixel (anti-aliasing)"));
    c.push_back(card_text("ORIGIN", "grrt", "GR ray tracer (github: gr_ray_tracer)"));
    c.push_back(fit_width("END", kCard));
    return c;
}

FitsCubeWriter::FitsCubeWriter(const std::string& path, int width, int height, int num_bins,
                               const std::vector<double>& freqs, const FitsMetadata& meta)
    : path_(path), width_(width), height_(height), bins_(num_bins) {
    f_ = std::fopen(path.c_str(), "wb");
    if (!f_) throw std::runtime_error("grrt: cannot open '" + path + "' for writing");
    const auto cards = fits_header_cards(width, height, num_bins, freqs, meta);
    const size_t per_block = kBlock / kCard;
    const size_t total = (cards.size() + per_block - 1) / per_block * per_block;
    for (const auto& c : cards) std::fwrite(c.data(), 1, kCard, f_);
    const std::string blank(kCard, ' ');
    for (size_t i = cards.size(); i < total; ++i) std::fwrite(blank.data(), 1, kCard, f_);
    if (std::ferror(f_)) throw std::runtime_error("grrt: write error on '" + path + "'");
}

FitsCubeWriter::~FitsCubeWriter() {
    if (f_) std::fclose(f_);
}

void FitsCubeWriter::write_planes(int k0, int k1, const void* planes_be) {
    if (k0 != next_plane_ || k1 < k0 || k1 > bins_) throw std::runtime_error("grrt: FITS planes must be written in order");
    const size_t n = static_cast<size_t>(width_) * height_ * 8 * static_cast<size_t>(k1 - k0);
    if (std::fwrite(planes_be, 1, n, f_) != n) throw std::runtime_error("grrt: write error on '" + path_ + "'");
    next_plane_ = k1;
}

void FitsCubeWriter::finalize() {
    if (next_plane_ != bins_) throw std::runtime_error("grrt: FITS cube incomplete");
    const size_t data = static_cast<size_t>(width_) * height_ * bins_ * 8;
    const size_t rem = data % kBlock;
    if (rem) {
        const std::vector<char> zeros(kBlock - rem, 0);
        std::fwrite(zeros.data(), 1, zeros.size(), f_);
    }
    const bool bad = std::fflush(f_) != 0 || std::ferror(f_);
    std::fclose(f_);
    f_ = nullptr;
    if (bad) throw std::runtime_error("grrt: write error during finalize");
}

}  // namespace grrt_b200
