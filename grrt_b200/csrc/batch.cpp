// The batched form: many thin-disk cameras (any mix of spins, inclinations,
// sizes) rendered by ONE persistent launch that pulls pixels from a device work
// queue, replayed as a captured CUDA graph. Each camera is a full GRRTContext
// (host tables built exactly as grrt_create builds them); their DevScene
// descriptions sit in one device array. An autotuner times candidate schedules
// (chunk size, chunk order across cameras, resident blocks per SM) and keeps
// the fastest, optionally caching the choice in a JSON file.
//
// In the mixed form the batch runs the mixed pipeline (FP32 speculation, star
// pass, FP64 re-trace, resolve) with each phase one launch over the samples
// of all cameras; the graph holds the four launches. Its phases take samples
// in camera order, so of the schedule only the resident blocks per SM apply.
//
// A batch of volumetric cameras renders spectra: one persistent launch of the
// warp-cooperative spectral kernel over the chunk table, each camera with its
// own frequency bins (grrt_batch_set_frequency_bins), its output cube at a
// prefix offset. The long rays that bound a single volumetric frame then
// overlap with the other cameras' work. The spectral batch runs the FP64 form
// in either precision setting (the volumetric mixed form's output is
// bit-identical to it).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "context.h"
#include "device/render_launch.h"

using namespace grrt_b200;

struct GRRTBatch {
    std::vector<std::unique_ptr<GRRTContext>> cams;
    std::vector<DevBatchItem> items;
    size_t total_pixels = 0;
    size_t total_samples = 0;  // mixed form's sample space (set with the device state)
    bool any_stars = false;
    bool spectral = false;     // volumetric cameras: spectral renders
    size_t total_spec = 0;     // spectral: output elements, sum of w * h * nb
    int nb_max = 0;
    double* d_freqs = nullptr;      // spectral: every camera's bins, back to back
    double* d_spec_scratch = nullptr;
    size_t spec_scratch_elems = 0;
    void* d_spec_out = nullptr;     // spectral output of the autotuner's runs
    int form = GRRT_FORM_FP64;
    // schedule
    int chunk_size = 256;
    int order = GRRT_BATCH_ORDER_ROUND_ROBIN;
    int blocks_per_sm = 0;  // 0 = as many as fit
    int block = 128;        // threads per block of the FP64 thin-disk batch kernel (64, 128, 256)
    bool tuned = false;
    // device
    int device = -1;
    DevScene* d_scenes = nullptr;
    DevBatchItem* d_items = nullptr;
    DevBatchChunk* d_chunks = nullptr;
    int n_chunks = 0;
    size_t chunks_cap = 0;
    unsigned* d_queue = nullptr;
    DevStats* d_stats = nullptr;
    float4* d_out = nullptr;  // output of the host-buffer entry point
    void* d_mixed = nullptr;  // mixed form's scratch
    size_t mixed_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    void* graph_out = nullptr;
    int graph_form = -1, graph_blocks = -1, graph_block = -1;
    bool graph_samples = false;
    bool schedule_dirty = true;
    std::string error;

    ~GRRTBatch() {
        if (device >= 0) cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(d_scenes);
        cudaFree(d_items);
        cudaFree(d_chunks);
        cudaFree(d_queue);
        cudaFree(d_stats);
        cudaFree(d_out);
        cudaFree(d_mixed);
        cudaFree(d_freqs);
        cudaFree(d_spec_scratch);
        cudaFree(d_spec_out);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    bool fail(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return false;
        error = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGetLastError();
        return true;
    }

    // Chunk table for the current schedule.
    std::vector<DevBatchChunk> make_chunks() const {
        std::vector<std::vector<DevBatchChunk>> per(items.size());
        for (size_t it = 0; it < items.size(); ++it) {
            const int n = items[it].w * items[it].h;
            for (int s = 0; s < n; s += chunk_size)
                per[it].push_back(DevBatchChunk{static_cast<int>(it), s, std::min(chunk_size, n - s)});
        }
        std::vector<DevBatchChunk> out;
        if (order != GRRT_BATCH_ORDER_ROUND_ROBIN) {
            for (auto& v : per) out.insert(out.end(), v.begin(), v.end());
        } else {
            size_t longest = 0;
            for (auto& v : per) longest = std::max(longest, v.size());
            for (size_t k = 0; k < longest; ++k)
                for (auto& v : per)
                    if (k < v.size()) out.push_back(v[k]);
        }
        return out;
    }

    bool upload_schedule() {
        if (!schedule_dirty) return true;
        const auto ch = make_chunks();
        if (ch.size() > chunks_cap) {
            cudaFree(d_chunks);
            d_chunks = nullptr;
            if (fail(cudaMalloc(&d_chunks, sizeof(DevBatchChunk) * ch.size()), "cudaMalloc(chunks)")) return false;
            chunks_cap = ch.size();
        }
        if (fail(cudaMemcpy(d_chunks, ch.data(), sizeof(DevBatchChunk) * ch.size(), cudaMemcpyHostToDevice),
                 "upload chunks"))
            return false;
        n_chunks = static_cast<int>(ch.size());
        schedule_dirty = false;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        return true;
    }

    DevBatch desc() const {
        DevBatch B;
        B.scenes = d_scenes;
        B.items = d_items;
        B.chunks = d_chunks;
        B.n_chunks = n_chunks;
        B.chunk_size = chunk_size;
        B.n_items = static_cast<int>(items.size());
        B.n_samples = static_cast<unsigned>(total_samples);
        B.n_pixels = total_pixels;
        return B;
    }

    // FP64 thin-disk batch traced by samples (GRRT_BATCH_ORDER_SAMPLES)
    bool by_samples() const { return !spectral && form != GRRT_FORM_MIXED && order == GRRT_BATCH_ORDER_SAMPLES; }

    int max_blocks_per_sm() const {
        if (spectral) return vol_spectral_batch_max_blocks_per_sm();
        if (by_samples()) return fp64_batch_max_blocks_per_sm();
        return form == GRRT_FORM_MIXED ? mixed_batch_max_blocks_per_sm() : thin_batch_max_blocks_per_sm(block);
    }

    // Re-uploads the cameras' scenes (they carry the mixed form's knobs).
    bool upload_scenes() {
        if (!d_scenes) return true;
        std::vector<DevScene> scenes;
        for (auto& c : cams) {
            c->form = form;
            scenes.push_back(c->scene_for_launch());
        }
        if (fail(cudaMemcpy(d_scenes, scenes.data(), sizeof(DevScene) * scenes.size(), cudaMemcpyHostToDevice),
                 "upload scenes"))
            return false;
        return true;
    }

    int blocks() const {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int maxb = max_blocks_per_sm();
        const int per = (blocks_per_sm > 0 && blocks_per_sm < maxb) ? blocks_per_sm : maxb;
        return sms * per;
    }

    // Enqueue one batched render (as a CUDA graph replay) on stream s: RGBA
    // (float4 per pixel) or, for a spectral batch, the cubes (doubles).
    int launch(void* out, cudaStream_t s) {
        if (!upload_schedule()) return -1;
        const int nb = blocks();
        const bool mixed = !spectral && form == GRRT_FORM_MIXED;
        const bool samples = by_samples();
        if (spectral) {
            const size_t need = static_cast<size_t>(4) * nb_max * nb * vol_spectral_batch_threads();
            if (need > spec_scratch_elems) {
                if (graph) cudaGraphExecDestroy(graph);
                graph = nullptr;
                cudaFree(d_spec_scratch);
                d_spec_scratch = nullptr;
                spec_scratch_elems = 0;
                if (fail(cudaMalloc(&d_spec_scratch, need * sizeof(double)), "cudaMalloc(spectral scratch)")) return -1;
                spec_scratch_elems = need;
            }
        }
        if (mixed || samples) {
            if (total_samples > 0x7f000000ull) {
                error = "the mixed form and the trace by samples index samples in 31 bits; this batch has " +
                        std::to_string(total_samples);
                return -1;
            }
            const size_t need = mixed_scratch_bytes_for(total_samples);
            if (need > mixed_bytes) {
                if (graph) cudaGraphExecDestroy(graph);
                graph = nullptr;
                cudaFree(d_mixed);
                d_mixed = nullptr;
                mixed_bytes = 0;
                if (fail(cudaMalloc(&d_mixed, need), "cudaMalloc(mixed scratch)")) return -1;
                mixed_bytes = need;
            }
        }
        if (!graph || graph_out != out || graph_form != form || graph_blocks != nb || graph_block != block ||
            graph_samples != samples) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            cudaGraph_t g = nullptr;
            if (fail(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
            cudaMemsetAsync(d_stats, 0, sizeof(DevStats), stream);
            const cudaError_t le =
                spectral ? launch_vol_spectral_batch(desc(), nb_max, static_cast<double*>(out), d_spec_scratch,
                                                     spec_scratch_elems, d_queue, d_stats, nb, stream)
                : mixed ? launch_thin_mixed_batch(desc(), any_stars, static_cast<float4*>(out), d_queue, d_stats,
                                                  d_mixed, mixed_bytes, blocks_per_sm, stream)
                : samples ? launch_thin_fp64_batch(desc(), static_cast<float4*>(out), d_queue, d_stats, d_mixed,
                                                   mixed_bytes, blocks_per_sm, stream)
                          : launch_thin_batch(desc(), static_cast<float4*>(out), d_queue, d_stats, nb, block, stream);
            const cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (fail(le, "batch launch") || fail(ce, "end capture")) {
                if (g) cudaGraphDestroy(g);
                return -1;
            }
            const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            if (fail(ie, "graph instantiate")) return -1;
            graph_out = out;
            graph_form = form;
            graph_blocks = nb;
            graph_block = block;
            graph_samples = samples;
        }
        cudaEventRecord(ev0, s);
        if (fail(cudaGraphLaunch(graph, s), "graph launch")) return -1;
        cudaEventRecord(ev1, s);
        return 0;
    }
};

namespace {
thread_local std::string g_batch_error;

std::string batch_key(const GRRTBatch& b) {
    std::ostringstream k;
    k << "form" << b.form << ";n" << b.cams.size() << (b.spectral ? ";spectral" : "");
    for (const auto& c : b.cams) {
        k << ";" << c->params.width << "x" << c->params.height << "s" << c->spp << "a" << c->spin_a << "t"
          << c->observer_theta;
        if (b.spectral) {
            k << "b" << c->freq_bins.size();
            for (double f : c->freq_bins) k << "," << f;
        }
    }
    std::hash<std::string> h;
    std::ostringstream out;
    out << std::hex << h(k.str());
    return out.str();
}
}  // namespace

extern "C" GRRT_EXPORT GRRTBatch* grrt_batch_create(const GRRTParams* params, int count) {
    if (!params || count <= 0) {
        g_batch_error = "grrt_batch_create: need at least one camera";
        return nullptr;
    }
    auto b = std::make_unique<GRRTBatch>();
    try {
        const bool vol0 = params[0].disk_enabled && params[0].disk_volumetric;
        b->spectral = vol0;
        for (int i = 0; i < count; ++i) {
            const bool vol = params[i].disk_enabled && params[i].disk_volumetric;
            if (vol != vol0) {
                g_batch_error = "grrt_batch_create: a batch holds either volumetric cameras (spectral renders) or "
                                "thin-disk cameras, not both (camera " + std::to_string(i) + " differs from camera 0)";
                return nullptr;
            }
            if (params[i].width <= 0 || params[i].height <= 0) {
                g_batch_error = "grrt_batch_create: camera " + std::to_string(i) + " has no pixels";
                return nullptr;
            }
            auto c = std::make_unique<GRRTContext>();
            c->build(params[i]);
            DevBatchItem it;
            it.scene = i;
            it.w = params[i].width;
            it.h = params[i].height;
            it.out_pitch = params[i].width;
            it.out_offset = b->total_pixels;
            b->total_pixels += static_cast<size_t>(it.w) * it.h;
            b->items.push_back(it);
            b->cams.push_back(std::move(c));
        }
    } catch (const std::exception& e) {
        g_batch_error = std::string("grrt_batch_create: ") + e.what();
        return nullptr;
    }
    return b.release();
}

extern "C" GRRT_EXPORT void grrt_batch_destroy(GRRTBatch* b) { delete b; }

extern "C" GRRT_EXPORT const char* grrt_batch_error(const GRRTBatch* b) {
    if (!b) return g_batch_error.empty() ? nullptr : g_batch_error.c_str();
    return b->error.empty() ? nullptr : b->error.c_str();
}

// Spectral batches: every camera's bins into one device array; each item gets
// its bins, bin count and output offset (the cubes back to back in camera
// order). The items are (re-)uploaded when the device state exists.
static bool batch_upload_bins(GRRTBatch* b) {
    size_t nf = 0;
    for (size_t i = 0; i < b->cams.size(); ++i) {
        if (b->cams[i]->freq_bins.empty()) {
            b->error = "camera " + std::to_string(i) + " has no frequency bins; call grrt_batch_set_frequency_bins";
            return false;
        }
        nf += b->cams[i]->freq_bins.size();
    }
    std::vector<double> all;
    all.reserve(nf);
    for (auto& c : b->cams) all.insert(all.end(), c->freq_bins.begin(), c->freq_bins.end());
    cudaFree(b->d_freqs);
    b->d_freqs = nullptr;
    if (b->fail(cudaMalloc(&b->d_freqs, sizeof(double) * nf), "cudaMalloc(bins)")) return false;
    if (b->fail(cudaMemcpy(b->d_freqs, all.data(), sizeof(double) * nf, cudaMemcpyHostToDevice), "upload bins"))
        return false;
    size_t f0 = 0, off = 0;
    int nb_max = 0;
    for (auto& it : b->items) {
        const auto& c = b->cams[static_cast<size_t>(it.scene)];
        it.freqs = b->d_freqs + f0;
        it.nb = static_cast<int>(c->freq_bins.size());
        it.spec_offset = off;
        f0 += c->freq_bins.size();
        off += static_cast<size_t>(it.w) * it.h * it.nb;
        nb_max = std::max(nb_max, it.nb);
    }
    b->total_spec = off;
    if (nb_max != b->nb_max) {
        b->nb_max = nb_max;
        cudaFree(b->d_spec_scratch);
        b->d_spec_scratch = nullptr;
        b->spec_scratch_elems = 0;
    }
    if (b->d_items &&
        b->fail(cudaMemcpy(b->d_items, b->items.data(), sizeof(DevBatchItem) * b->items.size(),
                           cudaMemcpyHostToDevice),
                "upload items"))
        return false;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaFree(b->d_spec_out);
    b->d_spec_out = nullptr;
    return true;
}

static bool batch_ensure_device(GRRTBatch* b) {
    if (b->d_scenes) {
        cudaSetDevice(b->device);
        return true;
    }
    std::vector<DevScene> scenes;
    for (auto& c : b->cams) {
        if (!c->ensure_device()) {
            b->error = c->error;
            return false;
        }
        c->form = b->form;
        scenes.push_back(c->scene_for_launch());
    }
    b->device = b->cams[0]->device;
    // the mixed form's sample space: each item's samples (pixel-major, grid^2
    // per pixel) after those of the items before it
    size_t s0 = 0;
    for (auto& it : b->items) {
        const DevScene& sc = scenes[static_cast<size_t>(it.scene)];
        it.sample0 = s0;
        s0 += static_cast<size_t>(it.w) * it.h * static_cast<size_t>(sc.grid) * static_cast<size_t>(sc.grid);
        b->any_stars = b->any_stars || sc.stars_on != 0;
    }
    b->total_samples = s0;
    if (b->spectral && !batch_upload_bins(b)) return false;
    if (b->fail(cudaMalloc(&b->d_scenes, sizeof(DevScene) * scenes.size()), "cudaMalloc(scenes)")) return false;
    if (b->fail(cudaMemcpy(b->d_scenes, scenes.data(), sizeof(DevScene) * scenes.size(), cudaMemcpyHostToDevice),
                "upload scenes"))
        return false;
    if (b->fail(cudaMalloc(&b->d_items, sizeof(DevBatchItem) * b->items.size()), "cudaMalloc(items)")) return false;
    if (b->fail(cudaMemcpy(b->d_items, b->items.data(), sizeof(DevBatchItem) * b->items.size(),
                           cudaMemcpyHostToDevice),
                "upload items"))
        return false;
    if (b->fail(cudaMalloc(&b->d_queue, 256), "cudaMalloc(queue)")) return false;
    if (b->fail(cudaMalloc(&b->d_stats, sizeof(DevStats)), "cudaMalloc(stats)")) return false;
    if (b->fail(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream")) return false;
    if (b->fail(cudaEventCreate(&b->ev0), "event") || b->fail(cudaEventCreate(&b->ev1), "event")) return false;
    return true;
}

extern "C" GRRT_EXPORT int grrt_batch_set_precision(GRRTBatch* b, int form) {
    if (!b || (form != GRRT_FORM_FP64 && form != GRRT_FORM_MIXED)) return -1;
    if (form == b->form) return 0;

    b->form = form;
    // scenes carry the form's knobs; re-upload
    return b->upload_scenes() ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_batch_set_tuning(GRRTBatch* b, int block, double tol_fp32, double r_factor) {
    if (!b || (block != 64 && block != 128 && block != 256) || !(tol_fp32 >= 1e-9 && tol_fp32 <= 1e-2) ||
        !(r_factor >= 1.0 && r_factor <= 100.0)) {
        if (b) b->error = "grrt_batch_set_tuning: block must be 64, 128 or 256, tol_fp32 in [1e-9, 1e-2], "
                          "r_factor in [1, 100]";
        return -1;
    }
    b->block = block;
    for (auto& c : b->cams) {
        c->tol_fp32 = tol_fp32;
        c->mixed_r_factor = r_factor;
    }
    if (b->d_scenes) cudaSetDevice(b->device);
    return b->upload_scenes() ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_batch_get_tuning(const GRRTBatch* b, int* block, double* tol_fp32, double* r_factor) {
    if (!b) return -1;
    if (block) *block = b->block;
    if (tol_fp32) *tol_fp32 = b->cams[0]->tol_fp32;
    if (r_factor) *r_factor = b->cams[0]->mixed_r_factor;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_set_schedule(GRRTBatch* b, int chunk_size, int order, int blocks_per_sm) {
    if (!b || chunk_size < 1 ||
        (order != GRRT_BATCH_ORDER_CAMERA_MAJOR && order != GRRT_BATCH_ORDER_ROUND_ROBIN &&
         order != GRRT_BATCH_ORDER_SAMPLES) ||
        blocks_per_sm < 0) {
        if (b) b->error = "grrt_batch_set_schedule: bad schedule";
        return -1;
    }
    b->chunk_size = chunk_size;
    b->order = order;
    b->blocks_per_sm = blocks_per_sm;
    b->schedule_dirty = true;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_get_schedule(const GRRTBatch* b, int* chunk_size, int* order,
                                                   int* blocks_per_sm) {
    if (!b) return -1;
    if (chunk_size) *chunk_size = b->chunk_size;
    if (order) *order = b->order;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_render_device(GRRTBatch* b, float* d_rgba, void* stream) {
    if (!b || !d_rgba) return -1;
    if (b->spectral) {
        b->error = "grrt_batch_render_device: this batch holds volumetric cameras; use grrt_batch_render_spectral*";
        return -1;
    }
    if (!batch_ensure_device(b)) return -1;
    return b->launch(d_rgba, static_cast<cudaStream_t>(stream));
}

extern "C" GRRT_EXPORT int grrt_batch_set_frequency_bins(GRRTBatch* b, int camera, const double* freqs, int n) {
    if (!b) return -1;
    if (!b->spectral) {
        b->error = "grrt_batch_set_frequency_bins: the batch holds thin-disk cameras (no spectra)";
        return -1;
    }
    if (!freqs || n < 1 || camera < -1 || camera >= static_cast<int>(b->cams.size())) {
        b->error = "grrt_batch_set_frequency_bins: bad camera or bins";
        return -1;
    }
    for (size_t i = 0; i < b->cams.size(); ++i)
        if (camera < 0 || static_cast<int>(i) == camera) b->cams[i]->freq_bins.assign(freqs, freqs + n);
    if (b->d_scenes) {
        cudaSetDevice(b->device);
        for (auto& c : b->cams)
            if (c->freq_bins.empty()) return 0;  // uploaded once every camera has bins
        if (!batch_upload_bins(b)) return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT long long grrt_batch_spectral_offset(GRRTBatch* b, int camera) {
    if (!b || !b->spectral || camera < 0 || camera > static_cast<int>(b->cams.size())) return -1;
    long long off = 0;
    for (int i = 0; i < camera; ++i) {
        const auto& it = b->items[static_cast<size_t>(i)];
        off += static_cast<long long>(it.w) * it.h * static_cast<long long>(b->cams[static_cast<size_t>(i)]->freq_bins.size());
    }
    return off;
}

extern "C" GRRT_EXPORT int grrt_batch_render_spectral_device(GRRTBatch* b, double* d_spec, void* stream) {
    if (!b || !d_spec) return -1;
    if (!b->spectral) {
        b->error = "grrt_batch_render_spectral_device: the batch holds thin-disk cameras (no spectra)";
        return -1;
    }
    if (!batch_ensure_device(b)) return -1;
    return b->launch(d_spec, static_cast<cudaStream_t>(stream));
}

extern "C" GRRT_EXPORT int grrt_batch_render_spectral(GRRTBatch* b, double* const* cubes) {
    if (!b || !cubes) return -1;
    if (!b->spectral) {
        b->error = "grrt_batch_render_spectral: the batch holds thin-disk cameras (no spectra)";
        return -1;
    }
    if (!batch_ensure_device(b)) return -1;
    if (!b->d_spec_out && b->fail(cudaMalloc(&b->d_spec_out, sizeof(double) * b->total_spec), "cudaMalloc(output)"))
        return -1;
    if (b->launch(b->d_spec_out, b->stream) != 0) return -1;
    if (b->fail(cudaStreamSynchronize(b->stream), "batch render")) return -1;
    const double* d = static_cast<const double*>(b->d_spec_out);
    for (size_t i = 0; i < b->items.size(); ++i) {
        const auto& it = b->items[i];
        if (!cubes[i]) continue;
        if (b->fail(cudaMemcpy(cubes[i], d + it.spec_offset, sizeof(double) * it.w * it.h * it.nb,
                               cudaMemcpyDeviceToHost),
                    "copy result"))
            return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_render(GRRTBatch* b, float* const* framebuffers) {
    if (!b || !framebuffers) return -1;
    if (b->spectral) {
        b->error = "grrt_batch_render: this batch holds volumetric cameras; use grrt_batch_render_spectral*";
        return -1;
    }
    if (!batch_ensure_device(b)) return -1;
    if (!b->d_out && b->fail(cudaMalloc(&b->d_out, sizeof(float4) * b->total_pixels), "cudaMalloc(output)")) return -1;
    if (b->launch(b->d_out, b->stream) != 0) return -1;
    if (b->fail(cudaStreamSynchronize(b->stream), "batch render")) return -1;
    for (size_t i = 0; i < b->items.size(); ++i) {
        const auto& it = b->items[i];
        if (!framebuffers[i]) continue;
        if (b->fail(cudaMemcpy(framebuffers[i], b->d_out + it.out_offset, sizeof(float4) * it.w * it.h,
                               cudaMemcpyDeviceToHost),
                    "copy result"))
            return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_get_stats(GRRTBatch* b, GRRTStats* out) {
    if (!b || !out) return -1;
    std::memset(out, 0, sizeof(*out));
    if (!b->d_stats) return 0;
    cudaSetDevice(b->device);
    if (b->fail(cudaDeviceSynchronize(), "synchronize")) return -1;
    DevStats s{};
    if (b->fail(cudaMemcpy(&s, b->d_stats, sizeof(s), cudaMemcpyDeviceToHost), "read stats")) return -1;
    out->attempts = s.attempts;
    out->accepted = s.accepted;
    out->crossings = s.crossings;
    out->rays = s.rays;
    out->horizon = s.horizon;
    out->escaped = s.escaped;
    out->max_steps = s.max_steps;
    out->fp64_attempts = s.fp64_attempts;
    out->clamp_evals = s.clamp_evals;
    out->march_steps = s.march_steps;
    out->physics_steps = s.physics_steps;
    out->bin_updates = s.bin_updates;
    std::memcpy(&out->hamiltonian_max, &s.h_max_bits, sizeof(double));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) out->kernel_ms = ms;
    cudaGetLastError();
    return 0;
}

// Times candidate schedules on the batch itself and keeps the fastest.
//   FP64 thin-disk batches: chunk size (64..4096) x chunk order x resident
//     blocks per SM at 128 threads per block, then threads per block (64,
//     128, 256) x resident blocks per SM at the best chunk and order; and the
//     trace by samples (GRRT_BATCH_ORDER_SAMPLES) x resident blocks per SM.
//   Spectral batches: chunk size x chunk order x resident blocks per SM.
//   Mixed batches (the phases take samples in camera order, so the chunk
//     table does not apply): resident blocks per SM x the FP32 tolerance
//     (1e-6, 3e-6, 1e-5) x r_factor (3, 4). Each candidate is held to the
//     mixed form's bar against the batch's FP64 render: every pixel within
//     1e-4 relative (floor 1e-6 x the camera's maximum). Candidates that miss
//     it are not taken.
// With a cache path, a choice stored for an identical batch (same cameras,
// sizes, spins, inclinations, bins and form) is reused without timing, and a
// new choice is appended. Returns 0 and writes the chosen time (ms) to *best_ms.
namespace {
struct Tuning {
    int chunk, order, bps, block;
    double tol_fp32, r_factor;
};

void apply(GRRTBatch* b, const Tuning& t) {
    grrt_batch_set_schedule(b, t.chunk, t.order, t.bps);
    grrt_batch_set_tuning(b, t.block, t.tol_fp32, t.r_factor);
}

// best of two timed runs; < 0 on error
double time_batch(GRRTBatch* b, void* out) {
    double t = 1e30;
    for (int rep = 0; rep < 2; ++rep) {
        if (b->launch(out, b->stream) != 0) return -1.0;
        if (b->fail(cudaStreamSynchronize(b->stream), "autotune run")) return -1.0;
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        t = std::min(t, static_cast<double>(ms));
    }
    return t;
}

// largest relative difference of the RGB channels against ref, floor 1e-6 x
// each camera's maximum
double max_rel_rgb(const GRRTBatch* b, const std::vector<float>& got, const std::vector<float>& ref) {
    double worst = 0.0;
    for (const auto& it : b->items) {
        const size_t p0 = it.out_offset, n = static_cast<size_t>(it.w) * it.h;
        double scale = 0.0;
        for (size_t p = p0; p < p0 + n; ++p)
            for (int c = 0; c < 3; ++c) scale = std::max(scale, static_cast<double>(ref[4 * p + c]));
        for (size_t p = p0; p < p0 + n; ++p)
            for (int c = 0; c < 3; ++c) {
                const double r = ref[4 * p + c], g = got[4 * p + c];
                const double d = std::fabs(g - r) / std::max(std::fabs(r), 1e-6 * scale);
                if (!(d <= worst)) worst = std::isnan(d) ? 1e30 : d;
            }
    }
    return worst;
}
}  // namespace

extern "C" GRRT_EXPORT int grrt_batch_autotune(GRRTBatch* b, const char* cache_path, double* best_ms) {
    if (!b) return -1;
    if (!batch_ensure_device(b)) return -1;
    const std::string key = batch_key(*b);
    if (cache_path && cache_path[0]) {
        std::ifstream in(cache_path);
        std::string line;
        while (std::getline(in, line)) {
            Tuning t{256, GRRT_BATCH_ORDER_ROUND_ROBIN, 0, 128, 3e-6, 3.0};
            double ms = 0;
            char kbuf[64] = {0};
            const int got = std::sscanf(line.c_str(),
                                        " {\"key\": \"%63[^\"]\", \"chunk\": %d, \"order\": %d, \"blocks_per_sm\": %d, "
                                        "\"ms\": %lf, \"block\": %d, \"tol_fp32\": %lf, \"r_factor\": %lf",
                                        kbuf, &t.chunk, &t.order, &t.bps, &ms, &t.block, &t.tol_fp32, &t.r_factor);
            if (got == 8 && key == kbuf) {
                apply(b, t);
                b->tuned = true;
                if (best_ms) *best_ms = ms;
                return 0;
            }
        }
    }
    void* tune_out = nullptr;
    if (b->spectral) {
        if (!b->d_spec_out &&
            b->fail(cudaMalloc(&b->d_spec_out, sizeof(double) * b->total_spec), "cudaMalloc(output)"))
            return -1;
        tune_out = b->d_spec_out;
    } else {
        if (!b->d_out && b->fail(cudaMalloc(&b->d_out, sizeof(float4) * b->total_pixels), "cudaMalloc(output)"))
            return -1;
        tune_out = b->d_out;
    }
    const bool mixed = !b->spectral && b->form == GRRT_FORM_MIXED;
    Tuning cur{b->chunk_size, b->order, b->blocks_per_sm, b->block, b->cams[0]->tol_fp32, b->cams[0]->mixed_r_factor};
    Tuning best_t = cur;
    double best = 1e30;
    auto consider = [&](const Tuning& t) -> int {
        apply(b, t);
        const double ms = time_batch(b, tune_out);
        if (ms < 0.0) return -1;
        if (ms < best) {
            best = ms;
            best_t = t;
        }
        return 0;
    };
    if (mixed) {
        // the FP64 render the candidates are held to
        std::vector<float> ref(4 * b->total_pixels), got(4 * b->total_pixels);
        b->form = GRRT_FORM_FP64;
        Tuning f64 = cur;
        f64.block = 128;
        apply(b, f64);
        if (b->launch(tune_out, b->stream) != 0 || b->fail(cudaStreamSynchronize(b->stream), "autotune reference") ||
            b->fail(cudaMemcpy(ref.data(), tune_out, sizeof(float4) * b->total_pixels, cudaMemcpyDeviceToHost),
                    "autotune reference")) {
            b->form = GRRT_FORM_MIXED;
            b->upload_scenes();
            return -1;
        }
        b->form = GRRT_FORM_MIXED;
        const int maxb = b->max_blocks_per_sm();
        for (int bp : {maxb, std::max(1, maxb - 1)})
            for (double tol : {1e-6, 3e-6, 1e-5})
                for (double rf : {3.0, 4.0}) {
                    Tuning t = cur;
                    t.bps = bp;
                    t.tol_fp32 = tol;
                    t.r_factor = rf;
                    apply(b, t);
                    const double ms = time_batch(b, tune_out);
                    if (ms < 0.0) return -1;
                    if (b->fail(cudaMemcpy(got.data(), tune_out, sizeof(float4) * b->total_pixels,
                                           cudaMemcpyDeviceToHost),
                                "autotune check"))
                        return -1;
                    if (max_rel_rgb(b, got, ref) > 1e-4) continue;  // misses the bar
                    if (ms < best) {
                        best = ms;
                        best_t = t;
                    }
                }
        if (best >= 1e30) {
            // no candidate met the bar (none is expected to miss it): keep the defaults
            best_t = cur;
            best_t.tol_fp32 = 3e-6;
            best_t.r_factor = 3.0;
        }
    } else {
        const std::vector<int> orders{GRRT_BATCH_ORDER_ROUND_ROBIN, GRRT_BATCH_ORDER_CAMERA_MAJOR};
        b->block = 128;
        const int maxb = b->max_blocks_per_sm();
        for (int order : orders)
            for (int cs : {64, 256, 1024, 4096})
                for (int bp : {maxb, std::max(1, maxb - 1)}) {
                    Tuning t = cur;
                    t.chunk = cs;
                    t.order = order;
                    t.bps = bp;
                    t.block = 128;
                    if (consider(t) != 0) return -1;
                }
        if (!b->spectral) {
            const Tuning base = best_t;
            for (int blk : {64, 256}) {
                b->block = blk;
                b->order = base.order;
                const int mb = b->max_blocks_per_sm();
                for (int bp : {mb, std::max(1, mb - 1)}) {
                    Tuning t = base;
                    t.block = blk;
                    t.bps = bp;
                    if (consider(t) != 0) return -1;
                }
            }
            // the trace by samples (its own kernel: 128 threads, no chunks)
            b->block = 128;
            b->order = GRRT_BATCH_ORDER_SAMPLES;
            const int mbs = b->max_blocks_per_sm();
            for (int bp : {mbs, std::max(1, mbs - 1)}) {
                Tuning t = base;
                t.order = GRRT_BATCH_ORDER_SAMPLES;
                t.block = 128;
                t.bps = bp;
                if (consider(t) != 0) return -1;
            }
        }
    }
    apply(b, best_t);
    b->tuned = true;
    if (best_ms) *best_ms = best;
    if (cache_path && cache_path[0]) {
        std::ofstream out(cache_path, std::ios::app);
        out.precision(17);
        out << "{\"key\": \"" << key << "\", \"chunk\": " << best_t.chunk << ", \"order\": " << best_t.order
            << ", \"blocks_per_sm\": " << best_t.bps << ", \"ms\": " << best << ", \"block\": " << best_t.block
            << ", \"tol_fp32\": " << best_t.tol_fp32 << ", \"r_factor\": " << best_t.r_factor << "}\n";
    }
    return 0;
}
