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
    int form = GRRT_FORM_FP64;
    // schedule
    int chunk_size = 256;
    int order = GRRT_BATCH_ORDER_ROUND_ROBIN;
    int blocks_per_sm = 0;  // 0 = as many as fit
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
    float4* graph_out = nullptr;
    int graph_form = -1, graph_blocks = -1;
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
        if (order == GRRT_BATCH_ORDER_CAMERA_MAJOR) {
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

    static int max_blocks_per_sm(int f) {
        return f == GRRT_FORM_MIXED ? mixed_batch_max_blocks_per_sm() : thin_batch_max_blocks_per_sm();
    }

    int blocks() const {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int maxb = max_blocks_per_sm(form);
        const int per = (blocks_per_sm > 0 && blocks_per_sm < maxb) ? blocks_per_sm : maxb;
        return sms * per;
    }

    // Enqueue one batched render (as a CUDA graph replay) on stream s.
    int launch(float4* out, cudaStream_t s) {
        if (!upload_schedule()) return -1;
        const int nb = blocks();
        const bool mixed = form == GRRT_FORM_MIXED;
        if (mixed) {
            if (total_samples > 0xffffffffull) {
                error = "the mixed form indexes samples in 32 bits; this batch has " + std::to_string(total_samples);
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
        if (!graph || graph_out != out || graph_form != form || graph_blocks != nb) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            cudaGraph_t g = nullptr;
            if (fail(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
            cudaMemsetAsync(d_stats, 0, sizeof(DevStats), stream);
            const cudaError_t le =
                mixed ? launch_thin_mixed_batch(desc(), any_stars, out, d_queue, d_stats, d_mixed, mixed_bytes,
                                                blocks_per_sm, stream)
                      : launch_thin_batch(desc(), out, d_queue, d_stats, nb, stream);
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
    k << "form" << b.form << ";n" << b.cams.size();
    for (const auto& c : b.cams)
        k << ";" << c->params.width << "x" << c->params.height << "s" << c->spp << "a" << c->spin_a << "t"
          << c->observer_theta;
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
        for (int i = 0; i < count; ++i) {
            if (params[i].disk_enabled && params[i].disk_volumetric) {
                g_batch_error = "grrt_batch_create: the batched form renders thin-disk scenes (camera " +
                                std::to_string(i) + " is volumetric)";
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
    if (b->d_scenes) {
        // scenes carry the form's knobs; re-upload
        std::vector<DevScene> scenes;
        for (auto& c : b->cams) {
            c->form = form;
            scenes.push_back(c->scene_for_launch());
        }
        if (b->fail(cudaMemcpy(b->d_scenes, scenes.data(), sizeof(DevScene) * scenes.size(), cudaMemcpyHostToDevice),
                    "upload scenes"))
            return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT int grrt_batch_set_schedule(GRRTBatch* b, int chunk_size, int order, int blocks_per_sm) {
    if (!b || chunk_size < 1 || (order != GRRT_BATCH_ORDER_CAMERA_MAJOR && order != GRRT_BATCH_ORDER_ROUND_ROBIN) ||
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
    if (!batch_ensure_device(b)) return -1;
    return b->launch(reinterpret_cast<float4*>(d_rgba), static_cast<cudaStream_t>(stream));
}

extern "C" GRRT_EXPORT int grrt_batch_render(GRRTBatch* b, float* const* framebuffers) {
    if (!b || !framebuffers) return -1;
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
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) out->kernel_ms = ms;
    cudaGetLastError();
    return 0;
}

// Times the candidate schedules on the batch itself and keeps the fastest.
// With a cache path, a schedule stored for an identical batch (same cameras,
// sizes, spins, inclinations and form) is reused without timing, and a new
// choice is appended. Returns 0 and writes the chosen time (ms) to *best_ms.
extern "C" GRRT_EXPORT int grrt_batch_autotune(GRRTBatch* b, const char* cache_path, double* best_ms) {
    if (!b) return -1;
    if (!batch_ensure_device(b)) return -1;
    const std::string key = batch_key(*b);
    if (cache_path && cache_path[0]) {
        std::ifstream in(cache_path);
        std::string line;
        while (std::getline(in, line)) {
            int cs = 0, od = 0, bp = 0;
            double ms = 0;
            char kbuf[64] = {0};
            if (std::sscanf(line.c_str(), " {\"key\": \"%63[^\"]\", \"chunk\": %d, \"order\": %d, \"blocks_per_sm\": %d, \"ms\": %lf",
                            kbuf, &cs, &od, &bp, &ms) == 5 &&
                key == kbuf) {
                grrt_batch_set_schedule(b, cs, od, bp);
                b->tuned = true;
                if (best_ms) *best_ms = ms;
                return 0;
            }
        }
    }
    if (!b->d_out && b->fail(cudaMalloc(&b->d_out, sizeof(float4) * b->total_pixels), "cudaMalloc(output)")) return -1;
    const int maxb = GRRTBatch::max_blocks_per_sm(b->form);
    double best = 1e30;
    int bc = b->chunk_size, bo = b->order, bb = b->blocks_per_sm;
    // the mixed form's phases ignore the chunk table: only the occupancy varies
    const bool mixed = b->form == GRRT_FORM_MIXED;
    const std::vector<int> orders = mixed ? std::vector<int>{b->order}
                                          : std::vector<int>{GRRT_BATCH_ORDER_ROUND_ROBIN, GRRT_BATCH_ORDER_CAMERA_MAJOR};
    const std::vector<int> chunks = mixed ? std::vector<int>{b->chunk_size} : std::vector<int>{64, 256, 1024, 4096};
    for (int order : orders)
        for (int cs : chunks)
            for (int bp : {maxb, std::max(1, maxb - 1)}) {
                grrt_batch_set_schedule(b, cs, order, bp);
                double t = 1e30;
                for (int rep = 0; rep < 2; ++rep) {
                    if (b->launch(b->d_out, b->stream) != 0) return -1;
                    if (b->fail(cudaStreamSynchronize(b->stream), "autotune run")) return -1;
                    float ms = 0;
                    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
                    t = std::min(t, static_cast<double>(ms));
                }
                if (t < best) {
                    best = t;
                    bc = cs;
                    bo = order;
                    bb = bp;
                }
            }
    grrt_batch_set_schedule(b, bc, bo, bb);
    b->tuned = true;
    if (best_ms) *best_ms = best;
    if (cache_path && cache_path[0]) {
        std::ofstream out(cache_path, std::ios::app);
        out.precision(17);
        out << "{\"key\": \"" << key << "\", \"chunk\": " << bc << ", \"order\": " << bo << ", \"blocks_per_sm\": " << bb
            << ", \"ms\": " << best << "}\n";
    }
    return 0;
}
