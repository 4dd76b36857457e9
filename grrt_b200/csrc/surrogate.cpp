// The learned surrogate (include/grrt_surrogate.h): an MLP 4 -> 256 x 4 -> 6
// (SiLU), BF16 weights with FP32 master copies, trained with Adam on the GPU.
//
// Training: layer 1 (K = 4) runs on the CUDA cores; layers 2-5 and every
// backward GEMM run on the tensor cores through umma_gemm_bf16 (tcgen05, FP32
// accumulation in TMEM). A training step is captured once as a CUDA graph and
// replayed. Inference: one fused tensor-core kernel (mlp_fused.cu).
//
// Rendering: per sample, the camera ray's closed-form margins (capture,
// graze) and the network's outputs decide the colour. A sample whose
// predicted crossing lies outside the disk but whose error band reaches it is
// handed to the mixed form's FP32 speculation, which settles it as dark or
// queues it; a sample whose colour could move by more than the error budget
// (predicted lit, emission thresholds, stars within reach), or that lies in
// the calibrated bands around the critical curve or a graze, is re-traced
// exactly with the FP64 method (the mixed form's re-trace kernel); pixels are
// resolved as in the plain form.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/grrt_surrogate.h"
#include "context.h"
#include "device/mlp_fused.h"
#include "device/render_launch.h"
#include "device/surrogate.h"
#include "device/umma_gemm.h"

using namespace grrt_b200;
using namespace grrt_b200::surr;

namespace {

template <typename T>
bool dalloc(T** p, size_t n) {
    *p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

thread_local std::string g_surr_error;

}  // namespace

struct GRRTSurrogate {
    int device = -1;
    cudaStream_t stream = nullptr;
    std::string error;

    // parameters (FP32 master), gradients, Adam moments, step counter
    float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
    unsigned* d_step = nullptr;
    __nv_bfloat16 *d_wb[3] = {}, *d_wt[3] = {}, *d_w5b = nullptr, *d_w5t = nullptr;
    int* d_err = nullptr;
    DevStats* d_stats = nullptr;
    unsigned* d_queue = nullptr;

    // training set
    float *d_X = nullptr, *d_Y = nullptr;
    size_t n_data = 0;

    // training workspace for one batch size
    int ws_batch = 0, splits = 1;
    float *Xb = nullptr, *Yb = nullptr, *Z[4] = {}, *O = nullptr, *part = nullptr, *colpart = nullptr;
    float *loss = nullptr, *loss_hist = nullptr;
    int hist_cap = 0;
    __nv_bfloat16 *H[4] = {}, *dO = nullptr, *dZ[4] = {}, *TA = nullptr, *TB = nullptr;
    static constexpr int kColParts = 64;

    // inference workspace
    size_t inf_chunk = 0;
    float *iX = nullptr, *iO = nullptr;
    SampleAux* iaux = nullptr;
    unsigned* icount = nullptr;  // samples of the chunk that go through the network
    static constexpr size_t kChunk = size_t(1) << 22;

    RenderBands bands;
    bool calibrated = false;
    long long steps_done = 0;
    float last_loss = NAN;
    LossWeights weights;
    size_t last_render_samples = 0;
    // counts of the last render, copied into the surrogate's own buffer
    // (icount[1..3]: network, exact, speculated) so they outlive the context
    bool have_counts = false;

    ~GRRTSurrogate() {
        if (device >= 0) cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        free_workspace();
        free_inference();
        for (auto* p : {d_params, d_grad, d_m, d_v, d_X, d_Y}) {
            if (p) cudaFree(p);
        }
        dfree(d_step);
        for (int l = 0; l < 3; ++l) {
            dfree(d_wb[l]);
            dfree(d_wt[l]);
        }
        dfree(d_w5b);
        dfree(d_w5t);
        dfree(d_err);
        dfree(d_stats);
        dfree(d_queue);
        if (stream) cudaStreamDestroy(stream);
    }

    bool fail(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return false;
        error = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGetLastError();
        return true;
    }
    bool fail_msg(const std::string& m) {
        error = m;
        return true;
    }
    // copies are ordered on the surrogate's (non-blocking) stream, then waited for
    cudaError_t copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) const {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        return e;
    }

    void free_workspace() {
        dfree(Xb);
        dfree(Yb);
        dfree(O);
        dfree(part);
        dfree(colpart);
        dfree(loss);
        dfree(loss_hist);
        for (int l = 0; l < 4; ++l) {
            dfree(Z[l]);
            dfree(H[l]);
            dfree(dZ[l]);
        }
        dfree(dO);
        dfree(TA);
        dfree(TB);
        ws_batch = 0;
    }
    void free_inference() {
        dfree(iX);
        dfree(iO);
        dfree(iaux);
        dfree(icount);
        inf_chunk = 0;
        have_counts = false;
    }

    bool init(unsigned seed) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            error = "no CUDA device available (the surrogate trains and renders on the GPU)";
            return false;
        }
        if (fail(cudaGetDevice(&device), "cudaGetDevice")) return false;
        cudaDeviceProp prop{};
        if (fail(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return false;
        if (prop.major < 10) {
            error = "the surrogate's tensor-core kernels need an sm_100 GPU";
            return false;
        }
        if (fail(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
        const size_t P = ParamLayout::total;
        if (!dalloc(&d_params, P) || !dalloc(&d_grad, P) || !dalloc(&d_m, P) || !dalloc(&d_v, P) ||
            !dalloc(&d_step, 1) || !dalloc(&d_err, 1) || !dalloc(&d_stats, 1) || !dalloc(&d_queue, 1))
            return !fail_msg("cudaMalloc(surrogate parameters) failed");
        for (int l = 0; l < 3; ++l)
            if (!dalloc(&d_wb[l], kHidden * kHidden) || !dalloc(&d_wt[l], kHidden * kHidden))
                return !fail_msg("cudaMalloc(bf16 weights) failed");
        if (!dalloc(&d_w5b, kOutPad * kHidden) || !dalloc(&d_w5t, kHidden * kDOutPad))
            return !fail_msg("cudaMalloc(bf16 weights) failed");
        cudaMemsetAsync(d_w5t, 0, sizeof(__nv_bfloat16) * kHidden * kDOutPad, stream);
        cudaMemsetAsync(d_err, 0, sizeof(int), stream);
        // uniform init with variance 1/fan_in; biases 0; unused output rows 0
        std::vector<float> h(P, 0.0f);
        std::mt19937 rng(seed);
        auto fill = [&](size_t off, int rows, int cols, int used_rows) {
            const float bound = std::sqrt(3.0f / cols);
            std::uniform_real_distribution<float> U(-bound, bound);
            for (int r = 0; r < rows; ++r)
                for (int c = 0; c < cols; ++c)
                    h[off + static_cast<size_t>(r) * cols + c] = r < used_rows ? U(rng) : 0.0f;
        };
        fill(ParamLayout::w1, kHidden, kIn, kHidden);
        for (int l = 2; l <= 4; ++l) fill(ParamLayout::w(l), kHidden, kHidden, kHidden);
        fill(ParamLayout::w5, kOutPad, kHidden, kUsedOut);
        return set_params(h.data(), P);
    }

    bool set_params(const float* h, size_t n) {
        if (n != ParamLayout::total) return !fail_msg("parameter count mismatch");
        cudaSetDevice(device);
        if (fail(copy(d_params, h, n * sizeof(float), cudaMemcpyHostToDevice), "upload parameters")) return false;
        cudaMemsetAsync(d_m, 0, n * sizeof(float), stream);
        cudaMemsetAsync(d_v, 0, n * sizeof(float), stream);
        cudaMemsetAsync(d_step, 0, sizeof(unsigned), stream);
        steps_done = 0;
        if (fail(launch_cast_weights(d_params, d_wb, d_wt, d_w5b, d_w5t, stream), "cast weights")) return false;
        return !fail(cudaStreamSynchronize(stream), "cast weights");
    }

    bool gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, int sp,
              const GemmEpilogue& ep) {
        return !fail(umma_gemm_bf16(A, lda, B, ldb, M, N, K, sp, ep, d_err, stream), "tensor-core GEMM");
    }

    bool check_gemm_errors() {
        int h = 0;
        if (fail(copy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost), "read error flag")) return false;
        if (h != 0) {
            error = "tensor-core kernel reported a timeout (code " + std::to_string(h) + ")";
            cudaMemsetAsync(d_err, 0, sizeof(int), stream);
            return false;
        }
        return true;
    }

    // ---- data --------------------------------------------------------------
    bool trace_set(const GRRTParams* cams, int n_cams, int n_side, int jitter_s, float** X, float** Y, size_t* n_out) {
        if (!cams || n_cams <= 0 || n_side <= 0 || n_side > 4096) return !fail_msg("bad camera list or size");
        std::vector<std::unique_ptr<GRRTContext>> ctxs;
        std::vector<DevScene> scenes;
        for (int c = 0; c < n_cams; ++c) {
            GRRTParams p = cams[c];
            p.width = n_side;
            p.height = n_side;
            p.samples_per_pixel = 1;
            if (p.disk_volumetric) return !fail_msg("the surrogate covers thin-disk scenes");
            auto ctx = std::make_unique<GRRTContext>();
            try {
                ctx->build(p);
            } catch (const std::exception& e) {
                return !fail_msg(std::string("camera build: ") + e.what());
            }
            if (!ctx->ensure_device()) return !fail_msg(ctx->error);
            scenes.push_back(ctx->scene_for_launch());
            ctxs.push_back(std::move(ctx));
        }
        cudaSetDevice(device);
        // the contexts' table uploads ran on the legacy stream
        if (fail(cudaDeviceSynchronize(), "scene upload")) return false;
        const size_t n = static_cast<size_t>(n_cams) * n_side * n_side;
        DevScene* d_sc = nullptr;
        if (!dalloc(&d_sc, scenes.size())) return !fail_msg("cudaMalloc(scenes)");
        float *x = nullptr, *y = nullptr;
        if (!dalloc(&x, n * kIn) || !dalloc(&y, n * kYCols)) {
            dfree(d_sc);
            dfree(x);
            return !fail_msg("cudaMalloc(training set) failed");
        }
        bool ok = !fail(cudaMemcpyAsync(d_sc, scenes.data(), sizeof(DevScene) * scenes.size(),
                                        cudaMemcpyHostToDevice, stream),
                        "upload scenes") &&
                  !fail(cudaMemsetAsync(d_stats, 0, sizeof(DevStats), stream), "memset") &&
                  !fail(launch_trace_dataset(d_sc, n_cams, n_side, jitter_s, x, y, d_queue, d_stats, stream),
                        "trace training set") &&
                  !fail(cudaStreamSynchronize(stream), "trace training set");
        cudaFree(d_sc);
        if (!ok) {
            dfree(x);
            dfree(y);
            return false;
        }
        *X = x;
        *Y = y;
        *n_out = n;
        return true;
    }

    // ---- training ------------------------------------------------------------
    bool ensure_workspace(int B) {
        if (ws_batch == B) return true;
        free_workspace();
        const size_t b = static_cast<size_t>(B);
        splits = std::max(1, std::min(32, B / 64 / 4));
        bool ok = dalloc(&Xb, b * kIn) && dalloc(&Yb, b * kYCols) && dalloc(&O, b * kOutPad) &&
                  dalloc(&part, static_cast<size_t>(splits) * kHidden * kHidden) &&
                  dalloc(&colpart, static_cast<size_t>(kColParts) * kHidden * 5) && dalloc(&loss, 1) &&
                  dalloc(&dO, b * kDOutPad) && dalloc(&TA, b * kHidden) && dalloc(&TB, b * kHidden);
        for (int l = 0; l < 4 && ok; ++l)
            ok = dalloc(&Z[l], b * kHidden) && dalloc(&H[l], b * kHidden) && dalloc(&dZ[l], b * kHidden);
        if (!ok) {
            free_workspace();
            return !fail_msg("cudaMalloc(training workspace) failed");
        }
        cudaMemsetAsync(dO, 0, b * kDOutPad * sizeof(__nv_bfloat16), stream);
        ws_batch = B;
        return true;
    }

    // splits the GEMM actually uses (every split gets at least one K-block)
    int effective_splits(int K) const {
        const int kbt = K / 64;
        const int per = (kbt + splits - 1) / splits;
        return (kbt + per - 1) / per;
    }

    // Forward + loss + backward of the batch in Xb/Yb; gradients into d_grad.
    bool enqueue_fwd_bwd(int B) {
        const size_t P = ParamLayout::total;
        if (fail(launch_layer1_fwd(Xb, B, d_params, Z[0], H[0], stream), "layer 1")) return false;
        for (int l = 2; l <= 4; ++l) {
            GemmEpilogue ep;
            ep.bias = d_params + ParamLayout::b(l);
            ep.out_f32 = Z[l - 1];
            ep.ld_f32 = kHidden;
            ep.out_bf16 = H[l - 1];
            ep.ld_bf16 = kHidden;
            ep.act = kActSilu;
            if (!gemm(H[l - 2], kHidden, d_wb[l - 2], kHidden, B, kHidden, kHidden, 1, ep)) return false;
        }
        {
            GemmEpilogue ep;
            ep.bias = d_params + ParamLayout::b5;
            ep.out_f32 = O;
            ep.ld_f32 = kOutPad;
            if (!gemm(H[3], kHidden, d_w5b, kHidden, B, kOutPad, kHidden, 1, ep)) return false;
        }
        if (fail(cudaMemsetAsync(loss, 0, sizeof(float), stream), "memset")) return false;
        if (fail(cudaMemsetAsync(d_grad, 0, P * sizeof(float), stream), "memset")) return false;
        if (fail(launch_loss(O, Yb, B, weights, dO, loss, stream), "loss")) return false;
        // output layer: dW5 = dO^T H4, db5 = colsum(dO), dZ4 = (dO W5) * silu'(Z4)
        if (fail(launch_transpose(dO, B, kOutPad, kDOutPad, TA, B, stream), "transpose")) return false;
        if (fail(launch_transpose(H[3], B, kHidden, kHidden, TB, B, stream), "transpose")) return false;
        {
            GemmEpilogue ep;
            ep.out_f32 = part;
            ep.ld_f32 = kHidden;
            ep.split_stride = static_cast<size_t>(kOutPad) * kHidden;
            if (!gemm(TA, B, TB, B, kOutPad, kHidden, B, splits, ep)) return false;
            if (fail(launch_reduce_splits(part, effective_splits(B), static_cast<size_t>(kOutPad) * kHidden,
                                          d_grad + ParamLayout::w5, stream),
                     "reduce"))
                return false;
        }
        if (fail(launch_colsum(dO, B, kOutPad, kDOutPad, colpart, kColParts, d_grad + ParamLayout::b5, stream),
                 "colsum"))
            return false;
        {
            GemmEpilogue ep;
            ep.gate_z = Z[3];
            ep.ld_gate = kHidden;
            ep.out_bf16 = dZ[3];
            ep.ld_bf16 = kHidden;
            if (!gemm(dO, kDOutPad, d_w5t, kDOutPad, B, kHidden, kDOutPad, 1, ep)) return false;
        }
        for (int l = 4; l >= 2; --l) {
            // dW_l = dZ_l^T H_{l-1}, db_l = colsum(dZ_l), dZ_{l-1} = (dZ_l W_l) * silu'(Z_{l-1})
            if (fail(launch_transpose(dZ[l - 1], B, kHidden, kHidden, TA, B, stream), "transpose")) return false;
            if (fail(launch_transpose(H[l - 2], B, kHidden, kHidden, TB, B, stream), "transpose")) return false;
            GemmEpilogue ep;
            ep.out_f32 = part;
            ep.ld_f32 = kHidden;
            ep.split_stride = static_cast<size_t>(kHidden) * kHidden;
            if (!gemm(TA, B, TB, B, kHidden, kHidden, B, splits, ep)) return false;
            if (fail(launch_reduce_splits(part, effective_splits(B), static_cast<size_t>(kHidden) * kHidden,
                                          d_grad + ParamLayout::w(l), stream),
                     "reduce"))
                return false;
            if (fail(launch_colsum(dZ[l - 1], B, kHidden, kHidden, colpart, kColParts, d_grad + ParamLayout::b(l),
                                   stream),
                     "colsum"))
                return false;
            GemmEpilogue eb;
            eb.gate_z = Z[l - 2];
            eb.ld_gate = kHidden;
            eb.out_bf16 = dZ[l - 2];
            eb.ld_bf16 = kHidden;
            if (!gemm(dZ[l - 1], kHidden, d_wt[l - 2], kHidden, B, kHidden, kHidden, 1, eb)) return false;
        }
        return !fail(launch_layer1_bwd(dZ[0], Xb, B, colpart, kColParts, d_grad, stream), "layer 1 backward");
    }

    bool enqueue_train_step(int B, float lr) {
        if (fail(launch_gather(d_X, d_Y, n_data, B, d_step, Xb, Yb, stream), "gather")) return false;
        if (!enqueue_fwd_bwd(B)) return false;
        if (fail(launch_adam(d_params, d_grad, d_m, d_v, ParamLayout::total, d_step, lr, 0.9f, 0.999f, 1e-8f, stream),
                 "adam"))
            return false;
        if (fail(launch_record_loss(loss, d_step, loss_hist, hist_cap, stream), "record loss")) return false;
        return !fail(launch_cast_weights(d_params, d_wb, d_wt, d_w5b, d_w5t, stream), "cast weights");
    }

    // `steps` Adam steps at batch B. Learning rate: lr for the first half, then
    // halved every eighth of the run (piecewise constant, one graph per rate).
    bool train(int steps, int B, double lr, float* loss_out) {
        if (n_data == 0) return !fail_msg("no training set: call grrt_surrogate_generate first");
        if (steps <= 0 || B < 128 || B % 128 != 0 || B > (1 << 20)) return !fail_msg("bad steps or batch size");
        cudaSetDevice(device);
        if (!ensure_workspace(B)) return false;
        dfree(loss_hist);
        hist_cap = 0;
        unsigned t0 = 0;
        if (fail(copy(&t0, d_step, sizeof(unsigned), cudaMemcpyDeviceToHost), "read step")) return false;
        // the loss history is indexed by the global step counter
        hist_cap = static_cast<int>(t0) + steps;
        if (!dalloc(&loss_hist, static_cast<size_t>(hist_cap))) return !fail_msg("cudaMalloc(loss history)");
        int done = 0;
        const int phases[] = {steps / 2, steps / 8, steps / 8, steps / 8, steps - steps / 2 - 3 * (steps / 8)};
        double rate = lr;
        for (int ph = 0; ph < 5; ++ph, rate *= 0.5) {
            int n = phases[ph];
            if (n <= 0) continue;
            // one eager step (it also sets the kernels' launch attributes), then a graph
            if (!enqueue_train_step(B, static_cast<float>(rate))) return false;
            --n;
            ++done;
            if (n > 0) {
                cudaGraph_t g = nullptr;
                cudaGraphExec_t ge = nullptr;
                if (fail(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
                    return false;
                const bool ok = enqueue_train_step(B, static_cast<float>(rate));
                const cudaError_t ce = cudaStreamEndCapture(stream, &g);
                if (!ok || fail(ce, "end capture")) {
                    if (g) cudaGraphDestroy(g);
                    return false;
                }
                const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (fail(ie, "graph instantiate")) return false;
                for (int i = 0; i < n; ++i) {
                    if (fail(cudaGraphLaunch(ge, stream), "graph launch")) {
                        cudaGraphExecDestroy(ge);
                        return false;
                    }
                }
                done += n;
                const cudaError_t se = cudaStreamSynchronize(stream);
                cudaGraphExecDestroy(ge);
                if (fail(se, "training")) return false;
            }
            if (!check_gemm_errors()) return false;
        }
        if (fail(cudaStreamSynchronize(stream), "training")) return false;
        std::vector<float> hist(static_cast<size_t>(steps));
        if (fail(copy(hist.data(), loss_hist + t0, sizeof(float) * steps, cudaMemcpyDeviceToHost), "read loss"))
            return false;
        if (loss_out) std::memcpy(loss_out, hist.data(), sizeof(float) * steps);
        last_loss = hist.back();
        steps_done += done;
        calibrated = false;
        return check_gemm_errors();
    }

    // ---- inference -----------------------------------------------------------
    bool ensure_inference(size_t chunk) {
        if (inf_chunk >= chunk) return true;
        free_inference();
        if (!dalloc(&iX, chunk * kIn) || !dalloc(&iO, chunk * kOutPad) || !dalloc(&iaux, chunk) ||
            !dalloc(&icount, 64)) {
            free_inference();
            return !fail_msg("cudaMalloc(inference workspace) failed");
        }
        inf_chunk = chunk;
        return true;
    }

    // O[n x 16] = network(X[n x 4]): the fused tensor-core kernel (rows
    // min(n, *d_n) when a device count is given)
    bool enqueue_forward(const float* X, size_t n, float* out, const unsigned* d_n = nullptr) {
        return !fail(launch_mlp_fused(X, static_cast<long long>(n), d_params, d_wb, d_w5b, out, d_err, stream, d_n),
                     "fused network");
    }

    bool render(GRRTContext* ctx, const DevTile& tile, float* d_rgba, double* d_rgb64, unsigned* d_fate,
                cudaStream_t s) {
        if (!ctx->ensure_device()) return !fail_msg(ctx->error);
        if (ctx->vol) return !fail_msg("the surrogate renders thin-disk scenes");
        if (ctx->device != device) return !fail_msg("context and surrogate are on different GPUs");
        const DevScene S = ctx->scene_for_launch();
        const int g2 = S.grid * S.grid;
        const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
        if (n == 0) return true;
        // scratch of the mixed form's layout: per-sample colour/fate + re-trace queue
        const size_t bytes = mixed_scratch_bytes(tile, g2);
        if (bytes > ctx->d_mixed_scratch_bytes) {
            cudaFree(ctx->d_mixed_scratch);
            ctx->d_mixed_scratch = nullptr;
            ctx->d_mixed_scratch_bytes = 0;
            if (fail(cudaMalloc(&ctx->d_mixed_scratch, bytes), "cudaMalloc(surrogate scratch)")) return false;
            ctx->d_mixed_scratch_bytes = bytes;
        }
        if (!ensure_inference(std::min(n, kChunk))) return false;
        DevMixedBuffers mb = mixed_buffers_with_list(ctx->d_mixed_scratch, n, ctx->d_queue);
        mb.r_near = ctx->mixed_r_near();
        mb.margin = ctx->mixed_margin;
        // the surrogate's kernels run on its own stream, ordered after the caller's
        cudaEvent_t e_in = nullptr;
        if (fail(cudaEventCreateWithFlags(&e_in, cudaEventDisableTiming), "event")) return false;
        cudaEventRecord(e_in, s);
        cudaStreamWaitEvent(stream, e_in, 0);
        cudaEventDestroy(e_in);
        cudaEventRecord(ctx->ev0, stream);
        cudaEventRecord(ctx->ev_phase[0], stream);
        if (fail(cudaMemsetAsync(ctx->d_stats, 0, sizeof(DevStats), stream), "memset") ||
            fail(cudaMemsetAsync(ctx->d_mixed_scratch, 0, 1024, stream), "memset"))
            return false;
        // On a black sky a sample whose closed-form smallest radius lies
        // outside the disk, r_near and every photon orbit is settled by the
        // prepare pass (colour 0, escaped) and skips the network.
        const double settle_radius =
            S.stars_on ? 0.0
                       : std::max(std::max(5.0 * S.M, mb.r_near), S.disk_on ? S.r_out + 2.0 * mb.margin : 0.0);
        // network and shading, chunk by chunk (icount[1]: the render's network samples)
        if (fail(cudaMemsetAsync(icount + 1, 0, sizeof(unsigned), stream), "memset")) return false;
        for (size_t q0 = 0; q0 < n; q0 += kChunk) {
            const size_t nq = std::min(kChunk, n - q0);
            if (fail(cudaMemsetAsync(icount, 0, sizeof(unsigned), stream), "memset") ||
                fail(launch_prepare(S, tile, q0, nq, settle_radius, iX, iaux, icount, icount + 1, mb, ctx->d_stats,
                                    stream),
                     "prepare"))
                return false;
            if (!enqueue_forward(iX, nq, iO, icount)) return false;
            if (fail(launch_shade(S, tile, icount, nq, iO, iaux, bands, mb, ctx->d_stats, stream), "shade"))
                return false;
        }
        cudaEventRecord(ctx->ev_phase[1], stream);
        // the uncertain samples: FP32 speculation (and its star pass) settles the
        // dark ones and adds the rest to the exact list
        if (fail(cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned), stream), "memset") ||
            fail(launch_mixed_speculate(S, tile, mb, ctx->d_stats, stream), "speculation") ||
            fail(launch_mixed_stars(S, tile, mb, stream), "star pass"))
            return false;
        cudaEventRecord(ctx->ev_phase[2], stream);
        if (fail(launch_mixed_retrace(S, tile, mb, ctx->d_stats, ctx->d_mixed_scratch, stream), "exact re-trace"))
            return false;
        cudaEventRecord(ctx->ev_phase[3], stream);
        ThinOutputs out;
        out.rgba = reinterpret_cast<float4*>(d_rgba);
        out.rgb64 = d_rgb64;
        out.fate = d_fate;
        if (fail(launch_mixed_resolve(S, tile, mb, out, ctx->d_stats, stream), "resolve")) return false;
        if (fail(cudaMemcpyAsync(icount + 2, mb.retrace_count, sizeof(unsigned), cudaMemcpyDeviceToDevice, stream),
                 "counts") ||
            fail(cudaMemcpyAsync(icount + 3, mb.spec_count, sizeof(unsigned), cudaMemcpyDeviceToDevice, stream),
                 "counts"))
            return false;
        cudaEventRecord(ctx->ev_phase[4], stream);
        cudaEventRecord(ctx->ev1, stream);
        ctx->n_phases = kMixedPhases;
        // the caller's stream waits for the render
        cudaEvent_t e_out = nullptr;
        if (fail(cudaEventCreateWithFlags(&e_out, cudaEventDisableTiming), "event")) return false;
        cudaEventRecord(e_out, stream);
        cudaStreamWaitEvent(s, e_out, 0);
        cudaEventDestroy(e_out);
        last_render_samples = n;
        have_counts = true;
        return true;
    }

    // ---- calibration ---------------------------------------------------------
    static double quantile(std::vector<float>& v, double q) {
        if (v.empty()) return 0.0;
        const size_t k = std::min(v.size() - 1, static_cast<size_t>(q * (v.size() - 1)));
        std::nth_element(v.begin(), v.begin() + k, v.end());
        return v[k];
    }

    bool calibrate(const GRRTParams* cams, int n_cams, int n_side, double q, double safety, double* report) {
        if (!(q > 0.0 && q <= 1.0) || !(safety >= 1.0)) return !fail_msg("bad quantile or safety factor");
        float *X = nullptr, *Y = nullptr;
        size_t n = 0;
        if (!trace_set(cams, n_cams, n_side, 1, &X, &Y, &n)) return false;
        bool ok = ensure_inference(std::min(n, kChunk));
        float* err = nullptr;
        ok = ok && dalloc(&err, n * 4);
        for (size_t q0 = 0; ok && q0 < n; q0 += kChunk) {
            const size_t nq = std::min(kChunk, n - q0);
            ok = enqueue_forward(X + q0 * kIn, nq, iO) &&
                 !fail(launch_eval_errors(iO, Y + q0 * kYCols, nq, err + q0 * 4, stream), "errors");
        }
        ok = ok && !fail(cudaStreamSynchronize(stream), "calibration") && check_gemm_errors();
        std::vector<float> he, hy;
        if (ok) {
            he.resize(n * 4);
            hy.resize(n * kYCols);
            ok = !fail(copy(he.data(), err, n * 4 * sizeof(float), cudaMemcpyDeviceToHost), "read errors") &&
                 !fail(copy(hy.data(), Y, n * kYCols * sizeof(float), cudaMemcpyDeviceToHost), "read targets");
        }
        dfree(err);
        dfree(X);
        dfree(Y);
        if (!ok) return false;
        // 1. critical band: holds every sample whose closed-form fate disagrees
        //    with the integrator's (x2) and every sample with a relevant crossing
        //    after the second that does not graze (x1.2); never below the
        //    training fit cut
        // 2. graze band: the training fit cut (mu of the turning point)
        // 3. network error quantiles over the samples outside both bands (u:
        //    the error in units of the network's own predicted sigma)
        float cap_bad = 0.0f, multi = 0.0f;
        size_t n_cap_bad = 0, n_multi = 0;
        for (size_t i = 0; i < n; ++i) {
            const float* y = &hy[kYCols * i];
            const int term = static_cast<int>(y[6]);
            if (term == kTermMaxSteps) continue;
            if ((y[8] > 0.0f) != (term == kTermHorizon)) {
                cap_bad = std::max(cap_bad, std::fabs(y[8]));
                ++n_cap_bad;
            }
            if (y[7] >= 1.0f && y[9] >= kFitGraze) {
                multi = std::max(multi, std::fabs(y[8]));
                ++n_multi;
            }
        }
        const double cap_band = std::max({static_cast<double>(kFitCapture), 2.0 * cap_bad, 1.2 * multi});
        std::vector<float> du, dir, cth;
        size_t in_band = 0;
        for (size_t i = 0; i < n; ++i) {
            const float* e = &he[4 * i];
            const float* y = &hy[kYCols * i];
            if (std::fabs(y[8]) < cap_band || y[9] < kFitGraze || static_cast<int>(y[6]) == kTermMaxSteps) {
                ++in_band;
                continue;
            }
            if (e[0] >= 0.0f) du.push_back(std::max(e[0], e[1]));
            if (e[2] >= 0.0f) {
                dir.push_back(e[2]);
                cth.push_back(e[3]);
            }
        }
        const double median_du = quantile(du, 0.5);
        bands.du = safety * quantile(du, q);  // multiple of the predicted sigma
        const double du_arc = 1.0 / 1000.0 - 1.0 / 7000.0;
        // direction: multiple of sigma_dir covering the arc-start error and the
        // arc-length error from c_theta
        bands.dir = safety * (quantile(dir, q) + quantile(cth, q) * du_arc);
        bands.capture = cap_band;
        bands.graze = kFitGraze;
        calibrated = true;
        if (report) {
            report[0] = bands.du;
            report[1] = bands.dir;
            report[2] = bands.capture;
            report[3] = bands.graze;
            report[4] = static_cast<double>(n);
            report[5] = static_cast<double>(n_cap_bad);
            report[6] = static_cast<double>(in_band) / static_cast<double>(n);
            report[7] = median_du;
        }
        (void)n_multi;
        return true;
    }
};

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT GRRTSurrogate* grrt_surrogate_create(unsigned seed) {
    auto s = std::make_unique<GRRTSurrogate>();
    if (!s->init(seed)) {
        g_surr_error = "grrt_surrogate_create: " + s->error;
        return nullptr;
    }
    return s.release();
}

extern "C" GRRT_EXPORT void grrt_surrogate_destroy(GRRTSurrogate* s) { delete s; }

extern "C" GRRT_EXPORT const char* grrt_surrogate_error(const GRRTSurrogate* s) {
    if (!s) return g_surr_error.empty() ? nullptr : g_surr_error.c_str();
    return s->error.empty() ? nullptr : s->error.c_str();
}

extern "C" GRRT_EXPORT int grrt_surrogate_generate(GRRTSurrogate* s, const GRRTParams* cams, int n_cams, int n_side) {
    if (!s) return -1;
    s->error.clear();
    cudaSetDevice(s->device);
    float *X = nullptr, *Y = nullptr;
    size_t n = 0;
    if (!s->trace_set(cams, n_cams, n_side, 0, &X, &Y, &n)) return -1;
    dfree(s->d_X);
    dfree(s->d_Y);
    s->d_X = X;
    s->d_Y = Y;
    s->n_data = n;
    return 0;
}

extern "C" GRRT_EXPORT long long grrt_surrogate_dataset(GRRTSurrogate* s, float* x_out, float* y_out,
                                                        long long capacity) {
    if (!s) return -1;
    const long long n = static_cast<long long>(s->n_data);
    if (x_out && y_out && capacity >= n && n > 0) {
        cudaSetDevice(s->device);
        if (s->copy(x_out, s->d_X, sizeof(float) * kIn * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
            s->copy(y_out, s->d_Y, sizeof(float) * kYCols * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
    }
    return n;
}

extern "C" GRRT_EXPORT int grrt_surrogate_train(GRRTSurrogate* s, int steps, int batch, double lr, float* loss_out) {
    if (!s) return -1;
    s->error.clear();
    return s->train(steps, batch, lr, loss_out) ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_surrogate_calibrate(GRRTSurrogate* s, const GRRTParams* cams, int n_cams, int n_side,
                                                    double quantile, double safety, double* report8) {
    if (!s) return -1;
    s->error.clear();
    cudaSetDevice(s->device);
    return s->calibrate(cams, n_cams, n_side, quantile, safety, report8) ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_surrogate_set_bands(GRRTSurrogate* s, double du, double dir, double capture,
                                                    double graze, double tol_rel) {
    if (!s || !(du >= 0.0) || !(dir >= 0.0) || !(capture >= 0.0) || !(graze >= 0.0) || !(tol_rel > 0.0)) return -1;
    s->bands.du = du;
    s->bands.dir = dir;
    s->bands.capture = capture;
    s->bands.graze = graze;
    s->bands.tol_rel = tol_rel;
    s->calibrated = true;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_surrogate_get_bands(const GRRTSurrogate* s, double* out5) {
    if (!s || !out5) return -1;
    out5[0] = s->bands.du;
    out5[1] = s->bands.dir;
    out5[2] = s->bands.capture;
    out5[3] = s->bands.graze;
    out5[4] = s->bands.tol_rel;
    return s->calibrated ? 1 : 0;
}

extern "C" GRRT_EXPORT long long grrt_surrogate_params(GRRTSurrogate* s, float* out, long long capacity) {
    if (!s) return -1;
    const long long n = static_cast<long long>(ParamLayout::total);
    if (out && capacity >= n) {
        cudaSetDevice(s->device);
        if (s->copy(out, s->d_params, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
    }
    return n;
}

extern "C" GRRT_EXPORT int grrt_surrogate_set_params(GRRTSurrogate* s, const float* in, long long n) {
    if (!s || !in || n != static_cast<long long>(ParamLayout::total)) return -1;
    s->error.clear();
    return s->set_params(in, static_cast<size_t>(n)) ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_surrogate_forward(GRRTSurrogate* s, const float* d_in, long long n, float* d_out) {
    if (!s || !d_in || !d_out || n <= 0) return -1;
    s->error.clear();
    cudaSetDevice(s->device);
    if (!s->enqueue_forward(d_in, static_cast<size_t>(n), d_out)) return -1;
    if (s->fail(cudaStreamSynchronize(s->stream), "forward")) return -1;
    return s->check_gemm_errors() ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_surrogate_gradients(GRRTSurrogate* s, const float* h_in, const float* h_y, int n,
                                                    float* h_grad, double* loss) {
    if (!s || !h_in || !h_y || !h_grad || n < 128 || n % 128 != 0) return -1;
    s->error.clear();
    cudaSetDevice(s->device);
    if (!s->ensure_workspace(n)) return -1;
    if (s->fail(s->copy(s->Xb, h_in, sizeof(float) * kIn * n, cudaMemcpyHostToDevice), "upload") ||
        s->fail(s->copy(s->Yb, h_y, sizeof(float) * kYCols * n, cudaMemcpyHostToDevice), "upload"))
        return -1;
    if (!s->enqueue_fwd_bwd(n)) return -1;
    if (s->fail(cudaStreamSynchronize(s->stream), "gradients") || !s->check_gemm_errors()) return -1;
    float l = 0.0f;
    if (s->fail(s->copy(h_grad, s->d_grad, sizeof(float) * ParamLayout::total, cudaMemcpyDeviceToHost), "read") ||
        s->fail(s->copy(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost), "read"))
        return -1;
    if (loss) *loss = l;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_surrogate_render_device(GRRTSurrogate* s, GRRTContext* ctx, float* d_rgba,
                                                        double* d_rgb64, unsigned int* d_fate, void* stream) {
    if (!s || !ctx) return -1;
    s->error.clear();
    ctx->error.clear();
    cudaSetDevice(s->device);
    DevTile tile;
    tile.w = ctx->params.width;
    tile.h = ctx->params.height;
    tile.out_pitch = tile.w;
    if (!s->render(ctx, tile, d_rgba, d_rgb64, d_fate, static_cast<cudaStream_t>(stream))) {
        ctx->error = s->error;
        return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT int grrt_surrogate_render(GRRTSurrogate* s, GRRTContext* ctx, float* framebuffer) {
    if (!s || !ctx || !framebuffer) return -1;
    const size_t npix = static_cast<size_t>(ctx->params.width) * ctx->params.height;
    float* d = nullptr;
    cudaSetDevice(s->device);
    if (cudaMalloc(&d, npix * 16) != cudaSuccess) {
        cudaGetLastError();
        s->error = "cudaMalloc(frame)";
        return -1;
    }
    int rc = grrt_surrogate_render_device(s, ctx, d, nullptr, nullptr, s->stream);
    if (rc == 0 && s->copy(framebuffer, d, npix * 16, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        s->error = "copy frame";
        rc = -1;
    }
    cudaFree(d);
    if (rc == 0 && !s->check_gemm_errors()) rc = -1;
    return rc;
}

extern "C" GRRT_EXPORT int grrt_surrogate_save(const GRRTSurrogate* s, const char* path) {
    if (!s || !path) return -1;
    std::vector<float> p(ParamLayout::total);
    cudaSetDevice(s->device);
    if (s->copy(p.data(), s->d_params, sizeof(float) * p.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    std::ofstream f(path, std::ios::binary);
    if (!f) return -1;
    const char magic[8] = {'G', 'R', 'R', 'T', 'S', 'U', 'R', '1'};
    f.write(magic, 8);
    const uint64_t n = p.size();
    f.write(reinterpret_cast<const char*>(&n), sizeof(n));
    f.write(reinterpret_cast<const char*>(p.data()), sizeof(float) * n);
    const double b[5] = {s->bands.du, s->bands.dir, s->bands.capture, s->bands.graze, s->bands.tol_rel};
    f.write(reinterpret_cast<const char*>(b), sizeof(b));
    const int cal = s->calibrated ? 1 : 0;
    f.write(reinterpret_cast<const char*>(&cal), sizeof(cal));
    return f.good() ? 0 : -1;
}

extern "C" GRRT_EXPORT int grrt_surrogate_load(GRRTSurrogate* s, const char* path) {
    if (!s || !path) return -1;
    std::ifstream f(path, std::ios::binary);
    if (!f) return -1;
    char magic[8];
    uint64_t n = 0;
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(&n), sizeof(n));
    if (!f || std::memcmp(magic, "GRRTSUR1", 8) != 0 || n != ParamLayout::total) return -1;
    std::vector<float> p(n);
    double b[5];
    int cal = 0;
    f.read(reinterpret_cast<char*>(p.data()), sizeof(float) * n);
    f.read(reinterpret_cast<char*>(b), sizeof(b));
    f.read(reinterpret_cast<char*>(&cal), sizeof(cal));
    if (!f) return -1;
    if (!s->set_params(p.data(), n)) return -1;
    s->bands.du = b[0];
    s->bands.dir = b[1];
    s->bands.capture = b[2];
    s->bands.graze = b[3];
    s->bands.tol_rel = b[4];
    s->calibrated = cal != 0;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_surrogate_last_counts(const GRRTSurrogate* s, long long* exact,
                                                      long long* speculated, long long* network, long long* samples) {
    if (!s || !exact || !samples) return -1;
    unsigned h[3] = {0, 0, 0};  // network, exact, speculated
    if (s->have_counts) {
        cudaSetDevice(s->device);
        if (s->copy(h, s->icount + 1, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            return -1;
        }
    }
    *exact = h[1];
    if (speculated) *speculated = h[2];
    if (network) *network = h[0];
    *samples = static_cast<long long>(s->last_render_samples);
    return 0;
}

extern "C" GRRT_EXPORT int grrt_surrogate_last_exact(const GRRTSurrogate* s, long long* exact, long long* samples) {
    return grrt_surrogate_last_counts(s, exact, nullptr, nullptr, samples);
}
