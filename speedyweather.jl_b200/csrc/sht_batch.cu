// Batches: many transforms of different plans (truncations, grids, layer counts) run as
// grouped launches, one per stage for all of them, and optionally as one CUDA graph.
//
// Replaces the per-call launch sequences of a SpeedyWeather time step, which runs its
// transforms one after another (SpeedyWeather/src/time_stepping/transform.jl:117-191,
// SpeedyWeather/src/dynamics/tendencies.jl:161-214) and caches one CUDA graph per
// transform keyed by the field's device pointer
// (SpeedyTransforms/ext/gpu_graphs_common.jl:296-343).
//
// A batch runs all its synthesis items, then all its analysis items, as
//   Legendre synthesis (all)  ->  FFT synthesis (all)  ->  FFT analysis (all)  ->
//   Legendre analysis (all)
// four persistent launches whose CTAs loop over the union of the items' work lists
// (costliest first). Every item has its own Fourier scratch, so several items may use
// one plan. The Legendre tile width of the grouped launch is chosen by
// sht_batch_autotune, which times the candidates on the batch itself.
#include <algorithm>
#include <vector>

#include "sht_internal.h"

namespace sht {
const Plan* plan_impl(const sht_plan* plan);
int set_error(int code, const char* msg);
}  // namespace sht

using namespace sht;

struct sht_batch {
    std::vector<sht_batch_item> items;
    int device = 0;
    int nsm = 148;
    int bn = 64;                       // FP32 Legendre tile width of the grouped launches
    int fft_smem = 0;
    std::vector<float2*> scratch;      // per item
    LegView* d_leg = nullptr;          // per item
    FftView* d_fft = nullptr;          // per item
    GroupItem* d_lists = nullptr;      // Legendre syn | FFT syn | FFT ana | Legendre ana
    int n_list[4] = {0, 0, 0, 0};
    int off_list[4] = {0, 0, 0, 0};
    int leg_grid[3] = {0, 0, 0};       // persistent grid per tile width 32, 64, 128
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

thread_local char g_msg[512];

int bfail(int code, const char* what) { return set_error(code, what); }
int bcuda(cudaError_t e, const char* what) {
    snprintf(g_msg, sizeof g_msg, "%s: %s", what, cudaGetErrorString(e));
    return set_error(e == cudaErrorMemoryAllocation ? SHT_ENOMEM : SHT_ECUDA, g_msg);
}

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Work lists of the grouped launches for Legendre tile width bn, costliest first.
void build_lists(const sht_batch& b, int bn, std::vector<GroupItem> (&lists)[4]) {
    std::vector<std::pair<double, GroupItem>> w[4];
    for (int t = 0; t < (int)b.items.size(); ++t) {
        const sht_batch_item& it = b.items[t];
        const Plan& p = *plan_impl(it.plan);
        if (p.d.precision != SHT_PREC_FP32) continue;      // tensor-core plans run as their own calls
        const int K = it.nlayers;
        const bool syn = it.direction == SHT_SYNTHESIS;
        const int nct = (2 * K + bn - 1) / bn;
        const std::vector<LegItem>& li = syn ? p.h_syn_items : p.h_ana_items;
        for (const LegItem& l : li) {
            // contraction depth: parity rows (synthesis) or rings from j0(m) (analysis)
            const double depth = syn ? p.rows[l.m] : (double)(p.nh - p.j0[l.m]);
            for (int ct = 0; ct < nct; ++ct)
                for (int par = 0; par < 2; ++par)
                    w[syn ? 0 : 3].push_back({depth * bn, GroupItem{t, l.m, l.tile, ct * 2 + par}});
        }
        for (int j = 0; j < p.nh; ++j) {
            const RingDesc& r = p.h_rings[j];
            for (int ci = 0; ci * r.chunk < K; ++ci) {
                const int c = std::min(r.chunk, K - ci * r.chunk);
                w[syn ? 1 : 2].push_back({c * p.h_ring_cost[j], GroupItem{t, j, ci, 0}});
            }
        }
    }
    for (int q = 0; q < 4; ++q) {
        std::stable_sort(w[q].begin(), w[q].end(),
                         [](const std::pair<double, GroupItem>& x, const std::pair<double, GroupItem>& y) {
                             return x.first > y.first;
                         });
        lists[q].clear();
        for (auto& e : w[q]) lists[q].push_back(e.second);
    }
}

cudaError_t upload_lists(sht_batch& b, int bn) {
    std::vector<GroupItem> lists[4];
    build_lists(b, bn, lists);
    std::vector<GroupItem> all;
    for (int q = 0; q < 4; ++q) {
        b.off_list[q] = (int)all.size();
        b.n_list[q] = (int)lists[q].size();
        all.insert(all.end(), lists[q].begin(), lists[q].end());
    }
    if (b.d_lists) cudaFree(b.d_lists);
    b.d_lists = nullptr;
    cudaError_t e = cudaMalloc(&b.d_lists, std::max<size_t>(1, all.size()) * sizeof(GroupItem));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(b.d_lists, all.data(), all.size() * sizeof(GroupItem), cudaMemcpyHostToDevice);
    b.bn = bn;
    return e;
}

int bn_index(int bn) { return bn == 32 ? 0 : bn == 64 ? 1 : 2; }

// The items of tensor-core plans in one direction, each as its own sht_synthesize /
// sht_analyze call on the stream (their Legendre stage is the persistent tcgen05 kernel).
cudaError_t run_tc_items(const sht_batch& b, bool synthesis, cudaStream_t s) {
    for (const sht_batch_item& it : b.items) {
        if (plan_impl(it.plan)->d.precision == SHT_PREC_FP32 || (it.direction == SHT_SYNTHESIS) != synthesis)
            continue;
        const int rc = synthesis
                           ? sht_synthesize(it.plan, it.coeffs, it.ldc, it.grid, it.ldg, it.nlayers, it.flags, s)
                           : sht_analyze(it.plan, it.grid, it.ldg, it.coeffs, it.ldc, it.nlayers, it.flags, s);
        if (rc != SHT_OK) return cudaErrorLaunchFailure;
    }
    return cudaSuccess;
}

// Every synthesis of the batch completes before any analysis starts (an analysis may read
// a grid a synthesis of the same batch writes): grouped Legendre and Fourier synthesis,
// tensor-core syntheses, grouped Fourier and Legendre analysis, tensor-core analyses.
cudaError_t run(const sht_batch& b, cudaStream_t s) {
    cudaError_t e;
    const int lg = b.leg_grid[bn_index(b.bn)];
    if ((e = launch_legendre_grouped(b.d_leg, b.d_lists + b.off_list[0], b.n_list[0], b.bn, true, lg, s)) !=
        cudaSuccess)
        return e;
    if ((e = launch_fft_grouped(b.d_fft, b.d_lists + b.off_list[1], b.n_list[1], true, b.fft_smem,
                                kFftCtasPerSm * b.nsm, s)) != cudaSuccess)
        return e;
    if ((e = run_tc_items(b, true, s)) != cudaSuccess) return e;
    if ((e = launch_fft_grouped(b.d_fft, b.d_lists + b.off_list[2], b.n_list[2], false, b.fft_smem,
                                kFftCtasPerSm * b.nsm, s)) != cudaSuccess)
        return e;
    if ((e = launch_legendre_grouped(b.d_leg, b.d_lists + b.off_list[3], b.n_list[3], b.bn, false, lg, s)) !=
        cudaSuccess)
        return e;
    return run_tc_items(b, false, s);
}

void release(sht_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    for (float2* q : b->scratch)
        if (q) cudaFree(q);
    if (b->d_leg) cudaFree(b->d_leg);
    if (b->d_fft) cudaFree(b->d_fft);
    if (b->d_lists) cudaFree(b->d_lists);
}

}  // namespace

int sht_batch_create(const sht_batch_item* items, int nitems, sht_batch** out) {
    if (!out) return bfail(SHT_EINVAL, "sht_batch_create: NULL output");
    *out = nullptr;
    if (nitems < 1 || !items) return bfail(SHT_EINVAL, "sht_batch_create: empty batch");
    int device = -1;
    for (int t = 0; t < nitems; ++t) {
        const sht_batch_item& it = items[t];
        if (!it.plan) return bfail(SHT_EINVAL, "sht_batch_create: NULL plan");
        const Plan& p = *plan_impl(it.plan);
        if (device >= 0 && p.device != device)
            return bfail(SHT_EINVAL, "sht_batch_create: plans on different devices");
        device = p.device;
        if (it.direction != SHT_SYNTHESIS && it.direction != SHT_ANALYSIS)
            return bfail(SHT_EINVAL, "sht_batch_create: direction must be SHT_SYNTHESIS or SHT_ANALYSIS");
        if (it.nlayers < 1 || it.nlayers > p.d.nlayers)
            return bfail(SHT_EINVAL, "sht_batch_create: DimensionMismatch: nlayers outside 1 .. plan nlayers");
        if (it.ldc < p.nlm || it.ldg < p.npoints)
            return bfail(SHT_EINVAL, "sht_batch_create: DimensionMismatch: leading dimension below nlm / npoints");
        if (!it.coeffs || !it.grid) return bfail(SHT_EINVAL, "sht_batch_create: NULL array");
    }
    sht_batch* b = new sht_batch();
    b->items.assign(items, items + nitems);
    b->device = device;
    DevGuard g(device);
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && nsm > 0) b->nsm = nsm;
    cudaError_t e = cudaSuccess;
    std::vector<LegView> lv(nitems);
    std::vector<FftView> fv(nitems);
    b->scratch.assign(nitems, nullptr);
    for (int t = 0; t < nitems && e == cudaSuccess; ++t) {
        const sht_batch_item& it = items[t];
        const Plan& p = *plan_impl(it.plan);
        if (p.d.precision != SHT_PREC_FP32) continue;      // runs as its own call on the plan's buffers
        e = cudaMalloc(&b->scratch[t], std::max<int64_t>(1, p.scratch_rows * 2 * it.nlayers) * sizeof(float2));
        if (e != cudaSuccess) break;
        const bool syn = it.direction == SHT_SYNTHESIS;
        lv[t] = leg_view(p, syn ? (const float2*)it.coeffs : nullptr, syn ? nullptr : (float2*)it.coeffs, it.ldc,
                         b->scratch[t], it.nlayers, !syn && (it.flags & SHT_ADD));
        fv[t] = fft_view(p, syn ? nullptr : it.grid, syn ? it.grid : nullptr, it.ldg, b->scratch[t], it.nlayers,
                         syn ? it.flags : 0u, false, false);
        b->fft_smem = std::max(b->fft_smem, p.smem_fft);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_leg, nitems * sizeof(LegView));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_leg, lv.data(), nitems * sizeof(LegView), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_fft, nitems * sizeof(FftView));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_fft, fv.data(), nitems * sizeof(FftView), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = upload_lists(*b, 64);
    if (e == cudaSuccess) e = legendre_grouped_grids(b->nsm, b->leg_grid);
    if (e != cudaSuccess) {
        release(b);
        delete b;
        return bcuda(e, "sht_batch_create");
    }
    *out = b;
    return SHT_OK;
}

int sht_batch_run(sht_batch* b, void* stream) {
    if (!b) return bfail(SHT_EINVAL, "sht_batch_run: NULL batch");
    DevGuard g(b->device);
    const cudaError_t e = run(*b, (cudaStream_t)stream);
    return e == cudaSuccess ? SHT_OK : bcuda(e, "sht_batch_run");
}

int sht_batch_run_each(sht_batch* b, void* stream) {
    if (!b) return bfail(SHT_EINVAL, "sht_batch_run_each: NULL batch");
    int rc;
    for (int pass = 0; pass < 2; ++pass)          // all syntheses, then all analyses
        for (const sht_batch_item& it : b->items) {
            if ((it.direction == SHT_SYNTHESIS) != (pass == 0)) continue;
            rc = it.direction == SHT_SYNTHESIS
                     ? sht_synthesize(it.plan, it.coeffs, it.ldc, it.grid, it.ldg, it.nlayers, it.flags, stream)
                     : sht_analyze(it.plan, it.grid, it.ldg, it.coeffs, it.ldc, it.nlayers, it.flags, stream);
            if (rc != SHT_OK) return rc;
        }
    return SHT_OK;
}

int sht_batch_capture(sht_batch* b, void* stream) {
    if (!b) return bfail(SHT_EINVAL, "sht_batch_capture: NULL batch");
    DevGuard g(b->device);
    cudaError_t e = cudaSuccess;
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) {                                     // the legacy stream cannot capture
        if (!b->capture_stream) e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
        s = b->capture_stream;
    }
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const cudaError_t er = run(*b, s);
        e = cudaStreamEndCapture(s, &graph);
        if (er != cudaSuccess) e = er;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    return e == cudaSuccess ? SHT_OK : bcuda(e, "sht_batch_capture");
}

int sht_batch_launch(sht_batch* b, void* stream) {
    if (!b) return bfail(SHT_EINVAL, "sht_batch_launch: NULL batch");
    if (!b->exec) return bfail(SHT_EINVAL, "sht_batch_launch: no captured graph (call sht_batch_capture)");
    DevGuard g(b->device);
    const cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? SHT_OK : bcuda(e, "sht_batch_launch");
}

int sht_batch_autotune(sht_batch* b, void* stream, int32_t* tile_columns) {
    if (!b) return bfail(SHT_EINVAL, "sht_batch_autotune: NULL batch");
    DevGuard g(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int best = b->bn;
    float best_ms = 1e30f;
    for (int bn : {32, 64, 128}) {
        if (e != cudaSuccess) break;
        if ((e = upload_lists(*b, bn)) != cudaSuccess) break;
        for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = run(*b, s);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) e = run(*b, s);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            best = bn;
        }
    }
    if (e == cudaSuccess) e = upload_lists(*b, best);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (b->exec) {                                // a captured graph holds the old lists
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (e != cudaSuccess) return bcuda(e, "sht_batch_autotune");
    if (tile_columns) *tile_columns = best;
    return SHT_OK;
}

int sht_batch_destroy(sht_batch* b) {
    if (!b) return SHT_OK;
    DevGuard g(b->device);
    release(b);
    delete b;
    return SHT_OK;
}
