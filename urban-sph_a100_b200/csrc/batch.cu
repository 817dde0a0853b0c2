// Ensembles of independent ISPH cases of uneven size on one GPU.
//
// Every case is an ordinary context on its own non-blocking stream.  A pool of
// host workers takes cases from a queue ordered largest first (LPT) and steps
// each one; the GPU runs the kernels of all streams side by side, so cases
// of 20k-200k particles, each too small to fill 148 SMs, fill the device
// together.  The number of workers, i.e. how many cases are in flight at
// once, is chosen by sph_batch_autotune from timed probe steps;
// sph_batch_autotune_shapes then also picks the thread-block size of the
// per-step pair passes (128, 64 or 32 threads: small cases fill the 148 SMs
// with more, smaller blocks).
//
// With ppe_refinement = 4 each case's pressure solve is one CUDA graph whose
// conditional nodes take the convergence decisions on the device (ppe.cu),
// and sph_step reads a case's statistics once, after its last step: a
// worker queues all the steps of its case without waiting on the GPU.
// Without it the Krylov solver tests convergence on the host every few
// iterations, the iterations between two tests being one graph.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "ctx.cuh"

struct sph_batch {
    int device = 0;
    int precision = 0;
    int workers = 0;   // 0: one per case
    std::vector<sph_ctx *> ctx;
    std::vector<cudaStream_t> streams;
    std::vector<int64_t> n;
    std::vector<int> order;   // case indices, largest first
};

#define SPH_TRY_BATCH(x) do { const int s_ = (x); if (s_ < 0) return s_; } while (0)

namespace {

int run(sph_batch *b, int nsteps, int workers, sph_ppe_stats *stats) {
    const int nc = (int)b->ctx.size();
    const int W = std::max(1, std::min(workers > 0 ? workers : nc, nc));
    std::atomic<int> next(0);
    std::vector<int> status(nc, SPH_OK);
    std::vector<sph_ppe_stats> last(nc);
    auto worker = [&]() {
        cudaSetDevice(b->device);
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= nc) break;
            const int k = b->order[q];
            status[k] = sph_step(b->ctx[k], nsteps, &last[k]);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < W; ++w) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    int worst = SPH_OK;
    for (int k = 0; k < nc; ++k) {
        if (stats) stats[k] = last[k];
        if (status[k] < 0) worst = std::min(worst, status[k]);
        else if (worst >= 0) worst = std::max(worst, status[k]);
    }
    return worst;
}

}  // namespace

extern "C" {

int sph_batch_create(int ncase, const sph_params *params, const sph_part1 *const *P1, const int32_t *n, int precision,
                     int device, sph_batch **out) {
    using namespace sph;
    if (!out || ncase <= 0 || !params || !P1 || !n) return SPH_ERR_BAD_ARG;
    *out = nullptr;
    SPH_CUDA_TRY(cudaSetDevice(device));
    sph_batch *b = new (std::nothrow) sph_batch();
    if (!b) return SPH_ERR_OUT_OF_MEMORY;
    b->device = device;
    b->precision = precision;
    for (int k = 0; k < ncase; ++k) {
        cudaStream_t s = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) { set_cuda_error(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__); sph_batch_destroy(b); return SPH_ERR_CUDA; }
        b->streams.push_back(s);
        sph_ctx *c = nullptr;
        int st = sph_create(&params[k], precision, device, s, &c);
        if (st == SPH_OK) {
            b->ctx.push_back(c);
            st = sph_upload(c, P1[k], nullptr, n[k]);
        }
        if (st < 0) { sph_batch_destroy(b); return st; }
        b->n.push_back(n[k]);
    }
    b->order.resize(ncase);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) { return b->n[a] > b->n[c]; });
    *out = b;
    return SPH_OK;
}

void sph_batch_destroy(sph_batch *b) {
    if (!b) return;
    for (sph_ctx *c : b->ctx) sph_destroy(c);
    for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
    delete b;
}

int sph_batch_set_workers(sph_batch *b, int workers) {
    if (!b || workers < 0) return SPH_ERR_BAD_ARG;
    b->workers = workers;
    return SPH_OK;
}

int sph_batch_step(sph_batch *b, int nsteps, sph_ppe_stats *stats) {
    if (!b || nsteps < 0) return SPH_ERR_BAD_ARG;
    return run(b, nsteps, b->workers, stats);
}

int sph_batch_autotune(sph_batch *b, int probe_steps, int *workers, double *ms_per_step) {
    if (!b || probe_steps <= 0) return SPH_ERR_BAD_ARG;
    const int nc = (int)b->ctx.size();
    std::vector<int> cand;
    for (int w = 1; w < nc; w *= 2) cand.push_back(w);
    cand.push_back(nc);
    int best = nc;
    double best_ms = 1e300;
    for (int w : cand) {
        for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
        const auto t0 = std::chrono::steady_clock::now();
        const int st = run(b, probe_steps, w, nullptr);
        for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (st < 0) return st;
        if (ms < best_ms) { best_ms = ms; best = w; }
    }
    b->workers = best;
    if (workers) *workers = best;
    if (ms_per_step) *ms_per_step = best_ms / probe_steps;
    return SPH_OK;
}

int sph_batch_autotune_shapes(sph_batch *b, int probe_steps, int *workers, int *pair_block, double *ms_per_step) {
    if (!b || probe_steps <= 0) return SPH_ERR_BAD_ARG;
    int w = 0;
    double best_ms = 0;
    SPH_TRY_BATCH(sph_batch_autotune(b, probe_steps, &w, &best_ms));
    int best = 128;
    for (int threads : {64, 32}) {
        for (sph_ctx *c : b->ctx) SPH_TRY_BATCH(sph_set_pair_block(c, threads));
        for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
        const auto t0 = std::chrono::steady_clock::now();
        const int st = run(b, probe_steps, b->workers, nullptr);
        for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (st < 0) return st;
        if (ms < best_ms) { best_ms = ms; best = threads; }
    }
    for (sph_ctx *c : b->ctx) SPH_TRY_BATCH(sph_set_pair_block(c, best));
    if (workers) *workers = w;
    if (pair_block) *pair_block = best;
    if (ms_per_step) *ms_per_step = best_ms / probe_steps;
    return SPH_OK;
}

int sph_batch_case(sph_batch *b, int k, sph_ctx **ctx) {
    if (!b || !ctx || k < 0 || k >= (int)b->ctx.size()) return SPH_ERR_BAD_ARG;
    *ctx = b->ctx[k];
    return SPH_OK;
}

int64_t sph_batch_particles(sph_batch *b) {
    if (!b) return 0;
    int64_t s = 0;
    for (int64_t v : b->n) s += v;
    return s;
}

}  // extern "C"
