// Batched Richardson-Lucy: many independent problems (the uneven tiles of a
// large volume, whole small volumes), each with its own convolution plan, run
// as one CUDA graph.
//
// The reference solves tiles one after another (tile_processing.py:226-288,
// one richardson_lucy_with_operator call per tile).  Here the iterations of
// every problem are recorded once into a CUDA graph: the capture forks the
// problems over internal streams (balanced by FFT canvas volume), so a replay
// is one launch whose independent branches fill the GPU together, small
// problems included, with no per-kernel host launch cost.  A graph holds K
// iterations of all problems; a run of n iterations replays it n / K times
// (plus one graph for the remainder).  Graphs are cached per K.
//
// Capture needs a stream other than the legacy default stream, and the
// problems' plans must be distinct (a plan's scratch spectra serve one
// problem at a time): the batch owns an origin stream, joined to the caller's
// stream by events before and after.
#include <algorithm>
#include <map>
#include <new>
#include <vector>

#include "conv_impl.cuh"

struct decon_batch {
    int device = 0;
    int n = 0;
    std::vector<decon_conv*> plans;
    std::vector<const float*> obs;
    std::vector<float> bg;
    std::vector<float*> x, sens, ratio;
    std::vector<int> lane;  // internal stream of each problem
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joins;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::map<int, std::pair<cudaGraphExec_t, int64_t>> graphs;  // K -> (graph, kernel nodes)
};

namespace dk {

static void batch_free(decon_batch* b) {
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.second.first);
    b->graphs.clear();
    for (auto e : b->joins) cudaEventDestroy(e);
    for (auto s : b->streams) cudaStreamDestroy(s);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->origin) cudaStreamDestroy(b->origin);
}

// Record K iterations of every problem into a graph.  On failure the
// capture is ended (the origin stream is usable again) and the error kept.
static int batch_capture(decon_batch* b, int K, cudaGraphExec_t* exec, int64_t* nodes) {
    const int64_t before = decon_launch_count();
    DK_CUDA(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    int st = DECON_OK;
    cudaError_t e = cudaEventRecord(b->fork, b->origin);
    for (size_t i = 0; e == cudaSuccess && i < b->streams.size(); ++i)
        e = cudaStreamWaitEvent(b->streams[i], b->fork, 0);
    if (e != cudaSuccess) st = fail(DECON_ERR_CUDA, "batch fork failed: %s", cudaGetErrorString(e));
    for (int k = 0; st == DECON_OK && k < K; ++k)
        for (int i = 0; st == DECON_OK && i < b->n; ++i)
            st = decon_rl_iteration(b->plans[i], b->obs[i], b->bg[i], b->sens[i], b->x[i], b->ratio[i],
                                    nullptr, (void*)b->streams[b->lane[i]]);
    for (size_t i = 0; st == DECON_OK && i < b->streams.size(); ++i) {
        e = cudaEventRecord(b->joins[i], b->streams[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->origin, b->joins[i], 0);
        if (e != cudaSuccess) st = fail(DECON_ERR_CUDA, "batch join failed: %s", cudaGetErrorString(e));
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(b->origin, &graph);
    if (st != DECON_OK) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return st;
    }
    if (e != cudaSuccess) return fail(DECON_ERR_CUDA, "batch capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(DECON_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    *nodes = decon_launch_count() - before;
    count_launches(-*nodes);  // recorded, not launched; replays count them
    return DECON_OK;
}

}  // namespace dk

using namespace dk;

extern "C" {

int decon_rl_run(decon_conv* p, const float* observed, float background, const float* sens, float* x,
                 float* ratio, int iterations, void* stream) {
    if (iterations < 0) return fail(DECON_ERR_VALUE, "iterations must be >= 0");
    for (int k = 0; k < iterations; ++k)
        DK_TRY(decon_rl_iteration(p, observed, background, sens, x, ratio, nullptr, stream));
    return DECON_OK;
}

int decon_batch_rl_create(int n, decon_conv* const* plans, const float* const* observed,
                          const float* background, float* const* x, float* const* sens,
                          float* const* ratio, int nstreams, decon_batch** out) {
    if (!out || !plans || !observed || !background || !x || !sens || !ratio)
        return fail(DECON_ERR_NULL, "decon_batch_rl_create: null pointer");
    *out = nullptr;
    if (n < 1) return fail(DECON_ERR_VALUE, "a batch needs at least one problem");
    if (nstreams < 1) return fail(DECON_ERR_VALUE, "nstreams must be >= 1");
    for (int i = 0; i < n; ++i) {
        if (!plans[i] || !observed[i] || !x[i] || !sens[i] || !ratio[i])
            return fail(DECON_ERR_NULL, "decon_batch_rl_create: null pointer in problem %d", i);
        for (int j = 0; j < i; ++j)
            if (plans[j] == plans[i])
                return fail(DECON_ERR_VALUE, "problems %d and %d share a plan; each needs its own", j, i);
    }
    decon_batch* b = new (std::nothrow) decon_batch();
    if (!b) return fail(DECON_ERR_OOM, "host allocation failed");
    cudaGetDevice(&b->device);
    b->n = n;
    b->plans.assign(plans, plans + n);
    b->obs.assign(observed, observed + n);
    b->bg.assign(background, background + n);
    b->x.assign(x, x + n);
    b->sens.assign(sens, sens + n);
    b->ratio.assign(ratio, ratio + n);
    const int ns = std::min(nstreams, n);
    // largest canvases first onto the least-loaded stream
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    auto work = [&](int i) { return (double)plans[i]->F[0] * plans[i]->F[1] * plans[i]->F[2]; };
    std::sort(order.begin(), order.end(), [&](int a, int c) { return work(a) > work(c); });
    std::vector<double> load(ns, 0.0);
    b->lane.assign(n, 0);
    for (int i : order) {
        const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->lane[i] = s;
        load[s] += work(i);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    for (int s = 0; e == cudaSuccess && s < ns; ++s) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) b->streams.push_back(st);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->joins.push_back(ev);
    }
    if (e != cudaSuccess) {
        batch_free(b);
        delete b;
        return fail(DECON_ERR_CUDA, "batch streams: %s", cudaGetErrorString(e));
    }
    *out = b;
    return DECON_OK;
}

int decon_batch_rl_setup(decon_batch* b, const float* const* x_init, void* stream) {
    if (!b) return fail(DECON_ERR_NULL, "null batch");
    for (int i = 0; i < b->n; ++i)
        DK_TRY(decon_rl_setup(b->plans[i], b->obs[i], b->bg[i], x_init ? x_init[i] : nullptr, b->x[i],
                              b->sens[i], stream));
    return DECON_OK;
}

int decon_batch_rl_run(decon_batch* b, int iterations, int iters_per_graph, void* stream) {
    if (!b) return fail(DECON_ERR_NULL, "null batch");
    if (iterations < 0 || iters_per_graph < 1) return fail(DECON_ERR_VALUE, "bad iteration counts");
    if (iterations == 0) return DECON_OK;
    const cudaStream_t caller = as_stream(stream);
    const int K = std::min(iters_per_graph, iterations);
    const int reps = iterations / K, rem = iterations % K;
    for (int k : {K, rem}) {
        if (k == 0 || b->graphs.count(k)) continue;
        cudaGraphExec_t exec = nullptr;
        int64_t nodes = 0;
        DK_TRY(batch_capture(b, k, &exec, &nodes));
        b->graphs[k] = {exec, nodes};
    }
    DK_CUDA(cudaEventRecord(b->fork, caller));
    DK_CUDA(cudaStreamWaitEvent(b->origin, b->fork, 0));
    for (int r = 0; r < reps; ++r) {
        DK_CUDA(cudaGraphLaunch(b->graphs[K].first, b->origin));
        count_launches(b->graphs[K].second);
    }
    if (rem) {
        DK_CUDA(cudaGraphLaunch(b->graphs[rem].first, b->origin));
        count_launches(b->graphs[rem].second);
    }
    DK_CUDA(cudaEventRecord(b->done, b->origin));
    DK_CUDA(cudaStreamWaitEvent(caller, b->done, 0));
    return DECON_OK;
}

int decon_batch_rl_predict(decon_batch* b, float* const* pred, void* stream) {
    if (!b || !pred) return fail(DECON_ERR_NULL, "null pointer");
    for (int i = 0; i < b->n; ++i)
        DK_TRY(decon_rl_predict(b->plans[i], b->obs[i], b->bg[i], b->x[i], pred[i], nullptr, stream));
    return DECON_OK;
}

int decon_batch_graph_nodes(const decon_batch* b, int iters_per_graph, int64_t* kernels) {
    if (!b || !kernels) return fail(DECON_ERR_NULL, "null pointer");
    auto it = b->graphs.find(iters_per_graph);
    *kernels = it == b->graphs.end() ? 0 : it->second.second;
    return DECON_OK;
}

int decon_batch_destroy(decon_batch* b) {
    if (!b) return DECON_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    cudaStreamSynchronize(b->origin);
    batch_free(b);
    if (cur != b->device) cudaSetDevice(cur);
    delete b;
    return DECON_OK;
}

}  // extern "C"
