// gpk_batch.cpp — a sweep of independent grids advanced together.
//
// A step of one grid is a sequence of small kernels separated by a few host
// round trips (candidate counts, remap passes).  For the small 2-D instances
// of a parameter sweep those round trips, not the kernels, set the time of a
// plain loop over instances.  The batch runs W worker threads; each takes
// the next instance (largest first, so the long ones start early), advances
// it on its own stream and takes the next, so up to W instances are in flight
// on the GPU at once.  Work per instance is unchanged, so results are
// bit-identical to a plain loop.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpk_batch.h"
#include "gpk_grid.h"

struct gpk_batch {
    std::vector<gpk_grid*> grids;
    std::vector<int> order;  // instance indices, most cells first
    int workers = 1;
    int device = 0;
    // the whole sweep as one graph: each instance's captured two-step graph
    // as a child node, no edges between instances
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraph_t> children;  // the instance graphs it was built from
    ~gpk_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int hw_workers() {
    const unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 8;
}

struct FirstError {
    std::mutex m;
    int code = GPK_OK;
    std::string msg;
    void set(int c, const std::string& s) {
        std::lock_guard<std::mutex> lk(m);
        if (code == GPK_OK) { code = c; msg = s; }
    }
};

// Runs fn(instance) for every instance on b->workers threads.
template <typename F>
int for_each_instance(gpk_batch* b, F fn) {
    const int n = (int)b->grids.size();
    const int w = std::max(1, std::min(b->workers, n));
    std::atomic<int> next{0};
    std::atomic<bool> stop{false};
    FirstError err;
    auto body = [&]() {
        if (cudaSetDevice(b->device) != cudaSuccess) {
            err.set(GPK_ERR_CUDA, "cudaSetDevice failed in a batch worker");
            stop = true;
            return;
        }
        while (!stop.load()) {
            const int k = next.fetch_add(1);
            if (k >= n) break;
            const int inst = b->order[k];
            const int rc = fn(inst);
            if (rc != GPK_OK) {
                err.set(rc, "instance " + std::to_string(inst) + ": " + gpk_last_error());
                stop = true;
            }
        }
    };
    if (w == 1) {
        body();
    } else {
        std::vector<std::thread> pool;
        pool.reserve(w);
        for (int t = 0; t < w; ++t) pool.emplace_back(body);
        for (auto& t : pool) t.join();
    }
    if (err.code != GPK_OK) {
        gpk_set_error("batch: " + err.msg);
        return err.code;
    }
    return GPK_OK;
}

}  // namespace

extern "C" int gpk_batch_create(int n, gpk_grid* const* grids, int workers, gpk_batch** out) {
    if (!out || !grids || n < 1) {
        gpk_set_error("batch: need n >= 1 grids and an output pointer");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    std::vector<gpk_grid*> g(grids, grids + n);
    for (int i = 0; i < n; ++i)
        if (!g[i]) {
            gpk_set_error("batch: grid " + std::to_string(i) + " is null");
            return GPK_ERR_INVALID_ARGUMENT;
        }
    std::vector<gpk_grid*> sorted(g);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) {
        gpk_set_error("batch: a grid appears twice");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    if (workers < 0) {
        gpk_set_error("batch: workers must be >= 0");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    gpk_batch* b = new gpk_batch();
    b->grids = g;
    b->order.resize(n);
    for (int i = 0; i < n; ++i) b->order[i] = i;
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int a, int c) { return g[a]->d.N > g[c]->d.N; });
    b->workers = workers ? std::min(workers, n) : std::min(hw_workers(), n);
    b->device = g[0]->device;
    *out = b;
    return GPK_OK;
}

extern "C" int gpk_batch_destroy(gpk_batch* b) {
    delete b;
    return GPK_OK;
}

extern "C" int gpk_batch_set_workers(gpk_batch* b, int workers) {
    if (!b || workers < 0) {
        gpk_set_error("batch: null handle or negative worker count");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const int n = (int)b->grids.size();
    b->workers = workers ? std::min(workers, n) : std::min(hw_workers(), n);
    return GPK_OK;
}

extern "C" int gpk_batch_workers(const gpk_batch* b, int* workers) {
    if (!b || !workers) {
        gpk_set_error("batch: null argument");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    *workers = b->workers;
    return GPK_OK;
}

extern "C" int gpk_batch_step(gpk_batch* b, int steps, double dt, double dt_cap) {
    if (!b || steps < 0) {
        gpk_set_error("batch: null handle or negative step count");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    return for_each_instance(b, [&](int i) {
        gpk_grid* G = b->grids[i];
        for (int s = 0; s < steps; ++s) {
            double used = 0;
            const int rc = gpk_grid_step(G, dt, dt_cap, &used);
            if (rc != GPK_OK) return rc;
        }
        return gpk_grid_sync(G);
    });
}

extern "C" int gpk_batch_run(gpk_batch* b, double t_end, double dt, int max_steps, int* steps_out) {
    if (!b) {
        gpk_set_error("batch: null handle");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    return for_each_instance(b, [&](int i) {
        int n = 0;
        const int rc = gpk_grid_run(b->grids[i], t_end, dt, max_steps, &n);
        if (steps_out) steps_out[i] = n;
        if (rc != GPK_OK) return rc;
        return gpk_grid_sync(b->grids[i]);
    });
}

// ---- the sweep as one captured graph -------------------------------------------
static int batch_graph_build(gpk_batch* b, double dt, double dt_cap) {
    const int n = (int)b->grids.size();
    // each instance's two-step graph, captured on its own stream (in parallel)
    GPK_TRY(for_each_instance(b, [&](int i) { return gpk_grid_graph_prepare(b->grids[i], dt, dt_cap); }));
    bool same = b->exec && (int)b->children.size() == n;
    for (int i = 0; same && i < n; ++i) same = b->children[i] == b->grids[i]->step_graph;
    if (same) return GPK_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->children.assign(n, nullptr);
    GPK_CUDA_TRY(cudaGraphCreate(&b->graph, 0));
    for (int k = 0; k < n; ++k) {
        const int i = b->order[k];
        cudaGraphNode_t node;
        GPK_CUDA_TRY(cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, b->grids[i]->step_graph));
        b->children[i] = b->grids[i]->step_graph;
    }
    GPK_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return GPK_OK;
}

extern "C" int gpk_batch_graph_stream(gpk_batch* b, void** stream) {
    if (!b || !stream) return GPK_ERR_INVALID_ARGUMENT;
    if (!b->stream) {
        if (cudaSetDevice(b->device) != cudaSuccess) return GPK_ERR_CUDA;
        GPK_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    }
    *stream = (void*)b->stream;
    return GPK_OK;
}

extern "C" int gpk_batch_step_graph(gpk_batch* b, int steps, double dt, double dt_cap) {
    if (!b || steps < 0) {
        gpk_set_error("batch: null handle or negative step count");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    if (cudaSetDevice(b->device) != cudaSuccess) {
        gpk_set_error("batch: cudaSetDevice failed");
        return GPK_ERR_CUDA;
    }
    if (!b->stream) GPK_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    int done = 0;
    bool fresh = false;
    for (gpk_grid* G : b->grids) fresh |= G->step_id == 0;
    if (steps > 0 && fresh) {
        // one ordinary step makes the buffers and settings a captured step relies on
        GPK_TRY(gpk_batch_step(b, 1, dt, dt_cap));
        ++done;
    }
    if (steps - done >= 2) {
        GPK_TRY(batch_graph_build(b, dt, dt_cap));
        for (gpk_grid* G : b->grids) GPK_CUDA_TRY(cudaStreamSynchronize(G->stream));
        for (; steps - done >= 2; done += 2) {
            GPK_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
            for (gpk_grid* G : b->grids) {
                G->step_id += 2;
                G->launches += G->graph_launches;
            }
        }
        GPK_CUDA_TRY(cudaStreamSynchronize(b->stream));
        // a device-side failure of any instance's steps
        GPK_TRY(for_each_instance(b, [&](int i) { return gpk_grid_sync(b->grids[i]); }));
    }
    if (steps - done > 0) GPK_TRY(gpk_batch_step(b, steps - done, dt, dt_cap));
    return GPK_OK;
}

extern "C" int gpk_batch_autotune_tiles(gpk_batch* b, int trial_steps, int* choice_out, int* steps_taken) {
    if (!b || trial_steps < 1) {
        gpk_set_error("batch: null handle or trial_steps < 1");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const int steps = trial_steps + (trial_steps & 1);
    auto group = [&](gpk_grid* G) {
        const int side = std::max(G->d.Nx, G->d.Ny);
        return side <= 160 ? 0 : (side <= 320 ? 1 : 2);
    };
    int choice[3] = {1, 1, 1}, taken = 0;
    if (!b->stream) {
        void* st = nullptr;
        GPK_TRY(gpk_batch_graph_stream(b, &st));
    }
    // a first call captures the graphs (and steps fresh instances once)
    GPK_TRY(gpk_batch_step_graph(b, steps, -1.0, 1e30));
    taken += steps;
    cudaEvent_t e0, e1;
    GPK_CUDA_TRY(cudaEventCreate(&e0));
    GPK_CUDA_TRY(cudaEventCreate(&e1));
    int rc = GPK_OK;
    for (int gidx = 0; gidx < 3 && rc == GPK_OK; ++gidx) {
        bool any = false;
        for (gpk_grid* G : b->grids) any |= group(G) == gidx;
        if (!any) continue;
        float best = 3.4e38f;
        int best_d = choice[gidx];
        for (int d : {1, 2, 4}) {
            for (gpk_grid* G : b->grids)
                if (group(G) == gidx) G->tile_rows_div = d;
            // capture for the new tiles outside the timed region
            rc = gpk_batch_step_graph(b, 2, -1.0, 1e30);
            taken += 2;
            if (rc != GPK_OK) break;
            cudaEventRecord(e0, b->stream);
            rc = gpk_batch_step_graph(b, steps, -1.0, 1e30);
            cudaEventRecord(e1, b->stream);
            taken += steps;
            if (rc != GPK_OK) break;
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; best_d = d; }
        }
        choice[gidx] = best_d;
        for (gpk_grid* G : b->grids)
            if (group(G) == gidx) G->tile_rows_div = best_d;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (choice_out)
        for (int k = 0; k < 3; ++k) choice_out[k] = choice[k];
    if (steps_taken) *steps_taken = taken;
    return rc;
}

extern "C" int gpk_batch_autotune(gpk_batch* b, int trial_steps, int* workers_out, int* steps_taken) {
    if (!b || trial_steps < 1) {
        gpk_set_error("batch: null handle or trial_steps < 1");
        return GPK_ERR_INVALID_ARGUMENT;
    }
    const int n = (int)b->grids.size();
    const int saved = b->workers;
    int best_w = saved, taken = 0;
    double best_t = 1e300;
    for (int w = 1; w <= std::min(n, 64); w *= 2) {
        b->workers = w;
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = gpk_batch_step(b, trial_steps, -1.0, 1e30);
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        taken += trial_steps;
        if (rc != GPK_OK) {
            b->workers = saved;
            if (steps_taken) *steps_taken = taken;
            return rc;
        }
        if (t < best_t) { best_t = t; best_w = w; }
    }
    b->workers = best_w;
    if (workers_out) *workers_out = best_w;
    if (steps_taken) *steps_taken = taken;
    return GPK_OK;
}
