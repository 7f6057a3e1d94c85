// Batched apply of many independent operators of uneven size (no reference
// counterpart: the reference applies one operator per call). Each operator's
// passes run on one of a few worker streams, so small operators overlap on
// the GPU with large ones; operators are dealt to the streams largest first
// onto the least-loaded stream (work estimated as upsampled grid x coils x
// rank). With MR_B200_BATCH_GRAPH the whole batch -- fork, every operator's
// launches, join -- is captured once as one CUDA graph and replayed with a
// single launch; the graph is captured again when the array pointers change.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "engine.h"
#include "mr_aha/mr_aha_b200.h"

struct mr_b200_batch_s {
    std::vector<mr_op> ops;
    std::vector<int> lane;           // worker stream of each operator
    std::vector<cudaStream_t> ws;    // worker streams
    std::vector<cudaEvent_t> ev;     // one per worker (join) + fork
    cudaStream_t origin;             // capture / launch stream
    int dev;
    int flags;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    std::vector<const void *> gx;    // pointers baked into the graph
    std::vector<void *> gout;
};

static void batch_release(mr_b200_batch b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : b->ws)
        if (s) cudaStreamDestroy(s);
    if (b->origin) cudaStreamDestroy(b->origin);
    cudaGetLastError();
    delete b;
}

static double op_work(mr_op op) {
    const mr_config *c = mr_op_config(op);
    return (double)mr_pad_size(c) * c->n_coils * c->L;
}

static int batch_create_impl(const mr_op *ops, int n, int n_streams, int flags,
                             mr_b200_batch *out) {
    mr_b200_batch b = new (std::nothrow) mr_b200_batch_s();
    if (!b) MR_FAIL(MR_ERR_ALLOC, "mr_b200_batch_create: out of host memory");
    b->ops.assign(ops, ops + n);
    b->dev = mr_op_device(ops[0]);
    b->flags = flags;
    const int ns = std::max(1, std::min(n_streams, n));
    b->ws.assign(ns, nullptr);
    b->ev.assign(ns + 1, nullptr);
    bool ok = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; ok && i < ns; ++i)
        ok = cudaStreamCreateWithFlags(&b->ws[i], cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; ok && i <= ns; ++i)
        ok = cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        batch_release(b);
        MR_FAIL(MR_ERR_CUDA, "mr_b200_batch_create: cannot create streams / events");
    }
    // largest first onto the least-loaded worker
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return op_work(ops[a]) > op_work(ops[c]); });
    std::vector<double> load(ns, 0.0);
    b->lane.assign(n, 0);
    for (int i : order) {
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->lane[i] = w;
        load[w] += op_work(ops[i]);
    }
    if (flags & MR_B200_BATCH_TUNE) {
        // one tuning per distinct geometry (later ones start from it)
        std::map<std::string, bool> done;
        for (int i : order) {
            const mr_config *c = mr_op_config(ops[i]);
            char key[160];
            std::snprintf(key, sizeof(key), "%d %lld %lld %lld %d %d %d", c->traj_type,
                          (long long)c->n_dim[0], (long long)c->n_dim[1], (long long)c->n_dim[2],
                          c->L, c->n_coils, c->is_masked);
            if (done.count(key)) continue;
            done[key] = true;
            const int rc = mr_b200_op_autotune(ops[i], 2, nullptr);
            if (rc != MR_SUCCESS) {
                batch_release(b);
                return rc;
            }
        }
    }
    *out = b;
    return MR_SUCCESS;
}

extern "C" int mr_b200_batch_create(const mr_op *ops, int n_ops, int n_streams, int flags,
                                    mr_b200_batch *batch) {
    mr_clear_error();
    MR_REQUIRE(batch != nullptr, "mr_b200_batch_create: batch is NULL");
    *batch = nullptr;
    MR_REQUIRE(ops != nullptr && n_ops >= 1, "mr_b200_batch_create: no operators");
    MR_REQUIRE(n_streams >= 1 && n_streams <= 64, "mr_b200_batch_create: n_streams = %d",
               n_streams);
    MR_REQUIRE((flags & ~(MR_B200_BATCH_GRAPH | MR_B200_BATCH_TUNE)) == 0,
               "mr_b200_batch_create: unknown flags 0x%x", flags);
    for (int i = 0; i < n_ops; ++i) {
        MR_REQUIRE(ops[i] != nullptr, "mr_b200_batch_create: ops[%d] is NULL", i);
        MR_REQUIRE(mr_op_device(ops[i]) == mr_op_device(ops[0]),
                   "mr_b200_batch_create: ops[%d] is on another device", i);
        for (int j = 0; j < i; ++j)
            MR_REQUIRE(ops[j] != ops[i],
                       "mr_b200_batch_create: ops[%d] repeats ops[%d] (its work buffers would "
                       "be used twice at once)", i, j);
    }
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    const int dev = mr_op_device(ops[0]);
    if (prev != dev) MR_CUDA_TRY(cudaSetDevice(dev));
    const int rc = batch_create_impl(ops, n_ops, n_streams, flags, batch);
    if (prev != dev) cudaSetDevice(prev);
    return rc;
}

// Fork from b->origin, every operator on its worker, join back to origin.
static int batch_issue(mr_b200_batch b, const mr_complex *const *x, mr_complex *const *y) {
    const int ns = (int)b->ws.size();
    cudaEvent_t fork = b->ev[ns];
    MR_CUDA_TRY(cudaEventRecord(fork, b->origin));
    for (int w = 0; w < ns; ++w) MR_CUDA_TRY(cudaStreamWaitEvent(b->ws[w], fork, 0));
    for (size_t i = 0; i < b->ops.size(); ++i) {
        const int rc = mr_op_execute_on(b->ops[i], reinterpret_cast<const float2 *>(x[i]),
                                        reinterpret_cast<float2 *>(y[i]), b->ws[b->lane[i]]);
        if (rc != MR_SUCCESS) return rc;
    }
    for (int w = 0; w < ns; ++w) {
        MR_CUDA_TRY(cudaEventRecord(b->ev[w], b->ws[w]));
        MR_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->ev[w], 0));
    }
    return MR_SUCCESS;
}

static int batch_execute_impl(mr_b200_batch b, const mr_complex *const *x,
                              mr_complex *const *y, cudaStream_t caller) {
    const size_t n = b->ops.size();
    const int ns = (int)b->ws.size();
    // origin waits for the caller's earlier work
    MR_CUDA_TRY(cudaEventRecord(b->ev[ns], caller));
    MR_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->ev[ns], 0));
    int rc = MR_SUCCESS;
    if (b->flags & MR_B200_BATCH_GRAPH) {
        bool same = b->exec && b->gx.size() == n;
        for (size_t i = 0; same && i < n; ++i)
            same = b->gx[i] == (const void *)x[i] && b->gout[i] == (void *)y[i];
        if (!same) {
            if (b->exec) cudaGraphExecDestroy(b->exec);
            if (b->graph) cudaGraphDestroy(b->graph);
            b->exec = nullptr;
            b->graph = nullptr;
            MR_CUDA_TRY(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
            rc = batch_issue(b, x, y);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->origin, &g);
            if (rc != MR_SUCCESS) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ce != cudaSuccess || cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
                cudaGetLastError();
                if (g) cudaGraphDestroy(g);
                b->exec = nullptr;
                MR_FAIL(MR_ERR_CUDA, "mr_b200_batch_execute: graph capture failed");
            }
            b->graph = g;
            b->gx.assign(x, x + n);
            b->gout.assign(y, y + n);
        }
        MR_CUDA_TRY(cudaGraphLaunch(b->exec, b->origin));
    } else {
        rc = batch_issue(b, x, y);
        if (rc != MR_SUCCESS) return rc;
    }
    // the caller's later work waits for the batch
    MR_CUDA_TRY(cudaEventRecord(b->ev[ns], b->origin));
    MR_CUDA_TRY(cudaStreamWaitEvent(caller, b->ev[ns], 0));
    return MR_SUCCESS;
}

extern "C" int mr_b200_batch_execute(mr_b200_batch b, const mr_complex *const *d_x,
                                     mr_complex *const *d_out, void *stream) {
    mr_clear_error();
    MR_REQUIRE(b != nullptr, "mr_b200_batch_execute: batch is NULL");
    MR_REQUIRE(d_x != nullptr && d_out != nullptr, "mr_b200_batch_execute: NULL array list");
    for (size_t i = 0; i < b->ops.size(); ++i) {
        MR_REQUIRE(d_x[i] != nullptr && d_out[i] != nullptr,
                   "mr_b200_batch_execute: array %zu is NULL", i);
        MR_REQUIRE((const void *)d_x[i] != (const void *)d_out[i],
                   "mr_b200_batch_execute: out[%zu] must not alias x[%zu]", i, i);
    }
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != b->dev) MR_CUDA_TRY(cudaSetDevice(b->dev));
    const int rc = batch_execute_impl(b, d_x, d_out, (cudaStream_t)stream);
    if (prev != b->dev) cudaSetDevice(prev);
    return rc;
}

extern "C" int mr_b200_batch_destroy(mr_b200_batch b) {
    mr_clear_error();
    if (!b) return MR_SUCCESS;
    int prev = 0;
    const cudaError_t ce = cudaGetDevice(&prev);
    cudaSetDevice(b->dev);
    cudaStreamSynchronize(b->origin);
    for (cudaStream_t s : b->ws) cudaStreamSynchronize(s);
    batch_release(b);
    if (ce == cudaSuccess) cudaSetDevice(prev);
    return MR_SUCCESS;
}
