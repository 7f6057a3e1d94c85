// Conjugate gradients on the device for (A^H A + lambda I) x = b, with A^H A
// an operator of this library. Vectors stay FP32 complex (the operator's
// precision); every inner product is accumulated in FP64 in a fixed order
// (per-block partial sums, then one block sums the partials by index), so a
// solve is deterministic run to run; the scalars alpha, beta and |r|^2 live
// in device memory, so an iteration launches no host synchronisation and can
// be captured in a CUDA graph. The iteration is textbook CG (Hestenes &
// Stiefel 1952):
//   q = (A^H A + lambda) p;  alpha = |r|^2 / Re<p, q>;  x += alpha p;
//   r -= alpha q;  beta = |r_new|^2 / |r|^2;  p = r + beta p.
// Re<a, b> of complex vectors is the dot product of their float arrays, so
// the kernels work on floats (four at a time).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>

#include "engine.h"
#include "mr_aha/mr_aha_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;  // 8 x 148 SMs

// scalar slots in device memory
enum { S_RR = 0, S_PQ, S_ALPHA, S_BETA, S_RR0, S_NSCAL };

struct cg_dev {
    double *scal;      // S_NSCAL scalars
    double *part;      // kMaxBlocks partial sums
    unsigned *count;   // blocks done (last-block reduction)
    int *iter;         // iterations done
    double *hist;      // |r_k|^2, k = 0 .. cap
    int cap;
};

// Block sum of v (double) into part[blockIdx.x]; returns true in every
// thread of the last block to finish, which then sees all partials.
__device__ __forceinline__ bool block_partial(double v, const cg_dev &d) {
    __shared__ double ws[kThreads / 32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < kThreads / 32 ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) {
            d.part[blockIdx.x] = s;
            __threadfence();
            const unsigned done = atomicAdd(d.count, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    return last;
}

// Sum of part[0 .. gridDim.x) in a fixed order (run by the last block).
__device__ __forceinline__ double final_sum(const cg_dev &d) {
    __shared__ double ws[kThreads / 32];
    __threadfence();
    double v = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) v += __ldcg(d.part + i);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kThreads / 32; ++w) s += ws[w];
        *d.count = 0;
    }
    return s;  // valid in thread 0
}

__device__ __forceinline__ double dot4(float4 a, float4 b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
}

// x = 0 (if zero_x), r = b - q - lambda x (q = A^H A x, or nothing if zero_x),
// p = r, |r|^2 -> S_RR, hist[0]; iteration counter reset.
__global__ void __launch_bounds__(kThreads) k_cg_init(const float4 *__restrict__ b, float4 *x,
                                                      const float4 *__restrict__ q, float4 *r,
                                                      float4 *p, int64_t n4, float lambda,
                                                      int zero_x, cg_dev d) {
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n4;
         i += (int64_t)gridDim.x * kThreads) {
        float4 v = b[i];
        if (zero_x) {
            x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            const float4 a = q[i], xi = x[i];
            v.x -= a.x + lambda * xi.x;
            v.y -= a.y + lambda * xi.y;
            v.z -= a.z + lambda * xi.z;
            v.w -= a.w + lambda * xi.w;
        }
        r[i] = v;
        p[i] = v;
        acc += dot4(v, v);
    }
    if (block_partial(acc, d)) {
        const double s = final_sum(d);
        if (threadIdx.x == 0) {
            d.scal[S_RR] = s;
            d.scal[S_RR0] = s;
            d.hist[0] = s;
            *d.iter = 0;
        }
    }
}

// q += lambda p; Re<p, q> -> S_PQ; alpha = |r|^2 / Re<p, q> (0 when the
// curvature is not positive: the iteration then leaves x unchanged).
__global__ void __launch_bounds__(kThreads) k_cg_pq(const float4 *__restrict__ p, float4 *q,
                                                    int64_t n4, float lambda, cg_dev d) {
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n4;
         i += (int64_t)gridDim.x * kThreads) {
        const float4 pi = p[i];
        float4 qi = q[i];
        if (lambda != 0.f) {
            qi.x += lambda * pi.x;
            qi.y += lambda * pi.y;
            qi.z += lambda * pi.z;
            qi.w += lambda * pi.w;
            q[i] = qi;
        }
        acc += dot4(pi, qi);
    }
    if (block_partial(acc, d)) {
        const double s = final_sum(d);
        if (threadIdx.x == 0) {
            d.scal[S_PQ] = s;
            d.scal[S_ALPHA] = s > 0.0 ? d.scal[S_RR] / s : 0.0;
        }
    }
}

// x += alpha p; r -= alpha q; |r|^2 -> S_RR, beta, hist[++iter].
__global__ void __launch_bounds__(kThreads) k_cg_xr(float4 *x, float4 *r,
                                                    const float4 *__restrict__ p,
                                                    const float4 *__restrict__ q, int64_t n4,
                                                    cg_dev d) {
    const float al = (float)d.scal[S_ALPHA];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n4;
         i += (int64_t)gridDim.x * kThreads) {
        const float4 pi = p[i], qi = q[i];
        float4 xi = x[i], ri = r[i];
        xi.x += al * pi.x;
        xi.y += al * pi.y;
        xi.z += al * pi.z;
        xi.w += al * pi.w;
        ri.x -= al * qi.x;
        ri.y -= al * qi.y;
        ri.z -= al * qi.z;
        ri.w -= al * qi.w;
        x[i] = xi;
        r[i] = ri;
        acc += dot4(ri, ri);
    }
    if (block_partial(acc, d)) {
        const double s = final_sum(d);
        if (threadIdx.x == 0) {
            const double rr = d.scal[S_RR];
            d.scal[S_BETA] = rr > 0.0 ? s / rr : 0.0;
            d.scal[S_RR] = s;
            const int it = *d.iter + 1;
            *d.iter = it;
            if (it <= d.cap) d.hist[it] = s;
        }
    }
}

// p = r + beta p
__global__ void __launch_bounds__(kThreads) k_cg_p(float4 *p, const float4 *__restrict__ r,
                                                   int64_t n4, const double *scal) {
    const float be = (float)scal[S_BETA];
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n4;
         i += (int64_t)gridDim.x * kThreads) {
        const float4 ri = r[i], pi = p[i];
        p[i] = make_float4(ri.x + be * pi.x, ri.y + be * pi.y, ri.z + be * pi.z,
                           ri.w + be * pi.w);
    }
}

}  // namespace

struct mr_b200_cg_s {
    mr_op op;
    int dev;
    cudaStream_t op_stream;  // the operator's stream (caller-visible ordering)
    cudaStream_t s;          // the solver's own stream (capturable)
    cudaEvent_t ev;
    int64_t n4;              // float4 groups (Vimg * L complex = 2 floats each)
    const float2 *b;
    float2 *x;
    float2 *r, *p, *q;
    cg_dev d;
    void *dmem;              // one allocation for scalars, partials, counters, history
    float lambda;
    int nblk;
    int use_graph;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int iters;               // iterations issued
};

static void cg_release(mr_b200_cg cg) {
    if (cg->exec) cudaGraphExecDestroy(cg->exec);
    if (cg->graph) cudaGraphDestroy(cg->graph);
    if (cg->r) cudaFree(cg->r);
    if (cg->dmem) cudaFree(cg->dmem);
    if (cg->ev) cudaEventDestroy(cg->ev);
    if (cg->s) cudaStreamDestroy(cg->s);
    cudaGetLastError();
    delete cg;
}

// Make `waiter` wait for the work issued so far on `from`.
static int cg_order(mr_b200_cg cg, cudaStream_t from, cudaStream_t waiter) {
    MR_CUDA_TRY(cudaEventRecord(cg->ev, from));
    MR_CUDA_TRY(cudaStreamWaitEvent(waiter, cg->ev, 0));
    return MR_SUCCESS;
}

// One iteration on cg->s.
static int cg_iter(mr_b200_cg cg) {
    float4 *x = reinterpret_cast<float4 *>(cg->x);
    float4 *r = reinterpret_cast<float4 *>(cg->r);
    float4 *p = reinterpret_cast<float4 *>(cg->p);
    float4 *q = reinterpret_cast<float4 *>(cg->q);
    int rc = mr_op_execute_on(cg->op, cg->p, cg->q, cg->s);
    if (rc != MR_SUCCESS) return rc;
    k_cg_pq<<<cg->nblk, kThreads, 0, cg->s>>>(p, q, cg->n4, cg->lambda, cg->d);
    MR_LAUNCH_CHECK("k_cg_pq");
    k_cg_xr<<<cg->nblk, kThreads, 0, cg->s>>>(x, r, p, q, cg->n4, cg->d);
    MR_LAUNCH_CHECK("k_cg_xr");
    k_cg_p<<<cg->nblk, kThreads, 0, cg->s>>>(p, r, cg->n4, cg->d.scal);
    MR_LAUNCH_CHECK("k_cg_p");
    return MR_SUCCESS;
}

static int cg_create_impl(mr_op op, const float2 *b, float2 *x, double lambda, int flags,
                          int max_iters, mr_b200_cg *out) {
    const mr_config *cfg = mr_op_config(op);
    const int64_t n = mr_image_size(cfg) * (int64_t)cfg->L;  // complex elements
    mr_b200_cg cg = new (std::nothrow) mr_b200_cg_s();
    if (!cg) MR_FAIL(MR_ERR_ALLOC, "mr_b200_cg_create: out of host memory");
    cg->op = op;
    cg->dev = mr_op_device(op);
    cg->op_stream = mr_op_stream(op);
    cg->b = b;
    cg->x = x;
    cg->lambda = (float)lambda;
    cg->use_graph = (flags & MR_B200_CG_GRAPH) != 0;
    cg->n4 = n / 2;  // Vimg * L * 2 floats; n is even whenever L is, else one tail pair
    if (n % 2) {
        cg_release(cg);
        MR_FAIL(MR_ERR_UNSUPPORTED,
                "mr_b200_cg_create: Vimg * L = %lld is odd (the solver works on float4 groups)",
                (long long)n);
    }
    cg->nblk = (int)std::min<int64_t>(kMaxBlocks, std::max<int64_t>(1, mr_cdiv(cg->n4, kThreads)));
    const size_t vb = (size_t)n * sizeof(float2);
    if (cudaMalloc(&cg->r, 3 * vb) != cudaSuccess) {
        cudaGetLastError();
        cg->r = nullptr;
        cg_release(cg);
        MR_FAIL(MR_ERR_ALLOC, "mr_b200_cg_create: cannot allocate 3 x %zu bytes of work vectors", vb);
    }
    cg->p = cg->r + n;
    cg->q = cg->p + n;
    cg->d.cap = max_iters;
    const size_t sb = sizeof(double) * (S_NSCAL + kMaxBlocks + max_iters + 1) + 64;
    if (cudaMalloc(&cg->dmem, sb) != cudaSuccess) {
        cudaGetLastError();
        cg->dmem = nullptr;
        cg_release(cg);
        MR_FAIL(MR_ERR_ALLOC, "mr_b200_cg_create: cannot allocate solver scalars");
    }
    double *dm = static_cast<double *>(cg->dmem);
    cg->d.scal = dm;
    cg->d.part = dm + S_NSCAL;
    cg->d.hist = cg->d.part + kMaxBlocks;
    cg->d.count = reinterpret_cast<unsigned *>(cg->d.hist + max_iters + 1);
    cg->d.iter = reinterpret_cast<int *>(cg->d.count + 4);
    if (cudaStreamCreateWithFlags(&cg->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&cg->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cg_release(cg);
        MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_create: cannot create the solver's stream");
    }
    int rc = MR_SUCCESS;
    if (cudaMemsetAsync(cg->dmem, 0, sb, cg->s) != cudaSuccess) rc = MR_ERR_CUDA;
    // the caller's b and x were written on the operator's stream
    if (rc == MR_SUCCESS) rc = cg_order(cg, cg->op_stream, cg->s);
    const int zero_x = (flags & MR_B200_CG_ZERO_X) != 0;
    if (rc == MR_SUCCESS && !zero_x) rc = mr_op_execute_on(op, x, cg->q, cg->s);
    if (rc == MR_SUCCESS) {
        k_cg_init<<<cg->nblk, kThreads, 0, cg->s>>>(
            reinterpret_cast<const float4 *>(b), reinterpret_cast<float4 *>(x),
            reinterpret_cast<const float4 *>(cg->q), reinterpret_cast<float4 *>(cg->r),
            reinterpret_cast<float4 *>(cg->p), cg->n4, cg->lambda, zero_x, cg->d);
        if (cudaGetLastError() != cudaSuccess) rc = MR_ERR_CUDA;
    }
    if (rc == MR_SUCCESS) rc = cg_order(cg, cg->s, cg->op_stream);
    if (rc != MR_SUCCESS) {
        cudaStreamSynchronize(cg->s);
        cg_release(cg);
        if (rc == MR_ERR_CUDA) MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_create: initialisation failed");
        return rc;
    }
    *out = cg;
    return MR_SUCCESS;
}

extern "C" int mr_b200_cg_create(mr_op op, const mr_complex *d_b, mr_complex *d_x, double lambda,
                                 int flags, int max_iters, mr_b200_cg *cg) {
    mr_clear_error();
    MR_REQUIRE(cg != nullptr, "mr_b200_cg_create: cg is NULL");
    *cg = nullptr;
    MR_REQUIRE(op != nullptr, "mr_b200_cg_create: op is NULL");
    MR_REQUIRE(d_b != nullptr && d_x != nullptr, "mr_b200_cg_create: b or x is NULL");
    MR_REQUIRE((const void *)d_b != (const void *)d_x, "mr_b200_cg_create: x must not alias b");
    MR_REQUIRE(((uintptr_t)d_b | (uintptr_t)d_x) % 16 == 0,
               "mr_b200_cg_create: b and x must be 16-byte aligned");
    MR_REQUIRE(max_iters >= 0, "mr_b200_cg_create: max_iters = %d < 0", max_iters);
    MR_REQUIRE(lambda >= 0.0, "mr_b200_cg_create: lambda = %g < 0", lambda);
    MR_REQUIRE((flags & ~(MR_B200_CG_ZERO_X | MR_B200_CG_GRAPH)) == 0,
               "mr_b200_cg_create: unknown flags 0x%x", flags);
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    const int dev = mr_op_device(op);
    if (prev != dev) MR_CUDA_TRY(cudaSetDevice(dev));
    const int rc = cg_create_impl(op, reinterpret_cast<const float2 *>(d_b),
                                  reinterpret_cast<float2 *>(d_x), lambda, flags, max_iters, cg);
    if (prev != dev) cudaSetDevice(prev);
    return rc;
}

static int cg_step_impl(mr_b200_cg cg, int n_iter) {
    int rc = cg_order(cg, cg->op_stream, cg->s);
    if (rc != MR_SUCCESS) return rc;
    if (cg->use_graph && n_iter > 0 && !cg->exec) {
        // one iteration eagerly (first launches set kernel attributes), then
        // capture one on the solver's stream, replayed below
        rc = cg_iter(cg);
        if (rc != MR_SUCCESS) return rc;
        ++cg->iters;
        --n_iter;
        MR_CUDA_TRY(cudaStreamBeginCapture(cg->s, cudaStreamCaptureModeThreadLocal));
        rc = cg_iter(cg);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cg->s, &g);
        if (rc != MR_SUCCESS) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) {
            cudaGetLastError();
            MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_step: graph capture failed: %s",
                    cudaGetErrorString(ce));
        }
        cg->graph = g;
        if (cudaGraphInstantiate(&cg->exec, g, 0) != cudaSuccess) {
            cudaGetLastError();
            cg->exec = nullptr;
            MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_step: graph instantiation failed");
        }
    }
    for (int i = 0; i < n_iter; ++i) {
        if (cg->exec) {
            MR_CUDA_TRY(cudaGraphLaunch(cg->exec, cg->s));
        } else {
            rc = cg_iter(cg);
            if (rc != MR_SUCCESS) return rc;
        }
        ++cg->iters;
    }
    return cg_order(cg, cg->s, cg->op_stream);
}

extern "C" int mr_b200_cg_step(mr_b200_cg cg, int n_iter) {
    mr_clear_error();
    MR_REQUIRE(cg != nullptr, "mr_b200_cg_step: cg is NULL");
    MR_REQUIRE(n_iter >= 0, "mr_b200_cg_step: n_iter = %d < 0", n_iter);
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != cg->dev) MR_CUDA_TRY(cudaSetDevice(cg->dev));
    const int rc = cg_step_impl(cg, n_iter);
    if (prev != cg->dev) cudaSetDevice(prev);
    return rc;
}

extern "C" int mr_b200_cg_busy(mr_b200_cg cg, int *busy) {
    mr_clear_error();
    MR_REQUIRE(cg != nullptr && busy != nullptr, "mr_b200_cg_busy: NULL argument");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != cg->dev) MR_CUDA_TRY(cudaSetDevice(cg->dev));
    const cudaError_t e = cudaStreamQuery(cg->s);
    if (prev != cg->dev) cudaSetDevice(prev);
    if (e == cudaSuccess) {
        *busy = 0;
    } else if (e == cudaErrorNotReady) {
        cudaGetLastError();
        *busy = 1;
    } else {
        cudaGetLastError();
        MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_busy: %s", cudaGetErrorString(e));
    }
    return MR_SUCCESS;
}

extern "C" int mr_b200_cg_iterations(mr_b200_cg cg, int *n) {
    mr_clear_error();
    MR_REQUIRE(cg != nullptr && n != nullptr, "mr_b200_cg_iterations: NULL argument");
    *n = cg->iters;
    return MR_SUCCESS;
}

extern "C" int mr_b200_cg_residuals(mr_b200_cg cg, double *rr, int max, int *n) {
    mr_clear_error();
    MR_REQUIRE(cg != nullptr, "mr_b200_cg_residuals: cg is NULL");
    MR_REQUIRE(n != nullptr, "mr_b200_cg_residuals: n is NULL");
    MR_REQUIRE(rr != nullptr || max == 0, "mr_b200_cg_residuals: rr is NULL");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != cg->dev) MR_CUDA_TRY(cudaSetDevice(cg->dev));
    const int have = std::min(cg->iters, cg->d.cap) + 1;
    const int k = std::min(have, max);
    cudaError_t ce = cudaStreamSynchronize(cg->s);
    if (ce == cudaSuccess && k > 0)
        ce = cudaMemcpy(rr, cg->d.hist, sizeof(double) * k, cudaMemcpyDeviceToHost);
    if (prev != cg->dev) cudaSetDevice(prev);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        MR_FAIL(MR_ERR_CUDA, "mr_b200_cg_residuals: %s", cudaGetErrorString(ce));
    }
    *n = have;
    return MR_SUCCESS;
}

extern "C" int mr_b200_cg_destroy(mr_b200_cg cg) {
    mr_clear_error();
    if (!cg) return MR_SUCCESS;
    int prev = 0;
    const cudaError_t ce = cudaGetDevice(&prev);
    cudaSetDevice(cg->dev);
    cudaStreamSynchronize(cg->s);
    cg_release(cg);
    if (ce == cudaSuccess) cudaSetDevice(prev);
    return MR_SUCCESS;
}

extern "C" int mr_b200_cg_solve(mr_op op, const mr_complex *d_b, mr_complex *d_x, int n_iter,
                                double lambda, int flags, double *rr) {
    mr_b200_cg cg = nullptr;
    int rc = mr_b200_cg_create(op, d_b, d_x, lambda, flags, n_iter, &cg);
    if (rc != MR_SUCCESS) return rc;
    rc = mr_b200_cg_step(cg, n_iter);
    if (rc == MR_SUCCESS && rr) {
        int n = 0;
        rc = mr_b200_cg_residuals(cg, rr, n_iter + 1, &n);
    }
    if (rc != MR_SUCCESS) {
        // keep the first error's message
        char msg[512];
        std::strncpy(msg, mr_last_error(), sizeof(msg) - 1);
        msg[sizeof(msg) - 1] = 0;
        mr_b200_cg_destroy(cg);
        mr_set_error("%s", msg);
        return rc;
    }
    return mr_b200_cg_destroy(cg);
}
