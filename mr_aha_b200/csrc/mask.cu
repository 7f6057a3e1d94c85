// Automatic k-space mask, mr_calc_mask (reference src/cuda/mr_calc_mask.cu).
//
// Every sample is mapped to its nearest point of the centred upsampled grid,
// rint(k * float(M / 2 pi)) + M / 2 (mod M) per transformed axis, computed in
// single precision exactly as the reference does (mr_calc_mask.cu:63-90) so
// that the retained set is bit-identical; the marks are dilated by a
// periodic (2r+1)^d box (one separable max pass per axis, :107-130); the
// retained linear indices are compacted in ascending order; for a stack the
// in-plane set is repeated over every kz plane (:144-152).
#include "engine.h"

#include <algorithm>
#include <vector>

namespace {

constexpr int kBlk = 1024;

__global__ void k_mark(unsigned char *marks, const float *__restrict__ traj, int64_t ns,
                       int ndim, int m0, int m1, int m2, float s0, float s1, float s2) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= ns) return;
    const int m[3] = {m0, m1, m2};
    const float sc[3] = {s0, s1, s2};
    int64_t idx = 0, stride = 1;
    for (int a = 0; a < ndim; ++a) {
        int64_t i = (int64_t)rintf(traj[t + ns * a] * sc[a]) + m[a] / 2;
        i %= m[a];
        if (i < 0) i += m[a];
        idx += i * stride;
        stride *= m[a];
    }
    marks[idx] = 1;
}

__global__ void k_dilate(unsigned char *out, const unsigned char *__restrict__ in, int64_t n,
                         int m, int64_t stride, int r) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)((t / stride) % m);
    const int64_t base = t - (int64_t)i * stride;
    unsigned char v = in[t];
    for (int d = -r; d <= r && !v; ++d) {
        int j = (i + d) % m;
        if (j < 0) j += m;
        v = in[base + (int64_t)j * stride];
    }
    out[t] = v;
}

__global__ void k_count(int *counts, const unsigned char *__restrict__ marks, int64_t n) {
    int64_t base = (int64_t)blockIdx.x * kBlk;
    int c = 0;
    for (int k = threadIdx.x; k < kBlk; k += blockDim.x) {
        const int64_t i = base + k;
        if (i < n && marks[i]) ++c;
    }
    // block reduction
    __shared__ int red[1024 / 32];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += red[w];
        counts[blockIdx.x] = s;
    }
}

// One thread per element of the block's 1024-element range, in order.
__global__ void __launch_bounds__(1024) k_compact(int64_t *out, const unsigned char *__restrict__ marks,
                                                  int64_t n, const int64_t *__restrict__ offs) {
    __shared__ int wsum[32];
    const int64_t i = (int64_t)blockIdx.x * kBlk + threadIdx.x;
    const bool f = i < n && marks[i];
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int k = 0; k < 32; ++k) {
            const int v = wsum[k];
            wsum[k] = s;
            s += v;
        }
    }
    __syncthreads();
    if (f) out[offs[blockIdx.x] + wsum[w] + __popc(bal & ((1u << lane) - 1u))] = i;
}

__global__ void k_replicate(int64_t *mask, int64_t n_plane, int64_t plane, int Mz) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t total = n_plane * (int64_t)(Mz - 1);
    if (t >= total) return;
    const int64_t i = t % n_plane;
    const int64_t kz = t / n_plane + 1;
    mask[i + n_plane * kz] = mask[i] + plane * kz;
}

}  // namespace

static int calc_mask_impl(const mr_config *cfg, const float *traj, int64_t Ntrajs, int64_t Nkx,
                          int64_t *d_mask, int64_t *num_out) {
    cudaStream_t s = (cudaStream_t)cfg->stream;
    const bool three = cfg->traj_type == MR_TRAJ_3D;
    const int m[3] = {cfg->phi2_dim[0], cfg->phi2_dim[1], three ? cfg->phi2_dim[2] : 1};
    const int64_t n = (int64_t)m[0] * m[1] * m[2];
    const int64_t ns = Ntrajs * Nkx;
    const double tau = 6.283185307179586;
    unsigned char *a = nullptr, *b = nullptr;
    int *counts = nullptr;
    int64_t *offs = nullptr;
    const int64_t nblk = mr_cdiv(n, kBlk);
    int rc = MR_SUCCESS;
    auto cleanup = [&]() {
        if (a) cudaFree(a);
        if (b) cudaFree(b);
        if (counts) cudaFree(counts);
        if (offs) cudaFree(offs);
    };
    if (cudaMalloc(&a, n) != cudaSuccess || cudaMalloc(&b, n) != cudaSuccess ||
        cudaMalloc(&counts, nblk * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&offs, nblk * sizeof(int64_t)) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        MR_FAIL(MR_ERR_ALLOC, "failed to allocate the %lld-point mask grid", (long long)n);
    }
    cudaMemsetAsync(a, 0, n, s);
    k_mark<<<(unsigned)mr_cdiv(ns, 256), 256, 0, s>>>(a, traj, ns, three ? 3 : 2, m[0], m[1], m[2],
                                                      (float)(m[0] / tau), (float)(m[1] / tau),
                                                      (float)(m[2] / tau));
    int64_t stride = 1;
    for (int ax = 0; ax < 3; ++ax) {
        if (m[ax] > 1 && cfg->mask_radius > 0) {
            k_dilate<<<(unsigned)mr_cdiv(n, 256), 256, 0, s>>>(b, a, n, m[ax], stride, cfg->mask_radius);
            std::swap(a, b);
        }
        stride *= m[ax];
    }
    k_count<<<(unsigned)nblk, 256, 0, s>>>(counts, a, n);
    if (cudaGetLastError() != cudaSuccess) {
        cleanup();
        MR_FAIL(MR_ERR_CUDA, "mask kernels failed to launch");
    }
    std::vector<int> hc(nblk);
    std::vector<int64_t> ho(nblk);
    if (cudaMemcpyAsync(hc.data(), counts, nblk * sizeof(int), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cleanup();
        MR_FAIL(MR_ERR_CUDA, "mask count failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    int64_t tot = 0;
    for (int64_t k = 0; k < nblk; ++k) {
        ho[k] = tot;
        tot += hc[k];
    }
    if (d_mask && tot > 0) {
        cudaMemcpyAsync(offs, ho.data(), nblk * sizeof(int64_t), cudaMemcpyHostToDevice, s);
        k_compact<<<(unsigned)nblk, kBlk, 0, s>>>(d_mask, a, n, offs);
        if (cfg->traj_type == MR_TRAJ_STACK && cfg->phi2_dim[2] > 1) {
            const int Mz = cfg->phi2_dim[2];
            const int64_t tot_rep = tot * (Mz - 1);
            k_replicate<<<(unsigned)mr_cdiv(tot_rep, 256), 256, 0, s>>>(
                d_mask, tot, (int64_t)m[0] * m[1], Mz);
        }
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
            cleanup();
            MR_FAIL(MR_ERR_CUDA, "mask compaction failed");
        }
    }
    if (cfg->traj_type == MR_TRAJ_STACK) tot *= cfg->phi2_dim[2];
    cleanup();
    if (cfg->verbose)
        printf("[mr_aha] calc_mask: kept %lld of %lld upsampled locations within radius %d\n",
               (long long)tot, (long long)mr_pad_size(cfg), cfg->mask_radius);
    *num_out = tot;
    return rc;
}

extern "C" int mr_calc_mask(const mr_config *cfg, const float *d_traj, int64_t Ntrajs,
                            int64_t Nkx, int64_t *d_mask, int64_t *num_masked_out) {
    mr_clear_error();
    MR_REQUIRE(num_masked_out != nullptr, "mr_calc_mask: num_masked_out is NULL");
    *num_masked_out = 0;
    MR_REQUIRE(cfg != nullptr, "mr_calc_mask: cfg is NULL");
    MR_REQUIRE(d_traj != nullptr, "mr_calc_mask: d_traj is NULL");
    MR_REQUIRE(Ntrajs > 0, "mr_calc_mask: Ntrajs = %lld must be > 0", (long long)Ntrajs);
    MR_REQUIRE(Nkx > 0, "mr_calc_mask: Nkx = %lld must be > 0", (long long)Nkx);
    mr_config c = *cfg;
    c.is_masked = 0;
    c.num_masked = 0;
    int rc = mr_config_validate(&c);
    if (rc != MR_SUCCESS) return rc;
    int prev = -1;
    rc = mr_push_device(cfg, &prev);
    if (rc == MR_SUCCESS) rc = calc_mask_impl(cfg, d_traj, Ntrajs, Nkx, d_mask, num_masked_out);
    mr_pop_device(prev);
    return rc;
}
