// Operator object: mr_op_create / execute / info / kernel / destroy /
// abandon (reference src/cuda/mr_op.cu, single-device "direct" path
// :1034-1304, 1348-1352, 1480-1640).
//
// One device: the primary (cfg->gpu_device_id, or the current device for
// -1). A request for further devices is accepted and served by the primary
// alone; mr_op_info reports one device. The operator owns (or, with
// MR_OP_SHARE_PRIMARY, borrows) the maps, the mask and the kernel, and an
// apply plan. Its kernel can be converted to 16-bit storage with a per-
// location scale (mr_b200_op_set_kernel_format), in which case the applies
// read the 16-bit copy. An MR_OP_NUFFT operator holds no kernel and no plan:
// its applies run the NUFFT engine of nufft.cu.
#include <algorithm>
#include <chrono>
#include <new>
#include <cstring>

#include "engine.h"
#include "mr_aha/mr_aha_b200.h"
#include "nufft.h"

struct mr_op_s {
    mr_config cfg;
    mr_op_options opt;
    int dev;
    cudaStream_t stream;
    mr_aha_plan plan;
    const float2 *S;        // maps (borrowed or owned)
    const int64_t *mask;    // mask (borrowed or owned)
    const float2 *K;        // complex64 kernel, reference layout (borrowed or owned)
    void *S_own, *mask_own, *K_own;
    // complex64 kernel in the blocked layout read by the half-length pass 3
    // (mr_kernel_ref::blk), NULL when not built
    float2 *K_blk;
    // 16-bit formats: the codes in a blocked layout (four components per
    // 16-byte word group, rank <= 16) in K_blk, with the locations' scales in
    // natural grid order here; blk_kf = format of the copy in K_blk, -1 if none
    float *K_blk_scale;
    int blk_kf;
    // 16-bit kernel copy (MR_B200_KF_BF16 / MR_B200_KF_I16) and its scales
    int kf;
    void *K16;
    float *K16_scale;
    mr_nufft_op *nu;        // MR_OP_NUFFT engine, NULL for the Toeplitz method
    mr_op_info_t info;
    struct host_pipe *hp;   // host-buffer applies (mr_b200_op_execute_host), NULL until used
};

// Two device slots (input, output) for applies from and to host memory, a
// copy stream per direction, and per slot the events that order the three
// stages of one apply: copy in -> apply on the operator's stream -> copy out.
// Slot k of call i is reused by call i + 2 once call i's apply has read its
// input and its copy out has read its output.
struct host_pipe {
    float2 *dx[2] = {nullptr, nullptr}, *dy[2] = {nullptr, nullptr};
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t in_done[2] = {}, apply_done[2] = {}, out_done[2] = {};
    bool used[2] = {false, false};
    int next = 0;
};

static void host_pipe_free(host_pipe *hp) {
    if (!hp) return;
    if (hp->h2d) cudaStreamSynchronize(hp->h2d);
    if (hp->d2h) cudaStreamSynchronize(hp->d2h);
    for (int k = 0; k < 2; ++k) {
        if (hp->dx[k]) cudaFree(hp->dx[k]);
        if (hp->dy[k]) cudaFree(hp->dy[k]);
        if (hp->in_done[k]) cudaEventDestroy(hp->in_done[k]);
        if (hp->apply_done[k]) cudaEventDestroy(hp->apply_done[k]);
        if (hp->out_done[k]) cudaEventDestroy(hp->out_done[k]);
    }
    if (hp->h2d) cudaStreamDestroy(hp->h2d);
    if (hp->d2h) cudaStreamDestroy(hp->d2h);
    cudaGetLastError();
    delete hp;
}

static void op_release(mr_op op, int skip_device) {
    if (!skip_device) {
        if (op->plan) mr_aha_plan_destroy(op->plan);
        if (op->S_own) cudaFree(op->S_own);
        if (op->mask_own) cudaFree(op->mask_own);
        if (op->K_own) cudaFree(op->K_own);
        if (op->K16) cudaFree(op->K16);
        if (op->K16_scale) cudaFree(op->K16_scale);
        if (op->K_blk) cudaFree(op->K_blk);
        if (op->K_blk_scale) cudaFree(op->K_blk_scale);
        mr_nufft_op_destroy(op->nu);
        host_pipe_free(op->hp);
        cudaGetLastError();
    }
    delete op;
}

static int copy_dev(void **dst, const void *src, size_t bytes, cudaStream_t s) {
    if (cudaMalloc(dst, bytes) != cudaSuccess) {
        cudaGetLastError();
        *dst = nullptr;
        MR_FAIL(MR_ERR_ALLOC, "failed to allocate %zu bytes for an operator copy", bytes);
    }
    MR_CUDA_TRY(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    return MR_SUCCESS;
}

// Blocked copy of the complex64 kernel (mr_kernel_ref::blk): natural grid
// order with x in blocks of 32 (block b = (jz My + jy) Mx/32 + jx/32), from
// the centred reference layout K[t Vpad + cent(jx) + Mx (cent(jy) + My
// cent(jz))]. pair (rank <= 16): with ntri2 = ceil(ntri / 2), element t at
// ((b ntri2 + t/2) 32 + jx % 32) 2 + t % 2, the pad component of an odd ntri
// zero; otherwise element t at (b ntri + t) 32 + jx % 32.
__global__ void k_block_kernel(float2 *__restrict__ out, const float2 *__restrict__ K, int Mx,
                               int My, int Mz, int64_t ntri, int pair) {
    const int64_t vpad = (int64_t)Mx * My * Mz;
    const int64_t ntri2 = (ntri + 1) / 2;
    const int64_t total = vpad * (pair ? 2 * ntri2 : ntri);
    const int nbx = Mx / 32;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
         o += (int64_t)gridDim.x * blockDim.x) {
        int lane;
        int64_t t, b;
        if (pair) {
            lane = (int)((o >> 1) & 31);
            const int64_t rest = o >> 6;
            t = 2 * (rest % ntri2) + (o & 1);
            b = rest / ntri2;
        } else {
            lane = (int)(o & 31);
            const int64_t rest = o >> 5;
            t = rest % ntri;
            b = rest / ntri;
        }
        const int jx = (int)(b % nbx) * 32 + lane;
        const int64_t yz = b / nbx;
        const int jy = (int)(yz % My), jz = (int)(yz / My);
        const int64_t row = mr_nat2cent_d(jx, Mx, Mx / 2) +
                            (int64_t)Mx * (mr_nat2cent_d(jy, My, My / 2) +
                                           (int64_t)My * mr_nat2cent_d(jz, Mz, Mz / 2));
        out[o] = t < ntri ? K[t * vpad + row] : make_float2(0.f, 0.f);
    }
}

// Blocked copy of a masked kernel ([ntri][num_masked], row r at the centred
// grid index mask[r]): every row scattered to its grid location in the layout
// of k_block_kernel; locations outside the mask keep the zeros of the
// preceding memset.
__global__ void k_block_kernel_masked(float2 *__restrict__ out, const float2 *__restrict__ K,
                                      const int64_t *__restrict__ mask, int64_t nm, int Mx,
                                      int My, int Mz, int64_t ntri, int pair) {
    const int64_t ntri2 = (ntri + 1) / 2;
    const int64_t total = nm * ntri;
    const int nbx = Mx / 32;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
         o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = o % nm;
        const int64_t t = o / nm;
        int64_t c = __ldg(mask + r);
        if (c < 0 || c >= (int64_t)Mx * My * Mz) continue;  // not a grid location
        const int kx = (int)(c % Mx);
        c /= Mx;
        const int ky = (int)(c % My);
        const int kz = (int)(c / My);
        // centred -> natural index along each axis (inverse of mr_nat2cent_d)
        const int jx = mr_nat2cent_d(kx, Mx, Mx - Mx / 2);
        const int jy = mr_nat2cent_d(ky, My, My - My / 2);
        const int jz = mr_nat2cent_d(kz, Mz, Mz - Mz / 2);
        const int64_t b = ((int64_t)jz * My + jy) * nbx + jx / 32;
        const int64_t pos = pair ? ((b * ntri2 + t / 2) * 32 + jx % 32) * 2 + (t & 1)
                                 : (b * ntri + t) * 32 + jx % 32;
        out[pos] = K[o];
    }
}

// 16-bit blocked copy: with ntri4 = ceil(ntri / 4), the code of element
// (t, jx, jy, jz) at word ((b ntri4 + t/4) 32 + jx % 32) 4 + t % 4 (block b as
// in k_block_kernel; pad components zero), and the location's scale at its
// natural grid index (b 32 + jx % 32), from the reference-layout codes and
// scales (row = centred grid index).
__global__ void k_block_kernel16(uint32_t *__restrict__ out, float *__restrict__ sout,
                                 const uint32_t *__restrict__ K16, const float *__restrict__ scale,
                                 int Mx, int My, int Mz, int64_t ntri) {
    const int64_t vpad = (int64_t)Mx * My * Mz;
    const int64_t ntri4 = (ntri + 3) / 4;
    const int64_t total = vpad * 4 * ntri4;
    const int nbx = Mx / 32;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
         o += (int64_t)gridDim.x * blockDim.x) {
        const int lane = (int)((o >> 2) & 31);
        const int64_t rest = o >> 7;
        const int64_t t = 4 * (rest % ntri4) + (o & 3);
        const int64_t b = rest / ntri4;
        const int jx = (int)(b % nbx) * 32 + lane;
        const int64_t yz = b / nbx;
        const int jy = (int)(yz % My), jz = (int)(yz / My);
        const int64_t row = mr_nat2cent_d(jx, Mx, Mx / 2) +
                            (int64_t)Mx * (mr_nat2cent_d(jy, My, My / 2) +
                                           (int64_t)My * mr_nat2cent_d(jz, Mz, Mz / 2));
        out[o] = t < ntri ? K16[t * vpad + row] : 0u;
        if (t == 0) sout[b * 32 + lane] = scale[row];
    }
}

static void op_free_blocked(mr_op op) {
    if (op->K_blk || op->K_blk_scale) cudaStreamSynchronize(op->stream);
    if (op->K_blk) cudaFree(op->K_blk);
    if (op->K_blk_scale) cudaFree(op->K_blk_scale);
    op->K_blk = nullptr;
    op->K_blk_scale = nullptr;
    op->blk_kf = -1;
    cudaGetLastError();
}

static size_t op_blocked_bytes(const mr_config *cfg, int kf) {
    const size_t vpad = (size_t)mr_pad_size(cfg);
    if (kf == MR_KF_F32) return vpad * mr_blk_tri(cfg->L) * sizeof(float2);
    return vpad * mr_blk16_tri(cfg->L) * 4 + vpad * sizeof(float);
}

// Build the blocked copy of the current kernel format when the plan can use
// it and the device has room (it doubles the kernel's footprint); otherwise
// leave it out (the apply then reads the reference layout). complex64: only
// for a kernel the operator owns (a borrowed one may change under it); a
// masked operator's copy covers the whole grid, zero outside the mask.
// 16-bit: unmasked, rank <= 16. A copy of another format is freed first.
// Never fails the caller.
static void op_build_blocked(mr_op op) {
    if (op->K_blk && op->blk_kf == op->kf) return;
    op_free_blocked(op);
    if (!op->plan || !mr_plan_half_pass3(op->plan) || mr_env_int("MR_AHA_B200_NO_BLOCKED", 0))
        return;
    const bool f32 = op->kf == MR_KF_F32;
    if (f32 ? !op->K_own : (!op->K16 || op->cfg.is_masked || op->cfg.L > 16)) return;
    mr_geom g;
    mr_geom_from_config(&op->cfg, &g);
    const int64_t ntri = mr_num_tri(op->cfg.L);
    const size_t bytes = op_blocked_bytes(&op->cfg, op->kf);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < bytes + ((size_t)2 << 30)) {
        cudaGetLastError();
        return;
    }
    const size_t sbytes = f32 ? 0 : (size_t)g.vpad * sizeof(float);
    if (cudaMalloc(&op->K_blk, bytes - sbytes) != cudaSuccess ||
        (sbytes && cudaMalloc(&op->K_blk_scale, sbytes) != cudaSuccess)) {
        cudaGetLastError();
        op_free_blocked(op);
        return;
    }
    if (!f32) {
        k_block_kernel16<<<148 * 16, 256, 0, op->stream>>>(
            reinterpret_cast<uint32_t *>(op->K_blk), op->K_blk_scale,
            reinterpret_cast<const uint32_t *>(op->K16), op->K16_scale, g.m[0], g.m[1], g.m[2],
            ntri);
    } else {
        const int pair = op->cfg.L <= 16 ? 1 : 0;
        if (op->cfg.is_masked) {
            if (cudaMemsetAsync(op->K_blk, 0, bytes, op->stream) != cudaSuccess) {
                cudaGetLastError();
                op_free_blocked(op);
                return;
            }
            k_block_kernel_masked<<<148 * 16, 256, 0, op->stream>>>(
                op->K_blk, op->K, op->mask, op->cfg.num_masked, g.m[0], g.m[1], g.m[2], ntri,
                pair);
        } else {
            k_block_kernel<<<148 * 16, 256, 0, op->stream>>>(op->K_blk, op->K, g.m[0], g.m[1],
                                                             g.m[2], ntri, pair);
        }
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(op->stream) != cudaSuccess) {
        cudaGetLastError();
        op_free_blocked(op);
        return;
    }
    op->blk_kf = op->kf;
}

static int op_check(const mr_config *cfg, const mr_op_inputs *in, const mr_op_options *o) {
    int rc = mr_config_validate(cfg);
    if (rc != MR_SUCCESS) return rc;
    MR_REQUIRE(o->method == MR_OP_TOEPLITZ || o->method == MR_OP_NUFFT,
               "mr_op_create: method = %d is neither MR_OP_TOEPLITZ nor MR_OP_NUFFT",
               (int)o->method);
    MR_REQUIRE(in->d_SEs != nullptr, "mr_op_create: d_SEs is NULL");
    const bool need_gram = o->method == MR_OP_NUFFT || in->d_phi2_toep == nullptr;
    if (need_gram) {
        MR_REQUIRE(in->d_phi2 != nullptr, "mr_op_create: d_phi2 is NULL");
        MR_REQUIRE(in->d_traj != nullptr, "mr_op_create: d_traj is NULL");
        MR_REQUIRE(in->Ntrajs > 0 && in->Nkx > 0,
                   "mr_op_create: Ntrajs = %lld and Nkx = %lld must be > 0",
                   (long long)in->Ntrajs, (long long)in->Nkx);
    }
    if (o->method == MR_OP_NUFFT) {
        MR_REQUIRE(!cfg->is_masked,
                   "mr_op_create: the NUFFT method has no kernel to mask; set is_masked = 0 "
                   "(or use the Toeplitz method)");
        MR_REQUIRE(in->d_phi2_toep == nullptr,
                   "mr_op_create: d_phi2_toep is only used by the Toeplitz method");
        MR_REQUIRE(o->nufft_upsampfac == 0.0 || o->nufft_upsampfac > 1.0,
                   "mr_op_create: nufft_upsampfac = %g must be 0 (default 2.0) or above 1",
                   o->nufft_upsampfac);
    }
    if (cfg->is_masked)
        MR_REQUIRE(in->d_mask != nullptr, "mr_op_create: d_mask is required when is_masked is set");
    return MR_SUCCESS;
}

static int op_create_impl(const mr_config *cfg, const mr_op_inputs *in, const mr_op_options *o,
                          mr_op *out) {
    const auto t_start = std::chrono::steady_clock::now();
    int rc = op_check(cfg, in, o);
    if (rc != MR_SUCCESS) return rc;
    mr_op op = new (std::nothrow) mr_op_s();
    if (!op) MR_FAIL(MR_ERR_ALLOC, "failed to allocate the operator");
    op->blk_kf = -1;
    op->cfg = *cfg;
    op->opt = *o;
    op->stream = (cudaStream_t)cfg->stream;
    if (cudaGetDevice(&op->dev) != cudaSuccess) {
        op_release(op, 1);
        MR_FAIL(MR_ERR_CUDA, "cudaGetDevice failed");
    }
    cudaStream_t s = op->stream;
    // Inputs produced on the caller's stream must be complete.
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        op_release(op, 1);
        MR_FAIL(MR_ERR_CUDA, "synchronising the caller's stream failed");
    }
    const bool share = (o->flags & MR_OP_SHARE_PRIMARY) != 0;
    const size_t se_bytes = (size_t)mr_se_size(cfg) * sizeof(float2);
    const size_t k_bytes = (size_t)mr_phi2_toep_size(cfg) * sizeof(float2);
    if (share) {
        op->S = reinterpret_cast<const float2 *>(in->d_SEs);
        op->mask = in->d_mask;
    } else {
        rc = copy_dev(&op->S_own, in->d_SEs, se_bytes, s);
        if (rc == MR_SUCCESS && cfg->is_masked)
            rc = copy_dev(&op->mask_own, in->d_mask, (size_t)cfg->num_masked * sizeof(int64_t), s);
        if (rc != MR_SUCCESS) {
            op_release(op, 0);
            return rc;
        }
        op->S = (const float2 *)op->S_own;
        op->mask = (const int64_t *)op->mask_own;
    }
    double toep_ms = 0.0;
    if (o->method == MR_OP_NUFFT) {
        mr_config c = *cfg;
        c.gpu_device_id = -1;
        rc = mr_nufft_op_create(&c, reinterpret_cast<const float2 *>(in->d_phi2), in->d_traj,
                                in->Ntrajs, in->Nkx, o->nufft_upsampfac, s, &op->nu);
        if (rc != MR_SUCCESS) {
            char msg[512];
            snprintf(msg, sizeof(msg), "%s", mr_last_error());
            op_release(op, 0);
            mr_set_error("%s", msg);
            return rc;
        }
        op->kf = MR_KF_F32;
        mr_op_info_t &inf = op->info;
        inf.method = MR_OP_NUFFT;
        inf.n_devices = 1;
        inf.devices[0] = op->dev;
        inf.coil_begin[0] = 0;
        inf.coil_count[0] = cfg->n_coils;
        inf.group[0] = 1;
        inf.toep_source = MR_OP_TOEP_NONE;
        inf.toep_devices = 0;
        inf.create_ms = std::chrono::duration<double, std::milli>(
                            std::chrono::steady_clock::now() - t_start)
                            .count();
        *out = op;
        return MR_SUCCESS;
    }
    if (in->d_phi2_toep) {
        if (share) {
            op->K = reinterpret_cast<const float2 *>(in->d_phi2_toep);
        } else {
            rc = copy_dev(&op->K_own, in->d_phi2_toep, k_bytes, s);
            if (rc != MR_SUCCESS) {
                op_release(op, 0);
                return rc;
            }
            op->K = (const float2 *)op->K_own;
        }
        op->info.toep_source = MR_OP_TOEP_SUPPLIED;
        op->info.toep_devices = 0;
    } else {
        if (cudaMalloc(&op->K_own, k_bytes) != cudaSuccess) {
            cudaGetLastError();
            op_release(op, 0);
            MR_FAIL(MR_ERR_ALLOC, "failed to allocate the %zu-byte Toeplitz kernel", k_bytes);
        }
        const auto t0 = std::chrono::steady_clock::now();
        mr_config c = *cfg;
        c.gpu_device_id = -1;
        rc = mr_calc_toep(&c, in->d_phi2, in->d_traj, in->Ntrajs, in->Nkx, op->mask,
                          (mr_complex *)op->K_own);
        if (rc != MR_SUCCESS) {
            char msg[512];
            snprintf(msg, sizeof(msg), "%s", mr_last_error());
            op_release(op, 0);
            mr_set_error("%s", msg);
            return rc;
        }
        toep_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
        op->K = (const float2 *)op->K_own;
        op->info.toep_source = MR_OP_TOEP_BROADCAST;
        op->info.toep_devices = 1;
    }
    mr_config c = *cfg;
    c.gpu_device_id = -1;
    rc = mr_aha_plan_create(&c, &op->plan);
    if (rc != MR_SUCCESS) {
        char msg[512];
        snprintf(msg, sizeof(msg), "%s", mr_last_error());
        op_release(op, 0);
        mr_set_error("%s", msg);
        return rc;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        op_release(op, 0);
        MR_FAIL(MR_ERR_CUDA, "operator creation failed: %s",
                cudaGetErrorString(cudaGetLastError()));
    }
    op->kf = MR_KF_F32;
    op_build_blocked(op);
    mr_op_info_t &inf = op->info;
    inf.method = MR_OP_TOEPLITZ;
    inf.n_devices = 1;
    inf.devices[0] = op->dev;
    inf.coil_begin[0] = 0;
    inf.coil_count[0] = cfg->n_coils;
    inf.group[0] = mr_plan_group(op->plan);
    inf.toep_ms = toep_ms;
    inf.create_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start)
            .count();
    *out = op;
    return MR_SUCCESS;
}

extern "C" int mr_op_options_defaults(mr_op_options *opt) {
    mr_clear_error();
    MR_REQUIRE(opt != nullptr, "mr_op_options_defaults: opt is NULL");
    std::memset(opt, 0, sizeof(*opt));
    opt->method = MR_OP_TOEPLITZ;
    opt->toep_dist = MR_TOEP_DIST_AUTO;
    opt->flags = MR_OP_SHARE_PRIMARY;
    return MR_SUCCESS;
}

extern "C" int mr_op_create(const mr_config *cfg, const mr_op_inputs *in,
                            const mr_op_options *opt, mr_op *op_out) {
    mr_clear_error();
    MR_REQUIRE(op_out != nullptr, "mr_op_create: op_out is NULL");
    *op_out = nullptr;
    MR_REQUIRE(cfg != nullptr, "mr_op_create: cfg is NULL");
    MR_REQUIRE(in != nullptr, "mr_op_create: in is NULL");
    mr_op_options o;
    if (opt) o = *opt;
    else mr_op_options_defaults(&o);
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    int rc = MR_SUCCESS;
    if (cfg->gpu_device_id >= 0 && cfg->gpu_device_id != prev) {
        if (cudaSetDevice(cfg->gpu_device_id) != cudaSuccess) {
            cudaGetLastError();
            MR_FAIL(MR_ERR_CUDA, "cannot select device %d", cfg->gpu_device_id);
        }
    }
    rc = op_create_impl(cfg, in, &o, op_out);
    cudaSetDevice(prev);
    return rc;
}

static mr_kernel_ref op_kernel_ref(mr_op op) {
    mr_kernel_ref K;
    std::memset(&K, 0, sizeof(K));
    if (op->kf == MR_KF_F32) {
        K.data = op->K;
    } else {
        K.data = op->K16;
        K.scale = op->K16_scale;
    }
    if (op->K_blk && op->blk_kf == op->kf) {
        K.blk = op->K_blk;
        K.sblk = op->K_blk_scale;
    }
    K.kf = op->kf;
    return K;
}

int mr_op_execute_on(mr_op op, const float2 *x, float2 *out, cudaStream_t s) {
    if (op->nu) return mr_nufft_op_apply(op->nu, x, op->S, out, s);
    return mr_plan_execute_k(op->plan, x, op->S, op_kernel_ref(op), op->mask, out, s);
}

const mr_config *mr_op_config(mr_op op) { return &op->cfg; }
int mr_op_device(mr_op op) { return op->dev; }
cudaStream_t mr_op_stream(mr_op op) { return op->stream; }

extern "C" int mr_op_execute(mr_op op, const mr_complex *d_x, mr_complex *d_AhAx) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_op_execute: op is NULL");
    MR_REQUIRE(d_x != nullptr, "mr_op_execute: d_x is NULL");
    MR_REQUIRE(d_AhAx != nullptr, "mr_op_execute: d_AhAx is NULL");
    MR_REQUIRE((const void *)d_AhAx != (const void *)d_x,
               "mr_op_execute: d_AhAx must not alias d_x");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != op->dev) MR_CUDA_TRY(cudaSetDevice(op->dev));
    const int rc = mr_op_execute_on(op, reinterpret_cast<const float2 *>(d_x),
                                    reinterpret_cast<float2 *>(d_AhAx), op->stream);
    if (prev != op->dev) cudaSetDevice(prev);
    return rc;
}

extern "C" int mr_op_info(mr_op op, mr_op_info_t *info) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_op_info: op is NULL");
    MR_REQUIRE(info != nullptr, "mr_op_info: info is NULL");
    *info = op->info;
    return MR_SUCCESS;
}

extern "C" int mr_op_kernel(mr_op op, int k, const mr_complex **d_phi2_toep) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_op_kernel: op is NULL");
    MR_REQUIRE(d_phi2_toep != nullptr, "mr_op_kernel: d_phi2_toep is NULL");
    if (op->opt.method != MR_OP_TOEPLITZ)
        MR_FAIL(MR_ERR_UNSUPPORTED, "mr_op_kernel: a NUFFT operator has no kernel");
    MR_REQUIRE(k >= 0 && k < op->info.n_devices, "mr_op_kernel: device index %d outside [0, %d)",
               k, op->info.n_devices);
    if (!op->K)
        MR_FAIL(MR_ERR_UNSUPPORTED,
                "mr_op_kernel: the complex64 kernel was released after conversion to 16-bit "
                "storage");
    *d_phi2_toep = reinterpret_cast<const mr_complex *>(op->K);
    return MR_SUCCESS;
}

// ---- applies from and to host memory ----

// Makes the operator's device current; *prev = the device to restore, or -1.
static int op_push_device(mr_op op, int *prev) {
    *prev = -1;
    int cur = 0;
    MR_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != op->dev) {
        MR_CUDA_TRY(cudaSetDevice(op->dev));
        *prev = cur;
    }
    return MR_SUCCESS;
}

static int host_pipe_create(mr_op op, size_t bytes, host_pipe **out) {
    host_pipe *hp = new host_pipe();
    bool ok = cudaStreamCreateWithFlags(&hp->h2d, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&hp->d2h, cudaStreamNonBlocking) == cudaSuccess;
    for (int k = 0; k < 2 && ok; ++k)
        ok = cudaEventCreateWithFlags(&hp->in_done[k], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&hp->apply_done[k], cudaEventDisableTiming) ==
                 cudaSuccess &&
             cudaEventCreateWithFlags(&hp->out_done[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        host_pipe_free(hp);
        MR_FAIL(MR_ERR_CUDA, "host-buffer apply: cannot create streams or events");
    }
    for (int k = 0; k < 2; ++k) {
        if (cudaMalloc(&hp->dx[k], bytes) != cudaSuccess ||
            cudaMalloc(&hp->dy[k], bytes) != cudaSuccess) {
            host_pipe_free(hp);
            MR_FAIL(MR_ERR_ALLOC, "host-buffer apply: cannot allocate 4 x %zu bytes", bytes);
        }
    }
    (void)op;
    *out = hp;
    return MR_SUCCESS;
}

static int execute_host_impl(mr_op op, const mr_complex *h_x, mr_complex *h_AhAx) {
    const size_t bytes = (size_t)mr_x_size(&op->cfg) * sizeof(float2);
    if (!op->hp) {
        const int rc = host_pipe_create(op, bytes, &op->hp);
        if (rc != MR_SUCCESS) return rc;
    }
    host_pipe *hp = op->hp;
    const int k = hp->next;
    // copy in, once the apply two calls back has read this slot's input
    if (hp->used[k]) MR_CUDA_TRY(cudaStreamWaitEvent(hp->h2d, hp->apply_done[k], 0));
    MR_CUDA_TRY(cudaMemcpyAsync(hp->dx[k], h_x, bytes, cudaMemcpyHostToDevice, hp->h2d));
    MR_CUDA_TRY(cudaEventRecord(hp->in_done[k], hp->h2d));
    // apply, once the input is in and the copy out two calls back has read
    // this slot's output
    MR_CUDA_TRY(cudaStreamWaitEvent(op->stream, hp->in_done[k], 0));
    if (hp->used[k]) MR_CUDA_TRY(cudaStreamWaitEvent(op->stream, hp->out_done[k], 0));
    const int rc = mr_op_execute_on(op, hp->dx[k], hp->dy[k], op->stream);
    if (rc != MR_SUCCESS) return rc;
    MR_CUDA_TRY(cudaEventRecord(hp->apply_done[k], op->stream));
    // copy out
    MR_CUDA_TRY(cudaStreamWaitEvent(hp->d2h, hp->apply_done[k], 0));
    MR_CUDA_TRY(cudaMemcpyAsync(h_AhAx, hp->dy[k], bytes, cudaMemcpyDeviceToHost, hp->d2h));
    MR_CUDA_TRY(cudaEventRecord(hp->out_done[k], hp->d2h));
    hp->used[k] = true;
    hp->next = k ^ 1;
    return MR_SUCCESS;
}

extern "C" int mr_b200_op_execute_host(mr_op op, const mr_complex *h_x, mr_complex *h_AhAx) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_execute_host: op is NULL");
    MR_REQUIRE(h_x != nullptr, "mr_b200_op_execute_host: h_x is NULL");
    MR_REQUIRE(h_AhAx != nullptr, "mr_b200_op_execute_host: h_AhAx is NULL");
    MR_REQUIRE((const void *)h_AhAx != (const void *)h_x,
               "mr_b200_op_execute_host: h_AhAx must not alias h_x");
    int prev = -1;
    int rc = op_push_device(op, &prev);
    if (rc == MR_SUCCESS) rc = execute_host_impl(op, h_x, h_AhAx);
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_b200_op_host_sync(mr_op op) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_host_sync: op is NULL");
    if (!op->hp) return MR_SUCCESS;
    int prev = -1;
    int rc = op_push_device(op, &prev);
    if (rc == MR_SUCCESS) {
        const cudaError_t e1 = cudaStreamSynchronize(op->hp->h2d);
        const cudaError_t e2 = cudaStreamSynchronize(op->stream);
        const cudaError_t e3 = cudaStreamSynchronize(op->hp->d2h);
        const cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
        if (e != cudaSuccess) {
            cudaGetLastError();
            mr_pop_device(prev);
            MR_FAIL(MR_ERR_CUDA, "mr_b200_op_host_sync: %s", cudaGetErrorString(e));
        }
    }
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_b200_op_host_release(mr_op op) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_host_release: op is NULL");
    if (!op->hp) return MR_SUCCESS;
    int prev = -1;
    int rc = op_push_device(op, &prev);
    if (rc == MR_SUCCESS) {
        cudaStreamSynchronize(op->stream);
        host_pipe_free(op->hp);
        op->hp = nullptr;
    }
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_op_destroy(mr_op op) {
    mr_clear_error();
    if (!op) return MR_SUCCESS;
    int prev = 0;
    const cudaError_t ce = cudaGetDevice(&prev);
    cudaSetDevice(op->dev);
    cudaStreamSynchronize(op->stream);
    cudaGetLastError();
    op_release(op, 0);
    if (ce == cudaSuccess) cudaSetDevice(prev);
    return MR_SUCCESS;
}

extern "C" int mr_op_abandon(mr_op op) {
    mr_clear_error();
    if (!op) return MR_SUCCESS;
    // The primary device was reset: its buffers are gone with the context.
    if (op->plan) {
        // the plan's host struct only
        free(op->plan);
        op->plan = nullptr;
    }
    op_release(op, 1);
    return MR_SUCCESS;
}

// ---------------------------------------------------------------------------
// 16-bit kernel storage
// ---------------------------------------------------------------------------

// One block per location q: scale_q = max |re|, |im| over its ntri elements
// divided by the largest code (int16: 32767; bf16: 1, the scale only
// normalises), then every element is stored relative to it.
template <int KF>
__global__ void k_quantize(void *out, float *scale, const float2 *__restrict__ K, int64_t nloc,
                           int64_t ntri) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nloc;
         q += (int64_t)gridDim.x * blockDim.x) {
        float m = 0.f;
        for (int64_t t = 0; t < ntri; ++t) {
            const float2 v = K[q + nloc * t];
            m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
        float sc;
        if constexpr (KF == MR_KF_I16) sc = m > 0.f ? m / 32767.f : 1.f;
        else sc = m > 0.f ? m : 1.f;
        scale[q] = sc;
        const float inv = 1.f / sc;
        for (int64_t t = 0; t < ntri; ++t) {
            const float2 v = K[q + nloc * t];
            if constexpr (KF == MR_KF_I16) {
                short2 c;
                c.x = (short)__float2int_rn(fminf(fmaxf(v.x * inv, -32767.f), 32767.f));
                c.y = (short)__float2int_rn(fminf(fmaxf(v.y * inv, -32767.f), 32767.f));
                reinterpret_cast<short2 *>(out)[q + nloc * t] = c;
            } else {
                reinterpret_cast<__nv_bfloat162 *>(out)[q + nloc * t] =
                    __floats2bfloat162_rn(v.x * inv, v.y * inv);
            }
        }
    }
}

extern "C" int mr_b200_op_set_kernel_format(mr_op op, int format, int keep_complex64) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_set_kernel_format: op is NULL");
    MR_REQUIRE(format == MR_B200_KF_COMPLEX64 || format == MR_B200_KF_BF16 ||
                   format == MR_B200_KF_INT16,
               "mr_b200_op_set_kernel_format: unknown format %d", format);
    if (op->nu)
        MR_FAIL(MR_ERR_UNSUPPORTED, "mr_b200_op_set_kernel_format: a NUFFT operator has no kernel");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != op->dev) MR_CUDA_TRY(cudaSetDevice(op->dev));
    int rc = MR_SUCCESS;
    cudaStream_t s = op->stream;
    if (format == MR_B200_KF_COMPLEX64) {
        if (!op->K) {
            rc = MR_ERR_UNSUPPORTED;
            mr_set_error("the complex64 kernel was released; it cannot be restored");
        } else {
            op->kf = MR_KF_F32;
            op_build_blocked(op);
        }
    } else if (!op->K) {
        rc = MR_ERR_UNSUPPORTED;
        mr_set_error("the complex64 kernel was released; it cannot be re-quantised");
    } else {
        const int64_t nloc = op->cfg.is_masked ? op->cfg.num_masked : mr_pad_size(&op->cfg);
        const int64_t ntri = mr_num_tri(op->cfg.L);
        // a blocked copy serves only its own format: give its memory back
        // before the 16-bit kernel is allocated
        op_free_blocked(op);
        if (op->K16) cudaFree(op->K16);
        if (op->K16_scale) cudaFree(op->K16_scale);
        op->K16 = nullptr;
        op->K16_scale = nullptr;
        if (cudaMalloc(&op->K16, (size_t)nloc * ntri * 4) != cudaSuccess ||
            cudaMalloc(&op->K16_scale, (size_t)nloc * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            rc = MR_ERR_ALLOC;
            mr_set_error("failed to allocate the 16-bit kernel");
        } else {
            const unsigned blocks = (unsigned)std::min<int64_t>(mr_cdiv(nloc, 256), 148 * 16);
            if (format == MR_B200_KF_INT16)
                k_quantize<MR_KF_I16><<<blocks, 256, 0, s>>>(op->K16, op->K16_scale, op->K, nloc, ntri);
            else
                k_quantize<MR_KF_BF16><<<blocks, 256, 0, s>>>(op->K16, op->K16_scale, op->K, nloc, ntri);
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
                rc = MR_ERR_CUDA;
                mr_set_error("kernel quantisation failed");
            } else {
                op->kf = format == MR_B200_KF_INT16 ? MR_KF_I16 : MR_KF_BF16;
                if (!keep_complex64) {
                    // an owned copy is freed; a borrowed kernel is handed
                    // back (the caller may free it)
                    if (op->K_own) cudaFree(op->K_own);
                    op->K_own = nullptr;
                    op->K = nullptr;
                }
                op_build_blocked(op);
            }
        }
    }
    if (prev != op->dev) cudaSetDevice(prev);
    return rc;
}

// Checkpoint of a 16-bit kernel: its codes ([ntri][nloc] (re, im) pairs of
// 16-bit codes) and per-location scales, copied out of or into the operator.
extern "C" int mr_b200_op_save_kernel16(mr_op op, int *format, void *d_codes, float *d_scale) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && format != nullptr && d_codes != nullptr && d_scale != nullptr,
               "mr_b200_op_save_kernel16: NULL argument");
    if (op->kf == MR_KF_F32 || !op->K16)
        MR_FAIL(MR_ERR_UNSUPPORTED,
                "mr_b200_op_save_kernel16: the operator's kernel is not stored in 16 bits");
    const int64_t nloc = op->cfg.is_masked ? op->cfg.num_masked : mr_pad_size(&op->cfg);
    const int64_t ntri = mr_num_tri(op->cfg.L);
    int prev = -1;
    int rc = op_push_device(op, &prev);
    if (rc == MR_SUCCESS) {
        const cudaError_t e1 = cudaMemcpyAsync(d_codes, op->K16, (size_t)nloc * ntri * 4,
                                               cudaMemcpyDeviceToDevice, op->stream);
        const cudaError_t e2 = cudaMemcpyAsync(d_scale, op->K16_scale, (size_t)nloc * sizeof(float),
                                               cudaMemcpyDeviceToDevice, op->stream);
        const cudaError_t e3 = cudaStreamSynchronize(op->stream);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
            cudaGetLastError();
            rc = MR_ERR_CUDA;
            mr_set_error("mr_b200_op_save_kernel16: copy failed");
        } else {
            *format = op->kf == MR_KF_I16 ? MR_B200_KF_INT16 : MR_B200_KF_BF16;
        }
    }
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_b200_op_load_kernel16(mr_op op, int format, const void *d_codes,
                                        const float *d_scale) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && d_codes != nullptr && d_scale != nullptr,
               "mr_b200_op_load_kernel16: NULL argument");
    MR_REQUIRE(format == MR_B200_KF_BF16 || format == MR_B200_KF_INT16,
               "mr_b200_op_load_kernel16: format %d is not a 16-bit format", format);
    if (op->nu)
        MR_FAIL(MR_ERR_UNSUPPORTED, "mr_b200_op_load_kernel16: a NUFFT operator has no kernel");
    const int64_t nloc = op->cfg.is_masked ? op->cfg.num_masked : mr_pad_size(&op->cfg);
    const int64_t ntri = mr_num_tri(op->cfg.L);
    int prev = -1;
    int rc = op_push_device(op, &prev);
    if (rc != MR_SUCCESS) return rc;
    void *codes = op->K16;
    float *scale = op->K16_scale;
    if (!codes && cudaMalloc(&codes, (size_t)nloc * ntri * 4) != cudaSuccess) codes = nullptr;
    if (codes && !scale && cudaMalloc(&scale, (size_t)nloc * sizeof(float)) != cudaSuccess)
        scale = nullptr;
    if (!codes || !scale) {
        cudaGetLastError();
        if (codes && codes != op->K16) cudaFree(codes);
        mr_pop_device(prev);
        MR_FAIL(MR_ERR_ALLOC, "mr_b200_op_load_kernel16: cannot allocate the 16-bit kernel");
    }
    op->K16 = codes;
    op->K16_scale = scale;
    const cudaError_t e1 = cudaMemcpyAsync(codes, d_codes, (size_t)nloc * ntri * 4,
                                           cudaMemcpyDeviceToDevice, op->stream);
    const cudaError_t e2 = cudaMemcpyAsync(scale, d_scale, (size_t)nloc * sizeof(float),
                                           cudaMemcpyDeviceToDevice, op->stream);
    const cudaError_t e3 = cudaStreamSynchronize(op->stream);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        cudaGetLastError();
        mr_pop_device(prev);
        MR_FAIL(MR_ERR_CUDA, "mr_b200_op_load_kernel16: copy failed");
    }
    // the loaded codes replace the kernel: the complex64 one (and its blocked
    // copy) no longer describe this operator
    op_free_blocked(op);
    if (op->K_own) cudaFree(op->K_own);
    op->K_own = nullptr;
    op->K = nullptr;
    op->kf = format == MR_B200_KF_INT16 ? MR_KF_I16 : MR_KF_BF16;
    op->info.toep_source = MR_OP_TOEP_SUPPLIED;
    op_build_blocked(op);
    mr_pop_device(prev);
    return MR_SUCCESS;
}

extern "C" int mr_b200_op_kernel_format(mr_op op, int *format) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && format != nullptr, "mr_b200_op_kernel_format: NULL argument");
    *format = op->kf == MR_KF_F32 ? MR_B200_KF_COMPLEX64
                                  : (op->kf == MR_KF_I16 ? MR_B200_KF_INT16 : MR_B200_KF_BF16);
    return MR_SUCCESS;
}

extern "C" int mr_b200_op_profile(mr_op op, const mr_complex *d_x, mr_complex *d_AhAx,
                                  float *ms, char *names, int max_passes, int *n_passes) {
    mr_clear_error();
    MR_REQUIRE(op && d_x && d_AhAx && ms && n_passes, "mr_b200_op_profile: NULL argument");
    MR_REQUIRE(max_passes >= 1, "mr_b200_op_profile: max_passes must be >= 1");
    if (op->nu)
        MR_FAIL(MR_ERR_UNSUPPORTED, "mr_b200_op_profile: per-pass timing is for Toeplitz operators");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != op->dev) MR_CUDA_TRY(cudaSetDevice(op->dev));
    mr_prof prof;
    std::memset(&prof, 0, sizeof(prof));
    int rc = MR_SUCCESS;
    for (int k = 0; k <= MR_PROF_MAX; ++k)
        if (cudaEventCreate(&prof.ev[k]) != cudaSuccess) rc = MR_ERR_CUDA;
    if (rc == MR_SUCCESS)
        rc = mr_plan_execute_k(op->plan, reinterpret_cast<const float2 *>(d_x), op->S,
                               op_kernel_ref(op), op->mask, reinterpret_cast<float2 *>(d_AhAx),
                               op->stream, &prof);
    if (rc == MR_SUCCESS && cudaStreamSynchronize(op->stream) != cudaSuccess) {
        rc = MR_ERR_CUDA;
        mr_set_error("profiled execute failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (rc == MR_SUCCESS) {
        const int n = std::min(prof.n, max_passes);
        for (int k = 0; k < n; ++k) {
            float t = 0.f;
            cudaEventElapsedTime(&t, prof.ev[k], prof.ev[k + 1]);
            ms[k] = t;
            if (names) {
                std::strncpy(names + 32 * k, prof.name[k], 31);
                names[32 * k + 31] = '\0';
            }
        }
        *n_passes = n;
    }
    for (int k = 0; k <= MR_PROF_MAX; ++k)
        if (prof.ev[k]) cudaEventDestroy(prof.ev[k]);
    if (prev != op->dev) cudaSetDevice(prev);
    return rc;
}

extern "C" int mr_b200_op_autotune(mr_op op, int reps, float *ms) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_autotune: op is NULL");
    MR_REQUIRE(reps >= 1 && reps <= 100, "mr_b200_op_autotune: reps = %d outside [1, 100]", reps);
    if (op->nu)
        MR_FAIL(MR_ERR_UNSUPPORTED, "mr_b200_op_autotune: a NUFFT operator has no pass choices");
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != op->dev) MR_CUDA_TRY(cudaSetDevice(op->dev));
    const size_t vb = (size_t)mr_x_size(&op->cfg) * sizeof(float2);
    float2 *buf = nullptr;
    int rc = MR_SUCCESS;
    if (cudaMalloc(&buf, 2 * vb) != cudaSuccess) {
        cudaGetLastError();
        buf = nullptr;
        mr_set_error("mr_b200_op_autotune: cannot allocate 2 x %zu bytes of trial vectors", vb);
        rc = MR_ERR_ALLOC;
    }
    // a constant non-zero trial input (timings do not depend on the values)
    if (rc == MR_SUCCESS && cudaMemsetAsync(buf, 0x3c, 2 * vb, op->stream) != cudaSuccess) {
        cudaGetLastError();
        mr_set_error("mr_b200_op_autotune: cudaMemsetAsync failed");
        rc = MR_ERR_CUDA;
    }
    if (rc == MR_SUCCESS)
        rc = mr_plan_autotune(op->plan, buf, op->S, op_kernel_ref(op), op->mask,
                              buf + vb / sizeof(float2), reps, ms);
    if (buf) {
        cudaStreamSynchronize(op->stream);
        cudaFree(buf);
    }
    if (prev != op->dev) cudaSetDevice(prev);
    return rc;
}

extern "C" int mr_b200_op_blocked_copy(mr_op op, int enable, int *built) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr, "mr_b200_op_blocked_copy: op is NULL");
    if (op->nu) {
        if (built) *built = 0;
        return MR_SUCCESS;
    }
    int prev = 0;
    MR_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != op->dev) MR_CUDA_TRY(cudaSetDevice(op->dev));
    if (enable) op_build_blocked(op);
    else op_free_blocked(op);
    if (prev != op->dev) cudaSetDevice(prev);
    if (built) *built = op->K_blk != nullptr && op->blk_kf == op->kf;
    return MR_SUCCESS;
}

extern "C" int mr_b200_op_device_bytes(mr_op op, uint64_t *bytes) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && bytes != nullptr, "mr_b200_op_device_bytes: NULL argument");
    const mr_config *c = &op->cfg;
    const uint64_t nloc = c->is_masked ? (uint64_t)c->num_masked : (uint64_t)mr_pad_size(c);
    const uint64_t ntri = (uint64_t)mr_num_tri(c->L);
    uint64_t b = op->plan ? mr_plan_device_bytes(op->plan) : 0;
    if (op->K_own) b += nloc * ntri * sizeof(float2);
    if (op->K16) b += nloc * ntri * 4 + nloc * sizeof(float);
    if (op->K_blk) b += op_blocked_bytes(c, op->blk_kf);
    if (op->S_own) b += (uint64_t)mr_se_size(c) * sizeof(float2);
    if (op->mask_own) b += (uint64_t)c->num_masked * sizeof(int64_t);
    b += mr_nufft_op_bytes(op->nu);
    *bytes = b;
    return MR_SUCCESS;
}

extern "C" int mr_b200_op_device_status(mr_op op, int *status) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && status != nullptr, "mr_b200_op_device_status: NULL argument");
    *status = 0;
    if (!op->plan) return MR_SUCCESS;
    int prev = -1;
    int rc = mr_push_device(&op->cfg, &prev);
    if (rc == MR_SUCCESS) rc = mr_plan_device_status(op->plan, status);
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_b200_op_launches(mr_op op, int *n) {
    mr_clear_error();
    MR_REQUIRE(op != nullptr && n != nullptr, "mr_b200_op_launches: NULL argument");
    // NUFFT operator: per coil, 4 (+2 for a stack) kernels around the NUFFTs,
    // each NUFFT 5 (2-D) or 6 (3-D) kernels per plane chunk
    *n = op->plan ? mr_plan_launch_count(op->plan) : 0;
    return MR_SUCCESS;
}
