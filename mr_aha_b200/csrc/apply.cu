// Stateless apply plan: mr_aha_plan_create / execute / destroy and the
// one-shot mr_aha_toeplitz (reference src/cuda/mr_aha.cu:375-834).
//
// Data flow of one execute, per coil group of G coils (P = G * L planes,
// plane p = c * L + l), for an image [Nx, Ny, Nz] and grid [Mx, My, Mz]:
//
//   pass 1 (3D / stack): z lines. Reads x and SEs, forms S_c x_l, transforms
//          along z (zero-padded to Mz) -> W0 [P][Mz][Ny][Nx].
//   pass 2: y lines. Reads W0 (or, in 2D, x * SEs directly), transforms
//          along y (zero-padded to My) -> W1 [P][Mz][My][Nx].
//   pass 3: x lines. Reads W1 rows, transforms along x (zero-padded to Mx),
//          multiplies every frequency's rank vector of every coil by the
//          packed Hermitian block, transforms back and crops to Nx -> W1
//          (in place).
//   pass 4: y lines back, cropped to Ny -> W0 (2D: conj(S_c) coil sum into
//          the output).
//   pass 5 (3D / stack): z lines back, cropped to Nz, multiplied by
//          conj(S_c) and summed over the group's coils into the output.
//
// The full upsampled spectrum is never written to memory: x is the last
// forward and first inverse axis, so only half-padded intermediates
// (Mz*My*Nx and Mz*Ny*Nx per plane) go through HBM. When the L lines of one
// coil do not fit in shared memory, pass 3 falls back to a plain x transform
// into a full-grid buffer, a stand-alone block multiply and a plain inverse.
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <nvtx3/nvToolsExt.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

struct mr_aha_plan_s {
    mr_config cfg;
    mr_geom g;
    cudaStream_t stream;
    int group;       // coils per group
    mr_fft_axis ax[3];
    float2 *d_tw;    // twiddle tables of the three axes
    int *d_status;   // device status word (MR_DEV_ERR_*), after the tables; NULL if none
    float2 *W0, *W1; // intermediates
    float2 *W2, *W3; // unfused pass 3 only: full-grid spectrum in / out
    int *d_inv;      // masked: natural grid index -> mask row
    int fused;       // pass 3 with the block multiply inside
    int v1_fused;    // the ping-pong fused pass 3 fits shared memory
    int nc_cta;      // coils per CTA in the fused pass 3
    int xt_z, xt_y;  // strided tile widths
    // in-place kernels (passes2.cu): tile exponents per (axis, store mode),
    // -1 when unavailable; coils per block-diagonal tile, 0 when unavailable
    int xts_z_buf, xts_z_cs, xts_y_buf, xts_y_cs;
    int nc2;
    // compile-time-specialised kernels (passes3.cu): tile widths, 0 if none
    int xt3_z_buf, xt3_z_cs, xt3_y_buf, xt3_y_cs;
    int nc3;
    // y inverse into the z buffer (3-D): its own tile choice, first equal
    // to the y forward one (the autotuner may separate them)
    int xts_yi, xt3_yi;
    // half-length y passes (3-D / stack, My = 2 Ny): tile widths of the
    // forward and inverse pass, both 0 when not used (they go together)
    int yh_f, yh_i;
    int nch;         // coils per tile of the half-length pass 3, 0 if none
    int launches;    // kernels per execute (accounting)
};

static void plan_apply_tuned(mr_aha_plan p);

// Choose the in-place kernels where the lengths allow them.
static void plan_pick_v2(mr_aha_plan p, size_t lim) {
    const mr_geom &g = p->g;
    const bool off = mr_env_int("MR_AHA_B200_FFT_V1", 0) != 0;
    p->xts_z_buf = p->xts_z_cs = p->xts_y_buf = p->xts_y_cs = -1;
    p->nc2 = 0;
    p->yh_f = p->yh_i = 0;
    if (off) return;
    if (p->ax[2].small) {
        p->xts_z_buf = mr_strided2_xts(g.m[2], g.m[2], MR_SM_BUF, g.n[0], lim);
        p->xts_z_cs = mr_strided2_xts(g.m[2], g.n[2], MR_SM_COILSUM, g.n[0], lim);
    }
    if (p->ax[1].small) {
        p->xts_y_buf = mr_strided2_xts(g.m[1], g.m[1], MR_SM_BUF, g.n[0], lim);
        p->xts_y_cs = mr_strided2_xts(g.m[1], g.n[1], MR_SM_COILSUM, g.n[0], lim);
    }
    if (p->ax[0].small && p->fused) p->nc2 = mr_xbd2_coils(g.m[0], g.L, p->cfg.n_coils, lim);
    p->xt3_z_buf = p->xt3_z_cs = p->xt3_y_buf = p->xt3_y_cs = 0;
    p->nc3 = p->nch = 0;
    p->xts_yi = p->xts_y_buf;
    p->xt3_yi = 0;
    if (mr_env_int("MR_AHA_B200_NO_FIXED", 0)) return;
    // tile widths may be forced per axis (tuning): MR_AHA_B200_XT_Z, _XT_Y.
    // Short z lines run fastest in narrow tiles (small CTAs, four per SM):
    // 32 columns of 56-point lines measured 5.3 ms (first pass) and 5.2 ms
    // (last pass) against 9.4 and 8.3 ms for 256 / 128 columns at
    // 320 x 320 x 56, L = 16, 12 coils.
    const int wz = mr_env_int("MR_AHA_B200_XT_Z", 0), wy = mr_env_int("MR_AHA_B200_XT_Y", 0);
    const int wz0 = wz ? wz : (g.m[2] <= 64 ? 32 : 0);
    p->xt3_z_buf = mr_fixed_strided_xt(g.m[2], MR_SM_BUF, wz0);
    p->xt3_z_cs = mr_fixed_strided_xt(g.m[2], MR_SM_COILSUM, wz0);
    p->xt3_y_buf = mr_fixed_strided_xt(g.m[1], MR_SM_BUF, wy);
    p->xt3_y_cs = mr_fixed_strided_xt(g.m[1], MR_SM_COILSUM, wy);
    if (p->fused) p->nc3 = mr_fixed_xbd_coils(g.m[0], g.L);
    // pass 3 pads x by cn[0] and crops the same window
    if (p->fused) p->nch = mr_fixed_xbdh_coils(g.m[0], g.n[0], g.L);
    p->xt3_yi = p->xt3_y_buf;
    p->yh_f = p->yh_i = 0;
    if (p->cfg.n_spatial == 3 && g.m[1] == 2 * g.n[1]) {
        // measured at 320 x 320 x 56, L = 16, 12 coils: forward 8.2 ms with
        // 8-column tiles (8.8 with 16), inverse 6.6 ms with 16 (7.2 with 8)
        p->yh_f = mr_half_strided_xt(g.n[1], wy ? wy : 8);
        const int wyi = mr_env_int("MR_AHA_B200_XT_YI", 0);  // inverse only (tuning)
        p->yh_i = p->yh_f > 0 ? mr_half_strided_xt(g.n[1], wyi ? wyi : (wy ? wy : 16)) : 0;
        if (p->yh_i == 0) p->yh_f = 0;
    }
}

// ---------------------------------------------------------------------------
// Stand-alone block multiply over a full-grid buffer (unfused pass 3)
// ---------------------------------------------------------------------------

template <int KF>
__global__ void __launch_bounds__(256) k_bd_full(const float2 *__restrict__ in,
                                                 float2 *__restrict__ out, mr_geom g,
                                                 mr_kernel_ref K, int ncoil) {
    const int64_t vpad = g.vpad;
    const int64_t total = vpad * ncoil * g.L;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = w % vpad;
        const int64_t rest = w / vpad;
        const int c = (int)(rest % g.L);
        const int k = (int)(rest / g.L);
        const int jx = (int)(q % g.m[0]);
        const int jy = (int)((q / g.m[0]) % g.m[1]);
        const int jz = (int)(q / ((int64_t)g.m[0] * g.m[1]));
        int64_t row;
        bool zero = false;
        if (K.inv) {
            const int r = __ldg(K.inv + q);
            zero = r < 0;
            row = zero ? 0 : r;
        } else {
            row = mr_nat2cent_d(jx, g.m[0], g.cm[0]) +
                  (int64_t)g.m[0] * (mr_nat2cent_d(jy, g.m[1], g.cm[1]) +
                                     (int64_t)g.m[1] * mr_nat2cent_d(jz, g.m[2], g.cm[2]));
        }
        float2 y = make_float2(0.f, 0.f);
        if (!zero) {
            const mr_kload<KF> kl = mr_kload_at<KF>(K, row);
            y = bd_one<KF>(in + (int64_t)k * g.L * vpad + q, vpad, g.L, c, kl, g.upper);
        }
        out[w] = y;
    }
}

static int launch_bd_full(const float2 *in, float2 *out, const mr_geom &g,
                          const mr_kernel_ref &K, int ncoil, cudaStream_t s) {
    const int64_t total = g.vpad * ncoil * g.L;
    const int64_t blocks = std::min<int64_t>(mr_cdiv(total, 256), 148 * 64);
    switch (K.kf) {
        case MR_KF_F32: k_bd_full<MR_KF_F32><<<(unsigned)blocks, 256, 0, s>>>(in, out, g, K, ncoil); break;
        case MR_KF_BF16: k_bd_full<MR_KF_BF16><<<(unsigned)blocks, 256, 0, s>>>(in, out, g, K, ncoil); break;
        case MR_KF_I16: k_bd_full<MR_KF_I16><<<(unsigned)blocks, 256, 0, s>>>(in, out, g, K, ncoil); break;
        default: MR_FAIL(MR_ERR_INTERNAL, "unknown kernel format");
    }
    MR_LAUNCH_CHECK("k_bd_full");
    return MR_SUCCESS;
}

// Grid -> mask row map (reference mr_kernels.cu:259-278): entries outside
// the mask stay -1 from the preceding memset.
__global__ void k_mask_inverse(int *inv, const int64_t *__restrict__ mask, int64_t nm,
                               mr_geom g) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nm) return;
    int64_t c = mask[i];
    if (c < 0 || c >= g.vpad) return;  // not a grid location
    const int kx = (int)(c % g.m[0]);
    c /= g.m[0];
    const int ky = (int)(c % g.m[1]);
    const int kz = (int)(c / g.m[1]);
    auto c2n = [](int k, int M, int cm) {
        const int j = k - cm;
        return j < 0 ? j + M : j;
    };
    const int64_t nat = c2n(kx, g.m[0], g.cm[0]) +
                        (int64_t)g.m[0] * (c2n(ky, g.m[1], g.cm[1]) +
                                           (int64_t)g.m[1] * c2n(kz, g.m[2], g.cm[2]));
    inv[nat] = (int)i;
}

// ---------------------------------------------------------------------------
// Plan construction
// ---------------------------------------------------------------------------

static void plan_release(mr_aha_plan p) {
    if (p->d_tw) cudaFree(p->d_tw);
    if (p->W0) cudaFree(p->W0);
    if (p->W1) cudaFree(p->W1);
    if (p->W2) cudaFree(p->W2);
    if (p->W3) cudaFree(p->W3);
    if (p->d_inv) cudaFree(p->d_inv);
    p->d_tw = nullptr;
    p->d_status = nullptr;
    p->W0 = p->W1 = p->W2 = p->W3 = nullptr;
    p->d_inv = nullptr;
    cudaGetLastError();
}

static size_t plan_bytes(const mr_aha_plan p, int group) {
    const mr_geom &g = p->g;
    const size_t P = (size_t)group * g.L;
    const bool has_z = p->cfg.n_spatial == 3;
    size_t b = P * g.m[2] * g.m[1] * g.n[0];                // W1
    if (has_z) b += P * g.m[2] * g.n[1] * g.n[0];           // W0
    if (!p->fused) b += 2 * P * (size_t)g.vpad;             // W2, W3
    b *= sizeof(float2);
    if (p->cfg.is_masked) b += (size_t)g.vpad * sizeof(int);
    return b;
}

int mr_plan_half_pass3(mr_aha_plan p) {
    return p->fused && p->nch > 0 && p->g.m[0] % 32 == 0;
}

size_t mr_plan_device_bytes(mr_aha_plan p) {
    const mr_geom &g = p->g;
    return plan_bytes(p, p->group) + (size_t)(g.m[0] + g.m[1] + g.m[2]) * sizeof(float2);
}

static int plan_alloc(mr_aha_plan p, int group) {
    const mr_geom &g = p->g;
    const size_t P = (size_t)group * g.L;
    const bool has_z = p->cfg.n_spatial == 3;
    cudaError_t e = cudaSuccess;
    if (has_z) e = cudaMalloc(&p->W0, P * g.m[2] * g.n[1] * g.n[0] * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&p->W1, P * g.m[2] * g.m[1] * g.n[0] * sizeof(float2));
    if (e == cudaSuccess && !p->fused) e = cudaMalloc(&p->W2, P * g.vpad * sizeof(float2));
    if (e == cudaSuccess && !p->fused) e = cudaMalloc(&p->W3, P * g.vpad * sizeof(float2));
    if (e == cudaSuccess && p->cfg.is_masked) e = cudaMalloc(&p->d_inv, g.vpad * sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (p->W0) cudaFree(p->W0);
        if (p->W1) cudaFree(p->W1);
        if (p->W2) cudaFree(p->W2);
        if (p->W3) cudaFree(p->W3);
        if (p->d_inv) cudaFree(p->d_inv);
        p->W0 = p->W1 = p->W2 = p->W3 = nullptr;
        p->d_inv = nullptr;
        MR_FAIL(MR_ERR_ALLOC, "failed to allocate the work buffers for a group of %d coil(s): %s",
                group, cudaGetErrorString(e));
    }
    p->group = group;
    return MR_SUCCESS;
}

static int plan_create_impl(const mr_config *cfg, mr_aha_plan *out) {
    int rc = mr_config_validate(cfg);
    if (rc != MR_SUCCESS) return rc;
    mr_aha_plan p = (mr_aha_plan)calloc(1, sizeof(struct mr_aha_plan_s));
    if (!p) MR_FAIL(MR_ERR_ALLOC, "failed to allocate the plan struct");
    p->cfg = *cfg;
    p->stream = (cudaStream_t)cfg->stream;
    mr_geom_from_config(cfg, &p->g);
    const mr_geom &g = p->g;

    // FFT factorisations and twiddle tables of the three axes.
    int off[3], tot = 0;
    for (int d = 0; d < 3; ++d) {
        rc = mr_fft_factor(g.m[d], &p->ax[d]);
        if (rc != MR_SUCCESS) {
            free(p);
            return rc;
        }
        off[d] = tot;
        tot += g.m[d];
    }
    std::vector<float2> h(tot);
    for (int d = 0; d < 3; ++d) mr_fft_twiddles(g.m[d], h.data() + off[d]);
    // the tables, then one 16-byte slot for the device status word
    if (cudaMalloc(&p->d_tw, (tot + 2) * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        free(p);
        MR_FAIL(MR_ERR_ALLOC, "failed to allocate the FFT tables");
    }
    if (cudaMemcpy(p->d_tw, h.data(), tot * sizeof(float2), cudaMemcpyHostToDevice) !=
        cudaSuccess) {
        plan_release(p);
        free(p);
        MR_FAIL(MR_ERR_CUDA, "failed to upload the FFT tables");
    }
    for (int d = 0; d < 3; ++d) p->ax[d].tw = p->d_tw + off[d];
    p->d_status = reinterpret_cast<int *>(p->d_tw + tot);
    if (cudaMemset(p->d_status, 0, 2 * sizeof(float2)) != cudaSuccess) {
        plan_release(p);
        free(p);
        MR_FAIL(MR_ERR_CUDA, "failed to clear the plan's status word");
    }

    // Pass geometry: strided tile widths and the fused pass 3.
    const size_t lim = (size_t)mr_smem_limit();
    const size_t half = lim / 2;  // aim for two CTAs per SM on strided passes
    p->xt_z = mr_pick_xt(g.m[2], g.m[2], MR_SM_COILSUM, g.n[0], half);
    p->xt_y = mr_pick_xt(g.m[1], g.m[1], MR_SM_COILSUM, g.n[0], half);
    if (mr_strided_smem(g.m[2], p->xt_z, g.m[2], MR_SM_COILSUM) > lim ||
        mr_strided_smem(g.m[1], p->xt_y, g.m[1], MR_SM_COILSUM) > lim) {
        plan_release(p);
        free(p);
        MR_FAIL(MR_ERR_UNSUPPORTED, "an FFT line of %d / %d points exceeds shared memory",
                g.m[1], g.m[2]);
    }
    p->nc_cta = 1;
    // fused pass 3 when a fused kernel fits: the ping-pong one, or the
    // half-length one (half the shared memory; M = 2N only)
    p->v1_fused = mr_xbd_smem(g.m[0], g.L, 1) <= lim;
    p->fused = p->v1_fused || (mr_env_int("MR_AHA_B200_NO_FIXED", 0) == 0 &&
                               mr_fixed_xbdh_coils(g.m[0], g.n[0], g.L) > 0);
    if (p->fused && g.L <= 16 && mr_xbd_smem(g.m[0], g.L, 2) <= lim && cfg->n_coils >= 2)
        p->nc_cta = 2;
    if (!p->fused && mr_xplain_smem(g.m[0], 1) > lim) {
        plan_release(p);
        free(p);
        MR_FAIL(MR_ERR_UNSUPPORTED, "an FFT line of %d points exceeds shared memory", g.m[0]);
    }
    if (mr_env_int("MR_AHA_B200_UNFUSED_BD", 0)) p->fused = 0;
    plan_pick_v2(p, lim);

    // Coil group: all coils if they fit the budget, else fewer.
    size_t budget = 0;
    rc = mr_memory_budget(cfg, &budget);
    if (rc != MR_SUCCESS) {
        plan_release(p);
        free(p);
        return rc;
    }
    int group = mr_env_int("MR_AHA_CUDA_COIL_GROUP", cfg->n_coils);
    if (group < 1 || group > cfg->n_coils) group = cfg->n_coils;
    while (group > 1 && plan_bytes(p, group) > budget) --group;
    for (;; --group) {
        rc = plan_alloc(p, group);
        if (rc == MR_SUCCESS || group == 1) break;
    }
    if (rc != MR_SUCCESS) {
        plan_release(p);
        free(p);
        return rc;
    }
    mr_clear_error();
    const int ngroups = (int)mr_cdiv(cfg->n_coils, group);
    const int per = (cfg->n_spatial == 3 ? 2 : 0) + 2 + (p->fused ? 1 : 3);
    p->launches = ngroups * per + (cfg->is_masked ? 1 : 0);
    plan_apply_tuned(p);
    if (cfg->verbose)
        printf("[mr_aha] plan: %s block multiply, %d coil(s) per group, tiles z %d y %d\n",
               p->fused ? "fused" : "stand-alone", p->group, p->xt_z, p->xt_y);
    *out = p;
    return MR_SUCCESS;
}

extern "C" int mr_aha_plan_create(const mr_config *cfg, mr_aha_plan *plan_out) {
    mr_clear_error();
    MR_REQUIRE(plan_out != nullptr, "mr_aha_plan_create: plan_out is NULL");
    *plan_out = nullptr;
    MR_REQUIRE(cfg != nullptr, "mr_aha_plan_create: cfg is NULL");
    int prev = -1;
    int rc = mr_push_device(cfg, &prev);
    if (rc == MR_SUCCESS) rc = plan_create_impl(cfg, plan_out);
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_aha_plan_destroy(mr_aha_plan plan) {
    mr_clear_error();
    if (!plan) return MR_SUCCESS;
    int prev = -1;
    (void)mr_push_device(&plan->cfg, &prev);
    plan_release(plan);
    mr_pop_device(prev);
    free(plan);
    return MR_SUCCESS;
}

int mr_plan_group(mr_aha_plan plan) { return plan->group; }
cudaStream_t mr_plan_stream(mr_aha_plan plan) { return plan->stream; }
int mr_plan_launch_count(mr_aha_plan plan) { return plan->launches; }

int mr_plan_device_status(mr_aha_plan p, int *status) {
    *status = 0;
    if (!p->d_status) return MR_SUCCESS;
    MR_CUDA_TRY(cudaStreamSynchronize(p->stream));
    MR_CUDA_TRY(cudaMemcpy(status, p->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    MR_CUDA_TRY(cudaMemset(p->d_status, 0, sizeof(int)));
    return MR_SUCCESS;
}

// ---------------------------------------------------------------------------
// Execution
// ---------------------------------------------------------------------------

// Strided pass with the in-place kernel when available (xts >= 0), else the
// ping-pong kernel with tile width xt_v1.
static int launch_strided_auto(int dir, int lm, int sm, mr_strided_args a, int xts, int xt_v1,
                               cudaStream_t s, int xt3 = 0) {
    if (xt3 > 0) {
        a.xt = xt3;
        a.nxt = (int)mr_cdiv(a.nfast, a.xt);
        return mr_launch_strided3(dir, lm, sm, a, s);
    }
    if (xts >= 0) {
        a.xt = 1 << xts;
        a.nxt = (int)mr_cdiv(a.nfast, a.xt);
        return mr_launch_strided2(dir, lm, sm, a, xts, s);
    }
    a.xt = xt_v1;
    a.nxt = (int)mr_cdiv(a.nfast, a.xt);
    return mr_launch_strided(dir, lm, sm, a, s);
}

// Host-side NVTX ranges of one execute ("mr_aha apply" > pass name, shown
// in Nsight Systems timelines; NVTX calls return at once when no tool is
// attached). Ranges still open at an early error return are closed on exit.
struct nvtx_scope {
    int depth = 0;
    void push(const char *name) {
        nvtxRangePushA(name);
        ++depth;
    }
    void pop() {
        if (depth > 0) {
            nvtxRangePop();
            --depth;
        }
    }
    ~nvtx_scope() {
        while (depth > 0) pop();
    }
};

// End of a pass: an event for mr_b200_op_profile and the end of its range.
static void prof_mark(mr_prof *prof, nvtx_scope &nv, const char *name, cudaStream_t s) {
    nv.pop();
    if (!prof || prof->n >= MR_PROF_MAX) return;
    prof->name[prof->n] = name;
    cudaEventRecord(prof->ev[++prof->n], s);
}

int mr_plan_execute_k(mr_aha_plan p, const float2 *x, const float2 *S,
                      const mr_kernel_ref &K0, const int64_t *d_mask, float2 *out,
                      cudaStream_t s, mr_prof *prof) {
    if (prof) {
        prof->n = 0;
        cudaEventRecord(prof->ev[0], s);
    }
    const mr_config &cfg = p->cfg;
    const mr_geom &g = p->g;
    const bool has_z = cfg.n_spatial == 3;
    const int Nx = g.n[0], Ny = g.n[1], Nz = g.n[2];
    const int Mx = g.m[0], My = g.m[1], Mz = g.m[2];
    mr_kernel_ref K = K0;
    int rc;

    nvtx_scope nv;
    nv.push("mr_aha apply");
    if (cfg.is_masked) {
        nv.push("mask_inverse");
        const int64_t nm = cfg.num_masked;
        MR_CUDA_TRY(cudaMemsetAsync(p->d_inv, 0xFF, g.vpad * sizeof(int), s));
        k_mask_inverse<<<(unsigned)mr_cdiv(nm, 256), 256, 0, s>>>(p->d_inv, d_mask, nm, g);
        MR_LAUNCH_CHECK("k_mask_inverse");
        K.inv = p->d_inv;
        K.stride = nm;
        // a blocked copy of a masked kernel is in grid order (zero outside
        // the mask); pass 3 still skips the locations outside the mask
        prof_mark(prof, nv, "mask_inverse", s);
    } else {
        K.inv = nullptr;
        K.stride = g.vpad;
    }

    for (int c0 = 0; c0 < cfg.n_coils; c0 += p->group) {
        const int G = std::min(p->group, cfg.n_coils - c0);
        const int P = G * g.L;
        const int accumulate = c0 > 0;
        const int64_t w0_plane = (int64_t)Mz * Ny * Nx;
        const int64_t w1_plane = (int64_t)Mz * My * Nx;

        // ---- pass 1: z lines, S_c x_l, zero-pad along z ----
        if (has_z) {
            nv.push("z_forward");
            mr_strided_args a;
            std::memset(&a, 0, sizeof(a));
            a.status = p->d_status;
            // z lines: the (y, x) plane is contiguous, so tiles run over the
            // flattened plane index
            a.ax = p->ax[2];
            a.nfast = Nx * Ny;
            a.nouter = 1;
            a.nplane = P;
            a.s_outer = 0;
            a.s_axis = (int64_t)Nx * Ny;
            a.n_in = Nz;
            a.shift_in = g.cn[2];
            a.xs_x = x;
            a.xs_s = S;
            a.img_plane = g.vimg;
            a.L = g.L;
            a.coil0 = c0;
            a.dst = p->W0;
            a.d_plane = w0_plane;
            a.d_outer = 0;
            a.d_axis = (int64_t)Ny * Nx;
            a.n_out = Mz;
            a.shift_out = 0;
            a.scale = 1.f;
            rc = launch_strided_auto(-1, MR_LM_XS, MR_SM_BUF, a, p->xts_z_buf, p->xt_z, s,
                                     p->xt3_z_buf);
            if (rc != MR_SUCCESS) return rc;
            prof_mark(prof, nv, "z_forward", s);
        }
        // ---- pass 2: y lines, zero-pad along y ----
        {
            nv.push("y_forward");
            mr_strided_args a;
            std::memset(&a, 0, sizeof(a));
            a.status = p->d_status;
            a.ax = p->ax[1];
            a.nfast = Nx;
            a.xt = p->xt_y;
            a.nxt = (int)mr_cdiv(Nx, a.xt);
            a.nouter = Mz;
            a.nplane = P;
            a.n_in = Ny;
            a.shift_in = g.cn[1];
            a.L = g.L;
            a.coil0 = c0;
            a.img_plane = g.vimg;
            a.dst = p->W1;
            a.d_plane = w1_plane;
            a.d_outer = (int64_t)My * Nx;
            a.d_axis = Nx;
            a.n_out = My;
            a.shift_out = 0;
            a.scale = 1.f;
            if (has_z) {
                a.src = p->W0;
                a.s_plane = w0_plane;
                a.s_outer = (int64_t)Ny * Nx;
                a.s_axis = Nx;
                if (p->yh_f > 0) {
                    a.xt = p->yh_f;
                    a.nxt = (int)mr_cdiv(Nx, a.xt);
                    rc = mr_launch_strided_half(-1, a, s);
                } else {
                    rc = launch_strided_auto(-1, MR_LM_BUF, MR_SM_BUF, a, p->xts_y_buf, p->xt_y,
                                             s, p->xt3_y_buf);
                }
            } else {
                a.xs_x = x;
                a.xs_s = S;
                a.s_outer = 0;
                a.s_axis = Nx;
                rc = launch_strided_auto(-1, MR_LM_XS, MR_SM_BUF, a, p->xts_y_buf, p->xt_y, s,
                                         p->xt3_y_buf);
            }
            if (rc != MR_SUCCESS) return rc;
            prof_mark(prof, nv, "y_forward", s);
        }
        // ---- pass 3: x lines with the block multiply ----
        {
            mr_x_args a;
            std::memset(&a, 0, sizeof(a));
            a.ax = p->ax[0];
            a.scale = 1.f;
            if (p->fused) {
                nv.push("x_blockdiag");
                a.src = p->W1;
                a.dst = p->W1;
                a.s_row = Nx;
                a.d_row = Nx;
                a.n_in = Nx;
                a.shift_in = g.cn[0];
                a.n_out = Nx;
                a.shift_out = g.cn[0];
                a.plane_rows = (int64_t)My * Mz;
                a.nloc = My * Mz;
                a.nc = p->nc_cta;
                a.ncoil = G;
                a.nchunk = (int)mr_cdiv(G, a.nc);
                a.L = g.L;
                a.upper = g.upper;
                a.My = My;
                a.Mz = Mz;
                a.cmx = g.cm[0];
                a.cmy = g.cm[1];
                a.cmz = g.cm[2];
                a.K = K;
                a.status = p->d_status;
                if (p->nch > 0) {
                    a.nc = p->nch;
                    a.nchunk = (int)mr_cdiv(G, a.nc);
                    rc = mr_launch_xbdh(a, s);
                } else if (p->nc3 > 0) {
                    a.nc = p->nc3;
                    a.nchunk = (int)mr_cdiv(G, a.nc);
                    rc = mr_launch_xbd3(a, s);
                } else if (p->nc2 > 0) {
                    a.nc = p->nc2;
                    a.nchunk = (int)mr_cdiv(G, a.nc);
                    rc = mr_launch_xbd2(a, s);
                } else {
                    if (!p->v1_fused)
                        MR_FAIL(MR_ERR_INTERNAL, "no fused pass-3 kernel fits this geometry");
                    rc = mr_launch_xbd(a, s);
                }
                if (rc != MR_SUCCESS) return rc;
                prof_mark(prof, nv, "x_blockdiag", s);
            } else {
                nv.push("x_forward");
                const int rows = 4;
                a.rows_cta = rows;
                a.src = p->W1;
                a.dst = p->W2;
                a.s_row = Nx;
                a.d_row = Mx;
                a.nrows = (int64_t)P * My * Mz;
                a.n_in = Nx;
                a.shift_in = g.cn[0];
                a.n_out = Mx;
                a.shift_out = 0;
                rc = mr_launch_xplain(-1, a, s);
                if (rc != MR_SUCCESS) return rc;
                prof_mark(prof, nv, "x_forward", s);
                nv.push("blockdiag");
                rc = launch_bd_full(p->W2, p->W3, g, K, G, s);
                if (rc != MR_SUCCESS) return rc;
                prof_mark(prof, nv, "blockdiag", s);
                nv.push("x_inverse");
                a.src = p->W3;
                a.dst = p->W1;
                a.s_row = Mx;
                a.d_row = Nx;
                a.n_in = Mx;
                a.shift_in = 0;
                a.n_out = Nx;
                a.shift_out = g.cn[0];
                rc = mr_launch_xplain(1, a, s);
                if (rc != MR_SUCCESS) return rc;
                prof_mark(prof, nv, "x_inverse", s);
            }
        }
        // ---- pass 4: y lines back, crop ----
        {
            nv.push("y_inverse");
            mr_strided_args a;
            std::memset(&a, 0, sizeof(a));
            a.status = p->d_status;
            a.ax = p->ax[1];
            a.nfast = Nx;
            a.xt = p->xt_y;
            a.nxt = (int)mr_cdiv(Nx, a.xt);
            a.nouter = Mz;
            a.src = p->W1;
            a.s_plane = w1_plane;
            a.s_outer = (int64_t)My * Nx;
            a.s_axis = Nx;
            a.n_in = My;
            a.shift_in = 0;
            a.n_out = Ny;
            a.shift_out = g.cn[1];
            a.L = g.L;
            a.coil0 = c0;
            a.img_plane = g.vimg;
            a.scale = 1.f;
            if (has_z) {
                a.nplane = P;
                a.dst = p->W0;
                a.d_plane = w0_plane;
                a.d_outer = (int64_t)Ny * Nx;
                a.d_axis = Nx;
                if (p->yh_i > 0) {
                    a.xt = p->yh_i;
                    a.nxt = (int)mr_cdiv(Nx, a.xt);
                    rc = mr_launch_strided_half(1, a, s);
                } else {
                    rc = launch_strided_auto(1, MR_LM_BUF, MR_SM_BUF, a, p->xts_yi, p->xt_y, s,
                                             p->xt3_yi);
                }
            } else {
                a.nplane = g.L;
                a.xs_s = S;
                a.dst = out;
                a.d_plane = g.vimg;
                a.d_outer = 0;
                a.d_axis = Nx;
                a.ncoil = G;
                a.accumulate = accumulate;
                rc = launch_strided_auto(1, MR_LM_BUF, MR_SM_COILSUM, a, p->xts_y_cs, p->xt_y, s,
                                         p->xt3_y_cs);
            }
            if (rc != MR_SUCCESS) return rc;
            prof_mark(prof, nv, "y_inverse", s);
        }
        // ---- pass 5: z lines back, crop, conj(S_c) coil sum ----
        if (has_z) {
            nv.push("z_inverse");
            mr_strided_args a;
            std::memset(&a, 0, sizeof(a));
            a.status = p->d_status;
            a.ax = p->ax[2];
            a.nfast = Nx * Ny;
            a.nouter = 1;
            a.nplane = g.L;
            a.src = p->W0;
            a.s_plane = w0_plane;
            a.s_outer = 0;
            a.s_axis = (int64_t)Ny * Nx;
            a.n_in = Mz;
            a.shift_in = 0;
            a.n_out = Nz;
            a.shift_out = g.cn[2];
            a.L = g.L;
            a.coil0 = c0;
            a.xs_s = S;
            a.img_plane = g.vimg;
            a.dst = out;
            a.d_plane = g.vimg;
            a.d_outer = 0;
            a.d_axis = (int64_t)Ny * Nx;
            a.ncoil = G;
            a.accumulate = accumulate;
            a.scale = 1.f;
            rc = launch_strided_auto(1, MR_LM_BUF, MR_SM_COILSUM, a, p->xts_z_cs, p->xt_z, s,
                                     p->xt3_z_cs);
            if (rc != MR_SUCCESS) return rc;
            prof_mark(prof, nv, "z_inverse", s);
        }
    }
    if (cfg.verbose) {
        MR_CUDA_TRY(cudaStreamSynchronize(s));
        printf("[mr_aha] AhA applied over %d coil(s) in groups of %d, grid [%d %d %d] -> "
               "[%d %d %d], L = %d%s\n",
               cfg.n_coils, p->group, Nx, Ny, Nz, Mx, My, Mz, g.L,
               cfg.is_masked ? ", masked" : "");
    }
    return MR_SUCCESS;
}

extern "C" int mr_aha_plan_execute(mr_aha_plan plan, const mr_complex *d_x,
                                   const mr_complex *d_SEs,
                                   const mr_complex *d_phi2_toep, const int64_t *d_mask,
                                   mr_complex *d_AhAx) {
    mr_clear_error();
    MR_REQUIRE(plan != nullptr, "mr_aha_plan_execute: plan is NULL");
    MR_REQUIRE(d_x != nullptr, "mr_aha_plan_execute: d_x is NULL");
    MR_REQUIRE(d_SEs != nullptr, "mr_aha_plan_execute: d_SEs is NULL");
    MR_REQUIRE(d_phi2_toep != nullptr, "mr_aha_plan_execute: d_phi2_toep is NULL");
    MR_REQUIRE(d_AhAx != nullptr, "mr_aha_plan_execute: d_AhAx is NULL");
    MR_REQUIRE((const void *)d_AhAx != (const void *)d_x,
               "mr_aha_plan_execute: d_AhAx must not alias d_x");
    if (plan->cfg.is_masked)
        MR_REQUIRE(d_mask != nullptr,
                   "mr_aha_plan_execute: d_mask is required when is_masked is set");
    mr_kernel_ref K;
    std::memset(&K, 0, sizeof(K));
    K.data = d_phi2_toep;
    K.kf = MR_KF_F32;
    int prev = -1;
    int rc = mr_push_device(&plan->cfg, &prev);
    if (rc == MR_SUCCESS)
        rc = mr_plan_execute_k(plan, reinterpret_cast<const float2 *>(d_x),
                               reinterpret_cast<const float2 *>(d_SEs), K, d_mask,
                               reinterpret_cast<float2 *>(d_AhAx), plan->stream);
    mr_pop_device(prev);
    return rc;
}

extern "C" int mr_aha_toeplitz(const mr_config *cfg, const mr_complex *d_x,
                               const mr_complex *d_SEs, const mr_complex *d_phi2_toep,
                               const int64_t *d_mask, mr_complex *d_AhAx) {
    mr_aha_plan plan = nullptr;
    int rc = mr_aha_plan_create(cfg, &plan);
    if (rc != MR_SUCCESS) return rc;
    rc = mr_aha_plan_execute(plan, d_x, d_SEs, d_phi2_toep, d_mask, d_AhAx);
    // Work is asynchronous: make sure it finished before the buffers go.
    cudaStreamSynchronize(plan->stream);
    const int rc2 = mr_aha_plan_destroy(plan);
    return rc != MR_SUCCESS ? rc : rc2;
}

// ---------------------------------------------------------------------------
// Plan over caller-provided device scratch (used by the allocation-free
// entry point in noalloc.cu; nothing here allocates device memory)
// ---------------------------------------------------------------------------

// W_M^e = exp(-2 pi i e / M) for the three axes, into one table.
__global__ void k_twiddle_table(float2 *tw, int m0, int m1, int m2) {
    const int total = m0 + m1 + m2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        int M = m0, k = e;
        if (k >= m0) {
            k -= m0;
            M = m1;
            if (k >= m1) {
                k -= m1;
                M = m2;
            }
        }
        double s, c;
        sincospi(-2.0 * (double)k / (double)M, &s, &c);
        tw[e] = make_float2((float)c, (float)s);
    }
}

size_t mr_plan_struct_size() { return sizeof(struct mr_aha_plan_s); }

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int mr_plan_setup_in_scratch(const mr_config *cfg, char *scratch, size_t bytes, void *storage,
                             size_t *needed) {
    int rc = mr_config_validate(cfg);
    if (rc != MR_SUCCESS) return rc;
    mr_aha_plan p = (mr_aha_plan)storage;
    std::memset(p, 0, sizeof(*p));
    p->cfg = *cfg;
    p->stream = (cudaStream_t)cfg->stream;
    mr_geom_from_config(cfg, &p->g);
    const mr_geom &g = p->g;
    for (int d = 0; d < 3; ++d) {
        rc = mr_fft_factor(g.m[d], &p->ax[d]);
        if (rc != MR_SUCCESS) return rc;
    }
    const size_t lim = (size_t)mr_smem_limit();
    p->xt_z = mr_pick_xt(g.m[2], g.m[2], MR_SM_COILSUM, g.n[0], lim / 2);
    p->xt_y = mr_pick_xt(g.m[1], g.m[1], MR_SM_COILSUM, g.n[0], lim / 2);
    if (mr_strided_smem(g.m[2], p->xt_z, g.m[2], MR_SM_COILSUM) > lim ||
        mr_strided_smem(g.m[1], p->xt_y, g.m[1], MR_SM_COILSUM) > lim)
        MR_FAIL(MR_ERR_UNSUPPORTED, "an FFT line of %d / %d points exceeds shared memory",
                g.m[1], g.m[2]);
    p->nc_cta = 1;
    p->fused = mr_xbd_smem(g.m[0], g.L, 1) <= lim;
    p->v1_fused = p->fused;
    if (p->fused && g.L <= 16 && mr_xbd_smem(g.m[0], g.L, 2) <= lim && cfg->n_coils >= 2)
        p->nc_cta = 2;
    if (!p->fused && mr_xplain_smem(g.m[0], 1) > lim)
        MR_FAIL(MR_ERR_UNSUPPORTED, "an FFT line of %d points exceeds shared memory", g.m[0]);
    plan_pick_v2(p, lim);
    // Layout: twiddles | inverse mask map | W0 | W1 | W2 | W3, each 256-byte aligned.
    const bool has_z = cfg->n_spatial == 3;
    const size_t tw_b = align256((size_t)(g.m[0] + g.m[1] + g.m[2]) * sizeof(float2));
    const size_t inv_b = cfg->is_masked ? align256((size_t)g.vpad * sizeof(int)) : 0;
    int group = cfg->n_coils;
    size_t w0_b = 0, w1_b = 0, wf_b = 0, total = 0;
    for (;; --group) {
        const size_t P = (size_t)group * g.L;
        w0_b = has_z ? align256(P * g.m[2] * g.n[1] * g.n[0] * sizeof(float2)) : 0;
        w1_b = align256(P * g.m[2] * g.m[1] * g.n[0] * sizeof(float2));
        wf_b = p->fused ? 0 : align256(P * (size_t)g.vpad * sizeof(float2));
        total = tw_b + inv_b + w0_b + w1_b + 2 * wf_b;
        if (total <= bytes || group == 1) break;
    }
    if (needed) *needed = total;
    if (total > bytes)
        MR_FAIL(MR_ERR_UNSUPPORTED,
                "this operator needs %zu bytes of work space even one coil at a time, more "
                "than the %zu bytes of the library's static scratch array",
                total, bytes);
    char *q = scratch;
    p->d_tw = (float2 *)q;
    q += tw_b;
    p->d_inv = cfg->is_masked ? (int *)q : nullptr;
    q += inv_b;
    p->W0 = has_z ? (float2 *)q : nullptr;
    q += w0_b;
    p->W1 = (float2 *)q;
    q += w1_b;
    p->W2 = p->fused ? nullptr : (float2 *)q;
    q += wf_b;
    p->W3 = p->fused ? nullptr : (float2 *)q;
    p->group = group;
    p->ax[0].tw = p->d_tw;
    p->ax[1].tw = p->d_tw + g.m[0];
    p->ax[2].tw = p->d_tw + g.m[0] + g.m[1];
    k_twiddle_table<<<(unsigned)mr_cdiv(g.m[0] + g.m[1] + g.m[2], 256), 256, 0, p->stream>>>(
        p->d_tw, g.m[0], g.m[1], g.m[2]);
    MR_LAUNCH_CHECK("k_twiddle_table");
    const int ngroups = (int)mr_cdiv(cfg->n_coils, group);
    const int per = (has_z ? 2 : 0) + 2 + (p->fused ? 1 : 3);
    p->launches = ngroups * per + (cfg->is_masked ? 1 : 0) + 1;
    return MR_SUCCESS;
}

// ---------------------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------------------
// The tunable choices of a plan: per strided pass the specialised kernel's
// tile width (xt3 > 0) or the in-place kernel's tile exponent (xts >= 0),
// and the pass-3 kernel (half-length nch / specialised nc3 / in-place nc2 /
// ping-pong). The tuner measures full applies, one choice at a time
// (coordinate descent, one sweep), and keeps each improvement; results are
// remembered per geometry for later plans in the process.

struct mr_tune_choice {
    int xt3_z_buf, xts_z_buf, xt3_z_cs, xts_z_cs, xt3_y_buf, xts_y_buf, xt3_yi, xts_yi;
    int xt3_y_cs, xts_y_cs, nch, nc3, nc2, yh_f, yh_i;
};

static mr_tune_choice tune_get(const mr_aha_plan p) {
    return {p->xt3_z_buf, p->xts_z_buf, p->xt3_z_cs, p->xts_z_cs, p->xt3_y_buf, p->xts_y_buf,
            p->xt3_yi,    p->xts_yi,    p->xt3_y_cs, p->xts_y_cs, p->nch,       p->nc3,
            p->nc2,       p->yh_f,      p->yh_i};
}

static void tune_set(mr_aha_plan p, const mr_tune_choice &c) {
    p->xt3_z_buf = c.xt3_z_buf;
    p->xts_z_buf = c.xts_z_buf;
    p->xt3_z_cs = c.xt3_z_cs;
    p->xts_z_cs = c.xts_z_cs;
    p->xt3_y_buf = c.xt3_y_buf;
    p->xts_y_buf = c.xts_y_buf;
    p->xt3_yi = c.xt3_yi;
    p->xts_yi = c.xts_yi;
    p->xt3_y_cs = c.xt3_y_cs;
    p->xts_y_cs = c.xts_y_cs;
    p->nch = c.nch;
    p->nc3 = c.nc3;
    p->nc2 = c.nc2;
    p->yh_f = c.yh_f;
    p->yh_i = c.yh_i;
}

static std::string tune_key(const mr_aha_plan p) {
    const mr_geom &g = p->g;
    char b[256];
    std::snprintf(b, sizeof(b), "t%d n%d,%d,%d m%d,%d,%d L%d C%d G%d k%d u%d f%d",
                  p->cfg.traj_type, g.n[0], g.n[1], g.n[2], g.m[0], g.m[1], g.m[2], g.L,
                  p->cfg.n_coils, p->group, p->cfg.is_masked, g.upper, p->fused);
    return b;
}

// Strided passes the autotuner sweeps: (xt3, xts) fields, axis length, store
// mode, whether the plan runs that pass.
struct mr_tune_knob {
    int mr_tune_choice::*xt3;
    int mr_tune_choice::*xts;
    int M, smode;
    bool on;
};

static void tune_knobs(const mr_aha_plan p, mr_tune_knob (&k)[5]) {
    const mr_geom &g = p->g;
    const bool has_z = p->cfg.n_spatial == 3;
    k[0] = {&mr_tune_choice::xt3_z_buf, &mr_tune_choice::xts_z_buf, g.m[2], MR_SM_BUF, has_z};
    k[1] = {&mr_tune_choice::xt3_y_buf, &mr_tune_choice::xts_y_buf, g.m[1], MR_SM_BUF, true};
    k[2] = {&mr_tune_choice::xt3_yi, &mr_tune_choice::xts_yi, g.m[1], MR_SM_BUF, has_z};
    k[3] = {&mr_tune_choice::xt3_y_cs, &mr_tune_choice::xts_y_cs, g.m[1], MR_SM_COILSUM, !has_z};
    k[4] = {&mr_tune_choice::xt3_z_cs, &mr_tune_choice::xts_z_cs, g.m[2], MR_SM_COILSUM, has_z};
}

static bool tune_in(int v, const int *l, int n) {
    for (int i = 0; i < n; ++i)
        if (l[i] == v) return true;
    return false;
}

// True when every field of c is a value the autotuner itself tries for this
// plan, whose fields still hold their defaults: a cached choice from a file
// is used only then, so a stale or edited line cannot select a kernel width
// or coil group the plan has no launch for.
static bool tune_valid(const mr_aha_plan p, const mr_tune_choice &c) {
    const mr_tune_choice d = tune_get(p);
    const mr_geom &g = p->g;
    const bool has_z = p->cfg.n_spatial == 3;
    const bool fixed_ok = mr_env_int("MR_AHA_B200_NO_FIXED", 0) == 0;
    // pass 3 coil grouping
    if (!p->fused) {
        if (c.nch != d.nch || c.nc3 != d.nc3 || c.nc2 != d.nc2) return false;
    } else {
        const int nch0 = fixed_ok ? mr_fixed_xbdh_coils(g.m[0], g.n[0], g.L) : 0;
        const int nc2_0 = p->ax[0].small && mr_env_int("MR_AHA_B200_FFT_V1", 0) == 0
                              ? mr_xbd2_coils(g.m[0], g.L, p->cfg.n_coils, (size_t)mr_smem_limit())
                              : 0;
        int ncs[8];
        const int nn = fixed_ok ? mr_fixed_xbd_list(g.m[0], g.L, ncs, 8) : 0;
        if (c.nch != d.nch && c.nch != 0 && c.nch != nch0) return false;
        if (c.nc3 != d.nc3 && c.nc3 != 0 && !tune_in(c.nc3, ncs, nn)) return false;
        if (c.nc2 != d.nc2 && c.nc2 != 0 && c.nc2 != nc2_0) return false;
        const bool d_v1 = d.nch == 0 && d.nc3 == 0 && d.nc2 == 0;
        if (c.nch == 0 && c.nc3 == 0 && c.nc2 == 0 && !d_v1 && !p->v1_fused) return false;
    }
    // half-length y passes
    if (has_z && g.m[1] == 2 * g.n[1] && mr_half_strided_xt(g.n[1], 0) > 0) {
        int ws[16];
        const int nw = mr_half_strided_list(g.n[1], ws, 16);
        if ((c.yh_f == 0) != (c.yh_i == 0)) return false;
        if (c.yh_f != d.yh_f && c.yh_f != 0 && !tune_in(c.yh_f, ws, nw)) return false;
        if (c.yh_i != d.yh_i && c.yh_i != 0 && !tune_in(c.yh_i, ws, nw)) return false;
    } else if (c.yh_f != d.yh_f || c.yh_i != d.yh_i) {
        return false;
    }
    // strided passes: a fixed width, or the generic kernel up to two steps
    // narrower than the default
    mr_tune_knob knobs[5];
    tune_knobs(p, knobs);
    for (const mr_tune_knob &k : knobs) {
        const int x3 = c.*k.xt3, xs = c.*k.xts, dx3 = d.*k.xt3, dxs = d.*k.xts;
        if (!k.on) {
            if (x3 != dx3 || xs != dxs) return false;
            continue;
        }
        int xts[16];
        const int nf = fixed_ok ? mr_fixed_strided_list(k.M, k.smode, xts, 16) : 0;
        if (x3 != dx3 && x3 != 0 && !tune_in(x3, xts, nf)) return false;
        if (xs != dxs && !(xs >= 0 && xs < dxs && xs >= dxs - 2)) return false;
    }
    return true;
}

static std::mutex g_tune_mu;
static std::map<std::string, mr_tune_choice> g_tuned;

// On-disk cache of tuned choices, shared by processes: the file named by
// MR_AHA_B200_TUNE_CACHE (none when unset), one line per geometry,
// "<device name>|<geometry key>|<the choices>". Lines of other devices or
// that do not parse are ignored; it is read once per process (under
// g_tune_mu) and rewritten whole (temporary file, then rename) after each
// autotune.
static const int kTuneFields = (int)(sizeof(mr_tune_choice) / sizeof(int));
static bool g_tune_loaded = false;

static std::string tune_device() {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    return prop.name;
}

static void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = std::getenv("MR_AHA_B200_TUNE_CACHE");
    if (!path || !path[0]) return;
    FILE *f = std::fopen(path, "r");
    if (!f) return;
    const std::string dev = tune_device();
    char line[1024];
    while (std::fgets(line, sizeof(line), f)) {
        std::string l(line);
        const size_t a = l.find('|'), b = l.find('|', a == std::string::npos ? a : a + 1);
        if (a == std::string::npos || b == std::string::npos || l.substr(0, a) != dev) continue;
        mr_tune_choice c;
        int *v = reinterpret_cast<int *>(&c);
        const char *q = l.c_str() + b + 1;
        int n = 0;
        for (; n < kTuneFields; ++n) {
            char *end = nullptr;
            const long x = std::strtol(q, &end, 10);
            if (end == q) break;
            v[n] = (int)x;
            q = end;
        }
        if (n == kTuneFields) g_tuned[l.substr(a + 1, b - a - 1)] = c;
    }
    std::fclose(f);
}

static void tune_save_locked() {
    const char *path = std::getenv("MR_AHA_B200_TUNE_CACHE");
    if (!path || !path[0]) return;
    const std::string dev = tune_device();
    // keep other devices' lines, replace this device's with the current map
    std::vector<std::string> keep;
    if (FILE *f = std::fopen(path, "r")) {
        char line[1024];
        while (std::fgets(line, sizeof(line), f)) {
            std::string l(line);
            const size_t a = l.find('|');
            if (a != std::string::npos && l.substr(0, a) != dev) keep.push_back(l);
        }
        std::fclose(f);
    }
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = std::fopen(tmp.c_str(), "w");
    if (!f) return;
    for (const std::string &l : keep) std::fputs(l.c_str(), f);
    for (const auto &kv : g_tuned) {
        std::fprintf(f, "%s|%s|", dev.c_str(), kv.first.c_str());
        const int *v = reinterpret_cast<const int *>(&kv.second);
        for (int n = 0; n < kTuneFields; ++n) std::fprintf(f, " %d", v[n]);
        std::fputc('\n', f);
    }
    const bool ok = std::fclose(f) == 0;
    if (ok) std::rename(tmp.c_str(), path);
    else std::remove(tmp.c_str());
}

// Tuned choices of an earlier plan of the same geometry (this process, or
// the on-disk cache), if any.
static void plan_apply_tuned(mr_aha_plan p) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tuned.find(tune_key(p));
    if (it != g_tuned.end() && tune_valid(p, it->second)) tune_set(p, it->second);
}

static int tune_time(mr_aha_plan p, const float2 *x, const float2 *S, const mr_kernel_ref &K,
                     const int64_t *mask, float2 *out, int reps, cudaEvent_t e0, cudaEvent_t e1,
                     float *ms) {
    cudaStream_t s = p->stream;
    int rc = mr_plan_execute_k(p, x, S, K, mask, out, s);
    if (rc != MR_SUCCESS) return rc;
    MR_CUDA_TRY(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) {
        rc = mr_plan_execute_k(p, x, S, K, mask, out, s);
        if (rc != MR_SUCCESS) return rc;
    }
    MR_CUDA_TRY(cudaEventRecord(e1, s));
    MR_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    MR_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / reps;
    return MR_SUCCESS;
}

int mr_plan_autotune(mr_aha_plan p, const float2 *x, const float2 *S, const mr_kernel_ref &K,
                     const int64_t *mask, float2 *out, int reps, float *best_ms) {
    if (reps < 1) reps = 1;
    const mr_geom &g = p->g;
    const bool has_z = p->cfg.n_spatial == 3;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        if (e0) cudaEventDestroy(e0);
        MR_FAIL(MR_ERR_CUDA, "autotune: cannot create events");
    }
    mr_tune_choice best = tune_get(p);
    float best_t = 0.f;
    int rc = tune_time(p, x, S, K, mask, out, reps, e0, e1, &best_t);
    auto trial = [&](const mr_tune_choice &c) {
        if (rc != MR_SUCCESS) return;
        tune_set(p, c);
        float t = 0.f;
        rc = tune_time(p, x, S, K, mask, out, reps, e0, e1, &t);
        if (rc == MR_SUCCESS && t < best_t) {
            best_t = t;
            best = c;
        }
        tune_set(p, best);
    };
    mr_tune_knob knobs[5];
    tune_knobs(p, knobs);
    const bool fixed_ok = mr_env_int("MR_AHA_B200_NO_FIXED", 0) == 0;
    // pass 3 first (the largest share), then the strided passes
    if (p->fused && rc == MR_SUCCESS) {
        const mr_tune_choice base = best;
        const int nch0 = fixed_ok ? mr_fixed_xbdh_coils(g.m[0], g.n[0], g.L) : 0;
        const int nc2_0 = p->ax[0].small && mr_env_int("MR_AHA_B200_FFT_V1", 0) == 0
                              ? mr_xbd2_coils(g.m[0], g.L, p->cfg.n_coils, (size_t)mr_smem_limit())
                              : 0;
        std::vector<mr_tune_choice> cands;
        if (nch0 > 0) {
            mr_tune_choice c = base;
            c.nch = nch0;
            cands.push_back(c);
        }
        int ncs[8];
        const int nn = fixed_ok ? mr_fixed_xbd_list(g.m[0], g.L, ncs, 8) : 0;
        for (int i = 0; i < nn; ++i) {
            mr_tune_choice c = base;
            c.nch = 0;
            c.nc3 = ncs[i];
            cands.push_back(c);
        }
        if (nc2_0 > 0) {
            mr_tune_choice c = base;
            c.nch = c.nc3 = 0;
            c.nc2 = nc2_0;
            cands.push_back(c);
        }
        if (p->v1_fused) {
            mr_tune_choice c = base;
            c.nch = c.nc3 = c.nc2 = 0;
            cands.push_back(c);
        }
        for (const mr_tune_choice &c : cands)
            if (std::memcmp(&c, &base, sizeof(c)) != 0) trial(c);
    }
    // half-length y passes: off, or each instantiated width for the forward
    // and (separately) the inverse pass
    if (has_z && g.m[1] == 2 * g.n[1] && rc == MR_SUCCESS) {
        const int w0 = mr_half_strided_xt(g.n[1], 0);
        int ws[16];
        const int nw = w0 > 0 ? mr_half_strided_list(g.n[1], ws, 16) : 0;
        for (int pass = 0; pass < 2 && nw > 0; ++pass) {
            const mr_tune_choice base = best;
            std::vector<mr_tune_choice> cands;
            if (pass == 0) {
                mr_tune_choice c = base;
                c.yh_f = c.yh_i = 0;
                cands.push_back(c);
            }
            for (int i = 0; i < nw; ++i) {
                mr_tune_choice c = base;
                if (c.yh_f == 0) c.yh_f = c.yh_i = w0;
                if (pass == 0) c.yh_f = ws[i];
                else c.yh_i = ws[i];
                cands.push_back(c);
            }
            for (const mr_tune_choice &c : cands)
                if (std::memcmp(&c, &base, sizeof(c)) != 0) trial(c);
        }
    }
    for (const mr_tune_knob &k : knobs) {
        if (!k.on || rc != MR_SUCCESS) continue;
        const mr_tune_choice base = best;
        std::vector<mr_tune_choice> cands;
        int xts[16];
        const int nf = fixed_ok ? mr_fixed_strided_list(k.M, k.smode, xts, 16) : 0;
        for (int i = 0; i < nf; ++i) {
            mr_tune_choice c = base;
            c.*k.xt3 = xts[i];
            cands.push_back(c);
        }
        const int e0x = base.*k.xts;
        for (int d = 0; d < 3 && e0x - d >= 0; ++d) {
            mr_tune_choice c = base;
            c.*k.xt3 = 0;
            c.*k.xts = e0x - d;
            cands.push_back(c);
        }
        for (const mr_tune_choice &c : cands)
            if (std::memcmp(&c, &base, sizeof(c)) != 0) trial(c);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != MR_SUCCESS) return rc;
    tune_set(p, best);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_load_locked();
        g_tuned[tune_key(p)] = best;
        tune_save_locked();
    }
    if (best_ms) *best_ms = best_t;
    if (p->cfg.verbose)
        printf("[mr_aha] autotune %s: %.3f ms per apply\n", tune_key(p).c_str(), best_t);
    return MR_SUCCESS;
}
