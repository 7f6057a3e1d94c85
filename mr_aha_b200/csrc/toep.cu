// Toeplitz kernel build: mr_calc_toep and mr_calc_toep_from_psf
// (reference src/cuda/mr_calc_toep.cu:498-856).
//
// The reference evaluates, per packed Gram component t, a type-1 NUFFT with
// sign -1 of the strengths c_{t,m} (the component broadcast along each
// readout) onto the centred grid, then a centred inverse FFT scaled by
// 1/prod(M) (mr_calc_toep.cu:10-23, 171-200). Composing the two in closed
// form, per transformed axis of extent M with s = floor(M/2),
//
//   out[k] = (1/M) sum_m c_m D(theta_m,k),  theta = 2 pi (k - s) / M - x_m,
//   D(theta) = sum_{f=-s}^{M-s-1} exp(i f theta)
//            = exp(i theta ((M-1)/2 - s)) sin(M theta / 2) / sin(theta / 2),
//
// and the 2-D / 3-D kernel is the product of the per-axis factors. This is
// the EXACT value of the reference's pipeline (cufinufft approximates the
// same sum to eps). Because c_{t,m} is constant along a readout s, the sum
// factors through per-readout point-spread functions:
//
//   K_s[k] = sum_{r in readout s} Dx(theta_x) Dy(theta_y) [Dz(theta_z)]
//   out_t[k] = scale * sum_s T[t, s] K_s[k]
//
// Both steps are complex GEMMs evaluated here in double precision (FP64
// accumulation throughout; the Dirichlet factors are computed in double), and
// the result is rounded once to complex64. Cost: Ntrajs*Nkx*prod(M) for the
// per-readout PSFs plus ntri*Nkz*Ntrajs*prod(M) for the contraction.
#include "engine.h"
#include "nufft.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

// D(theta) for an axis of extent M, theta already in double.
__device__ __forceinline__ double2 dirichlet(double theta, int M, int s) {
    // reduce to (-pi, pi]; D is 2 pi periodic
    theta -= kTwoPi * rint(theta / kTwoPi);
    const double ph = theta * (0.5 * (double)(M - 1) - (double)s);
    double sp, cp;
    sincos(ph, &sp, &cp);
    double ratio;
    if (fabs(theta) < 1e-9) {
        ratio = (double)M;
    } else {
        ratio = sin(0.5 * (double)M * theta) / sin(0.5 * theta);
    }
    return make_double2(ratio * cp, ratio * sp);
}

// Dirichlet tables D[s][r][k] (k fastest) for spokes [s0, s0 + ns) of one
// axis: coordinate of sample (s, r) is traj[s + Ntrajs * r + Msmp * axis].
__global__ void k_dirichlet(double2 *D, const float *__restrict__ traj, int64_t Ntrajs,
                            int64_t Nkx, int axis, int64_t s0, int64_t ns, int M) {
    const int64_t total = ns * Nkx * M;
    const int s = M / 2;
    const int64_t msmp = Ntrajs * Nkx;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(w % M);
        const int64_t rest = w / M;
        const int64_t r = rest % Nkx;
        const int64_t sp = s0 + rest / Nkx;
        const double xm = (double)traj[sp + Ntrajs * r + msmp * axis];
        const double theta = kTwoPi * (double)(k - s) / (double)M - xm;
        D[w] = dirichlet(theta, M, s);
    }
}

// Packed Gram components as double: T[(t * nkz + kz) * Ntrajs + s] from the
// column-major [Ntrajs, Nkz, L, L] blocks (element (i, j) of block b at
// b + nbatch * (i + L * j)); component t is stored element (i, j) of the
// requested triangle (reference mr_kernels.cu:307-333).
__global__ void k_pack_gram(double2 *T, const float2 *__restrict__ phi2, int64_t nbatch,
                            int L, int upper) {
    const int64_t total = nbatch * L * L;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = w % nbatch;
        const int64_t ij = w / nbatch;
        const int i = (int)(ij % L);
        const int j = (int)(ij / L);
        const bool keep = upper ? (i <= j) : (i >= j);
        if (!keep) continue;
        bool cj;
        const int t = bd_tri_offset(i, j, L, upper, &cj);
        const float2 v = phi2[w];
        T[b + nbatch * t] = make_double2(v.x, v.y);
    }
}

// Complex double GEMM, C(i, j) = scale * sum_k A(i, k) B(k, j), batched.
//   A(i, k) = A1[i1 * a1_i + k * a1_k] (* A2[i2 * a2_i + k * a2_k] when A2 is
//   given), with ii = i + i_off, i1 = ii % n1, i2 = ii / n1;
//   B(k, j) = B[k * b_k + j * b_j];  C row-major with row stride c_i.
// 64 x 64 tile per CTA, k-steps of 16, 4 x 4 outputs per thread.
struct gemm_args {
    const double2 *A1, *A2;
    int64_t a1_i, a1_k, a1_b, a2_i, a2_k, a2_b;
    int64_t n1, i_off;
    const double2 *B;
    int64_t b_k, b_j, b_batch;
    void *C;
    int64_t c_i, c_batch;
    int64_t m, n, k;
    double scale;
};

template <bool OUT_F32>
__global__ void __launch_bounds__(256, 2) k_zgemm(const gemm_args g) {
    __shared__ double2 As[16][64 + 1];
    __shared__ double2 Bs[16][64 + 1];
    const int64_t batch = blockIdx.z;
    const int64_t i0 = (int64_t)blockIdx.y * 64;
    const int64_t j0 = (int64_t)blockIdx.x * 64;
    const int tx = threadIdx.x % 16;  // column group
    const int ty = threadIdx.x / 16;  // row group
    double2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0.0, 0.0);
    const double2 *A1 = g.A1 + batch * g.a1_b;
    const double2 *A2 = g.A2 ? g.A2 + batch * g.a2_b : nullptr;
    const double2 *B = g.B + batch * g.b_batch;
    for (int64_t k0 = 0; k0 < g.k; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int kk = e / 64, ii = e % 64;
            const int64_t gi = i0 + ii, gk = k0 + kk;
            double2 v = make_double2(0.0, 0.0);
            if (gi < g.m && gk < g.k) {
                const int64_t ia = gi + g.i_off;
                if (A2) {
                    const int64_t i1 = ia % g.n1, i2 = ia / g.n1;
                    const double2 p = A1[i1 * g.a1_i + gk * g.a1_k];
                    const double2 q = A2[i2 * g.a2_i + gk * g.a2_k];
                    v = make_double2(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x);
                } else {
                    v = A1[ia * g.a1_i + gk * g.a1_k];
                }
            }
            As[kk][ii] = v;
        }
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int kk = e / 64, jj = e % 64;
            const int64_t gj = j0 + jj, gk = k0 + kk;
            Bs[kk][jj] = (gj < g.n && gk < g.k) ? B[gk * g.b_k + gj * g.b_j]
                                                 : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
            double2 a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = As[kk][ty + 16 * q];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = Bs[kk][tx + 16 * q];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    acc[p][q].x = fma(a[p].x, b[q].x, fma(-a[p].y, b[q].y, acc[p][q].x));
                    acc[p][q].y = fma(a[p].x, b[q].y, fma(a[p].y, b[q].x, acc[p][q].y));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int64_t gi = i0 + ty + 16 * p;
        if (gi >= g.m) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t gj = j0 + tx + 16 * q;
            if (gj >= g.n) continue;
            const double2 v = acc[p][q];
            const int64_t o = batch * g.c_batch + gi * g.c_i + gj;
            if (OUT_F32)
                reinterpret_cast<float2 *>(g.C)[o] =
                    make_float2((float)(v.x * g.scale), (float)(v.y * g.scale));
            else
                reinterpret_cast<double2 *>(g.C)[o] =
                    make_double2(v.x * g.scale, v.y * g.scale);
        }
    }
}

int launch_zgemm(const gemm_args &g, int64_t nbatch, bool out_f32, cudaStream_t s) {
    if (g.m <= 0 || g.n <= 0 || nbatch <= 0) return MR_SUCCESS;
    const int64_t gx = mr_cdiv(g.n, 64), gy = mr_cdiv(g.m, 64);
    if (gx > 0x7fffffff || gy > 65535 || nbatch > 65535)
        MR_FAIL(MR_ERR_UNSUPPORTED, "kernel build GEMM grid too large");
    dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)nbatch);
    if (out_f32) k_zgemm<true><<<grid, 256, 0, s>>>(g);
    else k_zgemm<false><<<grid, 256, 0, s>>>(g);
    MR_LAUNCH_CHECK("k_zgemm");
    return MR_SUCCESS;
}

// out[i + nm * (t0 + t)] = full[t * vpad + mask[i]] for t < nt
__global__ void k_gather_mask(float2 *out, const float2 *__restrict__ full,
                              const int64_t *__restrict__ mask, int64_t nm, int64_t vpad,
                              int64_t t0, int64_t nt) {
    const int64_t total = nm * nt;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = w % nm, t = w / nm;
        out[i + nm * (t0 + t)] = full[t * vpad + mask[i]];
    }
}

unsigned grid_for(int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(mr_cdiv(n, 256), 148 * 32));
}

struct dev_buf {
    void *p = nullptr;
    ~dev_buf() {
        if (p) cudaFree(p);
    }
    int alloc(size_t bytes, const char *what) {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            MR_FAIL(MR_ERR_ALLOC, "failed to allocate %zu bytes for %s", bytes, what);
        }
        return MR_SUCCESS;
    }
};

}  // namespace

static int from_psf_impl(const mr_config *cfg, const float2 *psf, int64_t t0, int64_t n,
                         const int64_t *mask, float2 *out_all);

// Kernel build by spreading, for geometries where the closed form's
// Ntrajs * Nkx * prod(M) cost is prohibitive (3-D kooshball grids): per
// packed component t (and kz plane of a stack), the type-1 non-uniform FFT
// (sign -1, centred modes phi2_dim) of the strengths c_{t,m} (component t of
// sample m's readout Gram block, broadcast along the readout) with FP64
// accumulation in the spreading step (nufft.cu), then the centred inverse
// FFT / prod(M) (from_psf_impl) -- the reference's pipeline
// (src/cuda/mr_calc_toep.cu:537-633) with this library's own NUFFT. Writes
// components [t0, t0 + nt) to out (component t0 first).
static int toep_spread_build(const mr_config *cfg, const double2 *T, const float *traj,
                             int64_t Ntrajs, int64_t Nkx, float2 *out, int64_t t0, int64_t nt,
                             cudaStream_t s) {
    const bool three = cfg->traj_type == MR_TRAJ_3D;
    const int Mx = cfg->phi2_dim[0], My = cfg->phi2_dim[1], Mz = cfg->phi2_dim[2];
    const int nkz = cfg->traj_type == MR_TRAJ_STACK ? Mz : 1;
    const int modes[3] = {Mx, My, Mz};
    const int dims = three ? 3 : 2;
    const double eps = std::min(cfg->eps > 0 ? cfg->eps : 1e-6, 1e-7);
    const int64_t vpad = mr_pad_size(cfg);
    size_t budget = 0;
    int rc = mr_memory_budget(cfg, &budget);
    if (rc != MR_SUCCESS) return rc;
    // planes per call: whole components (nkz planes each) within the budget
    const size_t per_comp = mr_nufft_plan_bytes(dims, modes, eps, 2.0, nkz, 1);
    int64_t tc = (int64_t)std::max<size_t>(1, (budget / 2) / std::max<size_t>(per_comp, 1));
    tc = std::min<int64_t>(std::min<int64_t>(tc, nt), 64);
    const int env_c = mr_env_int("MR_AHA_TOEP_MAX_CHUNK", 0);
    if (env_c > 0) tc = std::min<int64_t>(tc, env_c);
    mr_nufft *plan = nullptr;
    rc = mr_nufft_create(dims, modes, traj, Ntrajs * Nkx, eps, 2.0, (int)(tc * nkz), 1, &plan);
    if (rc != MR_SUCCESS) return rc;
    dev_buf psf;
    rc = psf.alloc((size_t)tc * vpad * sizeof(float2), "the spread PSFs");
    mr_config c = *cfg;
    c.is_masked = 0;
    c.num_masked = 0;
    for (int64_t a = 0; a < nt && rc == MR_SUCCESS; a += tc) {
        const int64_t n = std::min(tc, nt - a);
        // planes (t, kz) of components [t0 + a, t0 + a + n): strengths
        // T[(t nkz + kz) Ntrajs + s], sample m of readout s = m % Ntrajs
        rc = mr_nufft_type1(plan, -1, T + (t0 + a) * nkz * Ntrajs, Ntrajs, Ntrajs,
                            (int)(n * nkz), (float2 *)psf.p, s);
        if (rc == MR_SUCCESS) rc = from_psf_impl(&c, (const float2 *)psf.p, a, n, nullptr, out);
    }
    cudaStreamSynchronize(s);
    mr_nufft_destroy(plan);
    return rc;
}

// Which build a configuration takes: MR_AHA_B200_TOEP_METHOD = 1 forces the
// spreading build, 2 the closed form; otherwise the cheaper by a cost model
// calibrated on B200 (3-D 64^3 image, 128^3 grid, L = 4, 2000 x 128
// samples: closed form 0.59 s, about 8 TFLOP/s of FP64 GEMM; spreading in
// trajectory order 0.04 s, about 9e10 double atomic adds per second; with
// the samples in grid-bin order the 3-D kooshball build (256^3 grid, 10000 x
// 256 samples) runs 1.9x and the stack320 one 1.5x faster: 1e11 here, still
// pessimistic like the GEMM rate, so the ratio of the two decides).
static bool use_spread_build(const mr_config *cfg, int64_t Ntrajs, int64_t Nkx) {
    const int m = mr_env_int("MR_AHA_B200_TOEP_METHOD", 0);
    if (m == 1) return true;
    if (m == 2) return false;
    const bool three = cfg->traj_type == MR_TRAJ_3D;
    const double Mx = cfg->phi2_dim[0], My = cfg->phi2_dim[1], Mz = cfg->phi2_dim[2];
    const double nkz = cfg->traj_type == MR_TRAJ_STACK ? Mz : 1;
    const double ntri = (double)mr_num_tri(cfg->L);
    const double grid = Mx * My * (three ? Mz : 1);
    const double smp = (double)Ntrajs * Nkx;
    const double t_exact = 8.0 * (smp * grid + ntri * nkz * Ntrajs * grid) / 8e12;
    const double w = 9, wd = three ? w * w * w : w * w;
    const double fine = grid * (three ? 8.0 : 4.0);
    const double t_spread =
        ntri * nkz * (2.0 * smp * wd / 1e11 + 10.0 * fine * std::log2(fine) / 5e12);
    return t_spread < t_exact;
}

// Build the unmasked kernel rows [row0, row0 + nrows) of the output matrix
// (rows = components for 2D / 3D, (component, kz) for a stack) into
// `out` (row stride = columns), or all rows when nrows < 0.
static int toep_build(const mr_config *cfg, const float2 *phi2, const float *traj,
                      int64_t Ntrajs, int64_t Nkx, float2 *out, int64_t t0, int64_t nt,
                      cudaStream_t s) {
    const int tt = cfg->traj_type;
    const int L = cfg->L;
    const int64_t ntri = mr_num_tri(L);
    const int Mx = cfg->phi2_dim[0], My = cfg->phi2_dim[1], Mz = cfg->phi2_dim[2];
    const bool three = tt == MR_TRAJ_3D;
    const int nkz = tt == MR_TRAJ_STACK ? Mz : 1;
    const int64_t nbatch = Ntrajs * nkz;
    // rows of the "A" side of the per-readout PSF: ky (2D/stack) or (kz, ky) (3D)
    const int64_t prow = three ? (int64_t)My * Mz : My;
    const int64_t ncols = prow * Mx;  // positions per output row
    const double scale = 1.0 / ((double)Mx * My * (three ? Mz : 1));

    int rc;
    dev_buf Tb;
    rc = Tb.alloc((size_t)nbatch * ntri * sizeof(double2), "the packed Gram blocks");
    if (rc != MR_SUCCESS) return rc;
    double2 *T = (double2 *)Tb.p;
    k_pack_gram<<<grid_for(nbatch * L * L), 256, 0, s>>>(T, phi2, nbatch, L,
                                                        cfg->triangulation == MR_TRI_UPPER);
    MR_LAUNCH_CHECK("k_pack_gram");
    if (use_spread_build(cfg, Ntrajs, Nkx))
        return toep_spread_build(cfg, T, traj, Ntrajs, Nkx, out, t0, nt, s);

    // Memory plan: Ks for all readouts over a chunk of PSF rows, plus the
    // Dirichlet tables of a chunk of readouts.
    size_t budget = 0;
    rc = mr_memory_budget(cfg, &budget);
    if (rc != MR_SUCCESS) return rc;
    const size_t per_prow = (size_t)Ntrajs * Mx * sizeof(double2);
    int64_t rchunk = (int64_t)std::max<size_t>(1, (budget / 2) / std::max<size_t>(per_prow, 1));
    rchunk = std::min<int64_t>(rchunk, prow);
    const int env_chunk = mr_env_int("MR_AHA_TOEP_MAX_CHUNK", 0);
    if (env_chunk > 0) rchunk = std::min<int64_t>(rchunk, env_chunk);
    const size_t per_spoke_tab = (size_t)Nkx * (Mx + My + (three ? Mz : 0)) * sizeof(double2);
    int64_t schunk = (int64_t)std::max<size_t>(1, (budget / 4) / std::max<size_t>(per_spoke_tab, 1));
    schunk = std::min<int64_t>(std::min<int64_t>(schunk, Ntrajs), 65535);

    dev_buf Kb, Dxb, Dyb, Dzb;
    rc = Kb.alloc((size_t)Ntrajs * rchunk * Mx * sizeof(double2), "the per-readout PSFs");
    if (rc != MR_SUCCESS) return rc;
    rc = Dxb.alloc((size_t)schunk * Nkx * Mx * sizeof(double2), "the x Dirichlet table");
    if (rc != MR_SUCCESS) return rc;
    rc = Dyb.alloc((size_t)schunk * Nkx * My * sizeof(double2), "the y Dirichlet table");
    if (rc != MR_SUCCESS) return rc;
    if (three) {
        rc = Dzb.alloc((size_t)schunk * Nkx * Mz * sizeof(double2), "the z Dirichlet table");
        if (rc != MR_SUCCESS) return rc;
    }
    double2 *Ks = (double2 *)Kb.p;
    double2 *Dx = (double2 *)Dxb.p, *Dy = (double2 *)Dyb.p, *Dz = (double2 *)Dzb.p;

    // output rows: (t, kz) for t in [t0, t0 + nt)
    const int64_t orow0 = t0 * nkz;
    const int64_t norows = nt * nkz;

    for (int64_t pr0 = 0; pr0 < prow; pr0 += rchunk) {
        const int64_t npr = std::min<int64_t>(rchunk, prow - pr0);
        // ---- per-readout PSFs for PSF rows [pr0, pr0 + npr) ----
        for (int64_t s0 = 0; s0 < Ntrajs; s0 += schunk) {
            const int64_t ns = std::min<int64_t>(schunk, Ntrajs - s0);
            k_dirichlet<<<grid_for(ns * Nkx * Mx), 256, 0, s>>>(Dx, traj, Ntrajs, Nkx, 0, s0, ns, Mx);
            k_dirichlet<<<grid_for(ns * Nkx * My), 256, 0, s>>>(Dy, traj, Ntrajs, Nkx, 1, s0, ns, My);
            if (three)
                k_dirichlet<<<grid_for(ns * Nkx * Mz), 256, 0, s>>>(Dz, traj, Ntrajs, Nkx, 2, s0, ns, Mz);
            MR_LAUNCH_CHECK("k_dirichlet");
            // Ks[s][pr][kx] = sum_r A(pr, r) Dx[s][r][kx], batched over s;
            // A(pr, r) = Dy[s][r][ky] (2D / stack) or Dy[s][r][ky] Dz[s][r][kz]
            // (3D, pr = kz * My + ky).
            gemm_args g;
            std::memset(&g, 0, sizeof(g));
            g.A1 = Dy;
            g.a1_i = 1;
            g.a1_k = My;
            g.a1_b = (int64_t)Nkx * My;
            g.n1 = three ? My : ((int64_t)1 << 62);
            g.i_off = pr0;
            if (three) {
                g.A2 = Dz;
                g.a2_i = 1;
                g.a2_k = Mz;
                g.a2_b = (int64_t)Nkx * Mz;
            }
            g.B = Dx;
            g.b_k = Mx;
            g.b_j = 1;
            g.b_batch = (int64_t)Nkx * Mx;
            g.C = Ks + s0 * npr * Mx;
            g.c_i = Mx;
            g.c_batch = npr * Mx;
            g.m = npr;
            g.n = Mx;
            g.k = Nkx;
            g.scale = 1.0;
            rc = launch_zgemm(g, ns, false, s);
            if (rc != MR_SUCCESS) return rc;
        }
        // ---- contraction: out[row][pr0.., kx] = scale * sum_s T[row][s] Ks[s][pr][kx] ----
        gemm_args g;
        std::memset(&g, 0, sizeof(g));
        g.A1 = T + orow0 * Ntrajs;
        g.a1_i = Ntrajs;
        g.a1_k = 1;
        g.n1 = (int64_t)1 << 62;
        g.B = Ks;
        g.b_k = npr * Mx;
        g.b_j = 1;
        g.C = out + pr0 * Mx;
        g.c_i = ncols;
        g.m = norows;
        g.n = npr * Mx;
        g.k = Ntrajs;
        g.scale = scale;
        rc = launch_zgemm(g, 1, true, s);
        if (rc != MR_SUCCESS) return rc;
    }
    MR_CUDA_TRY(cudaStreamSynchronize(s));
    return MR_SUCCESS;
}

static int calc_toep_impl(const mr_config *cfg, const float2 *phi2, const float *traj,
                          int64_t Ntrajs, int64_t Nkx, const int64_t *mask, float2 *out) {
    cudaStream_t s = (cudaStream_t)cfg->stream;
    const int64_t ntri = mr_num_tri(cfg->L);
    const int64_t vpad = mr_pad_size(cfg);
    if (!cfg->is_masked) return toep_build(cfg, phi2, traj, Ntrajs, Nkx, out, 0, ntri, s);
    // masked: build component chunks into a full-grid scratch and gather
    size_t budget = 0;
    int rc = mr_memory_budget(cfg, &budget);
    if (rc != MR_SUCCESS) return rc;
    int64_t tc = (int64_t)std::max<size_t>(1, (budget / 4) / ((size_t)vpad * sizeof(float2)));
    tc = std::min(tc, ntri);
    float2 *full = nullptr;
    if (cudaMalloc(&full, (size_t)tc * vpad * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        MR_FAIL(MR_ERR_ALLOC, "failed to allocate the masked kernel scratch");
    }
    for (int64_t t0 = 0; t0 < ntri && rc == MR_SUCCESS; t0 += tc) {
        const int64_t nt = std::min(tc, ntri - t0);
        rc = toep_build(cfg, phi2, traj, Ntrajs, Nkx, full, t0, nt, s);
        if (rc != MR_SUCCESS) break;
        const int64_t nm = cfg->num_masked;
        k_gather_mask<<<grid_for(nm * nt), 256, 0, s>>>(out, full, mask, nm, vpad, t0, nt);
        if (cudaGetLastError() != cudaSuccess) {
            rc = MR_ERR_CUDA;
            mr_set_error("k_gather_mask failed to launch");
        }
        if (cudaStreamSynchronize(s) != cudaSuccess && rc == MR_SUCCESS) {
            rc = MR_ERR_CUDA;
            mr_set_error("masked kernel gather failed");
        }
    }
    cudaFree(full);
    return rc;
}

extern "C" int mr_calc_toep(const mr_config *cfg, const mr_complex *d_phi2,
                            const float *d_traj, int64_t Ntrajs, int64_t Nkx,
                            const int64_t *d_mask, mr_complex *d_phi2_toep) {
    mr_clear_error();
    MR_REQUIRE(cfg != nullptr, "mr_calc_toep: cfg is NULL");
    MR_REQUIRE(d_phi2 != nullptr, "mr_calc_toep: d_phi2 is NULL");
    MR_REQUIRE(d_traj != nullptr, "mr_calc_toep: d_traj is NULL");
    MR_REQUIRE(d_phi2_toep != nullptr, "mr_calc_toep: d_phi2_toep is NULL");
    MR_REQUIRE(Ntrajs > 0, "mr_calc_toep: Ntrajs = %lld must be > 0", (long long)Ntrajs);
    MR_REQUIRE(Nkx > 0, "mr_calc_toep: Nkx = %lld must be > 0", (long long)Nkx);
    if (cfg->is_masked)
        MR_REQUIRE(d_mask != nullptr, "mr_calc_toep: d_mask is required when is_masked is set");
    int rc = mr_config_validate(cfg);
    if (rc != MR_SUCCESS) return rc;
    int prev = -1;
    rc = mr_push_device(cfg, &prev);
    if (rc == MR_SUCCESS)
        rc = calc_toep_impl(cfg, reinterpret_cast<const float2 *>(d_phi2), d_traj, Ntrajs, Nkx,
                            d_mask, reinterpret_cast<float2 *>(d_phi2_toep));
    mr_pop_device(prev);
    return rc;
}

// ---------------------------------------------------------------------------
// mr_calc_toep_from_psf: centred inverse FFT / prod(M) of given PSFs
// ---------------------------------------------------------------------------

static int from_psf_impl(const mr_config *cfg, const float2 *psf, int64_t t0, int64_t n,
                         const int64_t *mask, float2 *out_all) {
    cudaStream_t s = (cudaStream_t)cfg->stream;
    const int Mx = cfg->phi2_dim[0], My = cfg->phi2_dim[1], Mz = cfg->phi2_dim[2];
    const bool three = cfg->traj_type == MR_TRAJ_3D;
    const int64_t vpad = mr_pad_size(cfg);
    const float scale = (float)(1.0 / ((double)Mx * My * (three ? Mz : 1)));
    mr_fft_axis ax[3];
    int rc;
    int off[3], tot = 0;
    for (int d = 0; d < 3; ++d) {
        rc = mr_fft_factor(cfg->phi2_dim[d], &ax[d]);
        if (rc != MR_SUCCESS) return rc;
        off[d] = tot;
        tot += cfg->phi2_dim[d];
    }
    std::vector<float2> h(tot);
    for (int d = 0; d < 3; ++d) mr_fft_twiddles(cfg->phi2_dim[d], h.data() + off[d]);
    dev_buf twb, work;
    rc = twb.alloc(tot * sizeof(float2), "the FFT tables");
    if (rc != MR_SUCCESS) return rc;
    MR_CUDA_TRY(cudaMemcpy(twb.p, h.data(), tot * sizeof(float2), cudaMemcpyHostToDevice));
    for (int d = 0; d < 3; ++d) ax[d].tw = (const float2 *)twb.p + off[d];
    float2 *dst;
    if (cfg->is_masked) {
        rc = work.alloc((size_t)n * vpad * sizeof(float2), "the PSF scratch");
        if (rc != MR_SUCCESS) return rc;
        dst = (float2 *)work.p;
    } else {
        dst = out_all + t0 * vpad;
    }
    const size_t lim = (size_t)mr_smem_limit();
    // x: rows of Mx, centred -> natural, inverse, natural -> centred
    {
        mr_x_args a;
        std::memset(&a, 0, sizeof(a));
        a.ax = ax[0];
        a.rows_cta = 4;
        while (a.rows_cta > 1 && mr_xplain_smem(Mx, a.rows_cta) > lim) a.rows_cta >>= 1;
        a.src = psf;
        a.dst = dst;
        a.s_row = Mx;
        a.d_row = Mx;
        a.nrows = n * Mz * My;
        a.n_in = Mx;
        a.shift_in = Mx / 2;
        a.n_out = Mx;
        a.shift_out = Mx / 2;
        a.scale = three || My > 1 ? 1.f : scale;
        rc = mr_launch_xplain(1, a, s);
        if (rc != MR_SUCCESS) return rc;
    }
    // y lines (in place)
    {
        mr_strided_args a;
        std::memset(&a, 0, sizeof(a));
        a.ax = ax[1];
        a.nfast = Mx;
        a.xt = mr_pick_xt(My, My, MR_SM_BUF, Mx, lim / 2);
        a.nxt = (int)mr_cdiv(Mx, a.xt);
        a.nouter = Mz;
        a.nplane = (int)n;
        a.src = dst;
        a.s_plane = vpad;
        a.s_outer = (int64_t)My * Mx;
        a.s_axis = Mx;
        a.n_in = My;
        a.shift_in = My / 2;
        a.dst = dst;
        a.d_plane = vpad;
        a.d_outer = (int64_t)My * Mx;
        a.d_axis = Mx;
        a.n_out = My;
        a.shift_out = My / 2;
        a.scale = three ? 1.f : scale;
        rc = mr_launch_strided(1, MR_LM_BUF, MR_SM_BUF, a, s);
        if (rc != MR_SUCCESS) return rc;
    }
    if (three) {
        mr_strided_args a;
        std::memset(&a, 0, sizeof(a));
        a.ax = ax[2];
        a.nfast = Mx;
        a.xt = mr_pick_xt(Mz, Mz, MR_SM_BUF, Mx, lim / 2);
        a.nxt = (int)mr_cdiv(Mx, a.xt);
        a.nouter = My;
        a.nplane = (int)n;
        a.src = dst;
        a.s_plane = vpad;
        a.s_outer = Mx;
        a.s_axis = (int64_t)My * Mx;
        a.n_in = Mz;
        a.shift_in = Mz / 2;
        a.dst = dst;
        a.d_plane = vpad;
        a.d_outer = Mx;
        a.d_axis = (int64_t)My * Mx;
        a.n_out = Mz;
        a.shift_out = Mz / 2;
        a.scale = scale;
        rc = mr_launch_strided(1, MR_LM_BUF, MR_SM_BUF, a, s);
        if (rc != MR_SUCCESS) return rc;
    }
    if (cfg->is_masked) {
        const int64_t nm = cfg->num_masked;
        k_gather_mask<<<grid_for(nm * n), 256, 0, s>>>(out_all, dst, mask, nm, vpad, t0, n);
        MR_LAUNCH_CHECK("k_gather_mask");
    }
    MR_CUDA_TRY(cudaStreamSynchronize(s));
    return MR_SUCCESS;
}

extern "C" int mr_calc_toep_from_psf(const mr_config *cfg, const mr_complex *d_psf, int64_t t0,
                                     int64_t n_comp, const int64_t *d_mask,
                                     mr_complex *d_phi2_toep) {
    mr_clear_error();
    MR_REQUIRE(cfg != nullptr, "mr_calc_toep_from_psf: cfg is NULL");
    MR_REQUIRE(d_psf != nullptr, "mr_calc_toep_from_psf: d_psf is NULL");
    MR_REQUIRE(d_phi2_toep != nullptr, "mr_calc_toep_from_psf: d_phi2_toep is NULL");
    int rc = mr_config_validate(cfg);
    if (rc != MR_SUCCESS) return rc;
    const int64_t ntri = mr_num_tri(cfg->L);
    MR_REQUIRE(t0 >= 0 && n_comp >= 1 && t0 + n_comp <= ntri,
               "mr_calc_toep_from_psf: components [%lld, %lld) outside [0, %lld)",
               (long long)t0, (long long)(t0 + n_comp), (long long)ntri);
    if (cfg->is_masked)
        MR_REQUIRE(d_mask != nullptr,
                   "mr_calc_toep_from_psf: d_mask is required when is_masked is set");
    int prev = -1;
    rc = mr_push_device(cfg, &prev);
    if (rc == MR_SUCCESS)
        rc = from_psf_impl(cfg, reinterpret_cast<const float2 *>(d_psf), t0, n_comp, d_mask,
                           reinterpret_cast<float2 *>(d_phi2_toep));
    mr_pop_device(prev);
    return rc;
}
