// Non-uniform FFTs with the "exponential of semicircle" (ES) spreading kernel
// of Barnett, Magland and af Klinteberg, "A parallel nonuniform fast Fourier
// transform library based on an exponential of semicircle kernel", SIAM J.
// Sci. Comput. 41(5), C479-C504 (2019):
//
//   psi(z) = exp(beta (sqrt(1 - z^2) - 1)),  |z| <= 1,
//
// spread over w points of an oversampled periodic grid of nf >= sigma M
// points per axis (spacing h = 2 pi / nf, z = (l h - x) / (w h / 2)).
// Type 1: b[l] = sum_m c_m psi(l h - x_m) (spreading), B = FFT_{iflag}(b),
// f_k = B[k] / psihat(k). Type 2 is its adjoint: b = FFT_{iflag}(f / psihat
// zero-padded to the grid), c_m = sum_l b[l] psi(l h - x_m) (interpolation).
// psihat(k) = (w / 2) int_{-1}^{1} psi(z) cos(k w h z / 2) dz, evaluated on
// the host by Gauss-Legendre quadrature in double precision.
//
// Parameters (section 3 of the paper): w = ceil(log10(1 / eps)) + 1 for
// sigma = 2 (plus one point of margin here), beta = 2.30 w; other sigma:
// w = ceil(-ln(eps) / (pi sqrt(1 - 1 / sigma))) + 1,
// beta = 0.97 pi (1 - 1 / (2 sigma)) w.
//
// Spreading runs one thread per (plane, sample) pair with atomic adds into
// global memory, in FP32 or (for the Toeplitz kernel build) FP64, visiting
// the samples of a plane in grid-bin order (a permutation sorted once per
// plan) so that neighbouring threads update neighbouring grid points and the
// atomics find their lines in L2; the FFTs
// along each axis are the library's strided / row passes, whose load and
// store windows also do the zero padding (type 2) and the cropping to the
// centred modes (type 1).
#include "nufft.h"

#include <thrust/execution_policy.h>
#include <thrust/sort.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

struct mr_nufft {
    int dims;
    int M[3], nf[3];
    int w;
    double beta;
    int64_t npts;
    const float *traj;
    int maxp;
    int fp64;
    mr_fft_axis ax[3];
    float2 *tw;          // twiddles of the grid axes
    float *ideconv;      // 1 / psihat per centred mode index: x | y | z
    float2 *fine;        // maxp grids
    double2 *fine64;     // maxp grids (fp64 spreading)
    float2 *A, *B, *D;   // FFT stage buffers
    int *perm;           // samples in grid-bin order, NULL for trajectory order
};

namespace {

constexpr double kPi = 3.14159265358979323846;

int es_width(double eps, double sigma) {
    eps = std::min(std::max(eps, 1e-14), 1e-1);
    int w;
    if (std::fabs(sigma - 2.0) < 1e-12) w = (int)std::ceil(std::log10(1.0 / eps)) + 2;
    else w = (int)std::ceil(-std::log(eps) / (kPi * std::sqrt(1.0 - 1.0 / sigma))) + 2;
    return std::min(16, std::max(3, w));
}

double es_beta(int w, double sigma) {
    if (std::fabs(sigma - 2.0) < 1e-12) return 2.30 * w;
    return 0.97 * kPi * (1.0 - 1.0 / (2.0 * sigma)) * w;
}

// Smallest even integer >= n with no prime factor above 7 (lengths the FFT
// passes run with radix butterflies only).
int smooth_even(int n) {
    for (int m = std::max(2, n + (n & 1));; m += 2) {
        int r = m;
        for (int p : {2, 3, 5, 7})
            while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on the
// three-term recurrence of the Legendre polynomials).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &wq) {
    x.resize(n);
    wq.resize(n);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-15) break;
        }
        x[i] = z;
        wq[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

void plan_dims(int dims, const int *modes, double eps, double sigma, int *M, int *nf, int *w,
               double *beta) {
    if (sigma <= 1.0) sigma = 2.0;
    *w = es_width(eps, sigma);
    *beta = es_beta(*w, sigma);
    for (int d = 0; d < 3; ++d) {
        M[d] = d < dims ? modes[d] : 1;
        nf[d] = d < dims ? smooth_even(std::max((int)std::ceil(sigma * M[d]), 2 * *w)) : 1;
    }
}

struct bytes_of {
    size_t fine, fine64, A, B, D, tw, dec;
};

bytes_of plan_sizes(int dims, const int *M, const int *nf, int maxp, int fp64) {
    const size_t nfvol = (size_t)nf[0] * nf[1] * nf[2];
    const size_t mvol = (size_t)M[0] * M[1] * M[2];
    bytes_of b;
    b.fine = (size_t)maxp * nfvol * sizeof(float2);
    b.fine64 = fp64 ? (size_t)maxp * nfvol * sizeof(double2) : 0;
    b.A = (size_t)maxp * nf[2] * nf[1] * M[0] * sizeof(float2);
    b.B = dims == 3 ? (size_t)maxp * nf[2] * M[1] * M[0] * sizeof(float2) : 0;
    b.D = (size_t)maxp * mvol * sizeof(float2);
    b.tw = (size_t)(nf[0] + nf[1] + nf[2]) * sizeof(float2);
    b.dec = (size_t)(M[0] + M[1] + M[2]) * sizeof(float);
    return b;
}

unsigned grid_of(int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
}

// ES weights of the w grid points of one axis near position x (radians):
// first point l0 (wrapped into [0, nf)) and psi at each.
template <typename R>
__device__ __forceinline__ int es_axis(float x, int nf, int w, double beta, R *wt) {
    const double u = (double)x * (double)nf * (1.0 / (2.0 * kPi));
    const double half = 0.5 * (double)w;
    const double i0 = ceil(u - half);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        if (i < w) {
            const double z = (i0 + i - u) / half;
            if constexpr (sizeof(R) == 8) {
                const double q = 1.0 - z * z;
                wt[i] = q > 0.0 ? exp(beta * (sqrt(q) - 1.0)) : 0.0;
            } else {
                const float zf = (float)z;
                const float q = 1.f - zf * zf;
                wt[i] = q > 0.f ? expf((float)beta * (sqrtf(q) - 1.f)) : 0.f;
            }
        }
    }
    int64_t l = (int64_t)i0 % nf;
    if (l < 0) l += nf;
    return (int)l;
}

template <typename R>
struct cplx;
template <>
struct cplx<float> {
    using T = float2;
};
template <>
struct cplx<double> {
    using T = double2;
};

// fine[p][(lz,) ly, lx] += c(p, m) psi_z psi_y psi_x over the w^dims points
// near sample m, for every (p, m) with p < n.
template <int DIMS, typename R>
__global__ void __launch_bounds__(256) k_spread(typename cplx<R>::T *fine, const void *cv,
                                                int64_t cstride, int64_t bcast, int n,
                                                const float *__restrict__ traj, int64_t npts,
                                                const int *__restrict__ perm, int nfx, int nfy,
                                                int nfz, int w, double beta) {
    using C = typename cplx<R>::T;
    const C *c = reinterpret_cast<const C *>(cv);
    const int64_t nfvol = (int64_t)nfx * nfy * nfz;
    const int64_t total = (int64_t)n * npts;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = perm ? (int64_t)__ldg(perm + q % npts) : q % npts;
        const int p = (int)(q / npts);
        const C v = c[p * cstride + (bcast > 0 ? m % bcast : m)];
        if (v.x == 0 && v.y == 0) continue;
        R wx[16], wy[16], wz[16];
        const int lx0 = es_axis<R>(__ldg(traj + m), nfx, w, beta, wx);
        const int ly0 = es_axis<R>(__ldg(traj + npts + m), nfy, w, beta, wy);
        int lz0 = 0;
        if constexpr (DIMS == 3) lz0 = es_axis<R>(__ldg(traj + 2 * npts + m), nfz, w, beta, wz);
        C *g = fine + p * nfvol;
        for (int iz = 0; iz < (DIMS == 3 ? w : 1); ++iz) {
            int lz = lz0 + iz;
            if (lz >= nfz) lz -= nfz;
            const R fz = DIMS == 3 ? wz[iz] : (R)1;
            for (int iy = 0; iy < w; ++iy) {
                int ly = ly0 + iy;
                if (ly >= nfy) ly -= nfy;
                const R fzy = fz * wy[iy];
                C *row = g + ((int64_t)lz * nfy + ly) * nfx;
                int lx = lx0;
                for (int ix = 0; ix < w; ++ix) {
                    const R f = fzy * wx[ix];
                    atomicAdd(&row[lx].x, (R)v.x * f);
                    atomicAdd(&row[lx].y, (R)v.y * f);
                    if (++lx == nfx) lx = 0;
                }
            }
        }
    }
}

// c[p * cstride + m] = sum over the w^dims grid points near sample m of
// fine[p][...] psi_z psi_y psi_x.
template <int DIMS>
__global__ void __launch_bounds__(256) k_interp(float2 *c, int64_t cstride, int n,
                                                const float2 *__restrict__ fine,
                                                const float *__restrict__ traj, int64_t npts,
                                                const int *__restrict__ perm, int nfx, int nfy,
                                                int nfz, int w, double beta) {
    const int64_t nfvol = (int64_t)nfx * nfy * nfz;
    const int64_t total = (int64_t)n * npts;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = perm ? (int64_t)__ldg(perm + q % npts) : q % npts;
        const int p = (int)(q / npts);
        float wx[16], wy[16], wz[16];
        const int lx0 = es_axis<float>(__ldg(traj + m), nfx, w, beta, wx);
        const int ly0 = es_axis<float>(__ldg(traj + npts + m), nfy, w, beta, wy);
        int lz0 = 0;
        if constexpr (DIMS == 3) lz0 = es_axis<float>(__ldg(traj + 2 * npts + m), nfz, w, beta, wz);
        const float2 *g = fine + p * nfvol;
        float2 acc = make_float2(0.f, 0.f);
        for (int iz = 0; iz < (DIMS == 3 ? w : 1); ++iz) {
            int lz = lz0 + iz;
            if (lz >= nfz) lz -= nfz;
            const float fz = DIMS == 3 ? wz[iz] : 1.f;
            for (int iy = 0; iy < w; ++iy) {
                int ly = ly0 + iy;
                if (ly >= nfy) ly -= nfy;
                const float fzy = fz * wy[iy];
                const float2 *row = g + ((int64_t)lz * nfy + ly) * nfx;
                float2 r = make_float2(0.f, 0.f);
                int lx = lx0;
                for (int ix = 0; ix < w; ++ix) {
                    const float2 v = __ldg(row + lx);
                    r.x += v.x * wx[ix];
                    r.y += v.y * wx[ix];
                    if (++lx == nfx) lx = 0;
                }
                acc.x += r.x * fzy;
                acc.y += r.y * fzy;
            }
        }
        c[p * cstride + m] = acc;
    }
}

// Grid bin of every sample's nearest grid point below it (bins of bs points
// per axis, nb[d] bins along axis d, x fastest) and the identity
// permutation, to be sorted by bin.
__global__ void k_bin_keys(const float *__restrict__ traj, int64_t npts, int dims, int nfx,
                           int nfy, int nfz, int bs, int nbx, int nby, int *keys, int *perm) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < npts;
         m += (int64_t)gridDim.x * blockDim.x) {
        const int nf[3] = {nfx, nfy, nfz};
        int b[3] = {0, 0, 0};
        for (int d = 0; d < dims; ++d) {
            const double u = (double)__ldg(traj + d * npts + m) * nf[d] * (1.0 / (2.0 * kPi));
            int64_t l = (int64_t)floor(u) % nf[d];
            if (l < 0) l += nf[d];
            b[d] = (int)(l / bs);
        }
        keys[m] = (b[2] * nby + b[1]) * nbx + b[0];
        perm[m] = (int)m;
    }
}

// out[p][z][y][x] = in[p][z][y][x] * dx[x] * dy[y] * dz[z] (in place allowed)
__global__ void k_deconv(float2 *out, const float2 *in, int n, int Mx, int My, int Mz,
                         const float *__restrict__ dx, const float *__restrict__ dy,
                         const float *__restrict__ dz) {
    const int64_t vol = (int64_t)Mx * My * Mz;
    const int64_t total = (int64_t)n * vol;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = q % vol;
        const int x = (int)(r % Mx);
        const int y = (int)((r / Mx) % My);
        const int z = (int)(r / ((int64_t)Mx * My));
        const float f = __ldg(dx + x) * __ldg(dy + y) * __ldg(dz + z);
        const float2 v = in[q];
        out[q] = make_float2(v.x * f, v.y * f);
    }
}

__global__ void k_narrow(float2 *out, const double2 *__restrict__ in, int64_t n) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = in[q];
        out[q] = make_float2((float)v.x, (float)v.y);
    }
}

// FFT along the contiguous axis: `rows` rows, from src (row stride s_row,
// n_in samples read from index shift_in, wrapping) to dst (row stride d_row,
// n_out outputs from index shift_out, wrapping).
int fft_rows(int dir, const mr_fft_axis &ax, const float2 *src, int64_t s_row, int n_in,
             int shift_in, float2 *dst, int64_t d_row, int n_out, int shift_out, int64_t rows,
             cudaStream_t s) {
    mr_x_args a;
    std::memset(&a, 0, sizeof(a));
    a.ax = ax;
    a.rows_cta = 4;
    const size_t lim = (size_t)mr_smem_limit();
    while (a.rows_cta > 1 && mr_xplain_smem(ax.M, a.rows_cta) > lim) a.rows_cta >>= 1;
    if (mr_xplain_smem(ax.M, a.rows_cta) > lim)
        MR_FAIL(MR_ERR_UNSUPPORTED, "NUFFT: a grid line of %d points exceeds shared memory", ax.M);
    a.src = src;
    a.dst = dst;
    a.s_row = s_row;
    a.d_row = d_row;
    a.nrows = rows;
    a.n_in = n_in;
    a.shift_in = shift_in;
    a.n_out = n_out;
    a.shift_out = shift_out;
    a.scale = 1.f;
    return mr_launch_xplain(dir, a, s);
}

// FFT along a strided axis of nplane planes of nouter blocks of
// [axis][nfast] elements.
int fft_strided(int dir, const mr_fft_axis &ax, int nfast, int nouter, int nplane,
                const float2 *src, int64_t s_plane, int64_t s_outer, int64_t s_axis, int n_in,
                int shift_in, float2 *dst, int64_t d_plane, int64_t d_outer, int64_t d_axis,
                int n_out, int shift_out, cudaStream_t s) {
    mr_strided_args a;
    std::memset(&a, 0, sizeof(a));
    const size_t lim = (size_t)mr_smem_limit();
    a.ax = ax;
    a.nfast = nfast;
    a.xt = mr_pick_xt(ax.M, n_out, MR_SM_BUF, nfast, lim / 2);
    if (a.xt <= 0 || mr_strided_smem(ax.M, a.xt, n_out, MR_SM_BUF) > lim)
        MR_FAIL(MR_ERR_UNSUPPORTED, "NUFFT: a grid line of %d points exceeds shared memory", ax.M);
    a.nxt = (int)mr_cdiv(nfast, a.xt);
    a.nouter = nouter;
    a.nplane = nplane;
    a.src = src;
    a.s_plane = s_plane;
    a.s_outer = s_outer;
    a.s_axis = s_axis;
    a.n_in = n_in;
    a.shift_in = shift_in;
    a.dst = dst;
    a.d_plane = d_plane;
    a.d_outer = d_outer;
    a.d_axis = d_axis;
    a.n_out = n_out;
    a.shift_out = shift_out;
    a.scale = 1.f;
    return mr_launch_strided(dir, MR_LM_BUF, MR_SM_BUF, a, s);
}

}  // namespace

size_t mr_nufft_plan_bytes(int dims, const int *modes, double eps, double sigma, int max_planes,
                           int fp64) {
    int M[3], nf[3], w;
    double beta;
    plan_dims(dims, modes, eps, sigma, M, nf, &w, &beta);
    const bytes_of b = plan_sizes(dims, M, nf, max_planes, fp64);
    return b.fine + b.fine64 + b.A + b.B + b.D + b.tw + b.dec;
}

int mr_nufft_width(const mr_nufft *p) { return p->w; }

void mr_nufft_grid(const mr_nufft *p, int *nf) {
    for (int d = 0; d < 3; ++d) nf[d] = p->nf[d];
}

void mr_nufft_destroy(mr_nufft *p) {
    if (!p) return;
    for (void *q : {(void *)p->tw, (void *)p->ideconv, (void *)p->fine, (void *)p->fine64,
                    (void *)p->A, (void *)p->B, (void *)p->D, (void *)p->perm})
        if (q) cudaFree(q);
    cudaGetLastError();
    delete p;
}

int mr_nufft_create(int dims, const int *modes, const float *traj, int64_t npts, double eps,
                    double sigma, int max_planes, int fp64, mr_nufft **out) {
    *out = nullptr;
    MR_REQUIRE(dims == 2 || dims == 3, "NUFFT: dims = %d must be 2 or 3", dims);
    MR_REQUIRE(npts >= 1 && max_planes >= 1, "NUFFT: empty plan");
    for (int d = 0; d < dims; ++d)
        MR_REQUIRE(modes[d] >= 1, "NUFFT: mode count %d of axis %d must be >= 1", modes[d], d);
    mr_nufft *p = new (std::nothrow) mr_nufft();
    if (!p) MR_FAIL(MR_ERR_ALLOC, "NUFFT: cannot allocate the plan");
    p->dims = dims;
    plan_dims(dims, modes, eps, sigma, p->M, p->nf, &p->w, &p->beta);
    p->npts = npts;
    p->traj = traj;
    p->maxp = max_planes;
    p->fp64 = fp64;
    int rc = MR_SUCCESS;
    int off[3], tot = 0;
    for (int d = 0; d < 3 && rc == MR_SUCCESS; ++d) {
        rc = mr_fft_factor(p->nf[d], &p->ax[d]);
        off[d] = tot;
        tot += p->nf[d];
    }
    if (rc != MR_SUCCESS) {
        mr_nufft_destroy(p);
        return rc;
    }
    // 1 / psihat(k) per axis, k = j - floor(M / 2)
    std::vector<float> dec((size_t)p->M[0] + p->M[1] + p->M[2]);
    {
        std::vector<double> zq, wq;
        gauss_legendre(2 * p->w + 48, zq, wq);
        size_t o = 0;
        for (int d = 0; d < 3; ++d) {
            for (int j = 0; j < p->M[d]; ++j, ++o) {
                if (d >= dims) {
                    dec[o] = 1.f;
                    continue;
                }
                const double k = (double)(j - p->M[d] / 2);
                const double th = k * p->w * kPi / p->nf[d];
                double acc = 0.0;
                for (size_t q = 0; q < zq.size(); ++q)
                    acc += wq[q] * std::exp(p->beta * (std::sqrt(1.0 - zq[q] * zq[q]) - 1.0)) *
                           std::cos(th * zq[q]);
                dec[o] = (float)(1.0 / (0.5 * p->w * acc));
            }
        }
    }
    std::vector<float2> h(tot);
    for (int d = 0; d < 3; ++d) mr_fft_twiddles(p->nf[d], h.data() + off[d]);
    const bytes_of b = plan_sizes(dims, p->M, p->nf, max_planes, fp64);
    cudaError_t e = cudaMalloc(&p->tw, b.tw);
    if (e == cudaSuccess) e = cudaMalloc(&p->ideconv, b.dec);
    if (e == cudaSuccess) e = cudaMalloc(&p->fine, b.fine);
    if (e == cudaSuccess && fp64) e = cudaMalloc(&p->fine64, b.fine64);
    if (e == cudaSuccess) e = cudaMalloc(&p->A, b.A);
    if (e == cudaSuccess && dims == 3) e = cudaMalloc(&p->B, b.B);
    if (e == cudaSuccess) e = cudaMalloc(&p->D, b.D);
    if (e != cudaSuccess) {
        mr_nufft_destroy(p);
        MR_FAIL(MR_ERR_ALLOC, "NUFFT: cannot allocate %.2f GB of grids and tables",
                (b.fine + b.fine64 + b.A + b.B + b.D) / 1e9);
    }
    e = cudaMemcpy(p->tw, h.data(), b.tw, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->ideconv, dec.data(), b.dec, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        mr_nufft_destroy(p);
        MR_FAIL(MR_ERR_CUDA, "NUFFT: uploading the tables failed: %s", cudaGetErrorString(e));
    }
    for (int d = 0; d < 3; ++d) p->ax[d].tw = p->tw + off[d];
    // samples in grid-bin order (16^3 bins in 3-D, 32^2 in 2-D)
    if (npts <= 0x7fffffffLL && mr_env_int("MR_AHA_B200_NUFFT_NOSORT", 0) == 0) {
        const int bs = dims == 3 ? 16 : 32;
        const int nbx = (int)mr_cdiv(p->nf[0], bs), nby = (int)mr_cdiv(p->nf[1], bs);
        int *keys = nullptr;
        e = cudaDeviceSynchronize();  // the caller's trajectory is complete
        if (e == cudaSuccess) e = cudaMalloc(&p->perm, (size_t)npts * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&keys, (size_t)npts * sizeof(int));
        if (e == cudaSuccess) {
            k_bin_keys<<<grid_of(npts), 256>>>(traj, npts, dims, p->nf[0], p->nf[1], p->nf[2], bs,
                                                nbx, nby, keys, p->perm);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            try {
                thrust::sort_by_key(thrust::device, keys, keys + npts, p->perm);
                e = cudaDeviceSynchronize();
            } catch (...) {
                e = cudaErrorUnknown;
            }
        }
        if (keys) cudaFree(keys);
        if (e != cudaSuccess) {
            cudaGetLastError();
            mr_nufft_destroy(p);
            MR_FAIL(MR_ERR_CUDA, "NUFFT: sorting the samples by grid bin failed: %s",
                    cudaGetErrorString(e));
        }
    }
    *out = p;
    return MR_SUCCESS;
}

int mr_nufft_type1(mr_nufft *p, int iflag, const void *c, int64_t cstride, int64_t bcast, int n,
                   float2 *f, cudaStream_t s) {
    MR_REQUIRE(n >= 1 && n <= p->maxp, "NUFFT: %d planes outside [1, %d]", n, p->maxp);
    const int dir = iflag < 0 ? -1 : 1;
    const int nfx = p->nf[0], nfy = p->nf[1], nfz = p->nf[2];
    const int Mx = p->M[0], My = p->M[1], Mz = p->M[2];
    const int64_t nfvol = (int64_t)nfx * nfy * nfz;
    const int64_t total = (int64_t)n * p->npts;
    if (p->fp64) {
        MR_CUDA_TRY(cudaMemsetAsync(p->fine64, 0, (size_t)n * nfvol * sizeof(double2), s));
        if (p->dims == 3)
            k_spread<3, double><<<grid_of(total), 256, 0, s>>>(p->fine64, c, cstride, bcast, n,
                                                               p->traj, p->npts, p->perm, nfx, nfy,
                                                               nfz, p->w, p->beta);
        else
            k_spread<2, double><<<grid_of(total), 256, 0, s>>>(p->fine64, c, cstride, bcast, n,
                                                               p->traj, p->npts, p->perm, nfx, nfy,
                                                               nfz, p->w, p->beta);
        MR_LAUNCH_CHECK("k_spread");
        k_narrow<<<grid_of(n * nfvol), 256, 0, s>>>(p->fine, p->fine64, n * nfvol);
        MR_LAUNCH_CHECK("k_narrow");
    } else {
        MR_CUDA_TRY(cudaMemsetAsync(p->fine, 0, (size_t)n * nfvol * sizeof(float2), s));
        if (p->dims == 3)
            k_spread<3, float><<<grid_of(total), 256, 0, s>>>(p->fine, c, cstride, bcast, n,
                                                              p->traj, p->npts, p->perm, nfx, nfy,
                                                              nfz, p->w, p->beta);
        else
            k_spread<2, float><<<grid_of(total), 256, 0, s>>>(p->fine, c, cstride, bcast, n,
                                                              p->traj, p->npts, p->perm, nfx, nfy,
                                                              nfz, p->w, p->beta);
        MR_LAUNCH_CHECK("k_spread");
    }
    // x: grid rows -> the Mx centred modes
    int rc = fft_rows(dir, p->ax[0], p->fine, nfx, nfx, 0, p->A, Mx, Mx, Mx / 2,
                      (int64_t)n * nfz * nfy, s);
    if (rc != MR_SUCCESS) return rc;
    // y: [nfz][nfy][Mx] -> [nfz][My][Mx] (3-D into B, else straight into f)
    float2 *ydst = p->dims == 3 ? p->B : f;
    rc = fft_strided(dir, p->ax[1], Mx, nfz, n, p->A, (int64_t)nfz * nfy * Mx, (int64_t)nfy * Mx,
                     Mx, nfy, 0, ydst, (int64_t)nfz * My * Mx, (int64_t)My * Mx, Mx, My, My / 2, s);
    if (rc != MR_SUCCESS) return rc;
    if (p->dims == 3) {
        rc = fft_strided(dir, p->ax[2], My * Mx, 1, n, p->B, (int64_t)nfz * My * Mx, 0,
                         (int64_t)My * Mx, nfz, 0, f, (int64_t)Mz * My * Mx, 0, (int64_t)My * Mx,
                         Mz, Mz / 2, s);
        if (rc != MR_SUCCESS) return rc;
    }
    const int64_t mvol = (int64_t)Mx * My * Mz;
    k_deconv<<<grid_of(n * mvol), 256, 0, s>>>(f, f, n, Mx, My, Mz, p->ideconv, p->ideconv + Mx,
                                               p->ideconv + Mx + My);
    MR_LAUNCH_CHECK("k_deconv");
    return MR_SUCCESS;
}

int mr_nufft_type2(mr_nufft *p, int iflag, const float2 *f, int n, float2 *c, int64_t cstride,
                   cudaStream_t s) {
    MR_REQUIRE(n >= 1 && n <= p->maxp, "NUFFT: %d planes outside [1, %d]", n, p->maxp);
    const int dir = iflag < 0 ? -1 : 1;
    const int nfx = p->nf[0], nfy = p->nf[1], nfz = p->nf[2];
    const int Mx = p->M[0], My = p->M[1], Mz = p->M[2];
    const int64_t mvol = (int64_t)Mx * My * Mz;
    k_deconv<<<grid_of(n * mvol), 256, 0, s>>>(p->D, f, n, Mx, My, Mz, p->ideconv,
                                               p->ideconv + Mx, p->ideconv + Mx + My);
    MR_LAUNCH_CHECK("k_deconv");
    int rc;
    const float2 *ysrc = p->D;
    if (p->dims == 3) {
        // z: [Mz][My][Mx] centred -> [nfz][My][Mx], zero-padded
        rc = fft_strided(dir, p->ax[2], My * Mx, 1, n, p->D, mvol, 0, (int64_t)My * Mx, Mz, Mz / 2,
                         p->B, (int64_t)nfz * My * Mx, 0, (int64_t)My * Mx, nfz, 0, s);
        if (rc != MR_SUCCESS) return rc;
        ysrc = p->B;
    }
    // y: [nfz][My][Mx] -> [nfz][nfy][Mx]
    rc = fft_strided(dir, p->ax[1], Mx, nfz, n, ysrc, (int64_t)nfz * My * Mx, (int64_t)My * Mx, Mx,
                     My, My / 2, p->A, (int64_t)nfz * nfy * Mx, (int64_t)nfy * Mx, Mx, nfy, 0, s);
    if (rc != MR_SUCCESS) return rc;
    // x: rows of Mx centred modes -> grid rows of nfx
    rc = fft_rows(dir, p->ax[0], p->A, Mx, Mx, Mx / 2, p->fine, nfx, nfx, 0,
                  (int64_t)n * nfz * nfy, s);
    if (rc != MR_SUCCESS) return rc;
    const int64_t total = (int64_t)n * p->npts;
    if (p->dims == 3)
        k_interp<3><<<grid_of(total), 256, 0, s>>>(c, cstride, n, p->fine, p->traj, p->npts,
                                                   p->perm, nfx, nfy, nfz, p->w, p->beta);
    else
        k_interp<2><<<grid_of(total), 256, 0, s>>>(c, cstride, n, p->fine, p->traj, p->npts,
                                                   p->perm, nfx, nfy, nfz, p->w, p->beta);
    MR_LAUNCH_CHECK("k_interp");
    return MR_SUCCESS;
}

// ---------------------------------------------------------------------------
// NUFFT-method operator
// ---------------------------------------------------------------------------

struct mr_nufft_op {
    mr_config cfg;
    mr_nufft *plan;
    float *traj;        // coordinate d of sample m at traj[d * M + m], m = t + Ntrajs r
    float2 *gram;       // phi2 copy: B_{t,kz}[p][l] at ((l L + p) nkz + kz) Ntrajs + t
    float2 *im;         // [L][Nz][Ny][Nx] (2-D: [L][Ny][Nx]) of one coil
    float2 *ks, *ks2;   // samples [L][nkz][M]
    float2 *zmod;       // stack: exp(2 pi i floor(Nz / 2) z / Nz)
    float2 *ztw;        // stack: twiddles of the z FFT
    mr_fft_axis zax;
    int64_t Ntrajs, Nkx, M;
    int nkz, planes, chunk;
    size_t bytes;
};

namespace {

// im[l][v] = x[l][v] S[v] (times zmod[z] for a stack), v over the image
__global__ void k_nu_expand(float2 *im, const float2 *__restrict__ x, const float2 *__restrict__ S,
                            const float2 *__restrict__ zmod, int L, int64_t vimg, int64_t plane) {
    const int64_t total = (int64_t)L * vimg;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q % vimg;
        float2 s = __ldg(S + v);
        if (zmod) s = c_mul(s, __ldg(zmod + v / plane));
        im[q] = c_mul(s, __ldg(x + q));
    }
}

// out[l][v] (+)= conj(S[v] zmod[z]) im[l][v]
__global__ void k_nu_coilsum(float2 *out, const float2 *__restrict__ im,
                             const float2 *__restrict__ S, const float2 *__restrict__ zmod, int L,
                             int64_t vimg, int64_t plane, int accumulate) {
    const int64_t total = (int64_t)L * vimg;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q % vimg;
        float2 s = __ldg(S + v);
        if (zmod) s = c_mul(s, __ldg(zmod + v / plane));
        const float2 r = c_mulc(s, __ldg(im + q));
        out[q] = accumulate ? c_add(out[q], r) : r;
    }
}

// ks2[l][kz][m] = sum_p ks[p][kz][m] B_{t,kz}[p][l], t = m % Ntrajs (the rank
// row vector of every sample multiplied by its readout's Gram block from
// the right)
template <int LMAX>
__global__ void k_nu_gram(float2 *ks2, const float2 *__restrict__ ks,
                          const float2 *__restrict__ gram, int L, int nkz, int64_t M,
                          int64_t Ntrajs) {
    const int64_t total = (int64_t)nkz * M;
    const int64_t pstride = (int64_t)nkz * M;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = q % M;
        const int kz = (int)(q / M);
        const int64_t t = m % Ntrajs;
        float2 v[LMAX];
        for (int p = 0; p < L; ++p) v[p] = __ldg(ks + p * pstride + q);
        for (int l = 0; l < L; ++l) {
            float2 acc = make_float2(0.f, 0.f);
            for (int p = 0; p < L; ++p) {
                const float2 b = __ldg(gram + (((int64_t)l * L + p) * nkz + kz) * Ntrajs + t);
                acc = c_add(acc, c_mul(v[p], b));
            }
            ks2[l * pstride + q] = acc;
        }
    }
}

// traj copy in sample order m = t + Ntrajs r, coordinate-major (the
// caller's row-major (ndim, Nkx, Ntrajs) array is already that layout)
}  // namespace

size_t mr_nufft_op_bytes(const mr_nufft_op *e) { return e ? e->bytes : 0; }

void mr_nufft_op_destroy(mr_nufft_op *e) {
    if (!e) return;
    mr_nufft_destroy(e->plan);
    for (void *q : {(void *)e->traj, (void *)e->gram, (void *)e->im, (void *)e->ks,
                    (void *)e->ks2, (void *)e->zmod, (void *)e->ztw})
        if (q) cudaFree(q);
    cudaGetLastError();
    delete e;
}

int mr_nufft_op_create(const mr_config *cfg, const float2 *phi2, const float *traj,
                       int64_t Ntrajs, int64_t Nkx, double upsampfac, cudaStream_t s,
                       mr_nufft_op **out) {
    *out = nullptr;
    MR_REQUIRE(cfg->L <= 64, "NUFFT method: L = %d above 64 is not supported", cfg->L);
    mr_nufft_op *e = new (std::nothrow) mr_nufft_op();
    if (!e) MR_FAIL(MR_ERR_ALLOC, "NUFFT method: cannot allocate the engine");
    e->cfg = *cfg;
    const bool stack = cfg->traj_type == MR_TRAJ_STACK;
    const bool three = cfg->traj_type == MR_TRAJ_3D;
    const int ndim = three ? 3 : 2;
    const int L = cfg->L;
    e->Ntrajs = Ntrajs;
    e->Nkx = Nkx;
    e->M = Ntrajs * Nkx;
    e->nkz = stack ? cfg->n_dim[2] : 1;
    e->planes = L * e->nkz;
    const int64_t vimg = mr_image_size(cfg);
    const int modes[3] = {cfg->n_dim[0], cfg->n_dim[1], three ? cfg->n_dim[2] : 1};
    // planes per NUFFT call within half the memory budget
    size_t budget = 0;
    int rc = mr_memory_budget(cfg, &budget);
    if (rc != MR_SUCCESS) {
        delete e;
        return rc;
    }
    const size_t fixed = (size_t)e->M * ndim * sizeof(float) +
                         (size_t)Ntrajs * e->nkz * L * L * sizeof(float2) +
                         (size_t)vimg * L * sizeof(float2) +
                         2 * (size_t)e->planes * e->M * sizeof(float2);
    const size_t per_plane = mr_nufft_plan_bytes(ndim, modes, cfg->eps, upsampfac, 1, 0);
    int64_t chunk = budget > fixed ? (int64_t)((budget - fixed) / 2 / per_plane) : 1;
    chunk = std::max<int64_t>(1, std::min<int64_t>(chunk, e->planes));
    e->chunk = (int)chunk;
    cudaError_t ce = cudaMalloc(&e->traj, (size_t)e->M * ndim * sizeof(float));
    if (ce == cudaSuccess)
        ce = cudaMalloc(&e->gram, (size_t)Ntrajs * e->nkz * L * L * sizeof(float2));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->im, (size_t)vimg * L * sizeof(float2));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->ks, (size_t)e->planes * e->M * sizeof(float2));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->ks2, (size_t)e->planes * e->M * sizeof(float2));
    if (ce != cudaSuccess) {
        mr_nufft_op_destroy(e);
        MR_FAIL(MR_ERR_ALLOC, "NUFFT method: cannot allocate the %.2f GB engine buffers",
                fixed / 1e9);
    }
    ce = cudaMemcpyAsync(e->traj, traj, (size_t)e->M * ndim * sizeof(float),
                         cudaMemcpyDeviceToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(e->gram, phi2, (size_t)Ntrajs * e->nkz * L * L * sizeof(float2),
                             cudaMemcpyDeviceToDevice, s);
    if (ce != cudaSuccess) {
        mr_nufft_op_destroy(e);
        MR_FAIL(MR_ERR_CUDA, "NUFFT method: copying the inputs failed: %s",
                cudaGetErrorString(ce));
    }
    e->bytes = fixed;
    if (stack) {
        const int nz = cfg->n_dim[2];
        std::vector<float2> zm(nz), tw(nz);
        for (int z = 0; z < nz; ++z) {
            const double ph = 2.0 * kPi * (double)(nz / 2) * (double)z / (double)nz;
            zm[z] = make_float2((float)std::cos(ph), (float)std::sin(ph));
        }
        rc = mr_fft_factor(nz, &e->zax);
        if (rc != MR_SUCCESS) {
            mr_nufft_op_destroy(e);
            return rc;
        }
        mr_fft_twiddles(nz, tw.data());
        ce = cudaMalloc(&e->zmod, nz * sizeof(float2));
        if (ce == cudaSuccess) ce = cudaMalloc(&e->ztw, nz * sizeof(float2));
        if (ce == cudaSuccess)
            ce = cudaMemcpy(e->zmod, zm.data(), nz * sizeof(float2), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess)
            ce = cudaMemcpy(e->ztw, tw.data(), nz * sizeof(float2), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) {
            mr_nufft_op_destroy(e);
            MR_FAIL(MR_ERR_CUDA, "NUFFT method: z tables failed: %s", cudaGetErrorString(ce));
        }
        e->zax.tw = e->ztw;
        e->bytes += 2 * nz * sizeof(float2);
    }
    rc = mr_nufft_create(ndim, modes, e->traj, e->M, cfg->eps, upsampfac, e->chunk, 0, &e->plan);
    if (rc != MR_SUCCESS) {
        mr_nufft_op_destroy(e);
        return rc;
    }
    e->bytes += mr_nufft_plan_bytes(ndim, modes, cfg->eps, upsampfac, e->chunk, 0);
    ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) {
        mr_nufft_op_destroy(e);
        MR_FAIL(MR_ERR_CUDA, "NUFFT method: creation failed: %s", cudaGetErrorString(ce));
    }
    *out = e;
    return MR_SUCCESS;
}

int mr_nufft_op_apply(mr_nufft_op *e, const float2 *x, const float2 *S, float2 *out,
                      cudaStream_t s) {
    const mr_config &cfg = e->cfg;
    const bool stack = cfg.traj_type == MR_TRAJ_STACK;
    const int L = cfg.L;
    const int64_t vimg = mr_image_size(&cfg);
    const int64_t plane = (int64_t)cfg.n_dim[0] * cfg.n_dim[1];
    const int64_t mvol = stack ? plane : vimg;  // modes of one NUFFT plane
    const int nz = cfg.n_dim[2];
    int rc = MR_SUCCESS;
    for (int c = 0; c < cfg.n_coils; ++c) {
        const float2 *Sc = S + (int64_t)c * vimg;
        k_nu_expand<<<grid_of(L * vimg), 256, 0, s>>>(e->im, x, Sc, stack ? e->zmod : nullptr, L,
                                                      vimg, plane);
        MR_LAUNCH_CHECK("k_nu_expand");
        if (stack) {
            // plain FFT along z of every rank (the z modulation makes it the
            // centred one up to a kz phase that cancels with the inverse)
            rc = fft_strided(-1, e->zax, (int)plane, 1, L, e->im, vimg, 0, plane, nz, 0, e->im,
                             vimg, 0, plane, nz, 0, s);
            if (rc != MR_SUCCESS) return rc;
        }
        for (int p0 = 0; p0 < e->planes; p0 += e->chunk) {
            const int n = std::min(e->chunk, e->planes - p0);
            rc = mr_nufft_type2(e->plan, -1, e->im + (int64_t)p0 * mvol, n, e->ks + p0 * e->M,
                                e->M, s);
            if (rc != MR_SUCCESS) return rc;
        }
        const int64_t tot = (int64_t)e->nkz * e->M;
        if (L <= 16)
            k_nu_gram<16><<<grid_of(tot), 256, 0, s>>>(e->ks2, e->ks, e->gram, L, e->nkz, e->M,
                                                      e->Ntrajs);
        else
            k_nu_gram<64><<<grid_of(tot), 256, 0, s>>>(e->ks2, e->ks, e->gram, L, e->nkz, e->M,
                                                      e->Ntrajs);
        MR_LAUNCH_CHECK("k_nu_gram");
        for (int p0 = 0; p0 < e->planes; p0 += e->chunk) {
            const int n = std::min(e->chunk, e->planes - p0);
            rc = mr_nufft_type1(e->plan, 1, e->ks2 + p0 * e->M, e->M, 0, n,
                                e->im + (int64_t)p0 * mvol, s);
            if (rc != MR_SUCCESS) return rc;
        }
        if (stack) {
            rc = fft_strided(1, e->zax, (int)plane, 1, L, e->im, vimg, 0, plane, nz, 0, e->im,
                             vimg, 0, plane, nz, 0, s);
            if (rc != MR_SUCCESS) return rc;
        }
        k_nu_coilsum<<<grid_of(L * vimg), 256, 0, s>>>(out, e->im, Sc, stack ? e->zmod : nullptr,
                                                       L, vimg, plane, c > 0);
        MR_LAUNCH_CHECK("k_nu_coilsum");
    }
    return MR_SUCCESS;
}
