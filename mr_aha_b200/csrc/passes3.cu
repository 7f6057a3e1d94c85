// Passes with a compile-time-specialised FFT (fftfix.cuh) for the common
// lengths of the plans: the same data flow as the in-place kernels of
// passes2.cu, with the transform length, tile width / coil count and rank as
// template parameters. The plan uses these kernels when its geometry matches
// an instantiated configuration (mr_fixed_*), else the generic ones.
#include "engine.h"
#include "fftfix.cuh"

namespace {

// Block sizes: 512 threads for tiles of more than 10240 elements (one CTA per
// SM), 256 threads for smaller tiles, with registers capped so that two
// independent CTAs share an SM (one loads or stores while the other computes).

template <int DIR, int LM, int SM, int M, int XT, int kNT>
__global__ void __launch_bounds__(kNT, 512 / kNT) k_strided3(const __grid_constant__ mr_strided_args a) {
    extern __shared__ float2 sm[];
    constexpr int TILE = M * XT;
    float2 *acc = sm + TILE;
    int64_t bid = blockIdx.x;
    const int plane = (int)(bid % a.nplane);
    bid /= a.nplane;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const int ncl = (SM == MR_SM_COILSUM) ? a.ncoil : 1;
    const int64_t off0 = (int64_t)outer * a.s_outer + x0;
    const int64_t doff0 = (int64_t)outer * a.d_outer + x0;
    for (int cc = 0; cc < ncl; ++cc) {
        const int sp = (SM == MR_SM_COILSUM) ? cc * a.L + plane : plane;
        const float2 *srcp = nullptr, *xp = nullptr, *sp_s = nullptr;
        if constexpr (LM == MR_LM_BUF) {
            srcp = a.src + (int64_t)sp * a.s_plane + off0;
        } else {
            xp = a.xs_x + (int64_t)(sp % a.L) * a.img_plane + off0;
            sp_s = a.xs_s + (int64_t)(a.coil0 + sp / a.L) * a.img_plane + off0;
        }
        if constexpr (mrfix::factor(M).n >= 2) {
            // first pass reads global memory, last pass writes it: the tile
            // is x-major, so consecutive threads touch consecutive x
            auto load = [&](int b, int e) -> float2 {
                int sa = e + a.shift_in;
                if (sa >= M) sa -= M;
                float2 v = make_float2(0.f, 0.f);
                if (b < nx && sa < a.n_in) {
                    const int64_t o = (int64_t)sa * a.s_axis + b;
                    if constexpr (LM == MR_LM_BUF) v = srcp[o];
                    else v = c_mul(__ldg(sp_s + o), __ldg(xp + o));
                }
                return v;
            };
            auto store = [&](int b, int q, float2 v) {
                int da = q + a.shift_out;
                if (da >= M) da -= M;
                if (da < a.n_out && b < nx) {
                    if constexpr (SM == MR_SM_BUF) {
                        a.dst[(int64_t)plane * a.d_plane + doff0 + (int64_t)da * a.d_axis + b] =
                            c_scale(v, a.scale);
                    } else {
                        const float2 w = c_mulc(
                            __ldg(a.xs_s + (int64_t)(a.coil0 + cc) * a.img_plane + doff0 +
                                  (int64_t)da * a.d_axis + b),
                            v);
                        const int ai = da * XT + b;
                        acc[ai] = (cc == 0) ? w : c_add(acc[ai], w);
                    }
                }
            };
            mrfix::fft_io<true, true, DIR, M, XT, XT, 1, kNT>(sm, a.ax.tw, load, store);
            __syncthreads();
            continue;
        }
#pragma unroll 4
        for (int idx = threadIdx.x; idx < TILE; idx += kNT) {
            const int j = idx / XT;
            const int xx = idx % XT;
            int sa = j + a.shift_in;
            if (sa >= M) sa -= M;
            float2 v = make_float2(0.f, 0.f);
            if (xx < nx && sa < a.n_in) {
                const int64_t o = (int64_t)sa * a.s_axis + xx;
                if constexpr (LM == MR_LM_BUF) v = srcp[o];
                else v = c_mul(__ldg(sp_s + o), __ldg(xp + o));
            }
            sm[idx] = v;
        }
        __syncthreads();
        mrfix::fft<DIR, M, XT, XT, 1, kNT>(sm, a.ax.tw);
#pragma unroll 4
        for (int idx = threadIdx.x; idx < a.n_out * XT; idx += kNT) {
            const int da = idx / XT;
            const int xx = idx % XT;
            int q = da - a.shift_out;
            if (q < 0) q += M;
            const float2 v = sm[q * XT + xx];
            if constexpr (SM == MR_SM_BUF) {
                if (xx < nx)
                    a.dst[(int64_t)plane * a.d_plane + doff0 + (int64_t)da * a.d_axis + xx] =
                        c_scale(v, a.scale);
            } else {
                float2 w = make_float2(0.f, 0.f);
                if (xx < nx)
                    w = c_mulc(__ldg(a.xs_s + (int64_t)(a.coil0 + cc) * a.img_plane + doff0 +
                                     (int64_t)da * a.d_axis + xx),
                               v);
                acc[idx] = (cc == 0) ? w : c_add(acc[idx], w);
            }
        }
        __syncthreads();
    }
    if constexpr (SM == MR_SM_COILSUM) {
        for (int idx = threadIdx.x; idx < a.n_out * XT; idx += kNT) {
            const int da = idx / XT;
            const int xx = idx % XT;
            if (xx < nx) {
                float2 *o = a.dst + (int64_t)plane * a.d_plane + doff0 + (int64_t)da * a.d_axis + xx;
                const float2 v = c_scale(acc[idx], a.scale);
                *o = a.accumulate ? c_add(*o, v) : v;
            }
        }
    }
}

template <int M>
constexpr int odd_stride() {
    return (M % 2 == 0) ? M + 1 : M + 2;
}

template <int M, int L, int NC, int KF, int kNT>
__global__ void __launch_bounds__(kNT, 512 / kNT) k_xbd3(const __grid_constant__ mr_x_args a) {
    extern __shared__ float2 sm[];
    constexpr int LS = odd_stride<M>();
    constexpr int NL = NC * L;
    const int chunk = (int)(blockIdx.x % a.nchunk);
    const int loc = (int)(blockIdx.x / a.nchunk);
    const int jy = loc % a.My;
    const int jz = loc / a.My;
    const int c0 = chunk * NC;
    const int ncoils = min(NC, a.ncoil - c0);
    const int64_t pbase = (int64_t)c0 * L;
    const float2 *src = a.src + (pbase * a.plane_rows + loc) * a.s_row;
    const int64_t rstride = a.plane_rows * a.s_row;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < NL * M; idx += kNT) {
        const int b = idx / M;
        const int j = idx - b * M;
        int sa = j + a.shift_in;
        if (sa >= M) sa -= M;
        float2 v = make_float2(0.f, 0.f);
        if (b < ncoils * L && sa < a.n_in) v = src[b * rstride + sa];
        sm[b * LS + j] = v;
    }
    __syncthreads();
    mrfix::fft<-1, M, NL, 1, LS, kNT>(sm, a.ax.tw);
    const int ky = mr_nat2cent_d(jy, a.My, a.cmy);
    const int kz = mr_nat2cent_d(jz, a.Mz, a.cmz);
    constexpr int GW = 32 / NC;
    constexpr int ITEMS = NC * ((M + GW - 1) / GW) * GW;
    for (int w = threadIdx.x; w < ITEMS; w += kNT) {
        const int lane = w & 31;
        const int k = lane / GW;
        const int jx = (w >> 5) * GW + (lane - k * GW);
        if (jx >= M || k >= ncoils) continue;
        float2 v[1][L], y[1][L];
#pragma unroll
        for (int l = 0; l < L; ++l) v[0][l] = sm[(k * L + l) * LS + jx];
        bool zero = false;
        int64_t row;
        if (a.K.inv) {
            const int r = __ldg(a.K.inv + jx + (int64_t)M * (jy + (int64_t)a.My * jz));
            zero = r < 0;
            row = zero ? 0 : r;
        } else {
            row = mr_nat2cent_d(jx, M, a.cmx) + (int64_t)M * (ky + (int64_t)a.My * kz);
        }
        if (zero) {
#pragma unroll
            for (int l = 0; l < L; ++l) y[0][l] = make_float2(0.f, 0.f);
        } else {
            const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
            bd_block<L, 1, KF>(v, y, kl, a.upper);
        }
#pragma unroll
        for (int l = 0; l < L; ++l) sm[(k * L + l) * LS + jx] = y[0][l];
    }
    __syncthreads();
    mrfix::fft<1, M, NL, 1, LS, kNT>(sm, a.ax.tw);
    float2 *dst = a.dst + (pbase * a.plane_rows + loc) * a.d_row;
    const int64_t dstride = a.plane_rows * a.d_row;
    for (int idx = threadIdx.x; idx < ncoils * L * a.n_out; idx += kNT) {
        const int b = idx / a.n_out;
        const int da = idx - b * a.n_out;
        int q = da - a.shift_out;
        if (q < 0) q += M;
        dst[b * dstride + da] = c_scale(sm[b * LS + q], a.scale);
    }
}

// Pass 3 when the transform length is M = 2N, the row holds N samples (zero
// padding to M) and the output is cropped to the same window. The pad and
// crop phase ramps then cancel (the block multiply is diagonal in k), and
// with t[n] = W_M^n (W_M = exp(-2 pi i / M)):
//   X[2m] = FFT_N(x)[m],  X[2m+1] = FFT_N(x t)[m],
//   y[n]  = IFFT_N(Z_even)[n] + conj(t[n]) IFFT_N(Z_odd)[n],
// four length-N transforms of N-sample lines in place of two length-M
// transforms of half-empty ones. Row b = (coil, rank) of the tile keeps its
// even half-spectrum in line 2b and its odd one in line 2b + 1.
template <int N, int L, int NC, int KF, int kNT>
__global__ void __launch_bounds__(kNT, 512 / kNT) k_xbdh(const __grid_constant__ mr_x_args a) {
    extern __shared__ float2 sm[];
    constexpr int LS = odd_stride<N>();
    constexpr int NR = NC * L;
    constexpr int NL = 2 * NR;
    const int chunk = (int)(blockIdx.x % a.nchunk);
    const int loc = (int)(blockIdx.x / a.nchunk);
    const int jy = loc % a.My;
    const int jz = loc / a.My;
    const int c0 = chunk * NC;
    const int ncoils = min(NC, a.ncoil - c0);
    const int nrow = ncoils * L;
    const int64_t pbase = (int64_t)c0 * L;
    const float2 *tw = a.ax.tw;  // W_M^e, e < M
    const float2 *src = a.src + (pbase * a.plane_rows + loc) * a.s_row;
    const int64_t rstride = a.plane_rows * a.s_row;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < NR * N; idx += kNT) {
        const int b = idx / N;
        const int n = idx - b * N;
        float2 v = make_float2(0.f, 0.f);
        if (b < nrow) v = src[b * rstride + n];
        sm[(2 * b) * LS + n] = v;
        sm[(2 * b + 1) * LS + n] = c_mul(v, __ldg(tw + n));
    }
    __syncthreads();
    mrfix::fft<-1, N, NL, 1, LS, kNT, 2>(sm, tw);
    const int ky = mr_nat2cent_d(jy, a.My, a.cmy);
    const int kz = mr_nat2cent_d(jz, a.Mz, a.cmz);
    // a warp takes 16 consecutive m of one coil in both parities: lanes 0-15
    // the even k = 2m, lanes 16-31 the odd k = 2m + 1 (each half-warp reads
    // 16 consecutive words of one line)
    constexpr int MB = (N + 15) / 16;
    constexpr int ITEMS = NC * MB * 32;
    for (int w = threadIdx.x; w < ITEMS; w += kNT) {
        const int lane = w & 31;
        const int wi = w >> 5;
        const int k = wi / MB;
        const int m = (wi - k * MB) * 16 + (lane & 15);
        const int par = lane >> 4;
        if (m >= N || k >= ncoils) continue;
        const int jx = 2 * m + par;
        float2 *line = sm + (2 * k * L + par) * LS + m;
        float2 v[1][L], y[1][L];
#pragma unroll
        for (int l = 0; l < L; ++l) v[0][l] = line[2 * l * LS];
        bool zero = false;
        int64_t row;
        if (a.K.inv) {
            const int r = __ldg(a.K.inv + jx + (int64_t)(2 * N) * (jy + (int64_t)a.My * jz));
            zero = r < 0;
            row = zero ? 0 : r;
        } else {
            row = mr_nat2cent_d(jx, 2 * N, a.cmx) + (int64_t)(2 * N) * (ky + (int64_t)a.My * kz);
        }
        if (zero) {
#pragma unroll
            for (int l = 0; l < L; ++l) y[0][l] = make_float2(0.f, 0.f);
        } else {
            const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
            bd_block<L, 1, KF>(v, y, kl, a.upper);
        }
#pragma unroll
        for (int l = 0; l < L; ++l) line[2 * l * LS] = y[0][l];
    }
    __syncthreads();
    mrfix::fft<1, N, NL, 1, LS, kNT, 2>(sm, tw);
    float2 *dst = a.dst + (pbase * a.plane_rows + loc) * a.d_row;
    const int64_t dstride = a.plane_rows * a.d_row;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < nrow * N; idx += kNT) {
        const int b = idx / N;
        const int n = idx - b * N;
        const float2 e = sm[(2 * b) * LS + n];
        const float2 o = sm[(2 * b + 1) * LS + n];
        dst[b * dstride + n] = c_scale(c_add(e, c_mulc(__ldg(tw + n), o)), a.scale);
    }
}

template <typename F>
void set_attr(F *f, unsigned long long &mask) {
    const int dev = mr_current_device();
    if (!(mask & (1ull << dev))) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, mr_smem_limit());
        mask |= 1ull << dev;
    }
}

template <int DIR, int LM, int SM, int M, int XT>
int launch_s3(const mr_strided_args &a, cudaStream_t s) {
    constexpr int kNT = (M * XT > 10240) ? 512 : 256;
    static unsigned long long attr = 0;
    set_attr(k_strided3<DIR, LM, SM, M, XT, kNT>, attr);
    size_t smem = (size_t)M * XT * sizeof(float2);
    if (SM == MR_SM_COILSUM) smem += (size_t)a.n_out * XT * sizeof(float2);
    const int64_t nblk = (int64_t)a.nxt * a.nouter * a.nplane;
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
    k_strided3<DIR, LM, SM, M, XT, kNT><<<(unsigned)nblk, kNT, smem, s>>>(a);
    MR_LAUNCH_CHECK("k_strided3");
    return MR_SUCCESS;
}

template <int M, int L, int NC, int KF>
int launch_x3(const mr_x_args &a, cudaStream_t s) {
    constexpr int kNT = (NC * L * M > 10240) ? 512 : 256;
    static unsigned long long attr = 0;
    set_attr(k_xbd3<M, L, NC, KF, kNT>, attr);
    const size_t smem = (size_t)NC * L * odd_stride<M>() * sizeof(float2);
    const int64_t nblk = (int64_t)a.nloc * a.nchunk;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "block-diagonal pass grid too large");
    k_xbd3<M, L, NC, KF, kNT><<<(unsigned)nblk, kNT, smem, s>>>(a);
    MR_LAUNCH_CHECK("k_xbd3");
    return MR_SUCCESS;
}

template <int N, int L, int NC, int KF>
int launch_xh(const mr_x_args &a, cudaStream_t s) {
    constexpr int kNT = (NC * L * 2 * N > 10240) ? 512 : 256;
    static unsigned long long attr = 0;
    set_attr(k_xbdh<N, L, NC, KF, kNT>, attr);
    const size_t smem = (size_t)2 * NC * L * odd_stride<N>() * sizeof(float2);
    const int64_t nblk = (int64_t)a.nloc * a.nchunk;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "block-diagonal pass grid too large");
    k_xbdh<N, L, NC, KF, kNT><<<(unsigned)nblk, kNT, smem, s>>>(a);
    MR_LAUNCH_CHECK("k_xbdh");
    return MR_SUCCESS;
}

}  // namespace

// Instantiated strided configurations (length, tile width) and block-diagonal
// configurations (length, rank, coils per tile). Every strided one is built in
// the four modes the plans use.
#define MR_S3_LIST(X) \
    X(640, 32) X(640, 16) X(640, 8) X(56, 256) X(56, 128) X(56, 64) X(56, 32) X(56, 16) \
    X(128, 64) X(128, 32) X(8, 256)
#define MR_X3_LIST(X) X(640, 16, 2) X(640, 16, 1) X(128, 4, 4)
// half-length block-diagonal configurations (N = M / 2, rank, coils per tile)
#define MR_XH_LIST(X) X(320, 16, 1) X(64, 4, 4)

namespace {
// Shared memory a tile may take: half the per-block limit (two CTAs per SM)
// unless MR_AHA_B200_FULL_TILES is set.
size_t tile_budget(bool half) { return (size_t)mr_smem_limit() / (half ? 2 : 1); }
bool half_tiles() { return mr_env_int("MR_AHA_B200_FULL_TILES", 0) == 0; }
}  // namespace

int mr_fixed_strided_xt(int M, int smode, int want) {
    // `want` when it is instantiated and fits; else the widest instantiated
    // tile of this length for the store mode within the tile budget, the
    // full limit when no tile fits half of it
    int best = 0;
    if (want > 0) {
#define MR_S3_WANT(m, xt)                                                      \
        if (M == m && want == xt &&                                            \
            (size_t)m * xt * sizeof(float2) * (smode == MR_SM_COILSUM ? 2 : 1) <= \
                (size_t)mr_smem_limit())                                       \
            return xt;
        MR_S3_LIST(MR_S3_WANT)
#undef MR_S3_WANT
    }
    for (int pass = 0; pass < 2 && best == 0; ++pass) {
        const size_t budget = tile_budget(pass == 0 && half_tiles());
#define MR_S3_PICK(m, xt)                                                 \
        if (M == m) {                                                     \
            size_t b = (size_t)m * xt * sizeof(float2);                   \
            if (smode == MR_SM_COILSUM) b += (size_t)m * xt * sizeof(float2); \
            if (b <= budget && xt > best) best = xt;                      \
        }
        MR_S3_LIST(MR_S3_PICK)
#undef MR_S3_PICK
    }
    return best;
}

int mr_launch_strided3(int dir, int lmode, int smode, const mr_strided_args &a, cudaStream_t s) {
    const int M = a.ax.M, XT = a.xt;
#define MR_S3_CASE(m, xt)                                                                     \
    if (M == m && XT == xt) {                                                                 \
        if (dir < 0 && lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_s3<-1, 0, 0, m, xt>(a, s); \
        if (dir < 0 && lmode == MR_LM_XS && smode == MR_SM_BUF) return launch_s3<-1, 1, 0, m, xt>(a, s);  \
        if (dir > 0 && lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_s3<1, 0, 0, m, xt>(a, s);  \
        if (dir > 0 && lmode == MR_LM_BUF && smode == MR_SM_COILSUM) return launch_s3<1, 0, 1, m, xt>(a, s); \
    }
    MR_S3_LIST(MR_S3_CASE)
#undef MR_S3_CASE
    MR_FAIL(MR_ERR_INTERNAL, "no specialised strided pass for M = %d, tile %d", M, XT);
}

int mr_fixed_xbd_coils(int M, int L) {
    // the most coils per tile within the tile budget (as above)
    int nc = 0;
    for (int pass = 0; pass < 2 && nc == 0; ++pass) {
        const size_t budget = tile_budget(pass == 0 && half_tiles());
#define MR_X3_PICK(m, l, c)                                                         \
        if (M == m && L == l && (size_t)c * l * odd_stride<m>() * sizeof(float2) <= budget && \
            c > nc)                                                                 \
            nc = c;
        MR_X3_LIST(MR_X3_PICK)
#undef MR_X3_PICK
    }
    return nc;
}

int mr_launch_xbd3(const mr_x_args &a, cudaStream_t s) {
    const int M = a.ax.M;
#define MR_X3_CASE(m, l, c)                                                     \
    if (M == m && a.L == l && a.nc == c) {                                      \
        switch (a.K.kf) {                                                       \
            case MR_KF_F32: return launch_x3<m, l, c, MR_KF_F32>(a, s);         \
            case MR_KF_BF16: return launch_x3<m, l, c, MR_KF_BF16>(a, s);       \
            default: return launch_x3<m, l, c, MR_KF_I16>(a, s);                \
        }                                                                       \
    }
    MR_X3_LIST(MR_X3_CASE)
#undef MR_X3_CASE
    MR_FAIL(MR_ERR_INTERNAL, "no specialised block-diagonal pass for M = %d, L = %d", M, a.L);
}

int mr_fixed_xbdh_coils(int M, int n_in, int L) {
    if (M != 2 * n_in || mr_env_int("MR_AHA_B200_NO_HALF", 0)) return 0;
    const int N = n_in;
    int nc = 0;
#define MR_XH_PICK(n, l, c)                                                                  \
    if (N == n && L == l && (size_t)2 * c * l * odd_stride<n>() * sizeof(float2) <=          \
                                (size_t)mr_smem_limit() && c > nc)                           \
        nc = c;
    MR_XH_LIST(MR_XH_PICK)
#undef MR_XH_PICK
    return nc;
}

int mr_launch_xbdh(const mr_x_args &a, cudaStream_t s) {
    const int N = a.n_in;
    if (a.ax.M != 2 * N || a.n_out != N || a.shift_out != a.shift_in)
        MR_FAIL(MR_ERR_INTERNAL, "half-length block-diagonal pass needs M = 2 N and equal windows");
#define MR_XH_CASE(n, l, c)                                                   \
    if (N == n && a.L == l && a.nc == c) {                                    \
        switch (a.K.kf) {                                                     \
            case MR_KF_F32: return launch_xh<n, l, c, MR_KF_F32>(a, s);       \
            case MR_KF_BF16: return launch_xh<n, l, c, MR_KF_BF16>(a, s);     \
            default: return launch_xh<n, l, c, MR_KF_I16>(a, s);              \
        }                                                                     \
    }
    MR_XH_LIST(MR_XH_CASE)
#undef MR_XH_CASE
    MR_FAIL(MR_ERR_INTERNAL, "no half-length block-diagonal pass for N = %d, L = %d", N, a.L);
}

int mr_fixed_strided_list(int M, int smode, int *xt, int max) {
    // every instantiated tile width of this length that fits the per-block
    // shared memory limit, for the autotuner
    int n = 0;
#define MR_S3_LISTPICK(m, w)                                                                \
    if (M == m && n < max &&                                                                \
        (size_t)m * w * sizeof(float2) * (smode == MR_SM_COILSUM ? 2 : 1) <=                \
            (size_t)mr_smem_limit())                                                        \
        xt[n++] = w;
    MR_S3_LIST(MR_S3_LISTPICK)
#undef MR_S3_LISTPICK
    return n;
}

int mr_fixed_xbd_list(int M, int L, int *nc, int max) {
    int n = 0;
#define MR_X3_LISTPICK(m, l, c)                                                             \
    if (M == m && L == l && n < max &&                                                      \
        (size_t)c * l * odd_stride<m>() * sizeof(float2) <= (size_t)mr_smem_limit())        \
        nc[n++] = c;
    MR_X3_LIST(MR_X3_LISTPICK)
#undef MR_X3_LISTPICK
    return n;
}
