// FFT passes of the apply and of the kernel finish.
//
// Every pass transforms lines along one axis inside shared memory (Stockham,
// fft_device.cuh) and fuses the index work around it:
//  * load map: natural index j of the transform reads source index
//    a = (j + shift_in) mod M, or zero when a >= n_in. With shift_in =
//    floor(N/2) this is the zero-pad scatter of the reference's
//    mr_k_pad_mul_se (src/cuda/mr_kernels.cu:98-142); with shift_in =
//    floor(M/2) and n_in = M it is the centred-to-natural shift of
//    mr_k_to_natural (mr_kernels.cu:364-393);
//  * store map: destination index a < n_out takes transform output
//    q = (a - shift_out) mod M: the crop of mr_k_crop_mul_conj_se
//    (mr_kernels.cu:144-176) or the natural-to-centred shift of
//    mr_k_to_centered_scale (mr_kernels.cu:395-425);
//  * the coil-map product S_c x_l on the first forward pass and the
//    conj(S_c) coil sum on the last inverse pass;
//  * the packed Hermitian block multiply between the forward and inverse
//    transform of the contiguous axis (bd_device.cuh).
#include "engine.h"

#include <cmath>
#include <vector>

// ---------------------------------------------------------------------------
// FFT plan helpers
// ---------------------------------------------------------------------------

int mr_fft_factor(int M, mr_fft_axis *ax) {
    ax->M = M;
    ax->npass = 0;
    int n = M, e2 = 0;
    while (n % 2 == 0) {
        n /= 2;
        ++e2;
    }
    auto push = [&](int r) -> bool {
        if (ax->npass >= MR_FFT_MAX_PASSES) return false;
        ax->radix[ax->npass++] = r;
        return true;
    };
    while (e2 >= 3) {
        if (!push(8)) return MR_ERR_UNSUPPORTED;
        e2 -= 3;
    }
    if (e2 == 2 && !push(4)) return MR_ERR_UNSUPPORTED;
    if (e2 == 1 && !push(2)) return MR_ERR_UNSUPPORTED;
    const int small[3] = {5, 3, 7};
    for (int p : small)
        while (n % p == 0) {
            if (!push(p)) return MR_ERR_UNSUPPORTED;
            n /= p;
        }
    for (int p = 11; n > 1 && p <= MR_FFT_MAX_GENERIC_RADIX; p += 2)
        while (n % p == 0) {
            if (!push(p)) return MR_ERR_UNSUPPORTED;
            n /= p;
        }
    if (n > 1)
        MR_FAIL(MR_ERR_UNSUPPORTED,
                "FFT length %d has a prime factor %d above the supported %d", M, n,
                MR_FFT_MAX_GENERIC_RADIX);
    int prod = 1;
    ax->small = 1;
    for (int s = 0; s < ax->npass; ++s) {
        ax->p[s] = prod;
        ax->fp[s] = mr_make_fdiv((unsigned)prod);
        const int r = ax->radix[s];
        if (!(r == 2 || r == 3 || r == 4 || r == 5 || r == 7 || r == 8)) ax->small = 0;
        prod *= r;
    }
    return MR_SUCCESS;
}

void mr_fft_twiddles(int M, float2 *h) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int e = 0; e < M; ++e) {
        const double a = -two_pi * (double)e / (double)M;
        h[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
}

int mr_current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev > 63) return 0;
    return dev;
}

int mr_smem_limit() {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 48 * 1024;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
        cudaSuccess)
        return 48 * 1024;
    return v;
}

size_t mr_strided_smem(int M, int xt, int n_out, int smode) {
    size_t b = (size_t)2 * M * xt * sizeof(float2);
    if (smode == MR_SM_COILSUM) b += (size_t)n_out * xt * sizeof(float2);
    return b;
}

int mr_pick_xt(int M, int n_out, int smode, int nfast, size_t limit) {
    int xt = 32;
    while (xt > 1 && mr_strided_smem(M, xt, n_out, smode) > limit) xt >>= 1;
    while (xt > 1 && (xt >> 1) >= nfast) xt >>= 1;
    return xt;
}

size_t mr_xbd_smem(int M, int L, int nc) { return (size_t)2 * nc * L * (M + 1) * sizeof(float2); }
size_t mr_xplain_smem(int M, int rows) { return (size_t)2 * rows * (M + 1) * sizeof(float2); }

// ---------------------------------------------------------------------------
// Strided-axis pass
// ---------------------------------------------------------------------------

template <int DIR, int LM, int SM>
__global__ void __launch_bounds__(256) k_strided(const mr_strided_args a) {
    extern __shared__ float2 sm[];
    const int M = a.ax.M;
    const int xt = a.xt;
    float2 *A = sm;
    float2 *B = sm + (size_t)M * xt;
    float2 *acc = sm + (size_t)2 * M * xt;

    int64_t bid = blockIdx.x;
    const int xtile = (int)(bid % a.nxt);
    bid /= a.nxt;
    const int outer = (int)(bid % a.nouter);
    const int plane = (int)(bid / a.nouter);
    const int x0 = xtile * xt;
    const int nx = min(xt, a.nfast - x0);
    const int ncl = (SM == MR_SM_COILSUM) ? a.ncoil : 1;

    for (int cc = 0; cc < ncl; ++cc) {
        // plane of the source: BUF: `plane` (or coil cc's plane of rank l in
        // COILSUM mode); XS: plane p = c * L + l of the group.
        const int sp = (SM == MR_SM_COILSUM) ? cc * a.L + plane : plane;
        // ---- load (zero-pad / shift map) ----
        for (int idx = threadIdx.x; idx < M * xt; idx += blockDim.x) {
            const int j = idx / xt;
            const int xx = idx - j * xt;
            int src_a = j + a.shift_in;
            if (src_a >= M) src_a -= M;
            float2 v = make_float2(0.f, 0.f);
            if (xx < nx && src_a < a.n_in) {
                const int64_t off = (int64_t)outer * a.s_outer + (int64_t)src_a * a.s_axis + x0 + xx;
                if constexpr (LM == MR_LM_BUF) {
                    v = a.src[(int64_t)sp * a.s_plane + off];
                } else {
                    const int l = sp % a.L;
                    const int c = a.coil0 + sp / a.L;
                    v = c_mul(__ldg(a.xs_s + (int64_t)c * a.img_plane + off),
                              __ldg(a.xs_x + (int64_t)l * a.img_plane + off));
                }
            }
            A[idx] = v;
        }
        __syncthreads();
        float2 *R = fft_lines<DIR>(A, B, a.ax, xt, xt, 1, true);
        // ---- store (crop / shift map) ----
        for (int idx = threadIdx.x; idx < a.n_out * xt; idx += blockDim.x) {
            const int da = idx / xt;
            const int xx = idx - da * xt;
            int q = da - a.shift_out;
            if (q < 0) q += M;
            float2 v = R[q * xt + xx];
            if constexpr (SM == MR_SM_BUF) {
                if (xx < nx)
                    a.dst[(int64_t)plane * a.d_plane + (int64_t)outer * a.d_outer +
                          (int64_t)da * a.d_axis + x0 + xx] = c_scale(v, a.scale);
            } else {
                float2 w = make_float2(0.f, 0.f);
                if (xx < nx) {
                    const int64_t off = (int64_t)outer * a.d_outer + (int64_t)da * a.d_axis + x0 + xx;
                    const float2 s = __ldg(a.xs_s + (int64_t)(a.coil0 + cc) * a.img_plane + off);
                    w = c_mulc(s, v);
                }
                acc[idx] = (cc == 0) ? w : c_add(acc[idx], w);
            }
        }
        __syncthreads();
    }
    if constexpr (SM == MR_SM_COILSUM) {
        for (int idx = threadIdx.x; idx < a.n_out * xt; idx += blockDim.x) {
            const int da = idx / xt;
            const int xx = idx - da * xt;
            if (xx < nx) {
                float2 *o = a.dst + (int64_t)plane * a.d_plane + (int64_t)outer * a.d_outer +
                            (int64_t)da * a.d_axis + x0 + xx;
                float2 v = c_scale(acc[idx], a.scale);
                *o = a.accumulate ? c_add(*o, v) : v;
            }
        }
    }
}

template <int DIR, int LM, int SM>
static int launch_strided_t(const mr_strided_args &a, cudaStream_t s) {
    const size_t smem = mr_strided_smem(a.ax.M, a.xt, a.n_out, SM);
    static unsigned long long attr_set = 0;
    const int dev = mr_current_device();
    if (!(attr_set & (1ull << dev))) {
        cudaFuncSetAttribute(k_strided<DIR, LM, SM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, mr_smem_limit());
        attr_set |= 1ull << dev;
    }
    const int64_t nblk = (int64_t)a.nxt * a.nouter * a.nplane;
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
    k_strided<DIR, LM, SM><<<(unsigned)nblk, 256, smem, s>>>(a);
    MR_LAUNCH_CHECK("k_strided");
    return MR_SUCCESS;
}

int mr_launch_strided(int dir, int lmode, int smode, const mr_strided_args &a,
                      cudaStream_t s) {
    if (dir < 0) {
        if (lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_strided_t<-1, 0, 0>(a, s);
        if (lmode == MR_LM_XS && smode == MR_SM_BUF) return launch_strided_t<-1, 1, 0>(a, s);
        if (lmode == MR_LM_BUF && smode == MR_SM_COILSUM) return launch_strided_t<-1, 0, 1>(a, s);
    } else {
        if (lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_strided_t<1, 0, 0>(a, s);
        if (lmode == MR_LM_BUF && smode == MR_SM_COILSUM) return launch_strided_t<1, 0, 1>(a, s);
        if (lmode == MR_LM_XS && smode == MR_SM_BUF) return launch_strided_t<1, 1, 0>(a, s);
    }
    MR_FAIL(MR_ERR_INTERNAL, "unsupported strided pass mode");
}

// ---------------------------------------------------------------------------
// Contiguous-axis pass, plain (rows)
// ---------------------------------------------------------------------------

template <int DIR>
__global__ void __launch_bounds__(256) k_xplain(const mr_x_args a) {
    extern __shared__ float2 sm[];
    const int M = a.ax.M;
    const int ls = M + 1;
    const int rows = a.rows_cta;
    float2 *A = sm;
    float2 *B = sm + (size_t)rows * ls;
    const int64_t r0 = (int64_t)blockIdx.x * rows;
    const int nr = (int)min((int64_t)rows, a.nrows - r0);
    for (int idx = threadIdx.x; idx < rows * M; idx += blockDim.x) {
        const int b = idx / M;
        const int j = idx - b * M;
        int sa = j + a.shift_in;
        if (sa >= M) sa -= M;
        float2 v = make_float2(0.f, 0.f);
        if (b < nr && sa < a.n_in) v = a.src[(r0 + b) * a.s_row + sa];
        A[b * ls + j] = v;
    }
    __syncthreads();
    float2 *R = fft_lines<DIR>(A, B, a.ax, rows, 1, ls, false);
    for (int idx = threadIdx.x; idx < rows * a.n_out; idx += blockDim.x) {
        const int b = idx / a.n_out;
        const int da = idx - b * a.n_out;
        int q = da - a.shift_out;
        if (q < 0) q += M;
        if (b < nr) a.dst[(r0 + b) * a.d_row + da] = c_scale(R[b * ls + q], a.scale);
    }
}

int mr_launch_xplain(int dir, const mr_x_args &a, cudaStream_t s) {
    const size_t smem = mr_xplain_smem(a.ax.M, a.rows_cta);
    const int64_t nblk = mr_cdiv(a.nrows, a.rows_cta);
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "row pass grid too large");
    static unsigned long long set_f = 0, set_i = 0;
    const int dev = mr_current_device();
    if (dir < 0) {
        if (!(set_f & (1ull << dev))) {
            cudaFuncSetAttribute(k_xplain<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 mr_smem_limit());
            set_f |= 1ull << dev;
        }
        k_xplain<-1><<<(unsigned)nblk, 256, smem, s>>>(a);
    } else {
        if (!(set_i & (1ull << dev))) {
            cudaFuncSetAttribute(k_xplain<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 mr_smem_limit());
            set_i |= 1ull << dev;
        }
        k_xplain<1><<<(unsigned)nblk, 256, smem, s>>>(a);
    }
    MR_LAUNCH_CHECK("k_xplain");
    return MR_SUCCESS;
}

// ---------------------------------------------------------------------------
// Contiguous-axis pass with the block-diagonal multiply
// ---------------------------------------------------------------------------

// Block multiply of one frequency jx for the nc coils of the CTA, compile-
// time rank. v is read from buffer R, y written to buffer O (line stride ls).
template <int L, int NC, int KF>
__device__ __forceinline__ void xbd_apply(const mr_x_args &a, const float2 *R, float2 *O,
                                          int ls, int ncoils, int jy, int jz, int ky, int kz) {
    const int M = a.ax.M;
    for (int jx = threadIdx.x; jx < M; jx += blockDim.x) {
        float2 v[NC][L], y[NC][L];
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
            for (int l = 0; l < L; ++l)
                v[k][l] = (k < ncoils) ? R[(k * L + l) * ls + jx] : make_float2(0.f, 0.f);
        int64_t row;
        bool zero = false;
        if (a.K.inv) {
            const int64_t nat = jx + (int64_t)M * (jy + (int64_t)a.My * jz);
            const int r = __ldg(a.K.inv + nat);
            zero = r < 0;
            row = zero ? 0 : r;
        } else {
            const int kx = mr_nat2cent_d(jx, M, a.cmx);
            row = kx + (int64_t)M * (ky + (int64_t)a.My * kz);
        }
        if (zero) {
#pragma unroll
            for (int k = 0; k < NC; ++k)
#pragma unroll
                for (int l = 0; l < L; ++l) y[k][l] = make_float2(0.f, 0.f);
        } else {
            const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
            bd_block<L, NC, KF>(v, y, kl, a.upper);
        }
#pragma unroll
        for (int k = 0; k < NC; ++k)
            if (k < ncoils)
#pragma unroll
                for (int l = 0; l < L; ++l) O[(k * L + l) * ls + jx] = y[k][l];
    }
}

// Runtime-rank block multiply (any L), one output component per thread.
template <int KF>
__device__ __forceinline__ void xbd_apply_generic(const mr_x_args &a, const float2 *R, float2 *O,
                                                  int ls, int ncoils, int jy, int jz, int ky,
                                                  int kz) {
    const int M = a.ax.M;
    const int L = a.L;
    const int total = ncoils * L * M;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int jx = w % M;
        const int rest = w / M;
        const int c = rest % L;
        const int k = rest / L;
        int64_t row;
        bool zero = false;
        if (a.K.inv) {
            const int64_t nat = jx + (int64_t)M * (jy + (int64_t)a.My * jz);
            const int r = __ldg(a.K.inv + nat);
            zero = r < 0;
            row = zero ? 0 : r;
        } else {
            const int kx = mr_nat2cent_d(jx, M, a.cmx);
            row = kx + (int64_t)M * (ky + (int64_t)a.My * kz);
        }
        float2 y = make_float2(0.f, 0.f);
        if (!zero) {
            const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
            y = bd_one<KF>(R + (int64_t)k * L * ls + jx, ls, L, c, kl, a.upper);
        }
        O[(k * L + c) * ls + jx] = y;
    }
}

// L == 0 selects the runtime-rank variant.
template <int L, int NC, int KF>
__global__ void __launch_bounds__(512) k_xbd(const mr_x_args a) {
    extern __shared__ float2 sm[];
    const int M = a.ax.M;
    const int ls = M + 1;
    const int Lr = (L > 0) ? L : a.L;
    const int chunk = (int)(blockIdx.x % a.nchunk);
    const int loc = (int)(blockIdx.x / a.nchunk);
    const int jy = loc % a.My;
    const int jz = loc / a.My;
    const int c0 = chunk * a.nc;
    const int ncoils = min(a.nc, a.ncoil - c0);
    const int nlines = ncoils * Lr;
    float2 *A = sm;
    float2 *B = sm + (size_t)a.nc * Lr * ls;
    const int64_t pbase = (int64_t)c0 * Lr;
    // load the nlines rows of this location
    for (int idx = threadIdx.x; idx < nlines * M; idx += blockDim.x) {
        const int b = idx / M;
        const int j = idx - b * M;
        int sa = j + a.shift_in;
        if (sa >= M) sa -= M;
        float2 v = make_float2(0.f, 0.f);
        if (sa < a.n_in) v = a.src[((pbase + b) * a.plane_rows + loc) * a.s_row + sa];
        A[b * ls + j] = v;
    }
    __syncthreads();
    float2 *R = fft_lines<-1>(A, B, a.ax, nlines, 1, ls, false);
    float2 *O = (R == A) ? B : A;
    const int ky = mr_nat2cent_d(jy, a.My, a.cmy);
    const int kz = mr_nat2cent_d(jz, a.Mz, a.cmz);
    if constexpr (L > 0) {
        xbd_apply<L, NC, KF>(a, R, O, ls, ncoils, jy, jz, ky, kz);
    } else {
        xbd_apply_generic<KF>(a, R, O, ls, ncoils, jy, jz, ky, kz);
    }
    __syncthreads();
    float2 *Y = fft_lines<1>(O, R, a.ax, nlines, 1, ls, false);
    for (int idx = threadIdx.x; idx < nlines * a.n_out; idx += blockDim.x) {
        const int b = idx / a.n_out;
        const int da = idx - b * a.n_out;
        int q = da - a.shift_out;
        if (q < 0) q += M;
        a.dst[((pbase + b) * a.plane_rows + loc) * a.d_row + da] = c_scale(Y[b * ls + q], a.scale);
    }
}

template <int L, int NC, int KF>
static int launch_xbd_t(const mr_x_args &a, cudaStream_t s) {
    const int Lr = L > 0 ? L : a.L;
    const size_t smem = mr_xbd_smem(a.ax.M, Lr, a.nc);
    static unsigned long long attr_set = 0;
    const int dev = mr_current_device();
    if (!(attr_set & (1ull << dev))) {
        cudaFuncSetAttribute(k_xbd<L, NC, KF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             mr_smem_limit());
        attr_set |= 1ull << dev;
    }
    const int64_t nblk = (int64_t)a.nloc * a.nchunk;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "block-diagonal pass grid too large");
    k_xbd<L, NC, KF><<<(unsigned)nblk, 512, smem, s>>>(a);
    MR_LAUNCH_CHECK("k_xbd");
    return MR_SUCCESS;
}

template <int NC, int KF>
static int dispatch_xbd_L(const mr_x_args &a, cudaStream_t s) {
    switch (a.L) {
#define MR_XBD_CASE(l) \
    case l: return launch_xbd_t<l, NC, KF>(a, s);
        MR_XBD_CASE(1) MR_XBD_CASE(2) MR_XBD_CASE(3) MR_XBD_CASE(4)
        MR_XBD_CASE(5) MR_XBD_CASE(6) MR_XBD_CASE(7) MR_XBD_CASE(8)
        MR_XBD_CASE(9) MR_XBD_CASE(10) MR_XBD_CASE(11) MR_XBD_CASE(12)
        MR_XBD_CASE(13) MR_XBD_CASE(14) MR_XBD_CASE(15) MR_XBD_CASE(16)
#undef MR_XBD_CASE
        default: return launch_xbd_t<0, 1, KF>(a, s);
    }
}

template <int KF>
static int dispatch_xbd_nc(const mr_x_args &a, cudaStream_t s) {
    if (a.L > 16) return launch_xbd_t<0, 1, KF>(a, s);
    if (a.nc >= 2) return dispatch_xbd_L<2, KF>(a, s);
    return dispatch_xbd_L<1, KF>(a, s);
}

int mr_launch_xbd(const mr_x_args &a, cudaStream_t s) {
    switch (a.K.kf) {
        case MR_KF_F32: return dispatch_xbd_nc<MR_KF_F32>(a, s);
        case MR_KF_BF16: return dispatch_xbd_nc<MR_KF_BF16>(a, s);
        case MR_KF_I16: return dispatch_xbd_nc<MR_KF_I16>(a, s);
        default: MR_FAIL(MR_ERR_INTERNAL, "unknown kernel format %d", a.K.kf);
    }
}
