// Second-generation FFT passes: in-place, register-staged Stockham.
//
// Each pass of a line transform reads every butterfly's R inputs from shared
// memory into registers, synchronises, then computes and writes the outputs
// over the same buffer (the Stockham index map only moves data within a
// line, and all reads of the pass complete before any write). This halves
// the shared memory of the ping-pong formulation in passes.cu, so tiles are
// twice as large: 32 consecutive x positions per strided tile (coalesced
// 256-byte rows) and two coils per block-diagonal tile. Consecutive threads
// take consecutive lines (conflict-free shared-memory banks for both the
// x-major strided tiles and the odd line stride of row tiles), and every
// division by a run-time divisor is a multiply-shift (mr_fdiv). Lengths whose
// factors are all in {2, 3, 4, 5, 7, 8} use these kernels; other lengths keep
// the passes.cu kernels.
#include "engine.h"

#include <algorithm>

namespace {

template <int R, int DIR, int NB, int UA>
__device__ __forceinline__ void ip_pass(float2 (&u)[UA], float2 *buf, const int M, const int p,
                                        const mr_fdiv fp, const float2 *__restrict__ tw,
                                        const int nlines, const mr_fdiv fl, const int es,
                                        const int ls) {
    static_assert(NB * R <= UA, "register stage too small");
    const int mr = M / R;
    const int total = nlines * mr;
    const int tstep = M / (p * R);
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = threadIdx.x + k * blockDim.x;
        if (w < total) {
            const int i = mr_div(w, fl);
            const int b = w - i * nlines;
            const float2 *s = buf + b * ls + i * es;
#pragma unroll
            for (int t = 0; t < R; ++t) u[k * R + t] = s[t * mr * es];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = threadIdx.x + k * blockDim.x;
        if (w < total) {
            const int i = mr_div(w, fl);
            const int b = w - i * nlines;
            const int q = mr_div(i, fp);
            const int kk = i - q * p;
            if (p > 1) {
                const int e1 = kk * tstep;
#pragma unroll
                for (int t = 1; t < R; ++t) u[k * R + t] = c_mul(u[k * R + t], tw_get<DIR>(tw, t * e1));
            }
            dft_small<R, DIR>(&u[k * R]);
            float2 *d = buf + b * ls + (q * p * R + kk) * es;
#pragma unroll
            for (int t = 0; t < R; ++t) d[t * p * es] = u[k * R + t];
        }
    }
    __syncthreads();
}

// Full in-place transform of nlines lines (element e of line b at
// buf[b * ls + e * es]); requires nlines * M <= EPT * blockDim.x. One register
// array serves every radix: separate per-case arrays made the register
// allocator spill heavily.
template <int DIR, int EPT>
__device__ __forceinline__ void fft2_lines(float2 *buf, const mr_fft_axis &ax, const int nlines,
                                        const mr_fdiv fl, const int es, const int ls) {
    constexpr int UA = EPT + 7;
    float2 u[UA];
    for (int s = 0; s < ax.npass; ++s) {
        const int p = ax.p[s];
        switch (ax.radix[s]) {
            case 2: ip_pass<2, DIR, (EPT + 1) / 2>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
            case 3: ip_pass<3, DIR, (EPT + 2) / 3>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
            case 4: ip_pass<4, DIR, (EPT + 3) / 4>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
            case 5: ip_pass<5, DIR, (EPT + 4) / 5>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
            case 7: ip_pass<7, DIR, (EPT + 6) / 7>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
            default: ip_pass<8, DIR, (EPT + 7) / 8>(u, buf, ax.M, p, ax.fp[s], ax.tw, nlines, fl, es, ls); break;
        }
    }
}

constexpr int kThreads = 512;
constexpr int kEpt = 40;

// Strided-axis pass: tile [M][xt] in shared memory (x fastest), xt = 2^xts.
// Blocks are ordered plane-fastest so that the 12 coils x 16 ranks of one
// tile run together and the x / SEs tiles they share stay in L2.
template <int DIR, int LM, int SM>
__global__ void __launch_bounds__(kThreads) k_strided2(const __grid_constant__ mr_strided_args a,
                                                       const int xts,
                                                       const mr_fdiv fl) {
    extern __shared__ float2 sm[];
    const int M = a.ax.M;
    const int xt = 1 << xts;
    const int tile_elems = M * xt;
    float2 *acc = sm + tile_elems;

    int64_t bid = blockIdx.x;
    const int plane = (int)(bid % a.nplane);
    bid /= a.nplane;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile << xts;
    const int nx = min(xt, a.nfast - x0);
    const int ncl = (SM == MR_SM_COILSUM) ? a.ncoil : 1;
    const int64_t off0 = (int64_t)outer * a.s_outer + x0;

    for (int cc = 0; cc < ncl; ++cc) {
        const int sp = (SM == MR_SM_COILSUM) ? cc * a.L + plane : plane;
        const float2 *srcp = nullptr;
        const float2 *xp = nullptr, *sp_s = nullptr;
        if constexpr (LM == MR_LM_BUF) {
            srcp = a.src + (int64_t)sp * a.s_plane + off0;
        } else {
            const int l = sp % a.L;
            const int c = a.coil0 + sp / a.L;
            xp = a.xs_x + (int64_t)l * a.img_plane + off0;
            sp_s = a.xs_s + (int64_t)c * a.img_plane + off0;
        }
        for (int idx = threadIdx.x; idx < tile_elems; idx += kThreads) {
            const int j = idx >> xts;
            const int xx = idx & (xt - 1);
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
        fft2_lines<DIR, kEpt>(sm, a.ax, xt, fl, xt, 1);
        const int64_t doff0 = (int64_t)outer * a.d_outer + x0;
        for (int idx = threadIdx.x; idx < a.n_out * xt; idx += kThreads) {
            const int da = idx >> xts;
            const int xx = idx & (xt - 1);
            int q = da - a.shift_out;
            if (q < 0) q += M;
            const float2 v = sm[(q << xts) + xx];
            if constexpr (SM == MR_SM_BUF) {
                if (xx < nx)
                    a.dst[(int64_t)plane * a.d_plane + doff0 + (int64_t)da * a.d_axis + xx] =
                        c_scale(v, a.scale);
            } else {
                float2 w = make_float2(0.f, 0.f);
                if (xx < nx) {
                    const float2 s = __ldg(a.xs_s + (int64_t)(a.coil0 + cc) * a.img_plane + doff0 +
                                           (int64_t)da * a.d_axis + xx);
                    w = c_mulc(s, v);
                }
                acc[idx] = (cc == 0) ? w : c_add(acc[idx], w);
            }
        }
        __syncthreads();
    }
    if constexpr (SM == MR_SM_COILSUM) {
        const int64_t doff0 = (int64_t)outer * a.d_outer + x0;
        for (int idx = threadIdx.x; idx < a.n_out * xt; idx += kThreads) {
            const int da = idx >> xts;
            const int xx = idx & (xt - 1);
            if (xx < nx) {
                float2 *o = a.dst + (int64_t)plane * a.d_plane + doff0 + (int64_t)da * a.d_axis + xx;
                const float2 v = c_scale(acc[idx], a.scale);
                *o = a.accumulate ? c_add(*o, v) : v;
            }
        }
    }
}

// Contiguous-axis pass with the block multiply: nc coils (power of two) x L
// lines of one (jy, jz) location, line stride ls (odd). In the multiply a
// warp covers 32 / nc consecutive frequencies for all nc coils, so the lanes
// of one frequency load each kernel element in the same instruction.
template <int L, int KF>
__global__ void __launch_bounds__(kThreads) k_xbd2(const __grid_constant__ mr_x_args a,
                                                   const int ls,
                                                   const mr_fdiv fM, const mr_fdiv fnl) {
    extern __shared__ float2 sm[];
    const int M = a.ax.M;
    const int nc = a.nc;
    const int chunk = (int)(blockIdx.x % a.nchunk);
    const int loc = (int)(blockIdx.x / a.nchunk);
    const int jy = loc % a.My;
    const int jz = loc / a.My;
    const int c0 = chunk * nc;
    const int ncoils = min(nc, a.ncoil - c0);
    const int nlines = nc * L;
    const int64_t pbase = (int64_t)c0 * L;
    for (int idx = threadIdx.x; idx < nlines * M; idx += kThreads) {
        const int b = mr_div(idx, fM);
        const int j = idx - b * M;
        int sa = j + a.shift_in;
        if (sa >= M) sa -= M;
        float2 v = make_float2(0.f, 0.f);
        if (b < ncoils * L && sa < a.n_in)
            v = a.src[((pbase + b) * a.plane_rows + loc) * a.s_row + sa];
        sm[b * ls + j] = v;
    }
    __syncthreads();
    fft2_lines<-1, kEpt>(sm, a.ax, nlines, fnl, 1, ls);
    const int ky = mr_nat2cent_d(jy, a.My, a.cmy);
    const int kz = mr_nat2cent_d(jz, a.Mz, a.cmz);
    const int gw = 32 / nc;
    for (int w = threadIdx.x; w < nc * ((M + gw - 1) / gw) * gw; w += kThreads) {
        const int lane = w & 31;
        const int k = lane / gw;
        const int jx = (w >> 5) * gw + (lane - k * gw);
        if (jx >= M || k >= ncoils) continue;
        float2 v[1][L], y[1][L];
#pragma unroll
        for (int l = 0; l < L; ++l) v[0][l] = sm[(k * L + l) * ls + jx];
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
        for (int l = 0; l < L; ++l) sm[(k * L + l) * ls + jx] = y[0][l];
    }
    __syncthreads();
    fft2_lines<1, kEpt>(sm, a.ax, nlines, fnl, 1, ls);
    for (int idx = threadIdx.x; idx < ncoils * L * a.n_out; idx += kThreads) {
        const int b = idx / a.n_out;
        const int da = idx - b * a.n_out;
        int q = da - a.shift_out;
        if (q < 0) q += M;
        a.dst[((pbase + b) * a.plane_rows + loc) * a.d_row + da] = c_scale(sm[b * ls + q], a.scale);
    }
}

template <typename F>
void set_smem_attr(F *f, unsigned long long &mask) {
    const int dev = mr_current_device();
    if (!(mask & (1ull << dev))) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, mr_smem_limit());
        mask |= 1ull << dev;
    }
}

template <int DIR, int LM, int SM>
int launch_strided2_t(const mr_strided_args &a, int xts, cudaStream_t s) {
    static unsigned long long attr = 0;
    set_smem_attr(k_strided2<DIR, LM, SM>, attr);
    const int xt = 1 << xts;
    size_t smem = (size_t)a.ax.M * xt * sizeof(float2);
    if (SM == MR_SM_COILSUM) smem += (size_t)a.n_out * xt * sizeof(float2);
    const int64_t nblk = (int64_t)a.nxt * a.nouter * a.nplane;
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
    k_strided2<DIR, LM, SM><<<(unsigned)nblk, kThreads, smem, s>>>(a, xts, mr_make_fdiv(xt));
    MR_LAUNCH_CHECK("k_strided2");
    return MR_SUCCESS;
}

template <int L, int KF>
int launch_xbd2_t(const mr_x_args &a, cudaStream_t s) {
    static unsigned long long attr = 0;
    set_smem_attr(k_xbd2<L, KF>, attr);
    const int ls = mr_xbd2_stride(a.ax.M);
    const size_t smem = (size_t)a.nc * L * ls * sizeof(float2);
    const int64_t nblk = (int64_t)a.nloc * a.nchunk;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "block-diagonal pass grid too large");
    k_xbd2<L, KF><<<(unsigned)nblk, kThreads, smem, s>>>(a, ls, mr_make_fdiv(a.ax.M),
                                                        mr_make_fdiv(a.nc * L));
    MR_LAUNCH_CHECK("k_xbd2");
    return MR_SUCCESS;
}

template <int KF>
int dispatch_xbd2(const mr_x_args &a, cudaStream_t s) {
    switch (a.L) {
#define MR_X2_CASE(l) \
    case l: return launch_xbd2_t<l, KF>(a, s);
        MR_X2_CASE(1) MR_X2_CASE(2) MR_X2_CASE(3) MR_X2_CASE(4)
        MR_X2_CASE(5) MR_X2_CASE(6) MR_X2_CASE(7) MR_X2_CASE(8)
        MR_X2_CASE(9) MR_X2_CASE(10) MR_X2_CASE(11) MR_X2_CASE(12)
        MR_X2_CASE(13) MR_X2_CASE(14) MR_X2_CASE(15) MR_X2_CASE(16)
#undef MR_X2_CASE
        default: MR_FAIL(MR_ERR_INTERNAL, "k_xbd2 has no instance for L = %d", a.L);
    }
}

}  // namespace

int mr_xbd2_stride(int M) { return (M % 2 == 0) ? M + 1 : M + 2; }

int mr_strided2_xts(int M, int n_out, int smode, int nfast, size_t limit) {
    // largest power-of-two tile with M * xt <= EPT * threads that fits smem
    int xts = 6;
    auto bytes = [&](int s) {
        size_t b = (size_t)M * (1u << s) * sizeof(float2);
        if (smode == MR_SM_COILSUM) b += (size_t)n_out * (1u << s) * sizeof(float2);
        return b;
    };
    while (xts > 0 && ((size_t)M * (1u << xts) > (size_t)kEpt * kThreads || bytes(xts) > limit))
        --xts;
    while (xts > 0 && (1 << (xts - 1)) >= nfast) --xts;
    if ((size_t)M * (1u << xts) > (size_t)kEpt * kThreads || bytes(xts) > limit) return -1;
    return xts;
}

int mr_xbd2_coils(int M, int L, int ncoil, size_t limit) {
    if (L > 16) return 0;
    const int ls = mr_xbd2_stride(M);
    int nc = 8;
    while (nc > 1 && (nc / 2 >= ncoil || (size_t)nc * L * M > (size_t)kEpt * kThreads ||
                      (size_t)nc * L * ls * sizeof(float2) > limit))
        nc >>= 1;
    if ((size_t)nc * L * M > (size_t)kEpt * kThreads || (size_t)nc * L * ls * sizeof(float2) > limit)
        return 0;
    return nc;
}

int mr_launch_strided2(int dir, int lmode, int smode, const mr_strided_args &a, int xts,
                       cudaStream_t s) {
    if (dir < 0) {
        if (lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_strided2_t<-1, 0, 0>(a, xts, s);
        if (lmode == MR_LM_XS && smode == MR_SM_BUF) return launch_strided2_t<-1, 1, 0>(a, xts, s);
    } else {
        if (lmode == MR_LM_BUF && smode == MR_SM_BUF) return launch_strided2_t<1, 0, 0>(a, xts, s);
        if (lmode == MR_LM_BUF && smode == MR_SM_COILSUM) return launch_strided2_t<1, 0, 1>(a, xts, s);
    }
    MR_FAIL(MR_ERR_INTERNAL, "unsupported strided pass mode");
}

int mr_launch_xbd2(const mr_x_args &a, cudaStream_t s) {
    switch (a.K.kf) {
        case MR_KF_F32: return dispatch_xbd2<MR_KF_F32>(a, s);
        case MR_KF_BF16: return dispatch_xbd2<MR_KF_BF16>(a, s);
        case MR_KF_I16: return dispatch_xbd2<MR_KF_I16>(a, s);
        default: MR_FAIL(MR_ERR_INTERNAL, "unknown kernel format %d", a.K.kf);
    }
}
