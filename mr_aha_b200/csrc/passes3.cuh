// Kernel templates of the compile-time-specialised passes (fftfix.cuh) and
// the lists of instantiated configurations. The instantiations are spread
// over several translation units (passes3.cu, p3_*.cu) so that they compile
// in parallel; passes3.cu dispatches to them.
#pragma once

#include "engine.h"
#include "fftfix.cuh"
#include "tma.cuh"

namespace {

// Block sizes: 512 threads for tiles of more than 10240 elements (one CTA per
// SM), 256 threads for smaller tiles, with registers capped so that two
// independent CTAs share an SM (one loads or stores while the other computes).

template <int DIR, int LM, int SM, int M, int XT, int kNT, int MINB>
__global__ void __launch_bounds__(kNT, MINB) k_strided3(const __grid_constant__ mr_strided_args a) {
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
// even half-spectrum in line 2b and its odd one in line 2b + 1. BLK: read
// the complex64 kernel from its blocked copy (a.K.blk; a masked kernel's copy
// is in grid order, zero outside the mask, whose locations are still skipped), where
// the 32 frequencies of a warp are contiguous for every component. TMAIN:
// the CTA's NC L input rows arrive by TMA tensor copies (a.in_map: extents
// {N, plane_rows, planes of the group}, box {N or N / 2, 1, NC L}; planes
// past the group read as zeros) into a staging area at the end of the line
// buffer, instead of per-thread loads; same values, same arithmetic.
template <int N, int L, int NC, int KF, int kNT, bool BLK = false, bool TMAIN = false>
__global__ void __launch_bounds__(kNT, 512 / kNT) k_xbdh(const __grid_constant__ mr_x_args a) {
    extern __shared__ __align__(128) float2 sm[];
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
    if constexpr (BLK) {
        // L2 prefetch of this coil chunk's share of the location's blocked
        // kernel rows, issued before the forward transform: the coil CTAs
        // of a location start together and would otherwise all wait for the
        // first one's DRAM reads in the block multiply (43.7 against 44.4 ms
        // at 320 x 320 x 56, L = 16, 12 coils)
        constexpr int64_t LOCB = KF == MR_KF_F32
                                     ? (int64_t)((N + 15) / 16) * mr_blk_tri(L) * 32 * 8
                                     : (int64_t)((N + 15) / 16) * mr_blk16_tri(L) * 32 * 4;
        const int64_t per = ((LOCB / a.nchunk) + 4095) / 4096 * 4096;
        const int64_t b0 = (int64_t)chunk * per, b1 = min(LOCB, b0 + per);
        const char *kb = reinterpret_cast<const char *>(a.K.blk) + (int64_t)loc * LOCB;
        for (int64_t o = b0 + (int64_t)threadIdx.x * 4096; o < b1; o += (int64_t)kNT * 4096)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(kb + o),
                         "r"((unsigned)min((int64_t)4096, b1 - o))
                         : "memory");
    }
    if constexpr (TMAIN) {
        constexpr int BX = N > 256 ? N / 2 : N;
        constexpr int NBOX = N / BX;
        constexpr int SOFF = ((NL * LS - NR * N) / 16) * 16;  // 128-byte aligned staging
        constexpr int PER = (NR * N + kNT - 1) / kNT;
        static_assert(N % BX == 0 && BX <= 256 && NR <= 256 && SOFF >= 0, "TMA box");
        float2 *stage = sm + SOFF;
        uint64_t *bar = reinterpret_cast<uint64_t *>(sm + NL * LS);
        if (threadIdx.x == 0) {
            mrtma::mbar_init(bar, 1);
            mrtma::fence_mbar_init();
            mrtma::mbar_arrive_expect_tx(bar, NR * N * (unsigned)sizeof(float2));
#pragma unroll
            for (int q = 0; q < NBOX; ++q)
                mrtma::tensor3d_g2s(stage + q * NR * BX, &a.in_map, q * BX, loc, (int)pbase, bar);
        }
        __syncthreads();
        mrtma::mbar_wait(bar, 0, a.status);
        float2 vals[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int idx = threadIdx.x + k * kNT;
            if (idx < NR * N) {
                const int b = idx / N;
                const int n = idx - b * N;
                const int q = n / BX;
                vals[k] = stage[(q * NR + b) * BX + (n - q * BX)];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int idx = threadIdx.x + k * kNT;
            if (idx < NR * N) {
                const int b = idx / N;
                const int n = idx - b * N;
                sm[(2 * b) * LS + n] = vals[k];
                sm[(2 * b + 1) * LS + n] = c_mul(vals[k], __ldg(tw + n));
            }
        }
    } else {
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
    }
    __syncthreads();
    mrfix::fft<-1, N, NL, 1, LS, kNT, 2>(sm, tw);
    const int ky = mr_nat2cent_d(jy, a.My, a.cmy);
    const int kz = mr_nat2cent_d(jz, a.Mz, a.cmz);
    // a warp takes 16 consecutive m of one coil in both parities: lanes 0-15
    // the even k = 2m, lanes 16-31 the odd k = 2m + 1 (each half-warp reads
    // 16 consecutive words of one line)
    constexpr int MB = (N + 15) / 16;
    if constexpr (L > 16) {
        // rank 32: two threads per (k, coil), in paired warps (2j: outputs
        // 0-15, 2j + 1: outputs 16-31); both read v before either writes y
        static_assert(L == 32 && (kNT / 32) % 2 == 0, "split block multiply is for rank 32");
        constexpr int ITEMS2 = NC * MB * 2 * 32;
        constexpr int NIT = (ITEMS2 + kNT - 1) / kNT;
        for (int it = 0; it < NIT; ++it) {
            const int w = threadIdx.x + it * kNT;
            const int lane = w & 31;
            const int h = (w >> 5) & 1;
            const int wi = w >> 6;
            const int k = wi / MB;
            const int m = (wi - k * MB) * 16 + (lane & 15);
            const int par = lane >> 4;
            const bool ok = w < ITEMS2 && m < N && k < ncoils;
            float2 *line = sm + (2 * k * L + par) * LS + m;
            float2 y[16];
            if (ok) {
                const int jx = 2 * m + par;
                bool zero = false;
                int64_t row;
                if (a.K.inv) {
                    const int r =
                        __ldg(a.K.inv + jx + (int64_t)(2 * N) * (jy + (int64_t)a.My * jz));
                    zero = r < 0;
                    row = zero ? 0 : r;
                } else {
                    row = mr_nat2cent_d(jx, 2 * N, a.cmx) +
                          (int64_t)(2 * N) * (ky + (int64_t)a.My * kz);
                }
                if (zero) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) y[i] = make_float2(0.f, 0.f);
                } else if constexpr (BLK) {
                    static_assert(KF == MR_KF_F32, "16-bit blocked copies are for rank <= 16");
                    const mr_kload_blk<false> kl{
                        a.K.blk + (((int64_t)jz * a.My + jy) * MB + (wi - k * MB)) *
                                      (mr_blk_tri(L) * 32) +
                            (2 * (lane & 15) + par),
                        1.f};
                    if (a.upper) {
                        if (h) bd_half32<1, true, KF>(line, 2 * LS, kl, y);
                        else bd_half32<0, true, KF>(line, 2 * LS, kl, y);
                    } else {
                        if (h) bd_half32<1, false, KF>(line, 2 * LS, kl, y);
                        else bd_half32<0, false, KF>(line, 2 * LS, kl, y);
                    }
                } else {
                    const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
                    if (a.upper) {
                        if (h) bd_half32<1, true, KF>(line, 2 * LS, kl, y);
                        else bd_half32<0, true, KF>(line, 2 * LS, kl, y);
                    } else {
                        if (h) bd_half32<1, false, KF>(line, 2 * LS, kl, y);
                        else bd_half32<0, false, KF>(line, 2 * LS, kl, y);
                    }
                }
            }
            __syncthreads();
            if (ok) {
#pragma unroll
                for (int i = 0; i < 16; ++i) line[2 * (16 * h + i) * LS] = y[i];
            }
        }
    } else {
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
        } else if constexpr (BLK) {
            const int64_t blk = ((int64_t)jz * a.My + jy) * MB + (wi - k * MB);
            const int f = 2 * (lane & 15) + par;
            if constexpr (KF == MR_KF_F32) {
                // rank <= 16: paired components, two per 16-byte load
                const mr_kload_blk<true> kl{a.K.blk + blk * (mr_blk_tri(L) * 32) + 2 * f, 1.f};
                bd_block<L, 1, KF>(v, y, kl, a.upper);
            } else {
                // four 16-bit codes per 16-byte load, the location's scale
                const mr_kload_blk16<KF> kl{
                    reinterpret_cast<const uint4 *>(a.K.blk) + blk * (mr_blk16_tri(L) / 4 * 32) + f,
                    __ldg(a.K.sblk + blk * 32 + f)};
                bd_block<L, 1, KF>(v, y, kl, a.upper);
            }
        } else {
            const mr_kload<KF> kl = mr_kload_at<KF>(a.K, row);
            bd_block<L, 1, KF>(v, y, kl, a.upper);
        }
#pragma unroll
        for (int l = 0; l < L; ++l) line[2 * l * LS] = y[0][l];
    }
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

// Asynchronous 16-byte copies global -> shared (zero-filled past `bytes`).
__device__ __forceinline__ void mr_cp_async16(void *sdst, const void *gsrc, unsigned bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mr_cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void mr_cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// `rows` rows of a tile of XT columns (row r at src + r * stride, nx valid
// columns) into dst[r * XT + c], as 16-byte copies; columns past nx read 0.
// src, stride and the tile start must be 16-byte aligned (even elements).
template <int XT, int kNT>
__device__ __forceinline__ void mr_cp_tile(float2 *dst, const float2 *src, int64_t stride,
                                           int rows, int nx) {
    constexpr int CPR = XT / 2;
    for (int c = threadIdx.x; c < rows * CPR; c += kNT) {
        const int r = c / CPR;
        const int e0 = 2 * (c - r * CPR);
        const int valid = nx - e0;
        const unsigned bytes = valid >= 2 ? 16u : (valid == 1 ? 8u : 0u);
        const float2 *g = bytes ? src + (int64_t)r * stride + e0 : src;
        mr_cp_async16(dst + r * XT + e0, g, bytes);
    }
}

// Strided passes of length M = 2N whose input (forward) or output (inverse)
// is the N image rows, without the zero half: the forward pass computes the
// ramp-free spectrum X'[k] = sum_n x[n] W_M^{kn} as X'[2m] = FFT_N(x)[m],
// X'[2m+1] = FFT_N(x t)[m] (t[n] = W_M^n), and the inverse pass
// y[n] = IFFT_N(Z'_even)[n] + conj(t[n]) IFFT_N(Z'_odd)[n]. Against the
// padded transforms with pad / crop offset s, X' = W_M^{ks} X and the inverse
// drops the conjugate ramp, so a forward and an inverse of this kind used
// together give the same operator (everything between them is diagonal in
// k). Column b of the tile keeps its even line at b and its odd line at
// XT + b (x-major layout, element e of line bl at e * 2XT + bl).
template <int N, int XT, int kNT, int MINB>
__global__ void __launch_bounds__(kNT, MINB) k_strided_hf(const __grid_constant__ mr_strided_args a) {
    extern __shared__ float2 sm[];
    constexpr int NL = 2 * XT;
    int64_t bid = blockIdx.x;
    const int plane = (int)(bid % a.nplane);
    bid /= a.nplane;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const float2 *srcp = a.src + (int64_t)plane * a.s_plane + (int64_t)outer * a.s_outer + x0;
    float2 *dstp = a.dst + (int64_t)plane * a.d_plane + (int64_t)outer * a.d_outer + x0;
    const float2 *tw = a.ax.tw;  // W_M^e
    // each row element is read once and feeds both lines (a plain loop keeps
    // many loads in flight)
#pragma unroll 4
    for (int idx = threadIdx.x; idx < N * XT; idx += kNT) {
        const int e = idx / XT;
        const int b = idx - e * XT;
        float2 v = make_float2(0.f, 0.f);
        if (b < nx) v = srcp[(int64_t)e * a.s_axis + b];
        sm[e * NL + b] = v;
        sm[e * NL + XT + b] = c_mul(v, __ldg(tw + e));
    }
    __syncthreads();
    auto store = [&](int bl, int q, float2 v) {
        const int b = bl % XT;
        const int k = 2 * q + (bl >= XT ? 1 : 0);
        if (b < nx) dstp[(int64_t)k * a.d_axis + b] = c_scale(v, a.scale);
    };
    mrfix::fft_io<false, true, -1, N, NL, NL, 1, kNT, 2>(sm, tw, [](int, int) {
        return make_float2(0.f, 0.f); }, store);
}

template <int N, int XT, int kNT, int MINB>
__global__ void __launch_bounds__(kNT, MINB) k_strided_hi(const __grid_constant__ mr_strided_args a) {
    extern __shared__ float2 sm[];
    constexpr int NL = 2 * XT;
    int64_t bid = blockIdx.x;
    const int plane = (int)(bid % a.nplane);
    bid /= a.nplane;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const float2 *srcp = a.src + (int64_t)plane * a.s_plane + (int64_t)outer * a.s_outer + x0;
    float2 *dstp = a.dst + (int64_t)plane * a.d_plane + (int64_t)outer * a.d_outer + x0;
    const float2 *tw = a.ax.tw;
    auto load = [&](int bl, int e) -> float2 {
        const int b = bl % XT;
        const int k = 2 * e + (bl >= XT ? 1 : 0);
        return b < nx ? srcp[(int64_t)k * a.s_axis + b] : make_float2(0.f, 0.f);
    };
    mrfix::fft_io<true, false, 1, N, NL, NL, 1, kNT, 2>(sm, tw, load, mrfix::no_store());
#pragma unroll 4
    for (int idx = threadIdx.x; idx < N * XT; idx += kNT) {
        const int n = idx / XT;
        const int b = idx - n * XT;
        if (b < nx) {
            const float2 e = sm[n * NL + b];
            const float2 o = sm[n * NL + XT + b];
            dstp[(int64_t)n * a.d_axis + b] = c_scale(c_add(e, c_mulc(__ldg(tw + n), o)), a.scale);
        }
    }
}

// The half-length forward y pass pipelined over planes: a CTA takes PG
// planes of one (x tile, z) position; the next plane's rows are copied
// (cp.async) into the other stage while the current plane is transformed.
// The first FFT pass reads the stage (the odd line times t[n]), the last one
// writes the spectrum rows. Same arithmetic as k_strided_hf.
// TMA: each plane's [N][XT] tile arrives as tensor copies of boxes of at
// most 256 rows (a.map0: {fast, y, outer, plane}; columns past the plane read
// as zeros) completing on the stage's mbarrier, instead of per-thread cp.async.
template <int N, int XT, int kNT, int MINB, int PG, bool TMA = false>
__global__ void __launch_bounds__(kNT, MINB) k_hf_pipe(const __grid_constant__ mr_strided_args a) {
    extern __shared__ __align__(128) float2 sm[];
    constexpr int NL = 2 * XT;
    constexpr int STG = N * XT;
    float2 *stg = sm;               // [2][N][XT]
    float2 *buf = sm + 2 * STG;     // [N][2 XT]
    const int ngrp = (a.nplane + PG - 1) / PG;
    int64_t bid = blockIdx.x;
    const int grp = (int)(bid % ngrp);
    bid /= ngrp;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const int p0 = grp * PG;
    const int np = min(PG, a.nplane - p0);
    const int64_t soff = (int64_t)outer * a.s_outer + x0;
    const int64_t doff = (int64_t)outer * a.d_outer + x0;
    const float2 *tw = a.ax.tw;
    constexpr int BY = N > 256 ? N / 2 : N;  // rows per tensor box
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * STG + N * NL);
    auto issue = [&](int pl, int st) {
        if constexpr (TMA) {
            if (threadIdx.x == 0) {
                mrtma::fence_proxy_async_smem();
                mrtma::mbar_arrive_expect_tx(bar + st, N * XT * (unsigned)sizeof(float2));
#pragma unroll
                for (int q = 0; q < N / BY; ++q)
                    mrtma::tensor4d_g2s(stg + st * STG + q * BY * XT, &a.map0, x0, q * BY, outer,
                                        pl, bar + st);
            }
        } else {
            mr_cp_tile<XT, kNT>(stg + st * STG, a.src + (int64_t)pl * a.s_plane + soff, a.s_axis,
                                N, nx);
            mr_cp_async_commit();
        }
    };
    if constexpr (TMA) {
        static_assert(N % BY == 0 && BY <= 256 && XT <= 256, "TMA box");
        if (threadIdx.x == 0) {
            mrtma::mbar_init(bar, 1);
            mrtma::mbar_init(bar + 1, 1);
            mrtma::fence_mbar_init();
        }
        __syncthreads();
    }
    issue(p0, 0);
    for (int i = 0; i < np; ++i) {
        const int st = i & 1;
        if (i + 1 < np) issue(p0 + i + 1, st ^ 1);
        if constexpr (TMA) {
            mrtma::mbar_wait(bar + st, (unsigned)(i >> 1) & 1u, a.status);
        } else {
            if (i + 1 < np) mr_cp_async_wait<1>();
            else mr_cp_async_wait<0>();
        }
        __syncthreads();
        const float2 *sv = stg + st * STG;
        float2 *dstp = a.dst + (int64_t)(p0 + i) * a.d_plane + doff;
        auto load = [&](int bl, int e) -> float2 {
            const int b = bl % XT;
            const float2 v = sv[e * XT + b];
            return bl >= XT ? c_mul(v, __ldg(tw + e)) : v;
        };
        auto store = [&](int bl, int q, float2 v) {
            const int b = bl % XT;
            const int k = 2 * q + (bl >= XT ? 1 : 0);
            if (b < nx) dstp[(int64_t)k * a.d_axis + b] = c_scale(v, a.scale);
        };
        mrfix::fft_io<true, true, -1, N, NL, NL, 1, kNT, 2>(buf, tw, load, store);
        __syncthreads();
    }
}

// The half-length inverse y pass pipelined over planes (as k_hf_pipe): the
// next plane's 2N spectrum rows are copied into the other stage while the
// current plane is transformed; the first FFT pass reads the stage (row
// 2e + p for element e of line parity p), the combine loop writes the N
// image rows. Same arithmetic as k_strided_hi.
template <int N, int XT, int kNT, int MINB, int PG>
__global__ void __launch_bounds__(kNT, MINB) k_hi_pipe(const __grid_constant__ mr_strided_args a) {
    extern __shared__ float2 sm[];
    constexpr int NL = 2 * XT;
    constexpr int STG = 2 * N * XT;
    float2 *stg = sm;               // [2][2N][XT]
    float2 *buf = sm + 2 * STG;     // [N][2 XT]
    const int ngrp = (a.nplane + PG - 1) / PG;
    int64_t bid = blockIdx.x;
    const int grp = (int)(bid % ngrp);
    bid /= ngrp;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const int p0 = grp * PG;
    const int np = min(PG, a.nplane - p0);
    const int64_t soff = (int64_t)outer * a.s_outer + x0;
    const int64_t doff = (int64_t)outer * a.d_outer + x0;
    const float2 *tw = a.ax.tw;
    mr_cp_tile<XT, kNT>(stg, a.src + (int64_t)p0 * a.s_plane + soff, a.s_axis, 2 * N, nx);
    mr_cp_async_commit();
    for (int i = 0; i < np; ++i) {
        const int st = i & 1;
        if (i + 1 < np) {
            mr_cp_tile<XT, kNT>(stg + (st ^ 1) * STG, a.src + (int64_t)(p0 + i + 1) * a.s_plane + soff,
                                a.s_axis, 2 * N, nx);
            mr_cp_async_commit();
            mr_cp_async_wait<1>();
        } else {
            mr_cp_async_wait<0>();
        }
        __syncthreads();
        const float2 *sv = stg + st * STG;
        auto load = [&](int bl, int e) -> float2 {
            const int b = bl % XT;
            return sv[(2 * e + (bl >= XT ? 1 : 0)) * XT + b];
        };
        mrfix::fft_io<true, false, 1, N, NL, NL, 1, kNT, 2>(buf, tw, load, mrfix::no_store());
        float2 *dstp = a.dst + (int64_t)(p0 + i) * a.d_plane + doff;
        for (int idx = threadIdx.x; idx < N * XT; idx += kNT) {
            const int n = idx / XT;
            const int b = idx - n * XT;
            if (b < nx) {
                const float2 e = buf[n * NL + b];
                const float2 o = buf[n * NL + XT + b];
                dstp[(int64_t)n * a.d_axis + b] =
                    c_scale(c_add(e, c_mulc(__ldg(tw + n), o)), a.scale);
            }
        }
        __syncthreads();
    }
}

template <int DIR, int N, int XT>
int launch_sh(const mr_strided_args &a, cudaStream_t s) {
    constexpr int T = 2 * N * XT;
    constexpr int kNT = (T > 10240) ? 512 : 256;
    constexpr int MINB = (T > 10240) ? 1 : (T <= 2048 ? 4 : (T <= 5120 ? 3 : 2));
    static unsigned long long attr = 0;
    const size_t smem = (size_t)T * sizeof(float2);
    const int64_t nblk = (int64_t)a.nxt * a.nouter * a.nplane;
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
    if constexpr (DIR < 0 && XT % 2 == 0 && 4 * N * XT * 8 <= 112 * 1024) {
        constexpr int PG = 8;
        if (mr_env_int("MR_AHA_B200_NO_PIPE", 0) == 0 && (((uintptr_t)a.src) & 15) == 0 &&
            ((a.s_plane | a.s_axis | a.s_outer) & 1) == 0) {
            const int64_t nb = (int64_t)a.nxt * a.nouter * ((a.nplane + PG - 1) / PG);
            if (mr_env_int("MR_AHA_B200_NO_TMA", 0) == 0 && N / (N > 256 ? 2 : 1) <= 256) {
                // planes {x, y, z (outer), plane}
                mr_strided_args b = a;
                const uint64_t dim[4] = {(uint64_t)a.nfast, (uint64_t)N, (uint64_t)a.nouter,
                                         (uint64_t)a.nplane};
                const uint64_t str[3] = {(uint64_t)a.s_axis * sizeof(float2),
                                         (uint64_t)a.s_outer * sizeof(float2),
                                         (uint64_t)a.s_plane * sizeof(float2)};
                const uint32_t box[4] = {(uint32_t)XT, (uint32_t)(N > 256 ? N / 2 : N), 1u, 1u};
                const int rc = mr_tma_encode(&b.map0, a.src, 4, dim, str, box);
                if (rc != MR_SUCCESS) return rc;
                static unsigned long long attr_t = 0;
                set_attr(k_hf_pipe<N, XT, kNT, 2, PG, true>, attr_t);
                k_hf_pipe<N, XT, kNT, 2, PG, true>
                    <<<(unsigned)nb, kNT, (size_t)4 * N * XT * sizeof(float2) + 16, s>>>(b);
                MR_LAUNCH_CHECK_T("k_hf_pipe", "k_hf_pipe<N=%d,XT=%d,tma>", N, XT);
                return MR_SUCCESS;
            }
            static unsigned long long attr_p = 0;
            set_attr(k_hf_pipe<N, XT, kNT, 2, PG>, attr_p);
            k_hf_pipe<N, XT, kNT, 2, PG><<<(unsigned)nb, kNT, (size_t)4 * N * XT * sizeof(float2),
                                           s>>>(a);
            MR_LAUNCH_CHECK_T("k_hf_pipe", "k_hf_pipe<N=%d,XT=%d>", N, XT);
            return MR_SUCCESS;
        }
    }
    if constexpr (DIR > 0 && XT % 2 == 0 && 6 * N * XT * 8 <= 64 * 1024) {
        constexpr int PG = 8;
        if (mr_env_int("MR_AHA_B200_NO_PIPE", 0) == 0 && (((uintptr_t)a.src) & 15) == 0 &&
            ((a.s_plane | a.s_axis | a.s_outer) & 1) == 0) {
            static unsigned long long attr_p = 0;
            set_attr(k_hi_pipe<N, XT, kNT, 3, PG>, attr_p);
            const int64_t nb = (int64_t)a.nxt * a.nouter * ((a.nplane + PG - 1) / PG);
            k_hi_pipe<N, XT, kNT, 3, PG><<<(unsigned)nb, kNT, (size_t)6 * N * XT * sizeof(float2),
                                           s>>>(a);
            MR_LAUNCH_CHECK_T("k_hi_pipe", "k_hi_pipe<N=%d,XT=%d>", N, XT);
            return MR_SUCCESS;
        }
    }
    if constexpr (DIR < 0) {
        set_attr(k_strided_hf<N, XT, kNT, MINB>, attr);
        k_strided_hf<N, XT, kNT, MINB><<<(unsigned)nblk, kNT, smem, s>>>(a);
    } else {
        set_attr(k_strided_hi<N, XT, kNT, MINB>, attr);
        k_strided_hi<N, XT, kNT, MINB><<<(unsigned)nblk, kNT, smem, s>>>(a);
    }
    MR_LAUNCH_CHECK_T("k_strided_h", "%s<N=%d,XT=%d>", DIR < 0 ? "k_strided_hf" : "k_strided_hi",
                      N, XT);
    return MR_SUCCESS;
}

// Inverse strided pass with the conj(S_c) coil sum (the last pass of 3-D /
// stack plans), pipelined over the coils: while coil c is transformed, the
// next coil's input tile and coil-map tile are already being copied into the
// other half of a double buffer (cp.async), so the loads overlap the FFT
// instead of stalling it. Same arithmetic and order as k_strided3<1, BUF,
// COILSUM>. Shared memory: input and map tiles x 2 stages, FFT buffer, sum.
// TMA: each tile is one tensor copy (a.map0: input planes {fast, z, plane},
// a.map1: coil maps {fast, z, coil}; columns past the plane read as zeros)
// completing on the stage's mbarrier, instead of per-thread cp.async.
template <int M, int XT, int kNT, int MINB, bool TMA = false>
__global__ void __launch_bounds__(kNT, MINB) k_coilsum_pipe(const __grid_constant__ mr_strided_args a) {
    extern __shared__ __align__(128) float2 sm[];
    constexpr int TILE = M * XT;
    float2 *wst = sm;                 // [2][M][XT] input tiles
    float2 *sst = sm + 2 * TILE;      // [2][M][XT] coil-map tiles (n_out rows used)
    float2 *buf = sm + 4 * TILE;      // FFT workspace
    float2 *acc = sm + 5 * TILE;      // coil sum (n_out rows)
    int64_t bid = blockIdx.x;
    const int plane = (int)(bid % a.nplane);
    bid /= a.nplane;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const int64_t off0 = (int64_t)outer * a.s_outer + x0;
    const int64_t doff0 = (int64_t)outer * a.d_outer + x0;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 6 * TILE);  // TMA: one per stage
    auto issue = [&](int cc, int st) {
        if constexpr (TMA) {
            if (threadIdx.x == 0) {
                mrtma::fence_proxy_async_smem();
                mrtma::mbar_arrive_expect_tx(bar + st, (a.n_in + a.n_out) * XT *
                                                           (unsigned)sizeof(float2));
                mrtma::tensor3d_g2s(wst + st * TILE, &a.map0, x0, 0, cc * a.L + plane, bar + st);
                mrtma::tensor3d_g2s(sst + st * TILE, &a.map1, x0, 0, a.coil0 + cc, bar + st);
            }
        } else {
            const float2 *srcp = a.src + (int64_t)(cc * a.L + plane) * a.s_plane + off0;
            mr_cp_tile<XT, kNT>(wst + st * TILE, srcp, a.s_axis, a.n_in, nx);
            const float2 *sp = a.xs_s + (int64_t)(a.coil0 + cc) * a.img_plane + doff0;
            mr_cp_tile<XT, kNT>(sst + st * TILE, sp, a.d_axis, a.n_out, nx);
            mr_cp_async_commit();
        }
    };
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            mrtma::mbar_init(bar, 1);
            mrtma::mbar_init(bar + 1, 1);
            mrtma::fence_mbar_init();
        }
        __syncthreads();
    }
    issue(0, 0);
    for (int cc = 0; cc < a.ncoil; ++cc) {
        const int st = cc & 1;
        if (cc + 1 < a.ncoil) issue(cc + 1, st ^ 1);
        if constexpr (TMA) {
            mrtma::mbar_wait(bar + st, (unsigned)(cc >> 1) & 1u, a.status);
        } else {
            if (cc + 1 < a.ncoil) mr_cp_async_wait<1>();
            else mr_cp_async_wait<0>();
        }
        __syncthreads();
        const float2 *w = wst + st * TILE;
        const float2 *sv = sst + st * TILE;
        auto load = [&](int b, int e) -> float2 {
            int sa = e + a.shift_in;
            if (sa >= M) sa -= M;
            return sa < a.n_in ? w[sa * XT + b] : make_float2(0.f, 0.f);
        };
        auto store = [&](int b, int q, float2 v) {
            int da = q + a.shift_out;
            if (da >= M) da -= M;
            if (da < a.n_out) {
                const int ai = da * XT + b;
                const float2 t = c_mulc(sv[ai], v);
                acc[ai] = (cc == 0) ? t : c_add(acc[ai], t);
            }
        };
        mrfix::fft_io<true, true, 1, M, XT, XT, 1, kNT>(buf, a.ax.tw, load, store);
        __syncthreads();
    }
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

// First pass of 3-D / stack plans (forward z lines of S_c x_l), pipelined
// over the ranks: a CTA takes one coil's L planes of a tile; the coil-map
// tile is copied once, and the next rank's image tile is copied (cp.async)
// while the current one is transformed. Same arithmetic as k_strided3<-1,
// XS, BUF> (S_c x_l, then the FFT), so the results are identical. TMA: each
// tile is one tensor copy (a.map0: image planes {fast, z, rank}, a.map1:
// coil maps {fast, z, coil}; columns past the plane read as zeros)
// completing on an mbarrier, instead of per-thread cp.async.
template <int M, int XT, int kNT, int MINB, bool TMA = false>
__global__ void __launch_bounds__(kNT, MINB) k_xs_pipe(const __grid_constant__ mr_strided_args a) {
    extern __shared__ __align__(128) float2 sm[];
    constexpr int TILE = M * XT;
    float2 *sst = sm;                // coil-map tile (n_in rows)
    float2 *xst = sm + TILE;         // [2] image tiles
    float2 *buf = sm + 3 * TILE;     // FFT workspace
    const int ncg = a.nplane / a.L;  // coils
    int64_t bid = blockIdx.x;
    const int cg = (int)(bid % ncg);
    bid /= ncg;
    const int xtile = (int)(bid % a.nxt);
    const int outer = (int)(bid / a.nxt);
    const int x0 = xtile * XT;
    const int nx = min(XT, a.nfast - x0);
    const int64_t off0 = (int64_t)outer * a.s_outer + x0;
    const int64_t doff0 = (int64_t)outer * a.d_outer + x0;
    // TMA: bar[0] the coil-map tile, bar[1 + st] the image tile of stage st
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 4 * TILE);
    const unsigned tb = a.n_in * XT * (unsigned)sizeof(float2);
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            for (int q = 0; q < 3; ++q) mrtma::mbar_init(bar + q, 1);
            mrtma::fence_mbar_init();
            mrtma::mbar_arrive_expect_tx(bar, tb);
            mrtma::tensor3d_g2s(sst, &a.map1, x0, 0, a.coil0 + cg, bar);
            mrtma::mbar_arrive_expect_tx(bar + 1, tb);
            mrtma::tensor3d_g2s(xst, &a.map0, x0, 0, 0, bar + 1);
        }
        __syncthreads();
        mrtma::mbar_wait(bar, 0, a.status);
    } else {
        mr_cp_tile<XT, kNT>(sst, a.xs_s + (int64_t)(a.coil0 + cg) * a.img_plane + off0, a.s_axis,
                            a.n_in, nx);
        mr_cp_tile<XT, kNT>(xst, a.xs_x + off0, a.s_axis, a.n_in, nx);
        mr_cp_async_commit();
    }
    for (int l = 0; l < a.L; ++l) {
        const int st = l & 1;
        if constexpr (TMA) {
            if (l + 1 < a.L && threadIdx.x == 0) {
                mrtma::fence_proxy_async_smem();
                mrtma::mbar_arrive_expect_tx(bar + 1 + (st ^ 1), tb);
                mrtma::tensor3d_g2s(xst + (st ^ 1) * TILE, &a.map0, x0, 0, l + 1,
                                    bar + 1 + (st ^ 1));
            }
            mrtma::mbar_wait(bar + 1 + st, (unsigned)(l >> 1) & 1u, a.status);
        } else {
            if (l + 1 < a.L) {
                mr_cp_tile<XT, kNT>(xst + (st ^ 1) * TILE,
                                    a.xs_x + (int64_t)(l + 1) * a.img_plane + off0, a.s_axis,
                                    a.n_in, nx);
                mr_cp_async_commit();
                mr_cp_async_wait<1>();
            } else {
                mr_cp_async_wait<0>();
            }
        }
        __syncthreads();
        const float2 *xv = xst + st * TILE;
        float2 *dstp = a.dst + (int64_t)(cg * a.L + l) * a.d_plane + doff0;
        auto load = [&](int b, int e) -> float2 {
            int sa = e + a.shift_in;
            if (sa >= M) sa -= M;
            return sa < a.n_in ? c_mul(sst[sa * XT + b], xv[sa * XT + b]) : make_float2(0.f, 0.f);
        };
        auto store = [&](int b, int q, float2 v) {
            int da = q + a.shift_out;
            if (da >= M) da -= M;
            if (da < a.n_out && b < nx) dstp[(int64_t)da * a.d_axis + b] = c_scale(v, a.scale);
        };
        mrfix::fft_io<true, true, -1, M, XT, XT, 1, kNT>(buf, a.ax.tw, load, store);
        __syncthreads();
    }
}

inline bool mr_xs_pipe_ok(const mr_strided_args &a) {
    return mr_env_int("MR_AHA_B200_NO_PIPE", 0) == 0 &&
           (((uintptr_t)a.xs_x | (uintptr_t)a.xs_s) & 15) == 0 &&
           ((a.s_axis | a.s_outer | a.img_plane) & 1) == 0 && a.L >= 1 &&
           a.nplane % a.L == 0;
}

// Whether a pipelined z pass may load its tiles by TMA: one outer block (the
// tiles are boxes of 3-D tensors {fast, z, plane}), lines of at most 256
// points (the box limit), not switched off (MR_AHA_B200_NO_TMA).
inline bool mr_tma_tiles_ok(const mr_strided_args &a) {
    return mr_env_int("MR_AHA_B200_NO_TMA", 0) == 0 && a.nouter == 1 && a.n_in <= 256 &&
           a.nfast >= 1;
}

// Whether the pipelined coil-sum pass can take these arguments: 16-byte
// aligned tiles (even strides and offsets, aligned bases).
inline bool mr_coilsum_pipe_ok(const mr_strided_args &a) {
    return mr_env_int("MR_AHA_B200_NO_PIPE", 0) == 0 &&
           (((uintptr_t)a.src | (uintptr_t)a.xs_s) & 15) == 0 &&
           ((a.s_plane | a.s_axis | a.s_outer | a.img_plane | a.d_axis | a.d_outer) & 1) == 0 &&
           a.ncoil >= 1;
}

template <int DIR, int LM, int SM, int M, int XT>
int launch_s3(const mr_strided_args &a, cudaStream_t s) {
    constexpr int kNT = (M * XT > 10240) ? 512 : 256;
    // CTAs per SM the register budget must allow: small tiles need few
    // registers per thread, so more independent CTAs overlap their phases
    constexpr int MINB = (M * XT > 10240) ? 1 : (M * XT <= 2048 ? 4 : (M * XT <= 5120 ? 3 : 2));
    if constexpr (SM == MR_SM_BUF && LM == MR_LM_XS && DIR < 0 && XT % 2 == 0 &&
                  mrfix::factor(M).n >= 2 && 4 * M * XT * 8 <= 112 * 1024) {
        if (mr_xs_pipe_ok(a)) {
            constexpr int PB = (4 * M * XT * 8 <= 48 * 1024) ? 4 : 2;
            const int64_t nb = (int64_t)a.nxt * a.nouter * (a.nplane / a.L);
            if (nb <= 0) return MR_SUCCESS;
            if (nb > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
            if constexpr ((M * XT) % 16 == 0 && M <= 256 && XT <= 256) {
                if (mr_tma_tiles_ok(a)) {
                    // image planes {fast, z, rank} and coil maps {fast, z, coil}
                    mr_strided_args b = a;
                    const uint64_t d0[3] = {(uint64_t)a.nfast, (uint64_t)a.n_in, (uint64_t)a.L};
                    const uint64_t d1[3] = {(uint64_t)a.nfast, (uint64_t)a.n_in,
                                            (uint64_t)(a.coil0 + a.nplane / a.L)};
                    const uint64_t st[2] = {(uint64_t)a.s_axis * sizeof(float2),
                                            (uint64_t)a.img_plane * sizeof(float2)};
                    const uint32_t box[3] = {(uint32_t)XT, (uint32_t)a.n_in, 1u};
                    int rc = mr_tma_encode_3d(&b.map0, a.xs_x, d0, st, box);
                    if (rc == MR_SUCCESS) rc = mr_tma_encode_3d(&b.map1, a.xs_s, d1, st, box);
                    if (rc != MR_SUCCESS) return rc;
                    static unsigned long long attr_t = 0;
                    set_attr(k_xs_pipe<M, XT, 256, PB, true>, attr_t);
                    k_xs_pipe<M, XT, 256, PB, true>
                        <<<(unsigned)nb, 256, (size_t)4 * M * XT * sizeof(float2) + 32, s>>>(b);
                    MR_LAUNCH_CHECK_T("k_xs_pipe", "k_xs_pipe<M=%d,XT=%d,tma>", M, XT);
                    return MR_SUCCESS;
                }
            }
            static unsigned long long attr_x = 0;
            set_attr(k_xs_pipe<M, XT, 256, PB>, attr_x);
            k_xs_pipe<M, XT, 256, PB><<<(unsigned)nb, 256, (size_t)4 * M * XT * sizeof(float2),
                                        s>>>(a);
            MR_LAUNCH_CHECK_T("k_xs_pipe", "k_xs_pipe<M=%d,XT=%d>", M, XT);
            return MR_SUCCESS;
        }
    }
    if constexpr (SM == MR_SM_COILSUM && LM == MR_LM_BUF && DIR > 0 && XT % 2 == 0 &&
                  mrfix::factor(M).n >= 2 && 6 * M * XT * 8 <= 112 * 1024) {
        if (mr_coilsum_pipe_ok(a)) {
            // CTAs per SM that the shared memory allows, at most 4
            constexpr int PB = (6 * M * XT * 8 <= 48 * 1024) ? 4 : 2;
            const int64_t nb = (int64_t)a.nxt * a.nouter * a.nplane;
            if (nb <= 0) return MR_SUCCESS;
            if (nb > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
            if constexpr ((M * XT) % 16 == 0 && M <= 256 && XT <= 256) {
                if (mr_tma_tiles_ok(a) && a.n_out <= 256) {
                    // input planes {fast, z, plane} and coil maps {fast, z, coil}
                    mr_strided_args b = a;
                    const uint64_t d0[3] = {(uint64_t)a.nfast, (uint64_t)a.n_in,
                                            (uint64_t)a.ncoil * a.L};
                    const uint64_t s0[2] = {(uint64_t)a.s_axis * sizeof(float2),
                                            (uint64_t)a.s_plane * sizeof(float2)};
                    const uint32_t b0[3] = {(uint32_t)XT, (uint32_t)a.n_in, 1u};
                    const uint64_t d1[3] = {(uint64_t)a.nfast, (uint64_t)a.n_out,
                                            (uint64_t)(a.coil0 + a.ncoil)};
                    const uint64_t s1[2] = {(uint64_t)a.d_axis * sizeof(float2),
                                            (uint64_t)a.img_plane * sizeof(float2)};
                    const uint32_t b1[3] = {(uint32_t)XT, (uint32_t)a.n_out, 1u};
                    int rc = mr_tma_encode_3d(&b.map0, a.src, d0, s0, b0);
                    if (rc == MR_SUCCESS) rc = mr_tma_encode_3d(&b.map1, a.xs_s, d1, s1, b1);
                    if (rc != MR_SUCCESS) return rc;
                    static unsigned long long attr_t = 0;
                    set_attr(k_coilsum_pipe<M, XT, 256, PB, true>, attr_t);
                    k_coilsum_pipe<M, XT, 256, PB, true>
                        <<<(unsigned)nb, 256, (size_t)6 * M * XT * sizeof(float2) + 32, s>>>(b);
                    MR_LAUNCH_CHECK_T("k_coilsum_pipe", "k_coilsum_pipe<M=%d,XT=%d,tma>", M, XT);
                    return MR_SUCCESS;
                }
            }
            static unsigned long long attr_p = 0;
            set_attr(k_coilsum_pipe<M, XT, 256, PB>, attr_p);
            k_coilsum_pipe<M, XT, 256, PB><<<(unsigned)nb, 256,
                                             (size_t)6 * M * XT * sizeof(float2), s>>>(a);
            MR_LAUNCH_CHECK_T("k_coilsum_pipe", "k_coilsum_pipe<M=%d,XT=%d>", M, XT);
            return MR_SUCCESS;
        }
    }
    static unsigned long long attr = 0;
    set_attr(k_strided3<DIR, LM, SM, M, XT, kNT, MINB>, attr);
    size_t smem = (size_t)M * XT * sizeof(float2);
    if (SM == MR_SM_COILSUM) smem += (size_t)a.n_out * XT * sizeof(float2);
    const int64_t nblk = (int64_t)a.nxt * a.nouter * a.nplane;
    if (nblk <= 0) return MR_SUCCESS;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "strided pass grid too large");
    k_strided3<DIR, LM, SM, M, XT, kNT, MINB><<<(unsigned)nblk, kNT, smem, s>>>(a);
    MR_LAUNCH_CHECK_T("k_strided3", "k_strided3<%s,M=%d,XT=%d,LM=%d,SM=%d>",
                      DIR < 0 ? "fwd" : "inv", M, XT, LM, SM);
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
    MR_LAUNCH_CHECK_T("k_xbd3", "k_xbd3<M=%d,L=%d,NC=%d,KF=%d>", M, L, NC, KF);
    return MR_SUCCESS;
}

template <int N, int L, int NC, int KF>
int launch_xh(const mr_x_args &a, cudaStream_t s) {
    constexpr int kNT = (NC * L * 2 * N > 10240) ? 512 : 256;
    const size_t smem = (size_t)2 * NC * L * odd_stride<N>() * sizeof(float2);
    const int64_t nblk = (int64_t)a.nloc * a.nchunk;
    if (nblk > 0x7fffffffLL) MR_FAIL(MR_ERR_UNSUPPORTED, "block-diagonal pass grid too large");
    constexpr const char *kfs = KF == MR_KF_F32 ? "F32" : (KF == MR_KF_BF16 ? "BF16" : "I16");
    // blocked kernel copies: complex64 (any rank), 16-bit (rank <= 16, TMA
    // tiles only; without them the 16-bit pass reads the reference layout)
    if constexpr (KF == MR_KF_F32 || L <= 16) {
        if (a.K.blk) {
            if (mr_env_int("MR_AHA_B200_NO_TMA", 0) == 0 && ((uintptr_t)a.src & 15) == 0 &&
                (a.s_row & 1) == 0 && a.plane_rows <= 0x7fffffff) {
                // the group's rows as a 3-D tensor {x, row of a plane, plane}
                mr_x_args b = a;
                const uint64_t dim[3] = {(uint64_t)N, (uint64_t)a.plane_rows,
                                         (uint64_t)a.ncoil * L};
                const uint64_t str[2] = {(uint64_t)a.s_row * sizeof(float2),
                                         (uint64_t)a.plane_rows * a.s_row * sizeof(float2)};
                const uint32_t box[3] = {(uint32_t)(N > 256 ? N / 2 : N), 1u, (uint32_t)(NC * L)};
                const int rc = mr_tma_encode_3d(&b.in_map, a.src, dim, str, box);
                if (rc != MR_SUCCESS) return rc;
                static unsigned long long attr_t = 0;
                set_attr(k_xbdh<N, L, NC, KF, kNT, true, true>, attr_t);
                k_xbdh<N, L, NC, KF, kNT, true, true><<<(unsigned)nblk, kNT, smem + 16, s>>>(b);
                MR_LAUNCH_CHECK_T("k_xbdh", "k_xbdh<N=%d,L=%d,NC=%d,%s,%d,blocked,tma%s>", N, L,
                                  NC, kfs, kNT, a.K.inv ? ",masked" : "");
                return MR_SUCCESS;
            }
            if constexpr (KF == MR_KF_F32) {
                static unsigned long long attr_b = 0;
                set_attr(k_xbdh<N, L, NC, KF, kNT, true>, attr_b);
                k_xbdh<N, L, NC, KF, kNT, true><<<(unsigned)nblk, kNT, smem, s>>>(a);
                MR_LAUNCH_CHECK_T("k_xbdh", "k_xbdh<N=%d,L=%d,NC=%d,F32,%d,blocked%s>", N, L, NC,
                                  kNT, a.K.inv ? ",masked" : "");
                return MR_SUCCESS;
            }
        }
    }
    static unsigned long long attr = 0;
    set_attr(k_xbdh<N, L, NC, KF, kNT>, attr);
    k_xbdh<N, L, NC, KF, kNT><<<(unsigned)nblk, kNT, smem, s>>>(a);
    MR_LAUNCH_CHECK_T("k_xbdh", "k_xbdh<N=%d,L=%d,NC=%d,%s,%d%s>", N, L, NC, kfs, kNT,
                      a.K.inv ? ",masked" : "");
    return MR_SUCCESS;
}

}  // namespace

// Instantiated strided configurations (length, tile width): list A in
// passes3.cu, list B in p3_strided_b.cu; each is built in the four modes the
// plans use. Block-diagonal configurations (length, rank, coils per tile) in
// passes3.cu; half-length ones (N = M / 2, rank, coils per tile): list A in
// passes3.cu, B in p3_xbdh_b.cu, C in p3_xbdh_c.cu.
#define MR_S3_LIST_A(X)                                                                      \
    X(640, 32) X(640, 16) X(640, 8) X(56, 256) X(56, 128) X(56, 64) X(56, 32) X(56, 16)     \
    X(128, 64) X(128, 32) X(8, 256)
#define MR_S3_LIST_B(X)                                                                      \
    X(512, 32) X(512, 16) X(384, 32) X(384, 16) X(256, 64) X(256, 32) X(256, 16) X(32, 256) \
    X(32, 128) X(32, 64) X(32, 32) X(16, 256) X(16, 128) X(16, 64) X(16, 32) X(8, 128)
#define MR_S3_LIST(X) MR_S3_LIST_A(X) MR_S3_LIST_B(X)
#define MR_X3_LIST(X) X(640, 16, 2) X(640, 16, 1) X(128, 4, 4)
#define MR_XH_LIST_A(X) X(320, 32, 1) X(320, 16, 1) X(320, 8, 2) X(320, 4, 4)
#define MR_XH_LIST_B(X)                                                                      \
    X(256, 32, 1) X(256, 16, 1) X(256, 8, 2) X(256, 4, 4) X(192, 32, 1) X(192, 16, 1)        \
    X(192, 8, 2) X(192, 4, 4)
#define MR_XH_LIST_C(X)                                                                      \
    X(128, 32, 1) X(128, 16, 1) X(128, 8, 2) X(128, 4, 4) X(64, 32, 1) X(64, 16, 1)          \
    X(64, 8, 2) X(64, 4, 4)
#define MR_XH_LIST(X) MR_XH_LIST_A(X) MR_XH_LIST_B(X) MR_XH_LIST_C(X)

// Half-length strided passes (N, tile width), in p3_yhalf.cu.
#define MR_SH_LIST(X) X(320, 16) X(320, 8) X(320, 4) X(256, 16) X(256, 8) X(192, 16) X(192, 8) \
    X(128, 16) X(128, 32) X(64, 32) X(64, 16)

// Dispatchers of the other translation units: launch when (M, tile) /
// (N, L, nc) is in their list and set *found, else leave *found false.
int mr_launch_strided3_b(int dir, int lmode, int smode, const mr_strided_args &a,
                         cudaStream_t s, bool *found);
int mr_launch_xbdh_b(const mr_x_args &a, cudaStream_t s, bool *found);
int mr_launch_xbdh_c(const mr_x_args &a, cudaStream_t s, bool *found);

// Strided dispatch body for one list (used by each translation unit).
#define MR_S3_DISPATCH(m, xt)                                                                \
    if (M == m && XT == xt) {                                                                \
        *found = true;                                                                       \
        if (dir < 0 && lmode == MR_LM_BUF && smode == MR_SM_BUF)                             \
            return launch_s3<-1, 0, 0, m, xt>(a, s);                                         \
        if (dir < 0 && lmode == MR_LM_XS && smode == MR_SM_BUF)                              \
            return launch_s3<-1, 1, 0, m, xt>(a, s);                                         \
        if (dir > 0 && lmode == MR_LM_BUF && smode == MR_SM_BUF)                             \
            return launch_s3<1, 0, 0, m, xt>(a, s);                                          \
        if (dir > 0 && lmode == MR_LM_BUF && smode == MR_SM_COILSUM)                         \
            return launch_s3<1, 0, 1, m, xt>(a, s);                                          \
        MR_FAIL(MR_ERR_INTERNAL, "no specialised strided pass for this mode");              \
    }
#define MR_XH_DISPATCH(n, l, c)                                                              \
    if (N == n && a.L == l && a.nc == c) {                                                   \
        *found = true;                                                                       \
        switch (a.K.kf) {                                                                    \
            case MR_KF_F32: return launch_xh<n, l, c, MR_KF_F32>(a, s);                      \
            case MR_KF_BF16: return launch_xh<n, l, c, MR_KF_BF16>(a, s);                    \
            default: return launch_xh<n, l, c, MR_KF_I16>(a, s);                             \
        }                                                                                    \
    }
