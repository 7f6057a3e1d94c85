// Device code of the block-diagonal Toeplitz multiply: at every upsampled
// k-space location the rank row vector of each coil is multiplied from the
// right by the location's Hermitian L x L block, y_c = sum_r v_r A_rc
// (reference include/mr_aha/mr_aha.h:48-62, src/cuda/mr_kernels_bd.cu:56-139).
// The block is stored as one packed triangle; each stored element A_rc is
// read once and contributes A_rc v_r to y_c and, off the diagonal,
// conj(A_rc) v_c to y_r.
//
// Kernel storage formats (template parameter KF):
//   0: complex64 elements, component t of location q at base[q + t * stride];
//   1: bfloat16 (re, im) pairs with one float scale per location;
//   2: int16 (re, im) pairs with one float scale per location (block
//      floating point: value = scale * int16).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_device.cuh"

#define MR_KF_F32 0
#define MR_KF_BF16 1
#define MR_KF_I16 2

struct mr_kernel_ref {
    const void *data;     // element array (format KF)
    const float *scale;   // per-location scale (KF 1, 2), indexed like the location
    int64_t stride;       // elements between consecutive packed components
    const int *inv;       // masked: natural grid index -> mask row, -1 outside; else NULL
    int kf;
    // optional complex64 copy in the blocked layout (unmasked, Mx % 32 == 0):
    // natural grid order, x in blocks of 32. Rank <= 16: components in pairs,
    // with ntri2 = ceil(ntri / 2) component t of block b at
    // blk[((b * ntri2 + t / 2) * 32 + x % 32) * 2 + t % 2] (an odd ntri pads
    // its last pair with zeros); rank > 16: component t of block b at
    // blk[(b * ntri + t) * 32 + x % 32]. 16-bit formats (rank <= 16): the
    // 4-byte codes in groups of four, with ntri4 = ceil(ntri / 4) code t of
    // block b at word ((b * ntri4 + t / 4) * 32 + x % 32) * 4 + t % 4, and the
    // locations' scales in natural grid order in sblk. NULL if absent.
    const float2 *blk;
    const float *sblk;
};

// An int16 (re, im) pair as two floats (exact: every 16-bit integer is a
// float) by integer-to-float conversions, which run beside the FMA pipe: in
// the issue-bound block multiply this measured faster than building the
// floats with byte permutes and float subtractions (int16 pass 3 at 320 x 320
// x 56, L = 16, 12 coils: 40.2 against 41.5 ms).
__device__ __forceinline__ float2 mr_i16x2_to_float2(uint32_t w) {
    return make_float2((float)(short)(w & 0xFFFFu), (float)(short)(w >> 16));
}

// A bfloat16 (re, im) pair as two floats (the bf16 bits are the high half
// of the float's).
__device__ __forceinline__ float2 mr_bf16x2_to_float2(uint32_t w) {
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u));
}

template <int KF>
struct mr_kload {
    const void *base;
    int64_t stride;
    float s;
    // element t without the location's scale (16-bit formats: the stored
    // code; the caller scales the block's result once)
    __device__ __forceinline__ float2 get_raw(int t) const {
        if constexpr (KF == MR_KF_F32) {
            return __ldg(reinterpret_cast<const float2 *>(base) + (int64_t)t * stride);
        } else {
            const uint32_t w =
                __ldg(reinterpret_cast<const unsigned int *>(base) + (int64_t)t * stride);
            if constexpr (KF == MR_KF_BF16) return mr_bf16x2_to_float2(w);
            else return mr_i16x2_to_float2(w);
        }
    }
    __device__ __forceinline__ float2 get(int t) const {
        if constexpr (KF == MR_KF_F32) {
            return __ldg(reinterpret_cast<const float2 *>(base) + (int64_t)t * stride);
        } else if constexpr (KF == MR_KF_BF16) {
            const __nv_bfloat162 v =
                __ldg(reinterpret_cast<const __nv_bfloat162 *>(base) + (int64_t)t * stride);
            const float2 f = __bfloat1622float2(v);
            return make_float2(f.x * s, f.y * s);
        } else {
            const short2 v = __ldg(reinterpret_cast<const short2 *>(base) + (int64_t)t * stride);
            return make_float2((float)v.x * s, (float)v.y * s);
        }
    }
};

// Components per frequency of the blocked layout: the packed triangle,
// padded to an even count when paired (rank <= 16).
__host__ __device__ constexpr int mr_blk_tri(int L) {
    return L <= 16 ? 2 * ((L * (L + 1) / 2 + 1) / 2) : L * (L + 1) / 2;
}

// Components per frequency of the 16-bit blocked layout: the packed triangle
// padded to a multiple of four (four 4-byte codes per 16-byte load).
__host__ __device__ constexpr int mr_blk16_tri(int L) { return 4 * ((L * (L + 1) / 2 + 3) / 4); }

// Loader of one location's 16-bit block from the blocked layout (rank <=
// 16): `base` points at the location's group 0, group p is 32 groups further
// per p, and the four codes of a group come from one 16-byte load that the
// rank-16 walk's consecutive reads share; `s` is the location's scale (the
// block multiply scales its result once).
template <int KF>
struct mr_kload_blk16 {
    const uint4 *base;
    float s;
    __device__ __forceinline__ float2 get_raw(int t) const {
        const uint4 q = __ldg(base + (t >> 2) * 32);
        const uint32_t w = (t & 3) == 0 ? q.x : ((t & 3) == 1 ? q.y : ((t & 3) == 2 ? q.z : q.w));
        if constexpr (KF == MR_KF_BF16) return mr_bf16x2_to_float2(w);
        else return mr_i16x2_to_float2(w);
    }
};

// Loader of one location's block from the blocked layout, paired (rank <=
// 16: `base` points at the location's component pair 0, pair p is 32 pairs
// further per p, and both components of a pair come from one 16-byte load --
// the rank-16 walk reads them one after the other, so the two reads share
// it) or single (component t is 32 elements further per t; the rank-32 walk
// reads half of its elements out of packed order).
template <bool PAIR>
struct mr_kload_blk {
    const float2 *base;
    float s;
    __device__ __forceinline__ float2 get_raw(int t) const {
        if constexpr (PAIR) {
            const float4 q = __ldg(reinterpret_cast<const float4 *>(base) + (t >> 1) * 32);
            return (t & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
        } else {
            return __ldg(base + t * 32);
        }
    }
};

// Loader for the block of location `loc` (row in the kernel array).
template <int KF>
__device__ __forceinline__ mr_kload<KF> mr_kload_at(const mr_kernel_ref &k, int64_t loc) {
    mr_kload<KF> l;
    if constexpr (KF == MR_KF_F32) {
        l.base = reinterpret_cast<const float2 *>(k.data) + loc;
        l.s = 1.0f;
    } else if constexpr (KF == MR_KF_BF16) {
        l.base = reinterpret_cast<const __nv_bfloat162 *>(k.data) + loc;
        l.s = __ldg(k.scale + loc);
    } else {
        l.base = reinterpret_cast<const short2 *>(k.data) + loc;
        l.s = __ldg(k.scale + loc);
    }
    l.stride = k.stride;
    return l;
}

// y[k] = v[k] A for NC vectors of compile-time rank L, walking the packed
// triangle once. All register indices are compile-time constants after
// unrolling. A 16-bit block is multiplied in its stored codes and the result
// scaled once by the location's scale (one multiply per output instead of
// one per element).
template <int L, int NC, int KF, class KL>
__device__ __forceinline__ void bd_block(const float2 (&v)[NC][L], float2 (&y)[NC][L],
                                         const KL &kl, int upper) {
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int i = 0; i < L; ++i) y[k][i] = make_float2(0.f, 0.f);
    int t = 0;
    if (!upper) {
#pragma unroll
        for (int c = 0; c < L; ++c) {
#pragma unroll
            for (int r = c; r < L; ++r) {
                const float2 a = kl.get_raw(t++);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    y[k][c] = c_add(y[k][c], c_mul(a, v[k][r]));
                    if (r != c) y[k][r] = c_add(y[k][r], c_mulc(a, v[k][c]));
                }
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < L; ++c) {
#pragma unroll
            for (int r = 0; r <= c; ++r) {
                const float2 a = kl.get_raw(t++);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    y[k][c] = c_add(y[k][c], c_mul(a, v[k][r]));
                    if (r != c) y[k][r] = c_add(y[k][r], c_mulc(a, v[k][c]));
                }
            }
        }
    }
    if constexpr (KF != MR_KF_F32) {
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
            for (int i = 0; i < L; ++i) y[k][i] = c_scale(y[k][i], kl.s);
    }
}

// Stored index of element (r, c) of a packed L x L triangle (r >= c in the
// lower packing, r <= c in the upper one).
template <int L, bool UPPER>
__host__ __device__ constexpr int bd_t(int r, int c) {
    return UPPER ? c * (c + 1) / 2 + r : c * L - c * (c - 1) / 2 + (r - c);
}

// A_rc of a Hermitian block: the stored element, or the conjugate of the
// stored A_cr (unscaled 16-bit codes for 16-bit formats).
template <int L, bool UPPER, class KL>
__device__ __forceinline__ float2 bd_a(const KL &kl, int r, int c) {
    const bool stored = UPPER ? (r <= c) : (r >= c);
    return stored ? kl.get_raw(bd_t<L, UPPER>(r, c)) : c_conj(kl.get_raw(bd_t<L, UPPER>(c, r)));
}

// Outputs y_c, c in [16 H, 16 H + 16), of y = v A for a rank-32 block, with
// v_r at vl[r * vs] (shared memory): first the diagonal 16 x 16 block, with
// this half of v in registers and each stored pair read once, then the
// off-diagonal block, streaming the other half of v. Two threads (H = 0, 1)
// cover one block, each reading 136 + 256 of its 528 elements and doing half
// of its multiply-adds; each needs 64 registers of vectors instead of 128.
template <int H, bool UPPER, int KF, class KL>
__device__ __forceinline__ void bd_half32(const float2 *vl, int vs, const KL &kl,
                                          float2 (&y)[16]) {
    constexpr int O = 16 * H, P = 16 - O;
    float2 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = vl[(O + i) * vs];
        y[i] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
#pragma unroll
        for (int r = c; r < 16; ++r) {
            const float2 a = bd_a<32, UPPER>(kl, O + r, O + c);
            y[c] = c_add(y[c], c_mul(a, v[r]));
            if (r != c) y[r] = c_add(y[r], c_mulc(a, v[c]));
        }
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const float2 vr = vl[(P + r) * vs];
#pragma unroll
        for (int c = 0; c < 16; ++c)
            y[c] = c_add(y[c], c_mul(bd_a<32, UPPER>(kl, P + r, O + c), vr));
    }
    if constexpr (KF != MR_KF_F32) {
#pragma unroll
        for (int i = 0; i < 16; ++i) y[i] = c_scale(y[i], kl.s);
    }
}

// Packed offset of element (i, j) of the block and whether the stored value
// must be conjugated (the element lies in the unstored triangle).
__device__ __forceinline__ int bd_tri_offset(int i, int j, int L, int upper, bool *cj) {
    int r = i, c = j;
    *cj = false;
    if (upper) {
        if (r > c) { int t = r; r = c; c = t; *cj = true; }
        return c * (c + 1) / 2 + r;
    }
    if (r < c) { int t = r; r = c; c = t; *cj = true; }
    return c * L - c * (c - 1) / 2 + (r - c);
}

// Runtime-rank variant: one output component y_c = sum_r v_r A_rc, with v
// read from `v` (element r at v[r * vs]).
template <int KF>
__device__ __forceinline__ float2 bd_one(const float2 *v, int64_t vs, int L, int c,
                                         const mr_kload<KF> &kl, int upper) {
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < L; ++r) {
        bool cj;
        const int t = bd_tri_offset(r, c, L, upper, &cj);
        float2 a = kl.get(t);
        if (cj) a = c_conj(a);
        acc = c_add(acc, c_mul(a, v[(int64_t)r * vs]));
    }
    return acc;
}

__device__ __forceinline__ int mr_nat2cent_d(int j, int M, int c) {
    int k = j + c;
    return k >= M ? k - M : k;
}
