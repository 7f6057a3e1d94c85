// Compile-time-specialised in-place Stockham FFT for the lengths the plans
// use most. The length, radix sequence, line count, strides and thread count
// are template parameters, so every index of every butterfly folds to a
// per-thread base plus constant offsets, and the passes contain no run-time
// radix switch and (when the work divides evenly) no bounds guards. Same
// formulation as fft_device.cuh: butterfly i of a radix-R pass with p =
// product of earlier radices reads x[i + t M/R], twiddles by
// W_{pR}^{t (i mod p)}, transforms, and writes y[(i - i mod p) R + i mod p + t p];
// all reads of a pass finish (barrier) before its writes, in place.
#pragma once

#include "fft_device.cuh"

namespace mrfix {

struct radix_list {
    int n;
    int r[16];
};

// Radix policy of the host planner (passes.cu mr_fft_factor): eights, then a
// four or a two, then fives, threes, sevens. Lengths with other factors are
// not specialised (n = 0). Exception: 320 (the half-length lines of the
// 640-point grids) runs as 16 x 20, two register-resident passes instead of
// three (8, 8, 5): one shared-memory round trip and barrier fewer per line.
// Measured at 320 x 320 x 56, L = 16, 12 coils: y forward 6.51 -> 5.84 ms,
// y inverse 6.52 -> 6.36 ms, x pass 3 (with its L2 kernel prefetch) 44.4 ->
// 42.6 ms. Other lengths keep radix 8, whose smaller register stages spill
// less.
constexpr radix_list factor(int M) {
    radix_list l{0, {}};
    if (M == 320) {
        l.n = 2;
        l.r[0] = 16;
        l.r[1] = 20;
        return l;
    }
    int e2 = 0;
    while (M % 2 == 0) {
        M /= 2;
        ++e2;
    }
    while (e2 >= 3) {
        l.r[l.n++] = 8;
        e2 -= 3;
    }
    if (e2 == 2) l.r[l.n++] = 4;
    if (e2 == 1) l.r[l.n++] = 2;
    while (M % 5 == 0) {
        l.r[l.n++] = 5;
        M /= 5;
    }
    while (M % 3 == 0) {
        l.r[l.n++] = 3;
        M /= 3;
    }
    while (M % 7 == 0) {
        l.r[l.n++] = 7;
        M /= 7;
    }
    if (M != 1) l.n = 0;
    return l;
}

constexpr int max_stage(int M, int NL, int NT) {
    const radix_list l = factor(M);
    int m = 0;
    for (int s = 0; s < l.n; ++s) {
        const int R = l.r[s];
        const int total = NL * (M / R);
        const int nb = (total + NT - 1) / NT;
        if (nb * R > m) m = nb * R;
    }
    return m;
}

template <int R, int DIR, int M, int P, int NL, int ES, int LS, int NT, int TWS, int UA>
__device__ __forceinline__ void pass(float2 *buf, const float2 *__restrict__ tw, float2 (&u)[UA]) {
    constexpr int MR = M / R;
    constexpr int TOTAL = NL * MR;
    constexpr int NB = (TOTAL + NT - 1) / NT;
    constexpr int TSTEP = TWS * (M / (P * R));
    constexpr bool EXACT = (TOTAL % NT) == 0;
    static_assert(NB * R <= UA, "register stage too small");
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = tid + k * NT;
        if (EXACT || w < TOTAL) {
            const int i = w / NL;
            const int b = w - i * NL;
            const float2 *s = buf + b * LS + i * ES;
#pragma unroll
            for (int t = 0; t < R; ++t) u[k * R + t] = s[t * MR * ES];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = tid + k * NT;
        if (EXACT || w < TOTAL) {
            const int i = w / NL;
            const int b = w - i * NL;
            const int kk = i % P;
            const int q = i / P;
            if constexpr (P > 1) {
                const int e1 = kk * TSTEP;
#pragma unroll
                for (int t = 1; t < R; ++t)
                    u[k * R + t] = c_mul(u[k * R + t], tw_get<DIR>(tw, t * e1));
            }
            dft_small<R, DIR>(&u[k * R]);
            float2 *d = buf + b * LS + (q * P * R + kk) * ES;
#pragma unroll
            for (int t = 0; t < R; ++t) d[t * P * ES] = u[k * R + t];
        }
    }
    __syncthreads();
}

template <int DIR, int M, int NL, int ES, int LS, int NT, int TWS, int S, int P, int UA>
__device__ __forceinline__ void run(float2 *buf, const float2 *tw, float2 (&u)[UA]) {
    constexpr radix_list l = factor(M);
    if constexpr (S < l.n) {
        constexpr int R = l.r[S];
        pass<R, DIR, M, P, NL, ES, LS, NT, TWS>(buf, tw, u);
        run<DIR, M, NL, ES, LS, NT, TWS, S + 1, P * R>(buf, tw, u);
    }
}

// In-place transform of NL lines of length M held in shared memory (element
// e of line b at buf[b * LS + e * ES]) by NT threads. The twiddle table holds
// W_{TWS M}^e: TWS = 1 for a table of this length, 2 for the table of the
// doubled length (a length-M transform inside a length-2M one).
template <int DIR, int M, int NL, int ES, int LS, int NT, int TWS = 1>
__device__ __forceinline__ void fft(float2 *buf, const float2 *tw) {
    static_assert(factor(M).n > 0, "length not specialised");
    constexpr int UA = max_stage(M, NL, NT);
    float2 u[UA];
    run<DIR, M, NL, ES, LS, NT, TWS, 0, 1>(buf, tw, u);
}

}  // namespace mrfix

namespace mrfix {

// First pass reading its inputs through load(b, e) (element e of line b)
// instead of shared memory: no barrier before it, outputs to shared memory.
template <int R, int DIR, int M, int NL, int ES, int LS, int NT, int UA, class LoadF>
__device__ __forceinline__ void pass_first(float2 *buf, float2 (&u)[UA], const LoadF &load) {
    constexpr int MR = M / R;
    constexpr int TOTAL = NL * MR;
    constexpr int NB = (TOTAL + NT - 1) / NT;
    constexpr bool EXACT = (TOTAL % NT) == 0;
    static_assert(NB * R <= UA, "register stage too small");
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = tid + k * NT;
        if (EXACT || w < TOTAL) {
            const int i = w / NL;
            const int b = w - i * NL;
#pragma unroll
            for (int t = 0; t < R; ++t) u[k * R + t] = load(b, i + t * MR);
        }
    }
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = tid + k * NT;
        if (EXACT || w < TOTAL) {
            const int i = w / NL;
            const int b = w - i * NL;
            dft_small<R, DIR>(&u[k * R]);
            float2 *d = buf + b * LS + (i * R) * ES;   // p = 1
#pragma unroll
            for (int t = 0; t < R; ++t) d[t * ES] = u[k * R + t];
        }
    }
    __syncthreads();
}

// Last pass writing its outputs through store(b, e, v) instead of shared
// memory (no barrier needed after its reads: shared memory is not written).
template <int R, int DIR, int M, int P, int NL, int ES, int LS, int NT, int TWS, int UA,
          class StoreF>
__device__ __forceinline__ void pass_last(const float2 *buf, const float2 *__restrict__ tw,
                                          float2 (&u)[UA], const StoreF &store) {
    constexpr int MR = M / R;
    constexpr int TOTAL = NL * MR;
    constexpr int NB = (TOTAL + NT - 1) / NT;
    constexpr int TSTEP = TWS * (M / (P * R));
    constexpr bool EXACT = (TOTAL % NT) == 0;
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int w = tid + k * NT;
        if (EXACT || w < TOTAL) {
            const int i = w / NL;
            const int b = w - i * NL;
            const float2 *s = buf + b * LS + i * ES;
#pragma unroll
            for (int t = 0; t < R; ++t) u[k * R + t] = s[t * MR * ES];
            const int kk = i % P;
            const int q = i / P;
            if constexpr (P > 1) {
                const int e1 = kk * TSTEP;
#pragma unroll
                for (int t = 1; t < R; ++t)
                    u[k * R + t] = c_mul(u[k * R + t], tw_get<DIR>(tw, t * e1));
            }
            dft_small<R, DIR>(&u[k * R]);
#pragma unroll
            for (int t = 0; t < R; ++t) store(b, q * P * R + kk + t * P, u[k * R + t]);
        }
    }
}

template <bool LASTG, int DIR, int M, int NL, int ES, int LS, int NT, int TWS, int S, int P,
          int UA, class StoreF>
__device__ __forceinline__ void run_io(float2 *buf, const float2 *tw, float2 (&u)[UA],
                                       const StoreF &store) {
    constexpr radix_list l = factor(M);
    if constexpr (S < l.n) {
        constexpr int R = l.r[S];
        if constexpr (LASTG && S + 1 == l.n) {
            pass_last<R, DIR, M, P, NL, ES, LS, NT, TWS>(buf, tw, u, store);
        } else {
            pass<R, DIR, M, P, NL, ES, LS, NT, TWS>(buf, tw, u);
            run_io<LASTG, DIR, M, NL, ES, LS, NT, TWS, S + 1, P * R>(buf, tw, u, store);
        }
    }
}

struct no_store {
    __device__ void operator()(int, int, float2) const {}
};

// Transform of NL lines (twiddle table of TWS times the length, as fft()).
// FIRSTG: the first pass reads load(b, e) (element e of line b) instead of
// shared memory. LASTG: the last pass writes
// store(b, e, v) instead of shared memory (the result is then not in buf;
// the caller synchronises before reusing buf). Otherwise the result is in
// buf in natural order.
template <bool FIRSTG, bool LASTG, int DIR, int M, int NL, int ES, int LS, int NT, int TWS = 1,
          class LoadF, class StoreF>
__device__ __forceinline__ void fft_io(float2 *buf, const float2 *tw, const LoadF &load,
                                       const StoreF &store) {
    constexpr radix_list l = factor(M);
    static_assert(l.n >= 1, "length not specialised");
    static_assert(!(FIRSTG && LASTG) || l.n >= 2, "one-pass transform cannot do both");
    constexpr int UA = max_stage(M, NL, NT);
    float2 u[UA];
    if constexpr (FIRSTG) {
        constexpr int R0 = l.r[0];
        pass_first<R0, DIR, M, NL, ES, LS, NT>(buf, u, load);
        run_io<LASTG, DIR, M, NL, ES, LS, NT, TWS, 1, R0>(buf, tw, u, store);
    } else {
        run_io<LASTG, DIR, M, NL, ES, LS, NT, TWS, 0, 1>(buf, tw, u, store);
    }
}

}  // namespace mrfix
