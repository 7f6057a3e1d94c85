// Device-side mixed-radix FFT used by every pass of the apply and of the
// kernel finish: a Stockham auto-sort transform of many short lines held in
// shared memory, computed cooperatively by all threads of a CTA.
//
// Formulation (for a length M = R_0 R_1 ... R_{k-1} and p = R_0 ... R_{s-1}
// before pass s): butterfly i in [0, M/R) reads u_t = x[i + t M/R],
// multiplies u_t by W_{pR}^{t (i mod p)}, takes an R-point DFT, and writes
// y[(i - i mod p) R + i mod p + t p]. After the last pass the result is in
// natural order. Twiddles come from a per-length table W_M^e, e in [0, M),
// computed on the host in double precision; the inverse uses conjugates.
// Transforms are unnormalised in both directions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MR_FFT_MAX_PASSES 24
#define MR_FFT_MAX_GENERIC_RADIX 256

// Division by an invariant 32-bit divisor d >= 1 for dividends n < 2^31:
// n / d = (umulhi(n, m) + n) >> s with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1 (Granlund and Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994).
struct mr_fdiv {
    unsigned d, m, s;
};

__host__ __device__ inline mr_fdiv mr_make_fdiv(unsigned d) {
    mr_fdiv f;
    f.d = d;
    unsigned s = 0;
    while ((1ull << s) < (unsigned long long)d) ++s;
    f.s = s;
    f.m = (unsigned)((((unsigned long long)1 << 32) * ((1ull << s) - d)) / d + 1);
    return f;
}

__device__ __forceinline__ int mr_div(int n, const mr_fdiv &f) {
    return (int)((__umulhi((unsigned)n, f.m) + (unsigned)n) >> f.s);
}

struct mr_fft_axis {
    int M;
    int npass;
    int radix[MR_FFT_MAX_PASSES];
    int p[MR_FFT_MAX_PASSES];        // product of the radices before pass s
    mr_fdiv fp[MR_FFT_MAX_PASSES];   // division by p[s]
    int small;                       // every radix in {2, 3, 4, 5, 7, 8}
    const float2 *tw;  // W_M^e = exp(-2 pi i e / M)
};

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward, DIR=-1) or +i (inverse, DIR=+1)
template <int DIR>
__device__ __forceinline__ float2 c_mul_i(float2 a) {
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// Twiddle from the table: forward uses W, inverse conj(W).
template <int DIR>
__device__ __forceinline__ float2 tw_get(const float2 *tw, int e) {
    float2 w = __ldg(tw + e);
    return DIR < 0 ? w : make_float2(w.x, -w.y);
}

// ---- small DFTs: X_q = sum_t u_t exp(DIR 2 pi i t q / R) ------------------

template <int DIR>
__device__ __forceinline__ void dft2(float2 *u) {
    float2 a = u[0], b = u[1];
    u[0] = c_add(a, b);
    u[1] = c_sub(a, b);
}

template <int DIR>
__device__ __forceinline__ void dft3(float2 *u) {
    // cos(2pi/3) = -1/2, sin(2pi/3) = sqrt(3)/2
    const float s3 = 0.86602540378443864676f;
    float2 a = u[0], b = u[1], c = u[2];
    float2 s = c_add(b, c), d = c_sub(b, c);
    float2 m = make_float2(a.x - 0.5f * s.x, a.y - 0.5f * s.y);
    // DIR * i * s3 * d
    float2 r = c_mul_i<DIR>(make_float2(s3 * d.x, s3 * d.y));
    u[0] = c_add(a, s);
    u[1] = c_add(m, r);
    u[2] = c_sub(m, r);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2 *u) {
    float2 a0 = c_add(u[0], u[2]), a1 = c_sub(u[0], u[2]);
    float2 b0 = c_add(u[1], u[3]), b1 = c_mul_i<DIR>(c_sub(u[1], u[3]));
    u[0] = c_add(a0, b0);
    u[2] = c_sub(a0, b0);
    u[1] = c_add(a1, b1);
    u[3] = c_sub(a1, b1);
}

template <int DIR>
__device__ __forceinline__ void dft5(float2 *u) {
    // c1 = cos(2pi/5), c2 = cos(4pi/5), s1 = sin(2pi/5), s2 = sin(4pi/5)
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 a = u[0];
    float2 p1 = c_add(u[1], u[4]), m1 = c_sub(u[1], u[4]);
    float2 p2 = c_add(u[2], u[3]), m2 = c_sub(u[2], u[3]);
    float2 r1 = make_float2(a.x + c1 * p1.x + c2 * p2.x, a.y + c1 * p1.y + c2 * p2.y);
    float2 r2 = make_float2(a.x + c2 * p1.x + c1 * p2.x, a.y + c2 * p1.y + c1 * p2.y);
    float2 i1 = c_mul_i<DIR>(make_float2(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y));
    float2 i2 = c_mul_i<DIR>(make_float2(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y));
    u[0] = make_float2(a.x + p1.x + p2.x, a.y + p1.y + p2.y);
    u[1] = c_add(r1, i1);
    u[4] = c_sub(r1, i1);
    u[2] = c_add(r2, i2);
    u[3] = c_sub(r2, i2);
}

template <int DIR>
__device__ __forceinline__ void dft7(float2 *u) {
    const float c1 = 0.62348980185873353053f, c2 = -0.22252093395631440429f,
                c3 = -0.90096886790241912624f;
    const float s1 = 0.78183148246802980871f, s2 = 0.97492791218182360702f,
                s3 = 0.43388373911755812048f;
    float2 a = u[0];
    float2 p1 = c_add(u[1], u[6]), m1 = c_sub(u[1], u[6]);
    float2 p2 = c_add(u[2], u[5]), m2 = c_sub(u[2], u[5]);
    float2 p3 = c_add(u[3], u[4]), m3 = c_sub(u[3], u[4]);
    float2 r1 = make_float2(a.x + c1 * p1.x + c2 * p2.x + c3 * p3.x,
                            a.y + c1 * p1.y + c2 * p2.y + c3 * p3.y);
    float2 r2 = make_float2(a.x + c2 * p1.x + c3 * p2.x + c1 * p3.x,
                            a.y + c2 * p1.y + c3 * p2.y + c1 * p3.y);
    float2 r3 = make_float2(a.x + c3 * p1.x + c1 * p2.x + c2 * p3.x,
                            a.y + c3 * p1.y + c1 * p2.y + c2 * p3.y);
    // sin(2pi q t / 7) for q = 1..3: rows (s1 s2 s3), (s2 -s3 -s1), (s3 -s1 s2)
    float2 i1 = c_mul_i<DIR>(make_float2(s1 * m1.x + s2 * m2.x + s3 * m3.x,
                                         s1 * m1.y + s2 * m2.y + s3 * m3.y));
    float2 i2 = c_mul_i<DIR>(make_float2(s2 * m1.x - s3 * m2.x - s1 * m3.x,
                                         s2 * m1.y - s3 * m2.y - s1 * m3.y));
    float2 i3 = c_mul_i<DIR>(make_float2(s3 * m1.x - s1 * m2.x + s2 * m3.x,
                                         s3 * m1.y - s1 * m2.y + s2 * m3.y));
    u[0] = make_float2(a.x + p1.x + p2.x + p3.x, a.y + p1.y + p2.y + p3.y);
    u[1] = c_add(r1, i1);
    u[6] = c_sub(r1, i1);
    u[2] = c_add(r2, i2);
    u[5] = c_sub(r2, i2);
    u[3] = c_add(r3, i3);
    u[4] = c_sub(r3, i3);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2 *u) {
    const float h = 0.70710678118654752440f;
    // Decimation in frequency: pairs (t, t + 4); the even outputs are the
    // 4-point DFT of the sums, the odd outputs that of the differences
    // twiddled by w^t, w = exp(DIR i pi / 4) = h (1 + DIR i).
    float2 e[4], o[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        e[t] = c_add(u[t], u[t + 4]);
        o[t] = c_sub(u[t], u[t + 4]);
    }
    float2 t1 = c_mul_i<DIR>(o[1]);
    o[1] = make_float2(h * (o[1].x + t1.x), h * (o[1].y + t1.y));   // w
    o[2] = c_mul_i<DIR>(o[2]);                                        // w^2 = DIR i
    float2 t3 = c_mul_i<DIR>(o[3]);
    o[3] = make_float2(h * (t3.x - o[3].x), h * (t3.y - o[3].y));   // w^3 = h(-1 + DIR i)
    dft4<DIR>(e);
    dft4<DIR>(o);
    u[0] = e[0]; u[2] = e[1]; u[4] = e[2]; u[6] = e[3];
    u[1] = o[0]; u[3] = o[1]; u[5] = o[2]; u[7] = o[3];
}

// cos(2 pi m / R) and sin(2 pi m / R) for R = 16 or 20, from the cosines of
// the first quadrant (cos(2 pi j / R), j = 0 .. R / 4) and the quadrant
// symmetries, so that every value is the correctly rounded float of the
// exact one.
__host__ __device__ constexpr float quad_cos(int R, int j) {
    constexpr double c16[5] = {1.0, 0.92387953251128675613, 0.70710678118654752440,
                               0.38268343236508977173, 0.0};
    constexpr double c20[6] = {1.0, 0.95105651629515357212, 0.80901699437494742410,
                               0.58778525229247312917, 0.30901699437494742410, 0.0};
    return (float)(R == 16 ? c16[j] : c20[j]);
}
__host__ __device__ constexpr float root_cos(int R, int m) {
    const int q = (m % R) / (R / 4), r = (m % R) % (R / 4), Q = R / 4;
    return q == 0 ? quad_cos(R, r) : q == 1 ? -quad_cos(R, Q - r)
                                 : q == 2 ? -quad_cos(R, r) : quad_cos(R, Q - r);
}
__host__ __device__ constexpr float root_sin(int R, int m) {
    const int q = (m % R) / (R / 4), r = (m % R) % (R / 4), Q = R / 4;
    return q == 0 ? quad_cos(R, Q - r) : q == 1 ? quad_cos(R, r)
                                     : q == 2 ? -quad_cos(R, Q - r) : -quad_cos(R, r);
}

template <int R, int DIR>
__device__ __forceinline__ void dft_small(float2 *u);

// R = P Q point DFT in registers by one Cooley-Tukey step (n = Q n1 + n2,
// k = k1 + P k2): X[k1 + P k2] = sum_{n2} W_Q^{n2 k2} W_R^{n2 k1}
// sum_{n1} x[Q n1 + n2] W_P^{n1 k1}, W_R = exp(DIR 2 pi i / R); the inner
// twiddles are compile-time constants (exact for multiples of pi / 2).
template <int P, int Q, int DIR>
__device__ __forceinline__ void dft_pq(float2 *u) {
    constexpr int R = P * Q;
    float2 a[Q][P];
#pragma unroll
    for (int n2 = 0; n2 < Q; ++n2) {
#pragma unroll
        for (int n1 = 0; n1 < P; ++n1) a[n2][n1] = u[Q * n1 + n2];
        dft_small<P, DIR>(a[n2]);
#pragma unroll
        for (int k1 = 1; k1 < P; ++k1) {
            const int m = (n2 * k1) % R;
            if (m == 0) continue;
            if (4 * m == R) a[n2][k1] = c_mul_i<DIR>(a[n2][k1]);
            else if (2 * m == R) a[n2][k1] = make_float2(-a[n2][k1].x, -a[n2][k1].y);
            else if (4 * m == 3 * R) a[n2][k1] = c_mul_i<-DIR>(a[n2][k1]);
            else
                a[n2][k1] = c_mul(a[n2][k1],
                                  make_float2(root_cos(R, m), DIR < 0 ? -root_sin(R, m)
                                                                      : root_sin(R, m)));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
        float2 b[Q];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) b[n2] = a[n2][k1];
        dft_small<Q, DIR>(b);
#pragma unroll
        for (int k2 = 0; k2 < Q; ++k2) u[k1 + P * k2] = b[k2];
    }
}

template <int R, int DIR>
__device__ __forceinline__ void dft_small(float2 *u) {
    if constexpr (R == 2) dft2<DIR>(u);
    else if constexpr (R == 3) dft3<DIR>(u);
    else if constexpr (R == 4) dft4<DIR>(u);
    else if constexpr (R == 5) dft5<DIR>(u);
    else if constexpr (R == 7) dft7<DIR>(u);
    else if constexpr (R == 8) dft8<DIR>(u);
    else if constexpr (R == 16) dft_pq<4, 4, DIR>(u);
    else if constexpr (R == 20) dft_pq<4, 5, DIR>(u);
}

// ---- one Stockham pass over nlines lines ----------------------------------
// Element e of line b lives at buf[b * ls + e * es]. line_fast selects the
// mapping of consecutive threads: to consecutive lines (ls == 1 layouts) or
// to consecutive butterflies of one line (es == 1 layouts).
template <int R, int DIR>
__device__ __forceinline__ void stockham_pass(const float2 *__restrict__ src,
                                              float2 *__restrict__ dst, int M,
                                              int p, const float2 *tw, int nlines,
                                              int es, int ls, bool line_fast) {
    const int mr = M / R;
    const int total = nlines * mr;
    const int tstep = M / (p * R);
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int b, i;
        if (line_fast) {
            b = w % nlines;
            i = w / nlines;
        } else {
            i = w % mr;
            b = w / mr;
        }
        const float2 *s = src + (int64_t)b * ls;
        float2 u[R];
#pragma unroll
        for (int t = 0; t < R; ++t) u[t] = s[(i + t * mr) * es];
        const int k = i % p;
        if (p > 1) {
            const int e1 = k * tstep;
#pragma unroll
            for (int t = 1; t < R; ++t) u[t] = c_mul(u[t], tw_get<DIR>(tw, t * e1));
        }
        dft_small<R, DIR>(u);
        const int j = (i - k) * R + k;
        float2 *d = dst + (int64_t)b * ls;
#pragma unroll
        for (int t = 0; t < R; ++t) d[(j + t * p) * es] = u[t];
    }
}

// Generic radix (any R <= MR_FFT_MAX_GENERIC_RADIX): direct R-point DFT with
// roots W_M^{(M/R)(t q mod R)} from the table.
template <int DIR>
__device__ __noinline__ void stockham_pass_generic(const float2 *__restrict__ src,
                                                   float2 *__restrict__ dst, int M,
                                                   int R, int p, const float2 *tw,
                                                   int nlines, int es, int ls,
                                                   bool line_fast) {
    const int mr = M / R;
    const int total = nlines * mr;
    const int tstep = M / (p * R);
    float2 u[MR_FFT_MAX_GENERIC_RADIX];
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int b, i;
        if (line_fast) {
            b = w % nlines;
            i = w / nlines;
        } else {
            i = w % mr;
            b = w / mr;
        }
        const float2 *s = src + (int64_t)b * ls;
        const int k = i % p;
        for (int t = 0; t < R; ++t) {
            float2 v = s[(i + t * mr) * es];
            if (p > 1 && t > 0) v = c_mul(v, tw_get<DIR>(tw, t * k * tstep));
            u[t] = v;
        }
        const int j = (i - k) * R + k;
        float2 *d = dst + (int64_t)b * ls;
        for (int q = 0; q < R; ++q) {
            float2 acc = u[0];
            int e = 0;
            for (int t = 1; t < R; ++t) {
                e += q;
                if (e >= R) e -= R;
                acc = c_add(acc, c_mul(u[t], tw_get<DIR>(tw, e * mr)));
            }
            d[(j + q * p) * es] = acc;
        }
    }
}

// Full transform of nlines lines; a holds the input, b is scratch of the
// same shape. Returns the buffer holding the result. Must be called by all
// threads of the CTA (it synchronises after every pass).
template <int DIR>
__device__ float2 *fft_lines(float2 *a, float2 *b, const mr_fft_axis &ax, int nlines,
                             int es, int ls, bool line_fast) {
    int p = 1;
    for (int s = 0; s < ax.npass; ++s) {
        const int R = ax.radix[s];
        switch (R) {
            case 2: stockham_pass<2, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            case 3: stockham_pass<3, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            case 4: stockham_pass<4, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            case 5: stockham_pass<5, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            case 7: stockham_pass<7, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            case 8: stockham_pass<8, DIR>(a, b, ax.M, p, ax.tw, nlines, es, ls, line_fast); break;
            default:
                stockham_pass_generic<DIR>(a, b, ax.M, R, p, ax.tw, nlines, es, ls, line_fast);
                break;
        }
        __syncthreads();
        float2 *t = a;
        a = b;
        b = t;
        p *= R;
    }
    return a;
}
