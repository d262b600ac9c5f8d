// Device building blocks of the split-operator step: complex arithmetic,
// in-register radix-2/3/4/5/6/8/10/12/16/20/32 DFTs, and one Stockham autosort stage over a
// tile of L lines held in shared memory.
//
// The line FFT is the forward unnormalised transform X_k = sum_n x_n e^{-2 pi i kn/N}
// of the reference (core/src/fft.ixx:14-18).  Inverse transforms use the
// conjugation identity ifft(X) = conj(fft(conj(X)))/N (fft.ixx:89-98), with the
// conjugations and 1/N folded into the neighbouring element-wise operations.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sesk {

constexpr int kMaxStages = 12;

template <typename T>
struct __align__(2 * sizeof(T)) cx {
    T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cx<T> mk(T a, T b) {
    cx<T> r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename T>
__device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) {
    return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T>
__device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) {
    return mk<T>(a.x - b.x, a.y - b.y);
}
// complex64 sums and differences as packed FP32 pairs (sm_100 add/sub.f32x2):
// per component the same IEEE round-to-nearest operation as the scalar form,
// in one instruction instead of two.
__device__ __forceinline__ float2 as_f2(cx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cx<float> from_f2(float2 a) { return mk<float>(a.x, a.y); }
__device__ __forceinline__ cx<float> operator+(cx<float> a, cx<float> b) {
    return from_f2(__fadd2_rn(as_f2(a), as_f2(b)));
}
__device__ __forceinline__ cx<float> operator-(cx<float> a, cx<float> b) {
    cx<float> c;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rc, ra, rb;\n\tmov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(c.x), "=f"(c.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return c;
}
// Complex product with the FMAs written out: the compiler may not contract the
// two products of a component differently in different kernels, so every pass
// that multiplies the same operands gets the same bits (a run split into two
// calls equals one call; the step forms agree).
template <typename T>
__device__ __forceinline__ cx<T> operator*(cx<T> a, cx<T> b) {
    return mk<T>(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
// a * s for an FP64 scale s such as 1/N, which is not a power of two for
// radix-3/5 sizes: complex64 carries s as hi + lo, so that the scale applied
// every step has no systematic rounding (a plain FP32 1/N is off by up to 6e-8,
// which would move the norm by ~1e-7 every step).
template <typename T>
__device__ __forceinline__ cx<T> scale_d(cx<T> a, double s) {
    if constexpr (sizeof(T) == 4) {
        const float hi = (float)s, lo = (float)(s - (double)hi);
        return mk<float>(fmaf(a.x, hi, a.x * lo), fmaf(a.y, hi, a.y * lo));
    } else {
        return mk<double>(a.x * s, a.y * s);
    }
}
// a * (-i)
template <typename T>
__device__ __forceinline__ cx<T> mul_mi(cx<T> a) {
    return mk<T>(a.y, -a.x);
}
template <typename T>
__device__ __forceinline__ cx<T> cconj(cx<T> a) {
    return mk<T>(a.x, -a.y);
}
template <typename T>
__device__ __forceinline__ cx<double> widen(cx<T> a) {
    return mk<double>((double)a.x, (double)a.y);
}
template <typename T>
__device__ __forceinline__ cx<T> narrow(cx<double> a) {
    return mk<T>((T)a.x, (T)a.y);
}

// Division by a run-time invariant divisor with one multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994).  Valid for dividends below 2^31.
struct FastDiv {
    uint32_t d, mul, shr;
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f{d, 0u, 0u};
    if (d <= 1) return f;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;            // ceil(log2 d)
    const uint32_t p = 31 + l;
    f.mul = (uint32_t)(((1ull << p) + d - 1) / d);
    f.shr = p - 32;
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t x, const FastDiv& f) {
    return f.d <= 1 ? x : (__umulhi(x, f.mul) >> f.shr);
}

// ---------------------------------------------------------------------------
// In-register DFTs of size R, forward (e^{-}), natural-order output.
// The constants are cos/sin of the R-th roots of unity.  In FP32 each constant
// is carried as hi + lo (lo = the FP32 rounding of its remainder) and applied
// with one extra FMA: a plain FP32 constant such as (float)(1/sqrt 2) is
// ~1.7e-8 small, and that bias would shrink the norm by ~1e-7 every step.
// ---------------------------------------------------------------------------
template <typename T>
struct CK {
    T hi, lo;
};

template <typename T>
__device__ __forceinline__ CK<T> ck(double c) {
    if constexpr (sizeof(T) == 4) {
        const float hi = (float)c;
        return CK<T>{hi, (float)(c - (double)hi)};
    } else {
        return CK<T>{c, 0.0};
    }
}

// a * c for complex a and a real compensated constant c = c.hi + c.lo,
// componentwise fma(a, c.hi, a * c.lo) (complex64 as two packed FP32 operations).
template <typename T>
__device__ __forceinline__ cx<T> kmulc(cx<T> a, CK<T> c) {
    if constexpr (sizeof(T) == 4)
        return from_f2(__ffma2_rn(as_f2(a), make_float2(c.hi, c.hi), __fmul2_rn(as_f2(a), make_float2(c.lo, c.lo))));
    else
        return mk<T>(a.x * c.hi, a.y * c.hi);
}

// v * (c - i s) with compensated constants
template <typename T>
__device__ __forceinline__ cx<T> rotc(cx<T> v, CK<T> c, CK<T> s) {
    if constexpr (sizeof(T) == 4) {
        return mk<T>(fmaf(v.x, c.hi, fmaf(v.y, s.hi, fmaf(v.x, c.lo, v.y * s.lo))),
                     fmaf(v.y, c.hi, fmaf(-v.x, s.hi, fmaf(v.y, c.lo, -v.x * s.lo))));
    } else {
        return mk<T>(fma(v.x, c.hi, v.y * s.hi), fma(v.y, c.hi, -(v.x * s.hi)));
    }
}

template <typename T>
__device__ __forceinline__ CK<T> neg(CK<T> c) {
    return CK<T>{-c.hi, -c.lo};
}

template <typename T>
__device__ __forceinline__ void dft2(cx<T>* v) {
    const cx<T> a = v[0];
    v[0] = a + v[1];
    v[1] = a - v[1];
}

template <typename T>
__device__ __forceinline__ void dft4(cx<T>* v) {
    const cx<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
    const cx<T> t2 = v[1] + v[3], t3 = mul_mi(v[1] - v[3]);
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + t3;
    v[3] = t1 - t3;
}

template <typename T>
__device__ __forceinline__ void dft8(cx<T>* v) {
    const CK<T> h = ck<T>(0.70710678118654752440);  // cos(pi/4)
    cx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e);
    dft4(o);
    o[1] = rotc(o[1], h, h);          // * e^{-i pi/4}
    o[2] = mul_mi(o[2]);              // * e^{-i pi/2}
    o[3] = rotc(o[3], neg(h), h);     // * e^{-3i pi/4}
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = e[k] + o[k];
        v[k + 4] = e[k] - o[k];
    }
}

template <typename T>
__device__ __forceinline__ void dft16(cx<T>* v) {
    const CK<T> c1 = ck<T>(0.92387953251128675613);  // cos(pi/8)
    const CK<T> s1 = ck<T>(0.38268343236508977173);  // sin(pi/8)
    const CK<T> h = ck<T>(0.70710678118654752440);   // cos(pi/4)
    cx<T> e[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        e[k] = v[2 * k];
        o[k] = v[2 * k + 1];
    }
    dft8(e);
    dft8(o);
    // o[k] *= e^{-2 pi i k / 16}
    o[1] = rotc(o[1], c1, s1);
    o[2] = rotc(o[2], h, h);
    o[3] = rotc(o[3], s1, c1);
    o[4] = mul_mi(o[4]);
    o[5] = rotc(o[5], neg(s1), c1);
    o[6] = rotc(o[6], neg(h), h);
    o[7] = rotc(o[7], neg(c1), s1);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[k] = e[k] + o[k];
        v[k + 8] = e[k] - o[k];
    }
}

// 32 = 2 x 16: the even and odd samples' 16-point DFTs, the odd ones rotated by
// w32^k = cos(pi k/16) - i sin(pi k/16), then one radix-2 combination.
template <typename T>
__device__ __forceinline__ void dft32(cx<T>* v) {
    const CK<T> c1 = ck<T>(0.98078528040323044913);  // cos(pi/16)
    const CK<T> s1 = ck<T>(0.19509032201612826785);  // sin(pi/16)
    const CK<T> c2 = ck<T>(0.92387953251128675613);  // cos(pi/8)
    const CK<T> s2 = ck<T>(0.38268343236508977173);  // sin(pi/8)
    const CK<T> c3 = ck<T>(0.83146961230254523708);  // cos(3pi/16)
    const CK<T> s3 = ck<T>(0.55557023301960222474);  // sin(3pi/16)
    const CK<T> h = ck<T>(0.70710678118654752440);   // cos(pi/4)
    cx<T> e[16], o[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        e[k] = v[2 * k];
        o[k] = v[2 * k + 1];
    }
    dft16(e);
    dft16(o);
    o[1] = rotc(o[1], c1, s1);
    o[2] = rotc(o[2], c2, s2);
    o[3] = rotc(o[3], c3, s3);
    o[4] = rotc(o[4], h, h);
    o[5] = rotc(o[5], s3, c3);
    o[6] = rotc(o[6], s2, c2);
    o[7] = rotc(o[7], s1, c1);
    o[8] = mul_mi(o[8]);
    o[9] = rotc(o[9], neg(s1), c1);
    o[10] = rotc(o[10], neg(s2), c2);
    o[11] = rotc(o[11], neg(s3), c3);
    o[12] = rotc(o[12], neg(h), h);
    o[13] = rotc(o[13], neg(c3), s3);
    o[14] = rotc(o[14], neg(c2), s2);
    o[15] = rotc(o[15], neg(c1), s1);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        v[k] = e[k] + o[k];
        v[k + 16] = e[k] - o[k];
    }
}

template <typename T>
__device__ __forceinline__ void dft3(cx<T>* v) {
    const CK<T> hs3 = ck<T>(0.86602540378443864676);  // sin(2 pi/3)
    const cx<T> t = v[1] + v[2];
    cx<T> m;  // v0 - t/2 (the halving is exact)
    if constexpr (sizeof(T) == 4)
        m = from_f2(__ffma2_rn(as_f2(t), make_float2(-0.5f, -0.5f), as_f2(v[0])));
    else
        m = mk<T>(fma(-0.5, t.x, v[0].x), fma(-0.5, t.y, v[0].y));
    if constexpr (sizeof(T) == 4) {
        const cx<T> d = kmulc(v[1] - v[2], hs3);
        v[0] = v[0] + t;
        v[1] = mk<T>(m.x + d.y, m.y - d.x);  // m - i d
        v[2] = mk<T>(m.x - d.y, m.y + d.x);  // m + i d
    } else {  // d = (v1 - v2) sin(2 pi/3), folded into explicit FMAs
        const cx<T> b = v[1] - v[2];
        v[0] = v[0] + t;
        v[1] = mk<T>(fma(b.y, hs3.hi, m.x), fma(-b.x, hs3.hi, m.y));
        v[2] = mk<T>(fma(-b.y, hs3.hi, m.x), fma(b.x, hs3.hi, m.y));
    }
}

template <typename T>
__device__ __forceinline__ void dft5(cx<T>* v) {
    const CK<T> c1 = ck<T>(0.30901699437494742410);   // cos(2 pi/5)
    const CK<T> c2 = ck<T>(-0.80901699437494742410);  // cos(4 pi/5)
    const CK<T> s1 = ck<T>(0.95105651629515357212);   // sin(2 pi/5)
    const CK<T> s2 = ck<T>(0.58778525229247312917);   // sin(4 pi/5)
    const cx<T> a1 = v[1] + v[4], a2 = v[2] + v[3];
    const cx<T> b1 = v[1] - v[4], b2 = v[2] - v[3];
    cx<T> p1, p2, q1, q2;
    if constexpr (sizeof(T) == 4) {
        p1 = v[0] + kmulc(a1, c1) + kmulc(a2, c2);
        p2 = v[0] + kmulc(a1, c2) + kmulc(a2, c1);
        q1 = kmulc(b1, s1) + kmulc(b2, s2);
        q2 = kmulc(b1, s2) - kmulc(b2, s1);
    } else {  // the same sums with the FMAs written out
        p1 = mk<T>(fma(a2.x, c2.hi, fma(a1.x, c1.hi, v[0].x)), fma(a2.y, c2.hi, fma(a1.y, c1.hi, v[0].y)));
        p2 = mk<T>(fma(a2.x, c1.hi, fma(a1.x, c2.hi, v[0].x)), fma(a2.y, c1.hi, fma(a1.y, c2.hi, v[0].y)));
        q1 = mk<T>(fma(b1.x, s1.hi, b2.x * s2.hi), fma(b1.y, s1.hi, b2.y * s2.hi));
        q2 = mk<T>(fma(b1.x, s2.hi, -(b2.x * s1.hi)), fma(b1.y, s2.hi, -(b2.y * s1.hi)));
    }
    v[0] = v[0] + a1 + a2;
    v[1] = mk<T>(p1.x + q1.y, p1.y - q1.x);  // p1 - i q1
    v[4] = mk<T>(p1.x - q1.y, p1.y + q1.x);  // p1 + i q1
    v[2] = mk<T>(p2.x + q2.y, p2.y - q2.x);
    v[3] = mk<T>(p2.x - q2.y, p2.y + q2.x);
}

// 6 = 2 x 3 and 10 = 2 x 5 by the prime-factor (Good-Thomas) mapping, which
// needs no twiddles between the factors: input n = (R n1 + 2 n2) mod 2R,
// output k = (R k1 + (R+1) k2) mod 2R for R = 3, 5 (CRT: R^{-1} = 1 mod 2,
// 2^{-1} mod 3 = 2, 2^{-1} mod 5 = 3).
template <typename T>
__device__ __forceinline__ void dft6(cx<T>* v) {
    cx<T> a[3] = {v[0], v[2], v[4]};
    cx<T> b[3] = {v[3], v[5], v[1]};
    dft3(a);
    dft3(b);
    v[0] = a[0] + b[0];
    v[3] = a[0] - b[0];
    v[4] = a[1] + b[1];
    v[1] = a[1] - b[1];
    v[2] = a[2] + b[2];
    v[5] = a[2] - b[2];
}

template <typename T>
__device__ __forceinline__ void dft10(cx<T>* v) {
    cx<T> a[5] = {v[0], v[2], v[4], v[6], v[8]};
    cx<T> b[5] = {v[5], v[7], v[9], v[1], v[3]};
    dft5(a);
    dft5(b);
    v[0] = a[0] + b[0];
    v[5] = a[0] - b[0];
    v[6] = a[1] + b[1];
    v[1] = a[1] - b[1];
    v[2] = a[2] + b[2];
    v[7] = a[2] - b[2];
    v[8] = a[3] + b[3];
    v[3] = a[3] - b[3];
    v[4] = a[4] + b[4];
    v[9] = a[4] - b[4];
}

// 12 = 4 x 3 by the same mapping: input n = (3 n1 + 4 n2) mod 12, output
// k = (9 k1 + 4 k2) mod 12 (3^{-1} = 3 mod 4, 4^{-1} = 1 mod 3).
template <typename T>
__device__ __forceinline__ void dft12(cx<T>* v) {
    cx<T> a[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
        cx<T> c[4];
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) c[n1] = v[(3 * n1 + 4 * n2) % 12];
        dft4(c);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) a[k1][n2] = c[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        dft3(a[k1]);
#pragma unroll
        for (int k2 = 0; k2 < 3; ++k2) v[(9 * k1 + 4 * k2) % 12] = a[k1][k2];
    }
}

// 20 = 4 x 5 by the same mapping: input n = (5 n1 + 4 n2) mod 20, output
// k = (5 k1 + 16 k2) mod 20 (5^{-1} = 1 mod 4, 4^{-1} = 4 mod 5).
template <typename T>
__device__ __forceinline__ void dft20(cx<T>* v) {
    cx<T> a[4][5];
#pragma unroll
    for (int n2 = 0; n2 < 5; ++n2) {
        cx<T> c[4];
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) c[n1] = v[(5 * n1 + 4 * n2) % 20];
        dft4(c);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) a[k1][n2] = c[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        dft5(a[k1]);
#pragma unroll
        for (int k2 = 0; k2 < 5; ++k2) v[(5 * k1 + 16 * k2) % 20] = a[k1][k2];
    }
}

template <typename T, int R>
__device__ __forceinline__ void dft(cx<T>* v) {
    if constexpr (R == 2) dft2(v);
    else if constexpr (R == 3) dft3(v);
    else if constexpr (R == 4) dft4(v);
    else if constexpr (R == 5) dft5(v);
    else if constexpr (R == 6) dft6(v);
    else if constexpr (R == 8) dft8(v);
    else if constexpr (R == 10) dft10(v);
    else if constexpr (R == 12) dft12(v);
    else if constexpr (R == 16) dft16(v);
    else if constexpr (R == 20) dft20(v);
    else if constexpr (R == 32) dft32(v);
}

// ---------------------------------------------------------------------------
// Geometry of one axis pass.  A CTA owns a tile of L lines (L a power of two)
// of one axis of length n.  Shared-memory address of element e of tile line l
// is l*ls + e*es: (ls, es) = (pitch, 1) for contiguous-axis tiles, (1, L) for
// strided-axis tiles.  Butterflies are numbered line-fastest (b -> l = b % L,
// j = b / L) so consecutive threads touch consecutive lines: conflict-free in
// both layouts (the contiguous layout pads its pitch to an odd length).
// ---------------------------------------------------------------------------
struct Geo {
    int n;         // axis length
    int L;         // lines per tile
    int lshift;    // log2(L)
    int nthreads;  // threads per CTA
    int ls, es;    // shared-memory strides
    int nst;       // Stockham stages
    int rad[kMaxStages];
    int Ns[kMaxStages];        // product of the previous radices
    int twstride[kMaxStages];  // n / (Ns * R)
    FastDiv fNs[kMaxStages];
    FastDiv fn;                // division by n
};

// One Stockham autosort stage of radix R (E. Bainville's formulation of the
// mixed-radix Stockham FFT): butterfly j of span Ns reads x[j + r n/R],
// applies twiddles w^{r k n/(Ns R)} (k = j mod Ns) and writes
// y[(j - k) R + k + r Ns].
//
// STREAM: source and destination are different memories (HBM -> tile or
// tile -> HBM), so each thread runs its butterflies start to finish.
// Otherwise the stage is in place in the tile: a thread reads all of its (up
// to B) butterflies into registers, the CTA synchronises, then writes.
template <typename T, int R, int B, bool STREAM, class LD, class ST>
__device__ __forceinline__ void stage(const Geo& g, int p, const cx<T>* __restrict__ tw, LD& ld,
                                      ST& st) {
    const int n = g.n;
    const int nR = n / R;
    const int nb = g.L * nR;
    const int Ns = g.Ns[p];
    const int tws = g.twstride[p];
    const FastDiv fNs = g.fNs[p];
    if constexpr (STREAM) {
        for (int b = (int)threadIdx.x; b < nb; b += g.nthreads) {
            const int l = b & (g.L - 1), j = b >> g.lshift;
            cx<T> v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = ld(l, j + r * nR);
            const int k = j - (int)fdiv((uint32_t)j, fNs) * Ns;
            if (Ns > 1) {
                const int t1 = k * tws;
#pragma unroll
                for (int r = 1; r < R; ++r) v[r] = v[r] * tw[r * t1];
            }
            dft<T, R>(v);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) st(l, base + r * Ns, v[r]);
        }
    } else {
        cx<T> v[B > 0 ? B : 1][R];
#pragma unroll
        for (int it = 0; it < B; ++it) {
            const int b = (int)threadIdx.x + it * g.nthreads;
            if (b < nb) {
                const int l = b & (g.L - 1), j = b >> g.lshift;
#pragma unroll
                for (int r = 0; r < R; ++r) v[it][r] = ld(l, j + r * nR);
                if (Ns > 1) {
                    const int k = j - (int)fdiv((uint32_t)j, fNs) * Ns;
                    const int t1 = k * tws;
#pragma unroll
                    for (int r = 1; r < R; ++r) v[it][r] = v[it][r] * tw[r * t1];
                }
                dft<T, R>(v[it]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < B; ++it) {
            const int b = (int)threadIdx.x + it * g.nthreads;
            if (b < nb) {
                const int l = b & (g.L - 1), j = b >> g.lshift;
                const int k = j - (int)fdiv((uint32_t)j, fNs) * Ns;
                const int base = (j - k) * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) st(l, base + r * Ns, v[it][r]);
            }
        }
    }
    __syncthreads();
}

template <typename T, int EPT, int R, class LD, class ST>
__device__ __forceinline__ void stage_any(const Geo& g, int p, bool stream, const cx<T>* tw, LD& ld,
                                          ST& st) {
    if (stream) stage<T, R, EPT / R, true>(g, p, tw, ld, st);
    else stage<T, R, EPT / R, false>(g, p, tw, ld, st);
}

// Full line FFT over the tile: stage 0 reads through ld0 (HBM when G_IN, the
// tile otherwise, with any element-wise pre-op), the last stage writes through
// stn (HBM when G_OUT, the tile otherwise, with any post-op); intermediate
// stages stay in the shared tile.  EPT bounds the elements a thread holds in
// an in-place stage (B = EPT / R butterflies).
template <typename T, int EPT, bool G_IN, bool G_OUT, class LD0, class STN>
__device__ __forceinline__ void fft_tile(const Geo& g, cx<T>* sm, const cx<T>* __restrict__ tw,
                                         LD0& ld0, STN& stn) {
    if (g.nst == 0) {  // length-1 axis: identity transform, element ops still apply
        for (int l = threadIdx.x; l < g.L; l += g.nthreads) stn(l, 0, ld0(l, 0));
        __syncthreads();
        return;
    }
    for (int p = 0; p < g.nst; ++p) {
        const bool first = p == 0, last = p == g.nst - 1;
        // stream only when the stage's source and destination cannot alias
        const bool stream = (first && G_IN && !last) || (last && G_OUT && !first);
        auto ld = [&](int l, int e) -> cx<T> {
            return first ? ld0(l, e) : sm[l * g.ls + e * g.es];
        };
        auto st = [&](int l, int e, cx<T> v) {
            if (last) stn(l, e, v);
            else sm[l * g.ls + e * g.es] = v;
        };
        switch (g.rad[p]) {
            case 2: stage_any<T, EPT, 2>(g, p, stream, tw, ld, st); break;
            case 3: stage_any<T, EPT, 3>(g, p, stream, tw, ld, st); break;
            case 4: stage_any<T, EPT, 4>(g, p, stream, tw, ld, st); break;
            case 5: stage_any<T, EPT, 5>(g, p, stream, tw, ld, st); break;
            case 8: stage_any<T, EPT, 8>(g, p, stream, tw, ld, st); break;
            case 16:
                if constexpr (EPT >= 16) stage_any<T, EPT, 16>(g, p, stream, tw, ld, st);
                break;
            default: break;
        }
    }
}

}  // namespace sesk
