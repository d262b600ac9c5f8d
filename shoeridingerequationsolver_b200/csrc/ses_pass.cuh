// Axis-pass kernels of the Strang step and the device table builders.
//
// A Strang step of the reference, V/2 . F^-1 K F . V/2 (core/src/propagator.ixx:110-119),
// is executed as a chain of axis passes over psi in HBM.  With the interior
// half-kicks merged into full kicks (reference GPU batch, solver/src/vk_engine.ixx:611-633):
//
//   3D step:  X[inv x, V*M, fwd x]  Y[fwd y]  Z[fwd z, K/N, inv z]  Y[inv y]
//   2D step:  X[inv x, V*M, fwd x]  Y[fwd y, K/N, inv y]
//   1D step:  X[V*M, fwd x, K/N, inv x]
//
// so one step reads and writes psi 4 / 2 / 1 times and reads the potential
// phase table once.  All diagonal factors (potential phase, absorbing mask,
// kinetic phase, 1/N) are applied in FP64 whatever the storage precision.
#pragma once

#include <type_traits>

#include "ses_fft.cuh"

namespace sesk {

constexpr int kEPTDev = 8;  // elements a thread holds per in-place Stockham stage

enum DiagKind : int { DG_NONE = 0, DG_HALF = 1, DG_FULL = 2 };

// Number of FP64 sums a k-space reduction produces:
// [0] sum|phi|^2  [1] sum k^2/(2m)|phi|^2  [2..4] sum k_a |phi|^2
constexpr int kRedK = 5;
// Real-space sums: [0] sum|psi|^2 [1] sum V|psi|^2 [2] sum_{x in [a,b)}|psi|^2
// [3..5] sum r_a|psi|^2 [6..8] sum r_a^2|psi|^2
constexpr int kRedR = 9;

struct Tables {
    const void* vtab;          // C128: cis(-V dt/2) as cx<double>; C64: cis(-V dt/2) - 1 as cx<float>
    const double* mask1[3];    // separable absorber profiles (all set or all null)
    const double* maskfull;    // non-separable absorber (nullable)
    const cx<double>* kd[3];   // per axis: cis(-k^2 dt/(2m)) - 1
    const double* kv[3];       // per axis: wavenumbers (fftfreq layout)
    // complex64 path: the same FP64-built per-axis tables rounded to FP32
    const float* mask1f[3];
    const cx<float>* kdf[3];
    double inv_mass;
    double kscale;             // 1/N, folded into the kinetic multiply
    // long 1D line (four-step layout N1 x N2); null / 0 otherwise
    const void* kfull;         // kinetic delta per stored k-space element (cx<T>)
    const void* tw4;           // W_N^{n1 k2} per element (cx<T>; complex64: FP32-rounded)
    const void* tw4l;          // complex64: FP32 remainder of tw4
    int long_n2;               // N2: stored element (k1, k2) is frequency k2 + N2 k1
    // dipole drive (drive.ixx:25-40): psi *= cis(-kick u), u = axis . r at cell (i, j, k),
    // r = origin + index * spacing; kick = 0 off
    double kick;
    double kax[3], korg[3], kh[3];
};

// complex64 phase multiplies in FP32 on the delta form: psi + psi*d, d = factor - 1.
__device__ __forceinline__ cx<float> add_mul(cx<float> p, cx<float> d) {  // p + p*d
    return mk<float>(fmaf(p.x, d.x, fmaf(-p.y, d.y, p.x)), fmaf(p.x, d.y, fmaf(p.y, d.x, p.y)));
}
// (1+a)(1+b) - 1 for the separable kinetic deltas
__device__ __forceinline__ cx<double> dmul1(cx<double> a, cx<double> b) { return a + b + a * b; }
__device__ __forceinline__ cx<float> dmul1f(cx<float> a, cx<float> b) {  // (1+a)(1+b) - 1
    return mk<float>(fmaf(a.x, b.x, fmaf(-a.y, b.y, a.x + b.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, a.y + b.y)));
}

template <typename T>
struct PassArgs {
    const cx<T>* src;
    cx<T>* dst;
    Geo g;
    int axis;  // 0 = x (contiguous lines), 1 = y, 2 = z
    int nx, ny, nz;
    long long nlines;
    // strided-axis addressing: line slot s -> base (s % nu) + (s / nu) * sw,
    // element stride se.  For the x axis: base = s * nx, se = 1.
    long long nu, sw, se;
    FastDiv fnu, fny, fnx;
    const cx<T>* tw;   // twiddles cis(-2 pi t / n), t < n (run-time plans)
    const cx<T>* stw;  // per-stage twiddle tables of a compiled plan (hi part)
    const cx<T>* stwl; // FP32: remainder (lo part) of the same tables
    // run-time parts of the pass program (the structure is the kernel's MODE)
    int d_load, d_mid, d_store;
    int m_load, m_mid, m_store;
    double out_scale;
    Tables tb;
    double* partials;
};

// Absorber value at flat index f, coordinates (i, j, k): m = mx[i] * (my[j] * mz[k]), in FP64.
template <typename T>
__device__ __forceinline__ double maskval(const Tables& tb, long long f, int i, int j, int k) {
    if (tb.maskfull) return tb.maskfull[f];
    return tb.mask1[0][i] * (tb.mask1[1][j] * tb.mask1[2][k]);
}

template <typename T>
__device__ __forceinline__ cx<T> apply_diag_tv(cx<T> v, int kind, cx<T> tab, int use_mask, double m);

// Dipole kick of cell (i, j, k): psi * cis(-kick (ax x + ay y + az z)), the phase in FP64;
// complex64 multiplies in FP32 on the delta form.  Out of line: the FP64 sincos
// stays out of the passes' register allocation, which only test kick != 0.
template <typename T>
__device__ __noinline__ cx<T> kick_apply(cx<T> v, double kick, double ax, double ay, double az, double x0,
                                         double y0, double z0, double hx, double hy, double hz, int i, int j,
                                         int k) {
    const double u = ax * (x0 + i * hx) + ay * (y0 + j * hy) + az * (z0 + k * hz);
    const double ang = -kick * u;
    if constexpr (sizeof(T) == 4) {
        double s2, c2;
        sincos(0.5 * ang, &s2, &c2);
        return add_mul(v, mk<float>((float)(-2.0 * s2 * s2), (float)(2.0 * s2 * c2)));
    } else {
        double s, c;
        sincos(ang, &s, &c);
        return v * mk<double>(c, s);
    }
}

template <typename T>
__device__ __forceinline__ cx<T> kick_mul(cx<T> v, const Tables& tb, int i, int j, int k) {
    if (tb.kick == 0.0) return v;
    return kick_apply<T>(v, tb.kick, tb.kax[0], tb.kax[1], tb.kax[2], tb.korg[0], tb.korg[1], tb.korg[2], tb.kh[0],
                         tb.kh[1], tb.kh[2], i, j, k);
}

// psi * (potential phase) * (mask) at flat index f, coordinates (i, j, k).
template <typename T>
__device__ __forceinline__ cx<T> apply_diag(cx<T> v, int kind, int use_mask, long long f, int i, int j,
                                            int k, const Tables& tb) {
    const cx<T> tab = kind != DG_NONE ? reinterpret_cast<const cx<T>*>(tb.vtab)[f] : v;
    return apply_diag_tv(v, kind, tab, use_mask, use_mask ? maskval<T>(tb, f, i, j, k) : 1.0);
}

// The same and the dipole kick: only the run-time-plan x pass carries the kick,
// which keeps its FP64 phase code out of the compiled passes' register budget
// (driven steps always run their x passes on those kernels).
template <typename T>
__device__ __forceinline__ cx<T> apply_diag_kick(cx<T> v, int kind, int use_mask, long long f, int i, int j,
                                                 int k, const Tables& tb) {
    return kick_mul(apply_diag(v, kind, use_mask, f, i, j, k, tb), tb, i, j, k);
}

// Same as apply_diag with the potential-table entry and mask value supplied
// by the caller (pipelined passes stage the table in shared memory).
//   DG_HALF: psi * h (* m)            h = cis(-V dt/2)
//   DG_FULL: (psi * h (* m)) * h      the kick between two steps, applied as the
//            half kick that ends one step (with the mask) followed by the half
//            kick that starts the next, in exactly that arithmetic -- so a run
//            of steps split into two calls gives the same bits as one call.
// The complex64 path multiplies in FP32 on the delta form psi + psi*d, d = h - 1.
template <typename T>
__device__ __forceinline__ cx<T> apply_diag_tv(cx<T> v, int kind, cx<T> tab, int use_mask, double m) {
    if constexpr (sizeof(T) == 4) {
        cx<float> p = v;
        if (kind != DG_NONE) p = add_mul(p, tab);
        if (use_mask) {  // p - p (1 - m): the FP32 rounding falls on the small 1 - m, not on m
            const float md = (float)(1.0 - m);
            p = mk<float>(fmaf(-p.x, md, p.x), fmaf(-p.y, md, p.y));
        }
        if (kind == DG_FULL) p = add_mul(p, tab);
        return p;
    } else {
        cx<double> p = v;
        if (kind != DG_NONE) p = p * tab;
        if (use_mask) p = mk<double>(p.x * m, p.y * m);
        if (kind == DG_FULL) p = p * tab;
        return p;
    }
}

// psi_k * K / N then conj (inverse FFT start); complex64: FP32 on the delta form.
__device__ __forceinline__ cx<float> kinetic_conj_f(cx<float> v, cx<float> d, double kscale) {
    return cconj(scale_d(add_mul(v, d), kscale));
}

template <typename T>
__device__ __forceinline__ cx<T> kinetic_apply(cx<T> v, cx<double> dother, const cx<double>* kda64,
                                               const cx<float>* kda32, int pos, double kscale) {
    if constexpr (sizeof(T) == 4) return kinetic_conj_f(v, dmul1f(narrow<float>(dother), kda32[pos]), kscale);
    else return kinetic_conj(v, dmul1(dother, kda64[pos]), kscale);
}


// psi_k * K(k) / N followed by the conjugation that starts the inverse FFT.
template <typename T>
__device__ __forceinline__ cx<T> kinetic_conj(cx<T> v, cx<double> d, double kscale) {
    cx<double> p = widen(v);
    p = p + p * d;
    return narrow<T>(mk<double>(p.x * kscale, -p.y * kscale));
}

// Kinetic multiply from a per-element delta table (long 1D lines).
template <typename T>
__device__ __forceinline__ cx<T> kinetic_full(cx<T> v, const void* kfull, long long idx, double kscale) {
    if constexpr (sizeof(T) == 4)
        return kinetic_conj_f(v, reinterpret_cast<const cx<float>*>(kfull)[idx], kscale);
    else
        return kinetic_conj(v, reinterpret_cast<const cx<double>*>(kfull)[idx], kscale);
}

// Kinetic multiply of element `pos` of an axis whose other two axes give the
// FP64 delta `dother`: complex128 -> FP64; complex64 -> FP32 delta form with
// the FP32-rounded tables (kda64 / kda32 are the axis's FP64 / FP32 deltas).
template <typename T>
__device__ __forceinline__ cx<T> kinetic_apply(cx<T> v, cx<double> dother, const cx<double>* kda64,
                                               const cx<float>* kda32, int pos, double kscale);

// kinetic_apply with the axis's delta at this element fetched beforehand (kde:
// the FP64 delta for complex128, the FP32-rounded one for complex64): the same
// arithmetic, so passes that prefetch their tables give the same bits.
template <typename T>
using KinDelta = typename std::conditional<sizeof(T) == 4, cx<float>, cx<double>>::type;

template <typename T>
__device__ __forceinline__ cx<T> kinetic_apply_pre(cx<T> v, cx<double> dother, KinDelta<T> kde, double kscale) {
    if constexpr (sizeof(T) == 4) return kinetic_conj_f(v, dmul1f(narrow<float>(dother), kde), kscale);
    else return kinetic_conj(v, dmul1(dother, kde), kscale);
}

template <typename T>
__device__ __forceinline__ KinDelta<T> kin_delta(const cx<double>* kda64, const cx<float>* kda32, int pos) {
    if constexpr (sizeof(T) == 4) return kda32[pos];
    else return kda64[pos];
}

template <int NR>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NR], double* out) {
    __shared__ double red[32][NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
        double v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        acc[q] = v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NR; ++q) red[warp][q] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x < NR) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
        out[(size_t)blockIdx.x * NR + threadIdx.x] = s;
    }
}

// Accumulate k-space sums of one element: axis wavenumber ka, other two
// wavenumbers (kb, kc) in fixed axis slots.
__device__ __forceinline__ void acc_k(double (&acc)[kRedK], double w, const double* k3,
                                      double inv_mass) {
    const double ksq = k3[0] * k3[0] + k3[1] * k3[1] + k3[2] * k3[2];
    acc[0] += w;
    acc[1] += 0.5 * ksq * inv_mass * w;
    acc[2] += k3[0] * w;
    acc[3] += k3[1] * w;
    acc[4] += k3[2] * w;
}

// ---------------------------------------------------------------------------
// Pass programs.  Each program is its own kernel so every kernel holds at most
// two tile FFTs (register allocation stays local; no run-time program flags in
// the butterfly loops).
// ---------------------------------------------------------------------------
enum XMode : int {
    XM_FWD = 0,     // fwd x                                   (fft3 surface, energy copy)
    XM_INV = 1,     // inv x, scaled                           (fft3 surface)
    XM_START = 2,   // V/2, fwd x                              (first step of a batch)
    XM_MID = 3,     // inv x, V (* M), fwd x                   (between steps)
    XM_END = 4,     // inv x, V/2 (* M)                        (end of a batch)
    XM_1D = 5,      // V/2 or V (* M), fwd x, K/N, inv x, [V/2 (* M)]   (x only axis)
    XM_REDUCE = 6   // fwd x, k-space sums                     (1D energy)
};
// Strided programs.  SM_TW_* are the strided halves of a long 1D line run as a
// four-step transform (line of N = N1 N2 points stored as N1 x N2, x fastest):
// the y pass is the length-N2 transform with the twiddles W_N^{n1 k2} on its
// k-space side, the x pass (XM_1D) the length-N1 transform with the kinetic
// phase of frequency k2 + N2 k1 between forward and inverse.
enum SModeK : int {
    SM_FWD = 0,       // fwd y/z
    SM_INV = 1,       // inv y/z, scaled
    SM_FUSED = 2,     // fwd, K/N, inv                 (last axis)
    SM_REDUCE = 3,    // fwd, k-space sums
    SM_TW_START = 4,  // [V/2 (* M)], fwd y, * W        (long line: batch start, or k-space copy)
    SM_TW_MID = 5,    // * conj W, inv y, V (* M), fwd y, * W   (between steps)
    SM_TW_END = 6     // * conj W, inv y, V/2 (* M)     (batch end)
};
constexpr int kSModes = 7;

// ---------------------------------------------------------------------------
// Contiguous-axis (x) pass.  Tile = L consecutive x-lines, loaded and stored
// with coalesced accesses; shared layout [l][e] with an odd pitch.
// ---------------------------------------------------------------------------
// Programmatic dependent launch: a pass kernel may be launched while the
// previous kernel of its stream drains; it waits here, before touching any
// field or argument table, until that kernel has completed and its writes are
// visible (a no-op for a normal launch).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename T, int MODE>
__global__ void __launch_bounds__(512, 1) xpass_kernel(const PassArgs<T> a) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ Geo g;  // stage tables are indexed at run time: keep them out of parameter space
    if (threadIdx.x == 0) g = a.g;
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    const int n = a.g.n, L = a.g.L;
    const long long m0 = (long long)blockIdx.x * L;
    const int tile = L * n;
    const int tid = threadIdx.x, nt = blockDim.x;
    constexpr bool kDiagLoad = MODE == XM_START || MODE == XM_1D;
    constexpr bool kDiagStore = MODE == XM_END || MODE == XM_1D;

    // load (coalesced), optional real-space diagonal
    for (int idx = tid; idx < tile; idx += nt) {
        const int l = (int)fdiv((uint32_t)idx, a.g.fn), e = idx - l * n;
        const long long m = m0 + l;
        cx<T> v = mk<T>((T)0, (T)0);
        if (m < a.nlines) {
            const long long f = m * n + e;
            v = a.src[f];
            if constexpr (kDiagLoad) {
                if (a.d_load != DG_NONE || a.m_load) {
                    const int k = (int)fdiv((uint32_t)m, a.fny);
                    const int j = (int)(m - (long long)k * a.ny);
                    v = apply_diag_kick(v, a.d_load, a.m_load, f, e, j, k, a.tb);
                }
            }
        }
        sm[l * a.g.ls + e] = v;
    }
    __syncthreads();

    auto lds = [&](int l, int e) -> cx<T> { return sm[l * g.ls + e]; };
    auto sts = [&](int l, int e, cx<T> v) { sm[l * g.ls + e] = v; };

    if constexpr (MODE == XM_INV || MODE == XM_MID || MODE == XM_END) {
        auto ldc = [&](int l, int e) -> cx<T> { return cconj(sm[l * g.ls + e]); };
        auto stc = [&](int l, int e, cx<T> v) {
            sm[l * g.ls + e] = MODE == XM_INV ? scale_d(cconj(v), a.out_scale) : cconj(v);
        };
        fft_tile<T, kEPTDev, false, false>(g, sm, a.tw, ldc, stc);
    }
    if constexpr (MODE == XM_MID) {
        if (a.d_mid != DG_NONE || a.m_mid) {
            for (int idx = tid; idx < tile; idx += nt) {
                const int l = (int)fdiv((uint32_t)idx, g.fn), e = idx - l * n;
                const long long m = m0 + l;
                if (m < a.nlines) {
                    const int k = (int)fdiv((uint32_t)m, a.fny);
                    const int j = (int)(m - (long long)k * a.ny);
                    sm[l * g.ls + e] =
                        apply_diag_kick(sm[l * g.ls + e], a.d_mid, a.m_mid, m * n + e, e, j, k, a.tb);
                }
            }
            __syncthreads();
        }
    }
    if constexpr (MODE == XM_FWD || MODE == XM_START || MODE == XM_MID) {
        fft_tile<T, kEPTDev, false, false>(g, sm, a.tw, lds, sts);
    }
    if constexpr (MODE == XM_1D) {
        // x is the only transformed axis: fwd, K/N, inverse, all in the tile
        auto stk = [&](int l, int e, cx<T> v) {
            const long long m0l = m0 + l;
            const long long m = m0l < a.nlines ? m0l : 0;
            const int k = (int)fdiv((uint32_t)m, a.fny);
            const int j = (int)(m - (long long)k * a.ny);
            sm[l * g.ls + e] = kinetic_apply(v, dmul1(a.tb.kd[1][j], a.tb.kd[2][k]), a.tb.kd[0], a.tb.kdf[0],
                                             e, a.tb.kscale);
        };
        fft_tile<T, kEPTDev, false, false>(g, sm, a.tw, lds, stk);
        auto stc = [&](int l, int e, cx<T> v) { sm[l * g.ls + e] = cconj(v); };
        fft_tile<T, kEPTDev, false, false>(g, sm, a.tw, lds, stc);
    }
    if constexpr (MODE == XM_REDUCE) {
        double acc[kRedK] = {0, 0, 0, 0, 0};
        auto str = [&](int l, int e, cx<T> v) {
            const long long m = m0 + l;
            if (m < a.nlines) {
                const int k = (int)fdiv((uint32_t)m, a.fny);
                const int j = (int)(m - (long long)k * a.ny);
                const double k3[3] = {a.tb.kv[0][e], a.tb.kv[1][j], a.tb.kv[2][k]};
                const cx<double> p = widen(v);
                acc_k(acc, p.x * p.x + p.y * p.y, k3, a.tb.inv_mass);
            }
        };
        fft_tile<T, kEPTDev, false, false>(g, sm, a.tw, lds, str);
        block_reduce_store<kRedK>(acc, a.partials);
        return;
    }

    // store (coalesced), optional real-space diagonal
    if constexpr (MODE != XM_REDUCE) for (int idx = tid; idx < tile; idx += nt) {
        const int l = (int)fdiv((uint32_t)idx, g.fn), e = idx - l * n;
        const long long m = m0 + l;
        if (m < a.nlines) {
            const long long f = m * n + e;
            cx<T> v = sm[l * g.ls + e];
            if constexpr (kDiagStore) {
                if (a.d_store != DG_NONE || a.m_store) {
                    const int k = (int)fdiv((uint32_t)m, a.fny);
                    const int j = (int)(m - (long long)k * a.ny);
                    v = apply_diag_kick(v, a.d_store, a.m_store, f, e, j, k, a.tb);
                }
            }
            a.dst[f] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Strided-axis (y or z) pass.  Tile = L line slots whose first elements are
// consecutive in memory, so every element load/store of a warp is a
// contiguous run.  Stage 0 reads HBM directly and the last stage writes HBM
// directly; intermediate stages use the shared tile ([e][l] layout).
// ---------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(512, 1) spass_kernel(const PassArgs<T> a) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ Geo g;  // stage tables are indexed at run time: keep them out of parameter space
    if (threadIdx.x == 0) g = a.g;
    const int n = a.g.n, L = a.g.L;
    cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
    // per-line data after the tile, 16-byte aligned: kinetic delta of the two
    // other axes, their wavenumbers, and the line's base offset in psi
    cx<double>* dother =
        reinterpret_cast<cx<double>*>(smraw + (((size_t)L * n * sizeof(cx<T>) + 15) & ~(size_t)15));
    double* kq = reinterpret_cast<double*>(dother + L);
    long long* lbase = reinterpret_cast<long long*>(kq + 2 * L);
    const long long s0 = (long long)blockIdx.x * L;
    constexpr bool kLineInfo = MODE == SM_FUSED || MODE == SM_REDUCE;
    // the two other axes, in increasing order: y-pass -> (x, z), z-pass -> (x, y)
    const bool ypass = a.axis == 1;
    const cx<double>* kd1 = a.tb.kd[0];
    const cx<double>* kd2 = ypass ? a.tb.kd[2] : a.tb.kd[1];
    const cx<double>* kda = ypass ? a.tb.kd[1] : a.tb.kd[2];
    const double* kv1 = a.tb.kv[0];
    const double* kv2 = ypass ? a.tb.kv[2] : a.tb.kv[1];
    const double* kva = ypass ? a.tb.kv[1] : a.tb.kv[2];

    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const long long s = s0 + l;
        long long base = -1;
        int c1 = 0, c2 = 0;
        if (s < a.nlines) {
            const long long w = (long long)fdiv((uint32_t)s, a.fnu);
            const long long u = s - w * a.nu;
            base = u + w * a.sw;
            if (ypass) {  // lines (i, k)
                c1 = (int)u;
                c2 = (int)w;
            } else {  // z: lines (i, j), u = i + nx j
                c2 = (int)fdiv((uint32_t)u, a.fnx);
                c1 = (int)(u - (long long)c2 * a.nx);
            }
        }
        lbase[l] = base;
        if constexpr (kLineInfo) {
            dother[l] = dmul1(kd1[c1], kd2[c2]);
            kq[2 * l] = kv1[c1];
            kq[2 * l + 1] = kv2[c2];
        }
    }
    __syncthreads();

    const long long se = a.se;
    auto ldg = [&](int l, int e) -> cx<T> {
        const long long b = lbase[l];
        return b >= 0 ? a.src[b + e * se] : mk<T>((T)0, (T)0);
    };
    auto stg = [&](int l, int e, cx<T> v) {
        const long long b = lbase[l];
        if (b >= 0) a.dst[b + e * se] = v;
    };

    if constexpr (MODE == SM_FWD) {
        fft_tile<T, kEPTDev, true, true>(g, sm, a.tw, ldg, stg);
    } else if constexpr (MODE == SM_INV) {
        auto ldc = [&](int l, int e) -> cx<T> { return cconj(ldg(l, e)); };
        auto stc = [&](int l, int e, cx<T> v) { stg(l, e, scale_d(cconj(v), a.out_scale)); };
        fft_tile<T, kEPTDev, true, true>(g, sm, a.tw, ldc, stc);
    } else if constexpr (MODE == SM_FUSED) {
        auto stk = [&](int l, int e, cx<T> v) {
            sm[l * g.ls + e * g.es] = kinetic_apply(v, dother[l], kda, ypass ? a.tb.kdf[1] : a.tb.kdf[2], e,
                                                    a.tb.kscale);
        };
        fft_tile<T, kEPTDev, true, false>(g, sm, a.tw, ldg, stk);
        auto lds = [&](int l, int e) -> cx<T> { return sm[l * g.ls + e * g.es]; };
        auto stc = [&](int l, int e, cx<T> v) { stg(l, e, cconj(v)); };
        fft_tile<T, kEPTDev, false, true>(g, sm, a.tw, lds, stc);
    } else {  // SM_REDUCE
        double acc[kRedK] = {0, 0, 0, 0, 0};
        auto str = [&](int l, int e, cx<T> v) {
            if (lbase[l] >= 0) {
                const double ka = kva[e], kb = kq[2 * l + 1];
                const double k3[3] = {kq[2 * l], ypass ? ka : kb, ypass ? kb : ka};
                const cx<double> p = widen(v);
                acc_k(acc, p.x * p.x + p.y * p.y, k3, a.tb.inv_mass);
            }
        };
        fft_tile<T, kEPTDev, true, true>(g, sm, a.tw, ldg, str);
        block_reduce_store<kRedK>(acc, a.partials);
    }
}

// ---------------------------------------------------------------------------
// Real-space observables: grid-stride FP64 sums, one partial row per CTA,
// fixed grid -> deterministic.
// ---------------------------------------------------------------------------
struct ObsArgs {
    long long N;
    int nx, ny;
    FastDiv fnx, fny;
    double x0, hx, y0, hy, z0, hz;
    double xlo, xhi;
};

template <typename T>
__global__ void __launch_bounds__(256) obs_real_kernel(const cx<T>* __restrict__ psi,
                                                       const double* __restrict__ V, ObsArgs o,
                                                       double* partials) {
    double acc[kRedR];
#pragma unroll
    for (int q = 0; q < kRedR; ++q) acc[q] = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < o.N; idx += stride) {
        const long long line = idx / o.nx;  // 64-bit: N may exceed 2^31
        const int i = (int)(idx - line * o.nx);
        const long long k = line / o.ny;
        const int j = (int)(line - k * o.ny);
        const cx<double> p = widen(psi[idx]);
        const double w = p.x * p.x + p.y * p.y;
        const double x = o.x0 + i * o.hx, y = o.y0 + j * o.hy, z = o.z0 + (double)k * o.hz;
        acc[0] += w;
        acc[1] += V[idx] * w;
        if (x >= o.xlo && x < o.xhi) acc[2] += w;
        acc[3] += x * w;
        acc[4] += y * w;
        acc[5] += z * w;
        acc[6] += x * x * w;
        acc[7] += y * y * w;
        acc[8] += z * z * w;
    }
    block_reduce_store<kRedR>(acc, partials);
}

template <typename S, typename D>
__global__ void convert_kernel(const cx<S>* __restrict__ src, cx<D>* dst, long long N) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        dst[i] = mk<D>((D)src[i].x, (D)src[i].y);
    }
}

}  // namespace sesk
