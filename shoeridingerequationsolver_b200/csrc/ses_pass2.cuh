// Compiled-plan axis passes: the line FFT of length N = R0*R1*R2 runs with
// each thread holding E elements of its line in registers.  Butterfly j of a
// stage belongs to thread q = j mod (N/E); between stages the elements are
// exchanged through shared memory.  On the contiguous x axis a line lives
// inside one warp (exchange = __syncwarp); on the strided y/z axes consecutive
// threads own consecutive lines (coalesced) and exchanges are CTA-wide.
//
// The last stage of an FFT leaves thread q holding positions
// q + (N/E) b + r N/R_last, exactly the inputs the FIRST stage of an FFT with
// the reversed radix order needs, so the two FFTs of a fused pass (inverse
// then forward, or forward then inverse) run back to back in registers.
#pragma once

#include "ses_pass.cuh"

namespace sesk {

// PK (complex64): hi points to the interleaved table {h.x, h.y, l.x, l.y} per
// entry (the shared-memory copy), read with one 16-byte load; lo is unused.
template <typename T, bool PK = false>
__device__ __forceinline__ cx<T> twmul(cx<T> v, const cx<T>* __restrict__ hi,
                                       const cx<T>* __restrict__ lo, int idx) {
    if constexpr (sizeof(T) == 4) {  // compensated: v * (h + l), l = FP32 remainder of the FP64 twiddle
        cx<T> h, l;
        if constexpr (PK) {
            const float4 t = reinterpret_cast<const float4*>(hi)[idx];
            h = mk<float>(t.x, t.y);
            l = mk<float>(t.z, t.w);
        } else {
            h = hi[idx];
            l = lo[idx];
        }
        return mk<T>(fmaf(v.x, h.x, fmaf(-v.y, h.y, fmaf(v.x, l.x, -v.y * l.y))),
                     fmaf(v.x, h.y, fmaf(v.y, h.x, fmaf(v.x, l.y, v.y * l.x))));
    } else {
        return v * hi[idx];
    }
}

// 16-byte asynchronous global -> shared copies (cp.async, L2 only), used to fetch
// the potential-table rows of a tile while its first FFT runs.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Four-step twiddle W_N^{n1 k2} of element f (long 1D lines).
template <typename T>
__device__ __forceinline__ cx<T> tw4_mul(cx<T> v, const Tables& tb, long long f) {
    return twmul(v, reinterpret_cast<const cx<T>*>(tb.tw4), reinterpret_cast<const cx<T>*>(tb.tw4l), (int)f);
}

// One Stockham stage of radix R after NS points per butterfly group: twiddle
// then DFT of each of the thread's E/R butterflies.  A stage's table holds
// R x NS entries, w^{r k N/(NS R)} at [OFF + r*NS + k].
template <typename T, int N, int E, int TL, int R, int NS, int OFF, bool PK = false>
__device__ __forceinline__ void rstage(cx<T> (&v)[E], int q, const cx<T>* __restrict__ twh,
                                       const cx<T>* __restrict__ twl) {
    constexpr int B = E / R;
#pragma unroll
    for (int b = 0; b < B; ++b) {
        if constexpr (NS > 1) {
            const int k = (q + TL * b) % NS;
#pragma unroll
            for (int r = 1; r < R; ++r) v[b * R + r] = twmul<T, PK>(v[b * R + r], twh, twl, OFF + r * NS + k);
        }
        dft<T, R>(&v[b * R]);
    }
}

template <typename T, int N, int E, int TL, int RP, int NSP, int RN, class X>
__device__ __forceinline__ void rexchange(cx<T> (&v)[E], int q, X& x) {
#pragma unroll
    for (int b = 0; b < E / RP; ++b) {
        const int j = q + TL * b;
        const int k = j % NSP;
        const int base = (j - k) * RP + k;
#pragma unroll
        for (int r = 0; r < RP; ++r) x.put(base + r * NSP, v[b * RP + r]);
    }
    x.sync();
#pragma unroll
    for (int b = 0; b < E / RN; ++b) {
        const int j = q + TL * b;
#pragma unroll
        for (int r = 0; r < RN; ++r) v[b * RN + r] = x.get(j + r * (N / RN));
    }
    x.sync();
}

// Forward FFT of plan (R0, R1, R2) (R = 1: stage absent), tables of that plan.
// In:  v[b*R0 + r] = x[q + TL b + r N/R0].   Out: v[b*RL + r] = X[q + TL b + r N/RL].
template <typename T, int N, int E, int R0, int R1, int R2, int TOFF, bool PK = false, class X>
__device__ __forceinline__ void rfft(cx<T> (&v)[E], int q, const cx<T>* twh, const cx<T>* twl, X& x) {
    constexpr int TL = N / E;
    rstage<T, N, E, TL, R0, 1, TOFF, PK>(v, q, twh, twl);
    if constexpr (R1 > 1) {
        rexchange<T, N, E, TL, R0, 1, R1>(v, q, x);
        rstage<T, N, E, TL, R1, R0, TOFF + R0, PK>(v, q, twh, twl);
    }
    if constexpr (R2 > 1) {
        rexchange<T, N, E, TL, R1, R0, R2>(v, q, x);
        rstage<T, N, E, TL, R2, R0 * R1, TOFF + R0 + R1 * R0, PK>(v, q, twh, twl);
    }
}

template <int R0, int R1, int R2>
struct PlanShape {
    static constexpr int last = R2 > 1 ? R2 : (R1 > 1 ? R1 : R0);
    // reversed order (R2, R1, R0) without absent stages
    static constexpr int v0 = R2 > 1 ? R2 : (R1 > 1 ? R1 : R0);
    static constexpr int v1 = R2 > 1 ? R1 : (R1 > 1 ? R0 : 1);
    static constexpr int v2 = R2 > 1 ? R0 : 1;
    static constexpr int fwd_tables = R0 + (R1 > 1 ? R1 * R0 : 0) + (R2 > 1 ? R2 * R0 * R1 : 0);
    static constexpr int rev_tables = v0 + (v1 > 1 ? v1 * v0 : 0) + (v2 > 1 ? v2 * v0 * v1 : 0);
    static constexpr int tables = fwd_tables + rev_tables;
};

// Shared-memory copy of a plan's stage twiddles (forward then reversed tables)
// for persistent kernels: loaded once per CTA, so the FFT stages read twiddles at
// shared-memory latency and the tables of many instances do not compete for L1.
// complex64 entries are interleaved {h.x, h.y, l.x, l.y} (hi part and FP32
// remainder), 16 bytes each, read by twmul<float, true> with one load.  The copy
// must start on a 16-byte boundary.
template <typename T, int R0, int R1, int R2>
struct TwStage {
    static constexpr int count = PlanShape<R0, R1, R2>::tables;
    static constexpr size_t bytes = (size_t)count * sizeof(cx<T>) * (sizeof(T) == 4 ? 2 : 1);
    static __device__ __forceinline__ void load(cx<T>* dst, const cx<T>* hi, const cx<T>* lo) {
        for (int i = threadIdx.x; i < count; i += blockDim.x) {
            if constexpr (sizeof(T) == 4)
                reinterpret_cast<float4*>(dst)[i] = make_float4(hi[i].x, hi[i].y, lo[i].x, lo[i].y);
            else
                dst[i] = hi[i];
        }
    }
    // the twl argument that goes with the copy (unused by the interleaved reads)
    static __device__ __forceinline__ const cx<T>* lo_of(const cx<T>* dst) { return dst; }
};

// FFT with the plan's own order (tables at 0) or reversed order (tables after).
// PK: the tables are the interleaved shared-memory copy of TwStage.
template <typename T, int N, int E, int R0, int R1, int R2, bool REV, bool PK = false, class X>
__device__ __forceinline__ void rfft_plan(cx<T> (&v)[E], int q, const cx<T>* twh, const cx<T>* twl,
                                          X& x) {
    using S = PlanShape<R0, R1, R2>;
    if constexpr (!REV) rfft<T, N, E, R0, R1, R2, 0, PK>(v, q, twh, twl, x);
    else rfft<T, N, E, S::v0, S::v1, S::v2, S::fwd_tables, PK>(v, q, twh, twl, x);
}

// Padded line in shared memory: element pos at pos + PM * (pos >> SH).
template <typename T, int SH, int PM>
struct XchWarp {
    cx<T>* p;
    __device__ __forceinline__ void put(int pos, cx<T> v) { p[pos + PM * (pos >> SH)] = v; }
    __device__ __forceinline__ cx<T> get(int pos) const { return p[pos + PM * (pos >> SH)]; }
    __device__ __forceinline__ void sync() { __syncwarp(); }
};

// Padding of the contiguous pass's lines: the layouts with the fewest shared-memory
// wavefronts over every exchange of the plan (forward and reversed orders, both
// half-warps of 64-bit accesses), found by modelling the access patterns.
template <int N, int E>
struct XPad {
    static constexpr bool k160e40 = N == 160 && E == 40;  // plan 20 x 8
    static constexpr int SH = N == 160 || N == 96 || N == 64 ? 3 : (N == 48 || N == 32 ? 2 : 4);
    static constexpr int PM = N == 48 ? 3 : 1;
    static constexpr int LPAD = k160e40 ? 0 : (N == 160 ? 4 : (N == 96 ? 12 : (N == 32 ? 4 : 0)));
    static constexpr int PITCH = N + PM * (N >> SH) + LPAD;
};

template <typename T, int L>
struct XchCta {
    cx<T>* p;
    int l;
    __device__ __forceinline__ void put(int pos, cx<T> v) { p[pos * L + l] = v; }
    __device__ __forceinline__ cx<T> get(int pos) const { return p[pos * L + l]; }
    __device__ __forceinline__ void sync() { __syncthreads(); }
};

template <typename T>
__device__ __forceinline__ cx<T> czero() {
    return mk<T>((T)0, (T)0);
}

// ---------------------------------------------------------------------------
// Contiguous-axis (x) pass, compiled plan.  4 warps per CTA; a warp owns
// 32/(N/E) lines.  Modes as in XMode.
// ---------------------------------------------------------------------------
// Warps per contiguous-pass CTA: up to 4, within 48 KB of static shared memory.
template <typename T, int N, int E>
struct XShape {
    static constexpr int TL = N / E;
    static constexpr int LPW = 32 / TL;          // lines per warp
    static constexpr int PITCH = XPad<N, E>::PITCH;
    static constexpr int per_warp = LPW * PITCH * (int)sizeof(cx<T>);
    static constexpr int NW = (48 * 1024) / per_warp >= 4 ? 4 : ((48 * 1024) / per_warp < 1 ? 1 : (48 * 1024) / per_warp);
    // CTAs per SM the register allocation is sized for: 20 or more elements per
    // thread need more than the 128 registers of four 4-warp CTAs
    static constexpr int MINB = E >= 40 ? 2 : (E >= 20 ? 3 : 4);
    // Pitch of the staged potential-table rows of the batched pass: a
    // half-warp reads 16/TL lines at the same positions, each line covering 2 TL
    // banks with 64-bit elements; a pitch of TL mod 16 puts those lines on
    // disjoint banks (a pitch of N, a multiple of 16, puts them on the same).
    // The pitch stays even: rows are filled by 16-byte cp.async copies, whose
    // shared-memory address must be 16-byte aligned (one thread per line, TL = 1,
    // takes pitch 2 mod 16 instead of 1).
    static constexpr int RTL = TL < 2 ? 2 : TL;
    static constexpr int RPITCH = TL >= 16 ? N : N + ((RTL - N % 16) % 16 + 16) % 16;
    static_assert(RPITCH % 2 == 0, "staged rows start on 16-byte boundaries");
};

// Body of the contiguous pass for CTA tile `blk` (NW * LPW lines); `a` is the
// kernel parameter (single field) or an entry of a per-instance array in
// global memory (batched passes).
// vt (optional): shared memory for this CTA's potential-table rows (NW * LPW
// lines of N entries); the between-steps and batch-end passes then fetch the
// rows asynchronously at the start of the tile and read them after the first FFT.
// FASTKICK (between-steps pass of the batched kernel only): the pass applies the
// full kick with a separable absorber from staged table and profile rows -- the
// run-time tests of the general path (table kind, mask kind, staged rows) are
// resolved at compile time, leaving straight-line code per element.
template <typename T, int MODE, int N, int E, int R0, int R1, int R2, bool FASTKICK = false, bool PK = false,
          class A>
__device__ __forceinline__ void xpass2_body(const A& a, long long blk, cx<T>* xb, const cx<T>* twh,
                                            const cx<T>* twl, cx<T>* vt = nullptr) {
    static_assert(!FASTKICK || MODE == XM_MID, "the fast kick is the between-steps pass");
    using XS = XShape<T, N, E>;
    constexpr int TL = XS::TL;
    constexpr int LPW = XS::LPW;
    constexpr int PITCH = XS::PITCH;
    constexpr int NW = XS::NW;
    using S = PlanShape<R0, R1, R2>;
    // The batch-start pass runs its forward FFT in the reversed radix order, the
    // order of the second FFT of the between-steps pass, so that a batch end
    // followed by a batch start computes what one between-steps pass computes.
    constexpr bool kRev = MODE == XM_START;
    constexpr int RF = kRev ? S::last : R0;  // radix of the first FFT's first stage
    constexpr int RL = kRev ? R0 : S::last;  // radix of its last stage (output layout)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lw = lane / TL, q = lane % TL;
    const long long m = (blk * NW + warp) * LPW + lw;
    const bool valid = m < a.nlines;
    const long long mc = valid ? m : 0;
    const int kz = (int)fdiv((uint32_t)mc, a.fny);
    const int jy = (int)(mc - (long long)kz * a.ny);
    XchWarp<T, XPad<N, E>::SH, XPad<N, E>::PM> x{xb + (warp * LPW + lw) * PITCH};
    const cx<T>* src = a.src + mc * N;
    cx<T>* dst = a.dst + mc * N;
    cx<T> v[E];
    constexpr bool kTabLate = MODE == XM_MID || MODE == XM_END;  // table used after the first FFT
    constexpr int RP = XS::RPITCH;
    cx<T>* vrow = vt ? vt + (size_t)(warp * LPW + lw) * RP : nullptr;
    const double* mfull = a.tb.maskfull;
    const double* mx = a.tb.mask1[0];
    // this warp's copy of the x profile of a separable absorber (N doubles after the
    // table rows of all warps), staged with the rows by the passes that use it
    double* ms = vt ? reinterpret_cast<double*>(vt + (size_t)NW * LPW * RP) + (size_t)warp * N : nullptr;
    // load the first FFT's inputs (coalesced along the line)
    constexpr bool kConjIn = MODE == XM_INV || MODE == XM_MID || MODE == XM_END;
#pragma unroll
    for (int b = 0; b < E / RF; ++b)
#pragma unroll
        for (int r = 0; r < RF; ++r) {
            const int pos = q + TL * b + r * (N / RF);
            cx<T> e = valid ? src[pos] : czero<T>();
            if constexpr (MODE == XM_START || MODE == XM_1D) {
                if (a.d_load != DG_NONE || a.m_load)
                    e = apply_diag(e, a.d_load, a.m_load, mc * N + pos, pos, jy, kz, a.tb);
            }
            v[b * RF + r] = kConjIn ? cconj(e) : e;
        }
    if constexpr (kTabLate) {
        const bool want = FASTKICK || (MODE == XM_MID ? a.d_mid != DG_NONE : a.d_store != DG_NONE);
        const bool wantm = FASTKICK || ((MODE == XM_MID ? a.m_mid : a.m_store) && !mfull && mx);
        if (FASTKICK || (vt && (want || wantm))) {  // this warp's rows, 16-byte chunks spread over the lanes
            __syncwarp();  // the previous tile's reads of these rows are done
            if (want) {  // line by line, lane-strided 16-byte chunks: constant offsets per copy
                constexpr int CH = N * (int)sizeof(cx<T>) / 16;
                const long long m0 = (blk * NW + warp) * LPW;
                const char* tsrc = reinterpret_cast<const char*>(reinterpret_cast<const cx<T>*>(a.tb.vtab) + m0 * N);
                char* tdst = reinterpret_cast<char*>(vt + (size_t)warp * LPW * RP);
#pragma unroll
                for (int ln = 0; ln < LPW; ++ln) {
                    if (m0 + ln < a.nlines) {
#pragma unroll
                        for (int k = 0; k < (CH + 31) / 32; ++k) {
                            const int ch = lane + 32 * k;
                            if (CH % 32 == 0 || ch < CH)
                                cp_async16(tdst + ((size_t)ln * RP * sizeof(cx<T>) + 16 * ch),
                                           tsrc + ((size_t)ln * N * sizeof(cx<T>) + 16 * ch));
                        }
                    }
                }
            }
            if (wantm) {
                constexpr int MCH = N * (int)sizeof(double) / 16;
                for (int c = lane; c < MCH; c += 32)
                    cp_async16(reinterpret_cast<char*>(ms) + 16 * c, reinterpret_cast<const char*>(mx) + 16 * c);
            }
            cp_async_commit();
        }
    }
    // potential / mask at element pos of this line; the table entry from vrow when
    // prefetched, the separable mask as mx[pos] times the line's my[j] mz[k]
    const double myz = (!mfull && mx) ? a.tb.mask1[1][jy] * a.tb.mask1[2][kz] : 1.0;
    auto diag = [&](cx<T> e, int kind, int msk, int pos) {
        const long long f = mc * N + pos;
        if (vrow) {
            const cx<T> tab = kind != DG_NONE ? vrow[pos] : e;
            const double mv = !msk ? 1.0 : (mfull ? mfull[f] : ms[pos] * myz);  // ms staged when msk
            return apply_diag_tv(e, kind, tab, msk, mv);
        }
        return apply_diag(e, kind, msk, f, pos, jy, kz, a.tb);
    };

    rfft_plan<T, N, E, R0, R1, R2, kRev, PK>(v, q, twh, twl, x);
    // v[b*RL + r] now at position q + TL b + r N/RL
    if constexpr (kTabLate) {
        if (FASTKICK || vt) {
            cp_async_wait_all();
            __syncwarp();
        }
    }

    if constexpr (MODE == XM_REDUCE) {
        double acc[kRedK] = {0, 0, 0, 0, 0};
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    const int n2 = a.tb.long_n2;  // long line: element (pos, jy) is frequency jy + N2 pos
                    const double k3[3] = {n2 ? a.tb.kv[0][jy + n2 * pos] : a.tb.kv[0][pos],
                                          n2 ? 0.0 : a.tb.kv[1][jy], n2 ? 0.0 : a.tb.kv[2][kz]};
                    const cx<double> p = widen(v[b * RL + r]);
                    acc_k(acc, p.x * p.x + p.y * p.y, k3, a.tb.inv_mass);
                }
        }
        block_reduce_store<kRedK>(acc, a.partials);
        return;
    }
    if constexpr (MODE == XM_FWD || MODE == XM_START || MODE == XM_INV || MODE == XM_END) {
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    cx<T> e = v[b * RL + r];
                    if constexpr (MODE == XM_INV) e = scale_d(cconj(e), a.out_scale);
                    if constexpr (MODE == XM_END) {
                        e = cconj(e);
                        if (a.d_store != DG_NONE || a.m_store) e = diag(e, a.d_store, a.m_store, pos);
                    }
                    dst[pos] = e;
                }
        }
        return;
    }
    if constexpr (MODE == XM_MID || MODE == XM_1D) {
        // between the FFTs: MID -> conj, V (* M) in real space; 1D -> K/N, conj
        const cx<double> dyz = dmul1(a.tb.kd[1][jy], a.tb.kd[2][kz]);
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int pos = q + TL * b + r * (N / RL);
                cx<T> e = v[b * RL + r];
                if constexpr (MODE == XM_MID && FASTKICK) {
                    // (psi h (m)) h with the staged row h and profile mx, m = mx[pos] my[j] mz[k]
                    e = apply_diag_tv(cconj(e), DG_FULL, vrow[pos], 1, ms[pos] * myz);
                } else if constexpr (MODE == XM_MID) {
                    e = cconj(e);
                    if (a.d_mid != DG_NONE || a.m_mid) e = diag(e, a.d_mid, a.m_mid, pos);
                } else if (a.tb.kfull) {  // long line: kinetic of frequency k2 + N2 k1
                    e = kinetic_full<T>(e, a.tb.kfull, mc * N + pos, a.tb.kscale);
                } else {
                    e = kinetic_apply(e, dyz, a.tb.kd[0], a.tb.kdf[0], pos, a.tb.kscale);
                }
                v[b * RL + r] = e;
            }
        rfft_plan<T, N, E, R0, R1, R2, true, PK>(v, q, twh, twl, x);
        // v[b*R0 + r] at position q + TL b + r N/R0
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / R0; ++b)
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int pos = q + TL * b + r * (N / R0);
                    cx<T> e = v[b * R0 + r];
                    if constexpr (MODE == XM_1D) {
                        e = cconj(e);
                        if (a.d_store != DG_NONE || a.m_store)
                            e = apply_diag(e, a.d_store, a.m_store, mc * N + pos, pos, jy, kz, a.tb);
                    }
                    dst[pos] = e;
                }
        }
    }
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2>
__global__ void __launch_bounds__(XShape<T, N, E>::NW * 32, XShape<T, N, E>::MINB) xpass2_kernel(const PassArgs<T> a) {
    using XS = XShape<T, N, E>;
    __shared__ cx<T> xb[XS::NW * XS::LPW * XS::PITCH];
    pdl_wait();
    xpass2_body<T, MODE, N, E, R0, R1, R2>(a, (long long)blockIdx.x, xb, a.stw, a.stwl);
}

// ---------------------------------------------------------------------------
// Strided-axis (y or z) pass, compiled plan.  CTA = L lines x N/E threads per
// line; thread (l = tid % L, q = tid / L).  Modes as in SModeK.
// ---------------------------------------------------------------------------
template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L, bool PK = false, class A>
__device__ __forceinline__ void spass2_body(const A& a, long long blk, cx<T>* tile, const cx<T>* twh,
                                            const cx<T>* twl) {
    constexpr int TL = N / E;
    using S = PlanShape<R0, R1, R2>;
    // SM_TW_START runs its FFT in the reversed radix order (the order of the
    // second FFT of SM_TW_MID), like the contiguous batch-start pass.
    constexpr bool kRev = MODE == SM_TW_START;
    constexpr int RF = kRev ? S::last : R0;
    constexpr int RL = kRev ? R0 : S::last;
    const int l = threadIdx.x % L, q = threadIdx.x / L;
    const long long s = blk * L + l;
    const bool valid = s < a.nlines;
    const long long sc_ = valid ? s : 0;
    const long long w = (long long)fdiv((uint32_t)sc_, a.fnu);
    const long long u = sc_ - w * a.nu;
    const long long base = u + w * a.sw;
    const long long se = a.se;
    const bool ypass = a.axis == 1;
    int c1, c2;  // the line's other two coordinates: y-pass (x, z), z-pass (x, y)
    if (ypass) {
        c1 = (int)u;
        c2 = (int)w;
    } else {
        c2 = (int)fdiv((uint32_t)u, a.fnx);
        c1 = (int)(u - (long long)c2 * a.nx);
    }
    // potential / mask at element pos of this line (coordinates i, j, k)
    auto diag = [&](cx<T> e, int kind, int msk, int pos) {
        const long long f = base + pos * se;
        return ypass ? apply_diag(e, kind, msk, f, c1, pos, c2, a.tb) : apply_diag(e, kind, msk, f, c1, c2, pos, a.tb);
    };
    XchCta<T, L> x{tile, l};
    cx<T> v[E];
#pragma unroll
    for (int b = 0; b < E / RF; ++b)
#pragma unroll
        for (int r = 0; r < RF; ++r) {
            const int pos = q + TL * b + r * (N / RF);
            cx<T> e = valid ? a.src[base + pos * se] : czero<T>();
            if constexpr (MODE == SM_INV) e = cconj(e);
            if constexpr (MODE == SM_TW_START) {
                if (a.d_load != DG_NONE || a.m_load) e = diag(e, a.d_load, a.m_load, pos);
            }
            if constexpr (MODE == SM_TW_MID || MODE == SM_TW_END)  // conj(e * conj W) = conj(e) * W
                e = tw4_mul<T>(cconj(e), a.tb, base + pos * se);
            v[b * RF + r] = e;
        }
    // fused pass: the line's kinetic deltas (when they fit in 32 registers a thread), fetched before the first FFT
    cx<double> dother = mk<double>(0.0, 0.0);
    constexpr bool kPre = MODE == SM_FUSED && E * sizeof(KinDelta<T>) <= 128;
    KinDelta<T> kde[kPre ? E : 1];
    if constexpr (kPre) {
        dother = dmul1(a.tb.kd[0][c1], ypass ? a.tb.kd[2][c2] : a.tb.kd[1][c2]);
        const cx<double>* kda = ypass ? a.tb.kd[1] : a.tb.kd[2];
        const cx<float>* kdaf = ypass ? a.tb.kdf[1] : a.tb.kdf[2];
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) kde[b * RL + r] = kin_delta<T>(kda, kdaf, q + TL * b + r * (N / RL));
    }

    rfft_plan<T, N, E, R0, R1, R2, kRev, PK>(v, q, twh, twl, x);

    if constexpr (MODE == SM_TW_START || MODE == SM_TW_END) {
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    cx<T> e = v[b * RL + r];
                    if constexpr (MODE == SM_TW_START) {
                        e = tw4_mul<T>(e, a.tb, base + pos * se);
                    } else {
                        e = cconj(e);
                        if (a.d_store != DG_NONE || a.m_store) e = diag(e, a.d_store, a.m_store, pos);
                    }
                    a.dst[base + pos * se] = e;
                }
        }
        return;
    }
    if constexpr (MODE == SM_TW_MID) {
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int pos = q + TL * b + r * (N / RL);
                cx<T> e = cconj(v[b * RL + r]);
                if (a.d_mid != DG_NONE || a.m_mid) e = diag(e, a.d_mid, a.m_mid, pos);
                v[b * RL + r] = e;
            }
        rfft_plan<T, N, E, R0, R1, R2, true, PK>(v, q, twh, twl, x);
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / R0; ++b)
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int pos = q + TL * b + r * (N / R0);
                    a.dst[base + pos * se] = tw4_mul<T>(v[b * R0 + r], a.tb, base + pos * se);
                }
        }
        return;
    }

    if constexpr (MODE == SM_REDUCE) {
        double acc[kRedK] = {0, 0, 0, 0, 0};
        if (valid) {
            const double* kva = ypass ? a.tb.kv[1] : a.tb.kv[2];
            const double k1 = a.tb.kv[0][c1], k2 = ypass ? a.tb.kv[2][c2] : a.tb.kv[1][c2];
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    const double ka = kva[pos];
                    const double k3[3] = {k1, ypass ? ka : k2, ypass ? k2 : ka};
                    const cx<double> p = widen(v[b * RL + r]);
                    acc_k(acc, p.x * p.x + p.y * p.y, k3, a.tb.inv_mass);
                }
        }
        block_reduce_store<kRedK>(acc, a.partials);
        return;
    }
    if constexpr (MODE == SM_FWD || MODE == SM_INV) {
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    cx<T> e = v[b * RL + r];
                    if constexpr (MODE == SM_INV) e = scale_d(cconj(e), a.out_scale);
                    a.dst[base + pos * se] = e;
                }
        }
        return;
    }
    if constexpr (MODE == SM_FUSED) {
        if constexpr (kPre) {
#pragma unroll
            for (int i2 = 0; i2 < E; ++i2) v[i2] = kinetic_apply_pre<T>(v[i2], dother, kde[i2], a.tb.kscale);
        } else {
            const cx<double> dl = dmul1(a.tb.kd[0][c1], ypass ? a.tb.kd[2][c2] : a.tb.kd[1][c2]);
            const cx<double>* kda = ypass ? a.tb.kd[1] : a.tb.kd[2];
            const cx<float>* kdaf = ypass ? a.tb.kdf[1] : a.tb.kdf[2];
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (N / RL);
                    v[b * RL + r] = kinetic_apply(v[b * RL + r], dl, kda, kdaf, pos, a.tb.kscale);
                }
        }
        rfft_plan<T, N, E, R0, R1, R2, true, PK>(v, q, twh, twl, x);
        if (valid) {
#pragma unroll
            for (int b = 0; b < E / R0; ++b)
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int pos = q + TL * b + r * (N / R0);
                    a.dst[base + pos * se] = cconj(v[b * R0 + r]);
                }
        }
    }
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L>
__global__ void __launch_bounds__(L*(N / E), 1) spass2_kernel(const PassArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    pdl_wait();
    spass2_body<T, MODE, N, E, R0, R1, R2, L>(a, (long long)blockIdx.x, reinterpret_cast<cx<T>*>(smraw), a.stw,
                                              a.stwl);
}

// ---------------------------------------------------------------------------
// Batched passes: the same bodies over many fields of one shape, one launch.
// Work item t is tile (t mod bpi) of instance t / bpi; each instance has its
// own PassArgs (field, potential table, axis tables) in global memory.  CTAs
// walk the items with a grid stride; the grid is sized to the resident CTAs.
// ---------------------------------------------------------------------------
struct BatchWork {
    uint32_t total;  // instances x tiles per instance
    uint32_t bpi;    // tiles per instance
    FastDiv fbpi;
};

template <typename T, int MODE, int N, int E, int R0, int R1, int R2>
__global__ void __launch_bounds__(XShape<T, N, E>::NW * 32, XShape<T, N, E>::MINB)
    xbatch_kernel(const PassArgs<T>* __restrict__ args, const BatchWork w) {
    using XS = XShape<T, N, E>;
    using TW = TwStage<T, R0, R1, R2>;
    __shared__ cx<T> xb[XS::NW * XS::LPW * XS::PITCH];
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smraw);
    cx<T>* vt = reinterpret_cast<cx<T>*>(smraw + TW::bytes);  // XBatchSmem: rows of the potential table
    pdl_wait();
    if (blockIdx.x < w.total) TW::load(tw, args[0].stw, args[0].stwl);  // one plan per class
    __syncthreads();
    for (uint32_t t = blockIdx.x; t < w.total; t += gridDim.x) {
        const uint32_t inst = fdiv(t, w.fbpi);
        const PassArgs<T>& a = args[inst];
        if constexpr (MODE == XM_MID) {
            // the common between-steps program: full kick and a separable absorber
            if (a.d_mid == DG_FULL && a.m_mid && a.tb.maskfull == nullptr && a.tb.mask1[0] != nullptr) {
                xpass2_body<T, MODE, N, E, R0, R1, R2, true, true>(a, (long long)(t - inst * w.bpi), xb, tw,
                                                                   TW::lo_of(tw),
                                                             vt);
                continue;
            }
        }
        xpass2_body<T, MODE, N, E, R0, R1, R2, false, true>(a, (long long)(t - inst * w.bpi), xb, tw, TW::lo_of(tw),
                                                            vt);
    }
}

// Dynamic shared memory of xbatch_kernel: stage twiddles, then NW * LPW table
// rows (pitch RPITCH), then one x profile of the absorber (N doubles) per warp.
template <typename T, int N, int E, int R0, int R1, int R2>
constexpr size_t xbatch_smem() {
    return TwStage<T, R0, R1, R2>::bytes +
           (size_t)XShape<T, N, E>::NW * XShape<T, N, E>::LPW * XShape<T, N, E>::RPITCH * sizeof(cx<T>) +
           (size_t)XShape<T, N, E>::NW * N * sizeof(double);
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L>
__global__ void __launch_bounds__(L*(N / E), 1)
    sbatch_kernel(const PassArgs<T>* __restrict__ args, const BatchWork w) {
    using TW = TwStage<T, R0, R1, R2>;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* tile = reinterpret_cast<cx<T>*>(smraw);
    cx<T>* tw = tile + (size_t)N * L;
    pdl_wait();
    if (blockIdx.x < w.total) TW::load(tw, args[0].stw, args[0].stwl);
    __syncthreads();
    for (uint32_t t = blockIdx.x; t < w.total; t += gridDim.x) {
        const uint32_t inst = fdiv(t, w.fbpi);
        spass2_body<T, MODE, N, E, R0, R1, R2, L, true>(args[inst], (long long)(t - inst * w.bpi), tile, tw,
                                                        TW::lo_of(tw));
    }
}

}  // namespace sesk
