// Pipelined compiled-plan passes: persistent CTAs walk the tiles of a pass
// while a ring of NBUF shared-memory tile buffers is filled asynchronously --
// strided axes by TMA tensor loads (boxes of L lines x up to 256 rows), the
// contiguous axis by 1D bulk copies of whole lines (psi and, where the pass
// applies the potential, the matching rows of the potential table).  The FFT
// of tile i overlaps the loads of tiles i+1 .. i+NBUF-1.  Exchanges between
// Stockham stages reuse the tile buffer in place; results go to HBM with
// coalesced stores.
#pragma once

#include "ses_pass2.cuh"
#include "ses_tma.cuh"

namespace sesk {

struct PipeArgs {
    int ntiles;         // tiles of the pass
    int kind;           // strided: 0 -> 3D map {nx, ny, nz} (y pass), 1 -> 2D map {nx*ny, nz} (z pass)
    int rows_per_box;   // <= 256
    int nbox;           // boxes per tile along the transformed axis
    unsigned* err;      // device error word (bit 0: a bounded wait expired)
    // failure-detection test hook (0 in normal launches): bounded-wait limit in SM
    // cycles (0: ~2 s) and bytes every tile's barrier expects beyond what its copies
    // deliver, so that the wait for it runs out; no copy is changed
    long long wait_limit;
    uint32_t extra_tx;
};

// Offset of the stage-twiddle copy: after the NBUF ring buffers and their
// mbarriers, rounded up to 16 bytes.
__host__ __device__ constexpr size_t pipe_tw_offset(size_t ring_bytes, int nbuf) {
    return (ring_bytes + (size_t)nbuf * 8 + 15) / 16 * 16;
}

// XOR-swizzled position inside a dense line: bijective on [0, N) for N % 16 == 0,
// spreads both exchange patterns of the compiled plans over the banks.
__device__ __forceinline__ int swz(int pos) { return pos ^ ((pos >> 4) & 15); }

template <typename T>
struct XchLine {
    cx<T>* p;
    __device__ __forceinline__ void put(int pos, cx<T> v) { p[swz(pos)] = v; }
    __device__ __forceinline__ cx<T> get(int pos) const { return p[swz(pos)]; }
    __device__ __forceinline__ void sync() { __syncwarp(); }
};

// Abort after an expired wait: record it, drain this CTA's outstanding copies
// (bounded), return.  Called by all threads of the CTA together.
__device__ __forceinline__ void pipe_abort(const PipeArgs& pa, const uint64_t* bars, int nbuf, int i,
                                           int nmine) {
    if (threadIdx.x == 0) atomicOr(pa.err, 1u);
    for (int j = i; j < nmine && j < i + nbuf; ++j)
        (void)mbar_wait(smem_u32(&bars[j % nbuf]), (uint32_t)((j / nbuf) & 1), pa.wait_limit);
}

// Where a pipelined pass finds the tile with global index t (t walks
// blockIdx.x, blockIdx.x + gridDim.x, ...): one field (kernel parameters) or
// many fields of one shape (per-instance arguments and tensor maps in global
// memory; tile t is tile t mod bpi of instance t / bpi).
template <typename T>
struct OneField {
    static constexpr bool kMany = false;
    const PassArgs<T>& a;
    const CUtensorMap* map;
    __device__ __forceinline__ const PassArgs<T>& args(uint32_t) const { return a; }
    __device__ __forceinline__ long long local(uint32_t t) const { return (long long)t; }
    __device__ __forceinline__ const CUtensorMap* tmap(uint32_t) const { return map; }
};

template <typename T>
struct ManyFields {
    static constexpr bool kMany = true;
    const PassArgs<T>* __restrict__ arr;
    const CUtensorMap* maps;
    BatchWork w;
    __device__ __forceinline__ uint32_t inst(uint32_t t) const { return fdiv(t, w.fbpi); }
    __device__ __forceinline__ const PassArgs<T>& args(uint32_t t) const { return arr[inst(t)]; }
    __device__ __forceinline__ long long local(uint32_t t) const { return (long long)(t - inst(t) * w.bpi); }
    __device__ __forceinline__ const CUtensorMap* tmap(uint32_t t) const { return maps + inst(t); }
};

// ---------------------------------------------------------------------------
// Strided axis (y or z).  CTA = L lines x N/E threads; tile = N rows x L lines.
// ---------------------------------------------------------------------------
template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L, int NBUF, class F>
__device__ __forceinline__ void spass3_body(const F& f, const PipeArgs& pa) {
    constexpr int TL = N / E;
    constexpr int EW = (int)sizeof(cx<T>) / 8;  // 8-byte words per element
    constexpr uint32_t TILE_BYTES = (uint32_t)(N * L * sizeof(cx<T>));
    using S = PlanShape<R0, R1, R2>;
    constexpr int RL = S::last;
    extern __shared__ __align__(1024) unsigned char smraw3[];
    cx<T>* tiles = reinterpret_cast<cx<T>*>(smraw3);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smraw3 + (size_t)NBUF * TILE_BYTES);
    using TW = TwStage<T, R0, R1, R2>;
    // many fields: one shared-memory copy of the class's twiddles; one field: its tables via L1
    constexpr bool kSmemTw = F::kMany;
    cx<T>* tws = reinterpret_cast<cx<T>*>(smraw3 + pipe_tw_offset((size_t)NBUF * TILE_BYTES, NBUF));
    const cx<T>* twh = kSmemTw ? tws : f.args(blockIdx.x).stw;
    const cx<T>* twl = kSmemTw ? TW::lo_of(tws) : f.args(blockIdx.x).stwl;
    const int l = threadIdx.x % L, q = threadIdx.x / L;
    const int nmine = blockIdx.x < (unsigned)pa.ntiles ? (pa.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(smem_u32(&bars[b]), 1);
        fence_mbar_init();
    }
    if (kSmemTw && nmine > 0) TW::load(tws, f.args(blockIdx.x).stw, f.args(blockIdx.x).stwl);
    __syncthreads();
    auto issue = [&](int i) {  // thread 0: load this CTA's i-th tile into buffer i % NBUF
        const int buf = i % NBUF;
        const uint32_t t = blockIdx.x + (uint32_t)i * gridDim.x;
        const long long s0 = f.local(t) * L;
        const long long nx = f.args(t).nx;
        const CUtensorMap* map = f.tmap(t);
        const uint32_t bar = smem_u32(&bars[buf]);
        const uint32_t dst = smem_u32(tiles + (size_t)buf * N * L);
        mbar_expect_tx(bar, TILE_BYTES + pa.extra_tx);
        for (int bx = 0; bx < pa.nbox; ++bx) {
            const uint32_t d = dst + (uint32_t)(bx * pa.rows_per_box * L * (int)sizeof(cx<T>));
            if (pa.kind == 0)
                tma_load_3d(d, map, (int)(s0 % nx) * EW, bx * pa.rows_per_box, (int)(s0 / nx), bar);
            else
                tma_load_2d(d, map, (int)s0 * EW, bx * pa.rows_per_box, bar);
        }
    };
    if (threadIdx.x == 0)
        for (int i = 0; i < NBUF && i < nmine; ++i) issue(i);

    for (int i = 0; i < nmine; ++i) {
        const int buf = i % NBUF;
        const uint32_t t = blockIdx.x + (uint32_t)i * gridDim.x;
        const PassArgs<T>& a = f.args(t);
        const bool ypass = a.axis == 1;
        cx<T>* tile = tiles + (size_t)buf * N * L;
        const long long s = f.local(t) * L + l;
        const bool valid = s < a.nlines;
        const long long sc_ = valid ? s : 0;
        const long long w = (long long)fdiv((uint32_t)sc_, a.fnu);
        const long long u = sc_ - w * a.nu;
        const long long base = u + w * a.sw;
        int c1, c2;  // the line's other two coordinates: y-pass (x, z), z-pass (x, y)
        if (ypass) {
            c1 = (int)u;
            c2 = (int)w;
        } else {
            c2 = (int)fdiv((uint32_t)u, a.fnx);
            c1 = (int)(u - (long long)c2 * a.nx);
        }
        // fused pass: the line's kinetic deltas (when they fit in 32 registers a thread), fetched while the tile's copy is in flight
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
        const bool ok = mbar_wait(smem_u32(&bars[buf]), (uint32_t)((i / NBUF) & 1), pa.wait_limit);
        if (__syncthreads_or(!ok)) {
            pipe_abort(pa, bars, NBUF, i, nmine);
            return;
        }
        XchCta<T, L> x{tile, l};
        cx<T> v[E];
#pragma unroll
        for (int b = 0; b < E / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const cx<T> e = tile[(q + TL * b + r * (N / R0)) * L + l];
                v[b * R0 + r] = MODE == SM_INV ? cconj(e) : e;
            }
        __syncthreads();  // all stage-0 reads before the tile is reused for exchanges
        rfft_plan<T, N, E, R0, R1, R2, false, kSmemTw>(v, q, twh, twl, x);

        if constexpr (MODE == SM_FWD || MODE == SM_INV) {
            if (valid) {
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int pos = q + TL * b + r * (N / RL);
                        cx<T> e = v[b * RL + r];
                        if constexpr (MODE == SM_INV) e = scale_d(cconj(e), a.out_scale);
                        a.dst[base + pos * a.se] = e;
                    }
            }
        } else if constexpr (MODE == SM_FUSED) {
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
            rfft_plan<T, N, E, R0, R1, R2, true, kSmemTw>(v, q, twh, twl, x);
            if (valid) {
#pragma unroll
                for (int b = 0; b < E / R0; ++b)
#pragma unroll
                    for (int r = 0; r < R0; ++r) {
                        const int pos = q + TL * b + r * (N / R0);
                        a.dst[base + pos * a.se] = cconj(v[b * R0 + r]);
                    }
            }
        }
        // release the buffer: generic accesses ordered before the next TMA write
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && i + NBUF < nmine) issue(i + NBUF);
    }
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L, int NBUF, int MINB>
__global__ void __launch_bounds__(L*(N / E), MINB)
    spass3_kernel(const PassArgs<T> a, const __grid_constant__ CUtensorMap tmap, const PipeArgs pa) {
    pdl_wait();
    spass3_body<T, MODE, N, E, R0, R1, R2, L, NBUF>(OneField<T>{a, &tmap}, pa);
}

// Batched: the fields of one shape class, per-instance tensor maps in global memory.
template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int L, int NBUF, int MINB>
__global__ void __launch_bounds__(L*(N / E), MINB)
    sbatch3_kernel(const PassArgs<T>* __restrict__ args, const CUtensorMap* maps, const BatchWork w,
                   const PipeArgs pa) {
    pdl_wait();
    spass3_body<T, MODE, N, E, R0, R1, R2, L, NBUF>(ManyFields<T>{args, maps, w}, pa);
}

// ---------------------------------------------------------------------------
// Contiguous axis (x).  NW warps per CTA, a warp owns 32/(N/E) lines; a tile
// is the CTA's consecutive lines, copied whole (plus the potential-table rows
// when the mode applies the potential).
// ---------------------------------------------------------------------------
template <int MODE>
struct XUsesTable {
    static constexpr bool value = MODE == XM_START || MODE == XM_MID || MODE == XM_END || MODE == XM_1D;
};

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int NW, int NBUF, class F>
__device__ __forceinline__ void xpass3_body(const F& f, const PipeArgs& pa) {
    constexpr int TL = N / E;
    constexpr int LPW = 32 / TL;
    constexpr int LPC = NW * LPW;
    constexpr bool kTab = XUsesTable<MODE>::value;
    constexpr uint32_t PSI_BYTES = (uint32_t)(LPC * N * sizeof(cx<T>));
    // Passes that apply the potential read the x profile of a separable absorber
    // (N doubles) from shared memory, not between the FFTs from global memory:
    // batched, each tile buffer carries its instance's profile after the table
    // rows; one field, the profile is loaded once into the (there unused) slot of
    // the stage-twiddle copy.
    constexpr bool kMrowRing = kTab && F::kMany;
    constexpr uint32_t MROW_BYTES = kMrowRing ? (uint32_t)(N * sizeof(double)) : 0u;
    constexpr uint32_t BUF_BYTES = kTab ? 2 * PSI_BYTES + MROW_BYTES : PSI_BYTES;
    using S = PlanShape<R0, R1, R2>;
    // batch start: reversed radix order, as the second FFT of the between-steps pass
    constexpr bool kRev = MODE == XM_START;
    constexpr int RF = kRev ? S::last : R0;
    constexpr int RL = kRev ? R0 : S::last;
    extern __shared__ __align__(1024) unsigned char smraw3[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smraw3 + (size_t)NBUF * BUF_BYTES);
    using TW = TwStage<T, R0, R1, R2>;
    constexpr bool kSmemTw = F::kMany;
    cx<T>* tws = reinterpret_cast<cx<T>*>(smraw3 + pipe_tw_offset((size_t)NBUF * BUF_BYTES, NBUF));
    const cx<T>* twh = kSmemTw ? tws : f.args(blockIdx.x).stw;
    const cx<T>* twl = kSmemTw ? TW::lo_of(tws) : f.args(blockIdx.x).stwl;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lw = lane / TL, q = lane % TL;
    const int nmine = blockIdx.x < (unsigned)pa.ntiles ? (pa.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(smem_u32(&bars[b]), 1);
        fence_mbar_init();
    }
    if (kSmemTw && nmine > 0) TW::load(tws, f.args(blockIdx.x).stw, f.args(blockIdx.x).stwl);
    static_assert(TW::bytes >= N * sizeof(double), "the absorber profile fits the twiddle slot");
    double* mrow1 = reinterpret_cast<double*>(tws);  // one field: the absorber's x profile
    if constexpr (kTab && !F::kMany) {
        const PassArgs<T>& a0 = f.args(0);
        if (nmine > 0 && a0.tb.maskfull == nullptr && a0.tb.mask1[0] != nullptr)
            for (int i = threadIdx.x; i < N; i += blockDim.x) mrow1[i] = a0.tb.mask1[0][i];
    }
    __syncthreads();
    auto issue = [&](int i) {
        const int buf = i % NBUF;
        const uint32_t t = blockIdx.x + (uint32_t)i * gridDim.x;
        const PassArgs<T>& a = f.args(t);
        const cx<T>* vtab = reinterpret_cast<const cx<T>*>(a.tb.vtab);
        const long long m0 = f.local(t) * LPC;
        const long long rem = a.nlines - m0;
        const int nval = rem < LPC ? (int)rem : LPC;
        const uint32_t bytes = (uint32_t)(nval * N * (int)sizeof(cx<T>));
        const uint32_t bar = smem_u32(&bars[buf]);
        const uint32_t dst = smem_u32(smraw3 + (size_t)buf * BUF_BYTES);
        const bool sepm = kMrowRing && a.tb.maskfull == nullptr && a.tb.mask1[0] != nullptr;
        mbar_expect_tx(bar, (kTab ? 2 * bytes : bytes) + (sepm ? MROW_BYTES : 0u) + pa.extra_tx);
        bulk_g2s(dst, a.src + m0 * N, bytes, bar);
        if constexpr (kTab) bulk_g2s(dst + PSI_BYTES, vtab + m0 * N, bytes, bar);
        if constexpr (kMrowRing)
            if (sepm) bulk_g2s(dst + 2 * PSI_BYTES, a.tb.mask1[0], MROW_BYTES, bar);
    };
    if (threadIdx.x == 0)
        for (int i = 0; i < NBUF && i < nmine; ++i) issue(i);

    for (int i = 0; i < nmine; ++i) {
        const int buf = i % NBUF;
        const bool ok = mbar_wait(smem_u32(&bars[buf]), (uint32_t)((i / NBUF) & 1), pa.wait_limit);
        if (__syncthreads_or(!ok)) {
            pipe_abort(pa, bars, NBUF, i, nmine);
            return;
        }
        const uint32_t t = blockIdx.x + (uint32_t)i * gridDim.x;
        const PassArgs<T>& a = f.args(t);
        cx<T>* ptile = reinterpret_cast<cx<T>*>(smraw3 + (size_t)buf * BUF_BYTES);
        const cx<T>* ttile = reinterpret_cast<const cx<T>*>(smraw3 + (size_t)buf * BUF_BYTES + PSI_BYTES);
        const int lc = warp * LPW + lw;  // line within the tile
        const long long m = f.local(t) * LPC + lc;
        const bool valid = m < a.nlines;
        const long long mc = valid ? m : 0;
        const int kz = (int)fdiv((uint32_t)mc, a.fny);
        const int jy = (int)(mc - (long long)kz * a.ny);
        // separable absorber: per-line factor my[j] * mz[k] (the mask is m = mx[i] * (my[j] * mz[k]))
        const bool sep = a.tb.maskfull == nullptr && a.tb.mask1[0] != nullptr;
        const double myz = sep ? a.tb.mask1[1][jy] * a.tb.mask1[2][kz] : 1.0;
        const double* mrow = kMrowRing ? reinterpret_cast<const double*>(smraw3 + (size_t)buf * BUF_BYTES + 2 * PSI_BYTES)
                                       : mrow1;
        auto mval = [&](int pos) -> double {  // == maskval<T>(a.tb, mc * N + pos, pos, jy, kz)
            if (!sep) return a.tb.maskfull ? a.tb.maskfull[mc * N + pos] : 1.0;
            return (kTab ? mrow[pos] : a.tb.mask1[0][pos]) * myz;
        };
        cx<T>* line = ptile + (size_t)lc * N;
        const cx<T>* tline = ttile + (size_t)lc * N;
        XchLine<T> x{line};
        cx<T>* dst = a.dst + mc * N;
        cx<T> v[E];
        constexpr bool kConjIn = MODE == XM_MID || MODE == XM_END;
#pragma unroll
        for (int b = 0; b < E / RF; ++b)
#pragma unroll
            for (int r = 0; r < RF; ++r) {
                const int pos = q + TL * b + r * (N / RF);
                cx<T> e = line[pos];
                if constexpr (MODE == XM_START || MODE == XM_1D) {
                    if (a.d_load != DG_NONE || a.m_load)
                        e = apply_diag_tv(e, a.d_load, tline[pos], a.m_load, a.m_load ? mval(pos) : 1.0);
                }
                v[b * RF + r] = kConjIn ? cconj(e) : e;
            }
        __syncwarp();  // the line is reused for exchanges: all stage-0 reads first
        rfft_plan<T, N, E, R0, R1, R2, kRev, kSmemTw>(v, q, twh, twl, x);

        if constexpr (MODE == XM_FWD || MODE == XM_START || MODE == XM_END) {
            if (valid) {
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int pos = q + TL * b + r * (N / RL);
                        cx<T> e = v[b * RL + r];
                        if constexpr (MODE == XM_END) {
                            e = cconj(e);
                            if (a.d_store != DG_NONE || a.m_store)
                                e = apply_diag_tv(e, a.d_store, tline[pos], a.m_store,
                                                  a.m_store ? mval(pos) : 1.0);
                        }
                        dst[pos] = e;
                    }
            }
        } else if constexpr (MODE == XM_MID || MODE == XM_1D) {
            // the common between-steps program -- full kick, separable absorber -- as
            // straight-line code (the same arithmetic as the general path below)
            bool fast = false;
            if constexpr (MODE == XM_MID) fast = a.d_mid == DG_FULL && a.m_mid && sep;
            if (fast) {
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int pos = q + TL * b + r * (N / RL);
                        const double m = (kTab ? mrow[pos] : a.tb.mask1[0][pos]) * myz;
                        v[b * RL + r] = apply_diag_tv(cconj(v[b * RL + r]), DG_FULL, tline[pos], 1, m);
                    }
            } else {
                const cx<double> dyz = dmul1(a.tb.kd[1][jy], a.tb.kd[2][kz]);
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int pos = q + TL * b + r * (N / RL);
                        cx<T> e = v[b * RL + r];
                        if constexpr (MODE == XM_MID) {
                            e = cconj(e);
                            if (a.d_mid != DG_NONE || a.m_mid)
                                e = apply_diag_tv(e, a.d_mid, tline[pos], a.m_mid, a.m_mid ? mval(pos) : 1.0);
                        } else {
                            e = kinetic_conj(e, dmul1(dyz, a.tb.kd[0][pos]), a.tb.kscale);
                        }
                        v[b * RL + r] = e;
                    }
            }
            rfft_plan<T, N, E, R0, R1, R2, true, kSmemTw>(v, q, twh, twl, x);
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
                                e = apply_diag_tv(e, a.d_store, tline[pos], a.m_store,
                                                  a.m_store ? mval(pos) : 1.0);
                        }
                        dst[pos] = e;
                    }
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && i + NBUF < nmine) issue(i + NBUF);
    }
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int NW, int NBUF, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) xpass3_kernel(const PassArgs<T> a, const PipeArgs pa) {
    pdl_wait();
    xpass3_body<T, MODE, N, E, R0, R1, R2, NW, NBUF>(OneField<T>{a, nullptr}, pa);
}

template <typename T, int MODE, int N, int E, int R0, int R1, int R2, int NW, int NBUF, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB)
    xbatch3_kernel(const PassArgs<T>* __restrict__ args, const BatchWork w, const PipeArgs pa) {
    pdl_wait();
    xpass3_body<T, MODE, N, E, R0, R1, R2, NW, NBUF>(ManyFields<T>{args, nullptr, w}, pa);
}

}  // namespace sesk
