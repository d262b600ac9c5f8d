// Plane pass of the two-sweep 3D step for grids whose x-y plane fits in shared
// memory.  The four axis passes of a merged Strang step,
//
//   X[inv x, V*M, fwd x]  Y[fwd y]  Z[fwd z, K/N, inv z]  Y[inv y],
//
// touch psi in HBM four times; here the y transforms move into the x pass, per
// z-plane, and a step becomes two sweeps:
//
//   P[inv y, inv x, V*M, fwd x, fwd y]  Z[fwd z, K/N, inv z]
//
// (batch start P[V/2, fwd x, fwd y], batch end P[inv y, inv x, V/2 (*M)]).
// One CTA holds one plane in shared memory; the y phases run the strided
// pass's line FFT on the plane's columns, the x phase the contiguous pass's on
// its rows, with the same plans, radix orders and diagonal arithmetic as the
// axis passes.  The two step forms agree to the last bits the compiler's FMA
// contraction may place differently in differently structured kernels; within
// one form the step is deterministic, and a run split into several calls gives
// the bits of one call (the batch end + batch start equal a between-steps pass).
#pragma once

#include <vector>

#include "ses_pass2.cuh"

namespace sesk {

enum PlaneMode : int {
    PL_START = 0,  // [V/2 (*M)] fwd x, fwd y                  (first step of a batch)
    PL_MID = 1,    // inv y, inv x, V (*M), fwd x, fwd y       (between steps)
    PL_END = 2     // inv y, inv x, V/2 (*M)                   (end of a batch)
};

// Plane of NX x NY points, x plan with EX elements per thread, y plan with EY,
// NT threads.  Rows are the x-lines at the contiguous pass's padded pitch
// (element x of row y at y PITCH + x + PM (x >> SH)); a y-line is a column.
template <typename T, int NX, int EX, int NY, int EY, int NT>
struct PlaneShape {
    static constexpr int TLX = NX / EX, TLY = NY / EY;
    static constexpr int LPW = 32 / TLX;  // x-lines per warp
    static constexpr int LX = NT / TLX;   // x-lines per round
    static constexpr int LY = NT / TLY;   // y-lines per round
    static constexpr int SH = XPad<NX, EX>::SH, PM = XPad<NX, EX>::PM;
    static constexpr int PITCH = XPad<NX, EX>::PITCH;
    static constexpr size_t plane_bytes = (size_t)NY * PITCH * sizeof(cx<T>);
    static_assert(NT % 32 == 0 && 32 % TLX == 0 && NY % LX == 0 && NX % LY == 0, "plane tiling");
    static_assert(plane_bytes % 16 == 0, "twiddle copies start on 16-byte boundaries");
    static __device__ __forceinline__ int col(int x) { return x + PM * (x >> SH); }
};

// A column of the plane as the exchange buffer of a y-line (CTA-wide sync: the
// line's threads sit in different warps).
template <typename T, int PITCH>
struct XchCol {
    cx<T>* p;
    __device__ __forceinline__ void put(int pos, cx<T> v) { p[pos * PITCH] = v; }
    __device__ __forceinline__ cx<T> get(int pos) const { return p[pos * PITCH]; }
    __device__ __forceinline__ void sync() { __syncthreads(); }
};

template <typename T, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2, int NT>
constexpr size_t plane_smem() {
    return PlaneShape<T, NX, EX, NY, EY, NT>::plane_bytes + TwStage<T, RX0, RX1, RX2>::bytes +
           TwStage<T, RY0, RY1, RY2>::bytes;
}

// y phase, inverse (strided pass SM_INV, out_scale s): the NCOL columns x0 + xl
// of the plane at `src` (global memory), L per round; conj, FFT in plan order
// with the exchanges in column xl of a buffer of pitch XP (colp(xl)), then
// out(x, pos, conj * s); before_out() runs once, before the first round's outputs.
template <typename T, int NX, int NY, int EY, int RY0, int RY1, int RY2, int L, int NCOL, int XP, bool PK, class COLP,
          class OUT, class PRE>
__device__ __forceinline__ void plane_y_inv(const cx<T>* __restrict__ src, int x0, COLP colp, const cx<T>* twy,
                                            double s, OUT out, PRE before_out) {
    constexpr int TL = NY / EY;
    constexpr int RL = PlanShape<RY0, RY1, RY2>::last;
    const int l = threadIdx.x % L, q = threadIdx.x / L;
#pragma unroll 1
    for (int it = 0; it < NCOL / L; ++it) {
        const int xl = it * L + l, x = x0 + xl;
        XchCol<T, XP> xc{colp(xl)};
        cx<T> v[EY];
#pragma unroll
        for (int b = 0; b < EY / RY0; ++b)
#pragma unroll
            for (int r = 0; r < RY0; ++r) v[b * RY0 + r] = cconj(src[(q + TL * b + r * (NY / RY0)) * NX + x]);
        rfft_plan<T, NY, EY, RY0, RY1, RY2, false, PK>(v, q, twy, twy, xc);
        if (it == 0) before_out();
#pragma unroll
        for (int b = 0; b < EY / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) out(x, q + TL * b + r * (NY / RL), scale_d(cconj(v[b * RL + r]), s));
    }
}

// y phase, forward (strided pass SM_FWD): the NCOL columns x0 + xl from column xl
// of a buffer of pitch XP (colp(xl)), FFT in plan order (exchanges in the same
// column), to the plane at `dst` (global memory).
template <typename T, int NX, int NY, int EY, int RY0, int RY1, int RY2, int L, int NCOL, int XP, bool PK, class COLP>
__device__ __forceinline__ void plane_y_fwd(cx<T>* __restrict__ dst, int x0, COLP colp, const cx<T>* twy) {
    constexpr int TL = NY / EY;
    constexpr int RL = PlanShape<RY0, RY1, RY2>::last;
    const int l = threadIdx.x % L, q = threadIdx.x / L;
#pragma unroll 1
    for (int it = 0; it < NCOL / L; ++it) {
        const int xl = it * L + l, x = x0 + xl;
        XchCol<T, XP> xc{colp(xl)};
        cx<T> v[EY];
#pragma unroll
        for (int b = 0; b < EY / RY0; ++b)
#pragma unroll
            for (int r = 0; r < RY0; ++r) v[b * RY0 + r] = xc.get(q + TL * b + r * (NY / RY0));
        __syncthreads();  // the column's other threads have read their inputs before the first exchange
        rfft_plan<T, NY, EY, RY0, RY1, RY2, false, PK>(v, q, twy, twy, xc);
#pragma unroll
        for (int b = 0; b < EY / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) dst[(q + TL * b + r * (NY / RL)) * NX + x] = v[b * RL + r];
    }
}

// x phase: the NROWS rows y0 + yl of plane z, row yl of the row buffer `rows`
// (pitch PITCH, padding SH / PM), LX per round.  START: from global memory with
// V/2 (*M) at the load, forward FFT in reversed radix order (the contiguous pass
// XM_START), out(y, pos, v).  MID: from the row buffer, conj, FFT, conj, V (*M),
// reversed-order FFT (XM_MID), out(y, pos, v).  END: from the row buffer, conj,
// FFT, conj, V/2 (*M), to global memory (XM_END).  The FFT exchanges use the row.
template <typename T, int MODE, int NX, int EX, int RX0, int RX1, int RX2, int NY, int NT, int NROWS, int SH, int PM,
          int PITCH, bool PK, class OUT>
__device__ __forceinline__ void plane_x(const PassArgs<T>& a, int z, int y0, cx<T>* rows, const cx<T>* twx,
                                        OUT out) {
    using S = PlanShape<RX0, RX1, RX2>;
    constexpr int TL = NX / EX;
    constexpr int NW = NT / 32;
    constexpr int LPW = 32 / TL;
    constexpr int LX = NT / TL;
    constexpr bool kRev = MODE == PL_START;
    constexpr int RF = kRev ? S::last : RX0;  // first stage's radix (input layout)
    constexpr int RL = kRev ? RX0 : S::last;  // last stage's radix (output layout)
    static_assert(NROWS % LX == 0, "whole rounds of rows");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, lw = lane / TL, q = lane % TL;
    const cx<T>* vtab = reinterpret_cast<const cx<T>*>(a.tb.vtab);
#pragma unroll 1
    for (int it = 0; it < NROWS / LX; ++it) {
        const int yl = (it * NW + warp) * LPW + lw, y = y0 + yl;
        const long long row = ((long long)z * NY + y) * NX;  // flat index of the line's first point
        XchWarp<T, SH, PM> xw{rows + yl * PITCH};
        cx<T> v[EX];
        if constexpr (MODE == PL_START) {
#pragma unroll
            for (int b = 0; b < EX / RF; ++b)
#pragma unroll
                for (int r = 0; r < RF; ++r) {
                    const int pos = q + TL * b + r * (NX / RF);
                    cx<T> e = a.src[row + pos];
                    if (a.d_load != DG_NONE || a.m_load)
                        e = apply_diag(e, a.d_load, a.m_load, row + pos, pos, y, z, a.tb);
                    v[b * RF + r] = e;
                }
        } else {
#pragma unroll
            for (int b = 0; b < EX / RF; ++b)
#pragma unroll
                for (int r = 0; r < RF; ++r) v[b * RF + r] = cconj(xw.get(q + TL * b + r * (NX / RF)));
            __syncwarp();  // the line's other lanes have read their inputs before the first exchange
        }
        // between-steps pass: the potential-table entries used after the first
        // FFT, fetched before it
        cx<T> tv[EX];
        if constexpr (MODE == PL_MID) {
            if (a.d_mid != DG_NONE) {
#pragma unroll
                for (int b = 0; b < EX / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) tv[b * RL + r] = vtab[row + q + TL * b + r * (NX / RL)];
            }
        }
        rfft_plan<T, NX, EX, RX0, RX1, RX2, kRev, PK>(v, q, twx, twx, xw);
        if constexpr (MODE == PL_START) {
#pragma unroll
            for (int b = 0; b < EX / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) out(y, q + TL * b + r * (NX / RL), v[b * RL + r]);
        } else if constexpr (MODE == PL_END) {
#pragma unroll
            for (int b = 0; b < EX / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (NX / RL);
                    cx<T> e = cconj(v[b * RL + r]);
                    if (a.d_store != DG_NONE || a.m_store)
                        e = apply_diag(e, a.d_store, a.m_store, row + pos, pos, y, z, a.tb);
                    a.dst[row + pos] = e;
                }
        } else {
#pragma unroll
            for (int b = 0; b < EX / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int pos = q + TL * b + r * (NX / RL);
                    cx<T> e = cconj(v[b * RL + r]);
                    if (a.d_mid != DG_NONE || a.m_mid) {
                        const cx<T> tab = a.d_mid != DG_NONE ? tv[b * RL + r] : e;
                        e = apply_diag_tv(e, a.d_mid, tab, a.m_mid,
                                          a.m_mid ? maskval<T>(a.tb, row + pos, pos, y, z) : 1.0);
                    }
                    v[b * RL + r] = e;
                }
            rfft_plan<T, NX, EX, RX0, RX1, RX2, true, PK>(v, q, twx, twx, xw);
#pragma unroll
            for (int b = 0; b < EX / RX0; ++b)
#pragma unroll
                for (int r = 0; r < RX0; ++r) out(y, q + TL * b + r * (NX / RX0), v[b * RX0 + r]);
        }
    }
}

// Plane z of the field of `ax` through the whole plane buffer P (element (x, y)
// at P[y PITCH + col(x)]: rows are x-lines, columns y-lines); s: the inverse y
// pass's scale.  In place: the plane is read whole before any of it is written.
template <typename T, int MODE, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2,
          int NT>
__device__ __forceinline__ void plane_body(const PassArgs<T>& ax, double s, int z, cx<T>* P, const cx<T>* twx,
                                           const cx<T>* twy) {
    using PS = PlaneShape<T, NX, EX, NY, EY, NT>;
    constexpr bool PK = sizeof(T) == 4;  // complex64: interleaved hi/lo twiddles
    const long long gz = (long long)z * NX * NY;
    auto colp = [&](int x) { return P + PS::col(x); };
    auto put = [&](int y, int x, cx<T> v) { P[y * PS::PITCH + PS::col(x)] = v; };
    if constexpr (MODE != PL_START) {
        plane_y_inv<T, NX, NY, EY, RY0, RY1, RY2, PS::LY, NX, PS::PITCH, PK>(
            ax.src + gz, 0, colp, twy, s, [&](int x, int pos, cx<T> v) { put(pos, x, v); }, [] {});
        __syncthreads();
    }
    plane_x<T, MODE, NX, EX, RX0, RX1, RX2, NY, NT, NY, PS::SH, PS::PM, PS::PITCH, PK>(
        ax, z, 0, P, twx, [&](int y, int pos, cx<T> v) { put(y, pos, v); });
    if constexpr (MODE != PL_END) {
        __syncthreads();
        plane_y_fwd<T, NX, NY, EY, RY0, RY1, RY2, PS::LY, NX, PS::PITCH, PK>(ax.dst + gz, 0, colp, twy);
    }
}

// One CTA per z-plane (grid = nz).  ax: the x pass's arguments (field, tables,
// diagonal program, x stage twiddles); ay: the y stage twiddles and the inverse
// y pass's scale.
template <typename T, int MODE, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2,
          int NT>
__global__ void __launch_bounds__(NT, 1) plane_kernel(const PassArgs<T> ax, const PassArgs<T> ay) {
    using PS = PlaneShape<T, NX, EX, NY, EY, NT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* P = reinterpret_cast<cx<T>*>(smraw);
    cx<T>* twx = reinterpret_cast<cx<T>*>(smraw + PS::plane_bytes);
    cx<T>* twy = reinterpret_cast<cx<T>*>(smraw + PS::plane_bytes + TwStage<T, RX0, RX1, RX2>::bytes);
    pdl_wait();
    TwStage<T, RX0, RX1, RX2>::load(twx, ax.stw, ax.stwl);
    TwStage<T, RY0, RY1, RY2>::load(twy, ay.stw, ay.stwl);
    __syncthreads();
    plane_body<T, MODE, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>(ax, ay.out_scale, (int)blockIdx.x, P, twx,
                                                                         twy);
}

// Batched plane pass: the planes of every member of a class (one shape, one
// plan), work item t = member w.bpi + z (w.bpi = nz), CTAs walking the items
// grid-stride; the class's stage twiddles (shared by its members) are loaded
// once per CTA.  axs / ays: per-member x-program and y-pass arguments.
template <typename T, int MODE, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2,
          int NT>
__global__ void __launch_bounds__(NT, 1)
    plane_batch_kernel(const PassArgs<T>* __restrict__ axs, const PassArgs<T>* __restrict__ ays, const BatchWork w) {
    using PS = PlaneShape<T, NX, EX, NY, EY, NT>;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* P = reinterpret_cast<cx<T>*>(smraw);
    cx<T>* twx = reinterpret_cast<cx<T>*>(smraw + PS::plane_bytes);
    cx<T>* twy = reinterpret_cast<cx<T>*>(smraw + PS::plane_bytes + TwStage<T, RX0, RX1, RX2>::bytes);
    pdl_wait();
    if (blockIdx.x < w.total) {
        TwStage<T, RX0, RX1, RX2>::load(twx, axs[0].stw, axs[0].stwl);
        TwStage<T, RY0, RY1, RY2>::load(twy, ays[0].stw, ays[0].stwl);
    }
    __syncthreads();
    for (uint32_t t = blockIdx.x; t < w.total; t += gridDim.x) {
        const uint32_t m = fdiv(t, w.fbpi);
        plane_body<T, MODE, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>(axs[m], ays[m].out_scale,
                                                                             (int)(t - m * w.bpi), P, twx, twy);
        __syncthreads();  // the plane buffer is free for the next item
    }
}

// ---------------------------------------------------------------------------
// Plane pass over a thread-block cluster of CS CTAs (CS = 2, 4): CTA c owns the
// columns x in [c NX/CS, (c+1) NX/CS) for the y phases and the rows y in
// [c NY/CS, (c+1) NY/CS) for the x phase, so a plane's shared-memory traffic
// (the exchanges of four line FFTs and the two transposes) is spread over CS
// SMs.  The transposes write straight into the owning CTA's buffer through
// distributed shared memory; hardware cluster barriers order them (no waits of
// this code).  Every remote access comes before the last cluster barrier, so
// no CTA reads or writes the shared memory of a CTA that may have exited.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of this CTA's shared-memory location p in the window of CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(uint32_t a, cx<double> v) {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, cx<float> v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
// All threads of all CTAs of the cluster; shared-memory writes before it
// (local and remote) are visible to every CTA after it.
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The two halves of a barrier that orders no memory: arrive (this thread has
// started), and wait (every thread of the cluster has arrived).
__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;" ::: "memory"); }

// Base (shared::cluster address) of the same buffer in CTA o, o < CS, from the CS
// bases mapped once per kernel (compile-time selects, no indexed local array).
template <int CS>
__device__ __forceinline__ uint32_t pick_base(const uint32_t (&b)[CS], int o) {
    uint32_t r = b[0];
#pragma unroll
    for (int i = 1; i < CS; ++i) r = o == i ? b[i] : r;
    return r;
}

template <typename T, int NX, int EX, int NY, int EY, int CS, int NT>
struct ClusterPlaneShape {
    static constexpr int NXC = NX / CS, NYC = NY / CS;  // columns / rows of one CTA
    static constexpr int TLX = NX / EX, TLY = NY / EY;
    static constexpr int LPW = 32 / TLX;
    static constexpr int LX = NT / TLX, LY = NT / TLY;  // lines per round
    static constexpr int SH = XPad<NX, EX>::SH, PM = XPad<NX, EX>::PM;
    static constexpr int PITCH = XPad<NX, EX>::PITCH;  // row buffer: NYC rows of the x pass's padded pitch
    // column buffer: NY positions x NXC columns; complex64 rows padded by 64 bytes so
    // the x phase's four rows per warp land on different banks
    static constexpr int CPITCH = NXC + (sizeof(T) == 4 ? 8 : 0);
    static constexpr size_t rows_bytes = (size_t)NYC * PITCH * sizeof(cx<T>);
    static constexpr size_t cols_bytes = (size_t)NY * CPITCH * sizeof(cx<T>);
    static_assert(NX % CS == 0 && NY % CS == 0, "whole columns and rows per CTA");
    static_assert(NT % 32 == 0 && 32 % TLX == 0 && NYC % LX == 0 && NXC % LY == 0, "cluster plane tiling");
    static_assert(rows_bytes % 16 == 0 && cols_bytes % 16 == 0, "16-byte aligned buffers");
    static __device__ __forceinline__ int col(int x) { return x + PM * (x >> SH); }
};

template <typename T, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2, int CS,
          int NT>
constexpr size_t cluster_plane_smem() {
    using S = ClusterPlaneShape<T, NX, EX, NY, EY, CS, NT>;
    return S::rows_bytes + S::cols_bytes + TwStage<T, RX0, RX1, RX2>::bytes + TwStage<T, RY0, RY1, RY2>::bytes;
}

// Cluster of CS CTAs per z-plane (grid = nz CS, cluster dims (CS, 1, 1)); CTA c
// of cluster z.  Row buffer: this CTA's NY/CS rows; column buffer: its NX/CS
// columns, element (xl, y) at y CPITCH + xl.
template <typename T, int MODE, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2,
          int CS, int NT>
__global__ void __launch_bounds__(NT, 1) cluster_plane_kernel(const PassArgs<T> ax, const PassArgs<T> ay) {
    using PS = ClusterPlaneShape<T, NX, EX, NY, EY, CS, NT>;
    constexpr bool PK = sizeof(T) == 4;
    constexpr uint32_t ES = sizeof(cx<T>);
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* R = reinterpret_cast<cx<T>*>(smraw);
    cx<T>* Cb = reinterpret_cast<cx<T>*>(smraw + PS::rows_bytes);
    cx<T>* twx = reinterpret_cast<cx<T>*>(smraw + PS::rows_bytes + PS::cols_bytes);
    cx<T>* twy = reinterpret_cast<cx<T>*>(smraw + PS::rows_bytes + PS::cols_bytes + TwStage<T, RX0, RX1, RX2>::bytes);
    pdl_wait();
    TwStage<T, RX0, RX1, RX2>::load(twx, ax.stw, ax.stwl);
    TwStage<T, RY0, RY1, RY2>::load(twy, ay.stw, ay.stwl);
    const int c = (int)cluster_ctarank();
    const int z = blockIdx.x / CS;
    const long long gz = (long long)z * NX * NY;
    uint32_t rb[CS], cb[CS];  // the row and column buffers of every CTA of the cluster
#pragma unroll
    for (int o = 0; o < CS; ++o) {
        rb[o] = cluster_map(R, (uint32_t)o);
        cb[o] = cluster_map(Cb, (uint32_t)o);
    }
    // every CTA of the cluster runs (its buffers exist) before any of them is
    // written remotely: arrive now, wait before the first remote store
    cluster_arrive_relaxed();
    __syncthreads();  // twiddles in place
    auto colp = [&](int xl) { return Cb + xl; };
    if constexpr (MODE == PL_START) cluster_wait();
    if constexpr (MODE != PL_START) {
        // column results (x, y) to row y of the CTA that owns it
        auto to_rows = [&](int x, int y, cx<T> v) {
            const int o = y / PS::NYC;
            st_cluster(pick_base<CS>(rb, o) + (uint32_t)((y - o * PS::NYC) * PS::PITCH + PS::col(x)) * ES, v);
        };
        plane_y_inv<T, NX, NY, EY, RY0, RY1, RY2, PS::LY, PS::NXC, PS::CPITCH, PK>(
            ax.src + gz, c * PS::NXC, colp, twy, ay.out_scale, to_rows, [] { cluster_wait(); });
        cluster_barrier();
    }
    // row results (x, y) to column x of the CTA that owns it
    auto to_cols = [&](int y, int x, cx<T> v) {
        const int o = x / PS::NXC;
        st_cluster(pick_base<CS>(cb, o) + (uint32_t)(y * PS::CPITCH + (x - o * PS::NXC)) * ES, v);
    };
    plane_x<T, MODE, NX, EX, RX0, RX1, RX2, NY, NT, PS::NYC, PS::SH, PS::PM, PS::PITCH, PK>(ax, z, c * PS::NYC, R,
                                                                                            twx, to_cols);
    if constexpr (MODE != PL_END) {
        cluster_barrier();  // the last remote access of the kernel is before this barrier
        plane_y_fwd<T, NX, NY, EY, RY0, RY1, RY2, PS::LY, PS::NXC, PS::CPITCH, PK>(ax.dst + gz, c * PS::NXC, colp,
                                                                                   twy);
    }
}

template <typename T>
using PlaneKernel = void (*)(const PassArgs<T>, const PassArgs<T>);
template <typename T>
using PlaneBatchKernel = void (*)(const PassArgs<T>*, const PassArgs<T>*, const BatchWork);

// A compiled plane pass: the x and y plans it was built with (the solver uses it
// only when its own x and y plans are these), threads and shared memory.
template <typename T>
struct PlaneEntry {
    int nx = 0, ny = 0, nt = 0;
    int xe = 0, xr[3] = {1, 1, 1};
    int ye = 0, yr[3] = {1, 1, 1};
    int cs = 1;  // CTAs per plane (a thread-block cluster when > 1)
    size_t smem = 0;
    PlaneKernel<T> k[3] = {nullptr, nullptr, nullptr};  // by PlaneMode
    // batched form (one-CTA planes only): every member of a class, by PlaneMode
    PlaneBatchKernel<T> kb[3] = {nullptr, nullptr, nullptr};
    int kb_bps = 0;  // resident CTAs per SM
};

// Plane pass entry with NT threads per CTA and CS CTAs per plane (1: plane_kernel,
// else a cluster of CS).
template <typename T, int NX, int EX, int RX0, int RX1, int RX2, int NY, int EY, int RY0, int RY1, int RY2, int NT,
          int CS = 1>
PlaneEntry<T> make_plane_entry() {
    PlaneEntry<T> p;
    p.nx = NX;
    p.ny = NY;
    p.nt = NT;
    p.cs = CS;
    p.xe = EX;
    p.xr[0] = RX0;
    p.xr[1] = RX1;
    p.xr[2] = RX2;
    p.ye = EY;
    p.yr[0] = RY0;
    p.yr[1] = RY1;
    p.yr[2] = RY2;
    if constexpr (CS == 1) {
        p.smem = plane_smem<T, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>();
        p.k[PL_START] = plane_kernel<T, PL_START, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        p.k[PL_MID] = plane_kernel<T, PL_MID, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        p.k[PL_END] = plane_kernel<T, PL_END, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        p.kb[PL_START] = plane_batch_kernel<T, PL_START, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        p.kb[PL_MID] = plane_batch_kernel<T, PL_MID, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        p.kb[PL_END] = plane_batch_kernel<T, PL_END, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, NT>;
        for (auto k : p.kb) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&p.kb_bps, p.kb[PL_MID], NT, p.smem,
                                                              cudaOccupancyDefault);
    } else {
        p.smem = cluster_plane_smem<T, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, CS, NT>();
        p.k[PL_START] = cluster_plane_kernel<T, PL_START, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, CS, NT>;
        p.k[PL_MID] = cluster_plane_kernel<T, PL_MID, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, CS, NT>;
        p.k[PL_END] = cluster_plane_kernel<T, PL_END, NX, EX, RX0, RX1, RX2, NY, EY, RY0, RY1, RY2, CS, NT>;
    }
    for (auto k : p.k) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    cudaGetLastError();
    return p;
}

void register_planes(std::vector<PlaneEntry<float>>& f, std::vector<PlaneEntry<double>>& d);

}  // namespace sesk
