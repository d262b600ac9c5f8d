// Non-template kernels of the solver (table builders, final reductions).
// Included by ses_gpu.cu only: __global__ functions defined here have one
// definition in the library.
#pragma once

#include "ses_pass.cuh"

namespace sesk {

// Fixed-order final sum of per-CTA partial rows: out[q] = sum_b partials[b][q].
__global__ void finalize_kernel(const double* __restrict__ partials, int nblocks, int nr, double* out) {
    const int q = threadIdx.x;
    if (q < nr) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partials[(size_t)b * nr + q];
        out[q] = s;
    }
}

// ---------------------------------------------------------------------------
// FP64 table builders.  Phase arguments use round-to-nearest intrinsics in the
// reference's evaluation order (no FMA contraction), so theta is bitwise the
// reference's: -0.5*V*dt (propagator.ixx:81) and
// -0.5*(kx^2+ky^2+kz^2)/mass*dt (propagator.ixx:95-96).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double theta_v(double V, double dt) {
    return __dmul_rn(__dmul_rn(-0.5, V), dt);
}

__device__ __forceinline__ double theta_k(double ksq, double mass, double dt) {
    return __dmul_rn(__ddiv_rn(__dmul_rn(-0.5, ksq), mass), dt);
}

// cis(theta) - 1 without cancellation: (-2 sin^2(theta/2), sin(theta))
__device__ __forceinline__ cx<double> cis_minus_one(double th) {
    double s2, c2;
    sincos(0.5 * th, &s2, &c2);
    return mk<double>(-2.0 * s2 * s2, 2.0 * s2 * c2);
}

__global__ void build_vtab_c128(const double* __restrict__ V, cx<double>* out, long long N, double dt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        double s, c;
        sincos(theta_v(V[i], dt), &s, &c);
        out[i] = mk<double>(c, s);
    }
}

__global__ void build_vtab_c64(const double* __restrict__ V, cx<float>* out, long long N, double dt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        out[i] = narrow<float>(cis_minus_one(theta_v(V[i], dt)));
    }
}

// Imaginary time (imaginary_time.ixx:71-95): real weights exp(-V dtau/2) and
// exp(-k^2 dtau/(2m)) in the tables' formats -- complex128 (w, 0), complex64
// the delta (w - 1, 0) from expm1, so small weights-minus-one stay accurate.
__global__ void build_vtab_imag_c128(const double* __restrict__ V, cx<double>* out, long long N, double dtau) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = mk<double>(exp(theta_v(V[i], dtau)), 0.0);
}

__global__ void build_vtab_imag_c64(const double* __restrict__ V, cx<float>* out, long long N, double dtau) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = mk<float>((float)expm1(theta_v(V[i], dtau)), 0.0f);
}

__global__ void build_axis_tables_imag(int n, double dtau, double mass, const double* kv, cx<double>* kd) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) kd[j] = mk<double>(expm1(theta_k(__dmul_rn(kv[j], kv[j]), mass, dtau)), 0.0);
}

// psi *= 1 / sqrt(sum |psi|^2 dV), the sum taken from sums[0] on the device;
// sums[0] is kept for the energy estimate.
template <typename T>
__global__ void renormalize_kernel(cx<T>* psi, long long N, const double* __restrict__ sums, double dv) {
    const double s = 1.0 / sqrt(sums[0] * dv);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        psi[i] = scale_d(psi[i], s);
}

// |psi|^2 of the plane index `at` along `axis` (0/1/2) of an nx x ny x nz field,
// the other two axes in their own order (first the lower axis), as FP32.
template <typename T>
__global__ void density_slice_kernel(const cx<T>* __restrict__ psi, int nx, int ny, int nz, int axis, int at,
                                     float* out) {
    const int na = axis == 0 ? ny : nx, nb = axis == 2 ? ny : nz;
    const long long cnt = (long long)na * nb;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
         t += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(t % na), b = (int)(t / na);
        const int i = axis == 0 ? at : a, j = axis == 0 ? a : (axis == 1 ? at : b), k = axis == 2 ? at : b;
        const cx<double> p = widen(psi[i + (long long)nx * (j + (long long)ny * k)]);
        out[t] = (float)(p.x * p.x + p.y * p.y);
    }
}

// per-axis wavenumbers k_j = (2 pi / L) * (j if 2j < n else j - n)  (spectral.ixx:14-23)
// and kinetic deltas cis(-k^2 dt/(2m)) - 1
__global__ void build_axis_tables(double xmin, double xmax, int n, double dt, double mass,
                                  double* kv, cx<double>* kd) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        const double dk = __ddiv_rn(2.0 * 3.14159265358979323846, __dsub_rn(xmax, xmin));
        const int shifted = (2 * j < n) ? j : j - n;
        const double k = __dmul_rn(dk, (double)shifted);
        kv[j] = k;
        kd[j] = cis_minus_one(theta_k(__dmul_rn(k, k), mass, dt));
    }
}

template <typename T>
__global__ void build_twiddles(int n, cx<T>* tw) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double s, c;
        sincospi(-2.0 * (double)t / (double)n, &s, &c);
        tw[t] = mk<T>((T)c, (T)s);
    }
}

// Long 1D line of N = N1 N2 points in the four-step layout: the element stored
// at (k1, k2) after the forward transform (flat k1 + N1 k2) is frequency
// k = k2 + N2 k1; its kinetic delta is cis(-k_phys^2 dt/(2m)) - 1 with k_phys the
// line's fftfreq wavenumber kv[k].  The twiddle of element (n1, k2) is
// W_N^{n1 k2} = e^{-2 pi i (n1 k2 mod N)/N}, in FP64 (complex64: hi + lo parts).
template <typename T>
__global__ void build_long_tables(const double* __restrict__ kv, int n1, int n2, double dt, double mass,
                                  cx<T>* kfull, cx<T>* tw_hi, cx<T>* tw_lo) {
    const long long N = (long long)n1 * n2;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < N;
         f += (long long)gridDim.x * blockDim.x) {
        const long long a = f % n1, b = f / n1;  // (k1, k2) for kfull, (n1, k2) for the twiddle
        const double k = kv[b + (long long)n2 * a];
        const cx<double> d = cis_minus_one(theta_k(__dmul_rn(k, k), mass, dt));
        kfull[f] = mk<T>((T)d.x, (T)d.y);
        const long long t = (a * b) % N;
        double sn, cs;
        sincospi(-2.0 * (double)t / (double)N, &sn, &cs);
        tw_hi[f] = mk<T>((T)cs, (T)sn);
        if (tw_lo) tw_lo[f] = mk<T>((T)(cs - (double)(T)cs), (T)(sn - (double)(T)sn));
    }
}

// Full-N reference tables (propagator-tables surface).
__global__ void build_full_tables(const double* __restrict__ V, const double* __restrict__ kvx,
                                  const double* __restrict__ kvy, const double* __restrict__ kvz,
                                  int nx, int ny, long long N, double dt, double mass,
                                  cx<double>* half_v, cx<double>* kin) {
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < N;
         f += (long long)gridDim.x * blockDim.x) {
        double s, c;
        if (half_v) {
            sincos(theta_v(V[f], dt), &s, &c);
            half_v[f] = mk<double>(c, s);
        }
        if (kin) {
            const long long line = f / nx;
            const int i = (int)(f - line * nx);
            const long long k = line / ny;
            const int j = (int)(line - k * ny);
            const double a = kvx[i], b = kvy[j], cz = kvz[k];
            const double ksq = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(cz, cz));
            sincos(theta_k(ksq, mass, dt), &s, &c);
            kin[f] = mk<double>(c, s);
        }
    }
}

}  // namespace sesk
