/* CPU FP64 oracle for the Strang split-operator step -- TEST INFRASTRUCTURE.
 *
 * Restates the reference core's algorithm (parkyere/ShoeridingerEquationSolver,
 * core/src/ modules) in plain C so tests can check the CUDA path against it on any
 * 2^a 3^b 5^c grid.  Power-of-two FFT lengths follow the reference's radix-2
 * steps and operation order exactly (bitwise-equal results when compiled with
 * the reference's flags -ffp-contract=off); other lengths use a mixed-radix
 * extension, pinned against an O(n^2) long-double DFT.  Built by
 * oracle/Makefile into oracle/libses_oracle.so.  The product never links it.
 */
#include "ses_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef struct {
    double re, im;
} cplx;

static const double kPi = 3.14159265358979323846;
/* integral of 1/r over the unit cube (potential.ixx:99-100) */
static const double kCoulombCellAverage = 2.3800774;

static inline cplx cmul(cplx a, cplx b) {
    /* (a.re b.re - a.im b.im, a.re b.im + a.im b.re): std::complex product
     * under -fcx-limited-range */
    cplx r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}

static inline double spacing(double lo, double hi, int n) { return (hi - lo) / n; }
static inline double coord(double lo, double hi, int n, int i) { return lo + i * spacing(lo, hi, n); }
static inline size_t flat(const int* n, int i, int j, int k) {
    return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k);
}
static inline size_t total(const int* n) { return (size_t)n[0] * (size_t)n[1] * (size_t)n[2]; }
static inline double cell_volume(const double* box, const int* n) {
    return spacing(box[0], box[1], n[0]) * spacing(box[2], box[3], n[1]) *
           spacing(box[4], box[5], n[2]);
}

int seso_supported_length(size_t n) {
    if (n == 0) return -1;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    while (n % 5 == 0) n /= 5;
    return n == 1 ? 0 : -1;
}

static int is_pow2(size_t n) { return (n & (n - 1)) == 0; }

void seso_fft_twiddles(size_t n, double* w) {
    const double ang = -2.0 * kPi / (double)n;
    for (size_t j = 0; j < n / 2; ++j) {
        const double th = ang * (double)j;
        w[2 * j] = cos(th);
        w[2 * j + 1] = sin(th);
    }
}

/* radix-2 DIT: bit-reversal permutation then len = 2..n butterfly stages using
 * w[j * n/len] (same steps as fft.ixx:39-73) */
static void fft_pow2(cplx* a, size_t n, const cplx* w) {
    if (n < 2) return;
    size_t j = 0;
    for (size_t i = 1; i < n; ++i) {
        size_t bit = n >> 1;
        while (j & bit) {
            j ^= bit;
            bit >>= 1;
        }
        j ^= bit;
        if (i < j) {
            cplx t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2, stride = n / len;
        for (size_t base = 0; base < n; base += len) {
            for (size_t q = 0; q < half; ++q) {
                const cplx u = a[base + q];
                const cplx v = cmul(a[base + q + half], w[q * stride]);
                a[base + q].re = u.re + v.re;
                a[base + q].im = u.im + v.im;
                a[base + q + half].re = u.re - v.re;
                a[base + q + half].im = u.im - v.im;
            }
        }
    }
}

/* Mixed-radix recursive decimation in time (extension for 3 | n or 5 | n):
 * X[k + q m] = sum_r W_n^{r (k + q m)} Y_r[k], Y_r = FFT_m(x[r::p]),
 * p = smallest prime factor, m = n/p.  wfull[t] = cis(-2 pi t / N_top). */
static void fft_mixed_rec(const cplx* in, size_t istride, cplx* out, size_t n, const cplx* wfull,
                          size_t ntop, cplx* tmp) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    size_t p = (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5;
    size_t m = n / p;
    for (size_t r = 0; r < p; ++r)
        fft_mixed_rec(in + r * istride, istride * p, out + r * m, m, wfull, ntop, tmp);
    const size_t wstep = ntop / n;
    for (size_t k = 0; k < m; ++k) {
        for (size_t q = 0; q < p; ++q) {
            const size_t kk = k + q * m;
            cplx acc = out[k];
            for (size_t r = 1; r < p; ++r) {
                const size_t t = ((r * kk) % n) * wstep;
                const cplx v = cmul(out[r * m + k], wfull[t]);
                acc.re += v.re;
                acc.im += v.im;
            }
            tmp[kk] = acc;
        }
    }
    memcpy(out, tmp, n * sizeof(cplx));
}

static void fft_line(cplx* a, size_t n, const cplx* w, cplx* scratch) {
    /* w: pow2 -> half table (seso_fft_twiddles); mixed -> full table cis(-2 pi t/n) */
    if (is_pow2(n)) {
        fft_pow2(a, n, w);
        return;
    }
    cplx* out = scratch;
    cplx* tmp = scratch + n;
    fft_mixed_rec(a, 1, out, n, w, n, tmp);
    memcpy(a, out, n * sizeof(cplx));
}

/* Worker threads for independent lines and elements.  Every line (element) is
 * computed by the same serial code whichever thread runs it, so results are
 * bit-identical to a single-threaded run -- the property the reference's
 * deterministic pool guarantees (core/src/parallel.ixx:14-16).  SESO_THREADS
 * sets the count (default: the online cores). */
typedef void (*range_fn)(void* ctx, size_t begin, size_t end);

enum { kMaxThreads = 256 };

static int oracle_threads(void) {
    const char* e = getenv("SESO_THREADS");
    long t = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
    if (t < 1) t = 1;
    if (t > kMaxThreads) t = kMaxThreads;
    return (int)t;
}

typedef struct {
    range_fn fn;
    void* ctx;
    size_t begin, end;
} range_job;

static void* run_range(void* p) {
    range_job* j = (range_job*)p;
    j->fn(j->ctx, j->begin, j->end);
    return NULL;
}

/* fn over [0, count) in contiguous chunks; `work` = rough cost of the whole call in
 * element operations, below which threads are not worth starting */
static void par_for(size_t count, size_t work, range_fn fn, void* ctx) {
    size_t t = (size_t)oracle_threads();
    if (t > count) t = count;
    if (t <= 1 || work < ((size_t)1 << 16)) {
        fn(ctx, 0, count);
        return;
    }
    pthread_t th[kMaxThreads];
    range_job jobs[kMaxThreads];
    int started[kMaxThreads];
    for (size_t i = 0; i < t; ++i) {
        jobs[i].fn = fn;
        jobs[i].ctx = ctx;
        jobs[i].begin = count * i / t;
        jobs[i].end = count * (i + 1) / t;
        started[i] = i > 0 && pthread_create(&th[i], NULL, run_range, &jobs[i]) == 0;
    }
    run_range(&jobs[0]);
    for (size_t i = 1; i < t; ++i) {
        if (started[i]) pthread_join(th[i], NULL);
        else run_range(&jobs[i]);  /* a thread that could not start runs here */
    }
}

static cplx* make_table(size_t n) {
    if (is_pow2(n)) {
        cplx* w = (cplx*)malloc((n / 2 + 1) * sizeof(cplx));
        seso_fft_twiddles(n, (double*)w);
        return w;
    }
    cplx* w = (cplx*)malloc(n * sizeof(cplx));
    for (size_t t = 0; t < n; ++t) {
        const double th = -2.0 * kPi * (double)t / (double)n;
        w[t].re = cos(th);
        w[t].im = sin(th);
    }
    return w;
}

int seso_fft1d(double* a, size_t n) {
    if (seso_supported_length(n) != 0) return -1;
    if (n < 2) return 0;
    cplx* w = make_table(n);
    cplx* s = (cplx*)malloc(2 * n * sizeof(cplx));
    fft_line((cplx*)a, n, w, s);
    free(s);
    free(w);
    return 0;
}

typedef struct {
    cplx* a;
    const cplx* ph;
    const double* m;
    double inv;
} elem_ctx;

static void conj_range(void* p, size_t b, size_t e) {
    cplx* a = ((elem_ctx*)p)->a;
    for (size_t i = b; i < e; ++i) a[i].im = -a[i].im;
}

static void conj_scale_range(void* p, size_t b, size_t e) {
    const elem_ctx* c = (const elem_ctx*)p;
    for (size_t i = b; i < e; ++i) {
        c->a[i].re = c->inv * c->a[i].re;
        c->a[i].im = c->inv * -c->a[i].im;
    }
}

static void phase_range(void* p, size_t b, size_t e) {
    const elem_ctx* c = (const elem_ctx*)p;
    for (size_t i = b; i < e; ++i) c->a[i] = cmul(c->a[i], c->ph[i]);
}

static void mask_range(void* p, size_t b, size_t e) {
    const elem_ctx* c = (const elem_ctx*)p;
    for (size_t i = b; i < e; ++i) {
        c->a[i].re *= c->m[i];
        c->a[i].im *= c->m[i];
    }
}

static void conj_all(cplx* a, size_t n) {
    elem_ctx c = {a, NULL, NULL, 0.0};
    par_for(n, n, conj_range, &c);
}

static void conj_scale_all(cplx* a, size_t n) {
    elem_ctx c = {a, NULL, NULL, 1.0 / (double)n};
    par_for(n, n, conj_scale_range, &c);
}

int seso_ifft1d(double* a, size_t n) {
    if (seso_supported_length(n) != 0) return -1;
    conj_all((cplx*)a, n);
    seso_fft1d(a, n);
    conj_scale_all((cplx*)a, n);
    return 0;
}

typedef struct {
    cplx* a;
    const int* n;
    const cplx* w;
    int axis;
} lines_ctx;

/* lines [begin, end) of one axis: x lines in place, y and z lines through a
 * gathered scratch line */
static void fft_lines(void* p, size_t begin, size_t end) {
    const lines_ctx* c = (const lines_ctx*)p;
    const int* n = c->n;
    const int len = n[c->axis];
    cplx* line = (cplx*)malloc((size_t)len * sizeof(cplx));
    cplx* scr = (cplx*)malloc(2 * (size_t)len * sizeof(cplx));
    for (size_t m = begin; m < end; ++m) {
        if (c->axis == 0) {
            fft_line(c->a + m * (size_t)n[0], (size_t)len, c->w, scr);
            continue;
        }
        /* y: line m = (i, k) with m = i + nx k; z: line m = (i, j) with m = i + nx j */
        const int i = (int)(m % (size_t)n[0]), o = (int)(m / (size_t)n[0]);
        for (int e = 0; e < len; ++e) line[e] = c->a[c->axis == 1 ? flat(n, i, e, o) : flat(n, i, o, e)];
        fft_line(line, (size_t)len, c->w, scr);
        for (int e = 0; e < len; ++e) c->a[c->axis == 1 ? flat(n, i, e, o) : flat(n, i, o, e)] = line[e];
    }
    free(scr);
    free(line);
}

/* Forward unnormalised 3D transform: all x lines, then all y lines, then all z
 * lines (core/src/fft.ixx:102-173). */
int seso_fft3d(double* data, const int* n) {
    for (int ax = 0; ax < 3; ++ax)
        if (seso_supported_length((size_t)n[ax]) != 0) return -1;
    const size_t N = total(n);
    for (int ax = 0; ax < 3; ++ax) {
        if (n[ax] <= 1) continue;
        cplx* w = make_table((size_t)n[ax]);
        lines_ctx c = {(cplx*)data, n, w, ax};
        par_for(N / (size_t)n[ax], N * 8, fft_lines, &c);
        free(w);
    }
    return 0;
}

int seso_ifft3d(double* data, const int* n) {
    for (int ax = 0; ax < 3; ++ax)
        if (seso_supported_length((size_t)n[ax]) != 0) return -1;
    const size_t N = total(n);
    conj_all((cplx*)data, N);
    seso_fft3d(data, n);
    conj_scale_all((cplx*)data, N);
    return 0;
}

void seso_dft_naive(const double* in, double* out, size_t n, int inverse) {
    const long double tw = (inverse ? 2.0L : -2.0L) * 3.141592653589793238462643383279502884L;
    for (size_t k = 0; k < n; ++k) {
        long double sr = 0.0L, si = 0.0L;
        for (size_t j = 0; j < n; ++j) {
            const long double th = tw * (long double)((j * k) % n) / (long double)n;
            const long double c = cosl(th), s = sinl(th);
            sr += (long double)in[2 * j] * c - (long double)in[2 * j + 1] * s;
            si += (long double)in[2 * j] * s + (long double)in[2 * j + 1] * c;
        }
        if (inverse) {
            sr /= (long double)n;
            si /= (long double)n;
        }
        out[2 * k] = (double)sr;
        out[2 * k + 1] = (double)si;
    }
}

void seso_wavenumbers(double xmin, double xmax, int n, double* k) {
    const double dk = 2.0 * kPi / (xmax - xmin);
    for (int j = 0; j < n; ++j) {
        const int shifted = (2 * j < n) ? j : j - n;
        k[j] = dk * shifted;
    }
}

void seso_tables3d(const double* box, const int* n, const double* V, double dt, double mass,
                   double* half_v, double* kin) {
    const size_t N = total(n);
    if (half_v) {
        for (size_t i = 0; i < N; ++i) {
            const double th = -0.5 * V[i] * dt;
            half_v[2 * i] = cos(th);
            half_v[2 * i + 1] = sin(th);
        }
    }
    if (kin) {
        double* kx = (double*)malloc((size_t)n[0] * sizeof(double));
        double* ky = (double*)malloc((size_t)n[1] * sizeof(double));
        double* kz = (double*)malloc((size_t)n[2] * sizeof(double));
        seso_wavenumbers(box[0], box[1], n[0], kx);
        seso_wavenumbers(box[2], box[3], n[1], ky);
        seso_wavenumbers(box[4], box[5], n[2], kz);
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i) {
                    const double s = kx[i] * kx[i] + ky[j] * ky[j] + kz[k] * kz[k];
                    const double th = -0.5 * s / mass * dt;
                    const size_t f = flat(n, i, j, k);
                    kin[2 * f] = cos(th);
                    kin[2 * f + 1] = sin(th);
                }
        free(kx);
        free(ky);
        free(kz);
    }
}

static void apply_phase(cplx* a, const cplx* ph, size_t N) {
    elem_ctx c = {a, ph, NULL, 0.0};
    par_for(N, N, phase_range, &c);
}

int seso_step3d(const double* box, const int* n, const double* V, double dt, double mass,
                const double* mask, double* psi, int nsteps) {
    for (int ax = 0; ax < 3; ++ax)
        if (seso_supported_length((size_t)n[ax]) != 0) return -1;
    const size_t N = total(n);
    cplx* half = (cplx*)malloc(N * sizeof(cplx));
    cplx* kin = (cplx*)malloc(N * sizeof(cplx));
    seso_tables3d(box, n, V, dt, mass, (double*)half, (double*)kin);
    cplx* a = (cplx*)psi;
    for (int s = 0; s < nsteps; ++s) {
        apply_phase(a, half, N);
        seso_fft3d(psi, n);
        apply_phase(a, kin, N);
        seso_ifft3d(psi, n);
        apply_phase(a, half, N);
        if (mask) {
            elem_ctx c = {a, NULL, mask, 0.0};
            par_for(N, N, mask_range, &c);
        }
    }
    free(half);
    free(kin);
    return 0;
}

/* Dipole-driven Strang steps (core/src/drive.ixx:25-65): kick(t) . step . kick(t + dt),
 * kick = psi * cis(-theta u), theta = amplitude cos(omega t) dt/2, u = axis . r. */
static void dipole_halfkick(cplx* a, const double* box, const int* n, const double* axis, double amplitude,
                            double omega, double t, double dt) {
    const double theta = amplitude * cos(omega * t) * 0.5 * dt;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double u = axis[0] * coord(box[0], box[1], n[0], i) + axis[1] * coord(box[2], box[3], n[1], j) +
                                 axis[2] * coord(box[4], box[5], n[2], k);
                const double ang = -theta * u;
                const cplx c = {cos(ang), sin(ang)};
                const size_t f = flat(n, i, j, k);
                a[f] = cmul(a[f], c);
            }
}

int seso_driven_step3d(const double* box, const int* n, const double* V, double dt, double mass,
                       const double* axis, double amplitude, double omega, double t0, double* psi,
                       int nsteps) {
    for (int ax = 0; ax < 3; ++ax)
        if (seso_supported_length((size_t)n[ax]) != 0) return -1;
    const size_t N = total(n);
    cplx* half = (cplx*)malloc(N * sizeof(cplx));
    cplx* kin = (cplx*)malloc(N * sizeof(cplx));
    seso_tables3d(box, n, V, dt, mass, (double*)half, (double*)kin);
    cplx* a = (cplx*)psi;
    for (int s = 0; s < nsteps; ++s) {
        const double t = t0 + s * dt;
        dipole_halfkick(a, box, n, axis, amplitude, omega, t, dt);
        apply_phase(a, half, N);
        seso_fft3d(psi, n);
        apply_phase(a, kin, N);
        seso_ifft3d(psi, n);
        apply_phase(a, half, N);
        dipole_halfkick(a, box, n, axis, amplitude, omega, t + dt, dt);
    }
    free(half);
    free(kin);
    return 0;
}

int seso_step1d(double xmin, double xmax, int n, const double* V, double dt, const double* mask,
                double* psi, int nsteps) {
    if (seso_supported_length((size_t)n) != 0) return -1;
    cplx* half = (cplx*)malloc((size_t)n * sizeof(cplx));
    cplx* kin = (cplx*)malloc((size_t)n * sizeof(cplx));
    double* k = (double*)malloc((size_t)n * sizeof(double));
    seso_wavenumbers(xmin, xmax, n, k);
    for (int i = 0; i < n; ++i) {
        const double th = -0.5 * V[i] * dt;
        half[i].re = cos(th);
        half[i].im = sin(th);
        const double tk = -0.5 * k[i] * k[i] * dt;
        kin[i].re = cos(tk);
        kin[i].im = sin(tk);
    }
    cplx* a = (cplx*)psi;
    for (int s = 0; s < nsteps; ++s) {
        apply_phase(a, half, (size_t)n);
        seso_fft1d(psi, (size_t)n);
        apply_phase(a, kin, (size_t)n);
        seso_ifft1d(psi, (size_t)n);
        apply_phase(a, half, (size_t)n);
        if (mask) {
            for (int i = 0; i < n; ++i) {
                a[i].re *= mask[i];
                a[i].im *= mask[i];
            }
        }
    }
    free(half);
    free(kin);
    free(k);
    return 0;
}

static void normalize3d(const double* box, const int* n, double* psi) {
    const double n2 = seso_norm3d(box, n, psi);
    if (n2 <= 0.0) return;
    const double inv = 1.0 / sqrt(n2);
    const size_t N = total(n);
    for (size_t i = 0; i < 2 * N; ++i) psi[i] = inv * psi[i];
}

int seso_relax3d(const double* box, const int* n, const double* V, double dtau, double mass,
                 double* psi, int nsteps) {
    for (int ax = 0; ax < 3; ++ax)
        if (seso_supported_length((size_t)n[ax]) != 0) return -1;
    const size_t N = total(n);
    double* half = (double*)malloc(N * sizeof(double));
    double* kin = (double*)malloc(N * sizeof(double));
    double* kx = (double*)malloc((size_t)n[0] * sizeof(double));
    double* ky = (double*)malloc((size_t)n[1] * sizeof(double));
    double* kz = (double*)malloc((size_t)n[2] * sizeof(double));
    seso_wavenumbers(box[0], box[1], n[0], kx);
    seso_wavenumbers(box[2], box[3], n[1], ky);
    seso_wavenumbers(box[4], box[5], n[2], kz);
    for (size_t i = 0; i < N; ++i) half[i] = exp(-0.5 * V[i] * dtau);
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i)
                kin[flat(n, i, j, k)] =
                    exp(-0.5 * (kx[i] * kx[i] + ky[j] * ky[j] + kz[k] * kz[k]) / mass * dtau);
    for (int s = 0; s < nsteps; ++s) {
        for (size_t i = 0; i < N; ++i) {
            psi[2 * i] = half[i] * psi[2 * i];
            psi[2 * i + 1] = half[i] * psi[2 * i + 1];
        }
        seso_fft3d(psi, n);
        for (size_t i = 0; i < N; ++i) {
            psi[2 * i] = kin[i] * psi[2 * i];
            psi[2 * i + 1] = kin[i] * psi[2 * i + 1];
        }
        seso_ifft3d(psi, n);
        for (size_t i = 0; i < N; ++i) {
            psi[2 * i] = half[i] * psi[2 * i];
            psi[2 * i + 1] = half[i] * psi[2 * i + 1];
        }
        normalize3d(box, n, psi);
    }
    free(half);
    free(kin);
    free(kx);
    free(ky);
    free(kz);
    return 0;
}

/* ---------------- potentials and masks ---------------- */

void seso_harmonic3d(const double* box, const int* n, double omega, const double* c, double* v) {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double dx = coord(box[0], box[1], n[0], i) - c[0];
                const double dy = coord(box[2], box[3], n[1], j) - c[1];
                const double dz = coord(box[4], box[5], n[2], k) - c[2];
                v[flat(n, i, j, k)] = 0.5 * omega * omega * (dx * dx + dy * dy + dz * dz);
            }
}

void seso_soft_coulomb3d(const double* box, const int* n, double Z, double a, const double* c,
                         double* v) {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double dx = coord(box[0], box[1], n[0], i) - c[0];
                const double dy = coord(box[2], box[3], n[1], j) - c[1];
                const double dz = coord(box[4], box[5], n[2], k) - c[2];
                v[flat(n, i, j, k)] = -Z / sqrt(dx * dx + dy * dy + dz * dz + a * a);
            }
}

void seso_regularized_coulomb3d(const double* box, const int* n, double Z, const double* c,
                                double* v) {
    const double h = spacing(box[0], box[1], n[0]);
    const double center = -Z * kCoulombCellAverage / h;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double dx = coord(box[0], box[1], n[0], i) - c[0];
                const double dy = coord(box[2], box[3], n[1], j) - c[1];
                const double dz = coord(box[4], box[5], n[2], k) - c[2];
                const double r = sqrt(dx * dx + dy * dy + dz * dz);
                v[flat(n, i, j, k)] = (r < 1e-6 * h) ? center : -Z / r;
            }
}

void seso_barrier3d(const double* box, const int* n, double v0, double xlo, double xhi, double* v) {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double x = coord(box[0], box[1], n[0], i);
                v[flat(n, i, j, k)] = (x >= xlo && x < xhi) ? v0 : 0.0;
            }
}

void seso_stark_fold3d(const double* box, const int* n, double e, double* v) {
    for (int k = 0; k < n[2]; ++k) {
        const double ez = e * coord(box[4], box[5], n[2], k);
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) v[flat(n, i, j, k)] += ez;
    }
}

void seso_stadium3d(const double* box, const int* n, double half_len, double r, double v_out,
                    double* v) {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double x = coord(box[0], box[1], n[0], i);
                const double y = coord(box[2], box[3], n[1], j);
                const double cx = x < -half_len ? -half_len : (x > half_len ? half_len : x);
                const double sdf = hypot(x - cx, y) - r;
                v[flat(n, i, j, k)] = sdf > 0.0 ? v_out : 0.0;
            }
}

void seso_harmonic1d(double xmin, double xmax, int n, double omega, double x0, double* v) {
    for (int i = 0; i < n; ++i) {
        const double dx = coord(xmin, xmax, n, i) - x0;
        v[i] = 0.5 * omega * omega * dx * dx;
    }
}

void seso_morse1d(double xmin, double xmax, int n, double d, double alpha, double x0, double* v) {
    for (int i = 0; i < n; ++i) {
        const double q = 1.0 - exp(-alpha * (coord(xmin, xmax, n, i) - x0));
        v[i] = d * q * q;
    }
}

void seso_double_well1d(double xmin, double xmax, int n, double vb, double a, double* v) {
    for (int i = 0; i < n; ++i) {
        const double s = coord(xmin, xmax, n, i) / a;
        const double q = s * s - 1.0;
        v[i] = vb * q * q;
    }
}

void seso_poschl_teller1d(double xmin, double xmax, int n, double v0, double a, double x0,
                          double* v) {
    for (int i = 0; i < n; ++i) {
        const double c = cosh((coord(xmin, xmax, n, i) - x0) / a);
        v[i] = -v0 / (c * c);
    }
}

void seso_mask1d(double xmin, double xmax, int n, double width, int profile, double* m) {
    if (n == 1) {
        m[0] = 1.0; /* collapsed axis: no walls */
        return;
    }
    for (int i = 0; i < n; ++i) {
        const double x = coord(xmin, xmax, n, i);
        const double d_lo = x - xmin, d_hi = xmax - x;
        const double d = d_lo < d_hi ? d_lo : d_hi;
        if (d >= width) {
            m[i] = 1.0;
            continue;
        }
        const double t = d / width;
        const double s = sin(0.5 * kPi * t); /* = cos(pi/2 (1 - t)) */
        m[i] = profile == 0 ? s * s : pow(s, 0.125);
    }
}

void seso_mask3d(const double* box, const int* n, double width, int profile, double* m) {
    double* mx = (double*)malloc((size_t)n[0] * sizeof(double));
    double* my = (double*)malloc((size_t)n[1] * sizeof(double));
    double* mz = (double*)malloc((size_t)n[2] * sizeof(double));
    seso_mask1d(box[0], box[1], n[0], width, profile, mx);
    seso_mask1d(box[2], box[3], n[1], width, profile, my);
    seso_mask1d(box[4], box[5], n[2], width, profile, mz);
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) m[flat(n, i, j, k)] = mx[i] * my[j] * mz[k];
    free(mx);
    free(my);
    free(mz);
}

/* ---------------- initial states ---------------- */

static double envelope(double u, double u0, double s) {
    return pow(2.0 * kPi * s * s, -0.25) * exp(-(u - u0) * (u - u0) / (4.0 * s * s));
}

void seso_gaussian3d(const double* box, const int* n, const double* r0, const double* sigma,
                     const double* k0, double* psi) {
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double x = coord(box[0], box[1], n[0], i);
                const double y = coord(box[2], box[3], n[1], j);
                const double z = coord(box[4], box[5], n[2], k);
                const double env = envelope(x, r0[0], sigma[0]) * envelope(y, r0[1], sigma[1]) *
                                   envelope(z, r0[2], sigma[2]);
                const double ph = k0[0] * x + k0[1] * y + k0[2] * z;
                const size_t f = flat(n, i, j, k);
                psi[2 * f] = env * cos(ph);
                psi[2 * f + 1] = env * sin(ph);
            }
    normalize3d(box, n, psi);
}

void seso_gaussian1d(double xmin, double xmax, int n, double x0, double sigma, double k0,
                     double* psi) {
    const double amp = pow(2.0 * kPi * sigma * sigma, -0.25);
    for (int i = 0; i < n; ++i) {
        const double x = coord(xmin, xmax, n, i);
        const double env = amp * exp(-(x - x0) * (x - x0) / (4.0 * sigma * sigma));
        psi[2 * i] = env * cos(k0 * x);
        psi[2 * i + 1] = env * sin(k0 * x);
    }
    const double inv = 1.0 / sqrt(seso_norm1d(xmin, xmax, n, psi));
    for (int i = 0; i < 2 * n; ++i) psi[i] = inv * psi[i];
}

/* ---------------- observables ---------------- */

static inline double ratio(double num, double den) { return den > 0.0 ? num / den : 0.0; }

double seso_norm3d(const double* box, const int* n, const double* psi) {
    const size_t N = total(n);
    double acc = 0.0;
    for (size_t i = 0; i < N; ++i) acc += psi[2 * i] * psi[2 * i] + psi[2 * i + 1] * psi[2 * i + 1];
    return acc * cell_volume(box, n);
}

double seso_norm1d(double xmin, double xmax, int n, const double* psi) {
    double acc = 0.0;
    for (int i = 0; i < n; ++i) acc += psi[2 * i] * psi[2 * i] + psi[2 * i + 1] * psi[2 * i + 1];
    return acc * spacing(xmin, xmax, n);
}

double seso_mean_energy3d(const double* box, const int* n, const double* psi, const double* V,
                          double mass) {
    const size_t N = total(n);
    double num_v = 0.0, den_x = 0.0;
    for (size_t i = 0; i < N; ++i) {
        const double w = psi[2 * i] * psi[2 * i] + psi[2 * i + 1] * psi[2 * i + 1];
        num_v += V[i] * w;
        den_x += w;
    }
    double* phi = (double*)malloc(2 * N * sizeof(double));
    memcpy(phi, psi, 2 * N * sizeof(double));
    seso_fft3d(phi, n);
    double* kx = (double*)malloc((size_t)n[0] * sizeof(double));
    double* ky = (double*)malloc((size_t)n[1] * sizeof(double));
    double* kz = (double*)malloc((size_t)n[2] * sizeof(double));
    seso_wavenumbers(box[0], box[1], n[0], kx);
    seso_wavenumbers(box[2], box[3], n[1], ky);
    seso_wavenumbers(box[4], box[5], n[2], kz);
    double num_t = 0.0, den_k = 0.0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const size_t f = flat(n, i, j, k);
                const double w = phi[2 * f] * phi[2 * f] + phi[2 * f + 1] * phi[2 * f + 1];
                num_t += 0.5 * (kx[i] * kx[i] + ky[j] * ky[j] + kz[k] * kz[k]) / mass * w;
                den_k += w;
            }
    free(phi);
    free(kx);
    free(ky);
    free(kz);
    return ratio(num_v, den_x) + ratio(num_t, den_k);
}

double seso_mean_energy1d(double xmin, double xmax, int n, const double* psi, const double* V) {
    const double box[6] = {xmin, xmax, 0.0, 1.0, 0.0, 1.0};
    const int nn[3] = {n, 1, 1};
    return seso_mean_energy3d(box, nn, psi, V, 1.0);
}

double seso_prob_x_range3d(const double* box, const int* n, const double* psi, double a, double b) {
    double acc = 0.0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double x = coord(box[0], box[1], n[0], i);
                if (x >= a && x < b) {
                    const size_t f = flat(n, i, j, k);
                    acc += psi[2 * f] * psi[2 * f] + psi[2 * f + 1] * psi[2 * f + 1];
                }
            }
    return acc * cell_volume(box, n);
}

static void moments(const double* box, const int* n, const double* psi, double* m1, double* m2) {
    double s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0}, den = 0.0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const size_t f = flat(n, i, j, k);
                const double w = psi[2 * f] * psi[2 * f] + psi[2 * f + 1] * psi[2 * f + 1];
                const double r[3] = {coord(box[0], box[1], n[0], i), coord(box[2], box[3], n[1], j),
                                     coord(box[4], box[5], n[2], k)};
                for (int a = 0; a < 3; ++a) {
                    s1[a] += r[a] * w;
                    s2[a] += r[a] * r[a] * w;
                }
                den += w;
            }
    for (int a = 0; a < 3; ++a) {
        m1[a] = ratio(s1[a], den);
        m2[a] = ratio(s2[a], den);
    }
}

void seso_mean_position3d(const double* box, const int* n, const double* psi, double* out3) {
    double m2[3];
    moments(box, n, psi, out3, m2);
}

void seso_sigma_position3d(const double* box, const int* n, const double* psi, double* out3) {
    double m1[3], m2[3];
    moments(box, n, psi, m1, m2);
    for (int a = 0; a < 3; ++a) {
        const double var = m2[a] - m1[a] * m1[a];
        out3[a] = sqrt(var > 0.0 ? var : 0.0);
    }
}

void seso_mean_momentum3d(const double* box, const int* n, const double* psi, double* out3) {
    const size_t N = total(n);
    double* phi = (double*)malloc(2 * N * sizeof(double));
    memcpy(phi, psi, 2 * N * sizeof(double));
    seso_fft3d(phi, n);
    double* kk[3];
    for (int a = 0; a < 3; ++a) {
        kk[a] = (double*)malloc((size_t)n[a] * sizeof(double));
        seso_wavenumbers(box[2 * a], box[2 * a + 1], n[a], kk[a]);
    }
    double num[3] = {0, 0, 0}, den = 0.0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const size_t f = flat(n, i, j, k);
                const double w = phi[2 * f] * phi[2 * f] + phi[2 * f + 1] * phi[2 * f + 1];
                num[0] += kk[0][i] * w;
                num[1] += kk[1][j] * w;
                num[2] += kk[2][k] * w;
                den += w;
            }
    for (int a = 0; a < 3; ++a) {
        out3[a] = ratio(num[a], den);
        free(kk[a]);
    }
    free(phi);
}
