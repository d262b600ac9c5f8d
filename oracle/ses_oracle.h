/* CPU FP64 oracle for the Strang split-operator step (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference core's algorithm for this path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
 * may load it, and only as the checker: the product library never links it.
 *
 * Complex arrays are interleaved (re, im) doubles, x-fastest flat layout
 * flat(i,j,k) = i + nx*(j + ny*k) (reference core/src/grid.ixx:20-30).
 * A grid is described by box[6] = {xmin,xmax,ymin,ymax,zmin,zmax} and n[3].
 */
#ifndef SES_ORACLE_H
#define SES_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 0 = ok, -1 = unsupported length (not 2^a 3^b 5^c) */
int seso_supported_length(size_t n);

/* w[j] = cis(-2 pi j / n), j < n/2, direct cos/sin (fft.ixx:29-37). */
void seso_fft_twiddles(size_t n, double* w);
/* In-place forward unnormalized 1D FFT.  Power-of-two n: radix-2 DIT with
 * bit reversal, identical steps to fft.ixx:39-73.  Other 2^a3^b5^c lengths:
 * recursive mixed-radix decimation in time (extension; the reference throws). */
int seso_fft1d(double* a, size_t n);
int seso_ifft1d(double* a, size_t n);      /* conj -> fft -> conj/N (fft.ixx:89-98) */
int seso_fft3d(double* a, const int* n);   /* x, y, z line passes (fft.ixx:102-173) */
int seso_ifft3d(double* a, const int* n);  /* conj identity (fft.ixx:177-188) */
/* O(n^2) long-double DFT, for pinning the mixed-radix path. */
void seso_dft_naive(const double* in, double* out, size_t n, int inverse);

void seso_wavenumbers(double xmin, double xmax, int n, double* k); /* spectral.ixx:14-23 */

/* Full-N phase tables (propagator.ixx:72-101): half_v = cis(-V dt/2),
 * kin = cis(-(kx^2+ky^2+kz^2)/(2m) dt). */
void seso_tables3d(const double* box, const int* n, const double* V, double dt, double mass,
                   double* half_v, double* kin);

/* nsteps reference Strang steps V/2 . F^-1 K F . V/2 (propagator.ixx:110-119),
 * optional real mask multiplied after every step (vkcheck_main.cpp:2469-2475). */
int seso_step3d(const double* box, const int* n, const double* V, double dt, double mass,
                const double* mask, double* psi, int nsteps);
int seso_step1d(double xmin, double xmax, int n, const double* V, double dt, const double* mask,
                double* psi, int nsteps);
/* dipole-driven steps kick(t) . step . kick(t + dt) (drive.ixx:25-65), no mask */
int seso_driven_step3d(const double* box, const int* n, const double* V, double dt, double mass,
                       const double* axis, double amplitude, double omega, double t0, double* psi,
                       int nsteps);
/* imaginary-time relaxation with renormalisation (imaginary_time.ixx:64-144) */
int seso_relax3d(const double* box, const int* n, const double* V, double dtau, double mass,
                 double* psi, int nsteps);

/* ---- potentials and masks (potential.ixx) ---- */
void seso_harmonic3d(const double* box, const int* n, double omega, const double* c, double* v);
void seso_soft_coulomb3d(const double* box, const int* n, double Z, double a, const double* c,
                         double* v);
void seso_regularized_coulomb3d(const double* box, const int* n, double Z, const double* c,
                                double* v);
void seso_barrier3d(const double* box, const int* n, double v0, double xlo, double xhi, double* v);
/* V += e * z  (Stark fold, hydrogen_director.ixx:1359-1370) */
void seso_stark_fold3d(const double* box, const int* n, double e, double* v);
/* stadium hard wall: v = v_out where the stadium SDF > 0, else 0, in the x-y plane
 * (billiard2d_director.ixx:26-29) */
void seso_stadium3d(const double* box, const int* n, double half_len, double r, double v_out,
                    double* v);
void seso_harmonic1d(double xmin, double xmax, int n, double omega, double x0, double* v);
void seso_morse1d(double xmin, double xmax, int n, double d, double alpha, double x0, double* v);
void seso_double_well1d(double xmin, double xmax, int n, double vb, double a, double* v);
void seso_poschl_teller1d(double xmin, double xmax, int n, double v0, double a, double x0,
                          double* v);
/* profile 0: sin^2 ramp (potential.ixx:192-233); profile 1: cos^(1/8) ramp
 * m = cos(pi/2 (1 - d/width))^(1/8) for wall distance d < width. */
void seso_mask1d(double xmin, double xmax, int n, double width, int profile, double* m);
void seso_mask3d(const double* box, const int* n, double width, int profile, double* m);

/* ---- initial states (wavepacket.ixx:16-49) ---- */
void seso_gaussian3d(const double* box, const int* n, const double* r0, const double* sigma,
                     const double* k0, double* psi);
void seso_gaussian1d(double xmin, double xmax, int n, double x0, double sigma, double k0,
                     double* psi);

/* ---- observables (field.ixx, observables.ixx), serial left-to-right sums ---- */
double seso_norm3d(const double* box, const int* n, const double* psi);
double seso_norm1d(double xmin, double xmax, int n, const double* psi);
double seso_mean_energy3d(const double* box, const int* n, const double* psi, const double* V,
                          double mass);
double seso_mean_energy1d(double xmin, double xmax, int n, const double* psi, const double* V);
/* absolute sum |psi|^2 dV over cells with x in [a, b) (observables.ixx:121-130) */
double seso_prob_x_range3d(const double* box, const int* n, const double* psi, double a, double b);
void seso_mean_position3d(const double* box, const int* n, const double* psi, double* out3);
void seso_sigma_position3d(const double* box, const int* n, const double* psi, double* out3);
void seso_mean_momentum3d(const double* box, const int* n, const double* psi, double* out3);

#ifdef __cplusplus
}
#endif
#endif
