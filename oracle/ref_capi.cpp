// C wrapper around the reference's FP64 CPU core (test infrastructure only).
//
// Compiled by oracle/build_ref.py against header-shimmed copies of the
// reference modules that it generates under oracle/_ref/gen/.  Every function
// forwards to the reference's public C++ API unchanged; the only code here is
// argument marshalling (interleaved re/im doubles <-> std::complex<double>).
// Used by tests/ to pin the oracle restatement and by bench.py's reference
// arm / cpu_baseline leg.  Never linked into the product library.

#include <complex>
#include <cstddef>
#include <cstring>
#include <vector>

#include "grid.hpp"
#include "vec.hpp"
#include "parallel.hpp"
#include "field.hpp"
#include "spectral.hpp"
#include "fft.hpp"
#include "propagator.hpp"
#include "potential.hpp"
#include "wavepacket.hpp"
#include "observables.hpp"
#include "imaginary_time.hpp"
#include "drive.hpp"

namespace {

using cd = std::complex<double>;

ses::Grid3D grid3(const double* box, const int* n) {
    return ses::Grid3D{ses::Grid1D{box[0], box[1], n[0]}, ses::Grid1D{box[2], box[3], n[1]},
                       ses::Grid1D{box[4], box[5], n[2]}};
}

void load(std::vector<cd>& dst, const double* src) {
    for (std::size_t i = 0; i < dst.size(); ++i) dst[i] = cd{src[2 * i], src[2 * i + 1]};
}

void store(const std::vector<cd>& src, double* dst) {
    for (std::size_t i = 0; i < src.size(); ++i) {
        dst[2 * i] = src[i].real();
        dst[2 * i + 1] = src[i].imag();
    }
}

struct Prop3 {
    ses::SplitOperator3D op;
};

struct Prop1 {
    ses::Grid1D g;
    ses::SplitOperator1D op;
};

}  // namespace

extern "C" {

int sesref_workers() { return ses::parallel_workers(); }

// ---- FFT (core/src/fft.ixx) ----
int sesref_fft1d(double* a, std::size_t n, int inverse) {
    std::vector<cd> v(n);
    load(v, a);
    try {
        if (inverse) ses::ifft(v); else ses::fft(v);
    } catch (...) {
        return -1;
    }
    store(v, a);
    return 0;
}

int sesref_fft3d(double* a, const int* n, int inverse) {
    const double box[6] = {0, 1, 0, 1, 0, 1};
    ses::Field3D f{grid3(box, n)};
    load(f.data(), a);
    try {
        if (inverse) ses::ifft(f); else ses::fft(f);
    } catch (...) {
        return -1;
    }
    store(f.data(), a);
    return 0;
}

void sesref_fft_twiddles(std::size_t n, double* out) { store(ses::fft_twiddles(n), out); }

void sesref_wavenumbers(double xmin, double xmax, int n, double* out) {
    const std::vector<double> k = ses::wavenumbers(ses::Grid1D{xmin, xmax, n});
    std::memcpy(out, k.data(), k.size() * sizeof(double));
}

// ---- potentials / masks / packets (core/src/potential.ixx, wavepacket.ixx) ----
void sesref_harmonic3d(const double* box, const int* n, double omega, const double* c, double* out) {
    const auto v = ses::harmonic_potential(grid3(box, n), omega, ses::Vec3d{c[0], c[1], c[2]});
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_soft_coulomb3d(const double* box, const int* n, double Z, double a, const double* c,
                           double* out) {
    const auto v = ses::soft_coulomb_potential(grid3(box, n), Z, a, ses::Vec3d{c[0], c[1], c[2]});
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_regularized_coulomb3d(const double* box, const int* n, double Z, const double* c,
                                  double* out) {
    const auto v = ses::regularized_coulomb_potential(grid3(box, n), Z, ses::Vec3d{c[0], c[1], c[2]});
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_barrier3d(const double* box, const int* n, double v0, double xlo, double xhi, double* out) {
    const auto v = ses::barrier_potential(grid3(box, n), v0, xlo, xhi);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_absorbing_mask3d(const double* box, const int* n, double width, double* out) {
    const auto v = ses::absorbing_mask(grid3(box, n), width);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_absorbing_mask1d(double xmin, double xmax, int n, double width, double* out) {
    const auto v = ses::absorbing_mask(ses::Grid1D{xmin, xmax, n}, width);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_harmonic1d(double xmin, double xmax, int n, double omega, double x0, double* out) {
    const auto v = ses::harmonic_potential(ses::Grid1D{xmin, xmax, n}, omega, x0);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_morse1d(double xmin, double xmax, int n, double d, double alpha, double x0, double* out) {
    const auto v = ses::morse_potential(ses::Grid1D{xmin, xmax, n}, d, alpha, x0);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_double_well1d(double xmin, double xmax, int n, double vb, double a, double* out) {
    const auto v = ses::double_well_potential(ses::Grid1D{xmin, xmax, n}, vb, a);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_poschl_teller1d(double xmin, double xmax, int n, double v0, double a, double x0,
                            double* out) {
    const auto v = ses::poschl_teller_potential(ses::Grid1D{xmin, xmax, n}, v0, a, x0);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_barrier1d(double xmin, double xmax, int n, double v0, double xlo, double xhi, double* out) {
    const auto v = ses::barrier_potential(ses::Grid1D{xmin, xmax, n}, v0, xlo, xhi);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void sesref_gaussian3d(const double* box, const int* n, const double* r0, const double* sigma,
                       const double* k0, double* out) {
    const ses::Field3D f = ses::gaussian_wavepacket(grid3(box, n), ses::Vec3d{r0[0], r0[1], r0[2]},
                                                    ses::Vec3d{sigma[0], sigma[1], sigma[2]},
                                                    ses::Vec3d{k0[0], k0[1], k0[2]});
    store(f.data(), out);
}
void sesref_gaussian1d(double xmin, double xmax, int n, double x0, double sigma, double k0,
                       double* out) {
    const ses::Field1D f = ses::gaussian_wavepacket(ses::Grid1D{xmin, xmax, n}, x0, sigma, k0);
    store(f.data(), out);
}

// ---- 3D split operator (core/src/propagator.ixx:68-134) ----
void* sesref_split3d_new(const double* box, const int* n, const double* V, double dt, double mass) {
    const ses::Grid3D g = grid3(box, n);
    std::vector<double> v(V, V + g.size());
    return new Prop3{ses::SplitOperator3D{g, v, dt, mass}};
}
void sesref_split3d_free(void* h) { delete static_cast<Prop3*>(h); }
void sesref_split3d_tables(void* h, double* half_v, double* kin) {
    const auto* p = static_cast<Prop3*>(h);
    if (half_v) store(p->op.half_potential_phase(), half_v);
    if (kin) store(p->op.kinetic_phase(), kin);
}

void* sesref_field3d_new(const double* box, const int* n) { return new ses::Field3D{grid3(box, n)}; }
void sesref_field3d_free(void* f) { delete static_cast<ses::Field3D*>(f); }
void sesref_field3d_set(void* f, const double* psi) { load(static_cast<ses::Field3D*>(f)->data(), psi); }
void sesref_field3d_get(void* f, double* psi) { store(static_cast<ses::Field3D*>(f)->data(), psi); }

// nsteps Strang steps; when mask != nullptr, psi *= mask after EVERY step (the
// CPU order the reference's absorber check uses, vkcheck_main.cpp:2469-2475).
void sesref_split3d_step(void* h, void* f, int nsteps, const double* mask) {
    const auto* p = static_cast<Prop3*>(h);
    auto* psi = static_cast<ses::Field3D*>(f);
    if (!mask) {
        p->op.step(*psi, nsteps);
        return;
    }
    std::vector<cd>& a = psi->data();
    for (int s = 0; s < nsteps; ++s) {
        p->op.step(*psi, 1);
        ses::parallel_for(static_cast<int>(a.size()), [&](int i) {
            a[static_cast<std::size_t>(i)] *= mask[i];
        });
    }
}

// ses::driven_step (drive.ixx:50-65) on the resident field.
void sesref_driven_step3d(void* h, void* f, const double* axis, double amplitude, double omega, double t0,
                          int nsteps) {
    const auto* p = static_cast<Prop3*>(h);
    ses::DipoleDrive d{ses::Vec3d{axis[0], axis[1], axis[2]}, amplitude, omega};
    ses::driven_step(*static_cast<ses::Field3D*>(f), p->op, d, t0, nsteps);
}

double sesref_norm3d(void* f) { return ses::norm_sq(*static_cast<ses::Field3D*>(f)); }
double sesref_mean_energy3d(void* f, const double* V, double mass) {
    auto* psi = static_cast<ses::Field3D*>(f);
    std::vector<double> v(V, V + psi->size());
    return ses::mean_energy(*psi, v, mass);
}
void sesref_mean_position3d(void* f, double* out) {
    const ses::Vec3d r = ses::mean_position(*static_cast<ses::Field3D*>(f));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void sesref_sigma_position3d(void* f, double* out) {
    const ses::Vec3d r = ses::sigma_position(*static_cast<ses::Field3D*>(f));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void sesref_mean_momentum3d(void* f, double* out) {
    const ses::Vec3d r = ses::mean_momentum(*static_cast<ses::Field3D*>(f));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// ---- 1D split operator (core/src/propagator.ixx:21-66) ----
void* sesref_split1d_new(double xmin, double xmax, int n, const double* V, double dt) {
    const ses::Grid1D g{xmin, xmax, n};
    std::vector<double> v(V, V + n);
    return new Prop1{g, ses::SplitOperator1D{g, v, dt}};
}
void sesref_split1d_free(void* h) { delete static_cast<Prop1*>(h); }
void sesref_split1d_step(void* h, double* psi_io, int nsteps, const double* mask) {
    auto* p = static_cast<Prop1*>(h);
    ses::Field1D f{p->g};
    load(f.data(), psi_io);
    for (int s = 0; s < nsteps; ++s) {
        p->op.step(f, 1);
        if (mask) {
            for (int i = 0; i < f.size(); ++i) f[i] *= mask[i];
        }
    }
    store(f.data(), psi_io);
}

static ses::Field1D field1(double xmin, double xmax, int n, const double* psi) {
    ses::Field1D f{ses::Grid1D{xmin, xmax, n}};
    load(f.data(), psi);
    return f;
}
double sesref_norm1d(double xmin, double xmax, int n, const double* psi) {
    return ses::norm_sq(field1(xmin, xmax, n, psi));
}
double sesref_mean_energy1d(double xmin, double xmax, int n, const double* psi, const double* V) {
    std::vector<double> v(V, V + n);
    return ses::mean_energy(field1(xmin, xmax, n, psi), v);
}
double sesref_mean_position1d(double xmin, double xmax, int n, const double* psi) {
    return ses::mean_position(field1(xmin, xmax, n, psi));
}
double sesref_sigma_x1d(double xmin, double xmax, int n, const double* psi) {
    return ses::sigma_x(field1(xmin, xmax, n, psi));
}
double sesref_mean_momentum1d(double xmin, double xmax, int n, const double* psi) {
    return ses::mean_momentum(field1(xmin, xmax, n, psi));
}
double sesref_probability_in_range1d(double xmin, double xmax, int n, const double* psi, double a,
                                     double b) {
    return ses::probability_in_range(field1(xmin, xmax, n, psi), a, b);
}

// ---- imaginary time (core/src/imaginary_time.ixx:64-144) ----
void sesref_relax3d(const double* box, const int* n, const double* V, double dtau, double mass,
                    double* psi_io, int nsteps) {
    const ses::Grid3D g = grid3(box, n);
    std::vector<double> v(V, V + g.size());
    const ses::ImaginaryTimePropagator3D itp{g, v, dtau, mass};
    ses::Field3D f{g};
    load(f.data(), psi_io);
    itp.relax(f, nsteps);
    store(f.data(), psi_io);
}

}  // extern "C"
