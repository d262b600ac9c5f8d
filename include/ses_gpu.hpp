// ses_gpu.hpp -- C++ adapter over the C ABI (ses_gpu.h) with the reference
// core's call surface, so director code written against ses::SplitOperator3D
// (core/src/propagator.ixx), ses::fft/ifft (core/src/fft.ixx) and ses::Field3D
// (core/src/field.ixx) switches to the B200 path by changing a namespace.
//
// Error behaviour follows the reference: unsupported sizes throw
// std::invalid_argument (fft.ixx:42-44); out-of-memory throws std::bad_alloc;
// device errors and expired bounded waits throw std::runtime_error.
#pragma once

#include <cmath>
#include <complex>
#include <cstddef>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ses_gpu.h"

namespace ses::gpu {

using cd = std::complex<double>;

inline void check(ses_status s) {
    if (s == SES_OK) return;
    const std::string msg = ses_last_error();
    if (s == SES_EINVAL) throw std::invalid_argument(msg);
    if (s == SES_ENOMEM) throw std::bad_alloc();
    throw std::runtime_error("ses_gpu: " + msg);
}

// Grid1D / Grid3D (core/src/grid.ixx:10-30)
struct Grid1D {
    double xmin{};
    double xmax{};
    int n{};
    constexpr int size() const noexcept { return n; }
    constexpr double spacing() const noexcept { return (xmax - xmin) / n; }
    constexpr double coord(int i) const noexcept { return xmin + i * spacing(); }
};

struct Grid3D {
    Grid1D x{}, y{}, z{};
    constexpr int size() const noexcept { return x.n * y.n * z.n; }
    constexpr int flat(int i, int j, int k) const noexcept { return i + x.n * (j + y.n * k); }
    constexpr double cell_volume() const noexcept {
        return x.spacing() * y.spacing() * z.spacing();
    }
    ses_grid_desc desc() const noexcept {
        return ses_grid_desc{{x.xmin, x.xmax, x.n}, {y.xmin, y.xmax, y.n}, {z.xmin, z.xmax, z.n}};
    }
};

// Field3D (core/src/field.ixx:47-66): owns complex128 values, x-fastest
class Field3D {
public:
    explicit Field3D(Grid3D g) : grid_(g), data_(static_cast<std::size_t>(g.size())) {}
    int size() const noexcept { return grid_.size(); }
    const Grid3D& grid() const noexcept { return grid_; }
    cd& operator()(int i, int j, int k) noexcept { return data_[grid_.flat(i, j, k)]; }
    const cd& operator()(int i, int j, int k) const noexcept { return data_[grid_.flat(i, j, k)]; }
    std::vector<cd>& data() noexcept { return data_; }
    const std::vector<cd>& data() const noexcept { return data_; }

private:
    Grid3D grid_;
    std::vector<cd> data_;
};

inline const double* raw(const std::vector<cd>& v) { return reinterpret_cast<const double*>(v.data()); }
inline double* raw(std::vector<cd>& v) { return reinterpret_cast<double*>(v.data()); }

// fft(Field3D&) / ifft(Field3D&) (fft.ixx:102-188) through the device
inline void fft(Field3D& f, ses_precision p = SES_C128) {
    const int32_t n[3] = {f.grid().x.n, f.grid().y.n, f.grid().z.n};
    check(ses_fft3_host(n, p, raw(f.data()), 0));
}
inline void ifft(Field3D& f, ses_precision p = SES_C128) {
    const int32_t n[3] = {f.grid().x.n, f.grid().y.n, f.grid().z.n};
    check(ses_fft3_host(n, p, raw(f.data()), 1));
}
// fft(std::vector<cd>&) / ifft (fft.ixx:75-98)
inline void fft(std::vector<cd>& a, ses_precision p = SES_C128) {
    const int32_t n[3] = {static_cast<int32_t>(a.size()), 1, 1};
    check(ses_fft3_host(n, p, raw(a), 0));
}
inline void ifft(std::vector<cd>& a, ses_precision p = SES_C128) {
    const int32_t n[3] = {static_cast<int32_t>(a.size()), 1, 1};
    check(ses_fft3_host(n, p, raw(a), 1));
}

// SplitOperator3D (propagator.ixx:68-134) plus the resident engine calls of
// the reference GPU engine (vk_engine.ixx: upload_state, step(n, absorb),
// set_absorber, readback, norm/energy).
class SplitOperator3D {
public:
    SplitOperator3D(const Grid3D& g, const std::vector<double>& potential, double dt,
                    double mass = 1.0, ses_precision prec = SES_C128)
        : grid_(g), dt_(dt) {
        if (static_cast<int>(potential.size()) != g.size())
            throw std::invalid_argument("potential size does not match the grid");
        const ses_grid_desc d = g.desc();
        check(ses_gpu_create(&d, prec, dt, mass, potential.data(), nullptr, &h_));
    }
    SplitOperator3D(const SplitOperator3D&) = delete;
    SplitOperator3D& operator=(const SplitOperator3D&) = delete;
    SplitOperator3D(SplitOperator3D&& o) noexcept : grid_(o.grid_), dt_(o.dt_), h_(o.h_) { o.h_ = nullptr; }
    ~SplitOperator3D() {
        if (h_) ses_gpu_destroy(h_);
    }

    double dt() const noexcept { return dt_; }
    const Grid3D& grid() const noexcept { return grid_; }

    std::vector<cd> half_potential_phase() const {
        std::vector<cd> t(static_cast<std::size_t>(grid_.size()));
        check(ses_gpu_tables(h_, raw(t), nullptr));
        return t;
    }
    std::vector<cd> kinetic_phase() const {
        std::vector<cd> t(static_cast<std::size_t>(grid_.size()));
        check(ses_gpu_tables(h_, nullptr, raw(t)));
        return t;
    }

    // In place on a caller-owned field, like the reference (propagator.ixx:110-119).
    void step(Field3D& psi, int nsteps = 1) const {
        if (psi.size() != grid_.size()) throw std::invalid_argument("field does not match the grid");
        check(ses_gpu_write_psi(h_, raw(psi.data())));
        check(ses_gpu_step(h_, nsteps, 0));
        check(ses_gpu_read_psi(h_, raw(psi.data())));
    }

    // ---- resident engine surface ----
    void upload_state(const std::vector<cd>& psi) { check(ses_gpu_write_psi(h_, raw(psi))); }
    void advance(int nsteps, bool absorb = false) { check(ses_gpu_step(h_, nsteps, absorb ? 1 : 0)); }
    std::vector<cd> readback() const {
        std::vector<cd> out(static_cast<std::size_t>(grid_.size()));
        check(ses_gpu_read_psi(h_, raw(out)));
        return out;
    }
    void set_absorber(const std::vector<double>& mask) { check(ses_gpu_set_absorber(h_, mask.data())); }
    void clear_absorber() { check(ses_gpu_set_absorber(h_, nullptr)); }
    void set_potential(const std::vector<double>& v) { check(ses_gpu_set_potential(h_, v.data())); }
    ses_observables observe(double xlo = -1e300, double xhi = 1e300) const {
        ses_observables o{};
        check(ses_gpu_observe(h_, xlo, xhi, &o));
        return o;
    }
    void sync(int timeout_ms = 0) const { check(ses_gpu_sync(h_, timeout_ms)); }
    ses_handle handle() const noexcept { return h_; }

    // Engine::norm_and_peak / Engine::scale (solver/src/vk_engine.ixx:1665-1692, 2120-2133)
    struct NormPeak {
        double sum = 0.0;   // sum |psi|^2 dV
        double peak = 0.0;  // max |psi|^2
    };
    NormPeak norm_and_peak() const {
        NormPeak np;
        check(ses_gpu_norm_and_peak(h_, &np.sum, &np.peak));
        return np;
    }
    void scale(double s) { check(ses_gpu_scale(h_, s)); }
    // records the step graph now rather than inside the first long advance
    void prepare(bool absorb = false) { check(ses_gpu_prepare(h_, absorb ? 1 : 0)); }

private:
    Grid3D grid_;
    double dt_;
    ses_handle h_ = nullptr;
};

// ImaginaryTimePropagator3D (core/src/imaginary_time.ixx:64-108): relax(psi, n)
// renormalises after every step, as the reference.
class ImaginaryTimePropagator3D {
public:
    ImaginaryTimePropagator3D(const Grid3D& g, const std::vector<double>& potential, double dtau,
                              double mass = 1.0, ses_precision prec = SES_C128)
        : grid_(g) {
        if (static_cast<int>(potential.size()) != g.size())
            throw std::invalid_argument("potential size does not match the grid");
        const ses_grid_desc d = g.desc();
        check(ses_gpu_create_imag(&d, prec, dtau, mass, potential.data(), nullptr, &h_));
    }
    ImaginaryTimePropagator3D(const ImaginaryTimePropagator3D&) = delete;
    ImaginaryTimePropagator3D& operator=(const ImaginaryTimePropagator3D&) = delete;
    ~ImaginaryTimePropagator3D() {
        if (h_) ses_gpu_destroy(h_);
    }
    void relax(Field3D& psi, int nsteps) const {
        if (psi.size() != grid_.size()) throw std::invalid_argument("field does not match the grid");
        check(ses_gpu_write_psi(h_, raw(psi.data())));
        check(ses_gpu_relax(h_, nsteps, 1, nullptr));
        check(ses_gpu_read_psi(h_, raw(psi.data())));
    }

private:
    Grid3D grid_;
    ses_handle h_ = nullptr;
};

struct Vec3d {
    double x{}, y{}, z{};
};

// norm_sq(Field3D) (core/src/field.ixx:68-74): sum |psi|^2 dV, left to right
inline double norm_sq(const Field3D& f) {
    double s = 0.0;
    for (const cd& v : f.data()) s += std::norm(v);
    return s * f.grid().cell_volume();
}

// probability_density (core/src/field.ixx:100-106)
inline std::vector<double> probability_density(const Field3D& f) {
    std::vector<double> rho(f.data().size());
    for (std::size_t i = 0; i < rho.size(); ++i) rho[i] = std::norm(f.data()[i]);
    return rho;
}

// gaussian_wavepacket(Grid3D, r0, sigma, k0) (core/src/wavepacket.ixx:29-49):
// separable Gaussian envelope (2 pi s^2)^(-1/4) exp(-(u - u0)^2 / (4 s^2)) per axis
// times e^{i k0 . r}, then normalised so that norm_sq = 1.
inline Field3D gaussian_wavepacket(const Grid3D& g, Vec3d r0, Vec3d sigma, Vec3d k0) {
    constexpr double kPi = 3.14159265358979323846;
    auto envelope = [](double u, double u0, double s) {
        return std::pow(2.0 * kPi * s * s, -0.25) * std::exp(-(u - u0) * (u - u0) / (4.0 * s * s));
    };
    Field3D psi(g);
    for (int k = 0; k < g.z.n; ++k)
        for (int j = 0; j < g.y.n; ++j)
            for (int i = 0; i < g.x.n; ++i) {
                const double x = g.x.coord(i), y = g.y.coord(j), z = g.z.coord(k);
                const double env = envelope(x, r0.x, sigma.x) * envelope(y, r0.y, sigma.y) * envelope(z, r0.z, sigma.z);
                const double phase = k0.x * x + k0.y * y + k0.z * z;
                psi(i, j, k) = cd{env * std::cos(phase), env * std::sin(phase)};
            }
    const double n2 = norm_sq(psi);
    if (n2 > 0.0) {
        const double inv = 1.0 / std::sqrt(n2);
        for (cd& v : psi.data()) v *= inv;
    }
    return psi;
}

// WavepacketSimulation (core/src/simulation.ixx:22-88): Config -> tables and
// psi0; advance(n) steps the field resident on the device, psi() / density()
// read it back when it changed, set_psi() uploads a field, relax(n, dtau) runs
// imaginary time on it.  The POVM measurement of the reference (measure) is not
// part of the step and is not provided.
class WavepacketSimulation {
public:
    struct Config {
        Grid3D grid;
        std::vector<double> potential;
        Vec3d r0;
        Vec3d sigma;
        Vec3d k0;
        double dt;
    };

    explicit WavepacketSimulation(Config cfg, ses_precision prec = SES_C128)
        : grid_(cfg.grid),
          dt_(cfg.dt),
          prec_(prec),
          potential_(std::move(cfg.potential)),
          propagator_(cfg.grid, potential_, cfg.dt, 1.0, prec),
          psi_(gaussian_wavepacket(cfg.grid, cfg.r0, cfg.sigma, cfg.k0)) {
        propagator_.upload_state(psi_.data());
    }

    void advance(int nsteps) {
        propagator_.advance(nsteps);
        steps_ += nsteps;
        stale_ = true;
    }

    // imaginary-time relaxation of the current field with step dtau (tau is not t)
    void relax(int nsteps, double dtau) {
        if (!relaxer_ || relaxer_dtau_ != dtau) {
            relaxer_.reset(new ImaginaryTimePropagator3D(grid_, potential_, dtau, 1.0, prec_));
            relaxer_dtau_ = dtau;
        }
        Field3D& p = current();
        relaxer_->relax(p, nsteps);
        propagator_.upload_state(p.data());
    }

    double time() const noexcept { return static_cast<double>(steps_) * dt_; }
    double dt() const noexcept { return dt_; }
    const Grid3D& grid() const noexcept { return grid_; }
    const Field3D& psi() const { return current(); }
    const std::vector<double>& potential() const noexcept { return potential_; }
    const SplitOperator3D& propagator() const noexcept { return propagator_; }
    SplitOperator3D& propagator() noexcept { return propagator_; }

    void set_psi(const Field3D& psi) {
        if (psi.size() != psi_.size()) throw std::invalid_argument("field does not match the grid");
        psi_ = psi;
        propagator_.upload_state(psi_.data());
        stale_ = false;
    }
    std::vector<double> density() const { return probability_density(current()); }

private:
    Field3D& current() const {
        if (stale_) {
            psi_.data() = propagator_.readback();
            stale_ = false;
        }
        return psi_;
    }

    Grid3D grid_;
    double dt_;
    ses_precision prec_;
    std::vector<double> potential_;
    SplitOperator3D propagator_;
    mutable Field3D psi_;
    mutable bool stale_ = false;
    long long steps_ = 0;
    std::unique_ptr<ImaginaryTimePropagator3D> relaxer_;
    double relaxer_dtau_ = 0.0;
};

// SplitOperator1D (propagator.ixx:21-66): the 3D engine on n x 1 x 1
class SplitOperator1D {
public:
    SplitOperator1D(const Grid1D& g, const std::vector<double>& potential, double dt,
                    ses_precision prec = SES_C128)
        : op_(Grid3D{g, Grid1D{0.0, 1.0, 1}, Grid1D{0.0, 1.0, 1}}, potential, dt, 1.0, prec), n_(g.n) {}
    double dt() const noexcept { return op_.dt(); }
    void step(std::vector<cd>& psi, int nsteps = 1) const {
        if (static_cast<int>(psi.size()) != n_) throw std::invalid_argument("field does not match the grid");
        check(ses_gpu_write_psi(op_.handle(), raw(psi)));
        check(ses_gpu_step(op_.handle(), nsteps, 0));
        check(ses_gpu_read_psi(op_.handle(), raw(psi)));
    }

private:
    SplitOperator3D op_;
    int n_;
};

// Many propagations advanced together (no counterpart in the reference core,
// whose directors loop over instances on the CPU: core/src/parallel.ixx:195-238).
// Members stay owned by the caller and must outlive their membership.
class Batch {
public:
    Batch() { check(ses_batch_create(&b_)); }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    ~Batch() {
        if (b_) ses_batch_destroy(b_);
    }

    void add(SplitOperator3D& op) {
        check(ses_batch_add(b_, op.handle()));
        members_.push_back(&op);
    }
    void remove(SplitOperator3D& op) {
        check(ses_batch_remove(b_, op.handle()));
        for (std::size_t i = 0; i < members_.size(); ++i)
            if (members_[i] == &op) {
                members_.erase(members_.begin() + static_cast<std::ptrdiff_t>(i));
                break;
            }
    }
    std::size_t size() const noexcept { return members_.size(); }
    void step(int nsteps, bool absorb = false) { check(ses_batch_step(b_, nsteps, absorb ? 1 : 0)); }
    void prepare(bool absorb = false) { check(ses_batch_prepare(b_, absorb ? 1 : 0)); }
    std::vector<ses_observables> observe(double xlo = -1e300, double xhi = 1e300) {
        std::vector<ses_observables> out(members_.size());
        check(ses_batch_observe(b_, xlo, xhi, out.data(), static_cast<int>(out.size())));
        return out;
    }
    void sync(int timeout_ms = 0) { check(ses_batch_sync(b_, timeout_ms)); }

    // One host round trip of every member (ses_batch_run): upload in[i] (skipped
    // where null), nsteps steps, observables, read back into out[i] (skipped
    // where null).  Fields match the members in the order they were added.
    std::vector<ses_observables> run(const std::vector<Field3D*>& in, int nsteps, bool absorb,
                                     const std::vector<Field3D*>& out, double xlo = -1e300,
                                     double xhi = 1e300) {
        const std::size_t m = members_.size();
        if ((!in.empty() && in.size() != m) || (!out.empty() && out.size() != m))
            throw std::invalid_argument("one field (or null) per member");
        std::vector<const double*> pin(m, nullptr);
        std::vector<double*> pout(m, nullptr);
        for (std::size_t i = 0; i < m; ++i) {
            for (Field3D* f : {in.empty() ? nullptr : in[i], out.empty() ? nullptr : out[i]})
                if (f && f->size() != members_[i]->grid().size())
                    throw std::invalid_argument("field does not match its member's grid");
            if (!in.empty() && in[i]) pin[i] = raw(in[i]->data());
            if (!out.empty() && out[i]) pout[i] = raw(out[i]->data());
        }
        std::vector<ses_observables> obs(m);
        check(ses_batch_run(b_, in.empty() ? nullptr : pin.data(), nsteps, absorb ? 1 : 0, xlo, xhi,
                            obs.data(), out.empty() ? nullptr : pout.data(), static_cast<int>(m), 0));
        return obs;
    }

private:
    ses_batch b_ = nullptr;
    std::vector<SplitOperator3D*> members_;
};

}  // namespace ses::gpu
