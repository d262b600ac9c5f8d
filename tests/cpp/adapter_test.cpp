// C++ caller of the B200 path through include/ses_gpu.hpp, written the way the
// reference's own gtest cases use ses::SplitOperator3D / ses::fft (reference
// tests/fft3_test.cpp, propagator_tables_test.cpp, solver/src/vkcheck_main.cpp
// check_engine_step), checked against the FP64 oracle (oracle/ses_oracle.h).
#include <cmath>
#include <complex>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "ses_gpu.hpp"
#include "ses_oracle.h"

using ses::gpu::cd;

static int failures = 0;
#define EXPECT(cond, what)                                   \
    do {                                                     \
        if (!(cond)) {                                       \
            std::printf("FAIL %s\n", what);                  \
            ++failures;                                      \
        } else {                                             \
            std::printf("PASS %s\n", what);                  \
        }                                                    \
    } while (0)

int main() {
    const double pi = 3.14159265358979323846;
    {  // fft3_test.cpp PlaneWaveSpikesAtItsBin
        const int nx = 8, ny = 16, nz = 4;
        ses::gpu::Field3D f{ses::gpu::Grid3D{{0, 1, nx}, {0, 1, ny}, {0, 1, nz}}};
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double th = 2 * pi * (3.0 * i / nx + 5.0 * j / ny + 1.0 * k / nz);
                    f(i, j, k) = cd{std::cos(th), std::sin(th)};
                }
        ses::gpu::fft(f);
        double worst = 0;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double e = (i == 3 && j == 5 && k == 1) ? 512.0 : 0.0;
                    worst = std::fmax(worst, std::abs(f(i, j, k) - cd{e, 0}));
                }
        EXPECT(worst < 1e-9, "fft3 plane wave spike");
    }
    {  // check_engine_step: 8^3 soft Coulomb, dt 0.02, 20 steps vs the FP64 core
        const double box[6] = {-4, 4, -4, 4, -4, 4};
        const int n[3] = {8, 8, 8};
        const double c[3] = {0, 0, 0}, r0[3] = {1, 0, 0}, sg[3] = {1.2, 1.2, 1.2}, k0[3] = {0, 0.5, 0};
        std::vector<double> V(512);
        seso_soft_coulomb3d(box, n, 1.0, 1.0, c, V.data());
        std::vector<cd> psi0(512);
        seso_gaussian3d(box, n, r0, sg, k0, reinterpret_cast<double*>(psi0.data()));
        std::vector<cd> ref = psi0;
        seso_step3d(box, n, V.data(), 0.02, 1.0, nullptr, reinterpret_cast<double*>(ref.data()), 20);
        const ses::gpu::Grid3D g{{-4, 4, 8}, {-4, 4, 8}, {-4, 4, 8}};
        for (ses_precision p : {SES_C128, SES_C64}) {
            ses::gpu::SplitOperator3D prop{g, V, 0.02, 1.0, p};
            ses::gpu::Field3D f{g};
            f.data() = psi0;
            prop.step(f, 20);
            double num = 0, den = 0;
            for (std::size_t i = 0; i < ref.size(); ++i) {
                num += std::norm(f.data()[i] - ref[i]);
                den += std::norm(ref[i]);
            }
            const double err = std::sqrt(num / den);
            std::printf("  rel L2 (%s) = %.3e\n", p == SES_C128 ? "c128" : "c64", err);
            EXPECT(err < (p == SES_C128 ? 20e-12 : 1e-5), "engine step vs FP64 core");
        }
    }
    {  // propagator_tables_test.cpp: entries == formula within EXPECT_DOUBLE_EQ (4 ulp)
        const double box[6] = {0, 4, 0, 4, 0, 4};
        const int n[3] = {4, 4, 4};
        const double c[3] = {1, 2, 3};
        std::vector<double> V(64);
        seso_harmonic3d(box, n, 2.0, c, V.data());
        std::vector<cd> half(64), kin(64);
        seso_tables3d(box, n, V.data(), 0.1, 1.0, reinterpret_cast<double*>(half.data()),
                      reinterpret_cast<double*>(kin.data()));
        const ses::gpu::Grid3D g{{0, 4, 4}, {0, 4, 4}, {0, 4, 4}};
        ses::gpu::SplitOperator3D prop{g, V, 0.1};
        const auto h = prop.half_potential_phase();
        const auto k = prop.kinetic_phase();
        double worst = 0;  // in units of 2^-52 (entries are <= 1 in magnitude)
        for (int i = 0; i < 64; ++i) {
            worst = std::fmax(worst, std::fabs(h[i].real() - half[i].real()) / std::ldexp(1.0, -52));
            worst = std::fmax(worst, std::fabs(h[i].imag() - half[i].imag()) / std::ldexp(1.0, -52));
            worst = std::fmax(worst, std::fabs(k[i].real() - kin[i].real()) / std::ldexp(1.0, -52));
            worst = std::fmax(worst, std::fabs(k[i].imag() - kin[i].imag()) / std::ldexp(1.0, -52));
        }
        EXPECT(worst <= 4.0, "propagator tables match the formula");
        EXPECT(prop.dt() == 0.1, "dt accessor");
    }
    {  // non-2^a3^b5^c size throws std::invalid_argument, like the reference
        bool threw = false;
        try {
            ses::gpu::SplitOperator3D bad{ses::gpu::Grid3D{{0, 1, 7}, {0, 1, 8}, {0, 1, 8}},
                                          std::vector<double>(448, 0.0), 0.1};
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw, "unsupported size throws std::invalid_argument");
    }
    {  // propagator_test.cpp ConservesNorm (1024 points, dt 0.05, 200 steps)
        std::vector<cd> psi(1024);
        seso_gaussian1d(-40, 40, 1024, -15, 1, 2, reinterpret_cast<double*>(psi.data()));
        ses::gpu::SplitOperator1D prop{ses::gpu::Grid1D{-40, 40, 1024}, std::vector<double>(1024, 0.0), 0.05};
        prop.step(psi, 200);
        const double nrm = seso_norm1d(-40, 40, 1024, reinterpret_cast<const double*>(psi.data()));
        EXPECT(std::fabs(nrm - 1.0) < 1e-12, "1D free packet conserves norm");
    }
    {  // a director sweeping several scenes through one batch: 16^3 and 32^3 (batched
       // kernels) and 8^3 (member by member), complex64, one host round trip each
        const int sizes[3] = {16, 32, 8};
        std::vector<ses::gpu::SplitOperator3D> ops;
        std::vector<ses::gpu::Field3D> in, out;
        std::vector<std::vector<cd>> want;
        for (int s : sizes) {
            const double box[6] = {-4, 4, -4, 4, -4, 4};
            const int n[3] = {s, s, s};
            const double c[3] = {0, 0, 0}, r0[3] = {0.5, 0, 0}, sg[3] = {1.0, 1.0, 1.0}, k0[3] = {1, 0, 0};
            const int N = s * s * s;
            std::vector<double> V(N);
            seso_harmonic3d(box, n, 1.0, c, V.data());
            const ses::gpu::Grid3D g{{-4, 4, s}, {-4, 4, s}, {-4, 4, s}};
            ops.emplace_back(g, V, 0.01, 1.0, SES_C64);
            in.emplace_back(g);
            out.emplace_back(g);
            seso_gaussian3d(box, n, r0, sg, k0, reinterpret_cast<double*>(in.back().data().data()));
            std::vector<cd> ref = in.back().data();
            seso_step3d(box, n, V.data(), 0.01, 1.0, nullptr, reinterpret_cast<double*>(ref.data()), 15);
            want.push_back(ref);
        }
        ses::gpu::Batch b;
        for (auto& op : ops) b.add(op);
        const std::vector<ses_observables> obs = b.run({&in[0], &in[1], &in[2]}, 15, false, {&out[0], &out[1], &out[2]});
        double worst = 0;
        for (std::size_t m = 0; m < ops.size(); ++m) {
            double num = 0, den = 0;
            for (std::size_t i = 0; i < want[m].size(); ++i) {
                num += std::norm(out[m].data()[i] - want[m][i]);
                den += std::norm(want[m][i]);
            }
            worst = std::fmax(worst, std::sqrt(num / den));
        }
        std::printf("  batch round trip: worst rel L2 vs the FP64 core %.3e\n", worst);
        EXPECT(worst < 1e-5, "batch round trip vs FP64 core");
        EXPECT(obs.size() == 3 && std::fabs(obs[1].norm - 1.0) < 1e-5, "batch observables");
        bool threw = false;
        try {
            b.run({&in[1], &in[0], &in[2]}, 1, false, {});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw, "batch run rejects a field of the wrong size");
    }
    {  // simulation_test.cpp: WavepacketSimulation on 16^3 harmonic, r0 (2,0,0), k0 (0,0.5,0), dt 0.02
        const double box[6] = {-8, 8, -8, 8, -8, 8};
        const int n[3] = {16, 16, 16};
        const double c[3] = {0, 0, 0}, r0[3] = {2, 0, 0}, sg[3] = {1, 1, 1}, k0[3] = {0, 0.5, 0};
        std::vector<double> V(4096);
        seso_harmonic3d(box, n, 1.0, c, V.data());
        const ses::gpu::Grid3D g{{-8, 8, 16}, {-8, 8, 16}, {-8, 8, 16}};
        ses::gpu::WavepacketSimulation sim{ses::gpu::WavepacketSimulation::Config{
            g, V, ses::gpu::Vec3d{2, 0, 0}, ses::gpu::Vec3d{1, 1, 1}, ses::gpu::Vec3d{0, 0.5, 0}, 0.02}};
        EXPECT(sim.time() == 0.0, "simulation time starts at 0");
        std::vector<cd> manual(4096);
        seso_gaussian3d(box, n, r0, sg, k0, reinterpret_cast<double*>(manual.data()));
        double d0 = 0;  // host builder vs the oracle's (bit-pinned to the reference's)
        for (int i = 0; i < 4096; ++i) d0 = std::fmax(d0, std::abs(sim.psi().data()[i] - manual[i]));
        EXPECT(d0 < 1e-15, "gaussian_wavepacket matches the reference builder");
        sim.advance(3);
        sim.advance(2);
        EXPECT(std::fabs(sim.time() - 5 * 0.02) < 1e-15, "time advances by steps x dt");
        seso_step3d(box, n, V.data(), 0.02, 1.0, nullptr, reinterpret_cast<double*>(manual.data()), 5);
        double md = 0;  // MatchesManualPropagation
        for (int i = 0; i < 4096; ++i) {
            md = std::fmax(md, std::fabs(sim.psi().data()[i].real() - manual[i].real()));
            md = std::fmax(md, std::fabs(sim.psi().data()[i].imag() - manual[i].imag()));
        }
        std::printf("  simulation vs manual propagation: max diff %.3e\n", md);
        EXPECT(md < 1e-13, "simulation matches manual propagation");
        const std::vector<double> rho = sim.density();
        double dd = 0;
        for (int i = 0; i < 4096; ++i) dd = std::fmax(dd, std::fabs(rho[i] - std::norm(sim.psi().data()[i])));
        EXPECT(dd == 0.0, "density is |psi|^2");
        EXPECT(std::fabs(ses::gpu::norm_sq(sim.psi()) - 1.0) < 1e-12, "simulation conserves norm");
        // Engine::norm_and_peak and scale on the resident field
        const auto np = sim.propagator().norm_and_peak();
        double peak = 0;
        for (double r : rho) peak = std::fmax(peak, r);
        EXPECT(std::fabs(np.sum - ses::gpu::norm_sq(sim.psi())) < 1e-13, "norm_and_peak sum");
        EXPECT(std::fabs(np.peak - peak) <= 1e-15 * peak, "norm_and_peak peak");
        sim.propagator().scale(0.5);
        const auto np2 = sim.propagator().norm_and_peak();
        EXPECT(std::fabs(np2.sum - 0.25 * np.sum) < 1e-13, "scale multiplies psi");
        sim.propagator().scale(2.0);
        ses::gpu::Field3D f{g};
        f.data() = manual;
        sim.set_psi(f);
        EXPECT(sim.psi().data() == manual, "set_psi replaces the field");
        sim.relax(50, 0.01);  // imaginary time keeps the field normalised
        EXPECT(std::fabs(ses::gpu::norm_sq(sim.psi()) - 1.0) < 1e-12, "relax renormalises");
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
