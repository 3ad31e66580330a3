// setups.cpp -- see setups.hpp.  The Python mirror (heraclespp_b200/setups.py)
// evaluates the same formulas; tests compare the two.
#include "setups.hpp"

#include <cmath>
#include <stdexcept>

namespace hcl::host {

namespace {

uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

constexpr double kPi = 3.141592653589793238462643383279502884;

template <class F>
void for_interior(SetupGrid const& g, F&& f)
{
    int b[3], e[3];
    for (int d = 0; d < 3; ++d) {
        b[d] = d < g.ndim ? g.ng : 0;
        e[d] = d < g.ndim ? g.n[d] - g.ng : 1;
    }
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const int64_t c = i + (int64_t)g.n[0] * (j + (int64_t)g.n[1] * k);
                f(c, i, j, k, i - b[0], j - b[1], k - b[2]);
            }
        }
    }
}

} // namespace

double hash_uniform(uint64_t seed, uint64_t i, uint64_t j, uint64_t k)
{
    uint64_t h = splitmix64(k);
    h = splitmix64(h ^ j);
    h = splitmix64(h ^ i);
    h = splitmix64(h ^ seed);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

void setup_initial_prim(std::string const& name, INIReader const& r, SetupGrid const& g, double* rho, double* u,
                        double* P)
{
    const int64_t N = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const int nd = g.ndim;
    const double* X = g.xc[0];
    const double* Y = g.xc[1];
    const double* Z = g.xc[2];
    if (name == "shock_tube") {
        // setups/shock_tube/setup.hpp:38-46 (defaults 1.0) and :74-91
        const double rho0 = r.GetReal("Initialisation", "rho0", 1.0);
        const double rho1 = r.GetReal("Initialisation", "rho1", 1.0);
        const double u0 = r.GetReal("Initialisation", "u0", 1.0);
        const double u1 = r.GetReal("Initialisation", "u1", 1.0);
        const double P0 = r.GetReal("Initialisation", "P0", 1.0);
        const double P1 = r.GetReal("Initialisation", "P1", 1.0);
        const double inter = r.GetReal("Initialisation", "inter", 1.0);
        for_interior(g, [&](int64_t c, int i, int, int, int, int, int) {
            const bool left = X[i] <= inter;
            rho[c] = left ? rho0 : rho1;
            P[c] = left ? P0 : P1;
            for (int d = 0; d < nd; ++d) {
                u[c + N * d] = left ? u0 : u1;
            }
        });
        return;
    }
    if (name == "advection_sinus") {
        // setups/advection_sinus/setup.hpp:32-72
        const double u0 = r.GetReal("Initialisation", "u0", 1.0);
        const double P0 = r.GetReal("Initialisation", "P0", 1.0);
        for_interior(g, [&](int64_t c, int i, int, int, int, int, int) {
            rho[c] = 1. + (1E-1 * std::sin(2 * kPi * X[i]));
            for (int d = 0; d < nd; ++d) {
                u[c + N * d] = u0;
            }
            P[c] = P0;
        });
        return;
    }
    if (name == "kelvin_helmholtz") {
        const uint64_t seed = (uint64_t)r.GetInteger("Initialisation", "seed", 1234);
        const double noise = r.GetReal("Initialisation", "noise", 1e-3);
        for_interior(g, [&](int64_t c, int i, int j, int, int ii, int jj, int kk) {
            const bool band = std::fabs(Y[j] - 0.5) < 0.25;
            rho[c] = band ? 2.0 : 1.0;
            u[c] = band ? 0.5 : -0.5;
            const double h = hash_uniform(seed, (uint64_t)ii, (uint64_t)jj, (uint64_t)kk);
            u[c + N] = 0.01 * std::sin(4 * kPi * X[i]) + noise * (2.0 * h - 1.0);
            P[c] = 2.5;
        });
        return;
    }
    if (name == "rayleigh_taylor3d") {
        const uint64_t seed = (uint64_t)r.GetInteger("Initialisation", "seed", 4321);
        const double noise = r.GetReal("Initialisation", "noise", 1e-4);
        const double gz = r.GetReal("Gravity", "gx2", -0.1);
        for_interior(g, [&](int64_t c, int i, int j, int k, int ii, int jj, int kk) {
            const bool upper = Z[k] > 0.5;
            rho[c] = upper ? 2.0 : 1.0;
            P[c] = 2.5 + (upper ? 2.0 : 1.0) * gz * (Z[k] - 0.5);
            u[c] = 0.0;
            u[c + N] = 0.0;
            const double h = hash_uniform(seed, (uint64_t)ii, (uint64_t)jj, (uint64_t)kk);
            const double mode =
                    0.01 * (1 + std::cos(4 * kPi * X[i])) * (1 + std::cos(4 * kPi * Y[j])) * (1 + std::cos(3 * kPi * Z[k])) / 8;
            u[c + 2 * N] = mode + noise * (2.0 * h - 1.0);
        });
        return;
    }
    if (name == "gresho_vortex") {
        const double p0 = r.GetReal("Initialisation", "p0", 5.0);
        const double rho0 = r.GetReal("Initialisation", "rho0", 1.0);
        for_interior(g, [&](int64_t c, int i, int j, int, int, int, int) {
            const double x = X[i] - 0.5;
            const double y = Y[j] - 0.5;
            const double rr = std::sqrt(x * x + y * y);
            const double th = std::atan2(y, x);
            double uphi, pr;
            if (rr < 0.2) {
                uphi = 5 * rr;
                pr = p0 + 12.5 * rr * rr;
            } else if (rr < 0.4) {
                uphi = 2 - 5 * rr;
                pr = p0 + 12.5 * rr * rr + 4 - 20 * rr + 4 * std::log(5 * rr);
            } else {
                uphi = 0.0;
                pr = p0 - 2 + 4 * std::log(2.0);
            }
            rho[c] = rho0;
            u[c] = -uphi * std::sin(th);
            u[c + N] = uphi * std::cos(th);
            P[c] = pr;
        });
        return;
    }
    if (name == "four_quadrant") {
        // seeded quadrant states: rho, p in U[0.1, 2], velocities in U[-1, 1]
        const uint64_t seed = (uint64_t)r.GetInteger("Initialisation", "seed", 7);
        double st[4][4];
        for (int q = 0; q < 4; ++q) {
            st[q][0] = 0.1 + 1.9 * hash_uniform(seed, (uint64_t)q, 0, 1);
            st[q][1] = -1.0 + 2.0 * hash_uniform(seed, (uint64_t)q, 1, 1);
            st[q][2] = -1.0 + 2.0 * hash_uniform(seed, (uint64_t)q, 2, 1);
            st[q][3] = 0.1 + 1.9 * hash_uniform(seed, (uint64_t)q, 3, 1);
        }
        for_interior(g, [&](int64_t c, int i, int j, int, int, int, int) {
            const int q = (X[i] > 0.5 ? 1 : 0) + 2 * (Y[j] > 0.5 ? 1 : 0);
            rho[c] = st[q][0];
            u[c] = st[q][1];
            u[c + N] = st[q][2];
            P[c] = st[q][3];
        });
        return;
    }
    throw std::runtime_error("Setup not implemented: " + name);
}

} // namespace hcl::host
