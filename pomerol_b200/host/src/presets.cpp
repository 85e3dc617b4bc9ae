// Lattice presets (same terms as LatticePresets.cpp:46-48, 75-83, 140-147,
// Pairing/NupNdown/Spinflip/PairHopping, 402-409, 423-448) and the core
// tables (Misc.cpp:41-66).
#include <map>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "pomerol.hpp"

namespace Pomerol {

std::array<Permutation3, 6> const permutations3 = {
    {{{0, 1, 2}, 1}, {{0, 2, 1}, -1}, {{1, 0, 2}, -1}, {{1, 2, 0}, 1}, {{2, 0, 1}, 1}, {{2, 1, 0}, -1}}};

std::array<Permutation4, 24> const permutations4 = {
    {{{0, 1, 2, 3}, 1},  {{0, 1, 3, 2}, -1}, {{0, 2, 1, 3}, -1}, {{0, 2, 3, 1}, 1},  {{0, 3, 1, 2}, 1},
     {{0, 3, 2, 1}, -1}, {{1, 0, 2, 3}, -1}, {{1, 0, 3, 2}, 1},  {{1, 2, 0, 3}, 1},  {{1, 2, 3, 0}, -1},
     {{1, 3, 0, 2}, -1}, {{1, 3, 2, 0}, 1},  {{2, 0, 1, 3}, 1},  {{2, 0, 3, 1}, -1}, {{2, 1, 0, 3}, -1},
     {{2, 1, 3, 0}, 1},  {{2, 3, 0, 1}, 1},  {{2, 3, 1, 0}, -1}, {{3, 0, 1, 2}, -1}, {{3, 0, 2, 1}, 1},
     {{3, 1, 0, 2}, 1},  {{3, 1, 2, 0}, -1}, {{3, 2, 0, 1}, -1}, {{3, 2, 1, 0}, 1}}};

// Contexts of destroyed Devices are kept per GPU and handed to the next
// Device on that GPU: its device buffers, streams and pinned staging memory
// are reused (pgx_set_blocks resets the problem, not the allocations), so a
// new Hamiltonian neither allocates nor frees device memory when a previous
// one of similar size existed.  Pooled contexts live until the process ends.
namespace {
std::mutex& pool_mutex() {
    static std::mutex m;
    return m;
}
std::map<int, std::vector<pgx_ctx*>>& context_pool() {
    static auto* p = new std::map<int, std::vector<pgx_ctx*>>();  // never destroyed: outlives static teardown
    return *p;
}
}  // namespace

Device::Device(int device) : device_(device) {
    {
        std::lock_guard<std::mutex> lk(pool_mutex());
        auto& free = context_pool()[device];
        if (!free.empty()) {
            ctx_ = free.back();
            free.pop_back();
            return;
        }
    }
    int rc = pgx_create(device, &ctx_);
    if (rc != PGX_OK) throw std::runtime_error("libpgx: no usable CUDA device (status " + std::to_string(rc) + ")");
}

Device::~Device() {
    if (!ctx_) return;
    std::lock_guard<std::mutex> lk(pool_mutex());
    context_pool()[device_].push_back(ctx_);
}

void Device::check(int rc, char const* what) const {
    if (rc != PGX_OK) throw std::runtime_error(std::string(what) + ": " + pgx_last_error(ctx_));
}

namespace LatticePresets {
using Operators::c;
using Operators::c_dag;
using Operators::n;

RealExpr Level(std::string const& Label, double Eps, unsigned short Orbital, spin Spin) {
    return Eps * n<double>(Label, Orbital, Spin);
}
ComplexExpr Level(std::string const& Label, std::complex<double> Eps, unsigned short Orbital, spin Spin) {
    return Eps * n<std::complex<double>>(Label, Orbital, Spin);
}
RealExpr Level(std::string const& Label, double Eps, unsigned short NOrbitals) {
    RealExpr r;
    for (unsigned short o = 0; o < NOrbitals; ++o) {
        r += Level(Label, Eps, o, up);
        r += Level(Label, Eps, o, down);
    }
    return r;
}

RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital1,
                 unsigned short Orbital2, spin Spin1, spin Spin2) {
    return (t * c_dag<double>(Label1, Orbital1, Spin1) * c<double>(Label2, Orbital2, Spin2)) + Operators::hc;
}
ComplexExpr Hopping(std::string const& Label1, std::string const& Label2, std::complex<double> t,
                    unsigned short Orbital1, unsigned short Orbital2, spin Spin1, spin Spin2) {
    using C = std::complex<double>;
    return (t * c_dag<C>(Label1, Orbital1, Spin1) * c<C>(Label2, Orbital2, Spin2)) + Operators::hc;
}
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital, spin Spin) {
    return Hopping(Label1, Label2, t, Orbital, Orbital, Spin, Spin);
}
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital1,
                 unsigned short Orbital2) {
    return Hopping(Label1, Label2, t, Orbital1, Orbital2, up, up) + Hopping(Label1, Label2, t, Orbital1, Orbital2, down, down);
}
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short NOrbitals) {
    RealExpr r;
    for (unsigned short o = 0; o < NOrbitals; ++o) {
        r += Hopping(Label1, Label2, t, o, up);
        r += Hopping(Label1, Label2, t, o, down);
    }
    return r;
}

RealExpr Magnetization(std::string const& Label, double H, unsigned short NOrbitals) {
    RealExpr r;
    for (unsigned short o = 0; o < NOrbitals; ++o) {
        r += Level(Label, H, o, up);
        r += Level(Label, -H, o, down);
    }
    return r;
}

RealExpr Pairing(std::string const& Label, double Delta, unsigned short NOrbitals) {
    RealExpr r;
    for (unsigned short o = 0; o < NOrbitals; ++o)
        r += (Delta * c_dag<double>(Label, o, up) * c_dag<double>(Label, o, down)) + Operators::hc;
    return r;
}

RealExpr NupNdown(std::string const& Label1, std::string const& Label2, double U, unsigned short Orbital1,
                  unsigned short Orbital2, spin Spin1, spin Spin2) {
    return U * n<double>(Label1, Orbital1, Spin1) * n<double>(Label2, Orbital2, Spin2);
}
RealExpr NupNdown(std::string const& Label, double U, unsigned short Orbital, spin Spin1, spin Spin2) {
    return NupNdown(Label, Label, U, Orbital, Orbital, Spin1, Spin2);
}

RealExpr Spinflip(std::string const& Label, double J, unsigned short Orbital1, unsigned short Orbital2, spin Spin1,
                  spin Spin2) {
    return J * c_dag<double>(Label, Orbital1, Spin1) * c_dag<double>(Label, Orbital2, Spin2) *
           c<double>(Label, Orbital2, Spin1) * c<double>(Label, Orbital1, Spin2);
}

RealExpr PairHopping(std::string const& Label, double J, unsigned short Orbital1, unsigned short Orbital2, spin Spin1,
                     spin Spin2) {
    return J * c_dag<double>(Label, Orbital1, Spin1) * c_dag<double>(Label, Orbital1, Spin2) *
           c<double>(Label, Orbital2, Spin1) * c<double>(Label, Orbital2, Spin2);
}

RealExpr CoulombS(std::string const& Label, double U, double Eps, unsigned short NOrbitals) {
    RealExpr r;
    for (unsigned short o = 0; o < NOrbitals; ++o)
        r += Level(Label, Eps, o, up) + Level(Label, Eps, o, down) + NupNdown(Label, Label, U, o, o, up, down);
    return r;
}

RealExpr CoulombP(std::string const& Label, double U, double U_p, double J, double Eps, unsigned short NOrbitals) {
    if (NOrbitals < 2) throw std::runtime_error("Cannot add multiorbital interaction to a site with 1 orbital");
    RealExpr r;
    for (unsigned short o1 = 0; o1 < NOrbitals; ++o1) {
        for (spin s1 : {up, down}) {
            r += Level(Label, Eps, o1, s1);
            for (unsigned short o2 = 0; o2 < NOrbitals; ++o2)
                if (o1 != o2) r += NupNdown(Label, Label, (U_p - J) / 2.0, o1, o2, s1, s1);
            for (spin s2 : {up, down}) {
                if (s2 >= s1) continue;
                r += NupNdown(Label, Label, U, o1, o1, s1, s2);
                for (unsigned short o2 = 0; o2 < NOrbitals; ++o2) {
                    if (o1 != o2) {
                        r += NupNdown(Label, Label, U_p, o1, o2, s1, s2);
                        r += Spinflip(Label, -J, o1, o2, s1, s2);
                        r += PairHopping(Label, -J, o1, o2, s1, s2);
                    }
                }
            }
        }
    }
    return r;
}

RealExpr CoulombP(std::string const& Label, double U, double J, double Eps, unsigned short NOrbitals) {
    return CoulombP(Label, U, U - 2.0 * J, J, Eps, NOrbitals);
}

}  // namespace LatticePresets
}  // namespace Pomerol
