// Core types of the drop-in host layer (namespace Pomerol), mirroring the
// reference's Misc.hpp (types, permutations: Misc.hpp:69-157, Misc.cpp:41-66),
// ComputableObject.hpp:28-59 (status machine) and Thermal.hpp:28-37.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pgx.h"

// The reference takes MPI communicators; this single-GPU build accepts and
// ignores them (no MPI exists here).
#ifndef POMEROL_B200_HAVE_MPI
using MPI_Comm = int;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
#endif

namespace Pomerol {

using RealType = double;
using ComplexType = std::complex<double>;
using ParticleIndex = unsigned int;
using QuantumState = std::uint64_t;
using BlockNumber = int;
using InnerQuantumState = std::uint64_t;
constexpr BlockNumber INVALID_BLOCK_NUMBER = -1;
static ComplexType const I = ComplexType(0.0, 1.0);

struct Permutation3 {
    std::array<std::size_t, 3> perm;
    int sign;
};
struct Permutation4 {
    std::array<std::size_t, 4> perm;
    int sign;
};
extern std::array<Permutation3, 6> const permutations3;
extern std::array<Permutation4, 24> const permutations4;

struct ComputableObject {
    enum StatusEnum { Constructed, Prepared, Computed };

    class StatusMismatch : public std::runtime_error {
    public:
        explicit StatusMismatch(std::string const& s) : std::runtime_error(s) {}
    };

    StatusEnum getStatus() const { return Status; }
    void setStatus(StatusEnum s) {
        if (s > Computed) throw StatusMismatch("Invalid computable object status");
        Status = s;
    }

protected:
    StatusEnum Status = Constructed;
};

struct Thermal {
    RealType beta;
    ComplexType MatsubaraSpacing;
    explicit Thermal(RealType beta) : beta(beta), MatsubaraSpacing(I * M_PI / beta) {}
};

// One GPU context shared by every object of an ED problem (owned through
// the Hamiltonian), taken from and returned to a per-GPU pool of contexts.
// Throws std::runtime_error on any non-OK status.
class Device {
public:
    explicit Device(int device = 0);
    ~Device();
    Device(Device const&) = delete;
    Device& operator=(Device const&) = delete;

    pgx_ctx* ctx() const { return ctx_; }
    void check(int rc, char const* what) const;

    // weights of the current temperature on the device
    RealType weights_beta = -1.0;

private:
    int device_ = 0;
    pgx_ctx* ctx_ = nullptr;
};

}  // namespace Pomerol
