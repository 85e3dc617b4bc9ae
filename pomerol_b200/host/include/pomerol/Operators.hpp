// Fermionic polynomial expressions and lattice presets.
//
// The reference builds these with libcommute (un-vendored dependency,
// v1.0.0): `Operators::c`, `c_dag`, `n`, `hc` (Operators.hpp) and the
// LatticePresets factories (LatticePresets.cpp:46-48 Level, :75-83 Hopping,
// :140-147 Magnetization, Pairing, NupNdown, Spinflip, PairHopping, :402-409
// CoulombS, :423-448 CoulombP).  This is an independent, fermion-only
// implementation with the same index tuples (label, orbital, spin).
#pragma once

#include <complex>
#include <map>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace Pomerol {

namespace LatticePresets {
enum spin : short { undef = -1, down = 0, up = 1 };
}
using LatticePresets::spin;

using IndexTuple = std::tuple<std::string, unsigned short, spin>;

// One creation (dagger) or annihilation operator.
struct Generator {
    bool dagger;
    IndexTuple index;
    bool operator<(Generator const& o) const { return std::tie(dagger, index) < std::tie(o.dagger, o.index); }
    bool operator==(Generator const& o) const { return dagger == o.dagger && index == o.index; }
};

// Product of generators in operator order (leftmost acts last).
using Monomial = std::vector<Generator>;

namespace Operators {

template <typename S> class expression {
public:
    using scalar_type = S;
    std::map<Monomial, S> terms;

    expression() = default;
    template <typename S2, typename = std::enable_if_t<!std::is_same<S, S2>::value && std::is_convertible<S2, S>::value>>
    expression(expression<S2> const& o) {
        for (auto const& kv : o.terms) terms[kv.first] = S(kv.second);
    }

    std::size_t size() const { return terms.size(); }

    expression& operator+=(expression const& o) {
        for (auto const& kv : o.terms) add(kv.first, kv.second);
        return *this;
    }
    expression& operator-=(expression const& o) {
        for (auto const& kv : o.terms) add(kv.first, -kv.second);
        return *this;
    }
    expression& operator*=(S s) {
        for (auto& kv : terms) kv.second *= s;
        return *this;
    }
    void add(Monomial const& m, S c) {
        auto it = terms.find(m);
        if (it == terms.end())
            terms.emplace(m, c);
        else {
            it->second += c;
            if (it->second == S(0)) terms.erase(it);
        }
    }
    expression dagger() const {
        expression r;
        for (auto const& kv : terms) {
            Monomial m;
            for (auto it = kv.first.rbegin(); it != kv.first.rend(); ++it) m.push_back(Generator{!it->dagger, it->index});
            r.add(m, conj_(kv.second));
        }
        return r;
    }
    bool is_complex() const {
        if constexpr (std::is_same<S, double>::value) return false;
        else {
            for (auto const& kv : terms)
                if (std::imag(kv.second) != 0.0) return true;
            return false;
        }
    }

private:
    static S conj_(S x) {
        if constexpr (std::is_same<S, double>::value) return x;
        else return std::conj(x);
    }
};

template <typename S> expression<S> operator+(expression<S> a, expression<S> const& b) { return a += b; }
template <typename S> expression<S> operator-(expression<S> a, expression<S> const& b) { return a -= b; }
template <typename S> expression<S> operator-(expression<S> a) { return a *= S(-1); }
inline expression<std::complex<double>> operator+(expression<double> const& a, expression<std::complex<double>> const& b) {
    return expression<std::complex<double>>(a) + b;
}
inline expression<std::complex<double>> operator+(expression<std::complex<double>> const& a, expression<double> const& b) {
    return a + expression<std::complex<double>>(b);
}
template <typename S> expression<S> operator*(expression<S> const& a, expression<S> const& b) {
    expression<S> r;
    for (auto const& x : a.terms)
        for (auto const& y : b.terms) {
            Monomial m = x.first;
            m.insert(m.end(), y.first.begin(), y.first.end());
            r.add(m, x.second * y.second);
        }
    return r;
}
template <typename S> expression<S> operator*(S s, expression<S> e) { return e *= s; }
template <typename S> expression<S> operator*(expression<S> e, S s) { return e *= s; }
inline expression<std::complex<double>> operator*(std::complex<double> s, expression<double> const& e) {
    return s * expression<std::complex<double>>(e);
}

// `x + hc` adds the Hermitian conjugate of x.
struct hc_tag {};
constexpr hc_tag hc{};
template <typename S> expression<S> operator+(expression<S> const& e, hc_tag) { return e + e.dagger(); }

template <typename S = double>
expression<S> c(std::string const& label, unsigned short orbital = 0, spin s = spin::down) {
    expression<S> e;
    e.add(Monomial{Generator{false, IndexTuple{label, orbital, s}}}, S(1));
    return e;
}
template <typename S = double>
expression<S> c_dag(std::string const& label, unsigned short orbital = 0, spin s = spin::down) {
    expression<S> e;
    e.add(Monomial{Generator{true, IndexTuple{label, orbital, s}}}, S(1));
    return e;
}
template <typename S = double>
expression<S> n(std::string const& label, unsigned short orbital = 0, spin s = spin::down) {
    return c_dag<S>(label, orbital, s) * c<S>(label, orbital, s);
}

}  // namespace Operators

using RealExpr = Operators::expression<double>;
using ComplexExpr = Operators::expression<std::complex<double>>;

namespace LatticePresets {

RealExpr Level(std::string const& Label, double Eps, unsigned short Orbital, spin Spin);
ComplexExpr Level(std::string const& Label, std::complex<double> Eps, unsigned short Orbital, spin Spin);
RealExpr Level(std::string const& Label, double Eps, unsigned short NOrbitals = 1);

RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital1,
                 unsigned short Orbital2, spin Spin1, spin Spin2);
ComplexExpr Hopping(std::string const& Label1, std::string const& Label2, std::complex<double> t,
                    unsigned short Orbital1, unsigned short Orbital2, spin Spin1, spin Spin2);
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital, spin Spin);
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short Orbital1,
                 unsigned short Orbital2);
RealExpr Hopping(std::string const& Label1, std::string const& Label2, double t, unsigned short NOrbitals = 1);

RealExpr Magnetization(std::string const& Label, double H, unsigned short NOrbitals = 1);
RealExpr Pairing(std::string const& Label, double Delta, unsigned short NOrbitals = 1);
RealExpr NupNdown(std::string const& Label1, std::string const& Label2, double U, unsigned short Orbital1,
                  unsigned short Orbital2, spin Spin1, spin Spin2);
RealExpr NupNdown(std::string const& Label, double U, unsigned short Orbital, spin Spin1 = up, spin Spin2 = down);
RealExpr Spinflip(std::string const& Label, double J, unsigned short Orbital1, unsigned short Orbital2, spin Spin1,
                  spin Spin2);
RealExpr PairHopping(std::string const& Label, double J, unsigned short Orbital1, unsigned short Orbital2, spin Spin1,
                     spin Spin2);
RealExpr CoulombS(std::string const& Label, double U, double Eps, unsigned short NOrbitals = 1);
RealExpr CoulombP(std::string const& Label, double U, double U_p, double J, double Eps, unsigned short NOrbitals = 3);
RealExpr CoulombP(std::string const& Label, double U, double J, double Eps, unsigned short NOrbitals = 3);

}  // namespace LatticePresets

}  // namespace Pomerol
