// A pomerol-style user program compiled against the drop-in headers
// (pomerol_b200/host/include) and linked with libpomerol_b200.so: the call
// sequence of the reference's two-particle GF test of a two-bath Anderson
// model (test/Anderson2PGFTest.cpp:37-152) -- expression, index
// classification, Hilbert space, StatesClassification, Hamiltonian,
// DensityMatrix, FieldOperatorContainer, TwoParticleGFContainer with both
// computeAll modes -- checked against that test's golden values.
//
// The model parameters and the golden values are read from a text file (the
// GPU test writes it from tests/golden/reference_kats.json):
//   U mu beta pole_resolution coefficient_tolerance tol
//   n_levels  level_0 hopping_0  level_1 hopping_1 ...
//   n_values  value_0 value_1 ...
// Exit status 0 when every value matches within tol, 1 otherwise.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "pomerol.hpp"

using namespace Pomerol;

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <parameters file>\n", argv[0]);
        return 2;
    }
    std::ifstream in(argv[1]);
    double U, mu, beta, pole_res, coef_tol, tol;
    int nlev, nval;
    in >> U >> mu >> beta >> pole_res >> coef_tol >> tol >> nlev;
    std::vector<double> levels(nlev), hops(nlev);
    for (int i = 0; i < nlev; ++i) in >> levels[i] >> hops[i];
    in >> nval;
    std::vector<double> golden(nval);
    for (auto& g : golden) in >> g;
    if (!in) {
        std::fprintf(stderr, "bad parameters file\n");
        return 2;
    }

    using namespace LatticePresets;
    auto HExpr = CoulombS("C", U, -mu);
    for (int i = 0; i < nlev; ++i) {
        const std::string b = "b" + std::to_string(i);
        HExpr += Level(b, levels[i]);
        HExpr += Hopping("C", b, hops[i]);
    }
    auto IndexInfo = MakeIndexClassification(HExpr);
    auto HS = MakeHilbertSpace(IndexInfo, HExpr);
    HS.compute();
    StatesClassification S;
    S.compute(HS);
    Hamiltonian H(S);
    H.prepare(HExpr, HS, MPI_COMM_WORLD);
    H.compute(MPI_COMM_WORLD);
    DensityMatrix rho(S, H, beta);
    rho.prepare();
    rho.compute();

    const ParticleIndex d0 = IndexInfo.getIndex("C", 0, down), u0 = IndexInfo.getIndex("C", 0, up);
    FieldOperatorContainer Ops(IndexInfo, HS, S, H, std::set<ParticleIndex>{u0, d0});
    Ops.prepareAll(HS);
    Ops.computeAll();

    const IndexCombination4 uuuu(u0, u0, u0, u0), dddd(d0, d0, d0, d0);
    // Each mode runs on a container of its own, as each SECTION of the
    // reference test re-runs the setup: a computed element returns an empty
    // list from a second compute() (TwoParticleGF.cpp:166-167).
    auto make_chi = [&]() {
        auto Chi = std::make_unique<TwoParticleGFContainer>(IndexInfo, S, H, rho, Ops);
        Chi->PoleResolution = pole_res;
        Chi->CoefficientTolerance = coef_tol;
        Chi->prepareAll({uuuu, IndexCombination4(u0, d0, u0, d0), dddd});
        return Chi;
    };

    const ComplexType w0 = I * M_PI / beta, W1 = I * 2.0 * M_PI / beta;
    int bad = 0;
    auto check = [&](const char* mode, int k, ComplexType v) {
        const double err = std::abs(v - ComplexType(golden[k], 0.0));
        if (!(err <= tol)) {
            std::fprintf(stderr, "%s: value %d = (%.12e, %.12e), golden %.12e, |diff| %.3e\n", mode, k, v.real(),
                         v.imag(), golden[k], err);
            ++bad;
        }
    };
    // mode 1: computeAll without frequencies, then point evaluation
    auto Chi1 = make_chi();
    Chi1->computeAll(false, {}, MPI_COMM_WORLD, true);
    TwoParticleGF const& cu = (*Chi1)(uuuu);
    TwoParticleGF const& cd = (*Chi1)(dddd);
    for (int k = 0; k < nval; ++k) {
        const ComplexType wp = I * (2.0 * k + 1.0) * M_PI / beta;
        check("point uuuu", k, cu(w0 + W1, wp, w0));
        check("point dddd", k, cd(w0 + W1, wp, w0));
    }
    // mode 2: computeAll on an explicit frequency list
    FreqVec3 freqs;
    for (int k = 0; k < nval; ++k) freqs.emplace_back(w0 + W1, I * (2.0 * k + 1.0) * M_PI / beta, w0);
    auto Chi2 = make_chi();
    auto data = Chi2->computeAll(true, freqs, MPI_COMM_WORLD, true);
    if ((int)data[uuuu].size() != nval || (int)data[dddd].size() != nval) {
        std::fprintf(stderr, "computeAll returned %zu and %zu values, expected %d\n", data[uuuu].size(),
                     data[dddd].size(), nval);
        return 1;
    }
    for (int k = 0; k < nval; ++k) {
        check("list uuuu", k, data[uuuu][k]);
        check("list dddd", k, data[dddd][k]);
    }
    std::printf("drop-in G2 program: %d mismatches of %d values\n", bad, 4 * nval);
    return bad == 0 ? 0 : 1;
}
