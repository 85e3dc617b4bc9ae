// Correlators of the drop-in API: GreensFunction, GFContainer,
// Susceptibility, EnsembleAverage, TwoParticleGF, TwoParticleGFContainer,
// ThreePointSusceptibility, ThreePointSusceptibilityContainer, Vertex4.
// Public members, signatures and frequency conventions follow the reference
// (GreensFunction.hpp:83-147, GFContainer.hpp:40-111, Susceptibility.hpp:75-171,
// EnsembleAverage.cpp:27-67, TwoParticleGF.hpp:111-187,
// TwoParticleGFContainer.hpp:52-93, IndexContainer4.hpp:138-273,
// ThreePointSusceptibility.hpp:67-177, ThreePointSusceptibilityContainer.hpp:35-108).
//
// Evaluation runs on the GPU: point queries by Matsubara index are served
// from a cache that is filled a whole frequency window (G, chi) or cube (G2)
// at a time by one device call.
#pragma once

#include <functional>
#include <map>
#include <memory>
#include <set>
#include <tuple>
#include <vector>

#include "ED.hpp"

namespace Pomerol {

struct IndexCombination2 {
    ParticleIndex Index1, Index2;
    IndexCombination2(ParticleIndex a, ParticleIndex b) : Index1(a), Index2(b) {}
    bool operator<(IndexCombination2 const& o) const { return std::tie(Index1, Index2) < std::tie(o.Index1, o.Index2); }
    bool operator==(IndexCombination2 const& o) const { return Index1 == o.Index1 && Index2 == o.Index2; }
};

struct IndexCombination4 {
    ParticleIndex Index1, Index2, Index3, Index4;
    IndexCombination4(ParticleIndex a, ParticleIndex b, ParticleIndex c, ParticleIndex d)
        : Index1(a), Index2(b), Index3(c), Index4(d) {}
    bool operator<(IndexCombination4 const& o) const {
        return std::tie(Index1, Index2, Index3, Index4) < std::tie(o.Index1, o.Index2, o.Index3, o.Index4);
    }
    bool operator==(IndexCombination4 const& o) const {
        return Index1 == o.Index1 && Index2 == o.Index2 && Index3 == o.Index3 && Index4 == o.Index4;
    }
};

using FreqTuple3 = std::tuple<ComplexType, ComplexType, ComplexType>;
using FreqVec3 = std::vector<FreqTuple3>;

// ------------------------------------------------------------ single particle
class GreensFunction : public Thermal, public ComputableObject {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-8;

    GreensFunction(StatesClassification const& S, Hamiltonian const& H, FieldOperator const& F1,
                   FieldOperator const& F2, DensityMatrix const& DM);
    void prepare();
    void compute();
    ParticleIndex getIndex(std::size_t Position) const;
    ComplexType operator()(long MatsubaraNumber) const;
    ComplexType operator()(ComplexType z) const;
    // Batched evaluation at many complex frequencies (one device call).
    std::vector<ComplexType> values(std::vector<ComplexType> const& z) const;
    bool isVanishing() const { return Vanishing; }

private:
    StatesClassification const& S;
    Hamiltonian const& H;
    FieldOperator const& F1;
    FieldOperator const& F2;
    DensityMatrix const& DM;
    bool Vanishing = true;
    std::vector<int> Outer, Inner;
    mutable std::map<long, ComplexType> Cache;
};

class GFContainer : public Thermal {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-8;

    GFContainer(IndexClassification const& IndexInfo, StatesClassification const& S, Hamiltonian const& H,
                DensityMatrix const& DM, FieldOperatorContainer const& Ops, bool Anomalous = false);
    void prepareAll(std::set<IndexCombination2> const& Indices = {});
    void computeAll();
    GreensFunction& operator()(IndexCombination2 const& Indices);
    GreensFunction& operator()(ParticleIndex Index1, ParticleIndex Index2) {
        return (*this)(IndexCombination2(Index1, Index2));
    }
    bool isInContainer(IndexCombination2 const& Indices) const { return ElementsMap.count(Indices) > 0; }

private:
    std::shared_ptr<GreensFunction> createElement(IndexCombination2 const& Indices) const;
    ParticleIndex NumIndices;
    StatesClassification const& S;
    Hamiltonian const& H;
    DensityMatrix const& DM;
    FieldOperatorContainer const& Operators;
    bool Anomalous;
    std::map<IndexCombination2, std::shared_ptr<GreensFunction>> ElementsMap;
};

// ------------------------------------------------------------ susceptibility
class EnsembleAverage : public Thermal, public ComputableObject {
public:
    EnsembleAverage(MonomialOperator const& A, DensityMatrix const& DM);
    void compute();
    ComplexType operator()() const { return Result; }
    ComplexType getResult() const { return Result; }

private:
    MonomialOperator const& A;
    DensityMatrix const& DM;
    ComplexType Result = 0;
};

class Susceptibility : public Thermal, public ComputableObject {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-8;

    Susceptibility(StatesClassification const& S, Hamiltonian const& H, MonomialOperator const& A,
                   MonomialOperator const& B, DensityMatrix const& DM);
    void prepare();
    void compute();
    void subtractDisconnected();
    void subtractDisconnected(ComplexType ave_A, ComplexType ave_B);
    void subtractDisconnected(EnsembleAverage& EA_A, EnsembleAverage& EA_B);
    ComplexType operator()(long MatsubaraNumber) const;
    ComplexType operator()(ComplexType z) const;
    std::vector<ComplexType> values(std::vector<ComplexType> const& z) const;
    bool isVanishing() const { return Vanishing; }

private:
    StatesClassification const& S;
    Hamiltonian const& H;
    MonomialOperator const& A;
    MonomialOperator const& B;
    DensityMatrix const& DM;
    bool Vanishing = true;
    bool SubtractDisconnected = false;
    ComplexType ave_A = 0, ave_B = 0;
    std::vector<int> Outer, Inner;
    mutable std::map<long, ComplexType> Cache;
};

// ------------------------------------------------------------ two particle
class TwoParticleGF : public Thermal, public ComputableObject {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-16;
    // Sub-terms are anchored on states with weight > AnchorTolerance (a
    // negative value, the default, takes CoefficientTolerance).  The part it
    // drops is bounded by (beta/pi)^3 times the Boltzmann weight of the
    // dropped states.  ExactSum = true sums every state quadruple instead.
    RealType AnchorTolerance = -1;
    bool ExactSum = false;
    // SplitProducts = true runs the anchored sum's largest products on the int8
    // tensor cores (six 7-bit slices per operand, FP64 recombination; about
    // 1e-11 relative error of G2).  Ignored with ExactSum.
    bool SplitProducts = false;
    int SplitSlices = 6;  // 7-bit digits per element of the split products (1..8)

    TwoParticleGF(StatesClassification const& S, Hamiltonian const& H, AnnihilationOperator const& C1,
                  AnnihilationOperator const& C2, CreationOperator const& CX3, CreationOperator const& CX4,
                  DensityMatrix const& DM);
    void prepare();
    std::vector<ComplexType> compute(bool clear = false, FreqVec3 const& freqs = {},
                                     MPI_Comm const& comm = MPI_COMM_WORLD);
    ParticleIndex getIndex(std::size_t Position) const;
    ComplexType operator()(ComplexType z1, ComplexType z2, ComplexType z3) const;
    ComplexType operator()(long MatsubaraNumber1, long MatsubaraNumber2, long MatsubaraNumber3) const;
    bool isVanishing() const { return Vanishing; }
    std::size_t getNumParts() const { return Parts.size(); }
    // Evaluate at many triples with one device call.
    std::vector<ComplexType> values(FreqVec3 const& freqs) const;
    // Block chains (S1..S4), operator order and permutation, for inspection.
    std::vector<pgx_g2_part> const& deviceParts() const { return Parts; }

private:
    StatesClassification const& S;
    Hamiltonian const& H;
    AnnihilationOperator const& C1;
    AnnihilationOperator const& C2;
    CreationOperator const& CX3;
    CreationOperator const& CX4;
    DensityMatrix const& DM;
    bool Vanishing = true;
    std::vector<pgx_g2_part> Parts;
    std::vector<std::array<MonomialOperator const*, 4>> PartOps;
    mutable std::map<std::tuple<long, long, long>, ComplexType> Cache;
};

template <typename ElementType> struct ElementWithPermFreq {
    std::shared_ptr<ElementType> pElement;
    Permutation4 FrequenciesPermutation;
    ComplexType operator()(long n1, long n2, long n3) const {
        long ns[4] = {n1, n2, n3, n1 + n2 - n3};
        return (*pElement)(ns[FrequenciesPermutation.perm[0]], ns[FrequenciesPermutation.perm[1]],
                           ns[FrequenciesPermutation.perm[2]]) *
               RealType(FrequenciesPermutation.sign);
    }
    operator ElementType&() { return *pElement; }
    ElementType& element() { return *pElement; }
};

class TwoParticleGFContainer : public Thermal {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-16;
    bool SplitProducts = false;  // passed to every element (TwoParticleGF::SplitProducts)
    RealType AnchorTolerance = -1;  // passed to every element (TwoParticleGF::AnchorTolerance)
    int SplitSlices = 6;            // passed to every element (TwoParticleGF::SplitSlices)

    TwoParticleGFContainer(IndexClassification const& IndexInfo, StatesClassification const& S, Hamiltonian const& H,
                           DensityMatrix const& DM, FieldOperatorContainer const& Ops);
    void prepareAll(std::set<IndexCombination4> const& Indices = {});
    std::map<IndexCombination4, std::vector<ComplexType>> computeAll(bool clearTerms = false,
                                                                     FreqVec3 const& freqs = {},
                                                                     MPI_Comm const& comm = MPI_COMM_WORLD,
                                                                     bool split = true);
    ElementWithPermFreq<TwoParticleGF>& operator()(IndexCombination4 const& Indices);
    ElementWithPermFreq<TwoParticleGF>& operator()(ParticleIndex i, ParticleIndex j, ParticleIndex k, ParticleIndex l) {
        return (*this)(IndexCombination4(i, j, k, l));
    }
    bool isInContainer(IndexCombination4 const& Indices) const { return ElementsMap.count(Indices) > 0; }
    std::map<IndexCombination4, std::shared_ptr<TwoParticleGF>> const& nonTrivialElements() const {
        return NonTrivialElements;
    }

private:
    ElementWithPermFreq<TwoParticleGF>& create(IndexCombination4 const& Indices);
    ParticleIndex NumIndices;
    StatesClassification const& S;
    Hamiltonian const& H;
    DensityMatrix const& DM;
    FieldOperatorContainer const& Operators;
    std::map<IndexCombination4, ElementWithPermFreq<TwoParticleGF>> ElementsMap;
    std::map<IndexCombination4, std::shared_ptr<TwoParticleGF>> NonTrivialElements;
};

// ------------------------------------------------------------ three point
// Channel of a three-point susceptibility (Misc.hpp:160-164).
enum Channel : int { PP = PGX_PP, PH = PGX_PH, xPH = PGX_XPH };

using FreqTuple2 = std::tuple<ComplexType, ComplexType>;
using FreqVec2 = std::vector<FreqTuple2>;

// Three-point fermion-boson susceptibility (ThreePointSusceptibility.hpp:67-158):
// part selection on the host as ThreePointSusceptibility::prepare does, the
// Lehmann sum over every state triple on the GPU (pgx_chi3).
class ThreePointSusceptibility : public Thermal, public ComputableObject {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-16;

    ThreePointSusceptibility(Channel channel, StatesClassification const& S, Hamiltonian const& H,
                             CreationOperator const& CX1, AnnihilationOperator const& C2, CreationOperator const& CX3,
                             AnnihilationOperator const& C4, DensityMatrix const& DM);
    void prepare();
    std::vector<ComplexType> compute(bool clear = false, FreqVec2 const& freqs = {},
                                     MPI_Comm const& comm = MPI_COMM_WORLD);
    ParticleIndex getIndex(std::size_t Position) const;
    ComplexType operator()(ComplexType z1, ComplexType z2) const;
    ComplexType operator()(long MatsubaraNumber1, long MatsubaraNumber2) const;
    bool isVanishing() const { return Vanishing; }
    std::size_t getNumParts() const { return Parts.size(); }
    // Evaluate at many duplets with one device call.
    std::vector<ComplexType> values(FreqVec2 const& freqs) const;
    std::vector<pgx_chi3_part> const& deviceParts() const { return Parts; }

private:
    MonomialOperator const& getF2() const;
    MonomialOperator const& getB1() const;
    MonomialOperator const& getB2() const;
    Channel channel;
    StatesClassification const& S;
    Hamiltonian const& H;
    CreationOperator const& CX1;
    AnnihilationOperator const& C2;
    CreationOperator const& CX3;
    AnnihilationOperator const& C4;
    DensityMatrix const& DM;
    bool Vanishing = true;
    std::vector<pgx_chi3_part> Parts;
    std::vector<std::array<MonomialOperator const*, 4>> PartOps;
    mutable std::map<std::pair<long, long>, ComplexType> Cache;
};

// Container of three-point susceptibilities over index quadruples
// (ThreePointSusceptibilityContainer.hpp:35-108 on IndexContainer4.hpp:138-237).
class ThreePointSusceptibilityContainer : public Thermal {
public:
    RealType PoleResolution = 1e-8;
    RealType CoefficientTolerance = 1e-16;

    ThreePointSusceptibilityContainer(Channel channel, IndexClassification const& IndexInfo,
                                      StatesClassification const& S, Hamiltonian const& H, DensityMatrix const& DM,
                                      FieldOperatorContainer const& Ops);
    void prepareAll(std::set<IndexCombination4> const& Indices = {});
    std::map<IndexCombination4, std::vector<ComplexType>> computeAll(bool clearTerms = false,
                                                                     FreqVec2 const& freqs = {},
                                                                     MPI_Comm const& comm = MPI_COMM_WORLD);
    ElementWithPermFreq<ThreePointSusceptibility>& operator()(IndexCombination4 const& Indices);
    ElementWithPermFreq<ThreePointSusceptibility>& operator()(ParticleIndex i, ParticleIndex j, ParticleIndex k,
                                                              ParticleIndex l) {
        return (*this)(IndexCombination4(i, j, k, l));
    }
    bool isInContainer(IndexCombination4 const& Indices) const { return ElementsMap.count(Indices) > 0; }

private:
    ElementWithPermFreq<ThreePointSusceptibility>& create(IndexCombination4 const& Indices);
    Channel channel;
    ParticleIndex NumIndices;
    StatesClassification const& S;
    Hamiltonian const& H;
    DensityMatrix const& DM;
    FieldOperatorContainer const& Operators;
    std::map<IndexCombination4, ElementWithPermFreq<ThreePointSusceptibility>> ElementsMap;
    std::map<IndexCombination4, std::shared_ptr<ThreePointSusceptibility>> NonTrivialElements;
};

// Two-particle vertex (Vertex4.hpp:38-104, Vertex4.cpp:34-53):
//   Gamma(n1, n2, n3) = chi(n1, n2, n3) + beta G13(n1) G24(n2) [n1 == n3]
//                                        - beta G14(n1) G23(n2) [n2 == n3].
// compute(N) caches the values on the box of MatsubaraContainer4
// (MatsubaraContainers.hpp:80-107: bosonic index Omega = n1 + n2 in
// [-2N, 2N - 2], n1 and n3 over the 2N - |Omega + 1| fermionic indices that
// keep n1, n2, n3 inside [-N, N)); chi is evaluated for the whole box in one
// device call.
class Vertex4 : public Thermal, public ComputableObject {
public:
    Vertex4(TwoParticleGF const& Chi, GreensFunction const& G13, GreensFunction const& G24, GreensFunction const& G14,
            GreensFunction const& G23);
    void compute(long NumberOfMatsubaras = 0);
    ComplexType operator()(long MatsubaraNumber1, long MatsubaraNumber2, long MatsubaraNumber3) const;
    ComplexType value(long MatsubaraNumber1, long MatsubaraNumber2, long MatsubaraNumber3) const;
    long getNumberOfMatsubaras() const { return NumberOfMatsubaras; }

private:
    ComplexType disconnected(long n1, long n2, long n3) const;
    TwoParticleGF const& Chi;
    GreensFunction const& G13;
    GreensFunction const& G24;
    GreensFunction const& G14;
    GreensFunction const& G23;
    long NumberOfMatsubaras = 0;
    std::vector<std::vector<ComplexType>> Values;  // per bosonic index: size x size, row n1, column n3
    std::vector<long> Offset, Size;
};

}  // namespace Pomerol
