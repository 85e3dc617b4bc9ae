// Exact-diagonalisation layer of the drop-in API: index classification,
// Hilbert-space partition, block Hamiltonian, density matrix and monomial
// operators.  Same class names, constructor arguments, status machine and
// exceptions as the reference (IndexClassification.hpp:40-141,
// HilbertSpace.hpp:48-169, StatesClassification.hpp:41-118,
// HamiltonianPart.hpp / Hamiltonian.hpp:60-113, DensityMatrix.hpp:56-87,
// MonomialOperator.hpp:60-439, FieldOperatorContainer.hpp:55-93); the
// numerical work runs on the GPU through libpgx.
#pragma once

#include <map>
#include <memory>
#include <set>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "Core.hpp"
#include "Operators.hpp"

namespace Pomerol {

// ---------------------------------------------------------------- indices
class IndexClassification {
public:
    using IndexInfo = IndexTuple;

    IndexClassification() = default;
    template <typename Sc> explicit IndexClassification(Operators::expression<Sc> const& H) {
        for (auto const& kv : H.terms)
            for (auto const& g : kv.first) InfoToIndices.emplace(g.index, 0);
        update();
    }
    void addInfo(IndexInfo const& info) {
        InfoToIndices.emplace(info, 0);
        update();
    }
    bool checkIndex(ParticleIndex in) const { return in < InfoToIndices.size(); }
    ParticleIndex getIndex(IndexInfo const& info) const;
    ParticleIndex getIndex(std::string const& label, unsigned short orbital, spin s) const {
        return getIndex(IndexInfo{label, orbital, s});
    }
    IndexInfo const& getInfo(ParticleIndex in) const;
    ParticleIndex getIndexSize() const { return (ParticleIndex)InfoToIndices.size(); }

private:
    void update();
    std::map<IndexInfo, ParticleIndex> InfoToIndices;
    std::vector<IndexInfo> IndicesToInfo;
};

template <typename Sc> IndexClassification MakeIndexClassification(Operators::expression<Sc> const& H) {
    return IndexClassification(H);
}

// Fock-space action of a monomial: (dagger, mode) pairs in operator order.
struct FockMonomial {
    std::vector<std::pair<bool, int>> ops;
    // |out> = sign * M |s>; false if M|s> = 0.
    bool apply(QuantumState s, QuantumState& out, double& sign) const;
};

// ------------------------------------------------------------ Hilbert space
class HilbertSpace : public ComputableObject {
public:
    template <typename Sc>
    HilbertSpace(IndexClassification const& IndexInfo, Operators::expression<Sc> const& H)
        : IndexInfo(IndexInfo), Complex(H.is_complex()) {
        for (auto const& kv : H.terms) HTerms.emplace_back(toFock(kv.first), std::complex<double>(kv.second));
    }
    // Two-phase partition (HilbertSpace.hpp:144-169).
    void compute();

    IndexClassification const& getIndexInfo() const { return IndexInfo; }
    QuantumState getDim() const { return QuantumState(1) << IndexInfo.getIndexSize(); }
    bool isComplex() const { return Complex; }
    FockMonomial toFock(Monomial const& m) const;
    std::vector<std::pair<FockMonomial, std::complex<double>>> const& getHTerms() const { return HTerms; }
    // block id of every Fock state (after compute())
    std::vector<BlockNumber> const& getBlockOf() const;
    BlockNumber getNumberOfBlocks() const { return NBlocks; }

private:
    IndexClassification const& IndexInfo;
    bool Complex;
    std::vector<std::pair<FockMonomial, std::complex<double>>> HTerms;
    std::vector<BlockNumber> BlockOf;
    BlockNumber NBlocks = 0;
};

template <typename Sc> HilbertSpace MakeHilbertSpace(IndexClassification const& IndexInfo, Operators::expression<Sc> const& H) {
    return HilbertSpace(IndexInfo, H);
}

// ------------------------------------------------------ states classification
class StatesClassification : public ComputableObject {
public:
    void compute(HilbertSpace const& HS);
    QuantumState getNumberOfStates() const { return StateBlockIndex.size(); }
    BlockNumber getNumberOfBlocks() const { return (BlockNumber)StatesContainer.size(); }
    InnerQuantumState getBlockSize(BlockNumber in) const;
    std::vector<QuantumState> const& getFockStates(BlockNumber in) const;
    QuantumState getFockState(BlockNumber in, InnerQuantumState i) const;
    BlockNumber getBlockNumber(QuantumState in) const;
    InnerQuantumState getInnerState(QuantumState in) const;

private:
    void checkComputed() const;
    std::vector<std::vector<QuantumState>> StatesContainer;
    std::vector<BlockNumber> StateBlockIndex;
    std::vector<InnerQuantumState> InnerIndex;
};

// ---------------------------------------------------------------- Hamiltonian
class Hamiltonian;

class HamiltonianPart {
public:
    HamiltonianPart(Hamiltonian const& H, BlockNumber Block) : H(&H), Block(Block) {}
    BlockNumber getBlockNumber() const { return Block; }
    InnerQuantumState getSize() const;
    bool isComplex() const;
    RealType getEigenValue(InnerQuantumState state) const;
    std::vector<RealType> const& getEigenValues() const;
    RealType getMinimumEigenvalue() const;
    // Dense block: the Hamiltonian before compute(), eigenvectors (columns) after.
    std::vector<RealType> getMatrix() const;
    std::vector<RealType> getEigenState(InnerQuantumState state) const;

private:
    Hamiltonian const* H;
    BlockNumber Block;
};

class Hamiltonian : public ComputableObject {
public:
    explicit Hamiltonian(StatesClassification const& S, int device = 0);

    template <typename Sc> void prepare(Operators::expression<Sc> const& HExpr, HilbertSpace const& HS,
                                       MPI_Comm const& comm = MPI_COMM_WORLD) {
        (void)HExpr;
        prepareImpl(HS, comm);
    }
    void compute(MPI_Comm const& comm = MPI_COMM_WORLD);
    // Hamiltonian::reduce / HamiltonianPart::reduce (Hamiltonian.cpp:115-119,
    // HamiltonianPart.cpp:151-172): every block keeps its eigenvalues up to
    // GroundEnergy + Cutoff and the top-left corner of that size of its
    // eigenvector matrix (a block with none left is kept whole).  The
    // accessors show the reduced blocks; quantities computed on the device
    // afterwards still use the full blocks.
    void reduce(RealType Cutoff);

    HamiltonianPart const& getPart(BlockNumber in) const;
    RealType getEigenValue(QuantumState state) const;
    std::vector<RealType> const& getEigenValues(BlockNumber in) const;
    std::vector<RealType> getEigenValues() const;
    RealType getGroundEnergy() const;
    InnerQuantumState getBlockSize(BlockNumber in) const { return S.getBlockSize(in); }
    bool isComplex() const { return Complex; }

    // GPU context shared by every object built on this Hamiltonian.
    Device& device() const { return *Dev; }
    StatesClassification const& getStates() const { return S; }
    std::vector<RealType> const& hostBlocks() const;  // packed blocks, fetched from the device when needed
    std::vector<long> const& matrixOffsets() const { return MOff; }
    std::vector<RealType> const& eigenvectors() const;  // packed, lazily fetched

private:
    void prepareImpl(HilbertSpace const& HS, MPI_Comm const& comm);
    StatesClassification const& S;
    std::shared_ptr<Device> Dev;
    bool Complex = false;
    mutable std::vector<RealType> HPacked;
    std::vector<long> MOff;
    std::vector<std::vector<RealType>> Eigenvalues;
    std::vector<long> Reduced;  // per block: kept eigenvalues after reduce(), 0 if not reduced
    mutable std::vector<RealType> UPacked;
    std::vector<HamiltonianPart> parts;
    RealType GroundEnergy = 0;
    friend class HamiltonianPart;
};

// ------------------------------------------------------------ density matrix
class DensityMatrix;

class DensityMatrixPart {
public:
    DensityMatrixPart(DensityMatrix const& DM, BlockNumber b) : DM(&DM), Block(b) {}
    RealType getWeight(InnerQuantumState s) const;
    RealType getAverageEnergy() const;
    bool isRetained() const;
    RealType beta() const;

private:
    DensityMatrix const* DM;
    BlockNumber Block;
};

class DensityMatrix : public Thermal, public ComputableObject {
public:
    DensityMatrix(StatesClassification const& S, Hamiltonian const& H, RealType beta);
    void prepare();
    void compute();
    RealType getWeight(QuantumState state) const;
    DensityMatrixPart const& getPart(BlockNumber in) const { return parts.at(in); }
    RealType getAverageEnergy() const;
    void truncateBlocks(RealType Tolerance, bool verbose = false);
    bool isRetained(BlockNumber in) const { return Retained.at(in) != 0; }
    // make the device hold this density matrix's weights (and retained flags)
    void bind() const;
    Hamiltonian const& getHamiltonian() const { return H; }
    std::vector<std::vector<RealType>> const& weights() const { return W; }

private:
    StatesClassification const& S;
    Hamiltonian const& H;
    std::vector<DensityMatrixPart> parts;
    std::vector<std::vector<RealType>> W;
    std::vector<int> Retained;
    bool Truncated = false;
    RealType TruncTol = 0;
    friend class DensityMatrixPart;
};

// ---------------------------------------------------------- monomial operators
class MonomialOperator;

class MonomialOperatorPart {
public:
    MonomialOperatorPart(MonomialOperator const& Op, BlockNumber Right, BlockNumber Left)
        : Op(&Op), Right(Right), Left(Left) {}
    BlockNumber getRightIndex() const { return Right; }
    BlockNumber getLeftIndex() const { return Left; }
    bool isComplex() const;
    InnerQuantumState getLeftSize() const;
    InnerQuantumState getRightSize() const;
    // Rotated block <Left| O |Right> (d_left x d_right, row-major, real or
    // interleaved complex), copied from the device.
    std::vector<RealType> getMatrix() const;

private:
    MonomialOperator const* Op;
    BlockNumber Right, Left;
};

class MonomialOperator : public ComputableObject {
public:
    struct BlocksBimap {
        std::map<BlockNumber, BlockNumber> left;   // left -> right
        std::map<BlockNumber, BlockNumber> right;  // right -> left
    };

    template <typename Sc>
    MonomialOperator(Operators::expression<Sc> const& MO, HilbertSpace const& HS, StatesClassification const& S_,
                     Hamiltonian const& H)
        : S(S_), H(H) {
        if (MO.size() != 1) throw std::runtime_error("Only monomial expressions are supported");
        auto const& kv = *MO.terms.begin();
        Mono = HS.toFock(kv.first);
        Coef = std::complex<double>(kv.second);
        if (std::imag(Coef) != 0.0) throw std::runtime_error("complex monomial coefficients are not supported");
    }

    void prepare(HilbertSpace const& HS);
    void compute(RealType Tolerance = 1e-8, MPI_Comm const& comm = MPI_COMM_WORLD);

    bool isComplex() const { return H.isComplex(); }
    MonomialOperatorPart const& getPartFromLeftIndex(BlockNumber LeftIndex) const;
    MonomialOperatorPart const& getPartFromRightIndex(BlockNumber RightIndex) const;
    BlockNumber getLeftIndex(BlockNumber RightIndex) const;
    BlockNumber getRightIndex(BlockNumber LeftIndex) const;
    BlocksBimap const& getBlockMapping() const;

    int deviceId() const { return OpId; }
    int devicePart(BlockNumber Right) const;
    // Fock action per part (right block, left block, inner target per right
    // state or -1, coefficient): the input of pgx_op_define.
    struct Action {
        BlockNumber right, left;
        std::vector<int32_t> target;
        std::vector<double> coef;
    };
    std::vector<Action> fockAction() const;
    Hamiltonian const& getHamiltonian() const { return H; }

protected:
    friend class FieldOperatorContainer;
    void setFromAdjoint(MonomialOperator const& src);
    void checkPrepared() const;

    StatesClassification const& S;
    Hamiltonian const& H;
    FockMonomial Mono;
    std::complex<double> Coef{1.0, 0.0};
    BlocksBimap Map;
    std::vector<MonomialOperatorPart> parts;
    std::unordered_map<BlockNumber, std::size_t> byLeft, byRight;
    int OpId = -1;
    std::unordered_map<BlockNumber, int> DevPartByRight;
};

class FieldOperator : public MonomialOperator {
public:
    template <typename Sc>
    FieldOperator(Operators::expression<Sc> const& FO, HilbertSpace const& HS, StatesClassification const& S_,
                  Hamiltonian const& H, ParticleIndex Index)
        : MonomialOperator(FO, HS, S_, H), Index(Index) {}
    ParticleIndex getIndex() const { return Index; }

private:
    ParticleIndex Index;
};

class CreationOperator : public FieldOperator {
public:
    CreationOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS, StatesClassification const& S,
                     Hamiltonian const& H, ParticleIndex Index);
};

class AnnihilationOperator : public FieldOperator {
public:
    AnnihilationOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS, StatesClassification const& S,
                         Hamiltonian const& H, ParticleIndex Index);
};

class QuadraticOperator : public MonomialOperator {
public:
    QuadraticOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS, StatesClassification const& S,
                      Hamiltonian const& H, ParticleIndex Index1, ParticleIndex Index2,
                      std::tuple<bool, bool> const& Dagger = std::tuple<bool, bool>(true, false));
    ParticleIndex getIndex1() const { return Index1; }
    ParticleIndex getIndex2() const { return Index2; }

private:
    ParticleIndex Index1, Index2;
};

class QuarticOperator : public MonomialOperator {
public:
    QuarticOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS, StatesClassification const& S,
                    Hamiltonian const& H, ParticleIndex Index1, ParticleIndex Index2, ParticleIndex Index3,
                    ParticleIndex Index4,
                    std::tuple<bool, bool, bool, bool> const& Dagger = std::tuple<bool, bool, bool, bool>(true, true,
                                                                                                           false, false));
};

class FieldOperatorContainer {
public:
    FieldOperatorContainer(IndexClassification const& IndexInfo, HilbertSpace const& HS, StatesClassification const& S,
                           Hamiltonian const& H, std::set<ParticleIndex> in = {});
    void prepareAll(HilbertSpace const& HS);
    void computeAll(RealType Tolerance = 1e-8);
    CreationOperator const& getCreationOperator(ParticleIndex in) const;
    AnnihilationOperator const& getAnnihilationOperator(ParticleIndex in) const;

private:
    std::map<ParticleIndex, std::unique_ptr<CreationOperator>> mapCreationOperators;
    std::map<ParticleIndex, std::unique_ptr<AnnihilationOperator>> mapAnnihilationOperators;
};

}  // namespace Pomerol
