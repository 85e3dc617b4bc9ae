// Exact-diagonalisation layer of the drop-in API (host side).
//
// Host work here is bookkeeping only: the Fock action of monomials, the
// invariant-subspace partition (HilbertSpace.hpp:144-169: connected
// components of H, then merges so that every c / c^+ maps a block into at
// most one block) and assembly of the dense block Hamiltonians
// (HamiltonianPart.cpp:56-76), which runs on the GPU (pgx_assemble_hamiltonian)
// from the terms' Fock action.  Eigensolve, weights and operator rotation run
// on the GPU through libpgx.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <unordered_map>

#include "pomerol.hpp"

namespace Pomerol {

// ------------------------------------------------------------ indices
void IndexClassification::update() {
    IndicesToInfo.clear();
    for (auto& kv : InfoToIndices) {
        kv.second = (ParticleIndex)IndicesToInfo.size();
        IndicesToInfo.push_back(kv.first);
    }
}

ParticleIndex IndexClassification::getIndex(IndexInfo const& info) const {
    auto it = InfoToIndices.find(info);
    if (it == InfoToIndices.end()) throw std::runtime_error("Wrong indices (" + std::get<0>(info) + ")");
    return it->second;
}

IndexClassification::IndexInfo const& IndexClassification::getInfo(ParticleIndex in) const {
    if (in >= IndicesToInfo.size()) throw std::runtime_error("Wrong particle index " + std::to_string(in));
    return IndicesToInfo[in];
}

bool FockMonomial::apply(QuantumState s, QuantumState& out, double& sign) const {
    sign = 1.0;
    for (auto it = ops.rbegin(); it != ops.rend(); ++it) {
        const QuantumState mask = QuantumState(1) << it->second;
        const bool occ = (s & mask) != 0;
        if (it->first == occ) return false;  // c^+ on occupied or c on empty
        if (__builtin_popcountll(s & (mask - 1)) & 1) sign = -sign;
        s ^= mask;
    }
    out = s;
    return true;
}

// ------------------------------------------------------------ Hilbert space
FockMonomial HilbertSpace::toFock(Monomial const& m) const {
    FockMonomial f;
    for (auto const& g : m) f.ops.emplace_back(g.dagger, (int)IndexInfo.getIndex(g.index));
    return f;
}

namespace {
struct UnionFind {
    std::vector<int64_t> p;
    explicit UnionFind(std::size_t n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int64_t find(int64_t a) {
        while (p[a] != a) {
            p[a] = p[p[a]];
            a = p[a];
        }
        return a;
    }
    bool unite(int64_t a, int64_t b) {
        a = find(a);
        b = find(b);
        if (a == b) return false;
        if (a < b) std::swap(a, b);
        p[a] = b;
        return true;
    }
};
}  // namespace

void HilbertSpace::compute() {
    if (getStatus() >= Computed) return;
    const QuantumState dim = getDim();
    UnionFind uf(dim);
    // phase I: connected components of H's matrix graph (non-zero elements)
    std::unordered_map<QuantumState, std::complex<double>> row;
    for (QuantumState s = 0; s < dim; ++s) {
        row.clear();
        for (auto const& t : HTerms) {
            QuantumState o;
            double sg;
            if (t.first.apply(s, o, sg)) row[o] += sg * t.second;
        }
        for (auto const& kv : row)
            if (kv.first != s && kv.second != std::complex<double>(0.0)) uf.unite((int64_t)s, (int64_t)kv.first);
    }
    // phase II: every c^+_i (and so c_i) maps a block into at most one block
    const int N = (int)IndexInfo.getIndexSize();
    bool merged = true;
    while (merged) {
        merged = false;
        for (int i = 0; i < N; ++i) {
            std::unordered_map<int64_t, int64_t> fwd, bwd;  // block -> first partner
            const QuantumState mask = QuantumState(1) << i;
            for (QuantumState s = 0; s < dim; ++s) {
                if (s & mask) continue;
                const int64_t a = uf.find((int64_t)s), b = uf.find((int64_t)(s | mask));
                auto f = fwd.emplace(a, b);
                if (!f.second && uf.find(f.first->second) != b) merged |= uf.unite(f.first->second, b);
                auto r = bwd.emplace(b, a);
                if (!r.second && uf.find(r.first->second) != uf.find(a)) merged |= uf.unite(r.first->second, a);
            }
        }
    }
    // blocks numbered by their smallest Fock state
    BlockOf.assign(dim, -1);
    std::unordered_map<int64_t, BlockNumber> id;
    for (QuantumState s = 0; s < dim; ++s) {
        const int64_t r = uf.find((int64_t)s);
        auto it = id.emplace(r, (BlockNumber)id.size()).first;
        BlockOf[s] = it->second;
    }
    NBlocks = (BlockNumber)id.size();
    setStatus(Computed);
}

std::vector<BlockNumber> const& HilbertSpace::getBlockOf() const {
    if (getStatus() < Computed) throw std::runtime_error("Hilbert space partition has not been computed");
    return BlockOf;
}

// ------------------------------------------------------ states classification
void StatesClassification::compute(HilbertSpace const& HS) {
    if (getStatus() == Computed) return;
    const QuantumState dim = HS.getDim();
    StateBlockIndex.assign(dim, 0);
    InnerIndex.assign(dim, 0);
    if (HS.getStatus() == ComputableObject::Computed) {
        auto const& bo = HS.getBlockOf();
        StatesContainer.assign(HS.getNumberOfBlocks(), {});
        for (QuantumState s = 0; s < dim; ++s) {
            StateBlockIndex[s] = bo[s];
            InnerIndex[s] = StatesContainer[bo[s]].size();
            StatesContainer[bo[s]].push_back(s);
        }
    } else {
        StatesContainer.assign(1, {});
        for (QuantumState s = 0; s < dim; ++s) {
            InnerIndex[s] = s;
            StatesContainer[0].push_back(s);
        }
    }
    setStatus(Computed);
}

void StatesClassification::checkComputed() const {
    if (getStatus() < Computed) throw StatusMismatch("StatesClassification is not computed yet.");
}
InnerQuantumState StatesClassification::getBlockSize(BlockNumber in) const {
    return getFockStates(in).size();
}
std::vector<QuantumState> const& StatesClassification::getFockStates(BlockNumber in) const {
    checkComputed();
    if (in < 0 || in >= getNumberOfBlocks()) throw std::runtime_error("Wrong block " + std::to_string(in));
    return StatesContainer[in];
}
QuantumState StatesClassification::getFockState(BlockNumber in, InnerQuantumState m) const {
    auto const& b = getFockStates(in);
    if (m < b.size()) return b[m];
    throw std::runtime_error("Wrong inner state " + std::to_string(m));
}
BlockNumber StatesClassification::getBlockNumber(QuantumState in) const {
    checkComputed();
    if (in >= StateBlockIndex.size()) throw std::runtime_error("Wrong state " + std::to_string(in));
    return StateBlockIndex[in];
}
InnerQuantumState StatesClassification::getInnerState(QuantumState in) const {
    checkComputed();
    if (in >= StateBlockIndex.size()) throw std::runtime_error("Wrong state " + std::to_string(in));
    return InnerIndex[in];
}

// ---------------------------------------------------------------- Hamiltonian
Hamiltonian::Hamiltonian(StatesClassification const& S, int device) : S(S), Dev(std::make_shared<Device>(device)) {}

void Hamiltonian::prepareImpl(HilbertSpace const& HS, MPI_Comm const&) {
    if (getStatus() >= Prepared) return;
    Complex = HS.isComplex();
    const BlockNumber nb = S.getNumberOfBlocks();
    const int sc = Complex ? 2 : 1;
    MOff.assign(nb + 1, 0);
    std::vector<int32_t> dims(nb);
    for (BlockNumber b = 0; b < nb; ++b) {
        dims[b] = (int32_t)S.getBlockSize(b);
        MOff[b + 1] = MOff[b] + (long)dims[b] * dims[b];
    }
    Dev->check(pgx_set_blocks(Dev->ctx(), nb, dims.data(), Complex ? 1 : 0), "pgx_set_blocks");
    auto const& terms = HS.getHTerms();
    const QuantumState dim = HS.getDim();
    int nmodes = 0;
    while ((QuantumState(1) << nmodes) < dim) ++nmodes;
    bool device_assembly = nmodes <= 30 && S.getNumberOfStates() == dim;
    for (auto const& t : terms) device_assembly = device_assembly && t.first.ops.size() <= PGX_TERM_OPS;
    HPacked.clear();
    if (device_assembly) {
        // the GPU builds the dense blocks from the terms' Fock action
        std::vector<int32_t> ops(std::max<std::size_t>(terms.size(), 1) * PGX_TERM_OPS, -1);
        std::vector<double> coef(std::max<std::size_t>(terms.size(), 1) * 2, 0.0);
        for (std::size_t t = 0; t < terms.size(); ++t) {
            auto const& m = terms[t].first.ops;
            for (std::size_t k = 0; k < m.size(); ++k) ops[t * PGX_TERM_OPS + k] = 2 * m[k].second + (m[k].first ? 1 : 0);
            coef[2 * t] = terms[t].second.real();
            coef[2 * t + 1] = terms[t].second.imag();
        }
        std::vector<uint64_t> fock;
        fock.reserve(dim);
        std::vector<int32_t> sb(dim, -1), si(dim, -1);
        for (BlockNumber b = 0; b < nb; ++b) {
            auto const& st = S.getFockStates(b);
            for (std::size_t i = 0; i < st.size(); ++i) {
                fock.push_back(st[i]);
                sb[st[i]] = b;
                si[st[i]] = (int32_t)i;
            }
        }
        Dev->check(pgx_assemble_hamiltonian(Dev->ctx(), (int32_t)terms.size(), ops.data(), coef.data(), nmodes,
                                            fock.data(), sb.data(), si.data()),
                   "pgx_assemble_hamiltonian");
    } else {
        // monomials longer than PGX_TERM_OPS operators: dense blocks built here
        HPacked.assign(MOff[nb] * sc, 0.0);
        for (BlockNumber b = 0; b < nb; ++b) {
            auto const& st = S.getFockStates(b);
            const long d = dims[b];
            double* Hb = HPacked.data() + MOff[b] * sc;
            for (long j = 0; j < d; ++j) {
                for (auto const& t : terms) {
                    QuantumState o;
                    double sg;
                    if (!t.first.apply(st[j], o, sg)) continue;
                    if (S.getBlockNumber(o) != b) throw std::logic_error("Hamiltonian connects different blocks");
                    const long i = (long)S.getInnerState(o);
                    if (Complex) {
                        Hb[2 * (i * d + j)] += sg * t.second.real();
                        Hb[2 * (i * d + j) + 1] += sg * t.second.imag();
                    } else {
                        Hb[i * d + j] += sg * t.second.real();
                    }
                }
            }
        }
        Dev->check(pgx_set_hamiltonian(Dev->ctx(), HPacked.data()), "pgx_set_hamiltonian");
    }
    parts.clear();
    for (BlockNumber b = 0; b < nb; ++b) parts.emplace_back(*this, b);
    setStatus(Prepared);
}

std::vector<RealType> const& Hamiltonian::hostBlocks() const {
    if (getStatus() < Prepared) throw StatusMismatch("Hamiltonian is not prepared yet.");
    if (HPacked.empty()) {
        HPacked.resize(MOff.back() * (Complex ? 2 : 1));
        Dev->check(pgx_get_hamiltonian(Dev->ctx(), HPacked.data()), "pgx_get_hamiltonian");
    }
    return HPacked;
}

void Hamiltonian::compute(MPI_Comm const&) {
    if (getStatus() >= Computed) return;
    if (getStatus() < Prepared) throw StatusMismatch("Hamiltonian is not prepared yet.");
    Dev->check(pgx_eigh(Dev->ctx()), "pgx_eigh");
    const BlockNumber nb = S.getNumberOfBlocks();
    std::vector<double> E(S.getNumberOfStates());
    Dev->check(pgx_get_eigensystem(Dev->ctx(), E.data(), nullptr), "pgx_get_eigensystem");
    Eigenvalues.assign(nb, {});
    long o = 0;
    GroundEnergy = std::numeric_limits<double>::infinity();
    for (BlockNumber b = 0; b < nb; ++b) {
        const long d = (long)S.getBlockSize(b);
        Eigenvalues[b].assign(E.begin() + o, E.begin() + o + d);
        o += d;
        GroundEnergy = std::min(GroundEnergy, *std::min_element(Eigenvalues[b].begin(), Eigenvalues[b].end()));
    }
    UPacked.clear();
    Reduced.assign(nb, 0);
    Dev->weights_beta = -1.0;
    setStatus(Computed);
}

void Hamiltonian::reduce(RealType Cutoff) {
    if (getStatus() < Computed) throw StatusMismatch("Hamiltonian is not computed yet.");
    const RealType level = GroundEnergy + Cutoff;
    for (BlockNumber b = 0; b < (BlockNumber)Eigenvalues.size(); ++b) {
        auto& e = Eigenvalues[b];
        long counter = 0;
        while (counter < (long)e.size() && e[counter] <= level) ++counter;  // ascending
        if (counter > 0) {
            e.resize(counter);
            Reduced[b] = counter;
        }
    }
}

std::vector<RealType> const& Hamiltonian::eigenvectors() const {
    if (getStatus() < Computed) throw StatusMismatch("Hamiltonian is not computed yet.");
    if (UPacked.empty()) {
        UPacked.resize(MOff.back() * (Complex ? 2 : 1));
        Dev->check(pgx_get_eigensystem(Dev->ctx(), nullptr, UPacked.data()), "pgx_get_eigensystem");
    }
    return UPacked;
}

HamiltonianPart const& Hamiltonian::getPart(BlockNumber in) const { return parts.at(in); }
RealType Hamiltonian::getEigenValue(QuantumState state) const {
    return parts.at(S.getBlockNumber(state)).getEigenValue(S.getInnerState(state));
}
std::vector<RealType> const& Hamiltonian::getEigenValues(BlockNumber in) const { return parts.at(in).getEigenValues(); }
std::vector<RealType> Hamiltonian::getEigenValues() const {
    std::vector<RealType> r;
    for (auto const& e : Eigenvalues) r.insert(r.end(), e.begin(), e.end());
    return r;
}
RealType Hamiltonian::getGroundEnergy() const {
    if (getStatus() < Computed) throw StatusMismatch("Hamiltonian is not computed yet.");
    return GroundEnergy;
}

InnerQuantumState HamiltonianPart::getSize() const { return H->S.getBlockSize(Block); }
bool HamiltonianPart::isComplex() const { return H->Complex; }
std::vector<RealType> const& HamiltonianPart::getEigenValues() const {
    if (H->getStatus() < ComputableObject::Computed)
        throw ComputableObject::StatusMismatch("HamiltonianPart is not computed yet.");
    return H->Eigenvalues[Block];
}
RealType HamiltonianPart::getEigenValue(InnerQuantumState s) const { return getEigenValues().at(s); }
RealType HamiltonianPart::getMinimumEigenvalue() const {
    auto const& e = getEigenValues();
    return *std::min_element(e.begin(), e.end());
}
std::vector<RealType> HamiltonianPart::getMatrix() const {
    const int sc = H->Complex ? 2 : 1;
    auto const& src = (H->getStatus() >= ComputableObject::Computed) ? H->eigenvectors() : H->hostBlocks();
    const long r = (H->getStatus() >= ComputableObject::Computed && Block < (BlockNumber)H->Reduced.size())
                       ? H->Reduced[Block]
                       : 0;
    if (r == 0)
        return std::vector<RealType>(src.begin() + H->MOff[Block] * sc, src.begin() + H->MOff[Block + 1] * sc);
    // the reduced block: the top-left r x r corner of the eigenvector matrix
    const long d = (long)getSize();
    std::vector<RealType> m(r * r * sc);
    for (long i = 0; i < r; ++i)
        for (long j = 0; j < r * sc; ++j) m[i * r * sc + j] = src[(H->MOff[Block] + i * d) * sc + j];
    return m;
}
std::vector<RealType> HamiltonianPart::getEigenState(InnerQuantumState state) const {
    const int sc = H->Complex ? 2 : 1;
    auto m = getMatrix();
    const long d = std::lround(std::sqrt((double)(m.size() / sc)));  // the block, or its reduced corner
    std::vector<RealType> v(d * sc);
    for (long i = 0; i < d; ++i)
        for (int c = 0; c < sc; ++c) v[i * sc + c] = m[(i * d + (long)state) * sc + c];
    return v;
}

// ------------------------------------------------------------ density matrix
DensityMatrix::DensityMatrix(StatesClassification const& S, Hamiltonian const& H, RealType beta)
    : Thermal(beta), S(S), H(H) {}

void DensityMatrix::prepare() {
    if (getStatus() >= Prepared) return;
    parts.clear();
    for (BlockNumber b = 0; b < S.getNumberOfBlocks(); ++b) parts.emplace_back(*this, b);
    Retained.assign(S.getNumberOfBlocks(), 1);
    setStatus(Prepared);
}

void DensityMatrix::compute() {
    if (getStatus() >= Computed) return;
    if (getStatus() < Prepared) prepare();
    Device& dev = H.device();
    std::vector<double> w(S.getNumberOfStates());
    double Z = 0;
    dev.check(pgx_weights(dev.ctx(), beta, w.data(), &Z), "pgx_weights");
    dev.weights_beta = beta;
    W.assign(S.getNumberOfBlocks(), {});
    long o = 0;
    for (BlockNumber b = 0; b < S.getNumberOfBlocks(); ++b) {
        const long d = (long)S.getBlockSize(b);
        W[b].assign(w.begin() + o, w.begin() + o + d);
        o += d;
    }
    setStatus(Computed);
}

void DensityMatrix::bind() const {
    if (getStatus() < Computed) throw StatusMismatch("DensityMatrix is not computed yet.");
    Device& dev = H.device();
    if (dev.weights_beta != beta) {
        dev.check(pgx_weights(dev.ctx(), beta, nullptr, nullptr), "pgx_weights");
        dev.weights_beta = beta;
    }
    // device retained flags follow this density matrix
    if (Truncated) dev.check(pgx_truncate_blocks(dev.ctx(), TruncTol, nullptr), "pgx_truncate_blocks");
    else dev.check(pgx_truncate_blocks(dev.ctx(), -1.0, nullptr), "pgx_truncate_blocks");
}

RealType DensityMatrix::getWeight(QuantumState state) const {
    if (getStatus() < Computed) throw StatusMismatch("DensityMatrix is not computed yet.");
    return W[S.getBlockNumber(state)][S.getInnerState(state)];
}

RealType DensityMatrix::getAverageEnergy() const {
    if (getStatus() < Computed) throw StatusMismatch("DensityMatrix is not computed yet.");
    RealType e = 0;
    for (auto const& p : parts) e += p.getAverageEnergy();
    return e;
}

void DensityMatrix::truncateBlocks(RealType Tolerance, bool) {
    if (getStatus() < Computed) throw StatusMismatch("DensityMatrix is not computed yet.");
    Device& dev = H.device();
    if (dev.weights_beta != beta) bind();
    Retained.assign(S.getNumberOfBlocks(), 0);
    dev.check(pgx_truncate_blocks(dev.ctx(), Tolerance, Retained.data()), "pgx_truncate_blocks");
    Truncated = true;
    TruncTol = Tolerance;
}

RealType DensityMatrixPart::getWeight(InnerQuantumState s) const { return DM->W.at(Block).at(s); }
RealType DensityMatrixPart::getAverageEnergy() const {
    auto const& e = DM->H.getEigenValues(Block);
    RealType r = 0;
    for (std::size_t i = 0; i < e.size(); ++i) r += e[i] * DM->W[Block][i];
    return r;
}
bool DensityMatrixPart::isRetained() const { return DM->isRetained(Block); }
RealType DensityMatrixPart::beta() const { return DM->beta; }

// ---------------------------------------------------------- monomial operators
void MonomialOperator::checkPrepared() const {
    if (getStatus() < Prepared) throw StatusMismatch("MonomialOperator is not prepared yet.");
}

void MonomialOperator::prepare(HilbertSpace const& HS) {
    (void)HS;
    if (getStatus() >= Prepared) return;
    parts.clear();
    Map = BlocksBimap();
    byLeft.clear();
    byRight.clear();
    for (BlockNumber R = 0; R < S.getNumberOfBlocks(); ++R) {
        BlockNumber L = INVALID_BLOCK_NUMBER;
        for (QuantumState s : S.getFockStates(R)) {
            QuantumState o;
            double sg;
            if (!Mono.apply(s, o, sg)) continue;
            const BlockNumber b = S.getBlockNumber(o);
            if (L == INVALID_BLOCK_NUMBER) L = b;
            else if (L != b) throw std::logic_error("partition violates the one-block rule for a monomial");
        }
        if (L == INVALID_BLOCK_NUMBER) continue;
        byRight[R] = parts.size();
        byLeft[L] = parts.size();
        Map.right[R] = L;
        Map.left[L] = R;
        parts.emplace_back(*this, R, L);
    }
    setStatus(Prepared);
}

std::vector<MonomialOperator::Action> MonomialOperator::fockAction() const {
    checkPrepared();
    std::vector<Action> out;
    for (auto const& p : parts) {
        Action a{p.getRightIndex(), p.getLeftIndex(), {}, {}};
        for (QuantumState s : S.getFockStates(p.getRightIndex())) {
            QuantumState o;
            double sg;
            if (Mono.apply(s, o, sg)) {
                a.target.push_back((int32_t)S.getInnerState(o));
                a.coef.push_back(sg * Coef.real());
            } else {
                a.target.push_back(-1);
                a.coef.push_back(0.0);
            }
        }
        out.push_back(std::move(a));
    }
    return out;
}

void MonomialOperator::compute(RealType, MPI_Comm const&) {
    checkPrepared();
    if (getStatus() >= Computed) return;
    Device& dev = H.device();
    std::vector<int32_t> rb, lb, tg;
    std::vector<double> cf;
    for (auto const& a : fockAction()) {
        rb.push_back(a.right);
        lb.push_back(a.left);
        tg.insert(tg.end(), a.target.begin(), a.target.end());
        cf.insert(cf.end(), a.coef.begin(), a.coef.end());
    }
    int32_t id = -1;
    dev.check(pgx_op_define(dev.ctx(), (int32_t)parts.size(), rb.data(), lb.data(), tg.data(), cf.data(), &id),
              "pgx_op_define");
    dev.check(pgx_op_rotate(dev.ctx(), id), "pgx_op_rotate");
    OpId = id;
    DevPartByRight.clear();
    for (std::size_t q = 0; q < parts.size(); ++q) DevPartByRight[parts[q].getRightIndex()] = (int)q;
    setStatus(Computed);
}

void MonomialOperator::setFromAdjoint(MonomialOperator const& src) {
    checkPrepared();
    if (getStatus() >= Computed) return;
    Device& dev = H.device();
    int32_t id = -1;
    dev.check(pgx_op_adjoint(dev.ctx(), src.OpId, &id), "pgx_op_adjoint");
    int32_t n = 0;
    dev.check(pgx_op_info(dev.ctx(), id, &n, nullptr, nullptr), "pgx_op_info");
    std::vector<int32_t> r(std::max(n, 1)), l(std::max(n, 1));
    dev.check(pgx_op_info(dev.ctx(), id, &n, r.data(), l.data()), "pgx_op_info");
    DevPartByRight.clear();
    for (int q = 0; q < n; ++q) {
        auto it = Map.right.find(r[q]);
        if (it == Map.right.end() || it->second != l[q])
            throw std::logic_error("adjoint block map disagrees with the prepared operator");
        DevPartByRight[r[q]] = q;
    }
    if ((std::size_t)n != parts.size()) throw std::logic_error("adjoint has a different number of parts");
    OpId = id;
    setStatus(Computed);
}

int MonomialOperator::devicePart(BlockNumber Right) const {
    auto it = DevPartByRight.find(Right);
    if (it == DevPartByRight.end()) throw std::runtime_error("operator has no part with this right block");
    return it->second;
}

MonomialOperatorPart const& MonomialOperator::getPartFromLeftIndex(BlockNumber LeftIndex) const {
    checkPrepared();
    return parts.at(byLeft.at(LeftIndex));
}
MonomialOperatorPart const& MonomialOperator::getPartFromRightIndex(BlockNumber RightIndex) const {
    checkPrepared();
    return parts.at(byRight.at(RightIndex));
}
BlockNumber MonomialOperator::getLeftIndex(BlockNumber RightIndex) const {
    checkPrepared();
    auto it = Map.right.find(RightIndex);
    return it == Map.right.end() ? INVALID_BLOCK_NUMBER : it->second;
}
BlockNumber MonomialOperator::getRightIndex(BlockNumber LeftIndex) const {
    checkPrepared();
    auto it = Map.left.find(LeftIndex);
    return it == Map.left.end() ? INVALID_BLOCK_NUMBER : it->second;
}
MonomialOperator::BlocksBimap const& MonomialOperator::getBlockMapping() const {
    checkPrepared();
    return Map;
}

bool MonomialOperatorPart::isComplex() const { return Op->isComplex(); }
InnerQuantumState MonomialOperatorPart::getLeftSize() const { return Op->getHamiltonian().getStates().getBlockSize(Left); }
InnerQuantumState MonomialOperatorPart::getRightSize() const {
    return Op->getHamiltonian().getStates().getBlockSize(Right);
}
std::vector<RealType> MonomialOperatorPart::getMatrix() const {
    if (Op->getStatus() < ComputableObject::Computed)
        throw ComputableObject::StatusMismatch("MonomialOperatorPart is not computed yet.");
    Hamiltonian const& H = Op->getHamiltonian();
    StatesClassification const& S = H.getStates();
    const long n = (long)S.getBlockSize(Left) * (long)S.getBlockSize(Right) * (isComplex() ? 2 : 1);
    std::vector<RealType> out(n);
    H.device().check(pgx_op_read(H.device().ctx(), Op->deviceId(), Op->devicePart(Right), out.data()), "pgx_op_read");
    return out;
}

static RealExpr single(bool dagger, IndexClassification const& ii, ParticleIndex p) {
    auto const& t = ii.getInfo(p);
    return dagger ? Operators::c_dag<double>(std::get<0>(t), std::get<1>(t), std::get<2>(t))
                  : Operators::c<double>(std::get<0>(t), std::get<1>(t), std::get<2>(t));
}

CreationOperator::CreationOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS,
                                   StatesClassification const& S, Hamiltonian const& H, ParticleIndex Index)
    : FieldOperator(single(true, IndexInfo, Index), HS, S, H, Index) {}

AnnihilationOperator::AnnihilationOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS,
                                           StatesClassification const& S, Hamiltonian const& H, ParticleIndex Index)
    : FieldOperator(single(false, IndexInfo, Index), HS, S, H, Index) {}

QuadraticOperator::QuadraticOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS,
                                     StatesClassification const& S, Hamiltonian const& H, ParticleIndex Index1,
                                     ParticleIndex Index2, std::tuple<bool, bool> const& Dagger)
    : MonomialOperator(single(std::get<0>(Dagger), IndexInfo, Index1) * single(std::get<1>(Dagger), IndexInfo, Index2),
                       HS, S, H),
      Index1(Index1),
      Index2(Index2) {}

QuarticOperator::QuarticOperator(IndexClassification const& IndexInfo, HilbertSpace const& HS,
                                 StatesClassification const& S, Hamiltonian const& H, ParticleIndex Index1,
                                 ParticleIndex Index2, ParticleIndex Index3, ParticleIndex Index4,
                                 std::tuple<bool, bool, bool, bool> const& Dagger)
    : MonomialOperator(single(std::get<0>(Dagger), IndexInfo, Index1) * single(std::get<1>(Dagger), IndexInfo, Index2) *
                           single(std::get<2>(Dagger), IndexInfo, Index3) *
                           single(std::get<3>(Dagger), IndexInfo, Index4),
                       HS, S, H) {}

FieldOperatorContainer::FieldOperatorContainer(IndexClassification const& IndexInfo, HilbertSpace const& HS,
                                               StatesClassification const& S, Hamiltonian const& H,
                                               std::set<ParticleIndex> in) {
    if (in.empty())
        for (ParticleIndex i = 0; i < IndexInfo.getIndexSize(); ++i) in.insert(i);
    for (ParticleIndex i : in) {
        mapCreationOperators.emplace(i, std::make_unique<CreationOperator>(IndexInfo, HS, S, H, i));
        mapAnnihilationOperators.emplace(i, std::make_unique<AnnihilationOperator>(IndexInfo, HS, S, H, i));
    }
}

void FieldOperatorContainer::prepareAll(HilbertSpace const& HS) {
    for (auto& kv : mapCreationOperators) kv.second->prepare(HS);
    for (auto& kv : mapAnnihilationOperators) kv.second->prepare(HS);
}

void FieldOperatorContainer::computeAll(RealType Tolerance) {
    for (auto& kv : mapCreationOperators) {
        kv.second->compute(Tolerance);
        mapAnnihilationOperators.at(kv.first)->setFromAdjoint(*kv.second);
    }
}

CreationOperator const& FieldOperatorContainer::getCreationOperator(ParticleIndex in) const {
    auto it = mapCreationOperators.find(in);
    if (it == mapCreationOperators.end()) throw std::runtime_error("Creation operator not found.");
    return *it->second;
}
AnnihilationOperator const& FieldOperatorContainer::getAnnihilationOperator(ParticleIndex in) const {
    auto it = mapAnnihilationOperators.find(in);
    if (it == mapAnnihilationOperators.end()) throw std::runtime_error("Annihilation operator not found.");
    return *it->second;
}

}  // namespace Pomerol
