// Correlators of the drop-in API: part selection on the host (as in
// GreensFunction.cpp:41-86, Susceptibility.cpp:42-92, TwoParticleGF.cpp:67-120,
// IndexContainer4.hpp:190-273), evaluation on the GPU through libpgx.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "pomerol.hpp"

namespace Pomerol {

namespace {

// Matsubara window cached per device call for single-index queries.
constexpr long GF_WINDOW = 512;

void pair_blocks(MonomialOperator const& F1, MonomialOperator const& F2, DensityMatrix const& DM, std::vector<int>& outer,
                 std::vector<int>& inner) {
    outer.clear();
    inner.clear();
    auto const& m1 = F1.getBlockMapping().left;   // left -> right
    auto const& m2 = F2.getBlockMapping().right;  // right -> left
    for (auto const& kv : m1) {
        const BlockNumber o = kv.first, i = kv.second;
        auto it = m2.find(o);
        if (it == m2.end() || it->second != i) continue;
        if (!(DM.isRetained(o) || DM.isRetained(i))) continue;
        outer.push_back(o);
        inner.push_back(i);
    }
}

}  // namespace

// ------------------------------------------------------------ GreensFunction
GreensFunction::GreensFunction(StatesClassification const& S, Hamiltonian const& H, FieldOperator const& F1,
                               FieldOperator const& F2, DensityMatrix const& DM)
    : Thermal(DM.beta), S(S), H(H), F1(F1), F2(F2), DM(DM) {}

void GreensFunction::prepare() {
    if (getStatus() >= Prepared) return;
    pair_blocks(F1, F2, DM, Outer, Inner);
    Vanishing = Outer.empty();
    setStatus(Prepared);
}

void GreensFunction::compute() {
    if (getStatus() >= Computed) return;
    if (getStatus() < Prepared) prepare();
    if (F1.getStatus() < Computed || F2.getStatus() < Computed)
        throw StatusMismatch("GreensFunction: operators are not computed");
    Cache.clear();
    setStatus(Computed);
}

ParticleIndex GreensFunction::getIndex(std::size_t Position) const {
    if (Position == 0) return F1.getIndex();
    if (Position == 1) return F2.getIndex();
    throw std::runtime_error("GreensFunction: Could not get operator index");
}

std::vector<ComplexType> GreensFunction::values(std::vector<ComplexType> const& z) const {
    std::vector<ComplexType> out(z.size(), 0.0);
    if (Vanishing || z.empty()) return out;
    if (getStatus() < Computed) throw StatusMismatch("GreensFunction is not computed yet.");
    DM.bind();
    Device& dev = H.device();
    dev.check(pgx_gf(dev.ctx(), F1.deviceId(), F2.deviceId(), (int32_t)Outer.size(), Outer.data(), Inner.data(),
                     (int32_t)z.size(), reinterpret_cast<double const*>(z.data()), CoefficientTolerance,
                     reinterpret_cast<double*>(out.data())),
              "pgx_gf");
    return out;
}

ComplexType GreensFunction::operator()(ComplexType z) const { return values({z})[0]; }

ComplexType GreensFunction::operator()(long n) const {
    if (Vanishing) return 0.0;
    auto it = Cache.find(n);
    if (it != Cache.end()) return it->second;
    std::vector<ComplexType> z;
    for (long k = n - GF_WINDOW / 2; k < n + GF_WINDOW / 2; ++k) z.push_back(MatsubaraSpacing * RealType(2 * k + 1));
    auto v = values(z);
    for (long k = 0; k < (long)z.size(); ++k) Cache[n - GF_WINDOW / 2 + k] = v[k];
    return Cache[n];
}

// ------------------------------------------------------------ GFContainer
GFContainer::GFContainer(IndexClassification const& IndexInfo, StatesClassification const& S, Hamiltonian const& H,
                         DensityMatrix const& DM, FieldOperatorContainer const& Ops, bool Anomalous)
    : Thermal(DM.beta), NumIndices(IndexInfo.getIndexSize()), S(S), H(H), DM(DM), Operators(Ops), Anomalous(Anomalous) {}

std::shared_ptr<GreensFunction> GFContainer::createElement(IndexCombination2 const& I) const {
    if (Anomalous)
        return std::make_shared<GreensFunction>(S, H, Operators.getAnnihilationOperator(I.Index1),
                                                Operators.getAnnihilationOperator(I.Index2), DM);
    return std::make_shared<GreensFunction>(S, H, Operators.getAnnihilationOperator(I.Index1),
                                            Operators.getCreationOperator(I.Index2), DM);
}

void GFContainer::prepareAll(std::set<IndexCombination2> const& Indices) {
    ElementsMap.clear();
    std::set<IndexCombination2> II = Indices;
    if (II.empty())
        for (ParticleIndex i = 0; i < NumIndices; ++i)
            for (ParticleIndex j = 0; j < NumIndices; ++j) II.emplace(i, j);
    for (auto const& ic : II) ElementsMap[ic] = createElement(ic);
    for (auto& kv : ElementsMap) {
        kv.second->PoleResolution = PoleResolution;
        kv.second->CoefficientTolerance = CoefficientTolerance;
        kv.second->prepare();
    }
}

void GFContainer::computeAll() {
    for (auto& kv : ElementsMap) kv.second->compute();
}

GreensFunction& GFContainer::operator()(IndexCombination2 const& I) {
    auto it = ElementsMap.find(I);
    if (it != ElementsMap.end()) return *it->second;
    auto e = createElement(I);
    e->PoleResolution = PoleResolution;
    e->CoefficientTolerance = CoefficientTolerance;
    e->prepare();
    e->compute();
    ElementsMap[I] = e;
    return *e;
}

// ------------------------------------------------------------ EnsembleAverage
EnsembleAverage::EnsembleAverage(MonomialOperator const& A, DensityMatrix const& DM)
    : Thermal(DM.beta), A(A), DM(DM) {}

void EnsembleAverage::compute() {
    if (getStatus() >= Prepared) return;
    DM.bind();
    Device& dev = A.getHamiltonian().device();
    double r[2] = {0, 0};
    dev.check(pgx_ensemble_average(dev.ctx(), A.deviceId(), r), "pgx_ensemble_average");
    Result = ComplexType(r[0], r[1]);
    setStatus(Prepared);
}

// ------------------------------------------------------------ Susceptibility
Susceptibility::Susceptibility(StatesClassification const& S, Hamiltonian const& H, MonomialOperator const& A,
                               MonomialOperator const& B, DensityMatrix const& DM)
    : Thermal(DM.beta), S(S), H(H), A(A), B(B), DM(DM) {}

void Susceptibility::prepare() {
    if (getStatus() >= Prepared) return;
    pair_blocks(A, B, DM, Outer, Inner);
    Vanishing = Outer.empty();
    setStatus(Prepared);
}

void Susceptibility::compute() {
    if (getStatus() >= Computed) return;
    if (getStatus() < Prepared) prepare();
    Cache.clear();
    setStatus(Computed);
}

void Susceptibility::subtractDisconnected() {
    EnsembleAverage a(A, DM), b(B, DM);
    subtractDisconnected(a, b);
}
void Susceptibility::subtractDisconnected(ComplexType a, ComplexType b) {
    SubtractDisconnected = true;
    ave_A = a;
    ave_B = b;
    Cache.clear();
}
void Susceptibility::subtractDisconnected(EnsembleAverage& a, EnsembleAverage& b) {
    a.compute();
    b.compute();
    subtractDisconnected(a(), b());
}

std::vector<ComplexType> Susceptibility::values(std::vector<ComplexType> const& z) const {
    std::vector<ComplexType> out(z.size(), 0.0);
    if (z.empty()) return out;
    if (!Vanishing) {
        if (getStatus() < Computed) throw StatusMismatch("Susceptibility is not computed yet.");
        DM.bind();
        Device& dev = H.device();
        dev.check(pgx_susc(dev.ctx(), A.deviceId(), B.deviceId(), (int32_t)Outer.size(), Outer.data(), Inner.data(),
                           (int32_t)z.size(), reinterpret_cast<double const*>(z.data()), PoleResolution,
                           CoefficientTolerance, beta, reinterpret_cast<double*>(out.data()), nullptr),
                  "pgx_susc");
    }
    if (SubtractDisconnected)
        for (std::size_t k = 0; k < z.size(); ++k)
            if (std::abs(z[k]) <= DBL_EPSILON) out[k] -= ave_A * ave_B * beta;
    return out;
}

ComplexType Susceptibility::operator()(ComplexType z) const { return values({z})[0]; }

ComplexType Susceptibility::operator()(long m) const {
    auto it = Cache.find(m);
    if (it != Cache.end()) return it->second;
    std::vector<ComplexType> z;
    for (long k = m - GF_WINDOW / 2; k < m + GF_WINDOW / 2; ++k) z.push_back(MatsubaraSpacing * RealType(2 * k));
    auto v = values(z);
    for (long k = 0; k < (long)z.size(); ++k) Cache[m - GF_WINDOW / 2 + k] = v[k];
    return Cache[m];
}

// ------------------------------------------------------------ TwoParticleGF
TwoParticleGF::TwoParticleGF(StatesClassification const& S, Hamiltonian const& H, AnnihilationOperator const& C1,
                             AnnihilationOperator const& C2, CreationOperator const& CX3, CreationOperator const& CX4,
                             DensityMatrix const& DM)
    : Thermal(DM.beta), S(S), H(H), C1(C1), C2(C2), CX3(CX3), CX4(CX4), DM(DM) {}

void TwoParticleGF::prepare() {
    if (getStatus() >= Prepared) return;
    MonomialOperator const* ops[3] = {&C1, &C2, &CX3};
    Parts.clear();
    PartOps.clear();
    for (auto const& kv : CX4.getBlockMapping().right) {  // right block S1 -> left block S4, ascending
        for (std::size_t p = 0; p < 6; ++p) {
            auto const& perm = permutations3[p].perm;
            const BlockNumber b0 = kv.first, b3 = kv.second;
            const BlockNumber b2 = ops[perm[2]]->getLeftIndex(b3);
            const BlockNumber b1 = ops[perm[0]]->getRightIndex(b0);
            if (b1 == INVALID_BLOCK_NUMBER || b2 == INVALID_BLOCK_NUMBER) continue;
            if (ops[perm[1]]->getRightIndex(b1) != b2) continue;
            if (!(DM.isRetained(b0) || DM.isRetained(b1) || DM.isRetained(b2) || DM.isRetained(b3))) continue;
            pgx_g2_part g{};
            g.op[0] = ops[perm[0]]->deviceId();
            g.op[1] = ops[perm[1]]->deviceId();
            g.op[2] = ops[perm[2]]->deviceId();
            g.op[3] = CX4.deviceId();
            g.block[0] = b0;
            g.block[1] = b1;
            g.block[2] = b2;
            g.block[3] = b3;
            for (int k = 0; k < 3; ++k) g.perm[k] = (int32_t)perm[k];
            g.sign = permutations3[p].sign;
            Parts.push_back(g);
            PartOps.push_back({ops[perm[0]], ops[perm[1]], ops[perm[2]], &CX4});
        }
    }
    Vanishing = Parts.empty();
    setStatus(Prepared);
}

std::vector<ComplexType> TwoParticleGF::values(FreqVec3 const& freqs) const {
    std::vector<ComplexType> out(freqs.size(), 0.0);
    if (Vanishing || freqs.empty()) return out;
    // device operator ids are resolved at evaluation time (operators may be
    // computed after prepare())
    std::vector<pgx_g2_part> parts = Parts;
    for (std::size_t q = 0; q < parts.size(); ++q)
        for (int k = 0; k < 4; ++k) {
            parts[q].op[k] = PartOps[q][k]->deviceId();
            if (parts[q].op[k] < 0) throw StatusMismatch("TwoParticleGF: operators are not computed");
        }
    std::vector<double> z(6 * freqs.size());
    for (std::size_t t = 0; t < freqs.size(); ++t) {
        ComplexType a = std::get<0>(freqs[t]), b = std::get<1>(freqs[t]), c = std::get<2>(freqs[t]);
        z[6 * t] = a.real();
        z[6 * t + 1] = a.imag();
        z[6 * t + 2] = b.real();
        z[6 * t + 3] = b.imag();
        z[6 * t + 4] = c.real();
        z[6 * t + 5] = c.imag();
    }
    DM.bind();
    Device& dev = H.device();
    // anchored sum: sub-terms whose Boltzmann weight is below the anchor
    // threshold are skipped (the same order as the coefficient filter);
    // ExactSum evaluates every state quadruple.
    const double anchor = AnchorTolerance < 0 ? CoefficientTolerance : AnchorTolerance;
    if (SplitProducts && !ExactSum) dev.check(pgx_set_g2_split_slices(dev.ctx(), SplitSlices), "pgx_set_g2_split_slices");
    dev.check(pgx_g2(dev.ctx(), (int32_t)parts.size(), parts.data(), (int32_t)freqs.size(), z.data(), PoleResolution,
                     ExactSum ? 0.0 : anchor,
                     ExactSum ? PGX_G2_EXACT : (PGX_G2_ANCHORED | (SplitProducts ? PGX_G2_SPLIT_I8 : 0)),
                     reinterpret_cast<double*>(out.data())),
              "pgx_g2");
    return out;
}

std::vector<ComplexType> TwoParticleGF::compute(bool clear, FreqVec3 const& freqs, MPI_Comm const&) {
    (void)clear;
    if (getStatus() < Prepared) throw StatusMismatch("TwoParticleGF is not prepared yet.");
    std::vector<ComplexType> m_data;
    if (getStatus() >= Computed) return m_data;
    if (!Vanishing) {
        m_data.assign(freqs.size(), 0.0);
        if (!freqs.empty()) m_data = values(freqs);
    }
    Cache.clear();
    setStatus(Computed);
    return m_data;
}

ParticleIndex TwoParticleGF::getIndex(std::size_t Position) const {
    switch (Position) {
        case 0: return C1.getIndex();
        case 1: return C2.getIndex();
        case 2: return CX3.getIndex();
        case 3: return CX4.getIndex();
        default: throw std::runtime_error("TwoParticleGF: Could not get operator index");
    }
}

ComplexType TwoParticleGF::operator()(ComplexType z1, ComplexType z2, ComplexType z3) const {
    if (Vanishing) return 0.0;
    return values({FreqTuple3{z1, z2, z3}})[0];
}

ComplexType TwoParticleGF::operator()(long n1, long n2, long n3) const {
    if (Vanishing) return 0.0;
    auto key = std::make_tuple(n1, n2, n3);
    auto it = Cache.find(key);
    if (it != Cache.end()) return it->second;
    // fill the cube [-W, W)^3 that contains the point with one device call
    long W = std::max({std::labs(n1) + 1, std::labs(n2) + 1, std::labs(n3) + 1, 8L});
    W = (W + 3) / 4 * 4;
    if (W > 24) return (*this)(MatsubaraSpacing * RealType(2 * n1 + 1), MatsubaraSpacing * RealType(2 * n2 + 1),
                               MatsubaraSpacing * RealType(2 * n3 + 1));
    FreqVec3 f;
    std::vector<std::tuple<long, long, long>> keys;
    for (long a = -W; a < W; ++a)
        for (long b = -W; b < W; ++b)
            for (long c = -W; c < W; ++c) {
                f.emplace_back(MatsubaraSpacing * RealType(2 * a + 1), MatsubaraSpacing * RealType(2 * b + 1),
                               MatsubaraSpacing * RealType(2 * c + 1));
                keys.emplace_back(a, b, c);
            }
    auto v = values(f);
    for (std::size_t k = 0; k < keys.size(); ++k) Cache[keys[k]] = v[k];
    return Cache[key];
}

// ------------------------------------------------------------ container
TwoParticleGFContainer::TwoParticleGFContainer(IndexClassification const& IndexInfo, StatesClassification const& S,
                                               Hamiltonian const& H, DensityMatrix const& DM,
                                               FieldOperatorContainer const& Ops)
    : Thermal(DM.beta), NumIndices(IndexInfo.getIndexSize()), S(S), H(H), DM(DM), Operators(Ops) {}

ElementWithPermFreq<TwoParticleGF>& TwoParticleGFContainer::create(IndexCombination4 const& I) {
    auto e = std::make_shared<TwoParticleGF>(S, H, Operators.getAnnihilationOperator(I.Index1),
                                             Operators.getAnnihilationOperator(I.Index2),
                                             Operators.getCreationOperator(I.Index3),
                                             Operators.getCreationOperator(I.Index4), DM);
    auto it = ElementsMap.emplace(I, ElementWithPermFreq<TwoParticleGF>{e, permutations4[0]}).first;
    NonTrivialElements.emplace(I, e);
    const bool sameC = I.Index1 == I.Index2, sameCX = I.Index3 == I.Index4;
    if (!sameC) ElementsMap.emplace(IndexCombination4(I.Index2, I.Index1, I.Index3, I.Index4),
                                    ElementWithPermFreq<TwoParticleGF>{e, permutations4[6]});
    if (!sameCX) ElementsMap.emplace(IndexCombination4(I.Index1, I.Index2, I.Index4, I.Index3),
                                     ElementWithPermFreq<TwoParticleGF>{e, permutations4[1]});
    if (!sameC && !sameCX)
        ElementsMap.emplace(IndexCombination4(I.Index2, I.Index1, I.Index4, I.Index3),
                            ElementWithPermFreq<TwoParticleGF>{e, permutations4[7]});
    return it->second;
}

void TwoParticleGFContainer::prepareAll(std::set<IndexCombination4> const& Indices) {
    ElementsMap.clear();
    NonTrivialElements.clear();
    std::set<IndexCombination4> II = Indices;
    if (II.empty())
        for (ParticleIndex i = 0; i < NumIndices; ++i)
            for (ParticleIndex j = i; j < NumIndices; ++j)
                for (ParticleIndex k = 0; k < NumIndices; ++k)
                    for (ParticleIndex l = k; l < NumIndices; ++l) II.emplace(i, j, k, l);
    for (auto const& ic : II)
        if (!isInContainer(ic)) create(ic);
    for (auto& kv : ElementsMap) {
        TwoParticleGF& g = kv.second.element();
        g.PoleResolution = PoleResolution;
        g.CoefficientTolerance = CoefficientTolerance;
        g.SplitProducts = SplitProducts;
        g.AnchorTolerance = AnchorTolerance;
        g.SplitSlices = SplitSlices;
        g.prepare();
    }
}

std::map<IndexCombination4, std::vector<ComplexType>> TwoParticleGFContainer::computeAll(bool clearTerms,
                                                                                         FreqVec3 const& freqs,
                                                                                         MPI_Comm const& comm,
                                                                                         bool split) {
    std::map<IndexCombination4, std::vector<ComplexType>> out;
    for (auto& kv : NonTrivialElements) {
        kv.second->SplitProducts = SplitProducts;
        kv.second->AnchorTolerance = AnchorTolerance;
        kv.second->SplitSlices = SplitSlices;
    }
    if (split) {
        for (auto& kv : NonTrivialElements) out[kv.first] = kv.second->compute(clearTerms, freqs, comm);
    } else {
        for (auto& kv : ElementsMap) out.emplace(kv.first, kv.second.element().compute(clearTerms, freqs, comm));
    }
    return out;
}

ElementWithPermFreq<TwoParticleGF>& TwoParticleGFContainer::operator()(IndexCombination4 const& I) {
    auto it = ElementsMap.find(I);
    if (it != ElementsMap.end()) return it->second;
    auto& e = create(I);
    e.element().PoleResolution = PoleResolution;
    e.element().CoefficientTolerance = CoefficientTolerance;
    e.element().SplitProducts = SplitProducts;
    e.element().AnchorTolerance = AnchorTolerance;
    e.element().SplitSlices = SplitSlices;
    e.element().prepare();
    return e;
}

// ------------------------------------------------------------ Vertex4
Vertex4::Vertex4(TwoParticleGF const& Chi, GreensFunction const& G13, GreensFunction const& G24,
                 GreensFunction const& G14, GreensFunction const& G23)
    : Thermal(Chi.beta), Chi(Chi), G13(G13), G24(G24), G14(G14), G23(G23) {}

ComplexType Vertex4::disconnected(long n1, long n2, long n3) const {
    ComplexType v = 0.0;
    if (n1 == n3) v += beta * G13(n1) * G24(n2);
    if (n2 == n3) v -= beta * G14(n1) * G23(n2);
    return v;
}

ComplexType Vertex4::value(long n1, long n2, long n3) const { return Chi(n1, n2, n3) + disconnected(n1, n2, n3); }

void Vertex4::compute(long N) {
    if (getStatus() >= Computed) return;
    NumberOfMatsubaras = N;
    Values.assign(N > 0 ? 4 * N - 1 : 0, {});
    Offset.assign(Values.size(), 0);
    Size.assign(Values.size(), 0);
    FreqVec3 freqs;
    std::vector<std::tuple<long, long, long>> idx;
    for (long bv = 0; bv < (long)Values.size(); ++bv) {
        const long Om = bv - 2 * N;
        Size[bv] = 2 * N - std::labs(Om + 1);
        Offset[bv] = (Om < 0 ? 0 : Om + 1) - N;
        for (long a = 0; a < Size[bv]; ++a)
            for (long c = 0; c < Size[bv]; ++c) {
                const long n1 = a + Offset[bv], n2 = Om - n1, n3 = c + Offset[bv];
                idx.emplace_back(n1, n2, n3);
                freqs.emplace_back(MatsubaraSpacing * RealType(2 * n1 + 1), MatsubaraSpacing * RealType(2 * n2 + 1),
                                   MatsubaraSpacing * RealType(2 * n3 + 1));
            }
    }
    const std::vector<ComplexType> chi = Chi.isVanishing() ? std::vector<ComplexType>(freqs.size(), 0.0) : Chi.values(freqs);
    std::size_t q = 0;
    for (long bv = 0; bv < (long)Values.size(); ++bv) {
        Values[bv].resize(Size[bv] * Size[bv]);
        for (long e = 0; e < Size[bv] * Size[bv]; ++e, ++q) {
            const auto& t = idx[q];
            Values[bv][e] = chi[q] + disconnected(std::get<0>(t), std::get<1>(t), std::get<2>(t));
        }
    }
    setStatus(Computed);
}

ComplexType Vertex4::operator()(long n1, long n2, long n3) const {
    const long bv = n1 + n2 + 2 * NumberOfMatsubaras;
    if (NumberOfMatsubaras > 0 && bv >= 0 && bv < (long)Values.size()) {
        const long a = n1 - Offset[bv], c = n3 - Offset[bv];
        if (a >= 0 && a < Size[bv] && c >= 0 && c < Size[bv]) return Values[bv][a * Size[bv] + c];
    }
    return value(n1, n2, n3);  // outside the cached box
}

}  // namespace Pomerol

namespace Pomerol {

// ------------------------------------------------------------ ThreePointSusceptibility
ThreePointSusceptibility::ThreePointSusceptibility(Channel channel, StatesClassification const& S,
                                                   Hamiltonian const& H, CreationOperator const& CX1,
                                                   AnnihilationOperator const& C2, CreationOperator const& CX3,
                                                   AnnihilationOperator const& C4, DensityMatrix const& DM)
    : Thermal(DM.beta), channel(channel), S(S), H(H), CX1(CX1), C2(C2), CX3(CX3), C4(C4), DM(DM) {}

// The operators of each channel (ThreePointSusceptibility.cpp:37-66): F1 = CX1;
// PP: F2 = CX3, B = C2 C4; PH: F2 = C2, B = CX3 C4; xPH: F2 = C4, B = CX3 C2.
MonomialOperator const& ThreePointSusceptibility::getF2() const {
    switch (channel) {
        case PP: return CX3;
        case PH: return C2;
        case xPH: return C4;
    }
    throw std::runtime_error("ThreePointSusceptibility: Wrong channel");
}
MonomialOperator const& ThreePointSusceptibility::getB1() const {
    switch (channel) {
        case PP: return C2;
        case PH: return CX3;
        case xPH: return CX3;
    }
    throw std::runtime_error("ThreePointSusceptibility: Wrong channel");
}
MonomialOperator const& ThreePointSusceptibility::getB2() const {
    switch (channel) {
        case PP: return C4;
        case PH: return C4;
        case xPH: return C2;
    }
    throw std::runtime_error("ThreePointSusceptibility: Wrong channel");
}

void ThreePointSusceptibility::prepare() {
    if (getStatus() >= Prepared) return;
    MonomialOperator const& F1 = CX1;
    MonomialOperator const& F2 = getF2();
    MonomialOperator const& B1 = getB1();
    MonomialOperator const& B2 = getB2();
    Parts.clear();
    PartOps.clear();
    auto add = [&](MonomialOperator const& Fa, MonomialOperator const& Fb, BlockNumber i, BlockNumber j,
                   BlockNumber k, BlockNumber m, bool swapped) {
        pgx_chi3_part p{};
        p.block[0] = i;
        p.block[1] = j;
        p.block[2] = k;
        p.block[3] = m;
        p.swapped = swapped ? 1 : 0;
        Parts.push_back(p);
        PartOps.push_back({&Fa, &Fb, &B1, &B2});
    };
    for (auto const& kv : B2.getBlockMapping().right) {  // right block -> left block, ascending
        const BlockNumber b2right = kv.first, b2left = kv.second;
        const BlockNumber b1left = B1.getLeftIndex(b2left);
        if (b1left == INVALID_BLOCK_NUMBER) continue;
        // <b2right|F1|j><j|F2|b1left><b1left|B1|b2left><b2left|B2|b2right>
        const BlockNumber f1right = F1.getRightIndex(b2right), f2left = F2.getLeftIndex(b1left);
        if (f1right == f2left && f1right != INVALID_BLOCK_NUMBER && DM.isRetained(b2right) &&
            DM.isRetained(f1right) && DM.isRetained(b1left))
            add(F1, F2, b2right, f1right, b1left, b2left, false);
        // <b2right|F2|j><j|F1|b1left><b1left|B1|b2left><b2left|B2|b2right>
        const BlockNumber f2right = F2.getRightIndex(b2right), f1left = F1.getLeftIndex(b1left);
        if (f2right == f1left && f2right != INVALID_BLOCK_NUMBER && DM.isRetained(b2right) &&
            DM.isRetained(f2right) && DM.isRetained(b1left))
            add(F2, F1, b2right, f2right, b1left, b2left, true);
    }
    Vanishing = Parts.empty();
    setStatus(Prepared);
}

std::vector<ComplexType> ThreePointSusceptibility::values(FreqVec2 const& freqs) const {
    std::vector<ComplexType> out(freqs.size(), 0.0);
    if (Vanishing || freqs.empty()) return out;
    std::vector<pgx_chi3_part> parts = Parts;
    for (std::size_t q = 0; q < parts.size(); ++q) {
        int32_t* ids[4] = {&parts[q].f1, &parts[q].f2, &parts[q].b1, &parts[q].b2};
        for (int k = 0; k < 4; ++k) {
            *ids[k] = PartOps[q][k]->deviceId();
            if (*ids[k] < 0) throw StatusMismatch("ThreePointSusceptibility: operators are not computed");
        }
    }
    std::vector<double> z(4 * freqs.size());
    for (std::size_t t = 0; t < freqs.size(); ++t) {
        const ComplexType a = std::get<0>(freqs[t]), b = std::get<1>(freqs[t]);
        z[4 * t] = a.real();
        z[4 * t + 1] = a.imag();
        z[4 * t + 2] = b.real();
        z[4 * t + 3] = b.imag();
    }
    DM.bind();
    Device& dev = H.device();
    dev.check(pgx_chi3(dev.ctx(), (int32_t)channel, (int32_t)parts.size(), parts.data(), (int32_t)freqs.size(),
                       z.data(), PoleResolution, reinterpret_cast<double*>(out.data())),
              "pgx_chi3");
    return out;
}

std::vector<ComplexType> ThreePointSusceptibility::compute(bool clear, FreqVec2 const& freqs, MPI_Comm const&) {
    (void)clear;
    if (getStatus() < Prepared) throw StatusMismatch("ThreePointSusceptibility is not prepared yet.");
    std::vector<ComplexType> m_data;
    if (getStatus() >= Computed) return m_data;
    if (!Vanishing) {
        m_data.assign(freqs.size(), 0.0);
        if (!freqs.empty()) m_data = values(freqs);
    }
    Cache.clear();
    setStatus(Computed);
    return m_data;
}

ParticleIndex ThreePointSusceptibility::getIndex(std::size_t Position) const {
    switch (Position) {
        case 0: return CX1.getIndex();
        case 1: return C2.getIndex();
        case 2: return CX3.getIndex();
        case 3: return C4.getIndex();
        default: throw std::runtime_error("ThreePointSusceptibility: Could not get operator index");
    }
}

ComplexType ThreePointSusceptibility::operator()(ComplexType z1, ComplexType z2) const {
    if (Vanishing) return 0.0;
    return values({FreqTuple2{z1, z2}})[0];
}

ComplexType ThreePointSusceptibility::operator()(long n1, long n2) const {
    if (Vanishing) return 0.0;
    const auto key = std::make_pair(n1, n2);
    auto it = Cache.find(key);
    if (it != Cache.end()) return it->second;
    // fill the square [-W, W)^2 that contains the point with one device call
    long W = std::max({std::labs(n1) + 1, std::labs(n2) + 1, 16L});
    W = (W + 7) / 8 * 8;
    if (W > 128) return (*this)(MatsubaraSpacing * RealType(2 * n1 + 1), MatsubaraSpacing * RealType(2 * n2 + 1));
    FreqVec2 f;
    for (long a = -W; a < W; ++a)
        for (long b = -W; b < W; ++b)
            f.emplace_back(MatsubaraSpacing * RealType(2 * a + 1), MatsubaraSpacing * RealType(2 * b + 1));
    auto v = values(f);
    std::size_t q = 0;
    for (long a = -W; a < W; ++a)
        for (long b = -W; b < W; ++b) Cache[std::make_pair(a, b)] = v[q++];
    return Cache[key];
}

// ------------------------------------------------------------ ThreePointSusceptibilityContainer
ThreePointSusceptibilityContainer::ThreePointSusceptibilityContainer(Channel channel,
                                                                     IndexClassification const& IndexInfo,
                                                                     StatesClassification const& S,
                                                                     Hamiltonian const& H, DensityMatrix const& DM,
                                                                     FieldOperatorContainer const& Ops)
    : Thermal(DM.beta), channel(channel), NumIndices(IndexInfo.getIndexSize()), S(S), H(H), DM(DM), Operators(Ops) {}

// IndexContainer4::create (IndexContainer4.hpp:190-237): the element and its
// aliases under exchange of the first or last two indices
ElementWithPermFreq<ThreePointSusceptibility>& ThreePointSusceptibilityContainer::create(IndexCombination4 const& I) {
    auto e = std::make_shared<ThreePointSusceptibility>(
        channel, S, H, Operators.getCreationOperator(I.Index1), Operators.getAnnihilationOperator(I.Index2),
        Operators.getCreationOperator(I.Index3), Operators.getAnnihilationOperator(I.Index4), DM);
    auto it = ElementsMap.emplace(I, ElementWithPermFreq<ThreePointSusceptibility>{e, permutations4[0]}).first;
    NonTrivialElements.emplace(I, e);
    const bool sameC = I.Index1 == I.Index2, sameCX = I.Index3 == I.Index4;
    if (!sameC)
        ElementsMap.emplace(IndexCombination4(I.Index2, I.Index1, I.Index3, I.Index4),
                            ElementWithPermFreq<ThreePointSusceptibility>{e, permutations4[6]});
    if (!sameCX)
        ElementsMap.emplace(IndexCombination4(I.Index1, I.Index2, I.Index4, I.Index3),
                            ElementWithPermFreq<ThreePointSusceptibility>{e, permutations4[1]});
    if (!sameC && !sameCX)
        ElementsMap.emplace(IndexCombination4(I.Index2, I.Index1, I.Index4, I.Index3),
                            ElementWithPermFreq<ThreePointSusceptibility>{e, permutations4[7]});
    return it->second;
}

void ThreePointSusceptibilityContainer::prepareAll(std::set<IndexCombination4> const& Indices) {
    ElementsMap.clear();
    NonTrivialElements.clear();
    std::set<IndexCombination4> II = Indices;
    if (II.empty())
        for (ParticleIndex i = 0; i < NumIndices; ++i)
            for (ParticleIndex j = i; j < NumIndices; ++j)
                for (ParticleIndex k = 0; k < NumIndices; ++k)
                    for (ParticleIndex l = k; l < NumIndices; ++l) II.emplace(i, j, k, l);
    for (auto const& ic : II)
        if (!isInContainer(ic)) create(ic);
    for (auto& kv : ElementsMap) {
        ThreePointSusceptibility& g = kv.second.element();
        g.PoleResolution = PoleResolution;
        g.CoefficientTolerance = CoefficientTolerance;
        g.prepare();
    }
}

// ThreePointSusceptibilityContainer::computeAll (ThreePointSusceptibilityContainer.cpp:30-40):
// every key of the map in order; an alias of an element computed earlier
// yields an empty vector, as there.
std::map<IndexCombination4, std::vector<ComplexType>> ThreePointSusceptibilityContainer::computeAll(
    bool clearTerms, FreqVec2 const& freqs, MPI_Comm const& comm) {
    std::map<IndexCombination4, std::vector<ComplexType>> out;
    for (auto& kv : ElementsMap) out.emplace(kv.first, kv.second.element().compute(clearTerms, freqs, comm));
    return out;
}

ElementWithPermFreq<ThreePointSusceptibility>& ThreePointSusceptibilityContainer::operator()(
    IndexCombination4 const& I) {
    auto it = ElementsMap.find(I);
    if (it != ElementsMap.end()) return it->second;
    auto& e = create(I);
    e.element().PoleResolution = PoleResolution;
    e.element().CoefficientTolerance = CoefficientTolerance;
    e.element().prepare();
    return e;
}

}  // namespace Pomerol
