// Python bindings of the drop-in host layer (module pomerol_b200._pomerol).
// The classes keep the reference's names and call patterns so that tests
// read like the reference's Catch2 tests.
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/operators.h>
#include <cmath>

#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "pomerol.hpp"

namespace py = pybind11;
using namespace Pomerol;
using C = std::complex<double>;

namespace {

py::array_t<double> as_real(std::vector<double> const& v, long rows, long cols) {
    py::array_t<double> a({rows, cols});
    std::copy(v.begin(), v.end(), a.mutable_data());
    return a;
}

py::object as_matrix(std::vector<double> const& v, long rows, long cols, bool cplx) {
    if (!cplx) return as_real(v, rows, cols);
    py::array_t<C> a({rows, cols});
    std::copy(reinterpret_cast<C const*>(v.data()), reinterpret_cast<C const*>(v.data()) + rows * cols,
              a.mutable_data());
    return a;
}

FreqVec3 to_freqs(std::vector<std::tuple<C, C, C>> const& f) { return FreqVec3(f.begin(), f.end()); }
FreqVec2 to_freqs2(std::vector<std::tuple<C, C>> const& f) { return FreqVec2(f.begin(), f.end()); }

template <typename E> void bind_expr(py::module& m, char const* name) {
    py::class_<E>(m, name)
        .def(py::init<>())
        .def("size", &E::size)
        .def("__len__", &E::size)
        .def("__iadd__", [](E& a, E const& b) { return a += b; })
        .def("__add__", [](E const& a, E const& b) { return E(a) += b; })
        .def("__sub__", [](E const& a, E const& b) { return E(a) -= b; })
        .def("__neg__", [](E const& a) { return E(a) *= typename E::scalar_type(-1); })
        .def("__mul__", [](E const& a, E const& b) { return a * b; })
        .def("__mul__", [](E const& a, typename E::scalar_type s) { return E(a) *= s; })
        .def("__rmul__", [](E const& a, typename E::scalar_type s) { return E(a) *= s; })
        .def("dagger", &E::dagger)
        .def("plus_hc", [](E const& a) { return a + Operators::hc; })
        .def("is_complex", &E::is_complex);
}

}  // namespace

PYBIND11_MODULE(_pomerol, m) {
    m.doc() = "Drop-in host layer of pomerol's G2/G/chi path on the B200 engine (libpgx)";

    py::enum_<spin>(m, "spin").value("undef", spin::undef).value("down", spin::down).value("up", spin::up).export_values();

    bind_expr<RealExpr>(m, "RealExpr");
    bind_expr<ComplexExpr>(m, "ComplexExpr");
    py::implicitly_convertible<RealExpr, ComplexExpr>();
    m.def("to_complex", [](RealExpr const& e) { return ComplexExpr(e); });
    m.def("add", [](RealExpr const& a, ComplexExpr const& b) { return a + b; });

    auto ops = m.def_submodule("Operators");
    ops.def("c", [](std::string const& l, unsigned short o, spin s) { return Operators::c<double>(l, o, s); },
            py::arg("label"), py::arg("orbital") = 0, py::arg("spin") = spin::down);
    ops.def("c_dag", [](std::string const& l, unsigned short o, spin s) { return Operators::c_dag<double>(l, o, s); },
            py::arg("label"), py::arg("orbital") = 0, py::arg("spin") = spin::down);
    ops.def("n", [](std::string const& l, unsigned short o, spin s) { return Operators::n<double>(l, o, s); },
            py::arg("label"), py::arg("orbital") = 0, py::arg("spin") = spin::down);

    auto lp = m.def_submodule("LatticePresets");
    namespace L = LatticePresets;
    lp.def("Level", py::overload_cast<std::string const&, double, unsigned short>(&L::Level), py::arg("label"),
           py::arg("eps"), py::arg("norbitals") = 1);
    lp.def("Level", py::overload_cast<std::string const&, double, unsigned short, spin>(&L::Level));
    lp.def("Hopping", py::overload_cast<std::string const&, std::string const&, double, unsigned short>(&L::Hopping),
           py::arg("label1"), py::arg("label2"), py::arg("t"), py::arg("norbitals") = 1);
    lp.def("Hopping", py::overload_cast<std::string const&, std::string const&, double, unsigned short, unsigned short,
                                        spin, spin>(&L::Hopping));
    lp.def("Hopping", py::overload_cast<std::string const&, std::string const&, C, unsigned short, unsigned short, spin,
                                        spin>(&L::Hopping));
    lp.def("Magnetization", &L::Magnetization, py::arg("label"), py::arg("h"), py::arg("norbitals") = 1);
    lp.def("Pairing", &L::Pairing, py::arg("label"), py::arg("delta"), py::arg("norbitals") = 1);
    lp.def("NupNdown", py::overload_cast<std::string const&, std::string const&, double, unsigned short, unsigned short,
                                         spin, spin>(&L::NupNdown));
    lp.def("Spinflip", &L::Spinflip);
    lp.def("PairHopping", &L::PairHopping);
    lp.def("CoulombS", &L::CoulombS, py::arg("label"), py::arg("U"), py::arg("eps"), py::arg("norbitals") = 1);
    lp.def("CoulombP", py::overload_cast<std::string const&, double, double, double, double, unsigned short>(&L::CoulombP),
           py::arg("label"), py::arg("U"), py::arg("U_p"), py::arg("J"), py::arg("eps"), py::arg("norbitals") = 3);

    py::class_<IndexClassification>(m, "IndexClassification")
        .def(py::init<RealExpr const&>())
        .def(py::init<ComplexExpr const&>())
        .def("getIndex", py::overload_cast<std::string const&, unsigned short, spin>(&IndexClassification::getIndex,
                                                                                     py::const_))
        .def("getInfo", &IndexClassification::getInfo)
        .def("getIndexSize", &IndexClassification::getIndexSize);
    m.def("MakeIndexClassification", [](RealExpr const& e) { return IndexClassification(e); });
    m.def("MakeIndexClassification", [](ComplexExpr const& e) { return IndexClassification(e); });

    py::class_<HilbertSpace>(m, "HilbertSpace")
        .def("compute", &HilbertSpace::compute)
        .def("getDim", &HilbertSpace::getDim)
        .def("getNumberOfBlocks", &HilbertSpace::getNumberOfBlocks);
    // one function for both expression types: keep_alive on the second of two
    // overloads faulted in pybind11's post-call handling
    m.def(
        "MakeHilbertSpace",
        [](IndexClassification const& ii, py::object const& e) -> HilbertSpace* {
            if (py::isinstance<RealExpr>(e)) return new HilbertSpace(ii, e.cast<RealExpr const&>());
            return new HilbertSpace(ii, e.cast<ComplexExpr const&>());
        },
        py::keep_alive<0, 1>());

    py::class_<StatesClassification>(m, "StatesClassification")
        .def(py::init<>())
        .def("compute", &StatesClassification::compute)
        .def("getNumberOfStates", &StatesClassification::getNumberOfStates)
        .def("getNumberOfBlocks", &StatesClassification::getNumberOfBlocks)
        .def("getBlockSize", &StatesClassification::getBlockSize)
        .def("getFockStates", &StatesClassification::getFockStates)
        .def("getBlockNumber", &StatesClassification::getBlockNumber)
        .def("getInnerState", &StatesClassification::getInnerState);

    py::class_<HamiltonianPart>(m, "HamiltonianPart")
        .def("getSize", &HamiltonianPart::getSize)
        .def("getEigenValues", &HamiltonianPart::getEigenValues)
        .def("getEigenValue", &HamiltonianPart::getEigenValue)
        .def("getMinimumEigenvalue", &HamiltonianPart::getMinimumEigenvalue)
        .def("getMatrix", [](HamiltonianPart const& p) {
            auto m = p.getMatrix();  // the block, or its reduced corner after Hamiltonian::reduce
            const long d = std::lround(std::sqrt((double)(m.size() / (p.isComplex() ? 2 : 1))));
            return as_matrix(m, d, d, p.isComplex());
        });

    py::class_<Hamiltonian>(m, "Hamiltonian")
        .def(py::init<StatesClassification const&, int>(), py::arg("S"), py::arg("device") = 0, py::keep_alive<1, 2>())
        .def("prepare", [](Hamiltonian& H, RealExpr const& e, HilbertSpace const& hs, int) { H.prepare(e, hs); },
             py::arg("HExpr"), py::arg("HS"), py::arg("comm") = 0)
        .def("prepare", [](Hamiltonian& H, ComplexExpr const& e, HilbertSpace const& hs, int) { H.prepare(e, hs); },
             py::arg("HExpr"), py::arg("HS"), py::arg("comm") = 0)
        .def("compute", [](Hamiltonian& H, int) { H.compute(); }, py::arg("comm") = 0)
        .def("reduce", &Hamiltonian::reduce, py::arg("Cutoff"))
        .def("getPart", &Hamiltonian::getPart, py::return_value_policy::reference_internal)
        .def("getGroundEnergy", &Hamiltonian::getGroundEnergy)
        .def("getEigenValues", py::overload_cast<>(&Hamiltonian::getEigenValues, py::const_))
        .def("getBlockEigenValues", py::overload_cast<BlockNumber>(&Hamiltonian::getEigenValues, py::const_))
        .def("isComplex", &Hamiltonian::isComplex);

    py::class_<DensityMatrix>(m, "DensityMatrix")
        .def(py::init<StatesClassification const&, Hamiltonian const&, double>(), py::keep_alive<1, 2>(),
             py::keep_alive<1, 3>())
        .def_readonly("beta", &DensityMatrix::beta)
        .def("prepare", &DensityMatrix::prepare)
        .def("compute", &DensityMatrix::compute)
        .def("getWeight", &DensityMatrix::getWeight)
        .def("getAverageEnergy", &DensityMatrix::getAverageEnergy)
        .def("truncateBlocks", &DensityMatrix::truncateBlocks, py::arg("tol"), py::arg("verbose") = false)
        .def("isRetained", &DensityMatrix::isRetained);

    py::class_<MonomialOperatorPart>(m, "MonomialOperatorPart")
        .def("getLeftIndex", &MonomialOperatorPart::getLeftIndex)
        .def("getRightIndex", &MonomialOperatorPart::getRightIndex)
        .def("getMatrix", [](MonomialOperatorPart const& p) {
            return as_matrix(p.getMatrix(), (long)p.getLeftSize(), (long)p.getRightSize(), p.isComplex());
        });

    py::class_<MonomialOperator>(m, "MonomialOperator")
        .def("prepare", &MonomialOperator::prepare)
        .def("compute", [](MonomialOperator& o, double tol, int) { o.compute(tol); }, py::arg("tol") = 1e-8,
             py::arg("comm") = 0)
        .def("getLeftIndex", &MonomialOperator::getLeftIndex)
        .def("getRightIndex", &MonomialOperator::getRightIndex)
        .def("getBlockMapping", [](MonomialOperator const& o) { return o.getBlockMapping().right; })
        .def("getPartFromRightIndex", &MonomialOperator::getPartFromRightIndex, py::return_value_policy::reference_internal)
        .def("getPartFromLeftIndex", &MonomialOperator::getPartFromLeftIndex, py::return_value_policy::reference_internal)
        .def("isComplex", &MonomialOperator::isComplex)
        .def("fockAction", [](MonomialOperator const& o) {
            std::vector<std::tuple<int, int, std::vector<int32_t>, std::vector<double>>> r;
            for (auto& a : o.fockAction()) r.emplace_back(a.right, a.left, a.target, a.coef);
            return r;
        });
    py::class_<FieldOperator, MonomialOperator>(m, "FieldOperator").def("getIndex", &FieldOperator::getIndex);
    py::class_<CreationOperator, FieldOperator>(m, "CreationOperator")
        .def(py::init<IndexClassification const&, HilbertSpace const&, StatesClassification const&, Hamiltonian const&,
                      ParticleIndex>(),
             py::keep_alive<1, 4>(), py::keep_alive<1, 5>());
    py::class_<AnnihilationOperator, FieldOperator>(m, "AnnihilationOperator")
        .def(py::init<IndexClassification const&, HilbertSpace const&, StatesClassification const&, Hamiltonian const&,
                      ParticleIndex>(),
             py::keep_alive<1, 4>(), py::keep_alive<1, 5>());
    py::class_<QuadraticOperator, MonomialOperator>(m, "QuadraticOperator")
        .def(py::init<IndexClassification const&, HilbertSpace const&, StatesClassification const&, Hamiltonian const&,
                      ParticleIndex, ParticleIndex, std::tuple<bool, bool> const&>(),
             py::arg("IndexInfo"), py::arg("HS"), py::arg("S"), py::arg("H"), py::arg("Index1"), py::arg("Index2"),
             py::arg("Dagger") = std::tuple<bool, bool>(true, false), py::keep_alive<1, 4>(), py::keep_alive<1, 5>());
    py::class_<QuarticOperator, MonomialOperator>(m, "QuarticOperator")
        .def(py::init<IndexClassification const&, HilbertSpace const&, StatesClassification const&, Hamiltonian const&,
                      ParticleIndex, ParticleIndex, ParticleIndex, ParticleIndex,
                      std::tuple<bool, bool, bool, bool> const&>(),
             py::arg("IndexInfo"), py::arg("HS"), py::arg("S"), py::arg("H"), py::arg("Index1"), py::arg("Index2"),
             py::arg("Index3"), py::arg("Index4"),
             py::arg("Dagger") = std::tuple<bool, bool, bool, bool>(true, true, false, false), py::keep_alive<1, 4>(),
             py::keep_alive<1, 5>());

    py::class_<FieldOperatorContainer>(m, "FieldOperatorContainer")
        .def(py::init<IndexClassification const&, HilbertSpace const&, StatesClassification const&, Hamiltonian const&,
                      std::set<ParticleIndex>>(),
             py::arg("IndexInfo"), py::arg("HS"), py::arg("S"), py::arg("H"), py::arg("indices") = std::set<ParticleIndex>(),
             py::keep_alive<1, 4>(), py::keep_alive<1, 5>())
        .def("prepareAll", &FieldOperatorContainer::prepareAll)
        .def("computeAll", &FieldOperatorContainer::computeAll, py::arg("tol") = 1e-8)
        .def("getCreationOperator", &FieldOperatorContainer::getCreationOperator, py::return_value_policy::reference_internal)
        .def("getAnnihilationOperator", &FieldOperatorContainer::getAnnihilationOperator,
             py::return_value_policy::reference_internal);

    py::class_<GreensFunction>(m, "GreensFunction")
        .def(py::init<StatesClassification const&, Hamiltonian const&, FieldOperator const&, FieldOperator const&,
                      DensityMatrix const&>(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(),
             py::keep_alive<1, 6>())
        .def_readwrite("PoleResolution", &GreensFunction::PoleResolution)
        .def_readwrite("CoefficientTolerance", &GreensFunction::CoefficientTolerance)
        .def("prepare", &GreensFunction::prepare)
        .def("compute", &GreensFunction::compute)
        .def("__call__", py::overload_cast<long>(&GreensFunction::operator(), py::const_))
        .def("__call__", py::overload_cast<C>(&GreensFunction::operator(), py::const_))
        .def("values", &GreensFunction::values)
        .def("isVanishing", &GreensFunction::isVanishing)
        .def("getIndex", &GreensFunction::getIndex);

    py::class_<GFContainer>(m, "GFContainer")
        .def(py::init<IndexClassification const&, StatesClassification const&, Hamiltonian const&, DensityMatrix const&,
                      FieldOperatorContainer const&, bool>(),
             py::arg("IndexInfo"), py::arg("S"), py::arg("H"), py::arg("DM"), py::arg("Ops"), py::arg("Anomalous") = false,
             py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(), py::keep_alive<1, 6>())
        .def("prepareAll",
             [](GFContainer& g, std::vector<std::pair<ParticleIndex, ParticleIndex>> const& idx) {
                 std::set<IndexCombination2> s;
                 for (auto const& p : idx) s.emplace(p.first, p.second);
                 g.prepareAll(s);
             },
             py::arg("indices") = std::vector<std::pair<ParticleIndex, ParticleIndex>>())
        .def("computeAll", &GFContainer::computeAll)
        .def("__call__", [](GFContainer& g, ParticleIndex i, ParticleIndex j) -> GreensFunction& { return g(i, j); },
             py::return_value_policy::reference_internal);

    py::class_<EnsembleAverage>(m, "EnsembleAverage")
        .def(py::init<MonomialOperator const&, DensityMatrix const&>(), py::keep_alive<1, 2>(), py::keep_alive<1, 3>())
        .def("compute", &EnsembleAverage::compute)
        .def("__call__", &EnsembleAverage::operator());

    py::class_<Susceptibility>(m, "Susceptibility")
        .def(py::init<StatesClassification const&, Hamiltonian const&, MonomialOperator const&, MonomialOperator const&,
                      DensityMatrix const&>(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(),
             py::keep_alive<1, 6>())
        .def_readwrite("PoleResolution", &Susceptibility::PoleResolution)
        .def_readwrite("CoefficientTolerance", &Susceptibility::CoefficientTolerance)
        .def("prepare", &Susceptibility::prepare)
        .def("compute", &Susceptibility::compute)
        .def("subtractDisconnected", py::overload_cast<>(&Susceptibility::subtractDisconnected))
        .def("subtractDisconnected", py::overload_cast<C, C>(&Susceptibility::subtractDisconnected))
        .def("subtractDisconnected", py::overload_cast<EnsembleAverage&, EnsembleAverage&>(&Susceptibility::subtractDisconnected))
        .def("__call__", py::overload_cast<long>(&Susceptibility::operator(), py::const_))
        .def("__call__", py::overload_cast<C>(&Susceptibility::operator(), py::const_))
        .def("values", &Susceptibility::values)
        .def("isVanishing", &Susceptibility::isVanishing);

    py::class_<TwoParticleGF>(m, "TwoParticleGF")
        .def(py::init<StatesClassification const&, Hamiltonian const&, AnnihilationOperator const&,
                      AnnihilationOperator const&, CreationOperator const&, CreationOperator const&, DensityMatrix const&>(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(),
             py::keep_alive<1, 6>(), py::keep_alive<1, 7>(), py::keep_alive<1, 8>())
        .def_readwrite("PoleResolution", &TwoParticleGF::PoleResolution)
        .def_readwrite("CoefficientTolerance", &TwoParticleGF::CoefficientTolerance)
        .def_readwrite("AnchorTolerance", &TwoParticleGF::AnchorTolerance)
        .def_readwrite("ExactSum", &TwoParticleGF::ExactSum)
        .def_readwrite("SplitProducts", &TwoParticleGF::SplitProducts)
        .def_readwrite("SplitSlices", &TwoParticleGF::SplitSlices)
        .def("prepare", &TwoParticleGF::prepare)
        .def("compute",
             [](TwoParticleGF& g, bool clear, std::vector<std::tuple<C, C, C>> const& f, int) {
                 return g.compute(clear, to_freqs(f));
             },
             py::arg("clear") = false, py::arg("freqs") = std::vector<std::tuple<C, C, C>>(), py::arg("comm") = 0)
        .def("__call__", py::overload_cast<long, long, long>(&TwoParticleGF::operator(), py::const_))
        .def("__call__", py::overload_cast<C, C, C>(&TwoParticleGF::operator(), py::const_))
        .def("values", [](TwoParticleGF const& g, std::vector<std::tuple<C, C, C>> const& f) { return g.values(to_freqs(f)); })
        .def("isVanishing", &TwoParticleGF::isVanishing)
        .def("getNumParts", &TwoParticleGF::getNumParts)
        .def("getIndex", &TwoParticleGF::getIndex)
        .def("parts", [](TwoParticleGF const& g) {
            std::vector<std::tuple<std::array<int, 4>, std::array<int, 3>, int>> r;
            for (auto const& p : g.deviceParts())
                r.emplace_back(std::array<int, 4>{p.block[0], p.block[1], p.block[2], p.block[3]},
                               std::array<int, 3>{p.perm[0], p.perm[1], p.perm[2]}, p.sign);
            return r;
        });

    py::class_<ElementWithPermFreq<TwoParticleGF>>(m, "TwoParticleGFElement")
        .def("__call__", &ElementWithPermFreq<TwoParticleGF>::operator())
        .def("element", &ElementWithPermFreq<TwoParticleGF>::element, py::return_value_policy::reference_internal);

    py::class_<TwoParticleGFContainer>(m, "TwoParticleGFContainer")
        .def(py::init<IndexClassification const&, StatesClassification const&, Hamiltonian const&, DensityMatrix const&,
                      FieldOperatorContainer const&>(),
             py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(), py::keep_alive<1, 6>())
        .def_readwrite("PoleResolution", &TwoParticleGFContainer::PoleResolution)
        .def_readwrite("CoefficientTolerance", &TwoParticleGFContainer::CoefficientTolerance)
        .def_readwrite("SplitProducts", &TwoParticleGFContainer::SplitProducts)
        .def_readwrite("AnchorTolerance", &TwoParticleGFContainer::AnchorTolerance)
        .def_readwrite("SplitSlices", &TwoParticleGFContainer::SplitSlices)
        .def("prepareAll",
             [](TwoParticleGFContainer& g, std::vector<std::array<ParticleIndex, 4>> const& idx) {
                 std::set<IndexCombination4> s;
                 for (auto const& p : idx) s.emplace(p[0], p[1], p[2], p[3]);
                 g.prepareAll(s);
             },
             py::arg("indices") = std::vector<std::array<ParticleIndex, 4>>())
        .def("computeAll",
             [](TwoParticleGFContainer& g, bool clear, std::vector<std::tuple<C, C, C>> const& f, int, bool split) {
                 auto r = g.computeAll(clear, to_freqs(f), 0, split);
                 std::map<std::tuple<int, int, int, int>, std::vector<C>> out;
                 for (auto& kv : r)
                     out[std::make_tuple(kv.first.Index1, kv.first.Index2, kv.first.Index3, kv.first.Index4)] = kv.second;
                 return out;
             },
             py::arg("clear") = false, py::arg("freqs") = std::vector<std::tuple<C, C, C>>(), py::arg("comm") = 0,
             py::arg("split") = true)
        .def("__call__",
             [](TwoParticleGFContainer& g, ParticleIndex i, ParticleIndex j, ParticleIndex k, ParticleIndex l)
                 -> ElementWithPermFreq<TwoParticleGF>& { return g(i, j, k, l); },
             py::return_value_policy::reference_internal)
        .def("isInContainer", [](TwoParticleGFContainer const& g, ParticleIndex i, ParticleIndex j, ParticleIndex k,
                                 ParticleIndex l) { return g.isInContainer(IndexCombination4(i, j, k, l)); });

    py::enum_<Channel>(m, "Channel").value("PP", PP).value("PH", PH).value("xPH", xPH).export_values();

    py::class_<ThreePointSusceptibility>(m, "ThreePointSusceptibility")
        .def(py::init<Channel, StatesClassification const&, Hamiltonian const&, CreationOperator const&,
                      AnnihilationOperator const&, CreationOperator const&, AnnihilationOperator const&,
                      DensityMatrix const&>(),
             py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(), py::keep_alive<1, 6>(),
             py::keep_alive<1, 7>(), py::keep_alive<1, 8>(), py::keep_alive<1, 9>())
        .def_readwrite("PoleResolution", &ThreePointSusceptibility::PoleResolution)
        .def_readwrite("CoefficientTolerance", &ThreePointSusceptibility::CoefficientTolerance)
        .def("prepare", &ThreePointSusceptibility::prepare)
        .def("compute",
             [](ThreePointSusceptibility& g, bool clear, std::vector<std::tuple<C, C>> const& f, int) {
                 return g.compute(clear, to_freqs2(f));
             },
             py::arg("clear") = false, py::arg("freqs") = std::vector<std::tuple<C, C>>(), py::arg("comm") = 0)
        .def("__call__", py::overload_cast<long, long>(&ThreePointSusceptibility::operator(), py::const_))
        .def("__call__", py::overload_cast<C, C>(&ThreePointSusceptibility::operator(), py::const_))
        .def("values",
             [](ThreePointSusceptibility const& g, std::vector<std::tuple<C, C>> const& f) {
                 return g.values(to_freqs2(f));
             })
        .def("isVanishing", &ThreePointSusceptibility::isVanishing)
        .def("getNumParts", &ThreePointSusceptibility::getNumParts)
        .def("getIndex", &ThreePointSusceptibility::getIndex)
        .def("parts", [](ThreePointSusceptibility const& g) {
            std::vector<std::tuple<std::array<int, 4>, int>> r;
            for (auto const& p : g.deviceParts())
                r.emplace_back(std::array<int, 4>{p.block[0], p.block[1], p.block[2], p.block[3]}, p.swapped);
            return r;
        });

    py::class_<ElementWithPermFreq<ThreePointSusceptibility>>(m, "ThreePointSusceptibilityElement")
        .def("element", &ElementWithPermFreq<ThreePointSusceptibility>::element,
             py::return_value_policy::reference_internal);

    py::class_<ThreePointSusceptibilityContainer>(m, "ThreePointSusceptibilityContainer")
        .def(py::init<Channel, IndexClassification const&, StatesClassification const&, Hamiltonian const&,
                      DensityMatrix const&, FieldOperatorContainer const&>(),
             py::keep_alive<1, 4>(), py::keep_alive<1, 5>(), py::keep_alive<1, 6>(), py::keep_alive<1, 7>())
        .def_readwrite("PoleResolution", &ThreePointSusceptibilityContainer::PoleResolution)
        .def_readwrite("CoefficientTolerance", &ThreePointSusceptibilityContainer::CoefficientTolerance)
        .def("prepareAll",
             [](ThreePointSusceptibilityContainer& g, std::vector<std::array<ParticleIndex, 4>> const& idx) {
                 std::set<IndexCombination4> s;
                 for (auto const& p : idx) s.emplace(p[0], p[1], p[2], p[3]);
                 g.prepareAll(s);
             },
             py::arg("indices") = std::vector<std::array<ParticleIndex, 4>>())
        .def("computeAll",
             [](ThreePointSusceptibilityContainer& g, bool clear, std::vector<std::tuple<C, C>> const& f, int) {
                 auto r = g.computeAll(clear, to_freqs2(f));
                 std::map<std::tuple<int, int, int, int>, std::vector<C>> out;
                 for (auto& kv : r)
                     out[std::make_tuple(kv.first.Index1, kv.first.Index2, kv.first.Index3, kv.first.Index4)] = kv.second;
                 return out;
             },
             py::arg("clear") = false, py::arg("freqs") = std::vector<std::tuple<C, C>>(), py::arg("comm") = 0)
        .def("__call__",
             [](ThreePointSusceptibilityContainer& g, ParticleIndex i, ParticleIndex j, ParticleIndex k,
                ParticleIndex l) -> ElementWithPermFreq<ThreePointSusceptibility>& { return g(i, j, k, l); },
             py::return_value_policy::reference_internal)
        .def("isInContainer", [](ThreePointSusceptibilityContainer const& g, ParticleIndex i, ParticleIndex j,
                                 ParticleIndex k, ParticleIndex l) {
            return g.isInContainer(IndexCombination4(i, j, k, l));
        });

    py::class_<Vertex4>(m, "Vertex4")
        .def(py::init<TwoParticleGF const&, GreensFunction const&, GreensFunction const&, GreensFunction const&,
                      GreensFunction const&>(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>(),
             py::keep_alive<1, 6>())
        .def("compute", &Vertex4::compute, py::arg("NumberOfMatsubaras") = 0)
        .def("__call__", &Vertex4::operator())
        .def("value", &Vertex4::value)
        .def("getNumberOfMatsubaras", &Vertex4::getNumberOfMatsubaras);
}
