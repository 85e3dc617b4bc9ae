// CPU oracle, part 4 (TEST INFRASTRUCTURE ONLY): the reference's G2 Lehmann
// algorithm restated in C++ for the reference-rule checker and the CPU
// baseline of bench.py.  Never linked into the product.
//
// Follows, per block chain (part):
//   TwoParticleGFPart::computeImpl   TwoParticleGFPart.cpp:189-265
//     - iterate index1 (states of S1) x index3 (states of S3), chase the
//       common index4 of row index3 of O3 and column index1 of CX4
//       (ChaseIndices.hpp:29-46), then the common index2 of row index1 of
//       O1 and column index3 of O2;
//     - keep quadruples with w1+w2+w3+w4 > CoefficientTolerance (:241);
//   TwoParticleGFPart::addMultiterm  TwoParticleGFPart.cpp:267-298
//   TermList::add_term               TermList.hpp:65-76 (merge in the same
//     binned-pole slot, Misc.cpp:83-86; weighted pole average
//     TwoParticleGFPart.cpp:35-43, 86-95; erase when negligible at
//     tolerance/(size+1); a re-inserted sum whose new slot is taken is
//     dropped, as std::unordered_set::emplace does);
//   NonResonantTerm / ResonantTerm::operator()  TwoParticleGFPart.hpp:475-495
//   TwoParticleGFPart::operator()    TwoParticleGFPart.cpp:309-322
//   the OpenMP loop over frequencies TwoParticleGF.cpp:136-144.
// "Non-zero" matrix elements are |x| > nz_tol: the reference's
// sparseView(Tolerance) (MonomialOperatorPart.cpp:87) keeps |x| > Tolerance *
// 1e-12 (Eigen's default dummy precision), i.e. |x| > 1e-20 at the default
// Tolerance 1e-8.
#include <omp.h>

#include <cmath>
#include <complex>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <unordered_map>
#include <vector>

using cplx = std::complex<double>;

namespace {

struct Key {
    int flag;
    int64_t b0, b1, b2;
    bool operator==(Key const& o) const { return flag == o.flag && b0 == o.b0 && b1 == o.b1 && b2 == o.b2; }
};
struct KeyHash {
    size_t operator()(Key const& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint64_t v : {(uint64_t)k.flag, (uint64_t)k.b0, (uint64_t)k.b1, (uint64_t)k.b2}) {
            h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        }
        return (size_t)h;
    }
};

struct Term {
    cplx c1, c2;   // NR: Coeff (c2 unused); Res: ResCoeff, NonResCoeff
    double p[3];
    long weight;
};

struct TermList {
    double res, tol;
    std::unordered_map<Key, Term, KeyHash> data;
    Key key(int flag, const double* p) const {
        return Key{flag, (int64_t)std::llround(p[0] / res), (int64_t)std::llround(p[1] / res),
                   (int64_t)std::llround(p[2] / res)};
    }
    bool negligible(Term const& t, size_t div, bool resonant) const {
        const double th = tol / (double)div;
        return resonant ? (std::abs(t.c1) <= th && std::abs(t.c2) <= th) : std::abs(t.c1) <= th;
    }
    void add(int flag, Term const& t, bool resonant) {
        Key k = key(flag, t.p);
        auto it = data.find(k);
        if (it == data.end()) {
            data.emplace(k, t);
            return;
        }
        Term s = it->second;
        const long w = s.weight + t.weight;
        for (int q = 0; q < 3; ++q) s.p[q] = (s.weight * s.p[q] + t.weight * t.p[q]) / (double)w;
        s.weight = w;
        s.c1 += t.c1;
        s.c2 += t.c2;
        data.erase(it);
        if (!negligible(s, data.size() + 1, resonant)) data.emplace(key(flag, s.p), s);
    }
};

}  // namespace

extern "C" {

// Count quadruples passing the reference's enumeration filter: all four
// elements non-zero and w1 + w2 + w3 + w4 > coef_tol, summed in that order
// (TwoParticleGFPart.cpp:241).
long long g2o_count(int d1, int d2, int d3, int d4, const double* O1, const double* O2, const double* O3,
                    const double* X4, const double* w1, const double* w2, const double* w3, const double* w4,
                    double coef_tol, double nz_tol) {
    long long n = 0;
#pragma omp parallel for reduction(+ : n) schedule(dynamic)
    for (int i1 = 0; i1 < d1; ++i1) {
        std::vector<int> l2, l4;
        for (int i3 = 0; i3 < d3; ++i3) {
            l2.clear();
            l4.clear();
            for (int i2 = 0; i2 < d2; ++i2)
                if (std::fabs(O1[(long)i1 * d2 + i2]) > nz_tol && std::fabs(O2[(long)i2 * d3 + i3]) > nz_tol) l2.push_back(i2);
            if (l2.empty()) continue;
            for (int i4 = 0; i4 < d4; ++i4)
                if (std::fabs(O3[(long)i3 * d4 + i4]) > nz_tol && std::fabs(X4[(long)i4 * d1 + i1]) > nz_tol) l4.push_back(i4);
            // a rounded sum of non-negative weights only grows as terms are added
            if (w1[i1] + w3[i3] > coef_tol) {
                n += (long long)l2.size() * (long long)l4.size();
                continue;
            }
            for (int i2 : l2)
                for (int i4 : l4) n += (w1[i1] + w2[i2] + w3[i3] + w4[i4] > coef_tol);
        }
    }
    return n;
}

// Reference-rule (rule=1) or exact (rule=0) evaluation of one part.
// z: nfreq triples (re,im)x3 BEFORE the part's permutation; out += values.
// row_begin/row_end/row_step restrict index1, col_step strides index3 and
// chase_step strides index2 and index4 (bounded samples: every sampled
// quadruple is filtered, split into sub-terms, merged and evaluated as the
// reference does); returns the number of
// quadruples enumerated; terms_out[0..1] = non-resonant / resonant terms kept.
long long g2o_part(int d1, int d2, int d3, int d4, const double* O1, const double* O2, const double* O3,
                   const double* X4, const double* E1, const double* E2, const double* E3, const double* E4,
                   const double* w1, const double* w2, const double* w3, const double* w4, const int* perm, int sign,
                   double beta, double pole_res, double coef_tol, double nz_tol, int rule, int nfreq, const double* z,
                   int row_begin, int row_end, int row_step, int col_step, int chase_step, double* out,
                   long long* terms_out, int nthreads) {
    TermList NR{pole_res, coef_tol, {}}, RS{pole_res, coef_tol, {}};
    std::vector<Term> nr_plain, rs_plain;  // exact mode keeps every term
    std::vector<int> flags_nr, flags_rs;
    long long nq = 0;
    std::vector<int> l4;
    const double ctol = rule ? coef_tol : -1.0;
    for (int i1 = row_begin; i1 < row_end; i1 += std::max(row_step, 1)) {
        for (int i3 = 0; i3 < d3; i3 += std::max(col_step, 1)) {
            l4.clear();
            for (int i4 = 0; i4 < d4; i4 += std::max(chase_step, 1))
                if (std::fabs(O3[(long)i3 * d4 + i4]) > nz_tol && std::fabs(X4[(long)i4 * d1 + i1]) > nz_tol)
                    l4.push_back(i4);
            if (l4.empty()) continue;
            for (int i2 = 0; i2 < d2; i2 += std::max(chase_step, 1)) {
                const double a12 = O1[(long)i1 * d2 + i2], a23 = O2[(long)i2 * d3 + i3];
                if (!(std::fabs(a12) > nz_tol && std::fabs(a23) > nz_tol)) continue;
                for (int i4 : l4) {
                    const double W1 = w1[i1], W2 = w2[i2], W3 = w3[i3], W4 = w4[i4];
                    if (rule && !(W1 + W2 + W3 + W4 > coef_tol)) continue;
                    ++nq;
                    const double M = sign * a12 * a23 * O3[(long)i3 * d4 + i4] * X4[(long)i4 * d1 + i1];
                    const double P[3] = {E2[i2] - E1[i1], E3[i3] - E2[i2], E4[i4] - E3[i3]};
                    Term t{};
                    std::memcpy(t.p, P, sizeof(P));
                    t.weight = 1;
                    // non-resonant z2 and z4 terms
                    t.c1 = -M * (W2 + W3);
                    if (std::abs(t.c1) > ctol) {
                        if (rule) NR.add(0, t, false);
                        else { nr_plain.push_back(t); flags_nr.push_back(0); }
                    }
                    t.c1 = M * (W1 + W4);
                    if (std::abs(t.c1) > ctol) {
                        if (rule) NR.add(1, t, false);
                        else { nr_plain.push_back(t); flags_nr.push_back(1); }
                    }
                    // resonant z1z2 and z2z3 terms
                    t.c1 = M * beta * W1;
                    t.c2 = M * (W3 - W1);
                    if (std::abs(t.c1) > ctol || std::abs(t.c2) > ctol) {
                        if (rule) RS.add(1, t, true);
                        else { rs_plain.push_back(t); flags_rs.push_back(1); }
                    }
                    t.c1 = -M * beta * W2;
                    t.c2 = M * (W2 - W4);
                    if (std::abs(t.c1) > ctol || std::abs(t.c2) > ctol) {
                        if (rule) RS.add(0, t, true);
                        else { rs_plain.push_back(t); flags_rs.push_back(0); }
                    }
                }
            }
        }
    }
    // flatten term lists
    if (rule) {
        for (auto const& kv : NR.data) { nr_plain.push_back(kv.second); flags_nr.push_back(kv.first.flag); }
        for (auto const& kv : RS.data) { rs_plain.push_back(kv.second); flags_rs.push_back(kv.first.flag); }
    }
    if (terms_out) {
        terms_out[0] = (long long)nr_plain.size();
        terms_out[1] = (long long)rs_plain.size();
    }
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int w = 0; w < nfreq; ++w) {
        const cplx F[3] = {cplx(z[6 * w], z[6 * w + 1]), cplx(z[6 * w + 2], z[6 * w + 3]), -cplx(z[6 * w + 4], z[6 * w + 5])};
        const cplx a = F[perm[0]], b = F[perm[1]], c = F[perm[2]];
        cplx s = 0.0;
        for (size_t k = 0; k < nr_plain.size(); ++k) {
            const Term& t = nr_plain[k];
            if (flags_nr[k])
                s += t.c1 / ((a - t.p[0]) * (a + b + c - t.p[0] - t.p[1] - t.p[2]) * (c - t.p[2]));
            else
                s += t.c1 / ((a - t.p[0]) * (b - t.p[1]) * (c - t.p[2]));
        }
        for (size_t k = 0; k < rs_plain.size(); ++k) {
            const Term& t = rs_plain[k];
            const cplx D = flags_rs[k] ? (a + b - t.p[0] - t.p[1]) : (b + c - t.p[1] - t.p[2]);
            s += (std::abs(D) <= pole_res ? t.c1 : (t.c2 / D)) / ((a - t.p[0]) * (c - t.p[2]));
        }
        out[2 * w] += s.real();
        out[2 * w + 1] += s.imag();
    }
    return nq;
}

int g2o_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
