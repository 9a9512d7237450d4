// Host-side parts of libpned_gpu.so: model input (local matrices, TPS shift,
// Sz-sector lists), the term-program compiler, and the small tridiagonal /
// continued-fraction routines that run on the CPU in the reference too.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>

#include "pned_internal.h"

namespace pned {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int fail(int code, const std::string &msg)
{
    set_error(msg);
    return code;
}

// ---------------------------------------------------------------------------
// Local two-site matrices
// ---------------------------------------------------------------------------
namespace {

// Spin-component matrices S^a (a = x, y, z) on one site, q x q, row-major.
// tree 0: S = 1/2 with digit 0 = up (S1/2 params.f90:1434-1439);
// tree 1: digit d <-> m = d - S, S^+/S^- from sqrt((S -+ m)(S +- m + 1)),
//         S^y = -(i/2)(su - sd) (Sa params.f90:1479-1494).
std::vector<cd> single_site_ops(int q, int tree)
{
    std::vector<cd> s(3 * q * q, cd(0, 0));
    auto at = [&](int a, int i, int j) -> cd & { return s[(a * q + i) * q + j]; };
    if (tree == 0) {
        at(0, 0, 1) = 0.5; at(0, 1, 0) = 0.5;
        at(1, 0, 1) = cd(0, -0.5); at(1, 1, 0) = cd(0, 0.5);
        at(2, 0, 0) = 0.5; at(2, 1, 1) = -0.5;
        return s;
    }
    const double S = 0.5 * (q - 1);
    for (int i = 0; i < q; ++i) {
        const double m = i - S;
        cd up = (i + 1 < q) ? cd(std::sqrt((S - m) * (S + m + 1.0)), 0) : cd(0, 0);  // row i, col i+1
        cd dn = (i > 0) ? cd(std::sqrt((S + m) * (S - m + 1.0)), 0) : cd(0, 0);      // row i, col i-1
        if (i + 1 < q) {
            at(0, i, i + 1) += 0.5 * up;
            at(1, i, i + 1) += cd(0, -0.5) * up;
        }
        if (i > 0) {
            at(0, i, i - 1) += 0.5 * dn;
            at(1, i, i - 1) -= cd(0, -0.5) * dn;
        }
        at(2, i, i) = m;
    }
    return s;
}

// The seven 3x3 exchange matrices J1x, J1y, J1z, J2x, J2y, J2z, J3z built from
// the coupling slots; ratio_l multiplies the non-Kitaev entries, with the
// tree-1 placement of params.f90:1497-1521.
void exchange_matrices(const double *c, int tree, cd J[7][3][3])
{
    enum { J1, K1, I11, I12, J1p, K1p, J1pp, K1pp, I11p, I12p, I11pp, I12pp, J2, K2, I21, I22, J3, K3, RL };
    const double rl = c[RL];
    const double j13 = tree ? c[J1pp] : c[J1pp] * rl, j12 = tree ? c[J1p] : c[J1p] * rl;
    const double j11 = tree ? c[J1] : c[J1] * rl;
    const double z[3][3] = {{j11, c[I11] * rl, c[I12] * rl}, {c[I11] * rl, j11, c[I12] * rl},
                            {c[I12] * rl, c[I12] * rl, c[K1]}};
    const double x[3][3] = {{c[K1p], c[I12pp] * rl, c[I12p] * rl}, {c[I12pp] * rl, j13, c[I11p] * rl},
                            {c[I12p] * rl, c[I11p] * rl, j12}};
    const double y[3][3] = {{j13, c[I12pp] * rl, c[I11p] * rl}, {c[I12pp] * rl, c[K1p], c[I12p] * rl},
                            {c[I11p] * rl, c[I12p] * rl, j12}};
    const double a2 = c[J2] * rl, k2 = c[K2] * rl, g1 = c[I21] * rl, g2 = c[I22] * rl;
    const double x2[3][3] = {{k2, g1, g2}, {g1, a2, g2}, {g2, g2, a2}};
    const double y2[3][3] = {{a2, g1, g2}, {g1, k2, g2}, {g2, g2, a2}};
    const double z2[3][3] = {{a2, g1, g2}, {g1, a2, g2}, {g2, g2, k2}};
    const double j3 = c[J3] * rl;
    const double z3[3][3] = {{j3, 0, 0}, {0, j3, 0}, {0, 0, j3}};
    const double (*mats[7])[3] = {x, y, z, x2, y2, z2, z3};
    for (int t = 0; t < 7; ++t)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) J[t][a][b] = mats[t][a][b];
}

}  // namespace

}  // namespace pned

using namespace pned;

extern "C" int pned_build_xlocal(int q, int tree, const double *cpl, int simple, const double *field, double coord,
                                 pned_c128 *xout, uint8_t *skip_out, int *parity_out)
{
    if (q < 2 || q > 8 || (tree == 0 && q != 2) || (tree != 0 && tree != 1) || !cpl || !xout)
        return fail(PNED_EINVAL, "pned_build_xlocal: bad q_spin/tree/pointers");
    const int Q = q * q;
    std::vector<cd> s = single_site_ops(q, tree);
    cd J[7][3][3];
    exchange_matrices(cpl, tree, J);
    // two-site operators P_ab(row = q*j1 + i1, col = q*j2 + i2) = S^a(i1,i2) S^b(j1,j2)
    std::vector<cd> P(9 * Q * Q);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int j1 = 0; j1 < q; ++j1)
                for (int i1 = 0; i1 < q; ++i1)
                    for (int j2 = 0; j2 < q; ++j2)
                        for (int i2 = 0; i2 < q; ++i2)
                            P[(3 * a + b) * Q * Q + (q * j1 + i1) * Q + (q * j2 + i2)] =
                                s[(a * q + i1) * q + i2] * s[(b * q + j1) * q + j2];
    std::vector<cd> X(9 * Q * Q, cd(0, 0));
    for (int row = 0; row < Q; ++row)
        for (int col = 0; col < Q; ++col) {
            cd v[7];
            for (int t = 0; t < 7; ++t) {
                // same term order as the reference: xx xy xz yx yy yz zx zy zz
                cd acc = J[t][0][0] * P[row * Q + col];
                for (int ab = 1; ab < 9; ++ab) acc = acc + J[t][ab / 3][ab % 3] * P[ab * Q * Q + row * Q + col];
                v[t] = acc;
            }
            cd x2x = v[3], x2y = v[4];
            const bool keep_second = tree == 0 || simple == 3 || simple == 4;
            if (simple == 3) { x2x = v[5]; x2y = v[5]; }
            if (!keep_second) { x2x = 0; x2y = 0; }
            const cd out[9] = {v[0], v[1], v[2], x2x, x2y, v[5], v[6], v[6], v[6]};
            for (int t = 0; t < 9; ++t) X[t * Q * Q + row + Q * col] += out[t];
        }
    if (field) {
        for (int t = 0; t < 3; ++t)
            for (int j1 = 0; j1 < q; ++j1)
                for (int i1 = 0; i1 < q; ++i1)
                    for (int j2 = 0; j2 < q; ++j2)
                        for (int i2 = 0; i2 < q; ++i2) {
                            cd acc = 0;
                            for (int a = 0; a < 3; ++a) {
                                if (j1 == j2) acc += field[a] * s[(a * q + i1) * q + i2];
                                if (i1 == i2) acc += field[a] * s[(a * q + j1) * q + j2];
                            }
                            X[t * Q * Q + (q * j1 + i1) + Q * (q * j2 + i2)] -= acc / coord;
                        }
    }
    // parity type and skip mask
    const double eps = .5e-28;
    auto mag2 = [](cd z) { return std::fabs((std::conj(z) * z).real()); };
    auto XA = [&](int r, int c, int t) { return X[t * Q * Q + r + Q * c]; };
    int pt = 0;
    std::vector<uint8_t> skip(9 * Q * Q, 1);
    if (tree == 0) {
        for (int t = 0; t < 9; ++t) {
            if (mag2(XA(1, 0, t)) > eps || mag2(XA(2, 0, t)) > eps) pt |= 2;
            if (mag2(XA(3, 0, t)) > eps) pt |= 1;
        }
        for (int t = 0; t < 9; ++t)
            for (int c = 0; c < Q; ++c)
                for (int r = 0; r < Q; ++r) {
                    bool keep;
                    if (pt == 0)
                        keep = (r == c) || (r == 1 && c == 2) || (r == 2 && c == 1);
                    else
                        keep = (r == c) || mag2(XA(r, c, t)) > eps;
                    skip[t * Q * Q + r + Q * c] = keep ? 0 : 1;
                }
    } else {
        auto dsum = [&](int st) { return st % q + st / q; };
        for (int t = 0; t < 9; ++t)
            for (int j = 0; j < Q; ++j)
                for (int i = j; i < Q; ++i)
                    if (dsum(j) != dsum(i) && mag2(XA(i, j, t)) > eps) pt |= 1;
        for (int t = 0; t < 9; ++t)
            for (int j = 0; j < Q; ++j)
                for (int i = 0; i < Q; ++i) {
                    bool keep = (i == j) || (pt == 0 ? dsum(i) == dsum(j) : mag2(XA(i, j, t)) > eps);
                    skip[t * Q * Q + i + Q * j] = keep ? 0 : 1;
                }
    }
    for (int k = 0; k < 9 * Q * Q; ++k) xout[k] = pned_c128{X[k].real(), X[k].imag()};
    if (skip_out) std::memcpy(skip_out, skip.data(), skip.size());
    if (parity_out) *parity_out = pt;
    return PNED_OK;
}

extern "C" int pned_tps_transform(int q, int tree, int nbond, double c_count, int mode, pned_c128 *x, double *L)
{
    if (q < 2 || !x || !L || nbond <= 0) return fail(PNED_EINVAL, "pned_tps_transform: bad arguments");
    const int Q = q * q;
    auto at = [&](int r, int c, int t) -> pned_c128 & { return x[t * Q * Q + r + Q * c]; };
    double lb;
    int ndiag = Q;
    if (mode == 0) {
        // reference: l_b from the diagonal entries 0..3 of all nine types
        double acc = 0;
        for (int t = 0; t < 9; ++t)
            for (int i = 0; i < 4 && i < Q; ++i) {
                const pned_c128 z = at(i, i, t);
                const double m2 = std::fabs(z.re * z.re + z.im * z.im);
                acc += tree == 0 ? m2 : 0.25 * double((q - 1) * (q - 1)) * std::sqrt(m2);
            }
        lb = tree == 0 ? acc / c_count : 2.0 * acc / c_count / double(Q);
        ndiag = std::min(4, Q);   // the reference shifts entries 0..3 only
        *L = lb * double(nbond);
    } else if (mode == 1) {
        lb = *L / double(nbond);
    } else {
        return fail(PNED_EINVAL, "pned_tps_transform: mode must be 0 or 1");
    }
    for (int k = 0; k < 9 * Q * Q; ++k) { x[k].re = -x[k].re; x[k].im = -x[k].im; }
    for (int t = 0; t < 9; ++t)
        for (int i = 0; i < ndiag; ++i) at(i, i, t).re = lb + at(i, i, t).re;
    return PNED_OK;
}

extern "C" int pned_mk_list12(int n, int q, int parity_type, int total_sz, int64_t *ldim, int64_t *list1,
                              int64_t *l3lo, int64_t *l3hi)
{
    if (n < 1 || q < 2 || !ldim) return fail(PNED_EINVAL, "pned_mk_list12: bad arguments");
    const int ihf0 = n / 2, ihf = (n + 1) / 2;
    int64_t nA = 1, nB = 1;
    for (int i = 0; i < ihf; ++i) nA *= q;
    for (int i = 0; i < ihf0; ++i) nB *= q;
    std::vector<int> dsum(nA);
    for (int64_t j = 0; j < nA; ++j) {
        int64_t x = j;
        int s = 0;
        for (int i = 0; i < ihf; ++i) { s += int(x % q); x /= q; }
        dsum[j] = s;
    }
    int64_t cnt = 0;
    int64_t ja = 0, jb = 0, ibpat = 0;
    const int64_t nmax = std::max(nA, nB);
    if (l3lo) std::fill(l3lo, l3lo + nmax, int64_t(-1));
    if (l3hi) std::fill(l3hi, l3hi + nmax, int64_t(-1));
    for (int64_t i2 = 0; i2 < nB; ++i2)
        for (int64_t i1 = 0; i1 < nA; ++i1) {
            if (parity_type == 0 && dsum[i1] + dsum[i2] != total_sz) continue;
            ++cnt;
            if (!list1) continue;
            if (i2 == ibpat) ++ja;
            else { ibpat = i2; ja = 1; jb = cnt - 1; }
            list1[cnt - 1] = i2 * nA + i1;
            if (l3lo) l3lo[i1] = ja;
            if (l3hi) l3hi[i2] = jb;
        }
    *ldim = cnt;
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// Term-program compiler
// ---------------------------------------------------------------------------
namespace pned {

namespace {

struct Bond { int s1, s2, t; };

// Bonds in schedule order: tree 0 keeps ipair order (sort_list of
// S1/2 MPIlib.f90:344-392 is stable when every item is local); tree 1 reorders
// by the larger site with the exchange sort of Sa MPIlib.f90:398-425.
std::vector<Bond> schedule_bonds(const pned_model_desc *d)
{
    std::vector<Bond> b(d->n_bonds);
    for (int i = 0; i < d->n_bonds; ++i) {
        int a = d->ipair[2 * i] - 1, c = d->ipair[2 * i + 1] - 1;
        b[i] = Bond{std::min(a, c), std::max(a, c), d->bond_type[i]};
    }
    if (d->tree == 1) {
        std::vector<int> key(b.size()), idx(b.size());
        for (size_t i = 0; i < b.size(); ++i) { key[i] = b[i].s2; idx[i] = int(i); }
        for (size_t i = 0; i + 1 < b.size(); ++i)
            for (size_t j = i + 1; j < b.size(); ++j)
                if (key[i] > key[j]) { std::swap(key[i], key[j]); std::swap(idx[i], idx[j]); }
        std::vector<Bond> o(b.size());
        for (size_t i = 0; i < b.size(); ++i) o[i] = b[idx[i]];
        b.swap(o);
    }
    return b;
}

}  // namespace

int eval_tables_on_structure(const HostProgram &S, const pned_model_desc *d, std::vector<cd> &table,
                             std::vector<cd> &dtab)
{
    if (S.q != 2 || d->q_spin != 2 || d->n_sites != S.n || d->n_bonds != S.nbond)
        return fail(PNED_EINVAL, "slot couplings: lattice differs from the slot batch's structure");
    std::vector<Bond> bonds = schedule_bonds(d);
    for (size_t i = 0; i < bonds.size(); ++i)
        if (bonds[i].s1 != S.dsite1[i] || bonds[i].s2 != S.dsite2[i])
            return fail(PNED_EINVAL, "slot couplings: bond list differs from the slot batch's structure");
    const int Q = 4;
    auto elem = [&](int t, int row, int col) -> cd {
        const size_t k = size_t(t - 1) * Q * Q + row + size_t(Q) * col;
        if (d->skip && d->skip[k]) return cd(0, 0);
        return cd(d->xlocal[k].re, d->xlocal[k].im);
    };
    table.assign(S.table.size(), cd(0, 0));
    for (size_t ti = 0; ti < S.xterms.size(); ++ti) {
        const XorTerm &term = S.xterms[ti];
        std::vector<int> deps;
        for (int k = 0; k < term.nb; ++k) deps.push_back((term.pos4 >> (8 * k)) & 0xff);
        for (int idx = 0; idx < (1 << term.nb); ++idx) {
            auto bit = [&](int site) {
                for (size_t k = 0; k < deps.size(); ++k)
                    if (deps[k] == site) return (idx >> k) & 1;
                return 0;
            };
            cd c = 0;
            for (const auto &bf : S.xcontrib[ti]) {
                const Bond &b = bonds[bf.first];
                const int st = 2 * bit(b.s2) + bit(b.s1);
                c += elem(b.t, st ^ bf.second, st);
            }
            table[term.tab + idx] = c;
        }
    }
    dtab.clear();
    for (const Bond &b : bonds)
        for (int st = 0; st < Q; ++st) dtab.push_back(elem(b.t, st, st));
    return PNED_OK;
}

int compile_program(const pned_model_desc *d, HostProgram &P)
{
    const int n = d->n_sites, q = d->q_spin, Q = q * q;
    if (n < 2 || q < 2 || d->n_bonds < 1 || !d->ipair || !d->bond_type || !d->xlocal)
        return fail(PNED_EINVAL, "pned_model_create: incomplete description");
    if (q == 2 && n > 32) return fail(PNED_EINVAL, "pned_model_create: n_sites > 32 for S = 1/2");
    double dimd = std::pow(double(q), n);
    if (dimd > 9.0e18) return fail(PNED_EINVAL, "pned_model_create: basis too large");
    if (q > 2 && (q > 4 || n > 32)) return fail(PNED_ENOTSUP, "pned_model_create: mixed radix needs q <= 4, n <= 32");
    for (int i = 0; i < 2 * d->n_bonds; ++i)
        if (d->ipair[i] < 1 || d->ipair[i] > n) return fail(PNED_EINVAL, "pned_model_create: ipair out of range");
    for (int i = 0; i < d->n_bonds; ++i) {
        if (d->bond_type[i] < 1 || d->bond_type[i] > 9) return fail(PNED_EINVAL, "pned_model_create: bond type");
        if (d->ipair[2 * i] == d->ipair[2 * i + 1]) return fail(PNED_EINVAL, "pned_model_create: bond on one site");
    }
    P = HostProgram{};
    P.n = n; P.q = q; P.nbond = d->n_bonds;
    P.dim = 1;
    for (int i = 0; i < n; ++i) P.dim *= q;
    if (d->parity_type == 0) {
        // Sz-conserving sector: mk_list12 (S1/2 parallel.f90:452-578, Sa :366-486)
        if (n > 40) return fail(PNED_ENOTSUP, "pned_model_create: sector basis above 40 sites");
        int64_t ldim = 0;
        int rc = pned_mk_list12(n, q, 0, d->total_sz, &ldim, nullptr, nullptr, nullptr);
        if (rc) return rc;
        if (ldim < 1) return fail(PNED_EINVAL, "pned_model_create: empty Sz sector");
        const int ihf0 = n / 2, ihf = (n + 1) / 2;
        int64_t nA = 1, nB = 1;
        for (int i = 0; i < ihf; ++i) nA *= q;
        for (int i = 0; i < ihf0; ++i) nB *= q;
        P.list1.resize(size_t(ldim));
        P.lin_lo.resize(size_t(std::max(nA, nB)));
        P.lin_hi.resize(size_t(std::max(nA, nB)));
        rc = pned_mk_list12(n, q, 0, d->total_sz, &ldim, P.list1.data(), P.lin_lo.data(), P.lin_hi.data());
        if (rc) return rc;
        P.sector = true;
        P.total = d->total_sz;
        P.ihf = ihf;
        P.dim = ldim;
    }
    std::vector<Bond> bonds = schedule_bonds(d);
    auto elem = [&](int t, int row, int col) -> cd {
        const size_t k = size_t(t - 1) * Q * Q + row + size_t(Q) * col;
        if (d->skip && d->skip[k]) return cd(0, 0);
        return cd(d->xlocal[k].re, d->xlocal[k].im);
    };
    for (const Bond &b : bonds) P.bond_type.push_back(b.t);
    // diagonal tables
    for (const Bond &b : bonds) {
        P.dsite1.push_back(b.s1);
        P.dsite2.push_back(b.s2);
        for (int st = 0; st < Q; ++st) {
            cd v = elem(b.t, st, st);
            if (v.imag() != 0) P.real = false;
            P.dtab.push_back(v);
        }
    }
    if (q == 2) {
        // group off-diagonal contributions by flip mask (first-appearance order)
        struct Contrib { int bond; int f; };
        std::vector<uint32_t> order;
        std::map<uint32_t, std::vector<Contrib>> groups;
        for (size_t bi = 0; bi < bonds.size(); ++bi) {
            const Bond &b = bonds[bi];
            for (int f = 1; f < 4; ++f) {
                bool any = false;
                for (int st = 0; st < 4; ++st) {
                    if (elem(b.t, st ^ f, st) == cd(0, 0)) continue;
                    any = true;
                    // the sector's Lin lookup is only defined for partners inside it
                    if (P.sector && __builtin_popcount(unsigned(st ^ f)) != __builtin_popcount(unsigned(st)))
                        return fail(PNED_EINVAL, "pned_model_create: a nonzero element changes Sz, "
                                                 "which parity_type 0 (the Sz sector basis) does not allow");
                }
                if (!any) continue;
                uint32_t mask = ((f & 1) ? (1u << b.s1) : 0u) | ((f & 2) ? (1u << b.s2) : 0u);
                if (!groups.count(mask)) order.push_back(mask);
                groups[mask].push_back(Contrib{int(bi), f});
            }
        }
        for (uint32_t mask : order) {
            const auto &cs = groups[mask];
            // split into pieces whose dependency sites number at most kMaxDeps
            size_t i = 0;
            while (i < cs.size()) {
                std::vector<int> deps;
                size_t j = i;
                for (; j < cs.size(); ++j) {
                    std::vector<int> nd = deps;
                    for (int s : {bonds[cs[j].bond].s1, bonds[cs[j].bond].s2})
                        if (std::find(nd.begin(), nd.end(), s) == nd.end()) nd.push_back(s);
                    if (int(nd.size()) > kMaxDeps) break;
                    deps = nd;
                }
                std::sort(deps.begin(), deps.end());
                XorTerm term{};
                term.xmask = mask;
                std::vector<std::pair<int, int>> contrib;
                for (size_t k = i; k < j; ++k) contrib.push_back({cs[k].bond, cs[k].f});
                P.xcontrib.push_back(contrib);
                term.nb = uint8_t(deps.size());
                term.pos4 = 0;
                for (size_t k = 0; k < deps.size(); ++k) term.pos4 |= uint32_t(deps[k]) << (8 * k);
                term.tab = uint16_t(P.table.size());
                for (int idx = 0; idx < (1 << deps.size()); ++idx) {
                    auto bit = [&](int site) {
                        for (size_t k = 0; k < deps.size(); ++k)
                            if (deps[k] == site) return (idx >> k) & 1;
                        return 0;
                    };
                    cd c = 0;
                    for (size_t k = i; k < j; ++k) {
                        const Bond &b = bonds[cs[k].bond];
                        const int st = 2 * bit(b.s2) + bit(b.s1);
                        c += elem(b.t, st ^ cs[k].f, st);
                    }
                    if (c.imag() != 0) P.real = false;
                    P.table.push_back(c);
                }
                P.xterms.push_back(term);
                i = j;
            }
        }
        if (P.xterms.size() > size_t(kMaxTerms)) return fail(PNED_ENOTSUP, "pned_model_create: too many terms");
    } else {
        int64_t pw[33];
        pw[0] = 1;
        for (int i = 1; i <= n; ++i) pw[i] = pw[i - 1] * q;
        for (const Bond &b : bonds) {
            for (int d2 = -(q - 1); d2 <= q - 1; ++d2)
                for (int d1 = -(q - 1); d1 <= q - 1; ++d1) {
                    if (d1 == 0 && d2 == 0) continue;
                    std::vector<cd> tab(Q, cd(0, 0));
                    bool any = false;
                    for (int st = 0; st < Q; ++st) {
                        const int a = st % q, c = st / q;
                        const int e1 = a + d1, e2 = c + d2;
                        if (e1 < 0 || e1 >= q || e2 < 0 || e2 >= q) continue;
                        cd v = elem(b.t, e1 + q * e2, st);
                        if (v != cd(0, 0)) { any = true; tab[st] = v; }
                    }
                    if (any && P.sector && d1 + d2 != 0)
                        return fail(PNED_EINVAL, "pned_model_create: a nonzero element changes Sz, "
                                                 "which parity_type 0 (the Sz sector basis) does not allow");
                    if (!any) continue;
                    RadixTerm t{};
                    t.offset = d1 * pw[b.s1] + d2 * pw[b.s2];
                    t.s1 = uint8_t(b.s1);
                    t.s2 = uint8_t(b.s2);
                    t.tab = uint16_t(P.table.size());
                    for (cd v : tab) {
                        if (v.imag() != 0) P.real = false;
                        P.table.push_back(v);
                    }
                    P.rterms.push_back(t);
                    P.rdelta.push_back({d1, d2});
                }
        }
        if (P.rterms.size() > size_t(kMaxTerms)) return fail(PNED_ENOTSUP, "pned_model_create: too many terms");
    }
    // the coefficient table is staged into 48 KB of shared memory per block
    if (P.table.size() > size_t(kMaxTable))
        return fail(PNED_ENOTSUP, "pned_model_create: coefficient table above 3072 complex entries");
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// Tile planner for the single-vector S = 1/2 kernel
// ---------------------------------------------------------------------------
namespace {

// Partner tiles a set of masks needs with tile bits `tm`: distinct out-of-tile parts.
int count_groups(const std::vector<uint32_t> &masks, uint32_t tm)
{
    std::vector<uint32_t> parts;
    for (uint32_t m : masks)
        if (m & ~tm) parts.push_back(m & ~tm);
    std::sort(parts.begin(), parts.end());
    return int(std::unique(parts.begin(), parts.end()) - parts.begin());
}

// Masks of the set that lie inside tile bits `tm`.
int count_inside(const std::vector<uint32_t> &masks, uint32_t tm)
{
    int c = 0;
    for (uint32_t m : masks) c += (m & ~tm) == 0;
    return c;
}

// Tile bits that hold the most masks (objective 1): the `fixed` low bits, then
// greedily the bit that brings the most masks inside (ties: the bit that the
// most masks use), then pairwise exchanges while they bring more masks
// inside, or as many with fewer partner tiles.
uint32_t tile_most_inside(const std::vector<uint32_t> &masks, int n, int target, int fixed)
{
    uint32_t tm = (1u << fixed) - 1u;
    for (int k = fixed; k < target; ++k) {
        int best = -1, bi = -1, bu = -1;
        for (int b = fixed; b < n; ++b) {
            if (tm & (1u << b)) continue;
            const int in = count_inside(masks, tm | (1u << b));
            int u = 0;
            for (uint32_t m : masks) u += (m >> b) & 1u;
            if (in > bi || (in == bi && u > bu)) { bi = in; bu = u; best = b; }
        }
        tm |= 1u << best;
    }
    int in = count_inside(masks, tm), g = count_groups(masks, tm);
    for (int round = 0; round < 32; ++round) {
        bool better = false;
        for (int a = fixed; a < n && !better; ++a) {
            if (!(tm & (1u << a))) continue;
            for (int b = fixed; b < n; ++b) {
                if (tm & (1u << b)) continue;
                const uint32_t t2 = (tm & ~(1u << a)) | (1u << b);
                const int in2 = count_inside(masks, t2), g2 = count_groups(masks, t2);
                if (in2 > in || (in2 == in && g2 < g)) { tm = t2; in = in2; g = g2; better = true; break; }
            }
        }
        if (!better) break;
    }
    return tm;
}

// Tile bits for a set of masks: the `fixed` low bits, then tbits + jb - fixed
// bits chosen to minimise the partner tiles (objective 0: greedy, then
// pairwise exchanges while they help) or to hold the most masks (objective 1,
// tile_most_inside); rows take the fixed bits and the lowest chosen ones, the
// j bits the rest.  Outer order: bits most used by out-of-tile masks first.
void choose_tile(const std::vector<uint32_t> &masks, int n, int tbits, int jb, int fixed, int objective,
                 std::vector<int> &rowpos, std::vector<int> &jpos, std::vector<int> &outer, uint32_t &tilemask)
{
    const int target = tbits + jb;
    tilemask = (1u << fixed) - 1u;
    auto usage = [&](int b) {
        int u = 0;
        for (uint32_t m : masks) if (m & (1u << b)) ++u;
        return u;
    };
    if (objective == 1) tilemask = tile_most_inside(masks, n, target, fixed);
    for (int k = __builtin_popcount(tilemask); k < target; ++k) {
        int best = -1, bestg = 1 << 30, bestu = -1;
        for (int b = fixed; b < n; ++b) {
            if (tilemask & (1u << b)) continue;
            const int g = count_groups(masks, tilemask | (1u << b));
            const int u = usage(b);
            if (g < bestg || (g == bestg && u > bestu)) { bestg = g; bestu = u; best = b; }
        }
        tilemask |= 1u << best;
    }
    int g = count_groups(masks, tilemask);
    for (int round = 0; round < 16 && objective != 1; ++round) {
        bool better = false;
        for (int a = fixed; a < n && !better; ++a) {
            if (!(tilemask & (1u << a))) continue;
            for (int b = fixed; b < n; ++b) {
                if (tilemask & (1u << b)) continue;
                const uint32_t t2 = (tilemask & ~(1u << a)) | (1u << b);
                const int g2 = count_groups(masks, t2);
                if (g2 < g) { tilemask = t2; g = g2; better = true; break; }
            }
        }
        if (!better) break;
    }
    std::vector<int> chosen;
    for (int b = 0; b < n; ++b) if (tilemask & (1u << b)) chosen.push_back(b);
    rowpos.assign(chosen.begin(), chosen.begin() + tbits);
    jpos.assign(chosen.begin() + tbits, chosen.end());
    std::vector<std::pair<int, int>> ob;
    for (int b = 0; b < n; ++b) {
        if (tilemask & (1u << b)) continue;
        int use = 0;
        for (uint32_t m : masks) if ((m & ~tilemask) && (m & (1u << b))) ++use;
        ob.push_back({-use, b});
    }
    std::sort(ob.begin(), ob.end());
    outer.clear();
    for (auto &x : ob) outer.push_back(x.second);
}

}  // namespace

int plan_tiles(const HostProgram &P, int tbits, int jb, int fixed, int window_bits, int max_passes,
               std::vector<HostProgram::TilePass> &passes, int objective)
{
    if (P.q != 2 || jb < 0 || jb > kTileMaxJB || tbits < 1 || tbits > 8 || fixed < 0 || fixed > tbits ||
        P.n < tbits + jb + 1)
        return PNED_ENOTSUP;
    const int n = P.n;
    std::vector<int> remaining(P.xterms.size());
    for (size_t i = 0; i < remaining.size(); ++i) remaining[i] = int(i);
    passes.clear();
    while (!remaining.empty()) {
        std::vector<uint32_t> rm;
        for (int i : remaining) rm.push_back(P.xterms[i].xmask);
        std::vector<int> rowpos, jpos, outer;
        uint32_t tilemask;
        choose_tile(rm, n, tbits, jb, fixed, objective, rowpos, jpos, outer, tilemask);
        uint32_t nearmask = tilemask;
        if (objective == 1) {
            // window bits one by one: the bit that brings the most masks into the pass
            // (ties: the bit that the most masks use)
            for (int k = 0; k < window_bits; ++k) {
                int best = -1, bi = -1, bu = -1;
                for (int b = 0; b < n; ++b) {
                    if (nearmask & (1u << b)) continue;
                    const int in = count_inside(rm, nearmask | (1u << b));
                    int u = 0;
                    for (uint32_t m : rm) u += (m >> b) & 1u;
                    if (in > bi || (in == bi && u > bu)) { bi = in; bu = u; best = b; }
                }
                if (best < 0) break;
                nearmask |= 1u << best;
            }
        } else {
            for (int k = 0; k < window_bits && k < int(outer.size()); ++k) nearmask |= 1u << outer[k];
        }
        std::vector<int> take, rest;
        const bool last = int(passes.size()) + 1 >= max_passes;
        for (int i : remaining) {
            if (last || (P.xterms[i].xmask & ~nearmask) == 0) take.push_back(i);
            else rest.push_back(i);
        }
        if (take.empty()) { take = rest; rest.clear(); }
        // re-plan the tile for the masks of this pass only
        std::vector<uint32_t> tm;
        for (int i : take) tm.push_back(P.xterms[i].xmask);
        choose_tile(tm, n, tbits, jb, fixed, objective, rowpos, jpos, outer, tilemask);
        HostProgram::TilePass pass;
        pass.tbits = tbits;
        pass.jb = jb;
        pass.rowpos = rowpos;
        for (int k = 0; k < kTileMaxJB; ++k) pass.jpos[k] = k < jb ? jpos[k] : 0;
        pass.outer = outer;
        auto local = [&](uint32_t m) {
            uint32_t l = 0;
            for (int k = 0; k < tbits; ++k) if (m & (1u << rowpos[k])) l |= 1u << k;
            for (int k = 0; k < jb; ++k) if (m & (1u << jpos[k])) l |= 1u << (tbits + k);
            return l;
        };
        std::vector<TileTerm> in;
        std::vector<std::pair<uint32_t, TileTerm>> out;   // (partner-tile xor, term)
        for (int i : take) {
            const XorTerm &t = P.xterms[i];
            TileTerm q{};
            q.pos4 = t.pos4;
            q.tab = t.tab;
            q.nb = t.nb;
            for (int j = 0; j < (1 << jb); ++j) {
                uint32_t bits = 0;
                for (int d = 0; d < t.nb; ++d) {
                    const int pos = (t.pos4 >> (8 * d)) & 0xff;
                    for (int k = 0; k < jb; ++k) {
                        if (pos != jpos[k]) continue;
                        q.hasj = 1;
                        if ((j >> k) & 1) bits |= 1u << d;
                    }
                }
                q.jtab |= uint64_t(bits) << (4 * j);
                q.jdep = uint8_t(q.jdep | bits);
            }
            // in-tile terms: the local xor inside the tile; out-of-tile terms: the global xor
            if ((t.xmask & ~tilemask) == 0) {
                q.mask = local(t.xmask);
                in.push_back(q);
            } else {
                q.mask = t.xmask;
                q.lmask = local(t.xmask & tilemask);
                out.push_back({t.xmask & ~tilemask, q});
            }
        }
        std::stable_sort(out.begin(), out.end(),
                         [](const std::pair<uint32_t, TileTerm> &a, const std::pair<uint32_t, TileTerm> &b) {
                             return a.first < b.first;
                         });
        pass.nin = int(in.size());
        pass.tterms = in;
        for (size_t k = 0; k < out.size(); ++k) {
            if (k == 0 || out[k].first != out[k - 1].first) {
                pass.gstart.push_back(int(pass.tterms.size()));
                pass.gxor.push_back(out[k].first);
            }
            pass.tterms.push_back(out[k].second);
        }
        pass.gstart.push_back(int(pass.tterms.size()));
        if (int(pass.gxor.size()) > kTileMaxGroups) return PNED_ENOTSUP;
        passes.push_back(pass);
        remaining = rest;
    }
    if (passes.empty()) {   // diagonal-only model: one pass with no terms
        HostProgram::TilePass pass;
        pass.tbits = tbits;
        pass.jb = jb;
        std::vector<int> rowpos, jpos, outer;
        uint32_t tilemask;
        choose_tile({}, n, tbits, jb, fixed, objective, rowpos, jpos, outer, tilemask);
        pass.rowpos = rowpos;
        for (int k = 0; k < kTileMaxJB; ++k) pass.jpos[k] = k < jb ? jpos[k] : 0;
        pass.outer = outer;
        pass.gstart.push_back(0);
        passes.push_back(pass);
    }
    return PNED_OK;
}

}  // namespace pned

// ---------------------------------------------------------------------------
// Tile planner for the mixed-radix kernel (q > 2)
// ---------------------------------------------------------------------------
namespace pned {

int plan_qtiles(const HostProgram &P, int k, int low, std::vector<QTilePass> &passes)
{
    passes.clear();
    const int n = P.n, q = P.q;
    if (q <= 2 || P.sector || k < 2 || k > kQTileMaxSites || k > n) return PNED_ENOTSUP;
    // bonds (site pairs) of the terms
    std::vector<std::pair<int, int>> bonds;
    for (const RadixTerm &t : P.rterms) {
        std::pair<int, int> b{std::min<int>(t.s1, t.s2), std::max<int>(t.s1, t.s2)};
        if (std::find(bonds.begin(), bonds.end(), b) == bonds.end()) bonds.push_back(b);
    }
    std::vector<char> covered(bonds.size(), 0);
    size_t left = bonds.size();
    auto touching = [&](int x) {
        int c = 0;
        for (size_t i = 0; i < bonds.size(); ++i)
            if (!covered[i] && (bonds[i].first == x || bonds[i].second == x)) ++c;
        return c;
    };
    while (left > 0) {
        if (int(passes.size()) >= kQTileMaxPasses) return PNED_ENOTSUP;
        // the site set grown from one seed bond: the `low` lowest sites (kept in
        // every tile for runs of q^low consecutive states), the seed's sites, then
        // the site that brings the most uncovered bonds inside (ties: the one
        // touching most uncovered bonds)
        auto grow = [&](size_t seed) {
            std::vector<int> T;
            for (int x = 0; x < low && x < k; ++x) T.push_back(x);
            for (int x : {bonds[seed].first, bonds[seed].second})
                if (int(T.size()) < k && std::find(T.begin(), T.end(), x) == T.end()) T.push_back(x);
            auto has = [&](int x) { return std::find(T.begin(), T.end(), x) != T.end(); };
            while (int(T.size()) < k) {
                int bx = -1, bg = -1, bt = -1;
                for (int x = 0; x < n; ++x) {
                    if (has(x)) continue;
                    int g = 0;
                    for (size_t i = 0; i < bonds.size(); ++i) {
                        if (covered[i]) continue;
                        const int a = bonds[i].first, b = bonds[i].second;
                        if ((a == x && (b == x || has(b))) || (b == x && has(a))) ++g;
                    }
                    const int t = touching(x);
                    if (g > bg || (g == bg && t > bt)) { bx = x; bg = g; bt = t; }
                }
                T.push_back(bx);
            }
            return T;
        };
        // every uncovered bond is tried as the seed; the set covering most wins
        std::vector<int> S;
        int best_gain = -1;
        for (size_t i = 0; i < bonds.size(); ++i) {
            if (covered[i]) continue;
            std::vector<int> T = grow(i);
            int gain = 0;
            for (size_t b = 0; b < bonds.size(); ++b)
                if (!covered[b] && std::find(T.begin(), T.end(), bonds[b].first) != T.end() &&
                    std::find(T.begin(), T.end(), bonds[b].second) != T.end())
                    ++gain;
            if (gain > best_gain) { best_gain = gain; S = T; }
        }
        auto in = [&](int x) { return std::find(S.begin(), S.end(), x) != S.end(); };
        std::sort(S.begin(), S.end());
        QTilePass pass;
        pass.sites = S;
        for (int x = 0; x < n; ++x)
            if (!in(x)) pass.outer.push_back(x);
        std::vector<int64_t> lpw(S.size() + 1, 1);
        for (size_t i = 1; i <= S.size(); ++i) lpw[i] = lpw[i - 1] * q;
        auto pos = [&](int x) { return int(std::find(S.begin(), S.end(), x) - S.begin()); };
        std::vector<char> take(bonds.size(), 0);
        for (size_t i = 0; i < bonds.size(); ++i)
            if (!covered[i] && in(bonds[i].first) && in(bonds[i].second)) take[i] = 1;
        for (size_t t = 0; t < P.rterms.size(); ++t) {
            const RadixTerm &T = P.rterms[t];
            std::pair<int, int> b{std::min<int>(T.s1, T.s2), std::max<int>(T.s1, T.s2)};
            const size_t bi = size_t(std::find(bonds.begin(), bonds.end(), b) - bonds.begin());
            if (!take[bi]) continue;
            QTileTerm qt{};
            qt.ls1 = uint8_t(pos(T.s1));
            qt.ls2 = uint8_t(pos(T.s2));
            qt.loff = int32_t(P.rdelta[t].first * lpw[qt.ls1] + P.rdelta[t].second * lpw[qt.ls2]);
            qt.tab = T.tab;
            pass.terms.push_back(qt);
        }
        for (size_t i = 0; i < bonds.size(); ++i)
            if (take[i]) { covered[i] = 1; --left; }
        passes.push_back(pass);
    }
    if (passes.empty()) {   // diagonal-only model: one pass, no terms
        QTilePass pass;
        for (int x = 0; x < k; ++x) pass.sites.push_back(x);
        for (int x = k; x < n; ++x) pass.outer.push_back(x);
        passes.push_back(pass);
    }
    return PNED_OK;
}

}  // namespace pned

// ---------------------------------------------------------------------------
// Tridiagonal routines (CPU, as in the reference)
// ---------------------------------------------------------------------------
// Tile plan of a model as the S = 1/2 tile kernels receive it (row_bits = 8:
// the single-vector kernel; log2(256 / G): the multi-vector kernel), computed on
// the host (no device work): the program's flip terms, then every pass.
extern "C" int pned_tile_plan_export(const pned_model_desc *d, int row_bits, const pned_tile_plan *plan,
                                     int64_t *out, int64_t cap, int64_t *len)
{
    using namespace pned;
    if (!d || !len || (cap > 0 && !out) || row_bits < 1 || row_bits > 8)
        return fail(PNED_EINVAL, "pned_tile_plan_export: bad arguments");
    HostProgram P;
    int rc = compile_program(d, P);
    if (rc) return rc;
    if (P.q != 2 || P.sector) return fail(PNED_ENOTSUP, "pned_tile_plan_export: tiles are planned for the S = 1/2 full basis");
    const pned_tile_plan def{-1, -1, -1, -1, -1, -1, -1, -1, -1};
    const pned_tile_plan &pl = plan ? *plan : def;
    if (pl.max_passes > kTileMaxPasses || pl.window_bits > 30 || pl.row_fixed_bits > 8 || pl.j_bits > kTileMaxJB ||
        pl.j_bits == 0 || pl.objective > 1)
        return fail(PNED_EINVAL, "pned_tile_plan_export: plan out of range");
    // the defaults of the model's own single-vector plan: with no plan, from
    // kTileBigSites sites on, the tuned tensor-copy plan (5 fixed row bits,
    // window 7, 2 passes, most terms inside the tile)
    const bool big = !plan && row_bits == 8 && P.n >= kTileBigSites;
    const int fixed = big ? 5 : std::min(row_bits, pl.row_fixed_bits >= 0 ? pl.row_fixed_bits : 8);
    const int window = big ? 7 : (pl.window_bits >= 0 ? pl.window_bits : kTileWindowBits);
    const int mp = big ? 2 : (pl.max_passes > 0 ? pl.max_passes : kTileMaxPasses);
    const int jb = pl.j_bits > 0 ? pl.j_bits : 3;
    std::vector<HostProgram::TilePass> passes;
    rc = plan_tiles(P, row_bits, jb, fixed, window, mp, passes, big ? 1 : (pl.objective > 0 ? pl.objective : 0));
    if (rc) return fail(rc, "pned_tile_plan_export: no tile plan for this model and plan");
    std::vector<int64_t> v;
    v.push_back(int64_t(P.xterms.size()));
    for (const XorTerm &t : P.xterms) v.insert(v.end(), {int64_t(t.xmask), int64_t(t.pos4), int64_t(t.tab), int64_t(t.nb)});
    v.push_back(int64_t(passes.size()));
    for (const auto &ps : passes) {
        const int ng = int(ps.gxor.size());
        v.insert(v.end(), {int64_t(ps.tbits), int64_t(ps.jb), int64_t(ps.outer.size()), int64_t(ps.tterms.size()),
                           int64_t(ps.nin), int64_t(ng)});
        for (int k = 0; k < ps.tbits; ++k) v.push_back(ps.rowpos[k]);
        for (int k = 0; k < ps.jb; ++k) v.push_back(ps.jpos[k]);
        for (int o : ps.outer) v.push_back(o);
        for (const TileTerm &t : ps.tterms)
            v.insert(v.end(), {int64_t(t.mask), int64_t(t.pos4), int64_t(t.jtab), int64_t(t.tab), int64_t(t.nb),
                               int64_t(t.hasj), int64_t(t.lmask)});
        for (int g = 0; g <= ng; ++g) v.push_back(ps.gstart[g]);
        for (int g = 0; g < ng; ++g) v.push_back(int64_t(ps.gxor[g]));
    }
    *len = int64_t(v.size());
    for (int64_t i = 0; i < std::min<int64_t>(cap, *len); ++i) out[i] = v[size_t(i)];
    return PNED_OK;
}

// Mixed-radix tile passes of k sites (the `low` lowest sites kept in every
// tile) as the tiled mixed-radix kernel receives them, computed on the host:
// the program's radix terms, which table entries are nonzero, then every pass.
extern "C" int pned_qtile_plan_export(const pned_model_desc *d, int k, int low, int64_t *out, int64_t cap,
                                      int64_t *len)
{
    using namespace pned;
    if (!d || !len || (cap > 0 && !out)) return fail(PNED_EINVAL, "pned_qtile_plan_export: bad arguments");
    HostProgram P;
    int rc = compile_program(d, P);
    if (rc) return rc;
    if (P.q <= 2 || P.sector) return fail(PNED_ENOTSUP, "pned_qtile_plan_export: mixed-radix tiles need q > 2, full basis");
    std::vector<QTilePass> passes;
    rc = plan_qtiles(P, k, low, passes);
    if (rc) return fail(rc, "pned_qtile_plan_export: no tile passes for this k");
    std::vector<int64_t> v{int64_t(P.q), int64_t(P.n), int64_t(P.rterms.size())};
    for (const RadixTerm &t : P.rterms) v.insert(v.end(), {t.offset, int64_t(t.s1), int64_t(t.s2), int64_t(t.tab)});
    v.push_back(int64_t(P.table.size()));
    for (const cd &z : P.table) v.push_back(z != cd(0, 0) ? 1 : 0);
    v.push_back(int64_t(passes.size()));
    for (const QTilePass &ps : passes) {
        v.insert(v.end(), {int64_t(ps.sites.size()), int64_t(ps.outer.size()), int64_t(ps.terms.size())});
        for (int x : ps.sites) v.push_back(x);
        for (int x : ps.outer) v.push_back(x);
        for (const QTileTerm &t : ps.terms)
            v.insert(v.end(), {int64_t(t.loff), int64_t(t.ls1), int64_t(t.ls2), int64_t(t.tab)});
    }
    *len = int64_t(v.size());
    for (int64_t i = 0; i < std::min<int64_t>(cap, *len); ++i) out[i] = v[size_t(i)];
    return PNED_OK;
}

extern "C" int pned_bisec(const double *alpha, const double *beta, int ndim, double *E, int ne, double eps)
{
    // Sturm-sequence bisection, S1/2 basic.f90:25-107
    if (ndim > 8000 || ndim < 1) return fail(PNED_EINVAL, "pned_bisec: ndim must be 1..8000");
    if (ne > ndim || ne < 0) return fail(PNED_EINVAL, "pned_bisec: ne out of range");
    double range = std::fabs(alpha[0]) + std::fabs(beta[0]);
    for (int k = 2; k <= ndim - 1; ++k)
        range = std::max(range, std::fabs(beta[k - 2]) + std::fabs(alpha[k - 1]) + std::fabs(beta[k - 1]));
    if (ndim >= 2) range = std::max(range, std::fabs(beta[ndim - 2]) + std::fabs(alpha[ndim - 1]));
    range = -range;
    std::vector<double> b2(ndim + 1, 0.0);
    for (int i = 2; i <= ndim; ++i) b2[i - 1] = beta[i - 2] * beta[i - 2];
    const double epsabs = std::fabs(range) * eps;
    for (int i = 0; i < ne; ++i) E[i] = -range;
    double b = range;
    for (int k = 1; k <= ne; ++k) {
        double a = E[k - 1];
        for (int it = 0; it < 100; ++it) {
            const double c = (a + b) / 2.0;
            if (std::fabs(a - b) < epsabs) continue;
            int numneg = 0, ipass = 0;
            double g = 1.0;
            for (int i = 1; i <= ndim; ++i) {
                if (ipass == 0) g = c - alpha[i - 1] - b2[i - 1] / g;
                else if (ipass == 1) ipass = 2;
                else { g = c - alpha[i - 1]; ipass = 0; }
                if (ipass == 0) {
                    if (g < 0.0) ++numneg;
                    if (std::fabs(g) < std::fabs(b2[i - 1] * epsabs * eps)) ipass = 1;
                }
            }
            numneg = ndim - numneg;
            if (numneg < k) b = c;
            else {
                a = c;
                for (int i = k; i <= std::min(numneg, ne); ++i) E[i - 1] = c;
            }
        }
    }
    return PNED_OK;
}

extern "C" int pned_vec12(const double *alpha, const double *beta, const double *E, int ndim, int nvec, double *v)
{
    // inverse iteration on the tridiagonal matrix, S1/2 basic.f90:112-213
    if (ndim < 1 || nvec < 1 || !v) return fail(PNED_EINVAL, "pned_vec12: bad arguments");
    std::vector<double> di(ndim + 3), bl(ndim + 3), bu(ndim + 3), bv(ndim + 3), cm(ndim + 3);
    std::vector<int> lex(ndim + 3);
    auto V = [&](int j, int k) -> double & { return v[size_t(k - 1) * ndim + j - 1]; };
    int km = 1;
    for (int k = 1; k <= nvec; ++k) {
        for (int j = 1; j <= ndim; ++j) {
            di[j] = E[k - 1] - alpha[j - 1];
            bl[j] = -beta[j - 1];
            bu[j] = -beta[j - 1];
        }
        bu[ndim + 1] = 0.0;
        for (int j = 1; j <= ndim - 1; ++j) {
            if (std::fabs(di[j]) > std::fabs(bl[j])) {
                lex[j] = 0;
                if (std::fabs(di[j]) < 1.e-13) di[j] = 1.e-13;
                cm[j + 1] = bl[j] / di[j];
                di[j + 1] = di[j + 1] - cm[j + 1] * bu[j];
                bv[j] = 0.0;
            } else {
                lex[j] = 1;
                cm[j + 1] = di[j] / bl[j];
                di[j] = bl[j];
                const double s = bu[j];
                bu[j] = di[j + 1];
                bv[j] = bu[j + 1];
                di[j + 1] = s - cm[j + 1] * bu[j];
                bu[j + 1] = -cm[j + 1] * bv[j];
            }
        }
        if (std::fabs(di[ndim]) < 1.e-13) di[ndim] = 1.e-13;
        for (int j = 1; j <= ndim; ++j) V(j, k) = 1.0 / (double(j) * 5.0);
        if (k == 1) km = k;
        else if (std::fabs(E[k - 1] - E[km - 1]) > 1.e-13) km = k;
        else
            for (int i = km; i <= k - 1; ++i) {
                double prd = 0.0;
                for (int j = 1; j <= ndim; ++j) prd += V(j, i) * V(j, k);
                for (int j = 1; j <= ndim; ++j) V(j, k) -= prd * V(j, i);
            }
        for (int l = 1; l <= k - km + 3; ++l) {
            if (l != 1 || k != km)
                for (int j = 1; j <= ndim - 1; ++j) {
                    if (lex[j] == 0) V(j + 1, k) -= cm[j + 1] * V(j, k);
                    else {
                        const double s = V(j, k);
                        V(j, k) = V(j + 1, k);
                        V(j + 1, k) = s - cm[j + 1] * V(j, k);
                    }
                }
            for (int j = ndim; j >= 1; --j) {
                double s = V(j, k);
                if (j <= ndim - 1) s -= bu[j] * V(j + 1, k);
                if (j <= ndim - 2) s -= bv[j] * V(j + 2, k);
                V(j, k) = s / di[j];
            }
            double dn = 0.0;
            for (int j = 1; j <= ndim; ++j) dn += V(j, k) * V(j, k);
            if (dn > 1.e-13) dn = 1.0 / std::sqrt(dn);
            for (int j = 1; j <= ndim; ++j) V(j, k) *= dn;
        }
    }
    return PNED_OK;
}

extern "C" int pned_exec_renbun(int i_range, int s_maxitr, double split, double ene, double epsln,
                                const double *salpha, const double *sbeta, double *w, int *conv, double *dsf)
{
    // modified-Lentz continued fraction per omega, S1/2 DSF.f90:263-334
    if (i_range < 1 || s_maxitr < 2) return fail(PNED_EINVAL, "pned_exec_renbun: bad sizes");
#pragma omp parallel for schedule(static, 1)
    for (int j = 1; j <= i_range; ++j) {
        const double omega = double(j - 1) * split;
        w[j - 1] = omega;
        int ic = 0;
        double xr = 1.0e-10, xi = 1.0e-10, cr = xr, ci = xi, dr = 0.0, di = 0.0;
        for (int m = 1; m <= s_maxitr - 1; ++m) {
            const double f1 = omega + ene - salpha[m - 1];
            const double f2 = -std::pow(sbeta[m - 1], 2.0);
            const double xr1 = xr, xi1 = xi;
            dr = dr * f2 + f1;
            di = di * f2 + epsln;
            double dd = dr * dr + di * di;
            if (dd == 0.0) { dr = 0.5e-28; di = 0.5e-28; }
            double c = cr * cr + ci * ci;
            cr = cr * f2 / c + f1;
            ci = -ci * f2 / c + epsln;
            c = cr * cr + ci * ci;
            if (c == 0.0) { cr = 0.5e-28; ci = 0.5e-28; }
            dd = dr * dr + di * di;
            dr = dr / dd;
            di = -di / dd;
            const double dlr = cr * dr - ci * di, dli = ci * dr + cr * di;
            xr = xr1 * dlr - xi1 * dli;
            xi = xr1 * dli + xi1 * dlr;
            if ((dlr - 1.0) * (dlr - 1.0) + dli * dli < 0.5e-28) { ic = m; break; }
        }
        if (conv) conv[j - 1] = ic;
        dsf[j - 1] = xi;
    }
    return PNED_OK;
}

extern "C" int pned_normalize_dsf(int i_range, double split, double sq_re, double *dsf)
{
    // trapezoid normalisation to S(q), S1/2 DSF.f90:337-351
    if (i_range < 2 || !dsf) return fail(PNED_EINVAL, "pned_normalize_dsf: bad arguments");
    double sum = 0.0;
    for (int i = 2; i <= i_range; ++i) sum += 0.5 * split * (dsf[i - 1] + dsf[i - 2]);
    for (int i = 0; i < i_range; ++i) dsf[i] = sq_re / sum * dsf[i];
    return PNED_OK;
}

extern "C" const char *pned_last_error(void) { return pned::g_err.c_str(); }
extern "C" int pned_abi_version(void) { return PNED_ABI_VERSION; }
