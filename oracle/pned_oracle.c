/*
 * pned_oracle.c -- CPU restatement of pNED's single-rank (lnp = 1) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or as the timed CPU baseline.  The product library
 * (pned_b200/libpned_gpu.so) never links or calls it.
 *
 * Parity status: the reference is Fortran 90 + MPI and no Fortran compiler
 * exists in this image, so the reference itself cannot be run here, and the
 * reference ships no tests, fixtures or golden vectors.  Parity is therefore
 * "unpinned" by the reference; this restatement is pinned instead by
 * project-written checks (dense FP64 diagonalisation of the same local
 * matrices, column-by-column H^T checks, analytic known answers for small
 * Heisenberg/Kitaev clusters) in tests/test_oracle.py.
 *
 * Every routine cites the reference routine it restates.  Paths are relative
 * to the pNED project root:
 *   S_one_half/Hybrid_TPS_*.f90     (S = 1/2 tree, bit arithmetic)
 *   S_arbitrary/Hybrid_TPS9_*.f90   (any S, base q = 2S+1 digits)
 *
 * Conventions kept from the reference:
 *   - local matrices xlocal_Ham(0:Q-1,0:Q-1,9) are column-major per bond type,
 *     element (row, col, type) at row + Q*col + Q*Q*(type-1), Q = q*q, with
 *     row = target pair state and col = current pair state;
 *   - the pair state of bond (s1 < s2) is d(s2)*q + d(s1);
 *   - H.v accumulates v0(l0) += X(target, current) * v1(partner), i.e. it
 *     applies H^T (S_one_half/Hybrid_TPS_parallel.f90:358);
 *   - basis index = state integer; bit (digit) j is site j+1.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef double _Complex cplx;

#define OR_OK 0
#define OR_EINVAL 1
#define OR_EBREAKDOWN 2
#define OR_ENOMEM 3

/* ------------------------------------------------------------------------ */
/* Coupling slots, in the order of the module variables of                  */
/* S_one_half/Hybrid_TPS_params.f90:17-26 (and S_arbitrary twin :12-21).    */
/* ------------------------------------------------------------------------ */
enum {
    C_J1, C_K1, C_I11, C_I12, C_J1p, C_K1p, C_J1pp, C_K1pp, C_I11p, C_I12p,
    C_I11pp, C_I12pp, C_J2, C_K2, C_I21, C_I22, C_J3, C_K3, C_RATIO_L, C_NCPL
};

/* 3x3 coupling matrices J1x..J3z of set_xlocal_Ham, index [a][b], a,b = x,y,z */
static void coupling_mats(const double *c, int tree_sa, cplx J[7][3][3])
{
    /* S_one_half/Hybrid_TPS_params.f90:1441-1465,
       S_arbitrary/Hybrid_TPS9_params.f90:1497-1521 (rl placement differs) */
    double rl = c[C_RATIO_L];
    memset(J, 0, sizeof(cplx) * 7 * 9);
    cplx J11 = c[C_J1], J12 = c[C_J1p], J13 = c[C_J1pp];
    cplx K11 = c[C_K1], K12 = c[C_K1p];
    cplx J2 = c[C_J2], J3 = c[C_J3], K2 = c[C_K2];
    cplx I111 = c[C_I11], I112 = c[C_I12], I121 = c[C_I11p], I122 = c[C_I12p];
    cplx I132 = c[C_I12pp], I211 = c[C_I21], I212 = c[C_I22];
    /* J1z = J[2] */
    if (!tree_sa) {
        J[2][0][0] = J11 * rl;  J[2][0][1] = I111 * rl; J[2][0][2] = I112 * rl;
        J[2][1][0] = I111 * rl; J[2][1][1] = J11 * rl;  J[2][1][2] = I112 * rl;
    } else {
        J[2][0][0] = J11;       J[2][0][1] = I111 * rl; J[2][0][2] = I112 * rl;
        J[2][1][0] = I111 * rl; J[2][1][1] = J11;       J[2][1][2] = I112 * rl;
    }
    J[2][2][0] = I112 * rl; J[2][2][1] = I112 * rl; J[2][2][2] = K11;
    /* J1x = J[0] */
    J[0][0][0] = K12;       J[0][0][1] = I132 * rl; J[0][0][2] = I122 * rl;
    J[0][1][0] = I132 * rl; J[0][1][1] = tree_sa ? J13 : J13 * rl; J[0][1][2] = I121 * rl;
    J[0][2][0] = I122 * rl; J[0][2][1] = I121 * rl; J[0][2][2] = tree_sa ? J12 : J12 * rl;
    /* J1y = J[1] */
    J[1][0][0] = tree_sa ? J13 : J13 * rl; J[1][0][1] = I132 * rl; J[1][0][2] = I121 * rl;
    J[1][1][0] = I132 * rl; J[1][1][1] = K12;       J[1][1][2] = I122 * rl;
    J[1][2][0] = I121 * rl; J[1][2][1] = I122 * rl; J[1][2][2] = tree_sa ? J12 : J12 * rl;
    /* J2x, J2y, J2z = J[3], J[4], J[5] */
    J[3][0][0] = K2 * rl;   J[3][0][1] = I211 * rl; J[3][0][2] = I212 * rl;
    J[3][1][0] = I211 * rl; J[3][1][1] = J2 * rl;   J[3][1][2] = I212 * rl;
    J[3][2][0] = I212 * rl; J[3][2][1] = I212 * rl; J[3][2][2] = J2 * rl;
    J[4][0][0] = J2 * rl;   J[4][0][1] = I211 * rl; J[4][0][2] = I212 * rl;
    J[4][1][0] = I211 * rl; J[4][1][1] = K2 * rl;   J[4][1][2] = I212 * rl;
    J[4][2][0] = I212 * rl; J[4][2][1] = I212 * rl; J[4][2][2] = J2 * rl;
    J[5][0][0] = J2 * rl;   J[5][0][1] = I211 * rl; J[5][0][2] = I212 * rl;
    J[5][1][0] = I211 * rl; J[5][1][1] = J2 * rl;   J[5][1][2] = I212 * rl;
    J[5][2][0] = I212 * rl; J[5][2][1] = I212 * rl; J[5][2][2] = K2 * rl;
    /* J3z = J[6] */
    J[6][0][0] = J3 * rl; J[6][1][1] = J3 * rl; J[6][2][2] = J3 * rl;
}

/* Single-site spin matrices s[a][i][j], a = x,y,z, i,j digits (q x q). */
static void spin_mats(int q, int tree_sa, cplx *s /* [3][q][q] */)
{
    memset(s, 0, sizeof(cplx) * 3 * q * q);
#define S(a, i, j) s[(a) * q * q + (i) * q + (j)]
    if (!tree_sa) {
        /* S_one_half/Hybrid_TPS_params.f90:1434-1439: bit 0 = up */
        S(0, 0, 1) = 0.5; S(0, 1, 0) = 0.5;
        S(1, 0, 1) = -0.5 * I; S(1, 1, 0) = 0.5 * I;
        S(2, 0, 0) = 0.5; S(2, 1, 1) = -0.5;
    } else {
        /* S_arbitrary/Hybrid_TPS9_params.f90:1479-1494: digit d <-> m = d - S */
        double ss = 0.5 * (double)(q - 1);
        cplx *su = calloc((size_t)q * q, sizeof(cplx));
        cplx *sd = calloc((size_t)q * q, sizeof(cplx));
        for (int i = 0; i <= q - 2; ++i) {
            double sm = (double)i - ss;
            su[i * q + i + 1] = sqrt((ss - sm) * (ss + sm + 1.0));
        }
        for (int i = 1; i <= q - 1; ++i) {
            double sm = (double)i - ss;
            sd[i * q + i - 1] = sqrt((ss + sm) * (ss - sm + 1.0));
        }
        for (int i = 0; i < q; ++i) S(2, i, i) = (double)i - ss;
        for (int i = 0; i < q * q; ++i) {
            s[0 * q * q + i] = 0.5 * (su[i] + sd[i]);
            s[1 * q * q + i] = (-0.5 * I) * (su[i] - sd[i]);
        }
        free(su);
        free(sd);
    }
#undef S
}

/*
 * set_xlocal_Ham, matrix part.  S_one_half/Hybrid_TPS_params.f90:1388-1563
 * (tree_sa = 0, q must be 2) and S_arbitrary/Hybrid_TPS9_params.f90:1412-1602
 * (tree_sa = 1).  X is [9][Q][Q] column-major per type (see header).
 */
int oracle_xlocal_matrices(int q, int tree_sa, const double *cpl, int simple, cplx *X)
{
    if (q < 2 || (!tree_sa && q != 2)) return OR_EINVAL;
    int Q = q * q;
    cplx *s = malloc(sizeof(cplx) * 3 * q * q);
    cplx *ss = malloc(sizeof(cplx) * 9 * Q * Q); /* s_ab(row, col), ab = 3a+b */
    cplx J[7][3][3];
    spin_mats(q, tree_sa, s);
    coupling_mats(cpl, tree_sa, J);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int j2 = 0; j2 < q; ++j2)
                for (int i2 = 0; i2 < q; ++i2)
                    for (int j1 = 0; j1 < q; ++j1)
                        for (int i1 = 0; i1 < q; ++i1)
                            ss[(3 * a + b) * Q * Q + (q * j1 + i1) + Q * (q * j2 + i2)] =
                                s[a * q * q + i1 * q + i2] * s[b * q * q + j1 * q + j2];
    /* Fortran sums J(1,1)*sxx + J(1,2)*sxy + J(1,3)*sxz + J(2,1)*syx + ... in
       this order (params.f90:1519-1545); ss index 3a+b follows the same order. */
    memset(X, 0, sizeof(cplx) * 9 * Q * Q);
    for (int i = 0; i < Q; ++i)
        for (int j = 0; j < Q; ++j) {
            cplx x[7];
            for (int t = 0; t < 7; ++t) {
                cplx acc = J[t][0][0] * ss[0 * Q * Q + j + Q * i];
                for (int ab = 1; ab < 9; ++ab)
                    acc = acc + J[t][ab / 3][ab % 3] * ss[ab * Q * Q + j + Q * i];
                x[t] = acc;
            }
            cplx x1x = x[0], x1y = x[1], x1z = x[2], x2x = x[3], x2y = x[4], x2z = x[5], x3z = x[6];
            cplx x3x = x3z, x3y = x3z;
            if (!tree_sa) {
                if (simple == 3) { x2x = x2z; x2y = x2z; }
            } else {
                if (simple == 3 || simple == 4) {
                    if (simple == 3) { x2x = x2z; x2y = x2z; }
                } else {
                    x2x = 0; x2y = 0;
                }
            }
            cplx xt[9] = {x1x, x1y, x1z, x2x, x2y, x2z, x3x, x3y, x3z};
            for (int t = 0; t < 9; ++t) X[t * Q * Q + j + Q * i] += xt[t];
        }
    free(s);
    free(ss);
    return OR_OK;
}

/*
 * Zeeman-field extension (not in the reference, which has no field term):
 * adds -(1/coord) * sum_a h_a (S^a x 1 + 1 x S^a) to the nearest-neighbour
 * bond types 1..3, so that a lattice where every site has `coord` such bonds
 * carries H_Z = -sum_i h.S_i exactly, using the tree's own spin matrices.
 */
int oracle_add_field(int q, int tree_sa, const double *h, double coord, cplx *X)
{
    int Q = q * q;
    cplx *s = malloc(sizeof(cplx) * 3 * q * q);
    spin_mats(q, tree_sa, s);
    for (int t = 0; t < 3; ++t)
        for (int j2 = 0; j2 < q; ++j2)
            for (int i2 = 0; i2 < q; ++i2)
                for (int j1 = 0; j1 < q; ++j1)
                    for (int i1 = 0; i1 < q; ++i1) {
                        cplx acc = 0;
                        for (int a = 0; a < 3; ++a) {
                            if (j1 == j2) acc += h[a] * s[a * q * q + i1 * q + i2];
                            if (i1 == i2) acc += h[a] * s[a * q * q + j1 * q + j2];
                        }
                        X[t * Q * Q + (q * j1 + i1) + Q * (q * j2 + i2)] -= acc / coord;
                    }
    free(s);
    return OR_OK;
}

/*
 * Parity type and skip mask llocal_Ham (plus plocal_Ham for the any-S tree).
 * S_one_half/Hybrid_TPS_params.f90:1565-1595,
 * S_arbitrary/Hybrid_TPS9_params.f90:1604-1655.
 * skip has the layout of X; 1 = .true. (element skipped).
 */
int oracle_parity_skip(int q, int tree_sa, const cplx *X, unsigned char *skip,
                       unsigned char *pskip, int *parity_type)
{
    const double eps = .5e-28;
    int Q = q * q;
    int pt = 0;
#define XA(r, c, t) X[(r) + Q * (c) + Q * Q * (t)]
#define AB2(z) fabs(creal(conj(z) * (z)))
    if (!tree_sa) {
        for (int t = 0; t < 9; ++t) {
            if (AB2(XA(1, 0, t)) > eps) pt |= 2;
            if (AB2(XA(2, 0, t)) > eps) pt |= 2;
            if (AB2(XA(3, 0, t)) > eps) pt |= 1;
        }
        for (int i = 0; i < 9 * Q * Q; ++i) skip[i] = 1;
        if (pt == 0) {
            for (int t = 0; t < 9; ++t) {
                skip[0 + Q * 0 + Q * Q * t] = 0;
                skip[1 + Q * 1 + Q * Q * t] = 0;
                skip[1 + Q * 2 + Q * Q * t] = 0;
                skip[2 + Q * 1 + Q * Q * t] = 0;
                skip[2 + Q * 2 + Q * Q * t] = 0;
                skip[3 + Q * 3 + Q * Q * t] = 0;
            }
        } else {
            for (int t = 0; t < 9; ++t)
                for (int i = 0; i < Q; ++i)
                    for (int k = 0; k < Q; ++k) {
                        if (AB2(XA(k, i, t)) > eps) skip[k + Q * i + Q * Q * t] = 0;
                        if (k == i) skip[k + Q * i + Q * Q * t] = 0;
                    }
        }
    } else {
        for (int t = 0; t < 9; ++t)
            for (int j = 0; j < Q; ++j)
                for (int i = j; i < Q; ++i) {
                    int s1 = j % q, s2 = j / q, s3 = i % q, s4 = i / q;
                    if (s1 + s2 - (s3 + s4) != 0)
                        if (AB2(XA(i, j, t)) > eps) pt |= 1;
                }
        for (int i = 0; i < 9 * Q * Q; ++i) skip[i] = 1;
        for (int t = 0; t < 9; ++t)
            for (int j = 0; j < Q; ++j)
                for (int i = 0; i < Q; ++i) {
                    int s1 = j % q, s2 = j / q, s3 = i % q, s4 = i / q;
                    if (pt == 0) {
                        if (s1 + s2 - (s3 + s4) == 0) skip[i + Q * j + Q * Q * t] = 0;
                    } else {
                        if (AB2(XA(i, j, t)) > eps) skip[i + Q * j + Q * Q * t] = 0;
                    }
                    if (i == j) skip[i + Q * j + Q * Q * t] = 0;
                }
        if (pskip) {
            for (int t = 0; t < 9; ++t)
                for (int i2 = 0; i2 < Q; ++i2) {
                    int check = 1;
                    for (int i1 = 0; i1 < Q; ++i1) {
                        int j2 = (i1 + i2) % Q;
                        if (AB2(XA(i1, j2, t)) > eps) check = 0;
                    }
                    pskip[i2 + Q * t] = check ? 0 : 1;
                }
        }
    }
#undef XA
#undef AB2
    *parity_type = pt;
    return OR_OK;
}

/*
 * change_to_TPS_hamiltonian as the reference does it: returns L (=
 * localHam_max*ibond) and overwrites X with l_b*1 - X.
 * S_one_half/Hybrid_TPS_params.f90:1600-1623 (l_b = sum_t sum_k |X_kk|^2 / c),
 * S_arbitrary/Hybrid_TPS9_params.f90:1660-1686 (only diagonal entries 0..3
 * are used and shifted, also for q = 3).
 */
double oracle_tps_reference(int q, int tree_sa, int nbond, double c_count, cplx *X)
{
    int Q = q * q;
    double lmax = 0.0;
    if (!tree_sa) {
        for (int t = 0; t < 9; ++t)
            for (int i = 0; i < 4; ++i)
                lmax += fabs(creal(conj(X[i + Q * i + Q * Q * t]) * X[i + Q * i + Q * Q * t]));
        lmax = lmax / c_count;
    } else {
        double ss = 0.25 * (double)((q - 1) * (q - 1));
        for (int t = 0; t < 9; ++t)
            for (int i = 0; i < 4; ++i)
                lmax += ss * sqrt(fabs(creal(conj(X[i + Q * i + Q * Q * t]) * X[i + Q * i + Q * Q * t])));
        lmax = 2.0 * lmax / c_count / (double)Q;
    }
    for (int i = 0; i < 9 * Q * Q; ++i) X[i] = -X[i];
    for (int t = 0; t < 9; ++t)
        for (int i = 0; i < 4; ++i) X[i + Q * i + Q * Q * t] = lmax + X[i + Q * i + Q * Q * t];
    return lmax * (double)nbond;
}

/* Explicit-shift TPS Hamiltonian: X <- (L/nbond)*1 - X on every diagonal entry. */
void oracle_tps_explicit(int q, int nbond, double L, cplx *X)
{
    int Q = q * q;
    double lb = L / (double)nbond;
    for (int i = 0; i < 9 * Q * Q; ++i) X[i] = -X[i];
    for (int t = 0; t < 9; ++t)
        for (int i = 0; i < Q; ++i) X[i + Q * i + Q * Q * t] = lb + X[i + Q * i + Q * Q * t];
}

/* ------------------------------------------------------------------------ */
/* Model: items of the lnp = 1 schedule                                     */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, q, Q, nbond, nitem;
    int tree_sa;
    int parity_type;
    int64_t ldim;
    int ihf, ihf0;
    int64_t irght, ilft;       /* S1/2: masks; Sa: q^ihf for both */
    int *it_s1, *it_s2, *it_t, *it_e; /* per item: site1, site2 (0-based), type (1..9), element */
    cplx *X;
    unsigned char *skip;
    int64_t *list1;            /* NULL for the full basis (list1(i) = i-1) */
    int64_t *list3a, *list3b;  /* Lin tables (1-based values as in Fortran) */
    int64_t nlist3;
} omodel;

static int64_t ipow(int64_t b, int e) { int64_t r = 1; while (e-- > 0) r *= b; return r; }

/*
 * Sa bond reordering of make_cpu_list2 (S_arbitrary/Hybrid_TPS9_MPIlib.f90:136-154)
 * using its exchange sort sort_list (:398-425) keyed on the larger site.
 */
static void sa_sort_bonds(int nb, int *p1, int *p2, int *ty)
{
    int *tp1 = malloc(sizeof(int) * nb), *tp2 = malloc(sizeof(int) * nb), *tt = malloc(sizeof(int) * nb);
    int *key = malloc(sizeof(int) * nb), *srt = malloc(sizeof(int) * nb);
    for (int i = 0; i < nb; ++i) {
        int a = p1[i], b = p2[i];
        tp1[i] = a < b ? a : b;
        tp2[i] = a < b ? b : a;
        tt[i] = ty[i];
        key[i] = tp2[i];
        srt[i] = i;
    }
    for (int i = 0; i < nb - 1; ++i)
        for (int j = i + 1; j < nb; ++j)
            if (key[i] > key[j]) {
                int k = key[i]; key[i] = key[j]; key[j] = k;
                k = srt[i]; srt[i] = srt[j]; srt[j] = k;
            }
    for (int i = 0; i < nb; ++i) {
        p1[i] = tp1[srt[i]];
        p2[i] = tp2[srt[i]];
        ty[i] = tt[srt[i]];
    }
    free(tp1); free(tp2); free(tt); free(key); free(srt);
}

/*
 * mk_list12 for one rank (lnp = 1, Iam = 0, p_bit = 0):
 * S_one_half/Hybrid_TPS_parallel.f90:452-578, S_arbitrary/Hybrid_TPS9_parallel.f90:366-486.
 * With parity_type /= 0 every state is kept (full basis); with parity_type == 0
 * the states whose digit sum is tot_sz (+is) are kept in ascending order.
 * Writes ldim; list1/list3 arrays are allocated when out pointers are given.
 */
int64_t oracle_mk_list12(int n, int q, int parity_type, int tot_sz, int is_shift,
                         int64_t **list1_out, int64_t **l3a_out, int64_t **l3b_out, int64_t *nl3_out)
{
    int b_bit = n;
    int ihf0 = b_bit / 2, ihf = (b_bit + 1) / 2;
    int64_t nA = ipow(q, ihf), nB = ipow(q, ihf0);
    int *szb = malloc(sizeof(int) * nA);
    for (int64_t j = 0; j < nA; ++j) {
        int64_t st = j; int bsz = 0;
        for (int i = 0; i < ihf; ++i) { bsz += (int)(st % q); st /= q; }
        szb[j] = bsz;
    }
    int64_t icnt = 0;
    for (int64_t i2 = 0; i2 < nB; ++i2)
        for (int64_t i1 = 0; i1 < nA; ++i1) {
            int isz = szb[i1] + szb[i2];
            if (parity_type == 0 && isz != is_shift + tot_sz) continue;
            icnt++;
        }
    int64_t ldim = icnt;
    if (list1_out) {
        int64_t nmax = nA > nB ? nA : nB;
        int64_t *list1 = malloc(sizeof(int64_t) * (ldim > 0 ? ldim : 1));
        int64_t *l3a = malloc(sizeof(int64_t) * nmax), *l3b = malloc(sizeof(int64_t) * nmax);
        for (int64_t i = 0; i < nmax; ++i) { l3a[i] = -1; l3b[i] = -1; }
        int64_t ja = 0, jb = 0, ibpatn = 0;
        icnt = 0;
        for (int64_t i2 = 0; i2 < nB; ++i2)
            for (int64_t i1 = 0; i1 < nA; ++i1) {
                int isz = szb[i1] + szb[i2];
                if (parity_type == 0 && isz != tot_sz + is_shift) continue;
                icnt++;
                int64_t ia = i1, ib = i2;
                if (ib == ibpatn) ja = ja + 1;
                else { ibpatn = ib; ja = 1; jb = icnt - 1; }
                list1[icnt - 1] = ib * nA + ia;
                l3a[ia] = ja;
                l3b[ib] = jb;
            }
        *list1_out = list1; *l3a_out = l3a; *l3b_out = l3b; *nl3_out = nmax;
    }
    free(szb);
    return ldim;
}

void oracle_free(void *p) { free(p); }

/*
 * Builds the model.  bonds: p1,p2 1-based sites as in ipair, ty bond types 1..9.
 * The S1/2 schedule keeps ipair order with (min,max) sites and elements 0..3
 * (make_cpu_list2, S_one_half/Hybrid_TPS_MPIlib.f90:139-209; sort_list keeps
 * the order when every item is local); the Sa schedule first reorders bonds
 * by their larger site.
 */
omodel *oracle_model_create(int n, int q, int tree_sa, int nbond, const int *ipair /* 2*nbond */,
                            const int *ibond_type, const cplx *X, const unsigned char *skip,
                            int parity_type, int tot_sz, int is_shift)
{
    omodel *m = calloc(1, sizeof(omodel));
    m->n = n; m->q = q; m->Q = q * q; m->nbond = nbond; m->tree_sa = tree_sa;
    m->parity_type = parity_type;
    int Q = m->Q;
    m->X = malloc(sizeof(cplx) * 9 * Q * Q);
    memcpy(m->X, X, sizeof(cplx) * 9 * Q * Q);
    m->skip = malloc(9 * Q * Q);
    memcpy(m->skip, skip, 9 * Q * Q);
    int *p1 = malloc(sizeof(int) * nbond), *p2 = malloc(sizeof(int) * nbond), *ty = malloc(sizeof(int) * nbond);
    for (int i = 0; i < nbond; ++i) { p1[i] = ipair[2 * i]; p2[i] = ipair[2 * i + 1]; ty[i] = ibond_type[i]; }
    if (tree_sa) sa_sort_bonds(nbond, p1, p2, ty);
    m->nitem = nbond * Q;
    m->it_s1 = malloc(sizeof(int) * m->nitem); m->it_s2 = malloc(sizeof(int) * m->nitem);
    m->it_t = malloc(sizeof(int) * m->nitem); m->it_e = malloc(sizeof(int) * m->nitem);
    int k = 0;
    for (int i = 0; i < nbond; ++i) {
        int a = p1[i] - 1, b = p2[i] - 1;
        int s1 = a < b ? a : b, s2 = a < b ? b : a;
        for (int e = 0; e < Q; ++e) {
            m->it_s1[k] = s1; m->it_s2[k] = s2; m->it_t[k] = ty[i]; m->it_e[k] = e;
            ++k;
        }
    }
    free(p1); free(p2); free(ty);
    /* PNED_ORACLE_ITEM_ORDER=reverse sums the items in the reverse order.  The
       order in which p_mltply_v3 sums its items is what the reference's rank
       decomposition changes (make_cpu_list2 groups the items by class,
       S_one_half/Hybrid_TPS_MPIlib.f90:104-341); a test uses it to measure how
       far long chains depend on that order.  Unset: the lnp = 1 order. */
    const char *ord = getenv("PNED_ORACLE_ITEM_ORDER");
    if (ord && strcmp(ord, "reverse") == 0) {
        for (int i = 0, j = m->nitem - 1; i < j; ++i, --j) {
            int t;
            t = m->it_s1[i]; m->it_s1[i] = m->it_s1[j]; m->it_s1[j] = t;
            t = m->it_s2[i]; m->it_s2[i] = m->it_s2[j]; m->it_s2[j] = t;
            t = m->it_t[i]; m->it_t[i] = m->it_t[j]; m->it_t[j] = t;
            t = m->it_e[i]; m->it_e[i] = m->it_e[j]; m->it_e[j] = t;
        }
    }
    m->ihf0 = n / 2; m->ihf = (n + 1) / 2;
    if (!tree_sa) {
        int64_t ihfbit = (int64_t)1 << m->ihf;
        m->irght = ihfbit - 1;
        m->ilft = (((int64_t)1 << n) - 1) ^ m->irght;
    } else {
        m->irght = ipow(q, m->ihf);
        m->ilft = ipow(q, m->ihf);
    }
    if (parity_type != 0) {
        m->ldim = ipow(q, n);
        m->list1 = NULL;
    } else {
        m->ldim = oracle_mk_list12(n, q, parity_type, tot_sz, is_shift, &m->list1, &m->list3a, &m->list3b, &m->nlist3);
    }
    return m;
}

int64_t oracle_model_ldim(const omodel *m) { return m->ldim; }
int oracle_model_nitem(const omodel *m) { return m->nitem; }
void oracle_model_item(const omodel *m, int k, int *s1, int *s2, int *t, int *e)
{
    *s1 = m->it_s1[k]; *s2 = m->it_s2[k]; *t = m->it_t[k]; *e = m->it_e[k];
}

void oracle_model_destroy(omodel *m)
{
    if (!m) return;
    free(m->X); free(m->skip); free(m->it_s1); free(m->it_s2); free(m->it_t); free(m->it_e);
    free(m->list1); free(m->list3a); free(m->list3b);
    free(m);
}

static inline int64_t lin_index(const omodel *m, int64_t it0)
{
    /* returns the 0-based index of state it0 (list_lib lookup, 1-based in Fortran) */
    if (!m->list1) return it0;
    int64_t it1, it2;
    if (!m->tree_sa) { it1 = it0 & m->irght; it2 = (it0 & m->ilft) >> m->ihf; }
    else { it1 = it0 % m->irght; it2 = it0 / m->ilft; }
    return m->list3a[it1] + m->list3b[it2] - 1;
}

/*
 * One item (bond x target element) of H.v over the whole local basis.
 * S_one_half/Hybrid_TPS_parallel.f90:415-440 (case 3, the only case when
 * lnp = 1) and S_arbitrary/Hybrid_TPS9_parallel.f90:339-353.
 */
static cplx hv_item(const omodel *m, int k, const cplx *v1, const cplx *vt, cplx *v0, double eperbd)
{
    const int q = m->q, Q = m->Q;
    const int s1 = m->it_s1[k], s2 = m->it_s2[k], t = m->it_t[k] - 1, ml = m->it_e[k];
    const cplx *hb = m->X + (size_t)Q * Q * t;
    const unsigned char *sk = m->skip + (size_t)Q * Q * t;
    const double Keperbd = -eperbd;
    const int64_t ldim = m->ldim;
    double pr = 0.0, pi = 0.0;
    if (!m->tree_sa) {
        const int64_t is1 = (int64_t)1 << s1, is2 = (int64_t)1 << s2;
        const int l1 = ml & 1, l2 = (ml >> 1) & 1;
#pragma omp parallel for reduction(+ : pr, pi) schedule(static)
        for (int64_t l0 = 0; l0 < ldim; ++l0) {
            int64_t it0 = m->list1 ? m->list1[l0] : l0;
            int ibit1 = (int)((it0 & is1) >> s1);
            int ibit2 = (int)((it0 & is2) >> s2);
            int istat = 2 * ibit2 + ibit1;
            int iex = ml;
            if (sk[iex + Q * istat]) continue;
            it0 = it0 + is1 * (l1 - ibit1);
            it0 = it0 + is2 * (l2 - ibit2);
            int64_t it = lin_index(m, it0);
            cplx factor2 = hb[iex + Q * istat];
            if (iex == istat) factor2 = factor2 + Keperbd;
            v0[l0] = v0[l0] + factor2 * vt[it];
            cplx c = factor2 * conj(v1[l0]) * vt[it];
            pr += creal(c); pi += cimag(c);
        }
    } else {
        const int64_t is1 = ipow(q, s1), is2 = ipow(q, s2);
        const int ml1 = ml % q, ml2 = ml / q;
#pragma omp parallel for reduction(+ : pr, pi) schedule(static)
        for (int64_t l0 = 0; l0 < ldim; ++l0) {
            int64_t it0 = m->list1 ? m->list1[l0] : l0;
            int ibit1 = (int)((it0 / is1) % q);
            int ibit2 = (int)((it0 / is2) % q);
            int istat = ibit2 * q + ibit1;
            if (sk[ml + Q * istat]) continue;
            it0 = it0 + is1 * (ml1 - ibit1) + is2 * (ml2 - ibit2);
            int64_t it = lin_index(m, it0);
            cplx factor2 = hb[ml + Q * istat];
            if (ml == istat) factor2 = factor2 + Keperbd;
            v0[l0] = v0[l0] + factor2 * vt[it];
            cplx c = factor2 * conj(v1[l0]) * vt[it];
            pr += creal(c); pi += cimag(c);
        }
    }
    return pr + I * pi;
}

/*
 * p_mltply_v3 for lnp = 1: v0 += (H - eperbd*ibond)^T v1 over items in
 * schedule order, prdct = sum of the per-item products.
 * S_one_half/Hybrid_TPS_parallel.f90:190-263 (loop :254-258).
 */
void oracle_p_mltply_v3(const omodel *m, const cplx *v1, cplx *v0, double eperbd, cplx *prdct)
{
    cplx p = 0;
    for (int k = 0; k < m->nitem; ++k) p = p + hv_item(m, k, v1, v1, v0, eperbd);
    *prdct = p;
}

/* Same, restricted to the states [lo, hi) of the output (timing samples). */
void oracle_p_mltply_v3_slice(const omodel *m, const cplx *v1, cplx *v0, double eperbd, int64_t lo, int64_t hi,
                              cplx *prdct)
{
    omodel tmp = *m;
    /* shift the output window: the gather source stays the whole v1 */
    cplx p = 0;
    if (m->list1 || lo < 0 || hi > m->ldim || lo >= hi) { *prdct = 0; return; }
    const int q = m->q, Q = m->Q;
    for (int k = 0; k < m->nitem; ++k) {
        const int s1 = m->it_s1[k], s2 = m->it_s2[k], t = m->it_t[k] - 1, ml = m->it_e[k];
        const cplx *hb = m->X + (size_t)Q * Q * t;
        const unsigned char *sk = m->skip + (size_t)Q * Q * t;
        double pr = 0.0, pi = 0.0;
        if (!m->tree_sa) {
            const int64_t is1 = (int64_t)1 << s1, is2 = (int64_t)1 << s2;
            const int l1 = ml & 1, l2 = (ml >> 1) & 1;
#pragma omp parallel for reduction(+ : pr, pi) schedule(static)
            for (int64_t l0 = lo; l0 < hi; ++l0) {
                int64_t it0 = l0;
                int ibit1 = (int)((it0 & is1) >> s1), ibit2 = (int)((it0 & is2) >> s2);
                int istat = 2 * ibit2 + ibit1;
                if (sk[ml + Q * istat]) continue;
                it0 = it0 + is1 * (l1 - ibit1) + is2 * (l2 - ibit2);
                cplx factor2 = hb[ml + Q * istat];
                if (ml == istat) factor2 = factor2 - eperbd;
                v0[l0 - lo] = v0[l0 - lo] + factor2 * v1[it0];
                cplx c = factor2 * conj(v1[l0]) * v1[it0];
                pr += creal(c); pi += cimag(c);
            }
        } else {
            const int64_t is1 = ipow(q, s1), is2 = ipow(q, s2);
            const int ml1 = ml % q, ml2 = ml / q;
#pragma omp parallel for reduction(+ : pr, pi) schedule(static)
            for (int64_t l0 = lo; l0 < hi; ++l0) {
                int64_t it0 = l0;
                int ibit1 = (int)((it0 / is1) % q), ibit2 = (int)((it0 / is2) % q);
                int istat = ibit2 * q + ibit1;
                if (sk[ml + Q * istat]) continue;
                it0 = it0 + is1 * (ml1 - ibit1) + is2 * (ml2 - ibit2);
                cplx factor2 = hb[ml + Q * istat];
                if (ml == istat) factor2 = factor2 - eperbd;
                v0[l0 - lo] = v0[l0 - lo] + factor2 * v1[it0];
                cplx c = factor2 * conj(v1[l0]) * v1[it0];
                pr += creal(c); pi += cimag(c);
            }
        }
        p = p + (pr + I * pi);
    }
    (void)tmp;
    *prdct = p;
}

/* calc_vec_inprdct: sum conj(x1) x2.  S_one_half/Hybrid_TPS_parallel.f90:104-126 */
cplx oracle_inprdct(int64_t n, const cplx *x1, const cplx *x2)
{
    double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
    for (int64_t j = 0; j < n; ++j) {
        cplx c = conj(x1[j]) * x2[j];
        re += creal(c); im += cimag(c);
    }
    return re + I * im;
}

/* calc_beta: sum |v0 - alpha v1|^2.  S_one_half/Hybrid_TPS_parallel.f90:161-188 */
double oracle_calc_beta(int64_t n, cplx alpha, const cplx *v1, const cplx *v0)
{
    double b = 0;
#pragma omp parallel for reduction(+ : b) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        cplx d = v0[i] - alpha * v1[i];
        b += creal(conj(d) * d);
    }
    return b;
}

/* calc_alpha_beta: S_one_half/Hybrid_TPS_parallel.f90:145-159 */
static void calc_alpha_beta(const omodel *m, double *alp, double *bet, const cplx *v1, cplx *v0)
{
    cplx a;
    oracle_p_mltply_v3(m, v1, v0, 0.0, &a);
    double b = oracle_calc_beta(m->ldim, a, v1, v0);
    *alp = creal(a);
    *bet = sqrt(b);
}

/* calc_alpha_beta2: S_one_half/Hybrid_TPS_parallel.f90:128-142 */
static void calc_alpha_beta2(const omodel *m, double *alp, double *bet, const cplx *v1, cplx *v0)
{
    cplx a;
    oracle_p_mltply_v3(m, v1, v0, 0.0, &a);
    cplx b = oracle_inprdct(m->ldim, v0, v0);
    *alp = creal(a);
    *bet = sqrt(creal(b));
}

/* ------------------------------------------------------------------------ */
/* Tridiagonal routines: S_one_half/Hybrid_TPS_basic.f90                    */
/* ------------------------------------------------------------------------ */

/* bisec: S_one_half/Hybrid_TPS_basic.f90:25-107 (1-based arrays shifted to 0) */
int oracle_bisec(const double *alpha, const double *beta, int ndim, double *E, int ne, double eps)
{
    if (ndim > 8000) return OR_EINVAL;
    if (ne > ndim || ne < 0) return OR_EINVAL;
    double range;
    if (ndim == 1) {
        range = fabs(alpha[0]) + fabs(beta[0]);
    } else {
        range = fabs(alpha[0]) + fabs(beta[0]);
        for (int k = 2; k <= ndim - 1; ++k) {
            double r2 = fabs(beta[k - 2]) + fabs(alpha[k - 1]) + fabs(beta[k - 1]);
            if (r2 > range) range = r2;
        }
        double r3 = fabs(beta[ndim - 2]) + fabs(alpha[ndim - 1]);
        if (r3 > range) range = r3;
    }
    range = -range;
    double *b2 = malloc(sizeof(double) * (ndim + 1));
    b2[0] = 0.0;
    for (int i = 2; i <= ndim; ++i) b2[i - 1] = beta[i - 2] * beta[i - 2];
    double epsabs = fabs(range) * eps;
    for (int i = 0; i < ne; ++i) E[i] = -range;
    double b = range;
    for (int k = 1; k <= ne; ++k) {
        double a = E[k - 1];
        for (int j = 1; j <= 100; ++j) {
            double c = (a + b) / 2.0;
            if (fabs(a - b) < epsabs) continue;
            int numneg = 0;
            double g = 1.0;
            int ipass = 0;
            for (int i = 1; i <= ndim; ++i) {
                if (ipass == 0) g = c - alpha[i - 1] - b2[i - 1] / g;
                else if (ipass == 1) ipass = 2;
                else { g = c - alpha[i - 1]; ipass = 0; }
                if (ipass == 0) {
                    if (g < 0.0) numneg++;
                    if (fabs(g) < fabs(b2[i - 1] * epsabs * eps)) ipass = 1;
                }
            }
            numneg = ndim - numneg;
            if (numneg < k) b = c;
            else {
                a = c;
                int up = numneg < ne ? numneg : ne;
                for (int i = k; i <= up; ++i) E[i - 1] = c;
            }
        }
    }
    free(b2);
    return OR_OK;
}

/* vec12: S_one_half/Hybrid_TPS_basic.f90:112-213.  v is [nvec][ndim]. */
int oracle_vec12(const double *alpha, const double *beta, double *v, const double *E, int ndim, int nvec)
{
    double *di = malloc(sizeof(double) * (ndim + 2)), *bl = malloc(sizeof(double) * (ndim + 2));
    double *bu = malloc(sizeof(double) * (ndim + 2)), *bv = malloc(sizeof(double) * (ndim + 2));
    double *cm = malloc(sizeof(double) * (ndim + 2));
    int *lex = malloc(sizeof(int) * (ndim + 2));
    /* 1-based helpers */
#define DI(j) di[(j)]
#define BL(j) bl[(j)]
#define BU(j) bu[(j)]
#define BV(j) bv[(j)]
#define CM(j) cm[(j)]
#define V(j, k) v[(size_t)((k) - 1) * ndim + (j) - 1]
    int km = 1;
    for (int k = 1; k <= nvec; ++k) {
        for (int j = 1; j <= ndim; ++j) {
            DI(j) = E[k - 1] - alpha[j - 1];
            BL(j) = -beta[j - 1];
            BU(j) = -beta[j - 1];
        }
        BU(ndim + 1) = 0.0;
        for (int j = 1; j <= ndim - 1; ++j) {
            if (fabs(DI(j)) > fabs(BL(j))) {
                lex[j] = 0;
                if (fabs(DI(j)) < 1.e-13) DI(j) = 1.e-13;
                CM(j + 1) = BL(j) / DI(j);
                DI(j + 1) = DI(j + 1) - CM(j + 1) * BU(j);
                BV(j) = 0.0;
            } else {
                lex[j] = 1;
                CM(j + 1) = DI(j) / BL(j);
                DI(j) = BL(j);
                double s = BU(j);
                BU(j) = DI(j + 1);
                BV(j) = BU(j + 1);
                DI(j + 1) = s - CM(j + 1) * BU(j);
                BU(j + 1) = -CM(j + 1) * BV(j);
            }
        }
        if (fabs(DI(ndim)) < 1.e-13) DI(ndim) = 1.e-13;
        for (int j = 1; j <= ndim; ++j) V(j, k) = 1.0 / ((double)j * 5.0);
        if (k == 1) km = k;
        else if (fabs(E[k - 1] - E[km - 1]) > 1.e-13) km = k;
        else {
            for (int i = km; i <= k - 1; ++i) {
                double prd = 0.0;
                for (int j = 1; j <= ndim; ++j) prd += V(j, i) * V(j, k);
                for (int j = 1; j <= ndim; ++j) V(j, k) = V(j, k) - prd * V(j, i);
            }
        }
        for (int l = 1; l <= k - km + 3; ++l) {
            if (l != 1 || k != km) {
                for (int j = 1; j <= ndim - 1; ++j) {
                    if (lex[j] == 0) V(j + 1, k) = V(j + 1, k) - CM(j + 1) * V(j, k);
                    else {
                        double s = V(j, k);
                        V(j, k) = V(j + 1, k);
                        V(j + 1, k) = s - CM(j + 1) * V(j, k);
                    }
                }
            }
            for (int j = ndim; j >= 1; --j) {
                double s = V(j, k);
                if (j <= ndim - 1) s = s - BU(j) * V(j + 1, k);
                if (j <= ndim - 2) s = s - BV(j) * V(j + 2, k);
                V(j, k) = s / DI(j);
            }
            double dnorm = 0.0;
            for (int j = 1; j <= ndim; ++j) dnorm += V(j, k) * V(j, k);
            if (dnorm > 1.e-13) dnorm = 1.0 / sqrt(dnorm);
            for (int j = 1; j <= ndim; ++j) V(j, k) = V(j, k) * dnorm;
        }
    }
#undef DI
#undef BL
#undef BU
#undef BV
#undef CM
#undef V
    free(di); free(bl); free(bu); free(bv); free(cm); free(lex);
    return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* Krylov loops                                                             */
/* ------------------------------------------------------------------------ */

/*
 * parallelized_lnc1z (S_one_half/Hybrid_TPS_Lanczos.f90:48-163) for a given
 * normalised initial vector.  Runs steps i = 2..nsteps (alpha/beta 0..nsteps-1);
 * with check_conv the nvec=8 convergence test of :133-155 may stop earlier.
 * v1 is overwritten with the last Lanczos vector; returns the number of
 * steps done in *itr (or an error on beta breakdown, :126-130).
 */
int oracle_lanczos(const omodel *m, cplx *v1, int nsteps, int check_conv, double *alpha, double *beta,
                   double *ene /* 8 */, int *itr)
{
    const int nvec2 = 8;
    int64_t ldim = m->ldim;
    cplx *v0 = calloc((size_t)ldim, sizeof(cplx));
    if (!v0) return OR_ENOMEM;
    double alpha1, beta1, ebefor = 0.0, eps = 1e-25;
    calc_alpha_beta(m, &alpha1, &beta1, v1, v0);
    alpha[0] = alpha1; beta[0] = beta1;
    int done = 1;
    int rc = OR_OK;
    for (int i = 2; i <= nsteps; ++i) {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < ldim; ++j) {
            cplx temp1 = v1[j];
            cplx temp2 = (v0[j] - alpha1 * v1[j]) / beta1;
            v0[j] = -beta1 * temp1;
            v1[j] = temp2;
        }
        calc_alpha_beta(m, &alpha1, &beta1, v1, v0);
        alpha[i - 1] = alpha1; beta[i - 1] = beta1;
        done = i;
        if (beta[i - 1] < 0.5e-30) { rc = OR_EBREAKDOWN; break; }
        if (check_conv) {
            if (i > 4 * nvec2 && i % 5 == 0) {
                oracle_bisec(alpha, beta, i, ene, nvec2, eps);
                int loop = fabs((ebefor - ene[nvec2 - 1]) / ene[nvec2 - 1]) < 1e-13;
                if (loop) break;
                ebefor = ene[nvec2 - 1];
            }
            if (i == 4 * nvec2) {
                eps = 1e-25;
                oracle_bisec(alpha, beta, 4 * nvec2, ene, nvec2, eps);
                ebefor = ene[nvec2 - 1];
            }
        }
    }
    if (ene) oracle_bisec(alpha, beta, done, ene, done < nvec2 ? done : nvec2, 1e-25);
    *itr = done;
    free(v0);
    return rc;
}

/*
 * One step of parallelized_lnc1z's loop (S_one_half/Hybrid_TPS_Lanczos.f90:
 * 111-122): the swap with the previous step's alpha/beta (in *alpha, *beta),
 * then p_mltply_v3 and calc_beta; *alpha, *beta receive the new values.  The
 * CPU timing of a whole step at full size calls this.
 */
void oracle_lanczos_step(const omodel *m, cplx *v1, cplx *v0, double *alpha, double *beta)
{
    const int64_t ldim = m->ldim;
    const double a = *alpha, b = *beta;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ldim; ++j) {
        cplx temp1 = v1[j];
        cplx temp2 = (v0[j] - a * v1[j]) / b;
        v0[j] = -b * temp1;
        v1[j] = temp2;
    }
    calc_alpha_beta(m, alpha, beta, v1, v0);
}

/*
 * The same step restricted to the output states [lo, hi) (a bounded sample
 * of a step): the swap on the slice of v1 and of v0s (v0s holds states lo ..
 * hi-1), p_mltply_v3 on the slice gathering from the whole v1, and calc_beta on
 * the slice.  *alpha receives the slice's part of Re prdct, *beta the square
 * root of the slice's part of calc_beta's sum.
 */
void oracle_lanczos_step_slice(const omodel *m, cplx *v1, cplx *v0s, int64_t lo, int64_t hi, double *alpha,
                               double *beta)
{
    const double a = *alpha, b = *beta;
#pragma omp parallel for schedule(static)
    for (int64_t j = lo; j < hi; ++j) {
        cplx temp1 = v1[j];
        cplx temp2 = (v0s[j - lo] - a * v1[j]) / b;
        v0s[j - lo] = -b * temp1;
        v1[j] = temp2;
    }
    cplx pr;
    oracle_p_mltply_v3_slice(m, v1, v0s, 0.0, lo, hi, &pr);
    const double bb = oracle_calc_beta(hi - lo, pr, v1 + lo, v0s);
    *alpha = creal(pr);
    *beta = sqrt(bb);
}

/*
 * Eigenvector by the Lanczos method, parallelized_lncv1z
 * (S_one_half/Hybrid_TPS_Lanczos.f90:183-329): the chain of the initial
 * vector is replayed with the alpha/beta stored by the first pass and
 * x = sum_{k=1..nsteps} coef[k-1] v_k is accumulated (:226-237, :270-309),
 * then normalised (:312-327).  As written, the reference zeroes v1 before its
 * first product (:205-214, :238), so its x comes out as the normalised
 * initial vector, which the following inverse iteration (parallelized_inv1z)
 * then refines; this restates the recurrence the routine sets up, with v_1 =
 * the initial vector.
 */
int oracle_lanczos_vector(const omodel *m, const cplx *v_init, int nsteps, const double *alpha, const double *beta,
                          const double *coef, cplx *x)
{
    int64_t ldim = m->ldim;
    cplx *v1 = malloc((size_t)ldim * sizeof(cplx));
    cplx *v0 = calloc((size_t)ldim, sizeof(cplx));
    if (!v1 || !v0) { free(v1); free(v0); return OR_ENOMEM; }
    memcpy(v1, v_init, (size_t)ldim * sizeof(cplx));
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ldim; ++j) x[j] = coef[0] * v1[j];
    cplx dummy;
    for (int k = 1; k < nsteps; ++k) {
        /* v0 = H v_k - beta_{k-1} v_{k-1} (v0 holds -beta_{k-1} v_{k-1}) */
        oracle_p_mltply_v3(m, v1, v0, 0.0, &dummy);
        const double a = alpha[k - 1], b = beta[k - 1], c = coef[k];
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < ldim; ++j) {
            cplx temp1 = v1[j];
            cplx temp2 = (v0[j] - a * v1[j]) / b;
            v0[j] = -b * temp1;
            v1[j] = temp2;
            x[j] += c * temp2;
        }
    }
    double dn = sqrt(creal(oracle_inprdct(ldim, x, x)));
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ldim; ++j) x[j] /= dn;
    free(v1); free(v0);
    return OR_OK;
}

/*
 * Diagonal observables of the TPS step (S_one_half/Hybrid_TPS_TPS.f90:128-321,
 * S_arbitrary/Hybrid_TPS9_TPS.f90 twin).  Every observable the reference
 * evaluates has the form
 *     O(s) = sum_t c_t * T[bit(s, a_t)][bit(s, b_t)]
 * with bit(s, p) = (s >> p) & 1 (0 for p >= n) -- the reference extracts bits
 * with iand/ishft in both trees, also for base-q states -- a 2x2 complex table
 * T per observable and complex weights c_t:
 *   calc_zz_bond_corr (:270-321): terms (ipair(2i-1), ipair(2i)) for z-bonds
 *       (the 1-based site numbers are used as bit shifts), c = 1,
 *       T[i][k] = (i - 1/2)(k - 1/2);
 *   calc_sq_zz (:153-199): terms (j, 0), c = e^{i q.r_j}, T[i][k] = (i-s)(k-s);
 *   calc_sq_pp (:201-249): terms (j, 0), c = e^{i q.r_j}, T = my_xor.
 * Layout: obs_off[o]..obs_off[o+1]-1 index the term arrays; obs_T is [o][2][2]
 * complex (T[i][k] at 2*i+k).
 */
static inline cplx obs_weight(int n, int64_t st, int t0, int t1, const int *ta, const int *tb,
                              const cplx *tc, const cplx *T)
{
    cplx acc = 0;
    for (int t = t0; t < t1; ++t) {
        int i = ta[t] >= n ? 0 : (int)((st >> ta[t]) & 1);
        int k = tb[t] >= n ? 0 : (int)((st >> tb[t]) & 1);
        acc += tc[t] * T[2 * i + k];
    }
    return acc;
}

/*
 * parallelized_TPSz (S_one_half/Hybrid_TPS_TPS.f90:325-409) for one seed with
 * the TPS-transformed model (X = l_b - X, L = l_b*ibond) and a normalised
 * random initial vector v1.  coef is [nsteps][ncoef] row-major with
 *   coef[i][0] = 2(i+1)/alpha, [1] = L, [2] = beta, [3] = L - alpha,
 *   [4] = Re(L<vg|v1> - <vg|v0>), then for each observable o two entries
 *   Re<v1|O v1>, Re<vg|O v1>  (eval_phys_val :83-111).
 * alpha_out[i] = L - alpha1 (<H>), beta_out[i] = ||(L-H)|k>||.
 */
int oracle_tps(const omodel *m, double L, cplx *v1, int nsteps, int nobs, const int *obs_off, const int *ta,
               const int *tb, const cplx *tc, const cplx *obs_T, double *alpha_out, double *beta_out, double *coef,
               int ncoef)
{
    int64_t ldim = m->ldim;
    cplx *v0 = calloc((size_t)ldim, sizeof(cplx));
    cplx *vg = calloc((size_t)ldim, sizeof(cplx));
    if (!v0 || !vg) { free(v0); free(vg); return OR_ENOMEM; }
    double alpha1 = 0, beta1 = 1;
    for (int i = 1; i <= nsteps; ++i) {
        if (i > 1) {
            double xnorm = 1.0 / beta1;
#pragma omp parallel for schedule(static)
            for (int64_t j = 0; j < ldim; ++j) {
                vg[j] = v1[j];
                v1[j] = xnorm * v0[j];
                v0[j] = 0;
            }
        }
        calc_alpha_beta2(m, &alpha1, &beta1, v1, v0);
        alpha_out[i - 1] = L - alpha1;
        beta_out[i - 1] = beta1;
        double *c = coef + (size_t)(i - 1) * ncoef;
        c[0] = (double)(2 * i) / alpha1;
        c[1] = L;
        c[2] = beta1;
        c[3] = L - alpha1;
        cplx val1 = oracle_inprdct(ldim, vg, v0);
        cplx val2 = oracle_inprdct(ldim, vg, v1);
        c[4] = creal(L * val2 - val1);
        for (int o = 0; o < nobs && 5 + 2 * o + 1 < ncoef; ++o) {
            double r1 = 0, r2 = 0;
            const int t0 = obs_off[o], t1 = obs_off[o + 1];
            const cplx *T = obs_T + 4 * o;
#pragma omp parallel for reduction(+ : r1, r2) schedule(static)
            for (int64_t j = 0; j < ldim; ++j) {
                int64_t st = m->list1 ? m->list1[j] : j;
                cplx ov = obs_weight(m->n, st, t0, t1, ta, tb, tc, T) * v1[j];
                r1 += creal(conj(v1[j]) * ov);
                r2 += creal(conj(vg[j]) * ov);
            }
            c[5 + 2 * o] = r1;
            c[5 + 2 * o + 1] = r2;
        }
    }
    free(v0); free(vg);
    return OR_OK;
}

/*
 * intalv_zz: v = sum_j (d_j - s) e^{i q.r_j} x, normalised; returns
 * cnorm = ||v_raw||^2 / n.  S_one_half/Hybrid_TPS_DSF.f90:18-87 (S1/2: bit 1
 * counts +1/2) and S_arbitrary/Hybrid_TPS9_DSF.f90:18-89 (digit - S).
 * qr[j] = q.r_j for site j.
 */
int oracle_intalv_zz(const omodel *m, const double *qr, const cplx *x, cplx *v, cplx *cnorm_out)
{
    int64_t ldim = m->ldim;
    int q = m->q;
    double ss = m->tree_sa ? 0.5 * (double)(q - 1) : 0.5;
    for (int64_t i = 0; i < ldim; ++i) v[i] = 0;
    for (int j = 0; j < m->n; ++j) {
        double qnorm = qr[j];
        double cq = cos(qnorm), sq = sin(qnorm);
        int64_t basis = ipow(q, j);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < ldim; ++i) {
            int64_t istate = m->list1 ? m->list1[i] : i;
            int64_t is = m->tree_sa ? (istate / basis) % q : (istate >> j) & 1;
            v[i] = v[i] + ((double)is - ss) * ((cq * creal(x[i]) - sq * cimag(x[i])) +
                                               I * (sq * creal(x[i]) + cq * cimag(x[i])));
        }
    }
    cplx cnorm = oracle_inprdct(ldim, v, v);
    if (cabs(cnorm) < 1e-25) cnorm = 1e-25;
    double norm2 = 1.0 / sqrt(creal(cnorm));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ldim; ++i) v[i] = v[i] * norm2;
    *cnorm_out = cnorm / (double)m->n;
    return OR_OK;
}

/*
 * intalv_xy, one rank (b_bit = n): v = sum_j fac e^{i q.r_j} S^{ipm}_j x,
 * normalised; returns cnorm = ||v_raw||^2 / n.  x lives on the source model's
 * basis (its sector states in list1 order, the reference's listt of
 * get_listt); v on the target model's (its Lin tables, list3(:,:,0)).
 * S_one_half/Hybrid_TPS_DSF.f90:91-193: ipm = +1 only, bit j 0 -> 1, no
 * factor.  S_arbitrary/Hybrid_TPS9_DSF.f90:91-286 (local_operation
 * :196-243): digit is -> is + ipm with fac = sqrt((s - sm)(s + sm + 1))
 * (ipm = +1) or sqrt((s + sm)(s - sm + 1)) (ipm = -1), sm = is - s; sites in
 * ascending order, each added over all source states.
 */
int oracle_intalv_xy(const omodel *mt, const omodel *ms, int ipm, const double *qr, const cplx *x, cplx *v,
                     cplx *cnorm_out)
{
    if (mt->n != ms->n || mt->q != ms->q || mt->tree_sa != ms->tree_sa) return OR_EINVAL;
    if (ipm != 1 && ipm != -1) return OR_EINVAL;
    if (!mt->tree_sa && ipm != 1) return OR_EINVAL;
    const int q = mt->q;
    const double ss = 0.5 * (double)(q - 1);
    for (int64_t i = 0; i < mt->ldim; ++i) v[i] = 0;
    for (int j = 0; j < mt->n; ++j) {
        const double qnorm = qr[j];
        const double cq = cos(qnorm), sq = sin(qnorm);
        const int64_t basis = ipow(q, j);
        /* one site: distinct source states reach distinct targets */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < ms->ldim; ++i) {
            const int64_t st = ms->list1 ? ms->list1[i] : i;
            const cplx rot = (cq * creal(x[i]) - sq * cimag(x[i])) + I * (sq * creal(x[i]) + cq * cimag(x[i]));
            if (!mt->tree_sa) {
                if (((st >> j) & 1) != 0) continue;
                v[lin_index(mt, st + basis)] += rot;
            } else {
                const int64_t is = (st / basis) % q;
                if (is + ipm < 0 || is + ipm >= q) continue;
                const double sm = (double)is - ss;
                const double fac = ipm == 1 ? sqrt((ss - sm) * (ss + sm + 1.0)) : sqrt((ss + sm) * (ss - sm + 1.0));
                v[lin_index(mt, st + ipm * basis)] += fac * rot;
            }
        }
    }
    cplx cnorm = oracle_inprdct(mt->ldim, v, v);
    if (cabs(cnorm) < 1e-25) cnorm = 1e-25;
    const double norm2 = 1.0 / sqrt(creal(cnorm));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < mt->ldim; ++i) v[i] = v[i] * norm2;
    *cnorm_out = cnorm / (double)mt->n;
    return OR_OK;
}

/*
 * parallelized_dsflnc1z (S_one_half/Hybrid_TPS_DSF.f90:195-261): with
 * s_maxitr = nsteps+1, salpha[0..nsteps-1], sbeta[0..nsteps] (sbeta[0] = cnorm).
 */
int oracle_dsf_chain(const omodel *m, cplx *v1, cplx cnorm, int nsteps, double *salpha, double *sbeta)
{
    int64_t ldim = m->ldim;
    cplx *v0 = calloc((size_t)ldim, sizeof(cplx));
    if (!v0) return OR_ENOMEM;
    double alpha1, beta1;
    sbeta[0] = creal(cnorm);
    calc_alpha_beta(m, &alpha1, &beta1, v1, v0);
    salpha[0] = alpha1;
    sbeta[1] = beta1;
    for (int i = 2; i <= nsteps; ++i) {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < ldim; ++j) {
            cplx temp1 = v1[j];
            cplx temp0 = (v0[j] - alpha1 * v1[j]) / beta1;
            v0[j] = -beta1 * temp1;
            v1[j] = temp0;
        }
        calc_alpha_beta(m, &alpha1, &beta1, v1, v0);
        salpha[i - 1] = alpha1;
        sbeta[i] = beta1;
    }
    free(v0);
    return OR_OK;
}

/*
 * exec_renbun (S_one_half/Hybrid_TPS_DSF.f90:263-334): modified-Lentz continued
 * fraction per omega = (j-1)*split; salpha/sbeta of length s_maxitr (zero
 * padded), levels m1 = 1..s_maxitr-1.
 */
void oracle_exec_renbun(int i_range, int s_maxitr, double split, double ene, double epsln, const double *salpha,
                        const double *sbeta, double *w, int *conv, double *dsf)
{
#pragma omp parallel for schedule(static, 1)
    for (int j = 1; j <= i_range; ++j) {
        double omega = (double)(j - 1) * split;
        w[j - 1] = omega;
        int i_conv = 0;
        double xr = 1.0e-10, xi = 1.0e-10, cr = xr, ci = xi, dr = 0.0, di = 0.0;
        for (int m1 = 1; m1 <= s_maxitr - 1; ++m1) {
            double f1 = omega + ene - salpha[m1 - 1];
            double f2 = (-1.0) * pow(sbeta[m1 - 1], 2.0);
            double xr1 = xr, xi1 = xi;
            dr = dr * f2; dr = dr + f1;
            di = di * f2; di = di + epsln;
            double d = dr * dr + di * di;
            if (d == 0.0) { dr = 0.5e-28; di = 0.5e-28; }
            double c = cr * cr + ci * ci;
            cr = cr * f2 / c; cr = cr + f1;
            ci = -ci * f2 / c; ci = ci + epsln;
            c = cr * cr + ci * ci;
            if (c == 0.0) { cr = 0.5e-28; ci = 0.5e-28; }
            d = dr * dr + di * di;
            dr = dr / d; di = -di / d;
            double dlr = cr * dr - ci * di, dli = ci * dr + cr * di;
            xr = xr1 * dlr - xi1 * dli;
            xi = xr1 * dli + xi1 * dlr;
            double dl = (dlr - 1.0) * (dlr - 1.0) + dli * dli;
            if (dl < 0.5e-28) { i_conv = m1; break; }
        }
        conv[j - 1] = i_conv;
        dsf[j - 1] = xi;
    }
}

/* nomalization_DSF: S_one_half/Hybrid_TPS_DSF.f90:337-351 */
void oracle_normalization_dsf(int i_range, double split, double sq_re, double *dsf)
{
    double sum = 0.0;
    for (int i = 2; i <= i_range; ++i) sum = sum + 0.5 * split * (dsf[i - 1] + dsf[i - 2]);
    for (int i = 1; i <= i_range; ++i) dsf[i - 1] = sq_re / sum * dsf[i - 1];
}

/*
 * parallelized_inv1z + parallelized_cg1 (S_one_half/Hybrid_TPS_cg.f90:18-196).
 * b: initial right-hand side (normalised random vector), x: result.
 * The `loop` flags of cg1 and inv1z are SAVEd Fortran variables: once cg1
 * converges, every later cg1 call returns after its first 5 iterations; this
 * is kept (state passed in cg_loop_saved).
 */
static int cg1(const omodel *m, double Eig, cplx *x, cplx *b, cplx *p, cplx *r, cplx *y, int *cg_loop_saved,
               int cg_max, int *iters)
{
    int64_t ldim = m->ldim;
    cplx bcnorm = oracle_inprdct(ldim, b, b);
    for (int64_t i = 0; i < ldim; ++i) { r[i] = b[i]; p[i] = b[i]; x[i] = 0; }
    double eperbd = Eig / (double)m->nbond;
    for (int itr = 1; itr <= cg_max; ++itr) {
        for (int64_t i = 0; i < ldim; ++i) y[i] = 0;
        cplx cdmm;
        oracle_p_mltply_v3(m, p, y, eperbd, &cdmm);
        cplx crp = oracle_inprdct(ldim, p, r);
        cplx cyp = oracle_inprdct(ldim, p, y);
        cplx calpha = crp / cyp;
        cplx rcnorm = oracle_inprdct(ldim, r, r);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < ldim; ++i) {
            x[i] = x[i] + calpha * p[i];
            r[i] = r[i] - calpha * y[i];
        }
        cplx rcnorm2 = oracle_inprdct(ldim, r, r);
        double beta = creal(rcnorm2) / creal(rcnorm);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < ldim; ++i) p[i] = r[i] + beta * p[i];
        *iters = itr;
        if (itr % 5 != 0) continue;
        if (sqrt(cabs(rcnorm2)) < 1.0e-9 * sqrt(cabs(bcnorm))) *cg_loop_saved = 1;
        if (*cg_loop_saved) return OR_OK;
    }
    return OR_OK;
}

int oracle_inverse_iteration(const omodel *m, double Eig, cplx *b_init, cplx *x, int inv_max, int cg_max,
                             int *n_inv, int *n_cg_total)
{
    int64_t ldim = m->ldim;
    cplx *b = malloc(sizeof(cplx) * ldim), *p = malloc(sizeof(cplx) * ldim);
    cplx *r = malloc(sizeof(cplx) * ldim), *y = malloc(sizeof(cplx) * ldim);
    if (!b || !p || !r || !y) { free(b); free(p); free(r); free(y); return OR_ENOMEM; }
    memcpy(b, b_init, sizeof(cplx) * ldim);
    int cg_loop_saved = 0;
    int total = 0;
    *n_inv = 0;
    for (int itr = 1; itr <= inv_max; ++itr) {
        int it = 0;
        cg1(m, Eig, x, b, p, r, y, &cg_loop_saved, cg_max, &it);
        total += it;
        cplx xcn = oracle_inprdct(ldim, x, x);
        double xnorm = 1.0 / sqrt(creal(xcn));
        for (int64_t i = 0; i < ldim; ++i) x[i] = x[i] * xnorm;
        cplx cxb = oracle_inprdct(ldim, x, b);
        *n_inv = itr;
        if (fabs(cabs(cxb) - 1.0) < 1.0e-12) break;
        for (int64_t i = 0; i < ldim; ++i) b[i] = x[i];
    }
    *n_cg_total = total;
    free(b); free(p); free(r); free(y);
    return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* Seeded complex-Gaussian vectors (shared definition with the GPU kernel)   */
/* ------------------------------------------------------------------------ */
static inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/*
 * v[g], g = s*R + r for s < dim, r < R: z = sqrt(-ln u1) * e^{2 pi i u2} with
 * u1 = (h1>>11 + 0.5) 2^-53, u2 = (h2>>11) 2^-53, h1/h2 = splitmix64 of the
 * mixed seed xor (2g, 2g+1); E|z|^2 = 1.  Not normalised.
 */
void oracle_gaussian(uint64_t seed, int64_t dim, int R, cplx *v)
{
    uint64_t key = splitmix64(seed ^ 0x5DEECE66Dull);
    int64_t n = dim * R;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; ++g) {
        uint64_t h1 = splitmix64(key ^ (uint64_t)(2 * g));
        uint64_t h2 = splitmix64(key ^ (uint64_t)(2 * g + 1));
        double u1 = ((double)(h1 >> 11) + 0.5) * 0x1.0p-53;
        double u2 = (double)(h2 >> 11) * 0x1.0p-53;
        double rad = sqrt(-log(u1));
        double ang = 2.0 * 3.14159265358979323846 * u2;
        v[g] = rad * cos(ang) + I * (rad * sin(ang));
    }
}

int oracle_num_threads(void) { return omp_get_max_threads(); }
void oracle_set_num_threads(int n) { omp_set_num_threads(n); }
