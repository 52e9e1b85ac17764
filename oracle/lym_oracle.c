/*
 * CPU oracle for the Wilson / Wilson-clover hot path of LeonardYM.
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Conventions and
 * provenance are described in lym_oracle.h.
 *
 * Arithmetic is FP64 complex with long double global reductions, as in the
 * reference (MatrixTypedef.h:28-30, AlgebraUtils.h:17-27).  The order of the
 * accumulations follows the reference loops so that results agree to a few
 * ulps, not only to tolerance.
 */
#include "lym_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SP(v, site, spin, nc) ((v) + ((size_t)(site) * 4 + (spin)) * (nc))

static int modulus(int value, int mod)
{
    /* LocalLayout::modulus (MPILattice/LocalLayout.h:164-169) */
    if (value >= mod) return value - mod;
    if (value < 0) return value + mod;
    return value;
}

static int lex_index(const int d[4], int x, int y, int z, int t)
{
    /* LocalLayout::getGlobalCoordinate (MPILattice/LocalLayout.h:149-163) */
    x = modulus(x, d[0]);
    y = modulus(y, d[1]);
    z = modulus(z, d[2]);
    t = modulus(t, d[3]);
    return d[3] * (d[2] * (d[1] * x + y) + z) + t;
}

int orc_geom_tables(const int d[4], int *sup, int *sdn, int *coord)
{
    /* LocalLayout::initialize (MPILattice/LocalLayout.h:34-110) */
    for (int x = 0; x < d[0]; ++x)
        for (int y = 0; y < d[1]; ++y)
            for (int z = 0; z < d[2]; ++z)
                for (int t = 0; t < d[3]; ++t) {
                    int s = lex_index(d, x, y, z, t);
                    int c[4] = {x, y, z, t};
                    for (int mu = 0; mu < 4; ++mu) {
                        int cp[4] = {x, y, z, t}, cm[4] = {x, y, z, t};
                        cp[mu] += 1;
                        cm[mu] -= 1;
                        if (sup) sup[s * 4 + mu] = lex_index(d, cp[0], cp[1], cp[2], cp[3]);
                        if (sdn) sdn[s * 4 + mu] = lex_index(d, cm[0], cm[1], cm[2], cm[3]);
                        if (coord) coord[s * 4 + mu] = c[mu];
                    }
                }
    return 0;
}

int orc_geom_init(orc_geom *g, const int dims[4])
{
    memset(g, 0, sizeof(*g));
    for (int mu = 0; mu < 4; ++mu) {
        if (dims[mu] < 1) return -1;
        g->dims[mu] = dims[mu];
    }
    g->V = dims[0] * dims[1] * dims[2] * dims[3];
    g->sup = (int *)malloc(sizeof(int) * 4 * (size_t)g->V);
    g->sdn = (int *)malloc(sizeof(int) * 4 * (size_t)g->V);
    g->coord = (int *)malloc(sizeof(int) * 4 * (size_t)g->V);
    if (!g->sup || !g->sdn || !g->coord) return -2;
    return orc_geom_tables(g->dims, g->sup, g->sdn, g->coord);
}

void orc_geom_free(orc_geom *g)
{
    free(g->sup);
    free(g->sdn);
    free(g->coord);
    memset(g, 0, sizeof(*g));
}

static int parity_of(const orc_geom *g, int site)
{
    const int *c = g->coord + 4 * site;
    return (c[0] + c[1] + c[2] + c[3]) % 2;
}

void orc_antiperiodic_bc(const int dims[4], void *links, int nc, int real_links)
{
    /* switchAntiperiodicBc (LatticeBoundaryConditions.h:8-14): U_t(x) -> -U_t(x) at t = L_t - 1 */
    int V = dims[0] * dims[1] * dims[2] * dims[3];
    int n2 = nc * nc;
    for (int s = 0; s < V; ++s) {
        if (s % dims[3] != dims[3] - 1) continue; /* t is the fastest index */
        if (real_links) {
            double *u = (double *)links + ((size_t)s * 4 + 3) * n2;
            for (int k = 0; k < n2; ++k) u[k] = -u[k];
        } else {
            orc_cplx *u = (orc_cplx *)links + ((size_t)s * 4 + 3) * n2;
            for (int k = 0; k < n2; ++k) u[k] = -u[k];
        }
    }
}

void orc_su2_to_adjoint(int nlinks, const orc_cplx *fund, double *adj)
{
    /* ConvertLattice::toAdjoint generic branch (utils/ConvertLattice.h:100-105):
     * adj(a,b) = 2 Re tr(T_a U T_b U^dagger), T_a = sigma_a / 2 (utils/LieGenerators.h:17-23). */
    const orc_cplx T[3][4] = {
        {0, 0.5, 0.5, 0},          /* column-major (0,0),(1,0),(0,1),(1,1) */
        {0, 0.5 * I, -0.5 * I, 0},
        {0.5, 0, 0, -0.5},
    };
    for (int l = 0; l < nlinks; ++l) {
        const orc_cplx *U = fund + 4 * (size_t)l;
        orc_cplx Ud[4];
        /* U^dagger, column-major */
        Ud[0] = conj(U[0]);
        Ud[1] = conj(U[2]);
        Ud[2] = conj(U[1]);
        Ud[3] = conj(U[3]);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                orc_cplx A[4], B[4], C[4];
                /* A = T_a U */
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j) {
                        A[j * 2 + i] = 0;
                        for (int k = 0; k < 2; ++k) A[j * 2 + i] += T[a][k * 2 + i] * U[j * 2 + k];
                    }
                /* B = A T_b */
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j) {
                        B[j * 2 + i] = 0;
                        for (int k = 0; k < 2; ++k) B[j * 2 + i] += A[k * 2 + i] * T[b][j * 2 + k];
                    }
                /* C = B U^dagger */
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j) {
                        C[j * 2 + i] = 0;
                        for (int k = 0; k < 2; ++k) C[j * 2 + i] += B[k * 2 + i] * Ud[j * 2 + k];
                    }
                adj[9 * (size_t)l + b * 3 + a] = 2.0 * creal(C[0] + C[3]);
            }
    }
}

/* ------------------------------------------------------------------------- */
/* small dense helpers on nc x nc column-major matrices held as complex      */

static void load_mat(const orc_op *op, const void *base, size_t idx, orc_cplx *m)
{
    int n2 = op->nc * op->nc;
    if (op->real_links) {
        const double *p = (const double *)base + idx * n2;
        for (int k = 0; k < n2; ++k) m[k] = p[k];
    } else {
        const orc_cplx *p = (const orc_cplx *)base + idx * n2;
        for (int k = 0; k < n2; ++k) m[k] = p[k];
    }
}

static void mat_mul(int n, const orc_cplx *a, const orc_cplx *b, orc_cplx *c)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            orc_cplx s = 0;
            for (int k = 0; k < n; ++k) s += a[k * n + i] * b[j * n + k];
            c[j * n + i] = s;
        }
}

static void mat_dag(int n, const orc_cplx *a, orc_cplx *c)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) c[j * n + i] = conj(a[i * n + j]);
}

/* product of four matrices, each optionally daggered: ((A B) C) D */
static void prod4(int n, const orc_cplx *m[4], const int dag[4], orc_cplx *out)
{
    orc_cplx t[4][64], acc[64], tmp[64];
    for (int k = 0; k < 4; ++k) {
        if (dag[k]) mat_dag(n, m[k], t[k]);
        else memcpy(t[k], m[k], sizeof(orc_cplx) * n * n);
    }
    mat_mul(n, t[0], t[1], acc);
    mat_mul(n, acc, t[2], tmp);
    mat_mul(n, tmp, t[3], out);
}

static void update_field_strength(orc_op *op)
{
    /* ImprovedDiracWilsonOperator::updateFieldStrength (ImprovedDiracWilsonOperator.cpp:502-523):
     * four-leaf clover Q_{mu nu}, F = (Q - Q^dagger)/8, planes (01,02,03,12,13,23). */
    const orc_geom *g = op->g;
    const int n = op->nc, n2 = n * n;
    static const int planes[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
#pragma omp parallel for
    for (int s = 0; s < g->V; ++s) {
        for (int p = 0; p < 6; ++p) {
            const int mu = planes[p][0], nu = planes[p][1];
            const int *sup = g->sup, *sdn = g->sdn;
            int dm = sdn[s * 4 + mu], dn = sdn[s * 4 + nu];
            int dmdn = sdn[dm * 4 + nu];
            int dnum = sup[dn * 4 + mu];
            int um = sup[s * 4 + mu], un = sup[s * 4 + nu];
            int dmun = sup[dm * 4 + nu];
            orc_cplx L[4][4][64];
            /* leaf 1: U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu) */
            load_mat(op, op->links, (size_t)dm * 4 + mu, L[0][0]);
            load_mat(op, op->links, (size_t)dmdn * 4 + nu, L[0][1]);
            load_mat(op, op->links, (size_t)dmdn * 4 + mu, L[0][2]);
            load_mat(op, op->links, (size_t)dn * 4 + nu, L[0][3]);
            /* leaf 2: U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+ */
            load_mat(op, op->links, (size_t)dn * 4 + nu, L[1][0]);
            load_mat(op, op->links, (size_t)dn * 4 + mu, L[1][1]);
            load_mat(op, op->links, (size_t)dnum * 4 + nu, L[1][2]);
            load_mat(op, op->links, (size_t)s * 4 + mu, L[1][3]);
            /* leaf 3: U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ */
            load_mat(op, op->links, (size_t)s * 4 + mu, L[2][0]);
            load_mat(op, op->links, (size_t)um * 4 + nu, L[2][1]);
            load_mat(op, op->links, (size_t)un * 4 + mu, L[2][2]);
            load_mat(op, op->links, (size_t)s * 4 + nu, L[2][3]);
            /* leaf 4: U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu) */
            load_mat(op, op->links, (size_t)s * 4 + nu, L[3][0]);
            load_mat(op, op->links, (size_t)dmun * 4 + mu, L[3][1]);
            load_mat(op, op->links, (size_t)dm * 4 + nu, L[3][2]);
            load_mat(op, op->links, (size_t)dm * 4 + mu, L[3][3]);
            static const int dags[4][4] = {{1, 1, 0, 0}, {1, 0, 0, 1}, {0, 0, 1, 1}, {0, 1, 1, 0}};
            orc_cplx Q[64], leaf[64];
            for (int k = 0; k < n2; ++k) Q[k] = 0;
            for (int l = 0; l < 4; ++l) {
                const orc_cplx *m[4] = {L[l][0], L[l][1], L[l][2], L[l][3]};
                prod4(n, m, dags[l], leaf);
                for (int k = 0; k < n2; ++k) Q[k] += leaf[k];
            }
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) {
                    orc_cplx f = (1. / 8.) * (Q[j * n + i] - conj(Q[i * n + j]));
                    size_t at = ((size_t)s * 6 + p) * n2 + j * n + i;
                    if (op->real_links) ((double *)op->F)[at] = creal(f);
                    else ((orc_cplx *)op->F)[at] = f;
                }
        }
    }
}

static inline orc_cplx Fat(const orc_op *op, int site, int k, int i, int j)
{
    size_t at = ((size_t)site * 6 + k) * op->nc * op->nc + (size_t)j * op->nc + i;
    if (op->real_links) return ((const double *)op->F)[at];
    return ((const orc_cplx *)op->F)[at];
}

static inline orc_cplx Uat(const orc_op *op, int site, int mu, int i, int j)
{
    size_t at = ((size_t)site * 4 + mu) * op->nc * op->nc + (size_t)j * op->nc + i;
    if (op->real_links) return ((const double *)op->links)[at];
    return ((const orc_cplx *)op->links)[at];
}

static inline orc_cplx times_i(orc_cplx a) { return CMPLX(-cimag(a), creal(a)); }

/* The clover term at one site, the intermediate "clover[4]" vector of
 * ImprovedDiracWilsonOperator.cpp:200-235 (fundamental and adjoint branches
 * coincide once F is read as complex: complex(a,b) == a + i b). */
static void clover_site(const orc_op *op, int site, const orc_cplx *in /* [4][nc] */,
                        orc_cplx *clover /* [4][nc] */)
{
    const int n = op->nc;
    for (int i = 0; i < n; ++i) {
        clover[0 * n + i] = 0;
        clover[1 * n + i] = 0;
        clover[2 * n + i] = 0;
        clover[3 * n + i] = 0;
        for (int j = 0; j < n; ++j) {
            orc_cplx F0 = Fat(op, site, 0, i, j), F5 = Fat(op, site, 5, i, j);
            clover[0 * n + i] += times_i((-F0 + F5) * in[0 * n + j]);
            clover[1 * n + i] += times_i((+F0 - F5) * in[1 * n + j]);
            clover[2 * n + i] += times_i((+F0 + F5) * in[2 * n + j]);
            clover[3 * n + i] += times_i((-F0 - F5) * in[3 * n + j]);
        }
    }
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            orc_cplx F1 = Fat(op, site, 1, i, j), F2 = Fat(op, site, 2, i, j);
            orc_cplx F3 = Fat(op, site, 3, i, j), F4 = Fat(op, site, 4, i, j);
            clover[0 * n + i] += (+F1 + F4 + times_i(+F2 - F3)) * in[1 * n + j];
            clover[1 * n + i] += (-F1 - F4 + times_i(+F2 - F3)) * in[0 * n + j];
            clover[2 * n + i] += (-F1 + F4 + times_i(+F2 + F3)) * in[3 * n + j];
            clover[3 * n + i] += (+F1 - F4 + times_i(+F2 + F3)) * in[2 * n + j];
        }
    }
}

/* Spin projection tables of DiracWilsonOperator.cpp:25-190.
 * h_k(minus, from x-mu) = psi_k + c[mu][k] psi_{p[mu][k]}
 * h_k(plus,  from x+mu) = psi_k - c[mu][k] psi_{p[mu][k]}                     */
static const int proj_p[4][2] = {{3, 2}, {3, 2}, {2, 3}, {2, 3}};

static inline orc_cplx proj_c(int mu, int k)
{
    static const double re[4][2] = {{0, 0}, {-1, 1}, {0, 0}, {1, 1}};
    static const double im[4][2] = {{-1, -1}, {0, 0}, {-1, 1}, {0, 0}};
    return CMPLX(re[mu][k], im[mu][k]);
}

/* Wilson (+ optional clover) full-lattice multiply / multiplyAdd, following
 * DiracWilsonOperator.cpp:16-202,204-391 and ImprovedDiracWilsonOperator.cpp:22-253,255-487.
 * Computes Q = gamma5 D directly, then undoes gamma5 when gamma5 == false. */
static void wilson_apply(const orc_op *op, orc_cplx *out, const orc_cplx *v1, const orc_cplx *v2,
                         orc_cplx alpha, int add, int with_clover)
{
    const orc_geom *g = op->g;
    const int n = op->nc;
    const double kappa = op->kappa;
#pragma omp parallel for
    for (int site = 0; site < g->V; ++site) {
        orc_cplx hm[8], hp[8], res[4][8];
        for (int mu = 0; mu < 4; ++mu) {
            const int sd = g->sdn[site * 4 + mu], su = g->sup[site * 4 + mu];
            for (int k = 0; k < 2; ++k) {
                const int pk = proj_p[mu][k];
                const orc_cplx c = proj_c(mu, k);
                for (int m = 0; m < n; ++m) {
                    hm[m] = SP(v1, sd, k, n)[m] + c * SP(v1, sd, pk, n)[m];
                    hp[m] = SP(v1, su, k, n)[m] - c * SP(v1, su, pk, n)[m];
                }
                for (int i = 0; i < n; ++i) {
                    orc_cplx tmp = 0, tmm = 0;
                    for (int m = 0; m < n; ++m) tmp += hm[m] * conj(Uat(op, sd, mu, m, i));
                    for (int m = 0; m < n; ++m) tmm += hp[m] * Uat(op, site, mu, i, m);
                    /* lower component: Q adds +kappa * conj(c) * (tmp - tmm) */
                    orc_cplx low = kappa * (conj(c) * (tmp - tmm));
                    if (mu == 0) {
                        if (add) {
                            res[k][i] = alpha * SP(v2, site, k, n)[i] + SP(v1, site, k, n)[i] - kappa * (tmp + tmm);
                            res[pk][i] = alpha * SP(v2, site, pk, n)[i] - SP(v1, site, pk, n)[i] + low;
                        } else {
                            res[k][i] = SP(v1, site, k, n)[i] - kappa * (tmp + tmm);
                            res[pk][i] = -SP(v1, site, pk, n)[i] + low;
                        }
                    } else {
                        res[k][i] -= kappa * (tmp + tmm);
                        res[pk][i] += low;
                    }
                }
            }
        }
        if (with_clover) {
            orc_cplx in[32], clover[32];
            for (int a = 0; a < 4; ++a)
                for (int i = 0; i < n; ++i) in[a * n + i] = SP(v1, site, a, n)[i];
            clover_site(op, site, in, clover);
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < 4; ++a) res[a][i] += (kappa * op->csw) * clover[a * n + i];
        }
        if (!op->gamma5) {
            for (int i = 0; i < n; ++i) {
                if (add) {
                    res[2][i] = -res[2][i] + 2.0 * alpha * SP(v2, site, 2, n)[i];
                    res[3][i] = -res[3][i] + 2.0 * alpha * SP(v2, site, 3, n)[i];
                } else {
                    res[2][i] = -res[2][i];
                    res[3][i] = -res[3][i];
                }
            }
        }
        for (int a = 0; a < 4; ++a)
            for (int i = 0; i < n; ++i) SP(out, site, a, n)[i] = res[a][i];
    }
}

/* ------------------------------------------------------------------------- */
/* even-odd operator (EvenOddImprovedDiracWilsonOperator.cpp)                */

static int inverse12(int N, orc_cplx *a /* N*N column-major, overwritten by inverse */)
{
    /* Gauss-Jordan with partial pivoting; the reference calls Eigen's inverse()
     * (EvenOddImprovedDiracWilsonOperator.cpp:315), an LU with partial pivoting. */
    orc_cplx m[24 * 48];
    const int W = 2 * N;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < W; ++j) m[i * W + j] = (j < N) ? a[j * N + i] : (j - N == i ? 1.0 : 0.0);
    for (int col = 0; col < N; ++col) {
        int piv = col;
        double best = cabs(m[col * W + col]);
        for (int r = col + 1; r < N; ++r)
            if (cabs(m[r * W + col]) > best) {
                best = cabs(m[r * W + col]);
                piv = r;
            }
        if (best == 0.0) return -1;
        if (piv != col)
            for (int j = 0; j < W; ++j) {
                orc_cplx t = m[col * W + j];
                m[col * W + j] = m[piv * W + j];
                m[piv * W + j] = t;
            }
        orc_cplx inv = 1.0 / m[col * W + col];
        for (int j = 0; j < W; ++j) m[col * W + j] *= inv;
        for (int r = 0; r < N; ++r) {
            if (r == col) continue;
            orc_cplx f = m[r * W + col];
            if (f == 0) continue;
            for (int j = 0; j < W; ++j) m[r * W + j] -= f * m[col * W + j];
        }
    }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) a[j * N + i] = m[i * W + N + j];
    return 0;
}

static int calculate_inverse_even_even(orc_op *op)
{
    /* EvenOddImprovedDiracWilsonOperator::calculateInverseEvenEven (.cpp:285-317).
     * Index 3*alpha + c as in the reference (valid for diracVectorLength == 3). */
    const orc_geom *g = op->g;
    const int n = op->nc, N = 4 * n;
    const double kc = op->kappa * op->csw;
    int bad = 0;
#pragma omp parallel for reduction(+ : bad)
    for (int s = 0; s < g->V; ++s) {
        orc_cplx *M = op->Tinv + (size_t)s * N * N;
        for (int k = 0; k < N * N; ++k) M[k] = 0;
        for (int k = 0; k < N; ++k) M[k * N + k] = 1;
#define AT(r, c) M[(size_t)(c) * N + (r)]
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                orc_cplx F0 = Fat(op, s, 0, i, j), F1 = Fat(op, s, 1, i, j), F2 = Fat(op, s, 2, i, j);
                orc_cplx F3 = Fat(op, s, 3, i, j), F4 = Fat(op, s, 4, i, j), F5 = Fat(op, s, 5, i, j);
                AT(n * 0 + i, n * 0 + j) += kc * I * (-F0 + F5);
                AT(n * 1 + i, n * 1 + j) += kc * I * (+F0 - F5);
                AT(n * 2 + i, n * 2 + j) -= kc * I * (+F0 + F5);
                AT(n * 3 + i, n * 3 + j) -= kc * I * (-F0 - F5);
                AT(n * 0 + i, n * 1 + j) += kc * (+F1 + F4 + times_i(+F2 - F3));
                AT(n * 1 + i, n * 0 + j) += kc * (-F1 - F4 + times_i(+F2 - F3));
                AT(n * 2 + i, n * 3 + j) -= kc * (-F1 + F4 + times_i(+F2 + F3));
                AT(n * 3 + i, n * 2 + j) -= kc * (+F1 - F4 + times_i(+F2 + F3));
            }
#undef AT
        if (inverse12(N, M) != 0) bad += 1;
    }
    return bad ? -3 : 0;
}

void orc_eo_multiply_even_even_inverse(const orc_op *op, orc_cplx *out)
{
    /* EvenOddImprovedDiracWilsonOperator::multiplyEvenEvenInverse (.cpp:61-89) */
    const orc_geom *g = op->g;
    const int n = op->nc, N = 4 * n;
#pragma omp parallel for
    for (int s = 0; s < g->V; ++s) {
        if (parity_of(g, s) != 0) continue;
        orc_cplx anti[32];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < n; ++c) anti[a * n + c] = SP(out, s, a, n)[c];
        const orc_cplx *M = op->Tinv + (size_t)s * N * N;
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < n; ++c) {
                orc_cplx t = 0;
                for (int b = 0; b < 4; ++b)
                    for (int bb = 0; bb < n; ++bb) t += M[(size_t)(n * b + bb) * N + (n * a + c)] * anti[b * n + bb];
                SP(out, s, a, n)[c] = t;
            }
    }
}

void orc_eo_multiply_odd_odd_minus_identity(const orc_op *op, orc_cplx *out, const orc_cplx *in, int part)
{
    /* EvenOddImprovedDiracWilsonOperator::multiplyOddOddMinusIdentity (.cpp:148-201):
     * out = T in - out on sites of the given parity */
    const orc_geom *g = op->g;
    const int n = op->nc;
    const double kc = op->kappa * op->csw;
#pragma omp parallel for
    for (int s = 0; s < g->V; ++s) {
        if (parity_of(g, s) != part) continue;
        orc_cplx vin[32], clover[32];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < n; ++c) vin[a * n + c] = SP(in, s, a, n)[c];
        clover_site(op, s, vin, clover);
        for (int c = 0; c < n; ++c) {
            SP(out, s, 0, n)[c] = vin[0 * n + c] + kc * clover[0 * n + c] - SP(out, s, 0, n)[c];
            SP(out, s, 1, n)[c] = vin[1 * n + c] + kc * clover[1 * n + c] - SP(out, s, 1, n)[c];
            SP(out, s, 2, n)[c] = vin[2 * n + c] - kc * clover[2 * n + c] - SP(out, s, 2, n)[c];
            SP(out, s, 3, n)[c] = vin[3 * n + c] - kc * clover[3 * n + c] - SP(out, s, 3, n)[c];
        }
    }
}

void orc_eo_multiply_even_odd(const orc_op *op, orc_cplx *out, const orc_cplx *in, int part)
{
    /* EvenOddImprovedDiracWilsonOperator::multiplyEvenOdd (.cpp:204-281):
     * on sites of parity `part`: out = -kappa H in; other sites: out = in.
     * In-place use (out == in) is safe: each site reads only the other parity. */
    const orc_geom *g = op->g;
    const int n = op->nc;
    const double kappa = op->kappa;
#pragma omp parallel for
    for (int s = 0; s < g->V; ++s) {
        if (parity_of(g, s) != part) {
            if (out != in)
                for (int a = 0; a < 4; ++a)
                    for (int c = 0; c < n; ++c) SP(out, s, a, n)[c] = SP(in, s, a, n)[c];
            continue;
        }
        orc_cplx tplus[4][2][8], tminus[4][2][8];
        for (int mu = 0; mu < 4; ++mu) {
            const int su = g->sup[s * 4 + mu], sd = g->sdn[s * 4 + mu];
            for (int k = 0; k < 2; ++k) {
                const int pk = proj_p[mu][k];
                const orc_cplx c = proj_c(mu, k);
                orc_cplx hp[8], hm[8];
                for (int m = 0; m < n; ++m) {
                    hp[m] = SP(in, su, k, n)[m] - c * SP(in, su, pk, n)[m];
                    hm[m] = SP(in, sd, k, n)[m] + c * SP(in, sd, pk, n)[m];
                }
                for (int i = 0; i < n; ++i) {
                    orc_cplx up = 0, dn = 0;
                    for (int m = 0; m < n; ++m) up += Uat(op, s, mu, i, m) * hp[m];
                    for (int m = 0; m < n; ++m) dn += conj(Uat(op, sd, mu, m, i)) * hm[m];
                    tminus[mu][k][i] = up - dn;
                    tplus[mu][k][i] = up + dn;
                }
            }
        }
        for (int i = 0; i < n; ++i) {
            orc_cplx u0 = tplus[0][0][i] + tplus[1][0][i] + tplus[2][0][i] + tplus[3][0][i];
            orc_cplx u1 = tplus[0][1][i] + tplus[1][1][i] + tplus[2][1][i] + tplus[3][1][i];
            /* lower spins: -kappa * conj(c) * (tmp - tmm) = +kappa * conj(c) * tminus */
            orc_cplx l2 = 0, l3 = 0;
            for (int mu = 0; mu < 4; ++mu)
                for (int k = 0; k < 2; ++k) {
                    orc_cplx v = conj(proj_c(mu, k)) * tminus[mu][k][i];
                    if (proj_p[mu][k] == 2) l2 += v;
                    else l3 += v;
                }
            SP(out, s, 0, n)[i] = -kappa * u0;
            SP(out, s, 1, n)[i] = -kappa * u1;
            SP(out, s, 2, n)[i] = kappa * l2;
            SP(out, s, 3, n)[i] = kappa * l3;
        }
    }
}

static void eo_multiply(const orc_op *op, orc_cplx *out, const orc_cplx *in)
{
    /* EvenOddImprovedDiracWilsonOperator::multiply (.cpp:26-47) */
    const orc_geom *g = op->g;
    const int n = op->nc;
    orc_eo_multiply_even_odd(op, out, in, 0);
    orc_eo_multiply_even_even_inverse(op, out);
    orc_eo_multiply_even_odd(op, out, out, 1);
    orc_eo_multiply_odd_odd_minus_identity(op, out, in, 1);
#pragma omp parallel for
    for (int s = 0; s < g->V; ++s) {
        if (parity_of(g, s) == 0) {
            for (int a = 0; a < 4; ++a)
                for (int c = 0; c < n; ++c) SP(out, s, a, n)[c] = SP(in, s, a, n)[c];
        } else if (op->gamma5) {
            for (int a = 2; a < 4; ++a)
                for (int c = 0; c < n; ++c) SP(out, s, a, n)[c] = -SP(out, s, a, n)[c];
        }
    }
}

/* ------------------------------------------------------------------------- */

int orc_op_init(orc_op *op, const orc_geom *g, int nc, int real_links, int kind, const void *links,
                double kappa, double csw, int gamma5)
{
    memset(op, 0, sizeof(*op));
    if (nc < 1 || nc > 8) return -1;
    op->g = g;
    op->nc = nc;
    op->real_links = real_links;
    op->kind = kind;
    op->links = links;
    op->kappa = kappa;
    op->csw = csw;
    op->gamma5 = gamma5;
    size_t esz = real_links ? sizeof(double) : sizeof(orc_cplx);
    op->F = calloc((size_t)g->V * 6 * nc * nc, esz);
    if (!op->F) return -2;
    if (kind != ORC_WILSON && kind != ORC_SQ_WILSON) update_field_strength(op);
    if (kind == ORC_EO_CLOVER || kind == ORC_SQ_EO_CLOVER) {
        if (nc != 3) return -1; /* the reference hard-codes 3*alpha + c (.cpp:81,295-311) */
        op->Tinv = (orc_cplx *)malloc(sizeof(orc_cplx) * (size_t)g->V * 16 * nc * nc);
        if (!op->Tinv) return -2;
        if (calculate_inverse_even_even(op) != 0) return -3;
    }
    return 0;
}

void orc_op_free(orc_op *op)
{
    free(op->F);
    free(op->Tinv);
    memset(op, 0, sizeof(*op));
}

const void *orc_op_field_strength(const orc_op *op) { return op->F; }

static size_t vec_len(const orc_op *op) { return (size_t)op->g->V * 4 * op->nc; }

static int base_multiply(const orc_op *op, int base_kind, orc_cplx *out, const orc_cplx *in)
{
    switch (base_kind) {
    case ORC_WILSON: wilson_apply(op, out, in, NULL, 0, 0, 0); return 0;
    case ORC_CLOVER: wilson_apply(op, out, in, NULL, 0, 0, 1); return 0;
    case ORC_EO_CLOVER: eo_multiply(op, out, in); return 0;
    default: return -1;
    }
}

int orc_multiply(const orc_op *op, orc_cplx *out, const orc_cplx *in)
{
    switch (op->kind) {
    case ORC_WILSON:
    case ORC_CLOVER:
    case ORC_EO_CLOVER: return base_multiply(op, op->kind, out, in);
    case ORC_SQ_WILSON:
    case ORC_SQ_CLOVER:
    case ORC_SQ_EO_CLOVER: {
        /* Square*Operator::multiply (SquareDiracWilsonOperator.cpp:12-16,
         * SquareImprovedDiracWilsonOperator.cpp:13-17, SquareEvenOdd...cpp:13-17) */
        int base = op->kind - 3;
        orc_cplx *tmp = (orc_cplx *)malloc(sizeof(orc_cplx) * vec_len(op));
        if (!tmp) return -2;
        base_multiply(op, base, tmp, in);
        base_multiply(op, base, out, tmp);
        free(tmp);
        return 0;
    }
    default: return -1;
    }
}

static int multiply_add_c(const orc_op *op, orc_cplx *out, const orc_cplx *v1, const orc_cplx *v2, orc_cplx alpha);

int orc_multiply_add(const orc_op *op, orc_cplx *out, const orc_cplx *v1, const orc_cplx *v2, double alpha_re,
                     double alpha_im)
{
    return multiply_add_c(op, out, v1, v2, CMPLX(alpha_re, alpha_im));
}

static int multiply_add_c(const orc_op *op, orc_cplx *out, const orc_cplx *v1, const orc_cplx *v2, orc_cplx alpha)
{
    switch (op->kind) {
    case ORC_WILSON: wilson_apply(op, out, v1, v2, alpha, 1, 0); return 0;
    case ORC_CLOVER: wilson_apply(op, out, v1, v2, alpha, 1, 1); return 0;
    case ORC_EO_CLOVER: return -5; /* not implemented in the reference: exit(5) (.cpp:49-52) */
    case ORC_SQ_WILSON:
    case ORC_SQ_CLOVER: {
        /* SquareDiracWilsonOperator.cpp:18-22, SquareImprovedDiracWilsonOperator.cpp:19-23 */
        orc_cplx *tmp = (orc_cplx *)malloc(sizeof(orc_cplx) * vec_len(op));
        if (!tmp) return -2;
        base_multiply(op, op->kind - 3, tmp, v1);
        wilson_apply(op, out, tmp, v2, alpha, 1, op->kind == ORC_SQ_CLOVER);
        free(tmp);
        return 0;
    }
    case ORC_SQ_EO_CLOVER: {
        /* SquareEvenOddImprovedDiracWilsonOperator.cpp:19-27 */
        orc_cplx *tmp = (orc_cplx *)malloc(sizeof(orc_cplx) * vec_len(op));
        if (!tmp) return -2;
        eo_multiply(op, tmp, v1);
        eo_multiply(op, out, tmp);
        size_t L = vec_len(op);
        for (size_t k = 0; k < L; ++k) out[k] += alpha * v2[k];
        free(tmp);
        return 0;
    }
    default: return -1;
    }
}

/* ------------------------------------------------------------------------- */
/* AlgebraUtils                                                               */

long double orc_squared_norm(const orc_geom *g, int nc, const orc_cplx *v)
{
    /* AlgebraUtils::squaredNorm (AlgebraUtils.h:17-27) */
    long double result = 0;
    const int per = 4 * nc;
#pragma omp parallel for reduction(+ : result)
    for (int s = 0; s < g->V; ++s) {
        for (int mu = 0; mu < 4; ++mu) {
            double part = 0; /* Eigen's dot of one GaugeVector, FP64 */
            for (int c = 0; c < nc; ++c) {
                orc_cplx z = v[(size_t)s * per + mu * nc + c];
                part += creal(conj(z) * z);
            }
            result += part;
        }
    }
    return result;
}

void orc_dot(const orc_geom *g, int nc, const orc_cplx *a, const orc_cplx *b, long double *re, long double *im)
{
    /* AlgebraUtils::dot (AlgebraUtils.h:182-196): sum conj(a) b */
    long double rr = 0, ii = 0;
    const int per = 4 * nc;
#pragma omp parallel for reduction(+ : rr, ii)
    for (int s = 0; s < g->V; ++s) {
        for (int mu = 0; mu < 4; ++mu) {
            orc_cplx part = 0;
            for (int c = 0; c < nc; ++c) part += conj(a[(size_t)s * per + mu * nc + c]) * b[(size_t)s * per + mu * nc + c];
            rr += creal(part);
            ii += cimag(part);
        }
    }
    *re = rr;
    *im = ii;
}

static orc_cplx dotc(const orc_op *op, const orc_cplx *a, const orc_cplx *b)
{
    long double re, im;
    orc_dot(op->g, op->nc, a, b, &re, &im);
    return CMPLX((double)re, (double)im);
}

/* ------------------------------------------------------------------------- */
/* solvers                                                                    */

int orc_cg(const orc_op *op, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess, double epsilon,
           int max_steps, int *steps)
{
    /* ConjugateGradient::solve (inverters/ConjugateGradient.cpp:10-74) */
    const size_t L = vec_len(op);
    orc_cplx *x = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *r = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!x || !r || !p || !t) return -2;
    memcpy(x, guess ? guess : src, sizeof(orc_cplx) * L);
    orc_multiply(op, t, x);
    for (size_t k = 0; k < L; ++k) {
        r[k] = src[k] - t[k];
        p[k] = r[k];
    }
    long double norm = orc_squared_norm(op->g, op->nc, r), norm_next = norm;
    int ok = 0;
    int step;
    for (step = 0; step < max_steps; ++step) {
        orc_multiply(op, t, p);
        norm = norm_next;
        long double dre, dim;
        orc_dot(op->g, op->nc, p, t, &dre, &dim);
        /* complex<long double>(norm) / dot, then cast to complex<double> */
        long double den = dre * dre + dim * dim;
        orc_cplx alpha = CMPLX((double)(norm * dre / den), (double)(-norm * dim / den));
        for (size_t k = 0; k < L; ++k) {
            x[k] = x[k] + alpha * p[k];
            r[k] = r[k] - alpha * t[k];
        }
        norm_next = orc_squared_norm(op->g, op->nc, r);
        if (norm_next < epsilon) {
            ok = 1;
            break;
        }
        double beta = (double)(norm_next / norm);
        for (size_t k = 0; k < L; ++k) p[k] = r[k] + beta * p[k];
    }
    if (steps) *steps = ok ? step : max_steps;
    memcpy(sol, x, sizeof(orc_cplx) * L);
    free(x); free(r); free(p); free(t);
    return ok;
}

static void seeded_uniform_vector(orc_cplx *v, size_t L)
{
    /* The reference draws a time-seeded uniform vector here
     * (AlgebraUtils.h:123-167); the oracle uses a fixed splitmix64 stream. */
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (size_t k = 0; k < L; ++k) {
        double re, im;
        for (int h = 0; h < 2; ++h) {
            s += 0x9E3779B97F4A7C15ull;
            uint64_t z = s;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
            if (h == 0) re = u; else im = u;
        }
        v[k] = CMPLX(re, im);
    }
}

static int bicgstab_impl(const orc_op *op, const orc_cplx *src, orc_cplx *sol, int shifted, orc_cplx shift,
                         const orc_cplx *guess, double precision, int max_steps, int *steps, double *last_error)
{
    /* BiConjugateGradient::solve (inverters/BiConjugateGradient.cpp:321-507) and the
     * shifted variant (A + shift) (BiConjugateGradient.cpp:510-690). */
    const size_t L = vec_len(op);
    orc_cplx *res = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *rhat = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *nu = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *s = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!res || !rhat || !p || !nu || !s || !t) return -2;
#define APPLY(o, i) (shifted ? multiply_add_c(op, (o), (i), (i), shift) : orc_multiply(op, (o), (i)))
    if (!guess) {
        long double ns = orc_squared_norm(op->g, op->nc, src);
        if (ns > precision) memcpy(sol, src, sizeof(orc_cplx) * L);
        else seeded_uniform_vector(sol, L);
    } else {
        memcpy(sol, guess, sizeof(orc_cplx) * L);
    }
    int rc = APPLY(p, sol);
    if (rc < 0) return rc;
    for (size_t k = 0; k < L; ++k) {
        res[k] = src[k] - p[k];
        rhat[k] = src[k] + p[k];
        p[k] = 0;
        nu[k] = 0;
    }
    orc_cplx alpha = 1, omega = 1;
    long double complex rho = 1;
    double last = 0;
    int step = 0, ok = 0;
    while (step < max_steps) {
        long double rre, rim;
        orc_dot(op->g, op->nc, rhat, res, &rre, &rim);
        long double complex rho_next = rre + rim * I;
        if (rre * rre + rim * rim == 0) {
            ok = 0;
            break; /* breakdown (BiConjugateGradient.cpp:381-384) */
        }
        orc_cplx beta = (orc_cplx)(rho_next / rho) * (alpha / omega);
        for (size_t k = 0; k < L; ++k) p[k] = res[k] + beta * (p[k] - omega * nu[k]);
        APPLY(nu, p);
        long double are, aim;
        orc_dot(op->g, op->nc, rhat, nu, &are, &aim);
        alpha = (orc_cplx)(rho_next / (are + aim * I));
        for (size_t k = 0; k < L; ++k) s[k] = res[k] - alpha * nu[k];
        APPLY(t, s);
        long double t1r, t1i, t2r, t2i;
        orc_dot(op->g, op->nc, t, s, &t1r, &t1i);
        orc_dot(op->g, op->nc, t, t, &t2r, &t2i);
        omega = (orc_cplx)((t1r + t1i * I) / (t2r + t2i * I));
        if (t2r == 0) {
            memcpy(sol, src, sizeof(orc_cplx) * L);
            ok = 1;
            break;
        }
        for (size_t k = 0; k < L; ++k) sol[k] += alpha * p[k] + omega * s[k];
        for (size_t k = 0; k < L; ++k) res[k] = s[k] - omega * t[k];
        long double norm = orc_squared_norm(op->g, op->nc, res);
        if (norm < precision) {
            ok = 1;
            last = (double)norm;
            break;
        }
        rho = rho_next;
        last = (double)norm;
        ++step;
    }
#undef APPLY
    if (steps) *steps = ok ? step : max_steps;
    if (last_error) *last_error = last;
    free(res); free(rhat); free(p); free(nu); free(s); free(t);
    return ok;
}

int orc_bicgstab(const orc_op *op, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess, double precision,
                 int max_steps, int *steps, double *last_error)
{
    return bicgstab_impl(op, src, sol, 0, 0, guess, precision, max_steps, steps, last_error);
}

int orc_bicgstab_shifted(const orc_op *op, const orc_cplx *src, orc_cplx *sol, double shift_re, double shift_im,
                         const orc_cplx *guess, double precision, int max_steps, int *steps, double *last_error)
{
    return bicgstab_impl(op, src, sol, 1, CMPLX(shift_re, shift_im), guess, precision, max_steps, steps,
                         last_error);
}

int orc_preconditioned_bicgstab(const orc_op *op, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess,
                                double precision, int max_steps, int *steps)
{
    /* PreconditionedBiCGStab::solve (inverters/PreconditionedBiCGStab.cpp:33-100) */
    const orc_geom *g = op->g;
    const int n = op->nc;
    const size_t L = vec_len(op);
    int even = (g->dims[0] % 2 == 0) && (g->dims[1] % 2 == 0) && (g->dims[2] % 2 == 0) && (g->dims[3] % 2 == 0);
    if (op->kind != ORC_CLOVER || !even) return orc_bicgstab(op, src, sol, guess, precision, max_steps, steps, NULL);

    orc_op eo, eo_sq;
    /* new EvenOdd... / SquareEvenOdd... : default-constructed, gamma5 = true (DiracOperator.cpp:14) */
    int rc = orc_op_init(&eo, g, n, op->real_links, ORC_EO_CLOVER, op->links, op->kappa, op->csw, 1);
    if (rc < 0) return rc;
    rc = orc_op_init(&eo_sq, g, n, op->real_links, ORC_SQ_EO_CLOVER, op->links, op->kappa, op->csw, 1);
    if (rc < 0) return rc;
    orc_cplx *odd_source = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *odd_source_eo = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *odd_inverse = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *even_inverse = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    memcpy(odd_source, src, sizeof(orc_cplx) * L);
    orc_eo_multiply_even_even_inverse(&eo, odd_source);
    orc_eo_multiply_even_odd(&eo, odd_source, odd_source, 1);
    for (int s = 0; s < g->V; ++s) {
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < n; ++c) {
                orc_cplx v = (parity_of(g, s) == 1) ? SP(src, s, a, n)[c] - SP(odd_source, s, a, n)[c]
                                                     : SP(src, s, a, n)[c];
                SP(odd_source, s, a, n)[c] = (a >= 2) ? -v : v;
            }
    }
    orc_multiply(&eo, odd_source_eo, odd_source);
    int res = orc_bicgstab(&eo_sq, odd_source_eo, odd_inverse, guess, precision, max_steps, steps, NULL);
    orc_eo_multiply_even_odd(&eo, even_inverse, odd_inverse, 0);
    for (int s = 0; s < g->V; ++s)
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < n; ++c) {
                if (parity_of(g, s) == 0) SP(even_inverse, s, a, n)[c] = SP(src, s, a, n)[c] - SP(even_inverse, s, a, n)[c];
                else SP(even_inverse, s, a, n)[c] = SP(odd_inverse, s, a, n)[c];
            }
    orc_eo_multiply_even_even_inverse(&eo, even_inverse);
    memcpy(sol, even_inverse, sizeof(orc_cplx) * L);
    free(odd_source); free(odd_source_eo); free(odd_inverse); free(even_inverse);
    orc_op_free(&eo);
    orc_op_free(&eo_sq);
    return res;
}

static int cg_shift_block(const orc_op *op, const orc_cplx *src, orc_cplx *x, orc_cplx *r, orc_cplx *p,
                          orc_cplx *t, double shift, double epsilon, int max_steps)
{
    /* inner CG of MEMultishiftSolver.cpp:38-79,100-142 (x, r, p initialised by the caller) */
    (void)src;
    const size_t L = vec_len(op);
    int noproblem = 1;
    long double norm_res = orc_squared_norm(op->g, op->nc, r);
    for (int i = 0; i < max_steps; ++i) {
        multiply_add_c(op, t, p, p, shift);
        long double dre, dim;
        orc_dot(op->g, op->nc, p, t, &dre, &dim);
        long double alpha = norm_res / dre;
        for (size_t k = 0; k < L; ++k) {
            x[k] = x[k] + (double)alpha * p[k];
            r[k] = r[k] - (double)alpha * t[k];
        }
        long double error = orc_squared_norm(op->g, op->nc, r);
        if (error < epsilon) break;
        long double beta = error / norm_res;
        for (size_t k = 0; k < L; ++k) p[k] = r[k] + (double)beta * p[k];
        norm_res = error;
        if (i == max_steps - 1) noproblem = 0;
    }
    return noproblem;
}

int orc_me_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols, const double *shifts, int nshift,
                      double epsilon, int max_steps)
{
    /* MEMultishiftSolver::solve (inverters/MEMultishiftSolver.cpp:10-143) */
    const size_t L = vec_len(op);
    orc_cplx *r = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!r || !p || !t) return -2;
    int ok = 1;
    for (size_t k = 0; k < L; ++k) {
        sols[0][k] = 0;
        p[k] = src[k];
        r[k] = src[k];
    }
    ok &= cg_shift_block(op, src, sols[0], r, p, t, shifts[0], epsilon, max_steps);
    for (int i = 1; i < nshift; ++i) {
        multiply_add_c(op, t, sols[i - 1], sols[i - 1], shifts[i]);
        for (size_t k = 0; k < L; ++k) {
            sols[i][k] = sols[i - 1][k];
            r[k] = src[k] - t[k];
            p[k] = src[k] - t[k];
        }
        ok &= cg_shift_block(op, src, sols[i], r, p, t, shifts[i], epsilon, max_steps);
    }
    free(r); free(p); free(t);
    return ok;
}

int orc_mmmr_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols, const double *shifts, int nshift,
                        double epsilon, int max_steps, int *steps)
{
    /* MMMRMultishiftSolver::solve, non-ALIGNED_OPT branch (inverters/MMMRMultishiftSolver.cpp:42-198),
     * over-relaxation omega = 0.95 (:37). */
    const size_t L = vec_len(op);
    const double omega = 0.95;
    orc_cplx *r = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!r || !p || !t) return -2;
    int flag = 1, first = 0;
    while (first < nshift && shifts[first] < 0) {
        for (size_t k = 0; k < L; ++k) {
            sols[first][k] = 0;
            p[k] = src[k];
            r[k] = src[k];
        }
        flag &= cg_shift_block(op, src, sols[first], r, p, t, shifts[first], epsilon, max_steps);
        ++first;
    }
    orc_cplx f[64];
    for (int i = 0; i < nshift; ++i) f[i] = 1;
    for (int i = first; i < nshift; ++i) memset(sols[i], 0, sizeof(orc_cplx) * L);
    memcpy(r, src, sizeof(orc_cplx) * L);
    const double last = shifts[nshift - 1];
    for (int it = 0; it < max_steps; ++it) {
        multiply_add_c(op, p, r, r, last);
        orc_cplx alpha = omega * (dotc(op, p, r) / dotc(op, p, p));
        for (size_t k = 0; k < L; ++k) sols[nshift - 1][k] += alpha * r[k];
        for (int idx = first; idx < nshift - 1; ++idx) {
            f[idx] = f[idx] / (1.0 + (shifts[idx] - last) * alpha);
            for (size_t k = 0; k < L; ++k) sols[idx][k] += f[idx] * alpha * r[k];
        }
        for (size_t k = 0; k < L; ++k) r[k] -= alpha * p[k];
        long double error = orc_squared_norm(op->g, op->nc, r);
        if (error < epsilon) {
            if (steps) *steps = it;
            free(r); free(p); free(t);
            return flag;
        }
    }
    if (steps) *steps = max_steps;
    free(r); free(p); free(t);
    return 0;
}

/* ---------------------------------------------------------------------------------
 * BiCGStab(l): BiConjugateGradient::solve(dirac, source, solution, int l, guess)
 * (inverters/BiConjugateGradient.cpp:130-317).  Inner products as the reference takes
 * them: dot(a, b) = sum conj(a) b in long double, cast to a double complex scalar. */
static orc_cplx cdot_c(const orc_op *op, const orc_cplx *a, const orc_cplx *b)
{
    long double re, im;
    orc_dot(op->g, op->nc, a, b, &re, &im);
    return (double)re + (double)im * I;
}

int orc_bicgstab_l(const orc_op *op, int l, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess,
                   double precision, int max_steps, int *steps, double *last_error)
{
    if (l < 1) return -1;
    const size_t L = vec_len(op);
    orc_cplx *tmp = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *rh = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx **u = (orc_cplx **)malloc(sizeof(orc_cplx *) * (l + 1)), **r = (orc_cplx **)malloc(sizeof(orc_cplx *) * (l + 1));
    for (int j = 0; j <= l; ++j) {
        u[j] = (orc_cplx *)calloc(L, sizeof(orc_cplx));
        r[j] = (orc_cplx *)calloc(L, sizeof(orc_cplx));
    }
    orc_cplx *tau = (orc_cplx *)calloc((size_t)(l + 1) * (l + 1), sizeof(orc_cplx));
    orc_cplx *sigma = (orc_cplx *)calloc(l + 1, sizeof(orc_cplx)), *gam = (orc_cplx *)calloc(l + 1, sizeof(orc_cplx));
    orc_cplx *gp = (orc_cplx *)calloc(l + 1, sizeof(orc_cplx)), *gpp = (orc_cplx *)calloc(l + 1, sizeof(orc_cplx));
#define TAU(i, j) tau[(size_t)(i) * (l + 1) + (j)]
    if (!guess) {
        long double ns = orc_squared_norm(op->g, op->nc, src);
        if (ns > precision) memcpy(sol, src, sizeof(orc_cplx) * L);
        else seeded_uniform_vector(sol, L);
    } else {
        memcpy(sol, guess, sizeof(orc_cplx) * L);
    }
    orc_multiply(op, tmp, sol);
    for (size_t k = 0; k < L; ++k) {
        r[0][k] = src[k] - tmp[k];
        rh[k] = src[k] + tmp[k];
        u[0][k] = 0;
    }
    orc_cplx rho0 = 1, alpha = 0, omega = 1;
    int step = 0, ok = 0;
    double last = 0;
    while (step < max_steps) {
        rho0 = -omega * rho0;
        for (int j = 0; j < l; ++j) {
            const orc_cplx rho1 = cdot_c(op, r[j], rh);
            const orc_cplx beta = (rho1 / rho0) * alpha;
            rho0 = rho1;
            for (int i = 0; i <= j; ++i)
                for (size_t k = 0; k < L; ++k) u[i][k] = r[i][k] - beta * u[i][k];
            orc_multiply(op, u[j + 1], u[j]);
            const orc_cplx gamma = cdot_c(op, u[j + 1], rh);
            alpha = rho0 / gamma;
            for (int i = 0; i <= j; ++i)
                for (size_t k = 0; k < L; ++k) r[i][k] = r[i][k] - alpha * u[i + 1][k];
            orc_multiply(op, r[j + 1], r[j]);
            for (size_t k = 0; k < L; ++k) sol[k] = sol[k] + alpha * u[0][k];
        }
        for (int j = 1; j <= l; ++j) {
            for (int i = 1; i < j; ++i) {
                TAU(i, j) = cdot_c(op, r[j], r[i]) / sigma[i];
                for (size_t k = 0; k < L; ++k) r[j][k] = r[j][k] - TAU(i, j) * r[i][k];
            }
            sigma[j] = cdot_c(op, r[j], r[j]);
            gp[j] = cdot_c(op, r[0], r[j]) / sigma[j];
        }
        gam[l] = gp[l];
        omega = gam[l];
        for (int j = l - 1; j > 0; --j) {
            orc_cplx t = 0;
            for (int i = j + 1; i <= l; ++i) t += TAU(j, i) * gam[i];
            gam[j] = gp[j] - t;
        }
        for (int j = 1; j < l; ++j) {
            orc_cplx t = 0;
            for (int i = j + 1; i < l; ++i) t += TAU(j, i) * gam[i + 1];
            gpp[j] = gam[j + 1] + t;
        }
        for (size_t k = 0; k < L; ++k) sol[k] = sol[k] + gam[1] * r[0][k];
        for (size_t k = 0; k < L; ++k) r[0][k] = r[0][k] - gp[l] * r[l][k];
        for (size_t k = 0; k < L; ++k) u[0][k] = u[0][k] - gam[l] * u[l][k];
        for (int j = 1; j < l; ++j) {
            for (size_t k = 0; k < L; ++k) u[0][k] = u[0][k] - gam[j] * u[j][k];
            for (size_t k = 0; k < L; ++k) sol[k] = sol[k] + gpp[j] * r[j][k];
            for (size_t k = 0; k < L; ++k) r[0][k] = r[0][k] - gp[j] * r[j][k];
        }
        const long double norm = orc_squared_norm(op->g, op->nc, r[0]);
        last = (double)norm;
        if (norm < precision) {
            ok = 1;
            break;
        }
        ++step;
    }
#undef TAU
    if (steps) *steps = ok ? step : max_steps;
    if (last_error) *last_error = last;
    for (int j = 0; j <= l; ++j) {
        free(u[j]);
        free(r[j]);
    }
    free(u); free(r); free(tmp); free(rh); free(tau); free(sigma); free(gam); free(gp); free(gpp);
    return ok;
}

/* ---------------------------------------------------------------------------------
 * BiCGStab with a preconditioner operator P: BiConjugateGradient::solve(dirac, source,
 * solution, preconditioner, guess) (inverters/BiConjugateGradient.cpp:11-128), with the
 * reference's steps as they are: t = A s (not A P s), convergence only after step 5. */
int orc_bicgstab_precond(const orc_op *op, const orc_op *pre, const orc_cplx *src, orc_cplx *sol,
                         const orc_cplx *guess, double precision, int max_steps, int *steps, double *last_error)
{
    const size_t L = vec_len(op);
    orc_cplx *res = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *rhat = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *nu = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *s = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *pt = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *st = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!guess) {
        long double ns = orc_squared_norm(op->g, op->nc, src);
        if (ns > precision) memcpy(sol, src, sizeof(orc_cplx) * L);
        else seeded_uniform_vector(sol, L);
    } else {
        memcpy(sol, guess, sizeof(orc_cplx) * L);
    }
    orc_multiply(op, p, sol);
    for (size_t k = 0; k < L; ++k) {
        res[k] = src[k] - p[k];
        rhat[k] = src[k] + p[k];
    }
    orc_cplx rho_prev = 0, alpha = 0, omega = 0;
    int step = 0, ok = 0, done = 0;
    double last = 0;
    while (step < max_steps) {
        const orc_cplx rho = cdot_c(op, rhat, res);
        if (creal(rho) * creal(rho) + cimag(rho) * cimag(rho) == 0.) {
            done = 1; /* breakdown: false, steps unchanged (BiConjugateGradient.cpp:40) */
            break;
        }
        if (step == 0) {
            memcpy(p, res, sizeof(orc_cplx) * L);
        } else {
            const orc_cplx beta = (rho / rho_prev) * (alpha / omega);
            for (size_t k = 0; k < L; ++k) p[k] = res[k] + beta * (p[k] - omega * nu[k]);
        }
        orc_multiply(pre, pt, p);
        orc_multiply(op, nu, pt);
        alpha = rho / cdot_c(op, rhat, nu);
        for (size_t k = 0; k < L; ++k) s[k] = res[k] - alpha * nu[k];
        orc_multiply(pre, st, s);
        orc_multiply(op, t, s);
        long double dre, dim;
        orc_dot(op->g, op->nc, t, s, &dre, &dim);
        const long double tt = orc_squared_norm(op->g, op->nc, t);
        omega = (double)(dre / tt) + (double)(dim / tt) * I;
        for (size_t k = 0; k < L; ++k) sol[k] = sol[k] + alpha * pt[k] + omega * st[k];
        for (size_t k = 0; k < L; ++k) res[k] = s[k] - omega * t[k];
        const long double norm = orc_squared_norm(op->g, op->nc, res);
        if (norm < precision && step > 5) {
            ok = 1;
            break;
        }
        rho_prev = rho;
        last = (double)norm;
        ++step;
    }
    if (steps) *steps = ok ? step : (done ? step : max_steps);
    if (last_error) *last_error = last;
    free(res); free(rhat); free(p); free(nu); free(s); free(t); free(pt); free(st);
    return ok;
}

/* ---------------------------------------------------------------------------------
 * Chronological multishift: ChronologicalMultishiftSolver::solve
 * (inverters/ChronologicalMultishiftSolver.cpp:11-194).  Shift 0 by CG from zero; every
 * further shift k starts CG from c1 x_{k-1} + c2 h_k, the combination minimising
 * |(A + s_k)(c1 x_{k-1} + c2 h_k) - b| (the reference's closed form).  h_k, the
 * chronological guess, is sols[k] on entry (the reference reads it from uninitialised
 * storage); when the 2x2 system is singular (h_k = 0 or parallel) c2 = 0 and c1
 * minimises the one-vector residual. */
int orc_chrono_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols, const double *shifts, int nshift,
                          double epsilon, int max_steps)
{
    const size_t L = vec_len(op);
    orc_cplx *r = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *p = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    orc_cplx *t = (orc_cplx *)malloc(sizeof(orc_cplx) * L), *gs = (orc_cplx *)malloc(sizeof(orc_cplx) * L);
    if (!r || !p || !t || !gs) return -2;
    int ok = 1;
    for (size_t k = 0; k < L; ++k) {
        sols[0][k] = 0;
        p[k] = src[k];
        r[k] = src[k];
    }
    ok &= cg_shift_block(op, src, sols[0], r, p, t, shifts[0], epsilon, max_steps);
    for (int i = 1; i < nshift; ++i) {
        multiply_add_c(op, p, sols[i - 1], sols[i - 1], shifts[i]);
        multiply_add_c(op, t, sols[i], sols[i], shifts[i]);
        long double re, im;
        const long double pApA = orc_squared_norm(op->g, op->nc, p), hAhA = orc_squared_norm(op->g, op->nc, t);
        orc_dot(op->g, op->nc, p, src, &re, &im);
        const long double complex pAb = re + im * I;
        orc_dot(op->g, op->nc, t, src, &re, &im);
        const long double complex hAb = re + im * I;
        orc_dot(op->g, op->nc, t, p, &re, &im);
        const long double complex hApA = re + im * I;
        const long double complex den = -(hAhA * pApA) + hApA * conjl(hApA);
        orc_cplx c1, c2;
        if (cabsl(den) > 1e-12L * hAhA * pApA && hAhA > 0) {
            const long double c1R = creall((-(hAhA * pAb) + hApA * conjl(hAb) + hAb * conjl(hApA) - hAhA * conjl(pAb)) /
                                           (2.0L * den));
            const long double c1I = creall((-0.5L * I) * (-(hAhA * pAb) - hApA * conjl(hAb) + hAb * conjl(hApA) +
                                                          hAhA * conjl(pAb)) / den);
            const long double c2R = creall((hApA * pAb - hAb * pApA - pApA * conjl(hAb) + conjl(hApA) * conjl(pAb)) /
                                           (2.0L * den));
            const long double c2I = creall((-0.5L * I) * (hApA * pAb - hAb * pApA + pApA * conjl(hAb) -
                                                          conjl(hApA) * conjl(pAb)) / den);
            c1 = (double)c1R + (double)c1I * I;
            c2 = (double)c2R + (double)c2I * I;
        } else {
            c1 = pApA > 0 ? (orc_cplx)(pAb / pApA) : 0;
            c2 = 0;
        }
        for (size_t k = 0; k < L; ++k) gs[k] = c1 * sols[i - 1][k] + c2 * sols[i][k];
        multiply_add_c(op, t, gs, gs, shifts[i]);
        for (size_t k = 0; k < L; ++k) {
            sols[i][k] = gs[k];
            r[k] = src[k] - t[k];
            p[k] = src[k] - t[k];
        }
        ok &= cg_shift_block(op, src, sols[i], r, p, t, shifts[i], epsilon, max_steps);
    }
    free(r); free(p); free(t); free(gs);
    return ok;
}
