/*
 * CPU oracle for the Wilson / Wilson-clover hot path of LeonardYM.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker.  Nothing in the product (leonardym_b200/) links,
 * loads or calls it.
 *
 * Every routine cites the reference file:line it restates (paths relative to
 * the LeonardYM source tree, source/...).  The restatement is pinned against
 * outputs of the reference's own code compiled from its sources
 * (oracle/build_ref.sh -> oracle/_ref/), see tests/test_oracle_pins.py and the
 * committed fixtures in tests/golden/.
 *
 * Memory conventions mirror the reference's raw Lattice storage
 * (MPILattice/Lattice.h:18-248, LatticeDefinitions.h:86-161):
 *   spinor  : double complex [V][4 spins][nc colours]           (GaugeVector[4])
 *   links   : [V][4 mu][nc*nc] column-major (i,j) -> j*nc+i;
 *             double complex (fundamental) or double (adjoint, real links)
 *   F       : [V][6][nc*nc]  same element type as the links
 *   site    : t + Lt*(z + Lz*(y + Ly*x))                (LocalLayout.h:149-163)
 */
#ifndef LYM_ORACLE_H
#define LYM_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double complex orc_cplx;

typedef struct {
    int dims[4];   /* glob_x, glob_y, glob_z, glob_t */
    int V;
    int *sup;      /* [V][4] */
    int *sdn;      /* [V][4] */
    int *coord;    /* [V][4] x,y,z,t */
} orc_geom;

enum orc_kind {
    ORC_WILSON = 0,         /* DiracWilsonOperator                      */
    ORC_CLOVER = 1,         /* ImprovedDiracWilsonOperator              */
    ORC_EO_CLOVER = 2,      /* EvenOddImprovedDiracWilsonOperator       */
    ORC_SQ_WILSON = 3,      /* SquareDiracWilsonOperator                */
    ORC_SQ_CLOVER = 4,      /* SquareImprovedDiracWilsonOperator        */
    ORC_SQ_EO_CLOVER = 5    /* SquareEvenOddImprovedDiracWilsonOperator */
};

typedef struct {
    const orc_geom *g;
    int nc;                 /* diracVectorLength */
    int real_links;         /* 1: adjoint representation, real links */
    int kind;
    const void *links;      /* fermion links (BCs folded in) */
    void *F;                /* field strength, owned */
    orc_cplx *Tinv;         /* 12x12 inverse clover matrices per site, owned (EO) */
    double kappa, csw;
    int gamma5;
} orc_op;

/* geometry: LocalLayout::initialize (MPILattice/LocalLayout.h:34-110) */
int  orc_geom_init(orc_geom *g, const int dims[4]);
void orc_geom_free(orc_geom *g);
int  orc_geom_tables(const int dims[4], int *sup, int *sdn, int *coord);

/* boundary conditions: switchAntiperiodicBc (LatticeBoundaryConditions.h:8-14) */
void orc_antiperiodic_bc(const int dims[4], void *links, int nc, int real_links);

/* SU(2) -> adjoint: ConvertLattice::toAdjoint (utils/ConvertLattice.h:24-34,100-105) */
void orc_su2_to_adjoint(int nlinks, const orc_cplx *fund, double *adj);

/* operator life cycle: setLattice / updateFieldStrength / calculateInverseEvenEven */
int  orc_op_init(orc_op *op, const orc_geom *g, int nc, int real_links, int kind,
                 const void *links, double kappa, double csw, int gamma5);
void orc_op_free(orc_op *op);

/* DiracOperator::multiply / multiplyAdd for every kind; 0 ok, <0 error */
int  orc_multiply(const orc_op *op, orc_cplx *out, const orc_cplx *in);
int  orc_multiply_add(const orc_op *op, orc_cplx *out, const orc_cplx *v1,
                      const orc_cplx *v2, double alpha_re, double alpha_im);

/* EO building blocks (EvenOddImprovedDiracWilsonOperator.cpp:61-281) */
void orc_eo_multiply_even_odd(const orc_op *op, orc_cplx *out, const orc_cplx *in, int part);
void orc_eo_multiply_even_even_inverse(const orc_op *op, orc_cplx *out);
void orc_eo_multiply_odd_odd_minus_identity(const orc_op *op, orc_cplx *out,
                                            const orc_cplx *in, int part);

/* field strength export (6 x nc x nc per site, same element type as links) */
const void *orc_op_field_strength(const orc_op *op);

/* AlgebraUtils (algebra_utils/AlgebraUtils.h:17-27,182-196) */
long double orc_squared_norm(const orc_geom *g, int nc, const orc_cplx *v);
void orc_dot(const orc_geom *g, int nc, const orc_cplx *a, const orc_cplx *b,
             long double *re, long double *im);

/* solvers; return 1 converged, 0 not converged, <0 error */
int orc_cg(const orc_op *op, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess,
           double epsilon, int max_steps, int *steps);
int orc_bicgstab(const orc_op *op, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess,
                 double precision, int max_steps, int *steps, double *last_error);
int orc_bicgstab_shifted(const orc_op *op, const orc_cplx *src, orc_cplx *sol,
                         double shift_re, double shift_im,
                         const orc_cplx *guess, double precision, int max_steps, int *steps,
                         double *last_error);
int orc_preconditioned_bicgstab(const orc_op *op, const orc_cplx *src, orc_cplx *sol,
                                const orc_cplx *guess, double precision, int max_steps,
                                int *steps);
int orc_me_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols,
                      const double *shifts, int nshift, double epsilon, int max_steps);
int orc_mmmr_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols,
                        const double *shifts, int nshift, double epsilon, int max_steps,
                        int *steps);
int orc_bicgstab_l(const orc_op *op, int l, const orc_cplx *src, orc_cplx *sol, const orc_cplx *guess,
                   double precision, int max_steps, int *steps, double *last_error);
int orc_bicgstab_precond(const orc_op *op, const orc_op *pre, const orc_cplx *src, orc_cplx *sol,
                         const orc_cplx *guess, double precision, int max_steps, int *steps, double *last_error);
int orc_chrono_multishift(const orc_op *op, const orc_cplx *src, orc_cplx **sols, const double *shifts, int nshift,
                          double epsilon, int max_steps);

#ifdef __cplusplus
}
#endif
#endif
