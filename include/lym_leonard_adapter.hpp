// lym_leonard_adapter.hpp -- header-only binding of liblym_b200 (include/lym_b200.h)
// into LeonardYM's own class hierarchy, for a maintainer to compile inside the
// reference (it includes the reference's headers).  The classes subclass the
// reference interfaces so existing callers (Solver::solve, MultishiftSolver::solve,
// DiracOperator::multiply/multiplyAdd) keep working unchanged:
//
//   GpuDiracOperator<Base, Kind>   : Base  (DiracWilsonOperator, ImprovedDiracWilsonOperator,
//                                           EvenOddImprovedDiracWilsonOperator and the Square* ones)
//     setLattice -> lym_gauge_upload of the raw extended_fermion_lattice_t storage
//     multiply / multiplyAdd -> lym_multiply / lym_multiply_add on the raw vector storage
//   GpuSolver       : Solver            -> lym_solve     (inverters/Solver.h:13)
//   GpuPreconditionedBiCGStab : PreconditionedBiCGStab -> lym_solve (LYM_SOLVER_EO_BICGSTAB), for
//                       the callers that build that solver themselves (MesonCorrelator.cpp:70,
//                       ChiralCondensate.cpp:51); any ImprovedDiracWilsonOperator, GPU or not
//   GpuMultishiftSolver : MultishiftSolver -> lym_multishift (inverters/MultishiftSolver.h:28)
//   GpuFermionForce : ImprovedFermionForce, what GpuDiracOperator::getForce returns
//     derivative(force, lattice, X, Y, weight) -> lym_fermion_force (hmc_forces/FermionForce.h:15)
//
// Requirements: single process (no ENABLE_MPI), LocalLayout initialised, even glob_t.
// Errors: the reference calls exit() on misuse; these adapters print the library's
// message and return false (solvers) or leave the output untouched (operators).
#ifndef LYM_LEONARD_ADAPTER_HPP
#define LYM_LEONARD_ADAPTER_HPP

#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "dirac_operators/DiracWilsonOperator.h"
#include "dirac_operators/EvenOddImprovedDiracWilsonOperator.h"
#include "dirac_operators/ImprovedDiracWilsonOperator.h"
#include "dirac_operators/SquareDiracWilsonOperator.h"
#include "dirac_operators/SquareEvenOddImprovedDiracWilsonOperator.h"
#include "dirac_operators/SquareImprovedDiracWilsonOperator.h"
#include "hmc_forces/ImprovedFermionForce.h"
#include "inverters/MultishiftSolver.h"
#include "inverters/PreconditionedBiCGStab.h"
#include "inverters/Solver.h"
#include "lym_b200.h"

namespace Update {

// One library context per process, for the geometry of the static LocalLayout.
inline lym_context *lym_global_context()
{
    static lym_context *ctx = nullptr;
    static int dims[4] = {0, 0, 0, 0};
    typedef Lattice::LocalLayout LL;
    const int want[4] = {LL::glob_x, LL::glob_y, LL::glob_z, LL::glob_t};
    if (ctx && (dims[0] != want[0] || dims[1] != want[1] || dims[2] != want[2] || dims[3] != want[3])) {
        lym_context_destroy(ctx);
        ctx = nullptr;
    }
    if (!ctx) {
#ifdef ADJOINT
        const int rep = LYM_REP_SU2_ADJOINT;
#else
        const int rep = LYM_REP_SU3_FUNDAMENTAL;
#endif
        if (lym_context_create(want, rep, 0, &ctx) != LYM_OK) {
            std::cerr << "lym_context_create failed" << std::endl;
            return nullptr;
        }
        for (int k = 0; k < 4; ++k) dims[k] = want[k];
    }
    return ctx;
}

inline int lym_next_gauge_id()
{
    static int next = 1;
    return next++;
}

class GpuFermionForce;

template <class Base, int Kind> class GpuDiracOperator : public Base {
public:
    GpuDiracOperator() : Base(), op_(-1), gauge_(lym_next_gauge_id()) {}
    ~GpuDiracOperator()
    {
        lym_context *c = lym_global_context();
        if (c && op_ >= 0) lym_operator_destroy(c, op_);
        if (c) lym_gauge_evict(c, gauge_);
    }

    virtual void setLattice(const extended_fermion_lattice_t &lat)
    {
        this->DiracOperator::setLattice(lat);  // keeps the host copy getLattice() returns
        lym_context *c = lym_global_context();
        if (!c) return;
        if (lym_gauge_upload(c, gauge_, reinterpret_cast<const double *>(lat.getRawData())) != LYM_OK) report(c);
        if (op_ < 0 && lym_operator_create(c, gauge_, Kind, this->kappa, csw_of(), this->gamma5, &op_) != LYM_OK)
            report(c);
        else if (op_ >= 0)
            lym_operator_set_gauge(c, op_, gauge_);
    }

    virtual void multiply(reduced_dirac_vector_t &output, const reduced_dirac_vector_t &input)
    {
        lym_context *c = sync();
        if (c && lym_multiply(c, op_, reinterpret_cast<double *>(output.getRawData()),
                              reinterpret_cast<const double *>(input.getRawData())) != LYM_OK)
            report(c);
    }

    virtual void multiplyAdd(reduced_dirac_vector_t &output, const reduced_dirac_vector_t &vector1,
                             const reduced_dirac_vector_t &vector2, const complex &alpha)
    {
        lym_context *c = sync();
        if (c && lym_multiply_add(c, op_, reinterpret_cast<double *>(output.getRawData()),
                                  reinterpret_cast<const double *>(vector1.getRawData()),
                                  reinterpret_cast<const double *>(vector2.getRawData()), alpha.real(),
                                  alpha.imag()) != LYM_OK)
            report(c);
    }

    int operatorId() { return sync() ? op_ : -1; }

    // DiracOperator::getForce (dirac_operators/DiracOperator.h:101): the fermion force of this
    // operator on the GPU (the library picks the Wilson or the improved force by the kind)
    virtual FermionForce *getForce() const;

protected:
    // kappa, csw and gamma5 are plain members of the reference classes (setGamma5 and
    // setCSW are not virtual), so they are pushed to the library before every use.
    lym_context *sync()
    {
        lym_context *c = lym_global_context();
        if (!c || op_ < 0) return nullptr;
        lym_operator_set_kappa(c, op_, this->kappa);
        lym_operator_set_csw(c, op_, csw_of());
        lym_operator_set_gamma5(c, op_, this->gamma5);
        return c;
    }
    double csw_of() const { return csw_helper(this); }
    static double csw_helper(const ImprovedDiracWilsonOperator *o) { return o->getCSW(); }
    static double csw_helper(const SquareImprovedDiracWilsonOperator *o) { return o->getCSW(); }
    static double csw_helper(const SquareEvenOddImprovedDiracWilsonOperator *o) { return o->getCSW(); }
    static double csw_helper(const void *) { return 0.0; }
    static void report(lym_context *c) { std::cerr << "liblym_b200: " << lym_last_error(c) << std::endl; }
    int op_;
    int gauge_;
};

typedef GpuDiracOperator<DiracWilsonOperator, LYM_OP_DIRAC_WILSON> GpuDiracWilsonOperator;
typedef GpuDiracOperator<ImprovedDiracWilsonOperator, LYM_OP_IMPROVED> GpuImprovedDiracWilsonOperator;
typedef GpuDiracOperator<EvenOddImprovedDiracWilsonOperator, LYM_OP_EVEN_ODD_IMPROVED> GpuEvenOddImprovedDiracWilsonOperator;
typedef GpuDiracOperator<SquareDiracWilsonOperator, LYM_OP_SQUARE_DIRAC_WILSON> GpuSquareDiracWilsonOperator;
typedef GpuDiracOperator<SquareImprovedDiracWilsonOperator, LYM_OP_SQUARE_IMPROVED> GpuSquareImprovedDiracWilsonOperator;
typedef GpuDiracOperator<SquareEvenOddImprovedDiracWilsonOperator, LYM_OP_SQUARE_EVEN_ODD_IMPROVED>
    GpuSquareEvenOddImprovedDiracWilsonOperator;

// operator id of a Gpu* operator, -1 for any other DiracOperator
inline int lym_operator_of(DiracOperator *d)
{
    if (auto o = dynamic_cast<GpuDiracWilsonOperator *>(d)) return o->operatorId();
    if (auto o = dynamic_cast<GpuImprovedDiracWilsonOperator *>(d)) return o->operatorId();
    if (auto o = dynamic_cast<GpuEvenOddImprovedDiracWilsonOperator *>(d)) return o->operatorId();
    if (auto o = dynamic_cast<GpuSquareDiracWilsonOperator *>(d)) return o->operatorId();
    if (auto o = dynamic_cast<GpuSquareImprovedDiracWilsonOperator *>(d)) return o->operatorId();
    if (auto o = dynamic_cast<GpuSquareEvenOddImprovedDiracWilsonOperator *>(d)) return o->operatorId();
    return -1;
}

// FermionForce::derivative (hmc_forces/FermionForce.cpp:11-20) on the GPU for the operator
// that created it: force[x][mu] -= weight * F_mu(x) on the raw force-lattice storage.
class GpuFermionForce : public ImprovedFermionForce {
public:
    GpuFermionForce(DiracOperator *op, real_t kappa, real_t csw) : ImprovedFermionForce(kappa, csw), op_(op) {}
    using ImprovedFermionForce::derivative;
    virtual void derivative(extended_fermion_force_lattice_t &fermionForce, const extended_fermion_lattice_t &,
                            const extended_dirac_vector_t &X, const extended_dirac_vector_t &Y, real_t weight)
    {
        lym_context *c = lym_global_context();
        const int op = lym_operator_of(op_);
        if (!c || op < 0)
            throw std::runtime_error("GpuFermionForce needs the Gpu* DiracOperator that created it");
        if (lym_fermion_force(c, op, reinterpret_cast<const double *>(X.getRawData()),
                              reinterpret_cast<const double *>(Y.getRawData()), weight,
                              reinterpret_cast<double *>(fermionForce.getRawData())) != LYM_OK)
            throw std::runtime_error(std::string("liblym_b200: ") + lym_last_error(c));
    }

private:
    DiracOperator *op_;
};

template <class Base, int Kind> FermionForce *GpuDiracOperator<Base, Kind>::getForce() const
{
    return new GpuFermionForce(const_cast<GpuDiracOperator *>(this), this->kappa, csw_of());
}

// Solver::solve on the GPU; `algorithm` is a lym_solver value.
class GpuSolver : public Solver {
public:
    explicit GpuSolver(int algorithm = LYM_SOLVER_EO_BICGSTAB) : Solver("GpuSolver"), algorithm_(algorithm) {}
    using Solver::solve;
    virtual bool solve(DiracOperator *dirac, const reduced_dirac_vector_t &source, reduced_dirac_vector_t &solution,
                       reduced_dirac_vector_t const *initial_guess = 0)
    {
        lym_context *c = lym_global_context();
        const int op = lym_operator_of(dirac);
        if (!c || op < 0) {
            std::cerr << "GpuSolver needs a Gpu* DiracOperator" << std::endl;
            return false;
        }
        lym_solve_stats st;
        const int rc = lym_solve(c, op, algorithm_, precision, (int)maxSteps,
                                 reinterpret_cast<const double *>(source.getRawData()),
                                 reinterpret_cast<double *>(solution.getRawData()),
                                 initial_guess ? reinterpret_cast<const double *>(initial_guess->getRawData()) : 0, &st);
        lastSteps = st.steps;
        lastError = st.last_error;
        if (rc < 0) std::cerr << "liblym_b200: " << lym_last_error(c) << std::endl;
        return rc == LYM_OK;
    }

private:
    int algorithm_;
};

// PreconditionedBiCGStab::solve (inverters/PreconditionedBiCGStab.cpp:33-100) with the whole
// solve on the GPU: source preparation, BiCGStab on the even-odd Schur system and the
// reconstruction run in the library (LYM_SOLVER_EO_BICGSTAB, the reference's iteration step
// for step in FP64; getLastSteps() is the inner BiCGStab's step count, as the reference's).
// The callers that create this solver themselves (MesonCorrelator.cpp:70,
// ChiralCondensate.cpp:51) switch to it by changing that one `new`.  A Gpu* Improved operator
// is solved as it is; any other ImprovedDiracWilsonOperator has its links, kappa and c_sw
// uploaded for the call (and released after it).  With even-odd preconditioning switched
// off through this class, the plain BiCGStab on D (PreconditionedBiCGStab.cpp:94-96,
// LYM_SOLVER_BICGSTAB).  Operators that are not ImprovedDiracWilsonOperator go to the
// reference's own solver, as before.
class GpuPreconditionedBiCGStab : public PreconditionedBiCGStab {
public:
    GpuPreconditionedBiCGStab() : PreconditionedBiCGStab(), even_odd_(true) {}
    using PreconditionedBiCGStab::solve;

    // PreconditionedBiCGStab::setUseEvenOddPreconditioning is not virtual: call it on this type
    void setUseEvenOddPreconditioning(bool eo)
    {
        even_odd_ = eo;
        PreconditionedBiCGStab::setUseEvenOddPreconditioning(eo);
    }

    virtual bool solve(DiracOperator *dirac, const reduced_dirac_vector_t &source, reduced_dirac_vector_t &solution,
                       reduced_dirac_vector_t const *initial_guess = 0)
    {
        ImprovedDiracWilsonOperator *imp = dynamic_cast<ImprovedDiracWilsonOperator *>(dirac);
        lym_context *c = imp ? lym_global_context() : nullptr;
        if (!c) return PreconditionedBiCGStab::solve(dirac, source, solution, 0, initial_guess);
        int op = lym_operator_of(dirac);
        int tmp_gauge = -1, tmp_op = -1;
        if (op < 0) {  // a CPU operator: its links, kappa, c_sw and gamma5 for this call
            tmp_gauge = lym_next_gauge_id();
            if (lym_gauge_upload(c, tmp_gauge, reinterpret_cast<const double *>(imp->getLattice()->getRawData())) !=
                    LYM_OK ||
                lym_operator_create(c, tmp_gauge, LYM_OP_IMPROVED, imp->getKappa(), imp->getCSW(), imp->getGamma5(),
                                    &tmp_op) != LYM_OK) {
                std::cerr << "liblym_b200: " << lym_last_error(c) << std::endl;
                release(c, tmp_gauge, tmp_op);
                return false;
            }
            op = tmp_op;
        }
        lym_solve_stats st;
        const int rc = lym_solve(c, op, even_odd_ ? LYM_SOLVER_EO_BICGSTAB : LYM_SOLVER_BICGSTAB, precision,
                                 (int)maxSteps, reinterpret_cast<const double *>(source.getRawData()),
                                 reinterpret_cast<double *>(solution.getRawData()),
                                 initial_guess ? reinterpret_cast<const double *>(initial_guess->getRawData()) : 0,
                                 &st);
        lastSteps = st.steps;
        lastError = st.last_error;
        if (rc < 0) std::cerr << "liblym_b200: " << lym_last_error(c) << std::endl;
        release(c, tmp_gauge, tmp_op);
        return rc == LYM_OK;
    }

private:
    static void release(lym_context *c, int gauge, int op)
    {
        if (op >= 0) lym_operator_destroy(c, op);
        if (gauge >= 0) lym_gauge_evict(c, gauge);
    }
    bool even_odd_;
};

// MultishiftSolver::solve on the GPU; `algorithm` is a lym_multishift_solver value.
class GpuMultishiftSolver : public MultishiftSolver {
public:
    explicit GpuMultishiftSolver(int algorithm = LYM_MULTISHIFT_CG, real_t epsilon = 0.00000001,
                                 unsigned int maxSteps = 3000)
        : MultishiftSolver(epsilon, maxSteps), algorithm_(algorithm)
    {
    }
    virtual bool solve(DiracOperator *dirac, const extended_dirac_vector_t &source,
                       std::vector<extended_dirac_vector_t> &solutions, const std::vector<real_t> &shifts)
    {
        lym_context *c = lym_global_context();
        const int op = lym_operator_of(dirac);
        if (!c || op < 0) return false;
        if (solutions.size() < shifts.size()) solutions.resize(shifts.size());
        std::vector<double *> out(shifts.size());
        for (size_t i = 0; i < shifts.size(); ++i) out[i] = reinterpret_cast<double *>(solutions[i].getRawData());
        lym_solve_stats st;
        const int rc = lym_multishift(c, op, algorithm_, (int)shifts.size(), shifts.data(), epsilon, (int)maxSteps,
                                      reinterpret_cast<const double *>(source.getRawData()), out.data(), &st);
        if (rc < 0) std::cerr << "liblym_b200: " << lym_last_error(c) << std::endl;
        return rc == LYM_OK;
    }

private:
    int algorithm_;
};

}  // namespace Update

#endif
