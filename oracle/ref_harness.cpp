// C entry points around LeonardYM's own hot-path classes, compiled from the
// reference sources by oracle/build_ref.sh into oracle/_ref/.  TEST
// INFRASTRUCTURE ONLY: it pins the oracle restatement (tests/test_oracle_pins.py)
// and generates the golden fixtures (tests/golden/make_golden.py).
//
// One library per representation: NUMCOLORS=3 (fundamental) and NUMCOLORS=2
// with ADJOINT.  The layout is the reference's process-global LocalLayout, so
// every entry point (re)initialises it for the requested extents.
#include <cstring>
#include <vector>

#include "algebra_utils/AlgebraUtils.h"
#include "dirac_functions/RationalApproximation.h"
#include "hmc_forces/DiracWilsonFermionForce.h"
#include "hmc_forces/ImprovedFermionForce.h"
#include "dirac_operators/DiracWilsonOperator.h"
#include "dirac_operators/EvenOddImprovedDiracWilsonOperator.h"
#include "dirac_operators/ImprovedDiracWilsonOperator.h"
#include "dirac_operators/SquareDiracWilsonOperator.h"
#include "dirac_operators/SquareEvenOddImprovedDiracWilsonOperator.h"
#include "dirac_operators/SquareImprovedDiracWilsonOperator.h"
#include "dirac_operators/BasicDiracWilsonOperator.h"
#include "inverters/BiConjugateGradient.h"
#include "inverters/ConjugateGradient.h"
#include "inverters/MEMultishiftSolver.h"
#include "inverters/MMMRMultishiftSolver.h"
#include "inverters/ChronologicalMultishiftSolver.h"
#include "inverters/PreconditionedBiCGStab.h"
#include "utils/ConvertLattice.h"
#include "correlators/MesonCorrelator.h"
#include "io/OutputSweep.h"
#include "starters/ReadStartGaugeConfiguration.h"
#include "fermion_measurements/ChiralCondensate.h"
#include <omp.h>
#include <sstream>
#include <string>

using namespace Update;

namespace {

int g_dims[4] = {0, 0, 0, 0};

void init_layout(const int d[4])
{
    if (g_dims[0] == d[0] && g_dims[1] == d[1] && g_dims[2] == d[2] && g_dims[3] == d[3]) return;
    Lattice::LocalLayout::glob_x = d[0];
    Lattice::LocalLayout::glob_y = d[1];
    Lattice::LocalLayout::glob_z = d[2];
    Lattice::LocalLayout::glob_t = d[3];
    Lattice::LocalLayout::initialize();
    for (int k = 0; k < 4; ++k) g_dims[k] = d[k];
}

template <class L> void load(L &lat, const double *raw)
{
    std::memcpy((void *)lat.getRawData(), raw, sizeof(typename L::TData) * lat.localsize);
}
template <class L> void store(const L &lat, double *raw)
{
    std::memcpy(raw, (const void *)lat.getRawData(), sizeof(typename L::TData) * lat.localsize);
}

// exposes the protected field strength of ImprovedDiracWilsonOperator
struct FieldStrengthAccess : public ImprovedDiracWilsonOperator {
    const reduced_field_strength_lattice_t &field() const { return F; }
};

DiracOperator *make_operator(int kind, double kappa, double csw, int gamma5, const extended_fermion_lattice_t &links)
{
    DiracOperator *op = nullptr;
    switch (kind) {
    case 0: op = new DiracWilsonOperator(); break;
    case 1: op = new ImprovedDiracWilsonOperator(); break;
    case 2: op = new EvenOddImprovedDiracWilsonOperator(); break;
    case 3: op = new SquareDiracWilsonOperator(); break;
    case 4: op = new SquareImprovedDiracWilsonOperator(); break;
    case 5: op = new SquareEvenOddImprovedDiracWilsonOperator(); break;
    case 6: op = new BasicDiracWilsonOperator(); break;
    default: return nullptr;
    }
    op->setKappa(kappa);
    if (kind == 1 || kind == 2) static_cast<ImprovedDiracWilsonOperator *>(op)->setCSW(csw);
    if (kind == 4) static_cast<SquareImprovedDiracWilsonOperator *>(op)->setCSW(csw);
    if (kind == 5) static_cast<SquareEvenOddImprovedDiracWilsonOperator *>(op)->setCSW(csw);
    op->setLattice(links);
    op->setGamma5(gamma5 != 0);
    return op;
}

}  // namespace

extern "C" {

int ref_dirac_vector_length() { return diracVectorLength; }
int ref_link_doubles() { return (int)(sizeof(FermionicGroup) / sizeof(double)); }

int ref_neighbours(const int dims[4], int *sup, int *sdn)
{
    init_layout(dims);
    const int V = Lattice::LocalLayout::localsize;
    for (int s = 0; s < V; ++s)
        for (int mu = 0; mu < 4; ++mu) {
            sup[s * 4 + mu] = reduced_dirac_vector_t::sup(s, mu);
            sdn[s * 4 + mu] = reduced_dirac_vector_t::sdn(s, mu);
        }
    return 0;
}

// switchAntiperiodicBc on a fermion link field (in place)
int ref_antiperiodic(const int dims[4], double *links)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    switchAntiperiodicBc(L);
    store(L, links);
    return 0;
}

#ifdef ADJOINT
// ConvertLattice::toAdjoint on nlinks SU(2) links (complex 2x2 column-major)
int ref_to_adjoint(int nlinks, const double *fund, double *adj)
{
    for (int l = 0; l < nlinks; ++l) {
        GaugeGroup U;
        std::memcpy((void *)U.data(), fund + 8 * (size_t)l, sizeof(GaugeGroup));
        AdjointGroup A;
        ConvertLattice<extended_fermion_lattice_t, extended_gauge_lattice_t>::toAdjoint(U, A);
        std::memcpy(adj + 9 * (size_t)l, (const void *)A.data(), sizeof(AdjointGroup));
    }
    return 0;
}
#endif

int ref_multiply(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links,
                 const double *in, double *out)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    reduced_dirac_vector_t x, y;
    load(x, in);
    op->multiply(y, x);
    store(y, out);
    delete op;
    return 0;
}

int ref_multiply_add(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links,
                     const double *v1, const double *v2, double are, double aim, double *out)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    reduced_dirac_vector_t a, b, y;
    load(a, v1);
    load(b, v2);
    op->multiplyAdd(y, a, b, complex(are, aim));
    store(y, out);
    delete op;
    return 0;
}

int ref_field_strength(const int dims[4], double kappa, double csw, const double *links, double *F)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    FieldStrengthAccess op;
    op.setKappa(kappa);
    op.setCSW(csw);
    op.setLattice(L);
    store(op.field(), F);
    return 0;
}

// solver = 0 ConjugateGradient, 1 BiConjugateGradient, 2 PreconditionedBiCGStab,
// 3 BiConjugateGradient shifted by (are, aim)
int ref_solve(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links, int solver,
              double precision, int max_steps, double are, double aim, const double *src, double *sol, int *steps)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    reduced_dirac_vector_t b, x;
    load(b, src);
    bool ok = false;
    if (solver == 0) {
        ConjugateGradient cg;
        cg.setPrecision(precision);
        cg.setMaximumSteps(max_steps);
        ok = cg.solve(op, b, x);
        *steps = cg.getLastSteps();
    } else if (solver == 1 || solver == 3) {
        BiConjugateGradient bi;
        bi.setPrecision(precision);
        bi.setMaximumSteps(max_steps);
        ok = solver == 1 ? bi.solve(op, b, x) : bi.solve(op, b, x, complex(are, aim));
        *steps = bi.getLastSteps();
    } else if (solver == 2) {
        PreconditionedBiCGStab pb;
        pb.setPrecision(precision);
        pb.setMaximumSteps(max_steps);
        ok = pb.solve(op, b, x);
        *steps = pb.getLastSteps();
    } else {
        delete op;
        return -1;
    }
    store(x, sol);
    delete op;
    return ok ? 1 : 0;
}

// solver 0: BiConjugateGradient::solve(op, b, x, int l) (BiCGStab(l), l = ival);
// solver 1: BiConjugateGradient::solve(op, b, x, preconditioner) with the preconditioner an
// operator of kind pkind (pkappa, pcsw, gamma5 as the solved operator)
int ref_solve2(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links, int solver,
               double precision, int max_steps, int ival, int pkind, double pkappa, double pcsw, const double *src,
               double *sol, int *steps)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    reduced_dirac_vector_t b, x;
    load(b, src);
    BiConjugateGradient bi;
    bi.setPrecision(precision);
    bi.setMaximumSteps(max_steps);
    bool ok = false;
    if (solver == 0) {
        ok = bi.solve(op, b, x, ival);
    } else if (solver == 1) {
        DiracOperator *pre = make_operator(pkind, pkappa, pcsw, gamma5, L);
        if (!pre) {
            delete op;
            return -1;
        }
        ok = bi.solve(op, b, x, pre);
        delete pre;
    } else {
        delete op;
        return -1;
    }
    *steps = bi.getLastSteps();
    store(x, sol);
    delete op;
    return ok ? 1 : 0;
}

// algorithm 0 MEMultishiftSolver, 1 MMMRMultishiftSolver, 2 ChronologicalMultishiftSolver
int ref_multishift(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links,
                   int algorithm, int nshift, const double *shifts, double epsilon, int max_steps, const double *src,
                   double **sols)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    extended_dirac_vector_t b;
    load(b, src);
    std::vector<extended_dirac_vector_t> xs(nshift);
    std::vector<real_t> sh(shifts, shifts + nshift);
    MultishiftSolver *ms = algorithm == 0   ? (MultishiftSolver *)new MEMultishiftSolver(epsilon, max_steps)
                           : algorithm == 1 ? (MultishiftSolver *)new MMMRMultishiftSolver(epsilon, max_steps)
                                            : (MultishiftSolver *)new ChronologicalMultishiftSolver(epsilon, max_steps);
    const bool ok = ms->solve(op, b, xs, sh);
    for (int i = 0; i < nshift; ++i) store(xs[i], sols[i]);
    delete ms;
    delete op;
    return ok ? 1 : 0;
}

// RationalApproximation::evaluate with MEMultishiftSolver (algorithm 0) or
// MMMRMultishiftSolver (1); precision / max_steps through setPrecision / setMaximumRecursion
int ref_rational_evaluate(const int dims[4], int kind, double kappa, double csw, int gamma5, const double *links,
                          int algorithm, int n, const double *alphas, const double *betas, double precision,
                          int max_steps, const double *src, double *out)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    DiracOperator *op = make_operator(kind, kappa, csw, gamma5, L);
    if (!op) return -1;
    extended_dirac_vector_t b, o;
    load(b, src);
    MultishiftSolver *ms = algorithm == 0 ? (MultishiftSolver *)new MEMultishiftSolver(precision, max_steps)
                                          : (MultishiftSolver *)new MMMRMultishiftSolver(precision, max_steps);
    RationalApproximation ra(std::vector<real_t>(alphas, alphas + n), std::vector<real_t>(betas, betas + n), ms);
    ra.setPrecision(precision);
    ra.setMaximumRecursion(max_steps);
    ra.evaluate(op, o, b);
    store(o, out);
    delete ms;
    delete op;
    return 1;
}

// FermionForce::derivative of DiracWilsonFermionForce (kind 0) or ImprovedFermionForce (1):
// force[x][mu] -= weight * derivative(x, mu), force read and written in place
int ref_fermion_force(const int dims[4], int kind, double kappa, double csw, const double *links, const double *X,
                      const double *Y, double weight, double *force)
{
    init_layout(dims);
    extended_fermion_lattice_t L;
    load(L, links);
    extended_dirac_vector_t x, y;
    load(x, X);
    load(y, Y);
    extended_fermion_force_lattice_t F;
    load(F, force);
    // the derived classes' per-link derivative(...) hides the base class's field overload
    if (kind == 0) {
        DiracWilsonFermionForce f(kappa);
        FermionForce &base = f;
        base.derivative(F, L, x, y, weight);
    } else {
        ImprovedFermionForce f(kappa, csw);
        f.setLattice(L);
        FermionForce &base = f;
        base.derivative(F, L, x, y, weight);
    }
    store(F, force);
    return 1;
}

// ---- CPU baseline of the benchmark --------------------------------------------------
// One ImprovedDiracWilsonOperator held on one link field, as a caller that solves many
// sources on one gauge configuration holds it (the field strength is built once), and
// PreconditionedBiCGStab::solve on it: per call the reference builds its even-odd
// operators (field strength and the 12x12 inverses of every site) and runs BiCGStab on
// the Schur system (inverters/PreconditionedBiCGStab.cpp:33-100).
static extended_fermion_lattice_t *g_bench_links = nullptr;
static ImprovedDiracWilsonOperator *g_bench_op = nullptr;

void ref_bench_release()
{
    delete g_bench_op;
    delete g_bench_links;
    g_bench_op = nullptr;
    g_bench_links = nullptr;
}

int ref_bench_prepare(const int dims[4], double kappa, double csw, const double *links)
{
    ref_bench_release();
    init_layout(dims);
    g_bench_links = new extended_fermion_lattice_t;
    load(*g_bench_links, links);
    g_bench_op = static_cast<ImprovedDiracWilsonOperator *>(make_operator(1, kappa, csw, 0, *g_bench_links));
    return g_bench_op ? 0 : -1;
}

// returns 1 when the solver reports convergence, 0 when not, -1 without a prepared operator
int ref_bench_solve(double precision, int max_steps, const double *src, double *sol, int *steps)
{
    if (!g_bench_op) return -1;
    reduced_dirac_vector_t b, x;
    load(b, src);
    PreconditionedBiCGStab pb;
    pb.setPrecision(precision);
    pb.setMaximumSteps(max_steps);
    const bool ok = pb.solve(g_bench_op, b, x);
    *steps = pb.getLastSteps();
    if (sol) store(x, sol);
    return ok ? 1 : 0;
}

// ---- the reference's propagator consumers ----------------------------------------------
// MesonCorrelator::execute and ChiralCondensate::execute on an Environment holding the given
// fermion links, with their registered default options and the Improved operator of kappa,
// c_sw.  Their results reach only std::cout (and GlobalOutput, off without a format), so the
// stream is captured with 17 significant digits and parsed.
namespace {

std::map<std::string, Option> consumer_options(double kappa, double csw)
{
    std::map<std::string, Option> m;
    MesonCorrelator::registerParameters(m);
    ChiralCondensate::registerParameters(m);
    m["dirac_operator"] = Option("dirac_operator", std::string("Improved"), "");
    m["kappa"] = Option("kappa", kappa, "");
    m["csw"] = Option("csw", csw, "");
    return m;
}

struct CoutCapture {
    std::ostringstream ss;
    std::streambuf *old;
    std::streamsize prec;
    CoutCapture() : old(std::cout.rdbuf(ss.rdbuf())), prec(std::cout.precision(17)) {}
    ~CoutCapture()
    {
        std::cout.rdbuf(old);
        std::cout.precision(prec);
    }
};

struct SeededChiralCondensate : public ChiralCondensate {
    // one generator per OpenMP thread, as the reference's constructor makes them, seeded
    void seed(unsigned int s)
    {
        // the integer generators hold a reference to their engine: reseeding it is enough
        for (int i = 0; i < omp_get_max_threads(); ++i) randomGenerator[i]->seed(s + 7919u * (unsigned int)i);
    }
};

}  // namespace

// out[4][Lt]: pion, scalar, PS correlators (with the 4 kappa^2 factor) and PCAC mass per t
int ref_meson_correlator(const int dims[4], double kappa, double csw, const double *links, double precision,
                         int max_steps, double *out)
{
    init_layout(dims);
    std::map<std::string, Option> opts = consumer_options(kappa, csw);
    opts["MesonCorrelator::inverter_precision"] = Option("MesonCorrelator::inverter_precision", precision, "");
    opts["MesonCorrelator::inverter_max_steps"] = Option("MesonCorrelator::inverter_max_steps", max_steps, "");
    environment_t env(opts);
    load(env.fermionicLinkConfiguration, links);
    env.measurement = true;
    std::string text;
    {
        CoutCapture cap;
        MesonCorrelator mc;
        mc.execute(env);
        text = cap.ss.str();
    }
    const char *keys[4] = {"Pion Exact Correlator at t", "Scalar Exact Correlator at t", "PS Exact Correlator at t",
                           "PCAC mass at t"};
    const int Lt = dims[3];
    for (int k = 0; k < 4; ++k) {
        std::vector<double> v;
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line))
            if (line.find(keys[k]) != std::string::npos) v.push_back(std::strtod(line.c_str() + line.rfind(" is ") + 4, nullptr));
        if ((int)v.size() != Lt) return -1;
        for (int t = 0; t < Lt; ++t) out[k * Lt + t] = v[t];
    }
    return 0;
}

// ChiralCondensate::execute with n estimators on one OpenMP thread, its generator seeded;
// out[16]: mean and standard deviation of the condensate (re, im), pseudo-condensate (re, im),
// connected part (re, im), pion norm (re, im); noise[n][V][4][3] (if not null): the real Z2
// noise the same seed gives, in the reference's order of drawing
int ref_chiral_condensate(const int dims[4], double kappa, double csw, const double *links, double precision,
                          int max_steps, int n, int connected, unsigned int seed, double *out, double *noise)
{
    init_layout(dims);
    std::map<std::string, Option> opts = consumer_options(kappa, csw);
    opts["ChiralCondensate::inverter_precision"] = Option("ChiralCondensate::inverter_precision", precision, "");
    opts["ChiralCondensate::inverter_max_steps"] = Option("ChiralCondensate::inverter_max_steps", max_steps, "");
    opts["ChiralCondensate::number_stochastic_estimators"] =
        Option("ChiralCondensate::number_stochastic_estimators", n, "");
    opts["ChiralCondensate::measure_condensate_connected"] =
        Option("ChiralCondensate::measure_condensate_connected", std::string(connected ? "true" : "false"), "");
    environment_t env(opts);
    load(env.fermionicLinkConfiguration, links);
    env.measurement = true;
    const int threads = omp_get_max_threads();
    omp_set_num_threads(1);  // one generator, drawn site after site
    std::string text;
    {
        CoutCapture cap;
        SeededChiralCondensate cc;
        cc.seed(seed);
        cc.execute(env);
        text = cap.ss.str();
    }
    if (noise) {
        random_generator_t g(seed);
        random_integer_generator_t ri = RandomSeed::getRandomIntegerGenerator(g);
        const size_t count = (size_t)n * Lattice::LocalLayout::localsize * 4 * diracVectorLength;
        for (size_t k = 0; k < count; ++k) noise[k] = ri() == 0 ? -1.0 : 1.0;
    }
    omp_set_num_threads(threads);
    const char *keys[8] = {"Chiral condensate is (re)", "Chiral condensate is (im)", "Pseudo condensate is (re)",
                           "Pseudo condensate is (im)", "Connected chiral condensate susceptibility is (re)",
                           "Connected chiral condensate susceptibility is (im)", "Pion norm is (re)",
                           "Pion norm is (im)"};
    for (int k = 0; k < 8; ++k) {
        std::istringstream in(text);
        std::string line;
        bool found = false;
        while (std::getline(in, line)) {
            const size_t p = line.find(keys[k]);
            if (p == std::string::npos) continue;
            const char *c = line.c_str() + p + std::strlen(keys[k]);
            char *end = nullptr;
            out[2 * k] = std::strtod(c, &end);
            const char *pm = std::strstr(end, "+/-");
            out[2 * k + 1] = pm ? std::strtod(pm + 3, nullptr) : 0.0;
            found = true;
        }
        if (!found) return -1;
    }
    return 0;
}

// ---- the reference's gauge-configuration files ------------------------------------------
// OutputSweep::execute writes, ReadStartGaugeConfiguration::readConfiguration reads the
// fundamental links (extended_gauge_lattice_t raw storage) of one process; format 0
// leonard_format, 1 muenster_format; `directory` ends with a separator; the file number is
// OutputSweep's sweep + output_offset (sweep 0 here).
namespace {
std::map<std::string, Option> file_options(int format, const char *directory, const char *name, int number,
                                           double beta, double kappa)
{
    std::map<std::string, Option> m;
    const std::string fmt = format ? "muenster_format" : "leonard_format";
    m["output_format_name"] = Option("output_format_name", fmt, "");
    m["input_format_name"] = Option("input_format_name", fmt, "");
    m["output_configuration_name"] = Option("output_configuration_name", std::string(name), "");
    m["input_name"] = Option("input_name", std::string(name), "");
    m["output_directory_configurations"] = Option("output_directory_configurations", std::string(directory), "");
    m["input_directory_configurations"] = Option("input_directory_configurations", std::string(directory), "");
    m["output_offset"] = Option("output_offset", number, "");
    m["input_number"] = Option("input_number", number, "");
    m["beta"] = Option("beta", beta, "");
    m["kappa"] = Option("kappa", kappa, "");
    // Environment::synchronize after reading: no smearing, the fermion links' boundary
    m["stout_smearing_levels"] = Option("stout_smearing_levels", 0, "");
    m["boundary_conditions"] = Option("boundary_conditions", std::string("fermion_antiperiodic"), "");
    return m;
}
}  // namespace

int ref_gauge_write(const int dims[4], int format, const char *directory, const char *name, int number,
                    const double *links, double beta, double kappa)
{
    init_layout(dims);
    environment_t env(file_options(format, directory, name, number, beta, kappa));
    load(env.gaugeLinkConfiguration, links);
    env.sweep = 0;
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    OutputSweep out;
    out.execute(env);
    std::cout.rdbuf(old);
    return 0;
}

// returns 1 when the reference's reader reports success
int ref_gauge_read(const int dims[4], int format, const char *directory, const char *name, int number, double *links,
                   double beta, double kappa)
{
    init_layout(dims);
    environment_t env(file_options(format, directory, name, number, beta, kappa));
    std::ostringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    const bool ok = ReadStartGaugeConfiguration::readConfiguration(env, number);
    std::cout.rdbuf(old);
    store(env.gaugeLinkConfiguration, links);
    return ok ? 1 : 0;
}

}  // extern "C"
