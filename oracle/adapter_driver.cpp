// The C++ adapter (include/lym_leonard_adapter.hpp) exercised from the reference side:
// LeonardYM's own classes, compiled from its sources (oracle/build_ref.sh), call the GPU
// library through the adapter's subclasses held by the reference's base-class pointers,
// and every result is compared with the reference's CPU classes on the same inputs.
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into oracle/_ref/, run by
// tests/test_gpu_adapter.py.
//
// usage: adapter_driver Lx Ly Lz Lt kappa csw links.bin source.bin
//   links.bin: the fermion links in the reference's raw layout (extended_fermion_lattice_t)
//   source.bin: one spinor in the reference's raw layout (reduced_dirac_vector_t)
// Prints one line per check ("ok"/"FAIL", name, measured value, bar); exit status 0 when
// every check passes.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "inverters/BiConjugateGradient.h"
#include "inverters/ConjugateGradient.h"
#include "inverters/MEMultishiftSolver.h"
#include "inverters/MMMRMultishiftSolver.h"
#include "inverters/PreconditionedBiCGStab.h"
#include "lym_leonard_adapter.hpp"

using namespace Update;

namespace {

int g_failures = 0;

void check(const std::string &name, double value, double bar)
{
    const bool ok = std::isfinite(value) && value <= bar;
    if (!ok) ++g_failures;
    std::printf("%s %s %.3e <= %.1e\n", ok ? "ok" : "FAIL", name.c_str(), value, bar);
    std::fflush(stdout);
}

template <class L> bool read_raw(L &lat, const char *path)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    const size_t n = sizeof(typename L::TData) * lat.localsize;
    const size_t got = std::fread((void *)lat.getRawData(), 1, n, f);
    std::fclose(f);
    return got == n;
}

template <class V> double norm2(const V &v)
{
    const double *p = reinterpret_cast<const double *>(v.getRawData());
    const size_t n = sizeof(typename V::TData) * v.localsize / sizeof(double);
    double s = 0.0;
    for (size_t k = 0; k < n; ++k) s += p[k] * p[k];
    return s;
}

template <class V> double rel(const V &a, const V &b)
{
    const double *p = reinterpret_cast<const double *>(a.getRawData());
    const double *q = reinterpret_cast<const double *>(b.getRawData());
    const size_t n = sizeof(typename V::TData) * a.localsize / sizeof(double);
    double d = 0.0, s = 0.0;
    for (size_t k = 0; k < n; ++k) {
        d += (p[k] - q[k]) * (p[k] - q[k]);
        s += q[k] * q[k];
    }
    return std::sqrt(d / (s > 0 ? s : 1.0));
}

// c_sw of the operator classes that have one (setCSW is not virtual in the reference)
void set_csw(ImprovedDiracWilsonOperator *o, double csw) { o->setCSW(csw); }
void set_csw(SquareImprovedDiracWilsonOperator *o, double csw) { o->setCSW(csw); }
void set_csw(SquareEvenOddImprovedDiracWilsonOperator *o, double csw) { o->setCSW(csw); }
void set_csw(void *, double) {}

// a reference operator of one kind and its GPU subclass, kappa / c_sw / gamma5 set through
// the concrete types
template <class Ref, class Gpu>
void make_pair(std::unique_ptr<DiracOperator> &ref, std::unique_ptr<DiracOperator> &gpu, double kappa, double csw,
               bool gamma5, const extended_fermion_lattice_t &links)
{
    Ref *r = new Ref();
    Gpu *g = new Gpu();
    r->setKappa(kappa);
    g->setKappa(kappa);
    set_csw(r, csw);
    set_csw(g, csw);
    r->setLattice(links);
    g->setLattice(links);
    r->setGamma5(gamma5);
    g->setGamma5(gamma5);
    ref.reset(r);
    gpu.reset(g);
}

void operators(double kappa, double csw, const extended_fermion_lattice_t &links, const reduced_dirac_vector_t &x,
               const reduced_dirac_vector_t &y)
{
    const char *names[6] = {"DiracWilson", "Improved", "EvenOddImproved", "SquareDiracWilson", "SquareImproved",
                            "SquareEvenOddImproved"};
    for (int kind = 0; kind < 6; ++kind)
        for (int g5 = 0; g5 < 2; ++g5) {
            std::unique_ptr<DiracOperator> ref, gpu;
            switch (kind) {
            case 0: make_pair<DiracWilsonOperator, GpuDiracWilsonOperator>(ref, gpu, kappa, csw, g5, links); break;
            case 1:
                make_pair<ImprovedDiracWilsonOperator, GpuImprovedDiracWilsonOperator>(ref, gpu, kappa, csw, g5, links);
                break;
            case 2:
                make_pair<EvenOddImprovedDiracWilsonOperator, GpuEvenOddImprovedDiracWilsonOperator>(ref, gpu, kappa,
                                                                                                    csw, g5, links);
                break;
            case 3:
                make_pair<SquareDiracWilsonOperator, GpuSquareDiracWilsonOperator>(ref, gpu, kappa, csw, g5, links);
                break;
            case 4:
                make_pair<SquareImprovedDiracWilsonOperator, GpuSquareImprovedDiracWilsonOperator>(ref, gpu, kappa, csw,
                                                                                                  g5, links);
                break;
            default:
                make_pair<SquareEvenOddImprovedDiracWilsonOperator, GpuSquareEvenOddImprovedDiracWilsonOperator>(
                    ref, gpu, kappa, csw, g5, links);
                break;
            }
            const std::string tag = std::string(names[kind]) + (g5 ? " gamma5" : "");
            reduced_dirac_vector_t a, b;
            ref->multiply(a, x);
            gpu->multiply(b, x);
            check("multiply " + tag, rel(b, a), 1e-13);
            if (kind == 2) continue;  // the reference exits on EvenOddImproved::multiplyAdd
            const complex alpha(0.3, -0.2);
            ref->multiplyAdd(a, x, y, alpha);
            gpu->multiplyAdd(b, x, y, alpha);
            check("multiplyAdd " + tag, rel(b, a), 1e-13);
        }
}

struct Solved {
    reduced_dirac_vector_t x;
    bool ok;
    int steps;
};

// any of the reference's solver classes (ConjugateGradient is not a Solver subclass)
template <class S> Solved run(S *s, DiracOperator *d, const reduced_dirac_vector_t &b, double precision)
{
    Solved r;
    s->setPrecision(precision);
    s->setMaximumSteps(5000);
    r.ok = s->solve(d, b, r.x);
    r.steps = (int)s->getLastSteps();
    return r;
}

void compare(const std::string &name, const Solved &gpu, const Solved &ref, int step_slack)
{
    check(name + " converged", gpu.ok && ref.ok ? 0.0 : 1.0, 0.0);
    check(name + " solution", rel(gpu.x, ref.x), 1e-8);
    check(name + " getLastSteps difference", std::abs(gpu.steps - ref.steps), step_slack);
    std::printf("   %s steps: gpu %d reference %d\n", name.c_str(), gpu.steps, ref.steps);
    std::fflush(stdout);
}

void solvers(double kappa, double csw, const extended_fermion_lattice_t &links, const reduced_dirac_vector_t &b)
{
    const double precision = 1e-20 * norm2(b);
    // (1) the reference's own BiConjugateGradient on a GPU operator (a multiply per call)
    {
        std::unique_ptr<DiracOperator> ref, gpu;
        make_pair<SquareEvenOddImprovedDiracWilsonOperator, GpuSquareEvenOddImprovedDiracWilsonOperator>(
            ref, gpu, kappa, csw, true, links);
        BiConjugateGradient s1, s2;
        compare("reference BiConjugateGradient on GpuSquareEvenOddImproved", run(&s1, gpu.get(), b, precision),
                run(&s2, ref.get(), b, precision), 2);
    }
    // (2) GpuSolver through Solver*: CG on Q^2 and BiCGStab on D
    {
        std::unique_ptr<DiracOperator> ref, gpu;
        make_pair<SquareImprovedDiracWilsonOperator, GpuSquareImprovedDiracWilsonOperator>(ref, gpu, kappa, csw, true,
                                                                                          links);
        std::unique_ptr<Solver> s1(new GpuSolver(LYM_SOLVER_CG));
        ConjugateGradient s2;
        compare("GpuSolver(CG) vs ConjugateGradient", run(s1.get(), gpu.get(), b, precision),
                run(&s2, ref.get(), b, precision), 0);
    }
    {
        std::unique_ptr<DiracOperator> ref, gpu;
        make_pair<ImprovedDiracWilsonOperator, GpuImprovedDiracWilsonOperator>(ref, gpu, kappa, csw, false, links);
        std::unique_ptr<Solver> s1(new GpuSolver(LYM_SOLVER_BICGSTAB));
        BiConjugateGradient s2;
        compare("GpuSolver(BiCGStab) vs BiConjugateGradient", run(s1.get(), gpu.get(), b, precision),
                run(&s2, ref.get(), b, precision), 2);
        // (3) GpuPreconditionedBiCGStab where the callers build PreconditionedBiCGStab, on the
        // GPU operator and on a plain CPU ImprovedDiracWilsonOperator
        std::unique_ptr<Solver> p1(new GpuPreconditionedBiCGStab());
        std::unique_ptr<Solver> p2(new GpuPreconditionedBiCGStab());
        PreconditionedBiCGStab p3;
        const Solved want = run(&p3, ref.get(), b, precision);
        compare("GpuPreconditionedBiCGStab (GPU operator) vs PreconditionedBiCGStab", run(p1.get(), gpu.get(), b,
                                                                                          precision), want, 2);
        compare("GpuPreconditionedBiCGStab (CPU operator) vs PreconditionedBiCGStab", run(p2.get(), ref.get(), b,
                                                                                          precision), want, 2);
        GpuPreconditionedBiCGStab p4;
        p4.setUseEvenOddPreconditioning(false);
        PreconditionedBiCGStab p5;
        p5.setUseEvenOddPreconditioning(false);
        compare("GpuPreconditionedBiCGStab without even-odd vs PreconditionedBiCGStab",
                run(&p4, gpu.get(), b, precision), run(&p5, ref.get(), b, precision), 2);
    }
    // (4) GpuMultishiftSolver through MultishiftSolver*
    {
        std::unique_ptr<DiracOperator> ref, gpu;
        make_pair<SquareImprovedDiracWilsonOperator, GpuSquareImprovedDiracWilsonOperator>(ref, gpu, kappa, csw, true,
                                                                                          links);
        const std::vector<real_t> shifts = {0.5, 0.1, 0.02};
        extended_dirac_vector_t src;
        src = b;
        const int algos[2] = {LYM_MULTISHIFT_ME, LYM_MULTISHIFT_MMMR};
        const char *names[2] = {"mass_estrapolation", "minimal_residual"};
        for (int a = 0; a < 2; ++a) {
            std::unique_ptr<MultishiftSolver> g(new GpuMultishiftSolver(algos[a], 1e-20 * norm2(b), 5000));
            std::unique_ptr<MultishiftSolver> r(MultishiftSolver::getInstance(names[a]));
            r->setPrecision(1e-20 * norm2(b));
            r->setMaxSteps(5000);
            // the reference's solvers write into solutions sized by the caller
            std::vector<extended_dirac_vector_t> xg(shifts.size()), xr(shifts.size());
            const bool okg = g->solve(gpu.get(), src, xg, shifts);
            const bool okr = r->solve(ref.get(), src, xr, shifts);
            check(std::string("GpuMultishiftSolver ") + names[a] + " converged", okg && okr ? 0.0 : 1.0, 0.0);
            for (size_t i = 0; i < shifts.size(); ++i) {
                reduced_dirac_vector_t u, v;
                u = xg[i];
                v = xr[i];
                check(std::string("GpuMultishiftSolver ") + names[a] + " shift " + std::to_string(shifts[i]),
                      rel(u, v), 1e-8);
            }
        }
    }
}

// DiracOperator::getForce of the GPU operator against the reference's ImprovedFermionForce
void force(double kappa, double csw, const extended_fermion_lattice_t &links, const reduced_dirac_vector_t &x,
           const reduced_dirac_vector_t &y)
{
    GpuImprovedDiracWilsonOperator gop;
    gop.setKappa(kappa);
    gop.setCSW(csw);
    gop.setLattice(links);
    extended_dirac_vector_t X, Y;
    X = x;
    Y = y;
    extended_fermion_force_lattice_t Fg, Fr;
    const size_t n = sizeof(extended_fermion_force_lattice_t::TData) * Fg.localsize;
    std::memset((void *)Fg.getRawData(), 0, n);
    std::memset((void *)Fr.getRawData(), 0, n);
    std::unique_ptr<FermionForce> gf(gop.getForce());
    gf->derivative(Fg, links, X, Y, 0.7);
    ImprovedFermionForce rf(kappa, csw);
    rf.setLattice(links);
    FermionForce &base = rf;
    base.derivative(Fr, links, X, Y, 0.7);
    const double *p = reinterpret_cast<const double *>(Fg.getRawData());
    const double *q = reinterpret_cast<const double *>(Fr.getRawData());
    double d = 0.0, s = 0.0;
    for (size_t k = 0; k < n / sizeof(double); ++k) {
        d += (p[k] - q[k]) * (p[k] - q[k]);
        s += q[k] * q[k];
    }
    check("getForce()->derivative vs ImprovedFermionForce", std::sqrt(d / s), 1e-12);
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s Lx Ly Lz Lt kappa csw links.bin source.bin\n", argv[0]);
        return 2;
    }
    Lattice::LocalLayout::glob_x = std::atoi(argv[1]);
    Lattice::LocalLayout::glob_y = std::atoi(argv[2]);
    Lattice::LocalLayout::glob_z = std::atoi(argv[3]);
    Lattice::LocalLayout::glob_t = std::atoi(argv[4]);
    Lattice::LocalLayout::initialize();
    const double kappa = std::atof(argv[5]), csw = std::atof(argv[6]);
    extended_fermion_lattice_t links;
    reduced_dirac_vector_t b, y;
    if (!read_raw(links, argv[7]) || !read_raw(b, argv[8])) {
        std::fprintf(stderr, "cannot read the input files\n");
        return 2;
    }
    // a second vector for multiplyAdd and the force: b with its spin blocks swapped and scaled
    for (int s = 0; s < b.localsize; ++s)
        for (int mu = 0; mu < 4; ++mu) y[s][mu] = 0.5 * b[s][3 - mu];
    operators(kappa, csw, links, b, y);
    solvers(kappa, csw, links, b);
    force(kappa, csw, links, b, y);
    std::printf("%s: %d failed checks\n", g_failures ? "FAILED" : "PASSED", g_failures);
    return g_failures ? 1 : 0;
}
