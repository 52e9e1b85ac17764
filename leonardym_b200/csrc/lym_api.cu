// C ABI of the library: contexts, resident gauge fields, operators, operator
// application and the Krylov solvers.  See include/lym_b200.h for the contract.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/lym_b200.h"
#include "lym_batch.cuh"
#include "lym_internal.h"
#include "lym_solver_ops.cuh"

using namespace lym;

namespace {

constexpr int kBlasGridMax = 148 * 8;

struct GaugeEntry {
    GaugeDev dev;
    int recon_err = 0;
};

struct OpEntry {
    int gauge_id = -1;
    int kind = LYM_OP_DIRAC_WILSON;
    double kappa = 0.0, csw = 0.0;
    int gamma5 = 1;
    CloverDev clover;
    bool clover_ok = false;
};

struct LymError {
    int code;
};

}  // namespace

// Batched stencil configuration picked by the autotuner: traversal column (by, bz) of
// the (y, z) plane (by = 0: plain half-site order) and the kernel variant (minimum
// resident blocks per SM).
struct BatchTile {
    int by = 0, bz = 0, minb = 1;
};

struct lym_context {
    Geom g;
    int rep = REP_SU3;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaStream_t st_copy = nullptr;  // host <-> device copies that overlap the solves
    std::recursive_mutex mu;  // entry points may call other entry points on the same thread
    std::string err;
    std::map<int, GaugeEntry> gauges;
    std::map<int, OpEntry> ops;
    int next_op = 1;
    // reductions
    double *partials = nullptr;
    double *bpartials = nullptr;  // per-RHS partial sums of the batched reductions
    double *spartials = nullptr;  // one partial sum per block of a single-RHS stencil launch
    int *nbr = nullptr;           // neighbour half-site table [2][8][stride] (batched stencil)
    std::map<int, int *> orders;  // traversal tables [stride] by column by * 4096 + bz
    std::map<int, BatchTile> tiles;  // tuned configuration by (precision, batch, clover)
    BatchTile forced_tile;
    bool tile_forced = false;
    unsigned int *counter = nullptr;
    int *d_err = nullptr;
    void *d_state = nullptr;      // solver state (device)
    void *h_state = nullptr;      // pinned mirror
    double *d_scal = nullptr;     // scratch scalars
    double *h_scal = nullptr;
    // host-layout staging buffers (V * 24 doubles)
    double *aos[3] = {nullptr, nullptr, nullptr};
    std::vector<Spinor> pool;
    // idle per-call device buffers (batched vectors, staging rings, scratch) kept for the
    // next call of the same size, like the spinor pool: given back by trim_pool
    std::vector<std::pair<size_t, void *>> blocks;
    size_t bytes = 0;
    unsigned long long launches = 0;  // kernels enqueued (graph replays count their nodes)
    double engine_stats[9] = {};      // block solves: lym_context_engine_stats
    bool capturing = false;
    int inject_alloc_failures = 0;  // the next n device allocations report failure (tests)
    bool inject_copy_wait = false;  // the next check of the bulk-copy wait word reports a give-up (tests)
    int link_reals = 12;            // FP32 SU(3) link format of the single-RHS stencils: 12 or 8
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

constexpr size_t kStateBytes = 8192;
static_assert(sizeof(MultishiftState) <= kStateBytes, "state buffer too small");
static_assert(sizeof(CGState) <= kStateBytes && sizeof(BiCGState) <= kStateBytes, "state buffer too small");

int fail(lym_context *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    throw LymError{code};
}

void ck(lym_context *c, cudaError_t e, const char *what)
{
    if (e != cudaSuccess) fail(c, LYM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call) ck(c, (call), #call)

template <class F> int guarded(lym_context *c, F f)
{
    if (!c) return LYM_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> lock(c->mu);
    try {
        cudaSetDevice(c->device);
        return f();
    } catch (const LymError &e) {
        return e.code;
    } catch (const std::bad_alloc &) {
        c->err = "host allocation failed";
        return LYM_ERR_MEMORY;
    }
}

size_t spinor_bytes(const Geom &g, int prec, int nparity);

// frees the idle spinors of the pool and the host-transfer staging buffers
void trim_pool(lym_context *c)
{
    if (c->st) cudaStreamSynchronize(c->st);
    for (auto &s : c->pool) {
        cudaFree(s.v);
        c->bytes -= spinor_bytes(c->g, s.prec, s.nparity);
    }
    c->pool.clear();
    for (auto &b : c->blocks) {
        cudaFree(b.second);
        c->bytes -= b.first;
    }
    c->blocks.clear();
    for (int k = 0; k < 3; ++k)
        if (c->aos[k]) {
            cudaFree(c->aos[k]);
            c->bytes -= (size_t)c->g.V * 24 * sizeof(double);
            c->aos[k] = nullptr;
        }
}

void *dev_alloc(lym_context *c, size_t bytes)
{
    if (c->inject_alloc_failures > 0) {  // host-side fault injection (lym_context_inject_alloc_failures)
        --c->inject_alloc_failures;
        fail(c, LYM_ERR_MEMORY, "device allocation of %zu bytes failed: injected failure", bytes);
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation && !c->capturing &&
        (!c->pool.empty() || !c->blocks.empty() || c->aos[0] || c->aos[1] || c->aos[2])) {
        // the idle pooled spinors are a cache: give them back and try once more
        cudaGetLastError();
        trim_pool(c);
        e = cudaMalloc(&p, bytes);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(c, LYM_ERR_MEMORY, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    CK(cudaMemsetAsync(p, 0, bytes, c->st));
    c->bytes += bytes;
    return p;
}

void dev_free(lym_context *c, void *p, size_t bytes)
{
    if (p) {
        cudaFree(p);
        c->bytes -= bytes;
    }
}

// a zeroed buffer of the given size from the idle blocks, else newly allocated
void *block_alloc(lym_context *c, size_t bytes)
{
    for (size_t i = 0; i < c->blocks.size(); ++i)
        if (c->blocks[i].first == bytes) {
            void *p = c->blocks[i].second;
            c->blocks.erase(c->blocks.begin() + i);
            CK(cudaMemsetAsync(p, 0, bytes, c->st));
            return p;
        }
    return dev_alloc(c, bytes);
}

// back to the idle blocks (its last uses are ordered before any later use on the
// context's stream; copies on the copy stream are drained by their owners first)
void block_free(lym_context *c, void *p, size_t bytes)
{
    if (p) c->blocks.emplace_back(bytes, p);
}

// device memory for the length of one call
struct DevBuf {
    lym_context *c;
    void *p = nullptr;
    size_t n = 0;
    DevBuf(lym_context *ctx, size_t bytes) : c(ctx), p(block_alloc(ctx, bytes)), n(bytes) {}
    ~DevBuf()
    {
        if (p) block_free(c, p, n);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

size_t spinor_bytes(const Geom &g, int prec, int nparity)
{
    const size_t s = g.stride;
    switch (prec) {
    case PREC_D: return nparity * 12 * s * sizeof(double2);
    case PREC_F: return nparity * 6 * s * sizeof(float4);
    default: return nparity * (3 * s * sizeof(int4) + s * sizeof(float));
    }
}

// --------------------------------------------------------- spinor pool -----
struct Vec {
    lym_context *c = nullptr;
    Spinor s;
    Vec() = default;
    Vec(lym_context *ctx, int prec, int nparity) : c(ctx)
    {
        for (size_t i = 0; i < c->pool.size(); ++i) {
            if (c->pool[i].prec == prec && c->pool[i].nparity == nparity) {
                s = c->pool[i];
                c->pool.erase(c->pool.begin() + i);
                return;
            }
        }
        s.prec = prec;
        s.nparity = nparity;
        s.stride = c->g.stride;
        const size_t b = spinor_bytes(c->g, prec, nparity);
        char *base = (char *)dev_alloc(c, b);
        s.v = base;
        if (prec == PREC_H) s.norm = (float *)(base + (size_t)nparity * 3 * c->g.stride * sizeof(int4));
        s.owned = true;
    }
    ~Vec()
    {
        if (c && s.v) c->pool.push_back(s);
    }
    Vec(const Vec &) = delete;
    Vec &operator=(const Vec &) = delete;
    const Spinor &operator*() const { return s; }
    Spinor par(int p) const { return s.parity(p); }
};

// --------------------------------------------------------- site kernels ----
void count(lym_context *c, int n)
{
    if (!c->capturing) c->launches += n;
}

template <class Op> void run_site(lym_context *c, const Op &op, int nparity, Gate gate = Gate{nullptr, nullptr})
{
    count(c, 1);
    int grid = (c->g.Vh + kBlasThreads - 1) / kBlasThreads;
    grid = std::min(grid, kBlasGridMax);
    site_kernel<Op><<<grid, kBlasThreads, 0, c->st>>>(op, c->g.Vh, nparity, RedBuf{c->partials, c->counter}, gate);
}

double2 C2(double re, double im = 0.0) { return make_double2(re, im); }

// y = a x + b y for any precisions of x and y
void axpby(lym_context *c, const Spinor &x, const Spinor &y, double2 a, double2 b)
{
    const int np = y.nparity;
    auto go = [&](auto X) {
        if (y.prec == PREC_D) run_site(c, OpAxpby<decltype(X), SpinorD>{X, y.d(), a, b}, np);
        else if (y.prec == PREC_F) run_site(c, OpAxpby<decltype(X), SpinorF>{X, y.f(), a, b}, np);
        else run_site(c, OpAxpby<decltype(X), SpinorH>{X, y.h(), a, b}, np);
    };
    if (x.prec == PREC_D) go(x.d());
    else if (x.prec == PREC_F) go(x.f());
    else go(x.h());
}

void copy(lym_context *c, const Spinor &dst, const Spinor &src)
{
    if (dst.prec == src.prec && dst.nparity == src.nparity) {
        CK(cudaMemcpyAsync(dst.v, src.v, spinor_bytes(c->g, src.prec, src.nparity), cudaMemcpyDeviceToDevice, c->st));
        return;
    }
    launch_convert(c->g, dst, src, c->st);
}

void zero(lym_context *c, const Spinor &s) { CK(cudaMemsetAsync(s.v, 0, spinor_bytes(c->g, s.prec, s.nparity), c->st)); }

double norm2_now(lym_context *c, const Spinor &x)
{
    run_site(c, OpNorm<SpinorD>{x.d(), c->d_scal}, x.nparity);
    CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return c->h_scal[0];
}

void gamma5_inplace(lym_context *c, const Spinor &x) { run_site(c, OpGamma5<SpinorD>{x.d()}, x.nparity); }

// ------------------------------------------------------------ operators ----
GaugeEntry &gauge_of(lym_context *c, int id)
{
    auto it = c->gauges.find(id);
    if (it == c->gauges.end()) fail(c, LYM_ERR_NOT_FOUND, "gauge field %d is not resident", id);
    return it->second;
}

OpEntry &op_of(lym_context *c, int id)
{
    auto it = c->ops.find(id);
    if (it == c->ops.end()) fail(c, LYM_ERR_NOT_FOUND, "operator %d does not exist", id);
    return it->second;
}

bool kind_has_clover(int kind)
{
    return kind == LYM_OP_IMPROVED || kind == LYM_OP_EVEN_ODD_IMPROVED || kind == LYM_OP_SQUARE_IMPROVED ||
           kind == LYM_OP_SQUARE_EVEN_ODD_IMPROVED;
}

size_t clover_bytes(const Geom &g, int prec)
{
    const size_t s = g.stride;
    if (prec == PREC_D) return 4 * 18 * s * sizeof(double2);
    if (prec == PREC_F) return 4 * 9 * s * sizeof(float4);
    return 4 * 9 * s * sizeof(uint2);
}

void free_clover(lym_context *c, OpEntry &op)
{
    for (int p = 0; p < 3; ++p) {
        dev_free(c, op.clover.T[p], clover_bytes(c->g, p));
        dev_free(c, op.clover.Tinv[p], clover_bytes(c->g, p));
        op.clover.T[p] = op.clover.Tinv[p] = nullptr;
    }
    op.clover_ok = false;
}

void ensure_clover(lym_context *c, OpEntry &op, double *F_out = nullptr)
{
    if (op.clover_ok && !F_out) return;
    if (c->capturing) fail(c, LYM_ERR_ARGUMENT, "clover term must be built before graph capture");
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    for (int p = 0; p < 3; ++p) {
        if (!op.clover.T[p]) op.clover.T[p] = dev_alloc(c, clover_bytes(c->g, p));
        if (!op.clover.Tinv[p]) op.clover.Tinv[p] = dev_alloc(c, clover_bytes(c->g, p));
    }
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
    launch_clover_build(c->g, ge.dev, op.kappa * op.csw, op.clover, F_out, c->d_err, c->st);
    launch_clover_compress(c->g, op.clover, c->st);
    int herr = 0;
    CK(cudaMemcpyAsync(c->h_scal, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    memcpy(&herr, c->h_scal, sizeof(int));
    CK(cudaGetLastError());
    if (herr) fail(c, LYM_ERR_NUMERIC, "clover block not invertible (error bits %d)", herr);
    op.clover_ok = true;
}

void require_recon(lym_context *c, GaugeEntry &ge, int prec)
{
    if (prec == PREC_D) return;
    if (!ge.dev.recon_ok)
        fail(c, LYM_ERR_UNSUPPORTED,
             "reduced-precision links need +-SU(3) / +-SO(3) links (unitarity check bits %d)", ge.recon_err);
}

// full operator: out = G5^g (T in_p - kappa H in_{1-p}) + alpha v2 on both parities
void apply_full(lym_context *c, OpEntry &op, int prec, const Spinor &out, const Spinor &in, int gamma5,
                const Spinor *v2, double2 alpha, const int *skip = nullptr)
{
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    const bool clov = kind_has_clover(op.kind);
    if (clov) ensure_clover(c, op);
    require_recon(c, ge, prec);
    for (int p = 0; p < 2; ++p) {
        DslashParams P;
        P.g = c->g;
        P.prec = prec;
        P.rep = c->rep;
        P.epi = EPI_XPAY_;
        P.parity = p;
        P.in = in.parity(1 - p);
        P.out = out.parity(p);
        P.y = in.parity(p);
        if (v2) {
            P.v2 = v2->parity(p);
            P.has_v2 = 1;
            P.alpha_re = alpha.x;
            P.alpha_im = alpha.y;
        } else {
            P.v2 = P.y;
        }
        P.U = &ge.dev;
        P.clover = clov ? op.clover.T[prec] : nullptr;
        P.gamma5 = gamma5;
        P.b = -op.kappa;
        P.skip_if = skip;
        launch_dslash(P, c->st);
        count(c, 1);
    }
}

// Schur complement on the odd sites:
//   out_o = G5^g (T_oo in_o - kappa^2 H_oe T_ee^{-1} H_eo in_o) + alpha v2_o
void apply_schur(lym_context *c, OpEntry &op, int prec, const Spinor &out_o, const Spinor &in_o, const Spinor &tmp_e,
                 int gamma5, const Spinor *v2 = nullptr, double2 alpha = make_double2(0, 0),
                 const int *skip = nullptr)
{
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    const bool clov = kind_has_clover(op.kind);
    if (clov) ensure_clover(c, op);
    require_recon(c, ge, prec);
    DslashParams P;
    P.g = c->g;
    P.prec = prec;
    P.rep = c->rep;
    P.U = &ge.dev;
    P.skip_if = skip;
    // K1: tmp_e = Tinv_ee H_eo in_o
    P.epi = clov ? EPI_CLOVINV_ : EPI_SCALE_;
    P.parity = 0;
    P.in = in_o;
    P.out = tmp_e;
    P.y = tmp_e;
    P.v2 = tmp_e;
    P.clover = clov ? op.clover.Tinv[prec] : nullptr;
    P.a = 1.0;
    launch_dslash(P, c->st);
    // K2: out_o = G5^g (T_oo in_o - kappa^2 H_oe tmp_e) + alpha v2
    P.epi = EPI_XPAY_;
    P.parity = 1;
    P.in = tmp_e;
    P.out = out_o;
    P.y = in_o;
    P.clover = clov ? op.clover.T[prec] : nullptr;
    P.b = -op.kappa * op.kappa;
    P.gamma5 = gamma5;
    if (v2) {
        P.v2 = *v2;
        P.has_v2 = 1;
        P.alpha_re = alpha.x;
        P.alpha_im = alpha.y;
    } else {
        P.v2 = in_o;
    }
    launch_dslash(P, c->st);
    count(c, 2);
}

// Q in_o = gamma5 S in_o inside the even-odd CG on (gamma5 S)^2, with the CG's vector work in
// the second launch (launch_dslash_cg): mode CG_NORM stores q = Q p in out_o and sets the
// state's alpha from |q|^2; mode CG_UPDATE (in_o = q) forms A p = Q q in registers and
// updates x and r with the state's alpha, then the CG step's scalars.  p, x, r: one parity.
void apply_schur_cg(lym_context *c, OpEntry &op, int prec, int mode, const Spinor &out_o, const Spinor &in_o,
                    const Spinor &tmp_e, const Spinor &p, const Spinor &x, const Spinor &r, void *state,
                    const int *skip)
{
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    const bool clov = kind_has_clover(op.kind);
    if (clov) ensure_clover(c, op);
    require_recon(c, ge, prec);
    DslashParams P;
    P.g = c->g;
    P.prec = prec;
    P.rep = c->rep;
    P.U = &ge.dev;
    P.skip_if = skip;
    P.epi = clov ? EPI_CLOVINV_ : EPI_SCALE_;
    P.parity = 0;
    P.in = in_o;
    P.out = tmp_e;
    P.y = tmp_e;
    P.v2 = tmp_e;
    P.clover = clov ? op.clover.Tinv[prec] : nullptr;
    P.a = 1.0;
    launch_dslash(P, c->st);
    P.epi = EPI_XPAY_;
    P.parity = 1;
    P.in = tmp_e;
    P.out = out_o;
    P.y = in_o;
    P.v2 = p;
    P.clover = clov ? op.clover.T[prec] : nullptr;
    P.b = -op.kappa * op.kappa;
    P.gamma5 = 1;
    launch_dslash_cg(P, mode, p, x, r, state, c->spartials, c->counter, c->st);
    count(c, 2);
}

bool is_even_odd(int kind) { return kind == LYM_OP_EVEN_ODD_IMPROVED || kind == LYM_OP_SQUARE_EVEN_ODD_IMPROVED; }

// DiracOperator::multiply / multiplyAdd on full device spinors (reference semantics).
void op_apply(lym_context *c, OpEntry &op, int prec, const Spinor &out, const Spinor &in, const Spinor *v2,
              double2 alpha, const int *skip = nullptr)
{
    const int g5 = op.gamma5;
    switch (op.kind) {
    case LYM_OP_DIRAC_WILSON:
    case LYM_OP_IMPROVED: apply_full(c, op, prec, out, in, g5, v2, alpha, skip); return;
    case LYM_OP_SQUARE_DIRAC_WILSON:
    case LYM_OP_SQUARE_IMPROVED: {
        Vec tmp(c, prec, 2);
        apply_full(c, op, prec, *tmp, in, g5, nullptr, alpha, skip);
        apply_full(c, op, prec, out, *tmp, g5, v2, alpha, skip);
        return;
    }
    case LYM_OP_EVEN_ODD_IMPROVED: {
        if (v2) fail(c, LYM_ERR_UNSUPPORTED, "EvenOddImprovedDiracWilsonOperator::multiplyAdd is not implemented");
        Vec te(c, prec, 1);
        copy(c, out.parity(0), in.parity(0));
        apply_schur(c, op, prec, out.parity(1), in.parity(1), *te, g5, nullptr, alpha, skip);
        return;
    }
    case LYM_OP_SQUARE_EVEN_ODD_IMPROVED: {
        Vec te(c, prec, 1), to(c, prec, 1);
        apply_schur(c, op, prec, *to, in.parity(1), *te, g5, nullptr, alpha, skip);
        Spinor v2o;
        if (v2) v2o = v2->parity(1);
        apply_schur(c, op, prec, out.parity(1), *to, *te, g5, v2 ? &v2o : nullptr, alpha, skip);
        copy(c, out.parity(0), in.parity(0));
        if (v2) axpby(c, v2->parity(0), out.parity(0), alpha, C2(1.0));
        return;
    }
    default: fail(c, LYM_ERR_ARGUMENT, "unknown operator kind %d", op.kind);
    }
}

// ------------------------------------------------------ host <-> device -----
double *staging(lym_context *c, int k)
{
    if (!c->aos[k]) c->aos[k] = (double *)dev_alloc(c, (size_t)c->g.V * 24 * sizeof(double));
    return c->aos[k];
}

void upload_vec(lym_context *c, const Spinor &dst, const double *src, bool device_ptr, int slot)
{
    const size_t b = (size_t)c->g.V * 24 * sizeof(double);
    const double *d = src;
    if (!device_ptr) {
        double *s = staging(c, slot);
        CK(cudaMemcpyAsync(s, src, b, cudaMemcpyHostToDevice, c->st));
        d = s;
    }
    launch_pack(c->g, d, dst, c->st);
}

void download_vec(lym_context *c, double *dst, const Spinor &src, bool device_ptr, int slot)
{
    const size_t b = (size_t)c->g.V * 24 * sizeof(double);
    if (device_ptr) {
        launch_unpack(c->g, src, dst, c->st);
        return;
    }
    double *s = staging(c, slot);
    launch_unpack(c->g, src, s, c->st);
    CK(cudaMemcpyAsync(dst, s, b, cudaMemcpyDeviceToHost, c->st));
}

// ------------------------------------------------------------- solvers -----
CGState *cg_state(lym_context *c) { return (CGState *)c->d_state; }
CGState &cg_host(lym_context *c) { return *(CGState *)c->h_state; }
BiCGState *bi_state(lym_context *c) { return (BiCGState *)c->d_state; }
BiCGState &bi_host(lym_context *c) { return *(BiCGState *)c->h_state; }

void pull_state(lym_context *c, size_t bytes)
{
    CK(cudaMemcpyAsync(c->h_state, c->d_state, bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
}
void push_state(lym_context *c, size_t bytes)
{
    CK(cudaMemcpyAsync(c->d_state, c->h_state, bytes, cudaMemcpyHostToDevice, c->st));
}

// Run `step` (one iteration; every kernel gated on the state's `pause` flag)
// until the device state pauses.  Batches of iterations are captured once into a
// CUDA graph and replayed; the host reads the state once per batch.
template <class S, class Step> void run_gated_state(lym_context *c, S *d, Step step, int batch, long max_iterations)
{
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    try {
        for (int k = 0; k < batch; ++k) step();
    } catch (...) {
        c->capturing = false;
        cudaStreamEndCapture(c->st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    c->capturing = false;
    CK(cudaStreamEndCapture(c->st, &graph));
    CK(cudaGraphInstantiate(&exec, graph, 0));
    size_t nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &nodes);
    // every iteration pauses the state by itself at its iteration limit; the host
    // bound below only guards against a state that never pauses
    const long max_launches = max_iterations / batch + 4;
    bool paused = false;
    for (long l = 0; l < max_launches; ++l) {
        CK(cudaGraphLaunch(exec, c->st));
        c->launches += nodes;
        CK(cudaMemcpyAsync(c->h_state, d, sizeof(S), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (((S *)c->h_state)->pause) {
            paused = true;
            break;
        }
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    CK(cudaGetLastError());
    if (!paused) fail(c, LYM_ERR_TIMEOUT, "solver state did not stop within %ld iterations", max_iterations);
}

// --- CG (ConjugateGradient::solve, inverters/ConjugateGradient.cpp:10-74) ---
template <class MatVec>
int cg_solve(lym_context *c, MatVec matvec, int nparity, const Spinor &b, const Spinor &x, const Spinor *guess,
             double eps, int max_steps, lym_solve_stats *st)
{
    Vec r(c, PREC_D, nparity), p(c, PREC_D, nparity), ap(c, PREC_D, nparity);
    copy(c, x, guess ? *guess : b);
    matvec(*ap, x, nullptr);
    run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{b.d(), (*ap).d(), (*r).d(), c->d_scal}, nparity);
    copy(c, *p, *r);
    CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CGState &H = cg_host(c);
    memset(&H, 0, sizeof(H));
    H.rr = c->h_scal[0];
    H.rr_max = H.rr;
    H.eps = eps;
    H.max_iter = max_steps;
    push_state(c, sizeof(CGState));
    CGState *S = cg_state(c);
    Gate gate{&S->pause, nullptr};
    auto step = [&]() {
        matvec(*ap, *p, &S->pause);
        run_site(c, OpCGAlpha<SpinorD, SpinorD>{(*p).d(), (*ap).d(), S}, nparity, gate);
        run_site(c, OpCGUpdate<SpinorD, SpinorD, SpinorD, SpinorD>{x.d(), (*p).d(), (*r).d(), (*ap).d(), S}, nparity,
                 gate);
        run_site(c, OpCGDirection<SpinorD, SpinorD>{(*p).d(), (*r).d(), S}, nparity, gate);
    };
    if (max_steps > 0) run_gated_state(c, S, step, 8, max_steps);
    else pull_state(c, sizeof(CGState));
    CGState &R = cg_host(c);
    if (st) {
        st->converged = R.converged;
        st->iterations = R.iter;
        st->steps = R.converged ? R.iter - 1 : max_steps;
        st->last_error = R.rr;
    }
    if (R.failed) fail(c, LYM_ERR_NUMERIC, "CG produced a non-finite residual");
    return R.converged ? LYM_OK : LYM_NOT_CONVERGED;
}

// Start vector of the reference's BiCGStab variants: the guess, else the source when its
// squared norm exceeds the precision, else a uniform random vector (BiConjugateGradient.cpp
// :333-340).  The reference seeds that vector from the clock (AlgebraUtils.h:123-167); a
// fixed deterministic stream is used instead.
void reference_start(lym_context *c, const Spinor &b, const Spinor &x, const Spinor *guess, double precision,
                     double norm_offset, int nparity)
{
    if (guess) {
        copy(c, x, *guess);
        return;
    }
    const double ns = norm2_now(c, b) + norm_offset;
    if (ns > precision) {
        copy(c, x, b);
        return;
    }
    std::vector<double> host((size_t)c->g.V * 24);
    unsigned long long z = 0x9E3779B97F4A7C15ull;
    for (auto &v : host) {
        z += 0x9E3779B97F4A7C15ull;
        unsigned long long q = z;
        q = (q ^ (q >> 30)) * 0xBF58476D1CE4E5B9ull;
        q = (q ^ (q >> 27)) * 0x94D049BB133111EBull;
        q ^= q >> 31;
        v = (double)(q >> 11) * (1.0 / 9007199254740992.0);
    }
    Vec full(c, PREC_D, 2);
    upload_vec(c, *full, host.data(), false, 2);
    CK(cudaStreamSynchronize(c->st));
    copy(c, x, nparity == 2 ? *full : full.par(1));
}

// --- BiCGStab (BiConjugateGradient::solve, BiConjugateGradient.cpp:321-507) ---
template <class MatVec>
int bicgstab_solve(lym_context *c, MatVec matvec, int nparity, const Spinor &b, const Spinor &x,
                   const Spinor *guess, double precision, int max_steps, double norm_offset, lym_solve_stats *st)
{
    Vec r(c, PREC_D, nparity), rhat(c, PREC_D, nparity), p(c, PREC_D, nparity), nu(c, PREC_D, nparity),
        s(c, PREC_D, nparity), t(c, PREC_D, nparity);
    reference_start(c, b, x, guess, precision, norm_offset, nparity);
    matvec(*p, x, nullptr);
    // r = b - A x ; rhat = b + A x
    copy(c, *r, b);
    axpby(c, *p, *r, C2(-1.0), C2(1.0));
    copy(c, *rhat, b);
    axpby(c, *p, *rhat, C2(1.0), C2(1.0));
    zero(c, *p);
    zero(c, *nu);
    BiCGState &H = bi_host(c);
    memset(&H, 0, sizeof(H));
    H.rho = C2(1.0);
    H.alpha = C2(1.0);
    H.omega = C2(1.0);
    H.precision = precision;
    H.max_steps = max_steps;
    push_state(c, sizeof(BiCGState));
    BiCGState *S = bi_state(c);
    Gate gate{&S->pause, nullptr};
    run_site(c, OpBiRho<SpinorD, SpinorD>{(*rhat).d(), (*r).d(), S}, nparity);
    auto step = [&]() {
        run_site(c, OpBiDirection<SpinorD, SpinorD, SpinorD>{(*p).d(), (*r).d(), (*nu).d(), S}, nparity, gate);
        matvec(*nu, *p, &S->pause);
        run_site(c, OpBiAlpha<SpinorD, SpinorD>{(*rhat).d(), (*nu).d(), S}, nparity, gate);
        run_site(c, OpBiS<SpinorD, SpinorD, SpinorD>{(*s).d(), (*r).d(), (*nu).d(), S}, nparity, gate);
        matvec(*t, *s, &S->pause);
        run_site(c, OpBiOmega<SpinorD, SpinorD>{(*t).d(), (*s).d(), S}, nparity, gate);
        run_site(c,
                 OpBiUpdate<SpinorD, SpinorD, SpinorD, SpinorD, SpinorD, SpinorD>{x.d(), (*p).d(), (*s).d(), (*t).d(),
                                                                                  (*r).d(), (*rhat).d(), S},
                 nparity, gate);
    };
    pull_state(c, sizeof(BiCGState));
    if (!bi_host(c).pause && max_steps > 0) run_gated_state(c, S, step, 4, max_steps);
    BiCGState &R = bi_host(c);
    if (R.degenerate) copy(c, x, b);  // BiConjugateGradient.cpp:455-464
    if (st) {
        st->converged = R.converged && !R.breakdown;
        st->iterations = R.step + (R.converged ? 1 : 0);
        st->steps = R.converged ? R.step : max_steps;
        st->last_error = R.last_error;
    }
    if (R.breakdown) {
        c->err = "BiConjugateGradient: breakdown (rho = 0 or non-finite residual)";
        return LYM_ERR_BREAKDOWN;
    }
    return R.converged ? LYM_OK : LYM_NOT_CONVERGED;
}

// b'_o = b_o + kappa H_oe Tinv_ee b_e  (source of the Schur system)
void schur_source(lym_context *c, OpEntry &op, const Spinor &b, const Spinor &bprime_o)
{
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    const bool clov = kind_has_clover(op.kind);
    if (clov) ensure_clover(c, op);
    Vec te(c, PREC_D, 1);
    if (clov) launch_clover(c->g, PREC_D, *te, b.parity(0), op.clover.Tinv[PREC_D], 0, 0, c->st);
    else copy(c, *te, b.parity(0));
    DslashParams P;
    P.g = c->g;
    P.prec = PREC_D;
    P.rep = c->rep;
    P.U = &ge.dev;
    P.epi = EPI_XPAY_;
    P.parity = 1;
    P.in = *te;
    P.out = bprime_o;
    P.y = b.parity(1);
    P.v2 = b.parity(1);
    P.b = op.kappa;
    launch_dslash(P, c->st);
}

// x_e = Tinv_ee (b_e + kappa H_eo x_o)
void schur_reconstruct(lym_context *c, OpEntry &op, const Spinor &b, const Spinor &x)
{
    GaugeEntry &ge = gauge_of(c, op.gauge_id);
    const bool clov = kind_has_clover(op.kind);
    DslashParams P;
    P.g = c->g;
    P.prec = PREC_D;
    P.rep = c->rep;
    P.U = &ge.dev;
    P.epi = clov ? EPI_XPAY_INV_ : EPI_XPAY_;
    P.parity = 0;
    P.in = x.parity(1);
    P.out = x.parity(0);
    P.y = b.parity(0);
    P.v2 = b.parity(0);
    P.clover = clov ? op.clover.Tinv[PREC_D] : nullptr;
    P.b = op.kappa;
    launch_dslash(P, c->st);
}

double true_residual(lym_context *c, OpEntry &op, const Spinor &b, const Spinor &x)
{
    // ||b - D x|| / ||b|| with the FP64 full operator D (gamma5 = false)
    Vec ax(c, PREC_D, 2), r(c, PREC_D, 2);
    apply_full(c, op, PREC_D, *ax, x, 0, nullptr, C2(0.0));
    run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{b.d(), (*ax).d(), (*r).d(), c->d_scal}, 2);
    CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double rr = c->h_scal[0];
    const double bb = norm2_now(c, b);
    return bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
}

// PreconditionedBiCGStab::solve (inverters/PreconditionedBiCGStab.cpp:33-100)
int eo_bicgstab(lym_context *c, OpEntry &op, const Spinor &b, const Spinor &x, const Spinor *guess, double precision,
                int max_steps, lym_solve_stats *st)
{
    const Geom &g = c->g;
    const bool even = g.L[0] % 2 == 0 && g.L[1] % 2 == 0 && g.L[2] % 2 == 0 && g.L[3] % 2 == 0;
    if (op.kind != LYM_OP_IMPROVED || !even) {
        auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
            op_apply(c, op, PREC_D, out, in, nullptr, C2(0.0), skip);
        };
        return bicgstab_solve(c, mv, 2, b, x, guess, precision, max_steps, 0.0, st);
    }
    // the even-odd operators of the reference are default-constructed: gamma5 = true (DiracOperator.cpp:14)
    OpEntry &eo = op;
    Vec bp(c, PREC_D, 1), src(c, PREC_D, 1), te(c, PREC_D, 1), tmp(c, PREC_D, 1);
    schur_source(c, op, b, *bp);
    gamma5_inplace(c, *bp);  // odd_source = gamma5 (b_o + kappa H Tinv b_e)
    apply_schur(c, eo, PREC_D, *src, *bp, *te, 1);  // odd_source_eo = gamma5 S odd_source
    const double norm_even = norm2_now(c, b.parity(0));  // the reference's full-lattice source norm includes gamma5 b_e
    auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
        apply_schur(c, eo, PREC_D, *tmp, in, *te, 1, nullptr, C2(0.0), skip);
        apply_schur(c, eo, PREC_D, out, *tmp, *te, 1, nullptr, C2(0.0), skip);
    };
    Spinor go;
    if (guess) go = guess->parity(1);
    const int rc = bicgstab_solve(c, mv, 1, *src, x.parity(1), guess ? &go : nullptr, precision, max_steps,
                                  norm_even, st);
    schur_reconstruct(c, op, b, x);
    return rc;
}

// Even-odd CG on (gamma5 S)^2 with reliable updates: D x = b to ||b - D x|| <= tol ||b||.
// Inner iterations run in `sprec` (FP64, FP32 or FP16 spinors); x and the true
// residual are FP64.  delta: reliable-update threshold on the recursive residual.
int eo_cg(lym_context *c, OpEntry &op, int sprec, const Spinor &b, const Spinor &x, const Spinor *guess, double tol,
          int max_steps, lym_solve_stats *st)
{
    const double delta = sprec == PREC_D ? 0.0 : 0.1;
    OpEntry &eo = op;  // apply_schur takes gamma5 explicitly
    if (kind_has_clover(op.kind)) ensure_clover(c, op);
    Vec bp(c, PREC_D, 1), rS(c, PREC_D, 1), rN(c, PREC_D, 1), te(c, PREC_D, 1), t1(c, PREC_D, 1);
    Vec xs(c, sprec == PREC_H ? PREC_F : sprec, 1), rs(c, sprec == PREC_H ? PREC_F : sprec, 1);
    Vec ps(c, sprec, 1), tes(c, sprec, 1), tos(c, sprec, 1);
    const Spinor xo = x.parity(1);
    schur_source(c, op, b, *bp);
    const double bb = norm2_now(c, b);
    const double eps_S = tol * tol * bb;
    if (guess) copy(c, xo, guess->parity(1));
    else zero(c, xo);

    // true residuals: r_S = b' - S x, r_N = g5 S g5 r_S ; returns |r_S|^2, |r_N|^2
    auto true_res = [&](double &rrS, double &rrN) {
        apply_schur(c, eo, PREC_D, *t1, xo, *te, 0);
        run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{(*bp).d(), (*t1).d(), (*rS).d(), c->d_scal}, 1);
        copy(c, *t1, *rS);
        gamma5_inplace(c, *t1);
        apply_schur(c, eo, PREC_D, *rN, *t1, *te, 1);
        run_site(c, OpNorm<SpinorD>{(*rN).d(), c->d_scal + 1}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        rrS = c->h_scal[0];
        rrN = c->h_scal[1];
    };
    double rrS, rrN;
    true_res(rrS, rrN);
    int iters = 0, updates = 0, rc = LYM_NOT_CONVERGED;
    CGState *S = cg_state(c);
    Gate gate{&S->pause, nullptr};
    if (rrS < eps_S || bb == 0.0) {
        rc = LYM_OK;
    } else {
        double eps_N = eps_S * (rrN / rrS);
        copy(c, *rs, *rN);
        copy(c, *ps, *rs);
        zero(c, *xs);
        CGState &H = cg_host(c);
        memset(&H, 0, sizeof(H));
        H.rr = rrN;
        H.rr_max = rrN;
        H.eps = eps_N;
        H.delta2 = delta * delta;
        H.max_iter = max_steps;
        push_state(c, sizeof(CGState));
        // one iteration, 5 launches: q = Q p with alpha from |q|^2 = <p, A p>; A p = Q q with
        // x += alpha p, r -= alpha A p and |r|^2 in the same launch; then p = r + beta p
        auto step = [&]() {
            apply_schur_cg(c, eo, sprec, CG_NORM, *tos, *ps, *tes, *ps, *xs, *rs, S, &S->pause);
            apply_schur_cg(c, eo, sprec, CG_UPDATE, *tos, *tos, *tes, *ps, *xs, *rs, S, &S->pause);
            if (sprec == PREC_D) run_site(c, OpCGDirection<SpinorD, SpinorD>{(*ps).d(), (*rs).d(), S}, 1, gate);
            else if (sprec == PREC_F) run_site(c, OpCGDirection<SpinorF, SpinorF>{(*ps).f(), (*rs).f(), S}, 1, gate);
            else run_site(c, OpCGDirection<SpinorH, SpinorF>{(*ps).h(), (*rs).f(), S}, 1, gate);
        };
        for (int outer = 0; outer < 10000; ++outer) {
            run_gated_state(c, S, step, 8, (long)max_steps - cg_host(c).iter + 8);
            CGState R = cg_host(c);
            iters = R.iter;
            if (R.failed) fail(c, LYM_ERR_NUMERIC, "CG produced a non-finite residual");
            // reliable update: x += x_sloppy, recompute the FP64 residuals
            axpby(c, *xs, xo, C2(1.0), C2(1.0));
            zero(c, *xs);
            true_res(rrS, rrN);
            ++updates;
            if (rrS < eps_S) {
                rc = LYM_OK;
                break;
            }
            if (R.iter >= max_steps) break;
            if (R.converged) {
                // recursion converged but the true residual did not: tighten
                eps_N = std::max(eps_N * 0.5 * eps_S / rrS, 1e-300);
            }
            copy(c, *rs, *rN);
            CGState &W = cg_host(c);
            W = R;
            W.beta = rrN / R.rr_prev;
            W.rr = rrN;
            W.rr_max = rrN;
            W.eps = eps_N;
            W.pause = 0;
            W.converged = 0;
            W.need_update = 0;
            push_state(c, sizeof(CGState));
            // p = r + beta p with the true residual
            if (sprec == PREC_D) run_site(c, OpCGDirection<SpinorD, SpinorD>{(*ps).d(), (*rs).d(), S}, 1);
            else if (sprec == PREC_F) run_site(c, OpCGDirection<SpinorF, SpinorF>{(*ps).f(), (*rs).f(), S}, 1);
            else run_site(c, OpCGDirection<SpinorH, SpinorF>{(*ps).h(), (*rs).f(), S}, 1);
        }
    }
    schur_reconstruct(c, op, b, x);
    if (st) {
        st->iterations = iters;
        st->steps = iters;
        st->reliable_updates = updates;
        st->converged = rc == LYM_OK;
        st->last_error = rrS;
    }
    return rc;
}

// Multishift CG on (A + shift_i), A Hermitian positive definite (a Square* kind).
int multishift_cg(lym_context *c, OpEntry &op, int nshift, const double *shifts, double eps, int max_steps,
                  const Spinor &b, std::vector<Spinor> &xs, lym_solve_stats *st)
{
    if (nshift < 1 || nshift > kMaxShifts) fail(c, LYM_ERR_ARGUMENT, "multishift: 1..%d shifts", kMaxShifts);
    int base = 0;
    for (int i = 1; i < nshift; ++i)
        if (shifts[i] < shifts[base]) base = i;
    const double s0 = shifts[base];
    std::vector<Vec *> ps;
    for (int i = 0; i < nshift; ++i) ps.push_back(new Vec(c, PREC_D, 2));
    Vec r(c, PREC_D, 2), ap(c, PREC_D, 2);
    std::vector<SpinorD> hx(nshift), hp(nshift);
    for (int i = 0; i < nshift; ++i) {
        zero(c, xs[i]);
        copy(c, **ps[i], b);
        hx[i] = xs[i].d();
        hp[i] = (**ps[i]).d();
    }
    copy(c, *r, b);
    SpinorD *dviews = (SpinorD *)dev_alloc(c, 2 * kMaxShifts * sizeof(SpinorD));
    CK(cudaMemcpyAsync(dviews, hx.data(), nshift * sizeof(SpinorD), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dviews + kMaxShifts, hp.data(), nshift * sizeof(SpinorD), cudaMemcpyHostToDevice, c->st));
    const double bb = norm2_now(c, b);
    // build the clover term and pool the operator's temporaries before graph capture
    op_apply(c, op, PREC_D, *ap, b, &b, C2(s0));
    MultishiftState &H = *(MultishiftState *)c->h_state;
    memset(&H, 0, sizeof(H));
    H.nshift = nshift;
    H.base = base;
    for (int i = 0; i < nshift; ++i) {
        H.sigma[i] = shifts[i] - s0;
        H.zeta[i] = H.zeta_prev[i] = 1.0;
        H.active[i] = 1;
    }
    H.rr = bb;
    H.alpha = 1.0;
    H.beta = 0.0;
    H.eps = eps;
    H.max_iter = max_steps;
    CK(cudaMemcpyAsync(c->d_state, c->h_state, sizeof(MultishiftState), cudaMemcpyHostToDevice, c->st));
    MultishiftState *S = (MultishiftState *)c->d_state;
    Gate gate{&S->pause, nullptr};
    const Spinor pb = **ps[base];
    auto step = [&]() {
        op_apply(c, op, PREC_D, *ap, pb, &pb, C2(s0), &S->pause);
        run_site(c, OpMsAlpha<SpinorD, SpinorD>{pb.d(), (*ap).d(), S}, 2, gate);
        run_site(c, OpMsResidual<SpinorD, SpinorD>{(*r).d(), (*ap).d(), S}, 2, gate);
        run_site(c, OpMsUpdate<SpinorD>{dviews, dviews + kMaxShifts, (*r).d(), S, nshift}, 2, gate);
    };
    int rc = LYM_OK;
    if (bb > 0 && max_steps > 0) {
        run_gated_state(c, S, step, 4, max_steps);
        MultishiftState &R = *(MultishiftState *)c->h_state;
        rc = R.converged ? LYM_OK : LYM_NOT_CONVERGED;
        if (st) {
            st->iterations = R.iter;
            st->steps = R.iter;
            st->converged = R.converged;
            st->last_error = R.rr;
        }
    }
    for (auto v : ps) delete v;
    dev_free(c, dviews, 2 * kMaxShifts * sizeof(SpinorD));
    return rc;
}

// The odd-site system of the RHMC operator with a shift, M = (G5 S)^2 + sigma, applied in
// `prec` through the Schur complement: out = G5 S (G5 S in) + sigma in.
void schur_square_shift(lym_context *c, OpEntry &op, int prec, const Spinor &out, const Spinor &in,
                        const Spinor &tmp_o, const Spinor &tmp_e, double sigma, const int *skip = nullptr)
{
    apply_schur(c, op, prec, tmp_o, in, tmp_e, 1, nullptr, C2(0.0), skip);
    apply_schur(c, op, prec, out, tmp_o, tmp_e, 1, &in, C2(sigma), skip);
}

// Mixed-precision CG on ((G5 S)^2 + sigma) x_o = b_o from the FP64 x_o it is given: directions
// and operator applications in `sprec`, residual and the solution accumulator in FP32 (FP64 for
// sprec FP64), every inner product and the recurrences in FP64; reliable updates (x += x_sloppy,
// FP64 true residual) whenever the recursive residual falls by delta, and a direction rebuilt
// from the true residual after each.  Stops when |b_o - M x_o|^2 < eps (FP64).
int shift_cg_mixed(lym_context *c, OpEntry &op, int sprec, double sigma, const Spinor &bo, const Spinor &xo,
                   double eps, int max_steps, int &iters, int &updates, double &rr_true)
{
    const int aprec = sprec == PREC_H ? PREC_F : sprec;
    Vec r64(c, PREC_D, 1), t64(c, PREC_D, 1), u64(c, PREC_D, 1), te64(c, PREC_D, 1);
    Vec rs(c, aprec, 1), xs(c, aprec, 1), ps(c, sprec, 1), aps(c, sprec, 1), tos(c, sprec, 1), tes(c, sprec, 1);
    auto true_res = [&]() {
        schur_square_shift(c, op, PREC_D, *u64, xo, *t64, *te64, sigma);
        run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{bo.d(), (*u64).d(), (*r64).d(), c->d_scal}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        return c->h_scal[0];
    };
    rr_true = true_res();
    if (rr_true < eps) return LYM_OK;
    if (max_steps <= 0) return LYM_NOT_CONVERGED;
    copy(c, *rs, *r64);
    copy(c, *ps, *rs);
    zero(c, *xs);
    CGState &H = cg_host(c);
    memset(&H, 0, sizeof(H));
    H.rr = rr_true;
    H.rr_max = rr_true;
    H.eps = eps;
    H.delta2 = sprec == PREC_D ? 0.0 : 0.01;
    H.max_iter = iters + max_steps;
    H.iter = iters;
    push_state(c, sizeof(CGState));
    CGState *S = cg_state(c);
    Gate gate{&S->pause, nullptr};
    double eps_rec = eps;
    auto step = [&]() {
        schur_square_shift(c, op, sprec, *aps, *ps, *tos, *tes, sigma, &S->pause);
        auto go = [&](auto P, auto AP, auto X, auto R) {
            run_site(c, OpCGAlpha<decltype(P), decltype(AP)>{P, AP, S}, 1, gate);
            run_site(c, OpCGUpdate<decltype(X), decltype(P), decltype(R), decltype(AP)>{X, P, R, AP, S}, 1, gate);
            run_site(c, OpCGDirection<decltype(P), decltype(R)>{P, R, S}, 1, gate);
        };
        if (sprec == PREC_D) go((*ps).d(), (*aps).d(), (*xs).d(), (*rs).d());
        else if (sprec == PREC_F) go((*ps).f(), (*aps).f(), (*xs).f(), (*rs).f());
        else go((*ps).h(), (*aps).h(), (*xs).f(), (*rs).f());
    };
    int rc = LYM_NOT_CONVERGED;
    for (int outer = 0; outer < 100000; ++outer) {
        run_gated_state(c, S, step, 8, (long)(H.max_iter - cg_host(c).iter) + 8);
        CGState R = cg_host(c);
        iters = R.iter;
        if (R.failed) fail(c, LYM_ERR_NUMERIC, "shifted CG produced a non-finite residual");
        axpby(c, *xs, xo, C2(1.0), C2(1.0));
        zero(c, *xs);
        rr_true = true_res();
        ++updates;
        if (rr_true < eps) {
            rc = LYM_OK;
            break;
        }
        if (R.iter >= R.max_iter) break;
        if (R.converged) eps_rec = std::max(eps_rec * 0.5 * eps / rr_true, 1e-300);
        copy(c, *rs, *r64);
        CGState &W = cg_host(c);
        W = R;
        W.beta = rr_true / R.rr_prev;
        W.rr = rr_true;
        W.rr_max = rr_true;
        W.eps = eps_rec;
        W.pause = 0;
        W.converged = 0;
        W.need_update = 0;
        push_state(c, sizeof(CGState));
        if (sprec == PREC_D) run_site(c, OpCGDirection<SpinorD, SpinorD>{(*ps).d(), (*rs).d(), S}, 1);
        else if (sprec == PREC_F) run_site(c, OpCGDirection<SpinorF, SpinorF>{(*ps).f(), (*rs).f(), S}, 1);
        else run_site(c, OpCGDirection<SpinorH, SpinorF>{(*ps).h(), (*rs).f(), S}, 1);
    }
    return rc;
}

// Mixed-precision multishift CG for the RHMC operator (SquareEvenOddImproved with gamma5:
// odd <- (G5 S)^2 x_o, even <- x_e; NFlavorFermionAction's multishift on the squared
// operator, actions/NFlavorFermionAction.cpp:76-96).  Even sites: x_e = b_e / (1 + sigma_i).
// Odd sites: one Krylov space on the smallest shift, FP32 storage and operator, the shift
// recurrences (Jegerlehner) and every inner product in FP64.  The shifted x_i and p_i are not
// touched every step: each step records its residual in a ring of kMsWin + 1 slots and
// updates, per shift, the coefficients of x_i and p_i on the window's residuals; one pass per
// window (ms_flush_kernel) applies them, so a step streams the base system's vectors only.
// Whenever the base residual falls by delta = 0.1, the FP32 accumulators are added to the
// FP64 solutions, the base residual is recomputed in FP64 and the directions are rebuilt from
// it (shifted residuals stay zeta_i r).  Then every shift whose FP64 true residual misses eps
// is refined by shift_cg_mixed in `rprec` from its multishift solution.
// eps: |b - (A + sigma_i) x_i|^2 (FP64).
int multishift_cg_mixed(lym_context *c, OpEntry &op, int rprec, int nshift, const double *shifts, double eps,
                        int max_steps, const Spinor &b, std::vector<Spinor> &xs, lym_solve_stats *st)
{
    if (op.kind != LYM_OP_SQUARE_EVEN_ODD_IMPROVED || !op.gamma5)
        fail(c, LYM_ERR_UNSUPPORTED,
             "mixed-precision multishift needs the squared even-odd operator with gamma5 (kind %d, gamma5 %d)",
             op.kind, op.gamma5);
    if (nshift < 1 || nshift > kMaxShifts) fail(c, LYM_ERR_ARGUMENT, "multishift: 1..%d shifts", kMaxShifts);
    for (int i = 0; i < nshift; ++i)
        if (!(1.0 + shifts[i] != 0.0) || !std::isfinite(shifts[i]))
            fail(c, LYM_ERR_ARGUMENT, "multishift: shift %d = %g gives a singular even-site system", i, shifts[i]);
    int base = 0;
    for (int i = 1; i < nshift; ++i)
        if (shifts[i] < shifts[base]) base = i;
    const double s0 = shifts[base];
    const Spinor bo = b.parity(1);
    for (int i = 0; i < nshift; ++i) {
        axpby(c, b.parity(0), xs[i].parity(0), C2(1.0 / (1.0 + shifts[i])), C2(0.0));
        zero(c, xs[i].parity(1));
    }
    const double bbo = norm2_now(c, bo);
    Vec ap(c, PREC_F, 1), tos(c, PREC_F, 1), tes(c, PREC_F, 1);
    Vec r64(c, PREC_D, 1), t64(c, PREC_D, 1), u64(c, PREC_D, 1), te64(c, PREC_D, 1);
    std::vector<Vec *> owned;
    struct Owner {
        std::vector<Vec *> &v;
        ~Owner()
        {
            for (auto p : v) delete p;
        }
    } owner{owned};
    auto fresh = [&]() {
        owned.push_back(new Vec(c, PREC_F, 1));
        return **owned.back();
    };
    std::vector<SpinorF> hring(kMsWin + 1), hacc(nshift), hp(nshift);
    for (int j = 0; j <= kMsWin; ++j) hring[j] = fresh().f();
    for (int i = 0; i < nshift; ++i) {
        const Spinor a = fresh(), p = fresh();
        zero(c, a);
        copy(c, p, bo);
        hacc[i] = a.f();
        hp[i] = p.f();
    }
    // ring slot 0 holds r_0 = b_o
    {
        Spinor r0 = **owned.front();
        copy(c, r0, bo);
    }
    // device arrays of views: ring, accumulators, directions
    const size_t vb = sizeof(SpinorF);
    const size_t nview = (kMsWin + 1) + 2 * kMaxShifts;
    char *dviews = (char *)dev_alloc(c, nview * vb);
    struct ViewsMem {
        lym_context *c;
        void *p;
        size_t n;
        ~ViewsMem() { dev_free(c, p, n); }
    } vmem{c, dviews, nview * vb};
    SpinorF *d_ring = (SpinorF *)dviews;
    SpinorF *d_acc = d_ring + (kMsWin + 1);
    SpinorF *d_p = d_acc + kMaxShifts;
    CK(cudaMemcpyAsync(d_ring, hring.data(), (kMsWin + 1) * vb, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(d_acc, hacc.data(), nshift * vb, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(d_p, hp.data(), nshift * vb, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    auto pview = [&](int i) {
        Spinor v;
        v.prec = PREC_F;
        v.nparity = 1;
        v.stride = c->g.stride;
        v.v = hp[i].v;
        return v;
    };
    auto ring_view = [&](int k) {
        Spinor v;
        v.prec = PREC_F;
        v.nparity = 1;
        v.stride = c->g.stride;
        v.v = hring[k % (kMsWin + 1)].v;
        return v;
    };
    // the base direction of the current step (the operator's input); P_base holds it as of
    // the window start, like every other shift's P_i
    Vec pcur(c, PREC_F, 1);
    copy(c, *pcur, bo);
    const Spinor pb = *pcur;

    // build the clover terms and pool the temporaries before graph capture
    schur_square_shift(c, op, PREC_F, *ap, pb, *tos, *tes, s0);
    schur_square_shift(c, op, PREC_D, *u64, bo, *t64, *te64, s0);

    MultishiftState &H = *(MultishiftState *)c->h_state;
    memset(&H, 0, sizeof(H));
    H.nshift = nshift;
    H.base = base;
    for (int i = 0; i < nshift; ++i) {
        H.sigma[i] = shifts[i] - s0;
        H.zeta[i] = H.zeta_prev[i] = 1.0;
        H.active[i] = 1;
        H.cp[i][0] = 1.0;
    }
    H.rr = bbo;
    H.rr_max = bbo;
    H.alpha = 1.0;
    H.beta = 0.0;
    H.eps = eps;
    H.max_iter = max_steps;
    H.delta2 = 0.01;
    CK(cudaMemcpyAsync(c->d_state, c->h_state, sizeof(MultishiftState), cudaMemcpyHostToDevice, c->st));
    MultishiftState *S = (MultishiftState *)c->d_state;
    Gate gate{&S->pause, nullptr};
    const Spinor xb = xs[base].parity(1);
    int nstep = 0;
    const int fgrid = std::min((c->g.Vh + kMsFlushThreads - 1) / kMsFlushThreads, 4 * 148);
    auto flush = [&]() {
        MsFlushArg fa{d_ring, d_acc, d_p, S, nshift, c->g.Vh};
        ms_flush_kernel<<<fgrid, kMsFlushThreads, 0, c->st>>>(fa);
        ms_window_reset_kernel<<<1, 32, 0, c->st>>>(S, nshift);
        count(c, 2);
    };
    auto step = [&]() {
        schur_square_shift(c, op, PREC_F, *ap, pb, *tos, *tes, s0, &S->pause);
        run_site(c, OpMsAlpha<SpinorF, SpinorF>{pb.f(), (*ap).f(), S}, 1, gate);
        run_site(c, OpMsResidualRing<SpinorF>{d_ring, (*ap).f(), S}, 1, gate);
        run_site(c, OpMsBaseDirection<SpinorF>{d_ring, pb.f(), S}, 1, gate);
        if (++nstep % kMsWin == 0) flush();
    };
    auto base_true_res = [&]() {
        schur_square_shift(c, op, PREC_D, *u64, xb, *t64, *te64, s0);
        run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{bo.d(), (*u64).d(), (*r64).d(), c->d_scal}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        return c->h_scal[0];
    };
    int iters = 0, updates = 0;
    std::vector<int> was_active(nshift, 1);
    if (!(bbo < eps || bbo == 0.0) && max_steps > 0) {
        for (int outer = 0; outer < 100000; ++outer) {
            nstep = 0;
            run_gated_state(c, S, step, kMsWin, (long)max_steps - ((MultishiftState *)c->h_state)->iter + kMsWin);
            MultishiftState R = *(MultishiftState *)c->h_state;
            iters = R.iter;
            if (R.failed) fail(c, LYM_ERR_NUMERIC, "multishift CG produced a non-finite residual");
            // fold the accumulators of every shift that ran since the last fold
            for (int i = 0; i < nshift; ++i) {
                if (!was_active[i]) continue;
                const Spinor a = **owned[(kMsWin + 1) + 2 * i];
                axpby(c, a, xs[i].parity(1), C2(1.0), C2(1.0));
                zero(c, a);
                was_active[i] = R.active[i] != 0;
            }
            const double rr = base_true_res();
            ++updates;
            if (R.converged && rr < eps) break;
            if (R.iter >= max_steps) break;
            MultishiftState &W = *(MultishiftState *)c->h_state;
            W = R;
            if (R.converged) W.eps = std::max(R.eps * 0.5 * eps / rr, 1e-300);
            W.beta = rr / R.rr_prev;
            for (int i = 0; i < nshift; ++i) {
                if (W.active[i] == 2) W.active[i] = 0;
                if (W.active[i] == 1) {
                    const double zr = W.zeta[i] / W.zeta_prev[i];
                    W.beta_s[i] = W.beta * zr * zr;
                }
            }
            W.active[base] = 1;
            W.rr = rr;
            W.rr_max = rr;
            W.pause = W.stop = W.converged = W.need_update = 0;
            CK(cudaMemcpyAsync(c->d_state, c->h_state, sizeof(MultishiftState), cudaMemcpyHostToDevice, c->st));
            const Spinor rcur = ring_view(R.iter);
            copy(c, rcur, *r64);
            run_site(c, OpMsDirection<SpinorF, SpinorF>{d_p, rcur.f(), S, nshift}, 1);
            copy(c, *pcur, pview(base));
        }
    }
    // refinement: every shift to the FP64 target on its own
    int rc = LYM_OK;
    int refine_its = iters;
    double worst = 0.0;
    for (int i = 0; i < nshift; ++i) {
        double rr_i = 0.0;
        const int budget = std::max(0, max_steps - refine_its);
        const int r_i = shift_cg_mixed(c, op, rprec, shifts[i], bo, xs[i].parity(1), eps, budget, refine_its,
                                       updates, rr_i);
        if (r_i != LYM_OK) rc = LYM_NOT_CONVERGED;
        worst = std::max(worst, rr_i);
    }
    if (st) {
        st->iterations = refine_its;
        st->steps = iters;
        st->reliable_updates = updates;
        st->converged = rc == LYM_OK;
        st->last_error = worst;
        const double bb = norm2_now(c, b);
        st->true_residual = bb > 0 ? std::sqrt(worst / bb) : 0.0;
    }
    return rc;
}

// MMMRMultishiftSolver::solve (inverters/MMMRMultishiftSolver.cpp:42-198): negative
// shifts by separate CG, the rest by one minimal-residual Krylov space on the last shift.
int multishift_mmmr(lym_context *c, OpEntry &op, int nshift, const double *shifts, double eps, int max_steps,
                    const Spinor &b, std::vector<Spinor> &xs, lym_solve_stats *st)
{
    if (nshift < 1 || nshift > kMaxShifts) fail(c, LYM_ERR_ARGUMENT, "multishift: 1..%d shifts", kMaxShifts);
    int first = 0, total = 0;
    bool flag = true;
    while (first < nshift && shifts[first] < 0) {
        const double sh = shifts[first];
        auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
            op_apply(c, op, PREC_D, out, in, &in, C2(sh), skip);
        };
        Vec z(c, PREC_D, 2);
        zero(c, *z);
        lym_solve_stats s1;
        memset(&s1, 0, sizeof(s1));
        flag = cg_solve(c, mv, 2, b, xs[first], &*z, eps, max_steps, &s1) == LYM_OK && flag;
        total += s1.iterations;
        ++first;
    }
    int rc = flag ? LYM_OK : LYM_NOT_CONVERGED;
    if (first < nshift) {
        const double last = shifts[nshift - 1];
        Vec r(c, PREC_D, 2), p(c, PREC_D, 2);
        for (int i = first; i < nshift; ++i) zero(c, xs[i]);
        copy(c, *r, b);
        std::vector<SpinorD> hx(nshift);
        for (int i = 0; i < nshift; ++i) hx[i] = xs[i].d();
        SpinorD *dviews = (SpinorD *)dev_alloc(c, kMaxShifts * sizeof(SpinorD));
        CK(cudaMemcpyAsync(dviews, hx.data(), nshift * sizeof(SpinorD), cudaMemcpyHostToDevice, c->st));
        op_apply(c, op, PREC_D, *p, *r, &*r, C2(last));  // clover and pooled temporaries before capture
        MMMRState &H = *(MMMRState *)c->h_state;
        memset(&H, 0, sizeof(H));
        H.nshift = nshift;
        H.first = first;
        H.max_iter = max_steps;
        H.omega = 0.95;
        H.eps = eps;
        for (int i = 0; i < nshift; ++i) {
            H.sigma[i] = shifts[i] - last;
            H.f[i] = C2(1.0);
        }
        CK(cudaMemcpyAsync(c->d_state, c->h_state, sizeof(MMMRState), cudaMemcpyHostToDevice, c->st));
        MMMRState *S = (MMMRState *)c->d_state;
        Gate gate{&S->pause, nullptr};
        auto step = [&]() {
            op_apply(c, op, PREC_D, *p, *r, &*r, C2(last), &S->pause);
            run_site(c, OpMMMRAlpha<SpinorD, SpinorD>{(*p).d(), (*r).d(), S}, 2, gate);
            run_site(c, OpMMMRUpdate<SpinorD>{dviews, (*r).d(), (*p).d(), S}, 2, gate);
        };
        if (max_steps > 0) run_gated_state(c, S, step, 4, max_steps);
        MMMRState &R = *(MMMRState *)c->h_state;
        total += R.iter;
        if (!R.converged) rc = LYM_NOT_CONVERGED;
        if (st) st->last_error = R.rr;
        dev_free(c, dviews, kMaxShifts * sizeof(SpinorD));
    }
    if (st) {
        st->iterations = total;
        st->steps = total;
        st->converged = rc == LYM_OK;
    }
    return rc;
}

// ------------------------------------------------------ multi-RHS (batched) --
size_t batch_bytes(const Geom &g, int prec, int nb)
{
    const size_t s = g.stride;
    return prec == PREC_F ? 6 * s * nb * sizeof(float4) : 3 * s * nb * sizeof(int4) + s * nb * sizeof(float);
}

struct BVec {
    lym_context *c;
    SpinorBatch s;
    size_t bytes;
    BVec(lym_context *ctx, int prec, int nb) : c(ctx)
    {
        if (nb < 2 || nb > kMaxBatch || (nb & (nb - 1))) fail(c, LYM_ERR_ARGUMENT, "batch width %d", nb);
        if ((double)12 * c->g.stride * nb / 2 >= 4294967296.0 || (double)72 * c->g.stride >= 4294967296.0)
            fail(c, LYM_ERR_UNSUPPORTED, "lattice too large for the batched stencil's 32-bit word indices");
        s.prec = prec;
        s.nb = nb;
        s.lognb = 0;
        while ((1 << s.lognb) < nb) ++s.lognb;
        s.stride = c->g.stride;
        bytes = batch_bytes(c->g, prec, nb);
        char *base = (char *)block_alloc(c, bytes);
        s.v = base;
        if (prec == PREC_H) s.norm = (float *)(base + (size_t)3 * s.stride * nb * sizeof(int4));
    }
    ~BVec() { block_free(c, s.v, bytes); }
    BVec(const BVec &) = delete;
    BVec &operator=(const BVec &) = delete;
    BatchF f() const { return BatchF{(float4 *)s.v, s.stride, s.lognb - 1}; }
    BatchH h() const { return BatchH{(int4 *)s.v, (float2 *)s.norm, s.stride, s.lognb - 1}; }
};

template <class Op> void run_batch(lym_context *c, const Op &op, int lognb, Gate gate = Gate{nullptr, nullptr})
{
    count(c, 1);
    const int lognp = lognb - 1;
    const long threads = (long)c->g.Vh << lognp;
    const int grid = (int)std::min<long>((threads + kBlasThreads - 1) / kBlasThreads, kBlasGridMax);
    static_assert(Op::NRED <= kBatchMaxRed, "the per-RHS partial sums are sized for kBatchMaxRed reductions");
    site_batch_kernel<Op><<<grid, kBlasThreads, 0, c->st>>>(op, c->g.Vh, lognp, c->bpartials, c->counter, gate);
}

const int *order_table(lym_context *c, int by, int bz)
{
    if (by == 0) return nullptr;
    const int key = by * 4096 + bz;
    auto it = c->orders.find(key);
    if (it != c->orders.end()) return it->second;
    if (c->capturing) fail(c, LYM_ERR_ARGUMENT, "traversal tables must be built before graph capture");
    int *t = (int *)dev_alloc(c, (size_t)c->g.stride * sizeof(int));
    launch_order_table(c->g, by, bz, t, c->st);
    count(c, 1);
    c->orders[key] = t;
    return t;
}

// Traversal columns worth timing: plain half-site order (x slowest), columns of 2, 4, 8
// and 12 y-rows spanning z, and square (y, z) columns of 4 and 8.
std::vector<BatchTile> tile_candidates(const Geom &g)
{
    std::vector<BatchTile> out;
    out.push_back(BatchTile{0, 0, 1});
    const int Ly = g.L[1], Lz = g.L[2];
    auto add = [&](int by, int bz) {
        if (by < 1 || bz < 1 || Ly % by || Lz % bz || (by == Ly && bz == Lz)) return;
        for (auto &t : out)
            if (t.by == by && t.bz == bz) return;
        out.push_back(BatchTile{by, bz, 1});
    };
    for (int by : {2, 4, 8, 12}) add(by, Lz);
    for (int b : {4, 8}) add(b, b);
    return out;
}

// Schur complement on a batch whose slots share the gauge field and may carry their own
// kappa and clover terms (per-slot tables b_slot = -kappa^2, T, Tinv in device memory):
//   out_r = G5^g (T_oo,r in_r - kappa_r^2 H_oe T_ee,r^-1 H_eo in_r)
// res_r, res_s, res_alpha (optional): with the second launch, s = r - alpha out per RHS
// om_rhat, om_scratch, om_state (optional, batch_omega_fusable variants): with the second
// launch, the BiCGStab omega sums of out, in and rhat, then the omega update of the state
void apply_schur_batch(lym_context *c, const GaugeDev &U, bool clov, int prec, const SpinorBatch &out,
                       const SpinorBatch &in, const SpinorBatch &tmp, int gamma5, const int *skip, const int *active,
                       const double *b_slot, const void *const *T_slot, const void *const *Ti_slot,
                       const BatchTile &tile, const int *uniform, const SpinorBatch *res_r = nullptr,
                       const SpinorBatch *res_s = nullptr, const double2 *res_alpha = nullptr,
                       const SpinorBatch *om_rhat = nullptr, double *om_scratch = nullptr, void *om_state = nullptr)
{
    if (!U.recon_ok)  // the batched stencil reads the 12-real FP32 links
        fail(c, LYM_ERR_UNSUPPORTED, "batched solves need +-SU(3) / +-SO(3) links (their FP32 links are reconstructed)");
    DslashBatchParams P;
    P.g = c->g;
    P.prec = prec;
    P.rep = c->rep;
    P.U = &U;
    P.skip_if = skip;
    P.active = active;
    P.nbr = c->nbr;
    P.order = order_table(c, tile.by, tile.bz);
    P.err = c->d_err + 1;  // the copy-wait word of the bulk-copy variant
    P.walk_by = tile.by;
    P.walk_bz = tile.bz;
    P.minb = tile.minb;
    P.has_clover = clov;
    P.uniform = uniform;
    P.epi = clov ? EPI_CLOVINV_ : EPI_SCALE_;
    P.parity = 0;
    P.in = in;
    P.out = tmp;
    P.y = tmp;
    P.clover_slot = clov ? Ti_slot : nullptr;
    P.a = 1.0;
    launch_dslash_batch(P, c->st);
    P.epi = res_r ? EPI_XPAY_RES_ : EPI_XPAY_;
    P.parity = 1;
    P.in = tmp;
    P.out = out;
    P.y = in;
    P.clover_slot = clov ? T_slot : nullptr;
    P.b_slot = b_slot;
    P.gamma5 = gamma5;
    if (res_r) {
        P.res_r = *res_r;
        P.res_s = *res_s;
        P.res_alpha = res_alpha;
    }
    if (om_rhat) {
        if (!batch_omega_fusable(tile.minb, prec) || res_r || gamma5)
            fail(c, LYM_ERR_ARGUMENT, "the omega sums need the FP32 staged stencil without other fusions");
        P.epi = EPI_XPAY_OMEGA_;
        P.om_rhat = *om_rhat;
        P.om_partials = om_scratch;
    }
    launch_dslash_batch(P, c->st);
    count(c, 2);
    if (om_rhat) {
        launch_omega_finalize(om_scratch, c->g, out.lognb, om_state, c->st);
        count(c, 2);
    }
}

// the squared fall of the recursive residual that triggers a block solve's FP64 reliable
// update with FP32 inner storage, and the fraction (1/n) of busy slots parked for their
// updates that pauses the batched loop
#ifndef LYM_BLOCK_DELTA2_F
#define LYM_BLOCK_DELTA2_F 1e-4
#endif
#ifndef LYM_BLOCK_PARK_FRACTION
#define LYM_BLOCK_PARK_FRACTION 8
#endif

// The bulk-copy variant of the batched stencil (minb & 32) gives up a copy wait after a
// bounded number of polls and sets a word of its own (d_err[1]); the calls that ran it read
// that word once they have synchronised and fail with LYM_ERR_TIMEOUT when it is set.
void check_copy_waits(lym_context *c, const BatchTile &t)
{
    if (!(t.minb & 32)) return;
    CK(cudaMemcpyAsync(c->h_scal, c->d_err + 1, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int e = 0;
    memcpy(&e, c->h_scal, sizeof(int));
    if (c->inject_copy_wait) {  // host-side fault injection (lym_context_inject_copy_wait_timeout)
        c->inject_copy_wait = false;
        e = 1;
    }
    if (e) {
        CK(cudaMemsetAsync(c->d_err + 1, 0, sizeof(int), c->st));
        fail(c, LYM_ERR_TIMEOUT, "a bulk copy of the batched stencil did not complete in its bounded wait");
    }
}

// Autotuner of the batched stencil: times one batched Schur application for every
// traversal column and kernel variant on the caller's fields (in is read, tmp and out
// are overwritten) and keeps the fastest per (precision, batch width, clover).
BatchTile tune_batch(lym_context *c, const GaugeDev &U, bool clov, int prec, const SpinorBatch &out,
                     const SpinorBatch &in, const SpinorBatch &tmp, const double *b_slot, const void *const *T_slot,
                     const void *const *Ti_slot, const int *uniform)
{
    if (c->tile_forced) {
        order_table(c, c->forced_tile.by, c->forced_tile.bz);  // built now, before any capture
        return c->forced_tile;
    }
    const int key = (prec * 64 + in.nb) * 2 + (clov ? 1 : 0);
    auto it = c->tiles.find(key);
    if (it != c->tiles.end()) return it->second;
    if (c->capturing) fail(c, LYM_ERR_ARGUMENT, "the batched stencil must be tuned before graph capture");
    // one tuning at a time in the process: contexts that tune together (a server's lanes
    // taking their first requests) would time each other's launches
    static std::mutex tune_mu;
    std::lock_guard<std::mutex> tune_lock(tune_mu);
    auto time_of = [&](const BatchTile &t, int reps) {
        CK(cudaEventRecord(c->ev0, c->st));
        for (int r = 0; r < reps; ++r)
            apply_schur_batch(c, U, clov, prec, out, in, tmp, 1, nullptr, nullptr, b_slot, T_slot, Ti_slot, t, uniform);
        CK(cudaEventRecord(c->ev1, c->st));
        CK(cudaEventSynchronize(c->ev1));
        CK(cudaGetLastError());
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        return ms / reps;
    };
    // a first pass of 3 applications per candidate (after one untimed), then the six
    // fastest again, 5 applications each in 3 interleaved rounds, keeping each one's best
    // round: single short timings differ by several per cent from launch to launch
    std::vector<std::pair<float, BatchTile>> timed;
    for (BatchTile t : tile_candidates(c->g)) {
        for (int k = 0; k < kBatchTunedCount; ++k) {
            t.minb = kBatchMinBlocks[k];
            apply_schur_batch(c, U, clov, prec, out, in, tmp, 1, nullptr, nullptr, b_slot, T_slot, Ti_slot, t, uniform);
            timed.emplace_back(time_of(t, 3), t);
        }
    }
    std::stable_sort(timed.begin(), timed.end(),
                     [](const std::pair<float, BatchTile> &a, const std::pair<float, BatchTile> &b) {
                         return a.first < b.first;
                     });
    timed.resize(std::min<size_t>(timed.size(), 6));
    std::vector<float> best_round(timed.size(), 1e30f);
    for (int round = 0; round < 3; ++round)
        for (size_t i = 0; i < timed.size(); ++i) best_round[i] = std::min(best_round[i], time_of(timed[i].second, 5));
    size_t pick = 0;
    for (size_t i = 1; i < timed.size(); ++i)
        if (best_round[i] < best_round[pick]) pick = i;
    const BatchTile best = timed[pick].second;
    c->tiles[key] = best;
    return best;
}

// y = a x + b y between a slot of a batch and a single FP64 half spinor (either way)
template <class X, class Y> void axpby_views(lym_context *c, const X &x, const Y &y, double2 a, double2 b)
{
    run_site(c, OpAxpby<X, Y>{x, y, a, b}, 1);
}

// Per-slot operator tables of a batch in device memory: b = -kappa^2 and the FP32
// clover bases T / Tinv of every slot (freed with the object).
struct SlotTables {
    lym_context *c;
    char *mem;
    double *b;
    const void **T, **Ti;
    int *uniform;
    static constexpr size_t kBytes = 3 * kMaxBatch * sizeof(double) + 16;
    SlotTables(lym_context *ctx, const std::vector<const OpEntry *> &ops) : c(ctx)
    {
        mem = (char *)dev_alloc(c, kBytes);
        b = (double *)mem;
        T = (const void **)(mem + kMaxBatch * sizeof(double));
        Ti = (const void **)(mem + 2 * kMaxBatch * sizeof(double));
        uniform = (int *)(mem + 3 * kMaxBatch * sizeof(double));
        std::vector<double> hb(ops.size());
        std::vector<const void *> hT(ops.size()), hTi(ops.size());
        for (size_t j = 0; j < ops.size(); ++j) {
            const bool clov = kind_has_clover(ops[j]->kind);
            hb[j] = -ops[j]->kappa * ops[j]->kappa;
            hT[j] = clov ? ops[j]->clover.T[PREC_F] : nullptr;
            hTi[j] = clov ? ops[j]->clover.Tinv[PREC_F] : nullptr;
        }
        try {
            CK(cudaMemcpyAsync(b, hb.data(), ops.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(T, hT.data(), ops.size() * sizeof(void *), cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(Ti, hTi.data(), ops.size() * sizeof(void *), cudaMemcpyHostToDevice, c->st));
            int uni = 1;
            for (size_t j = 1; j < ops.size(); ++j) uni &= hT[j] == hT[0];
            CK(cudaMemcpyAsync(uniform, &uni, sizeof(int), cudaMemcpyHostToDevice, c->st));
            CK(cudaStreamSynchronize(c->st));
        } catch (...) {
            dev_free(c, mem, kBytes);
            throw;
        }
    }
    ~SlotTables() { dev_free(c, mem, kBytes); }
    SlotTables(const SlotTables &) = delete;
    SlotTables &operator=(const SlotTables &) = delete;
};

// ----------------------------------------- reference solver variants (FP64) --
double2 dot_now(lym_context *c, const Spinor &a, const Spinor &b)
{
    run_site(c, OpDot<SpinorD, SpinorD>{a.d(), b.d(), c->d_scal}, a.nparity);
    CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return make_double2(c->h_scal[0], c->h_scal[1]);
}
typedef std::complex<double> zc;
inline zc zc_of(double2 v) { return zc(v.x, v.y); }
inline double2 d2_of(zc v) { return make_double2(v.real(), v.imag()); }

// BiCGStab(l): BiConjugateGradient::solve(dirac, source, solution, int l, guess)
// (inverters/BiConjugateGradient.cpp:130-317), step for step: the l BiCG steps, then the
// minimal-residual polynomial update (tau, sigma, gamma, gamma', gamma'').
int bicgstab_l_solve(lym_context *c, OpEntry &op, int l, const Spinor &b, const Spinor &x, const Spinor *guess,
                     double precision, int max_steps, lym_solve_stats *st)
{
    auto A = [&](const Spinor &out, const Spinor &in) { op_apply(c, op, PREC_D, out, in, nullptr, C2(0.0)); };
    std::vector<std::unique_ptr<Vec>> u, r;
    for (int j = 0; j <= l; ++j) {
        u.emplace_back(new Vec(c, PREC_D, 2));
        r.emplace_back(new Vec(c, PREC_D, 2));
    }
    Vec rh(c, PREC_D, 2), tmp(c, PREC_D, 2);
    reference_start(c, b, x, guess, precision, 0.0, 2);
    A(*tmp, x);
    copy(c, **r[0], b);
    axpby(c, *tmp, **r[0], C2(-1.0), C2(1.0));
    copy(c, *rh, b);
    axpby(c, *tmp, *rh, C2(1.0), C2(1.0));
    zero(c, **u[0]);
    zc rho0 = 1.0, alpha = 0.0, omega = 1.0;
    std::vector<zc> tau((l + 1) * (l + 1)), sigma(l + 1), gam(l + 1), gp(l + 1), gpp(l + 1);
    auto T = [&](int i, int j) -> zc & { return tau[i * (l + 1) + j]; };
    int step = 0;
    bool ok = false;
    double last = 0.0;
    while (step < max_steps) {
        rho0 = -omega * rho0;
        for (int j = 0; j < l; ++j) {
            const zc rho1 = zc_of(dot_now(c, **r[j], *rh));
            const zc beta = (rho1 / rho0) * alpha;
            rho0 = rho1;
            for (int i = 0; i <= j; ++i) axpby(c, **r[i], **u[i], C2(1.0), d2_of(-beta));
            A(**u[j + 1], **u[j]);
            alpha = rho0 / zc_of(dot_now(c, **u[j + 1], *rh));
            for (int i = 0; i <= j; ++i) axpby(c, **u[i + 1], **r[i], d2_of(-alpha), C2(1.0));
            A(**r[j + 1], **r[j]);
            axpby(c, **u[0], x, d2_of(alpha), C2(1.0));
        }
        for (int j = 1; j <= l; ++j) {
            for (int i = 1; i < j; ++i) {
                T(i, j) = zc_of(dot_now(c, **r[j], **r[i])) / sigma[i];
                axpby(c, **r[i], **r[j], d2_of(-T(i, j)), C2(1.0));
            }
            sigma[j] = zc_of(dot_now(c, **r[j], **r[j]));
            gp[j] = zc_of(dot_now(c, **r[0], **r[j])) / sigma[j];
        }
        gam[l] = gp[l];
        omega = gam[l];
        for (int j = l - 1; j > 0; --j) {
            zc t = 0.0;
            for (int i = j + 1; i <= l; ++i) t += T(j, i) * gam[i];
            gam[j] = gp[j] - t;
        }
        for (int j = 1; j < l; ++j) {
            zc t = 0.0;
            for (int i = j + 1; i < l; ++i) t += T(j, i) * gam[i + 1];
            gpp[j] = gam[j + 1] + t;
        }
        axpby(c, **r[0], x, d2_of(gam[1]), C2(1.0));
        axpby(c, **r[l], **r[0], d2_of(-gp[l]), C2(1.0));
        axpby(c, **u[l], **u[0], d2_of(-gam[l]), C2(1.0));
        for (int j = 1; j < l; ++j) {
            axpby(c, **u[j], **u[0], d2_of(-gam[j]), C2(1.0));
            axpby(c, **r[j], x, d2_of(gpp[j]), C2(1.0));
            axpby(c, **r[j], **r[0], d2_of(-gp[j]), C2(1.0));
        }
        last = norm2_now(c, **r[0]);
        if (last < precision) {
            ok = true;
            break;
        }
        if (!(last == last)) break;  // diverged to non-finite values
        ++step;
    }
    if (st) {
        st->iterations = ok ? step + 1 : step;
        st->steps = ok ? step : max_steps;
        st->converged = ok;
        st->last_error = last;
    }
    return ok ? LYM_OK : LYM_NOT_CONVERGED;
}

// BiCGStab with a preconditioner operator P: BiConjugateGradient::solve(dirac, source,
// solution, preconditioner, guess) (inverters/BiConjugateGradient.cpp:11-128), step for
// step, including its t = A s (not A P s) and its convergence test only after step 5.
int bicgstab_precond_solve(lym_context *c, OpEntry &op, OpEntry &pre, const Spinor &b, const Spinor &x,
                           const Spinor *guess, double precision, int max_steps, lym_solve_stats *st)
{
    auto A = [&](const Spinor &out, const Spinor &in) { op_apply(c, op, PREC_D, out, in, nullptr, C2(0.0)); };
    auto P = [&](const Spinor &out, const Spinor &in) { op_apply(c, pre, PREC_D, out, in, nullptr, C2(0.0)); };
    Vec r(c, PREC_D, 2), rh(c, PREC_D, 2), p(c, PREC_D, 2), nu(c, PREC_D, 2), s(c, PREC_D, 2), t(c, PREC_D, 2),
        pt(c, PREC_D, 2), sts(c, PREC_D, 2);
    reference_start(c, b, x, guess, precision, 0.0, 2);
    A(*p, x);
    copy(c, *r, b);
    axpby(c, *p, *r, C2(-1.0), C2(1.0));
    copy(c, *rh, b);
    axpby(c, *p, *rh, C2(1.0), C2(1.0));
    zc rho_prev = 0.0, alpha = 0.0, omega = 0.0;
    int step = 0, rc = LYM_NOT_CONVERGED;
    double last = 0.0;
    while (step < max_steps) {
        const zc rho = zc_of(dot_now(c, *rh, *r));
        if (std::norm(rho) == 0.0) {
            rc = LYM_ERR_BREAKDOWN;
            break;
        }
        if (step == 0) {
            copy(c, *p, *r);
        } else {
            const zc beta = (rho / rho_prev) * (alpha / omega);
            axpby(c, *nu, *p, d2_of(-omega), C2(1.0));
            axpby(c, *r, *p, C2(1.0), d2_of(beta));
        }
        P(*pt, *p);
        A(*nu, *pt);
        alpha = rho / zc_of(dot_now(c, *rh, *nu));
        copy(c, *s, *r);
        axpby(c, *nu, *s, d2_of(-alpha), C2(1.0));
        P(*sts, *s);
        A(*t, *s);
        omega = zc_of(dot_now(c, *t, *s)) / norm2_now(c, *t);
        axpby(c, *pt, x, d2_of(alpha), C2(1.0));
        axpby(c, *sts, x, d2_of(omega), C2(1.0));
        copy(c, *r, *s);
        axpby(c, *t, *r, d2_of(-omega), C2(1.0));
        const double norm = norm2_now(c, *r);
        if (norm < precision && step > 5) {
            rc = LYM_OK;
            last = norm;
            break;
        }
        rho_prev = rho;
        last = norm;
        ++step;
    }
    if (st) {
        st->iterations = rc == LYM_OK ? step + 1 : step;
        st->steps = rc == LYM_OK ? step : max_steps;
        st->converged = rc == LYM_OK;
        st->last_error = last;
    }
    return rc;
}

// Chronological multishift: ChronologicalMultishiftSolver::solve
// (inverters/ChronologicalMultishiftSolver.cpp:11-194).  Shift 0 by CG from zero; shift k
// by CG from c1 x_{k-1} + c2 h_k, the combination minimising |(A + s_k)(.) - b| in the
// reference's closed form, where h_k (the chronological guess) is what xs[k] holds on
// entry.  A singular 2x2 system (h_k = 0 or parallel) takes c2 = 0 and the one-vector
// minimiser for c1.
int multishift_chrono(lym_context *c, OpEntry &op, int nshift, const double *shifts, double eps, int max_steps,
                      const Spinor &b, const std::vector<Spinor> &xs, lym_solve_stats *st)
{
    Vec pA(c, PREC_D, 2), hA(c, PREC_D, 2), g(c, PREC_D, 2);
    int total = 0;
    bool ok = true;
    for (int i = 0; i < nshift; ++i) {
        const double sh = shifts[i];
        auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
            op_apply(c, op, PREC_D, out, in, &in, C2(sh), skip);
        };
        if (i == 0) {
            zero(c, *g);
        } else {
            mv(*pA, xs[i - 1], nullptr);
            mv(*hA, xs[i], nullptr);
            typedef std::complex<long double> lz;
            const long double pApA = norm2_now(c, *pA), hAhA = norm2_now(c, *hA);
            const double2 d1 = dot_now(c, *pA, b), d2 = dot_now(c, *hA, b), d3 = dot_now(c, *hA, *pA);
            const lz pAb(d1.x, d1.y), hAb(d2.x, d2.y), hApA(d3.x, d3.y);
            const lz den = -(hAhA * pApA) + hApA * std::conj(hApA);
            zc c1, c2;
            if (std::abs(den) > 1e-12L * hAhA * pApA && hAhA > 0) {
                const lz mi(0.0L, -0.5L);
                const long double c1R = std::real((-(hAhA * pAb) + hApA * std::conj(hAb) + hAb * std::conj(hApA) -
                                                   hAhA * std::conj(pAb)) / (lz(2.0L) * den));
                const long double c1I = std::real(mi * (-(hAhA * pAb) - hApA * std::conj(hAb) +
                                                        hAb * std::conj(hApA) + hAhA * std::conj(pAb)) / den);
                const long double c2R = std::real((hApA * pAb - hAb * pApA - pApA * std::conj(hAb) +
                                                   std::conj(hApA) * std::conj(pAb)) / (lz(2.0L) * den));
                const long double c2I = std::real(mi * (hApA * pAb - hAb * pApA + pApA * std::conj(hAb) -
                                                        std::conj(hApA) * std::conj(pAb)) / den);
                c1 = zc((double)c1R, (double)c1I);
                c2 = zc((double)c2R, (double)c2I);
            } else {
                c1 = pApA > 0 ? zc((double)(pAb.real() / pApA), (double)(pAb.imag() / pApA)) : zc(0.0);
                c2 = 0.0;
            }
            copy(c, *g, xs[i]);
            axpby(c, xs[i - 1], *g, d2_of(c1), d2_of(c2));
        }
        lym_solve_stats s1;
        memset(&s1, 0, sizeof(s1));
        const int rc = cg_solve(c, mv, 2, b, xs[i], &*g, eps, max_steps, &s1);
        ok = ok && rc == LYM_OK;
        total += s1.iterations;
    }
    if (st) {
        st->iterations = st->steps = total;
        st->converged = ok;
    }
    return ok ? LYM_OK : LYM_NOT_CONVERGED;
}

enum BlockAlgo : int { ALGO_CG = 0, ALGO_BICGSTAB = 1 };

// Block even-odd CG engine: nb slots on one resident gauge field.  Every slot solves its
// own D_slot x = b (its own kappa / clover term) by CG on (gamma5 S)^2 with its own FP64
// scalars, convergence mask and FP64 reliable updates; one batched stencil serves all
// slots.  Slots are filled with add(), advanced together with advance(), and can be
// refilled as soon as they finish (continuous batching).  The engine uses the context's
// device solver state exclusively while it lives.
class BlockEngine {
public:
    struct Slot {
        bool busy = false, finished = false;
        OpEntry *op = nullptr;
        Spinor B, X;
        Vec *bp = nullptr;
        double epsS = 0.0, bb = 0.0;
        int start_iter = 0, iters = 0, updates = 0, max_iter = 0, converged = 0;
        long long tag = -1;
        // BiCGStab progress: the best true residual so far, updates without a halving of it,
        // breakdown restarts; gave_up: stopped without convergence for another solver
        double best_rr = 0.0;
        int stalls = 0, restarts = 0;
        bool gave_up = false;
        // the source or the FP64 true residual is not finite: the slot stops unconverged,
        // alone (its batch mates go on), and is not handed to another solver
        bool nonfinite = false;
    };

    // algo ALGO_CG: CG on (gamma5 S)^2 (per iteration S^+ S p); ALGO_BICGSTAB: BiCGStab on S
    // itself (per iteration S p and S s), both with FP64 reliable updates
    BlockEngine(lym_context *ctx, int sprec_, int nb_, int algo_ = ALGO_CG)
        : c(ctx), sprec(sprec_), nb(nb_), algo(algo_), te(ctx, PREC_D, 1), t1(ctx, PREC_D, 1), rS(ctx, PREC_D, 1),
          rN(ctx, PREC_D, 1), xs(ctx, PREC_F, nb_), rs(ctx, PREC_F, nb_), ps(ctx, sprec_, nb_), aps(ctx, sprec_, nb_),
          tes(ctx, sprec_, nb_), tos(ctx, sprec_, nb_)
    {
        if (algo == ALGO_BICGSTAB) {
            svec.reset(new BVec(c, sprec, nb));
            rhat.reset(new BVec(c, PREC_F, nb));
            what.reset(new BVec(c, PREC_F, nb));
            for (BVec *v : {svec.get(), rhat.get(), what.get()}) CK(cudaMemsetAsync(v->s.v, 0, v->bytes, c->st));
            for (int j = 0; j < nb; ++j) {
                rhat_c[j].reset(new Vec(c, PREC_F, 1));
                what_c[j].reset(new Vec(c, PREC_F, 1));
            }
        }
        tables = (char *)dev_alloc(c, kTableBytes);
        d_b = (double *)tables;
        d_T = (const void **)(tables + kMaxBatch * sizeof(double));
        d_Ti = (const void **)(tables + 2 * kMaxBatch * sizeof(double));
        d_uniform = (int *)(tables + 3 * kMaxBatch * sizeof(double));
        CK(cudaMemsetAsync(tables, 0, kTableBytes, c->st));
        for (BVec *v : {&xs, &rs, &ps, &aps, &tes, &tos}) CK(cudaMemsetAsync(v->s.v, 0, v->bytes, c->st));
        memset(&hs, 0, sizeof(hs));
        hs.nb = nb;
        // reliable update when the recursive residual fell by 10x (FP16 inner storage) or
        // by 100x (FP32, whose rounding drift stays far below that between updates)
        hs.delta2 = sprec == PREC_H ? 0.01 : LYM_BLOCK_DELTA2_F;
        static_assert(sizeof(BatchCGState) <= kStateBytes, "state buffer too small");
    }
    ~BlockEngine()
    {
        if (exec) cudaGraphExecDestroy(exec);
        for (int j = 0; j < nb; ++j) delete slot[j].bp;
        dev_free(c, tables, kTableBytes);
    }

    int free_slot() const
    {
        for (int j = 0; j < nb; ++j)
            if (!slot[j].busy) return j;
        return -1;
    }
    bool working() const
    {
        for (int j = 0; j < nb; ++j)
            if (slot[j].busy && !slot[j].finished) return true;
        return false;
    }
    const Slot &info(int j) const { return slot[j]; }

    // Puts D x = b in slot j.  B, X: full FP64 spinors that stay alive until release(j).
    void add(int j, OpEntry &op, const Spinor &B, const Spinor &X, double tol, int max_iter, long long tag)
    {
        const bool clov = kind_has_clover(op.kind);
        if (gauge_id >= 0 && (op.gauge_id != gauge_id || clov != has_clover))
            fail(c, LYM_ERR_ARGUMENT, "the slots of one batch share the gauge field and operator kind");
        if (clov) ensure_clover(c, op);
        const double b = -op.kappa * op.kappa;
        const void *T = clov ? op.clover.T[PREC_F] : nullptr, *Ti = clov ? op.clover.Tinv[PREC_F] : nullptr;
        if (gauge_id < 0) {
            // first operator: every slot's table entry points at it (an idle lane of a pair
            // borrows valid operator data), then the batched stencil is tuned on it; the
            // engine takes the operator only once that has succeeded
            for (int k = 0; k < nb; ++k) set_tables(k, b, T, Ti);
            const BatchTile t =
                tune_batch(c, gauge_of(c, op.gauge_id).dev, clov, sprec, tos.s, ps.s, tes.s, d_b, d_T, d_Ti, d_uniform);
            if (algo == ALGO_BICGSTAB && batch_omega_fusable(t.minb, sprec))
                om_scratch.reset(new DevBuf(c, omega_scratch_doubles(c->g, xs.s.lognb) * sizeof(double)));
            tile = t;
            gauge_id = op.gauge_id;
            has_clover = clov;
        }
        Slot &s = slot[j];
        delete s.bp;
        s = Slot();
        s.busy = true;
        hs.its[j] = 0;
        s.op = &op;
        s.B = B;
        s.X = X;
        s.tag = tag;
        s.max_iter = max_iter;
        s.start_iter = hs.iter;
        s.bp = new Vec(c, PREC_D, 1);
        schur_source(c, op, B, **s.bp);
        s.bb = norm2_now(c, B);
        if (!std::isfinite(s.bb)) {
            s.nonfinite = true;
            zero(c, X);
            finish(j);
            return;
        }
        s.epsS = tol * tol * s.bb;
        zero(c, X.parity(1));
        set_tables(j, b, T, Ti);
        hs.x_reset[j] = 1;  // the slot's FP32 accumulator starts from zero in its first update pass
        double rrS, rrN = 0.0;
        // x = 0: the residual is the Schur source itself (S 0 = 0), so no operator is applied
        if (algo == ALGO_BICGSTAB) true_res_S(j, rrS, true);  // synchronises: the host values above were consumed
        else true_res(j, rrS, rrN, true);
        if (rrS < s.epsS || s.bb == 0.0) {
            s.converged = 1;
            finish(j);
            return;
        }
        hs.converged[j] = hs.need_update[j] = hs.restart[j] = 0;
        hs.last_update_its[j] = 0;
        if (algo == ALGO_BICGSTAB) {
            s.best_rr = rrS;
            restart_bicg(j, rrS);
            hs.eps[j] = s.epsS;
        } else {
            axpby_views(c, (*rN).d(), rs.f().slot(j), C2(1.0), C2(0.0));
            set_direction(j, 0.0);
            hs.active[j] = 1;
            hs.rr[j] = hs.rr_max[j] = rrN;
            hs.eps[j] = s.epsS * (rrN / rrS);
        }
    }

    static double wall() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
    // Iterates the running slots until the captured loop pauses (slots parked for their
    // FP64 reliable update, iteration limit, nothing left running), then services the
    // parked slots.  Returns the slots that finished since the last call.
    std::vector<int> advance()
    {
        service();
        if (any_active()) {
            int left = 1 << 30, busy = 0;
            for (int j = 0; j < nb; ++j)
                if (slot[j].busy && !slot[j].finished) {
                    ++busy;
                    if (hs.active[j]) left = std::min(left, slot[j].max_iter - hs.its[j]);
                }
            left = std::max(left, 1);
            hs.max_iter = hs.iter + left;
            hs.park_limit = std::max(1, busy / kParkFraction);
            hs.pause = 0;
            *(BatchCGState *)c->h_state = hs;
            CK(cudaMemcpyAsync(c->d_state, c->h_state, sizeof(BatchCGState), cudaMemcpyHostToDevice, c->st));
            BatchCGState *S = (BatchCGState *)c->d_state;
            const int iter0 = hs.iter;
            long its0 = 0;
            for (int j = 0; j < nb; ++j) its0 += hs.its[j];
            const double t0 = wall();
            run_loop(S, (long)left + kGraphIters);
            c->engine_stats[0] += wall() - t0;
            c->engine_stats[5] += 1;
            hs = *(BatchCGState *)c->h_state;
            long its1 = 0;
            for (int j = 0; j < nb; ++j) its1 += hs.its[j];
            c->engine_stats[7] += hs.iter - iter0;  // batch iterations
            c->engine_stats[8] += its1 - its0;      // iterations of the slots taking part
            if (hs.failed) fail(c, LYM_ERR_NUMERIC, "block CG produced a non-finite residual");
            direction_rest(S);
            for (int j = 0; j < nb; ++j) {
                Slot &s = slot[j];
                if (s.busy && !s.finished && hs.active[j] && hs.its[j] >= s.max_iter) {
                    if (!hs.x_reset[j]) axpby_views(c, xs.f().slot(j), s.X.parity(1).d(), C2(1.0), C2(1.0));
                    finish(j);
                }
            }
            service();
        }
        std::vector<int> out;
        out.swap(done_list);
        return out;
    }

    // forget a finished slot (its B and X are the caller's again)
    void release(int j)
    {
        delete slot[j].bp;
        slot[j] = Slot();
        hs.active[j] = 0;
    }

private:
    lym_context *c;
    int sprec, nb, algo;
    Vec te, t1, rS, rN;
    BVec xs, rs, ps, aps, tes, tos;       // CG: p, S^+S p (aps), tmp, S p (tos); BiCGStab: p, v, tmp, t
    std::unique_ptr<BVec> svec, rhat, what;  // BiCGStab only: s, the shadow residual rhat, S^+ rhat
    // BiCGStab: each slot's rhat and S^+ rhat again as contiguous FP32 spinors (the same
    // rounded values), which a reliable update reads coalesced: in the pair layout one
    // right-hand side is 8 bytes of every 32-byte sector it touches
    std::unique_ptr<Vec> rhat_c[kMaxBatch], what_c[kMaxBatch];
    std::unique_ptr<DevBuf> om_scratch;      // BiCGStab: partial omega sums of the fused stencil epilogue
    static constexpr size_t kTableBytes = 3 * kMaxBatch * sizeof(double) + 16;
    char *tables = nullptr;
    double *d_b = nullptr;
    const void **d_T = nullptr, **d_Ti = nullptr;
    int *d_uniform = nullptr;
    const void *h_T[kMaxBatch] = {};
    int gauge_id = -1;
    bool has_clover = false;
    BatchTile tile;
    cudaGraphExec_t exec = nullptr;  // kGraphIters captured iterations, replayed
    size_t nodes = 0;
    static constexpr int kGraphIters = 8;
    // the loop pauses once a kParkFraction-th of the busy slots waits for its update
    static constexpr int kParkFraction = LYM_BLOCK_PARK_FRACTION;
    // BiCGStab gives a source up after kMaxStalls reliable updates in a row that did not
    // halve its best true residual, or after kMaxRestarts breakdowns
    static constexpr int kMaxStalls = 3, kMaxRestarts = 3;
    Slot slot[kMaxBatch];

    // the operator of slot j in the device tables: b = -kappa^2 and the FP32 T / Tinv bases,
    // and the flag telling the stencil whether all slots now share one operator
    void set_tables(int j, double b, const void *T, const void *Ti)
    {
        h_T[j] = T;
        int uni = 1;
        for (int k = 1; k < nb; ++k) uni &= h_T[k] == h_T[0];
        CK(cudaMemcpyAsync(d_b + j, &b, sizeof(double), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(d_T + j, &T, sizeof(void *), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(d_Ti + j, &Ti, sizeof(void *), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(d_uniform, &uni, sizeof(int), cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    BatchCGState hs;
    std::vector<int> done_list;

    bool any_active() const
    {
        for (int j = 0; j < nb; ++j)
            if (hs.active[j]) return true;
        return false;
    }
    // |b' - S x|^2 and |S^+ (b' - S x)|^2 of slot j (zero_x: x = 0, the residual is b')
    void true_res(int j, double &rrS, double &rrN, bool zero_x = false)
    {
        Slot &s = slot[j];
        const Spinor xo = s.X.parity(1);
        if (zero_x) {
            copy(c, *rS, **s.bp);
            run_site(c, OpNorm<SpinorD>{(*rS).d(), c->d_scal}, 1);
        } else {
            apply_schur(c, *s.op, PREC_D, *t1, xo, *te, 0);
            run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{(**s.bp).d(), (*t1).d(), (*rS).d(), c->d_scal}, 1);
        }
        copy(c, *t1, *rS);
        gamma5_inplace(c, *t1);
        apply_schur(c, *s.op, PREC_D, *rN, *t1, *te, 1);
        run_site(c, OpNorm<SpinorD>{(*rN).d(), c->d_scal + 1}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        rrS = c->h_scal[0];
        rrN = c->h_scal[1];
    }
    // |b' - S x|^2 of slot j, the residual left in rS (zero_x: x = 0, the residual is b')
    void true_res_S(int j, double &rrS, bool zero_x = false)
    {
        Slot &s = slot[j];
        if (zero_x) {
            copy(c, *rS, **s.bp);
            run_site(c, OpNorm<SpinorD>{(*rS).d(), c->d_scal}, 1);
        } else {
            apply_schur(c, *s.op, PREC_D, *t1, s.X.parity(1), *te, 0);
            run_site(c, OpSubNorm<SpinorD, SpinorD, SpinorD>{(**s.bp).d(), (*t1).d(), (*rS).d(), c->d_scal}, 1);
        }
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        rrS = c->h_scal[0];
    }
    // BiCGStab (re)start of slot j from the true residual in rS: r = rhat = p = rS
    // what = S^+ rhat = g5 S g5 rhat (S is gamma5-hermitian), in FP64 into rN and the slot;
    // returns <what, p> for p = rhat = rS
    double2 shadow_image(int j)
    {
        copy(c, *t1, *rS);
        gamma5_inplace(c, *t1);
        apply_schur(c, *slot[j].op, PREC_D, *rN, *t1, *te, 1);
        axpby_views(c, (*rN).d(), what->f().slot(j), C2(1.0), C2(0.0));
        copy(c, **what_c[j], *rN);
        run_site(c, OpDot<SpinorD, SpinorD>{(*rN).d(), (*rS).d(), c->d_scal}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        return make_double2(c->h_scal[0], c->h_scal[1]);
    }
    // <a, b> of two views of slot j
    template <class SA, class SB> double2 slot_dot(const SA &a, const SB &b)
    {
        run_site(c, OpDot<SA, SB>{a, b, c->d_scal}, 1);
        CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        return make_double2(c->h_scal[0], c->h_scal[1]);
    }
    // BiCGStab (re)start of slot j from the true residual in rS: r = rhat = p = rS,
    // rho = |rS|^2, what = S^+ rhat, alpha = rho / <what, p>
    void restart_bicg(int j, double rrS)
    {
        axpby_views(c, (*rS).d(), rs.f().slot(j), C2(1.0), C2(0.0));
        axpby_views(c, (*rS).d(), rhat->f().slot(j), C2(1.0), C2(0.0));
        copy(c, **rhat_c[j], *rS);
        set_direction(j, 0.0);
        hs.rho[j] = make_double2(rrS, 0.0);
        hs.alpha[j] = cdiv(hs.rho[j], shadow_image(j));
        hs.rr[j] = hs.rr_max[j] = rrS;
        hs.restart[j] = 0;
        hs.active[j] = 1;
    }
    void reliable_update_bicg(int j)
    {
        Slot &s = slot[j];
        // x += the FP32 accumulator (unless a non-finite recursion (restart 2) drops it); the
        // accumulator counts as zero from the next update pass on
        if (hs.restart[j] != 2 && !hs.x_reset[j])
            axpby_views(c, xs.f().slot(j), s.X.parity(1).d(), C2(1.0), C2(1.0));
        hs.x_reset[j] = 1;
        double rrS;
        true_res_S(j, rrS);
        ++s.updates;
        hs.last_update_its[j] = hs.its[j];
        if (rrS < 0.5 * s.best_rr) {
            s.best_rr = rrS;
            s.stalls = 0;
        } else {
            ++s.stalls;
        }
        if (hs.restart[j]) ++s.restarts;
        if (!std::isfinite(rrS)) {
            s.nonfinite = true;
            finish(j);
        } else if (rrS < s.epsS) {
            s.converged = 1;
            finish(j);
        } else if (s.stalls >= kMaxStalls || s.restarts >= kMaxRestarts) {
            s.gave_up = true;  // BiCGStab does not converge on this source
            finish(j);
        } else {
            if (hs.converged[j]) hs.eps[j] = std::max(hs.eps[j] * 0.5 * s.epsS / rrS, 1e-300);
            if (hs.restart[j]) {
                restart_bicg(j, rrS);
            } else {
                // the recursion goes on with the true residual in place of the recursive
                // one: p += r_true - r_rec (p was formed from r_rec), r = r_true,
                // rho = <rhat, r>, alpha = rho / <what, p>
                if (sprec == PREC_F)
                    run_site(c, OpBiContinue<SlotF, SlotF, SpinorD, SpinorF, SpinorF>{
                                    rs.f().slot(j), ps.f().slot(j), (*rS).d(), (**rhat_c[j]).f(), (**what_c[j]).f(),
                                    c->d_scal}, 1);
                else
                    run_site(c, OpBiContinue<SlotF, SlotH, SpinorD, SpinorF, SpinorF>{
                                    rs.f().slot(j), ps.h().slot(j), (*rS).d(), (**rhat_c[j]).f(), (**what_c[j]).f(),
                                    c->d_scal}, 1);
                CK(cudaMemcpyAsync(c->h_scal, c->d_scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
                CK(cudaStreamSynchronize(c->st));
                hs.rho[j] = make_double2(c->h_scal[0], c->h_scal[1]);
                const double2 wp = make_double2(c->h_scal[2], c->h_scal[3]);
                hs.alpha[j] = cdiv(hs.rho[j], wp);
                hs.rr[j] = hs.rr_max[j] = rrS;
                hs.active[j] = 1;
            }
        }
        hs.restart[j] = 0;
        hs.converged[j] = 0;
        hs.need_update[j] = 0;
    }
    void set_direction(int j, double b)  // p_j = r_j + b p_j in the precision of p
    {
        if (sprec == PREC_F) axpby_views(c, rs.f().slot(j), ps.f().slot(j), C2(1.0), C2(b));
        else axpby_views(c, rs.f().slot(j), ps.h().slot(j), C2(1.0), C2(b));
    }
    // the reliable updates of the parked slots; a slot past its iteration limit finishes
    void service()
    {
        const double t0 = wall();
        check_copy_waits(c, tile);
        for (int j = 0; j < nb; ++j) {
            Slot &s = slot[j];
            if (!s.busy || s.finished || !hs.need_update[j]) continue;
            reliable_update(j);
            c->engine_stats[6] += 1;
            if (!s.finished && hs.its[j] >= s.max_iter) finish(j);
        }
        c->engine_stats[1] += wall() - t0;
    }
    // captures kGraphIters iterations once, then replays them until the state pauses
    void run_loop(BatchCGState *S, long max_iterations)
    {
        if (!exec) {
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
            c->capturing = true;
            try {
                for (int k = 0; k < kGraphIters; ++k) step(S);
            } catch (...) {
                c->capturing = false;
                cudaStreamEndCapture(c->st, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            c->capturing = false;
            CK(cudaStreamEndCapture(c->st, &graph));
            const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphGetNodes(graph, nullptr, &nodes);
            cudaGraphDestroy(graph);
            CK(e);
        }
        const long max_launches = max_iterations / kGraphIters + 4;
        for (long l = 0; l < max_launches; ++l) {
            CK(cudaGraphLaunch(exec, c->st));
            c->launches += nodes;
            c->engine_stats[4] += 1;
            CK(cudaMemcpyAsync(c->h_state, S, sizeof(BatchCGState), cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            if (((BatchCGState *)c->h_state)->pause) return;
        }
        fail(c, LYM_ERR_TIMEOUT, "block CG state did not pause within %ld iterations", max_iterations);
    }
    void reliable_update(int j)
    {
        if (algo == ALGO_BICGSTAB) {
            reliable_update_bicg(j);
            return;
        }
        Slot &s = slot[j];
        // x += the FP32 accumulator (unless a non-finite recursion (restart 2) drops it); the
        // accumulator counts as zero from the next update pass on
        if (hs.restart[j] != 2 && !hs.x_reset[j])
            axpby_views(c, xs.f().slot(j), s.X.parity(1).d(), C2(1.0), C2(1.0));
        hs.x_reset[j] = 1;
        const bool restarted = hs.restart[j] != 0;
        hs.restart[j] = 0;
        double rrS, rrN;
        true_res(j, rrS, rrN);
        ++s.updates;
        if (!std::isfinite(rrS) || !std::isfinite(rrN)) {
            s.nonfinite = true;
            finish(j);
        } else if (rrS < s.epsS) {
            s.converged = 1;
            finish(j);
        } else if (restarted) {  // CG again from the true residual
            axpby_views(c, (*rN).d(), rs.f().slot(j), C2(1.0), C2(0.0));
            set_direction(j, 0.0);
            hs.rr[j] = hs.rr_max[j] = rrN;
            hs.active[j] = 1;
        } else {
            if (hs.converged[j]) hs.eps[j] = std::max(hs.eps[j] * 0.5 * s.epsS / rrS, 1e-300);
            const double b = rrN / hs.rr_prev[j];
            if (sprec == PREC_F)
                run_site(c, OpCGContinue<SlotF, SlotF, SpinorD>{rs.f().slot(j), ps.f().slot(j), (*rN).d(), b}, 1);
            else
                run_site(c, OpCGContinue<SlotF, SlotH, SpinorD>{rs.f().slot(j), ps.h().slot(j), (*rN).d(), b}, 1);
            hs.rr[j] = hs.rr_max[j] = rrN;
            hs.active[j] = 1;  // back into the iteration
        }
        hs.converged[j] = 0;
        hs.need_update[j] = 0;
    }
    void finish(int j)
    {
        Slot &s = slot[j];
        s.finished = true;
        if (s.gave_up || s.nonfinite) {  // nothing to reconstruct (solved again elsewhere, or not finite)
            s.iters = hs.its[j];
            hs.active[j] = 0;
            hs.need_update[j] = 0;
            done_list.push_back(j);
            return;
        }
        s.iters = hs.its[j];
        hs.active[j] = 0;
        hs.need_update[j] = 0;
        schur_reconstruct(c, *s.op, s.B, s.X);
        done_list.push_back(j);
    }
    template <class SP> void step_bicg(BatchCGState *S, const SP &p, const SP &v, const SP &sv, const SP &t)
    {
        const GaugeDev &U = gauge_of(c, gauge_id).dev;
        Gate gate{&S->pause, nullptr};
        const int lognb = xs.s.lognb;
        // alpha is known when the iteration starts (<rhat, S p> = <S^+ rhat, p>, reduced with p)
        // v = S p, and s = r - alpha v in the same launch's epilogue
        apply_schur_batch(c, U, has_clover, sprec, aps.s, ps.s, tes.s, 0, &S->pause, S->active, d_b, d_T, d_Ti, tile,
                          d_uniform, &rs.s, &svec->s, S->alpha);
        if (om_scratch) {  // t = S s with the omega sums in its epilogue
            apply_schur_batch(c, U, has_clover, sprec, tos.s, svec->s, tes.s, 0, &S->pause, S->active, d_b, d_T,
                              d_Ti, tile, d_uniform, nullptr, nullptr, nullptr, &rhat->s,
                              (double *)om_scratch->p, S);
        } else {
            apply_schur_batch(c, U, has_clover, sprec, tos.s, svec->s, tes.s, 0, &S->pause, S->active, d_b, d_T,
                              d_Ti, tile, d_uniform);
            run_batch(c, OpBBOmega<SP, SP, BatchF>{t, sv, rhat->f(), S}, lognb, gate);
        }
        run_batch(c, OpBBUpdate<BatchF, SP, SP, SP, SP, BatchF, BatchF>{xs.f(), p, sv, t, v, rs.f(), what->f(), S},
                  lognb, gate);
    }
    void step(BatchCGState *S)
    {
        if (algo == ALGO_BICGSTAB) {
            if (sprec == PREC_F) step_bicg(S, ps.f(), aps.f(), svec->f(), tos.f());
            else step_bicg(S, ps.h(), aps.h(), svec->h(), tos.h());
            return;
        }
        const GaugeDev &U = gauge_of(c, gauge_id).dev;
        Gate gate{&S->pause, nullptr};
        const int lognb = xs.s.lognb;
        apply_schur_batch(c, U, has_clover, sprec, tos.s, ps.s, tes.s, 1, &S->pause, S->active, d_b, d_T, d_Ti, tile, d_uniform);
        apply_schur_batch(c, U, has_clover, sprec, aps.s, tos.s, tes.s, 1, &S->pause, S->active, d_b, d_T, d_Ti, tile, d_uniform);
        if (sprec == PREC_F) {
            run_batch(c, OpBAlpha<BatchF, BatchF>{ps.f(), aps.f(), S}, lognb, gate);
            run_batch(c, OpBUpdate<BatchF, BatchF, BatchF, BatchF>{xs.f(), ps.f(), rs.f(), aps.f(), S}, lognb,
                      gate);
            run_batch(c, OpBDirection<BatchF, BatchF>{ps.f(), rs.f(), S}, lognb, gate);
        } else {
            run_batch(c, OpBAlpha<BatchH, BatchH>{ps.h(), aps.h(), S}, lognb, gate);
            run_batch(c, OpBUpdate<BatchF, BatchH, BatchF, BatchH>{xs.f(), ps.h(), rs.f(), aps.h(), S}, lognb,
                      gate);
            run_batch(c, OpBDirection<BatchH, BatchF>{ps.h(), rs.f(), S}, lognb, gate);
        }
    }
    void direction_rest(BatchCGState *S)  // the direction update the pause skipped, for slots without an update
    {
        if (algo == ALGO_BICGSTAB) return;  // the direction is updated in the same pass as x and r
        if (sprec == PREC_F) run_batch(c, OpBDirection<BatchF, BatchF>{ps.f(), rs.f(), S}, xs.s.lognb);
        else run_batch(c, OpBDirection<BatchH, BatchF>{ps.h(), rs.f(), S}, xs.s.lognb);
    }
};

// upload of source and guess, device timing and download around one FP64 solve
template <class F>
int solve_framed(lym_context *c, const double *source, double *solution, const double *guess,
                        lym_solve_stats *stats, F solve)
{
    lym_solve_stats local;
    memset(&local, 0, sizeof(local));
    Vec b(c, PREC_D, 2), x(c, PREC_D, 2);
    std::unique_ptr<Vec> gs;
    upload_vec(c, *b, source, false, 0);
    if (guess) {
        gs.reset(new Vec(c, PREC_D, 2));
        upload_vec(c, **gs, guess, false, 1);
    }
    CK(cudaEventRecord(c->ev0, c->st));
    const int rc = solve(*b, *x, gs ? &**gs : nullptr, &local);
    CK(cudaEventRecord(c->ev1, c->st));
    download_vec(c, solution, *x, false, 2);
    CK(cudaStreamSynchronize(c->st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    local.seconds = ms * 1e-3;
    if (stats) *stats = local;
    CK(cudaGetLastError());
    return rc;
}

}  // namespace

// =============================================================== C ABI =====
extern "C" {

int lym_context_create(const int dims[4], int rep, int device, lym_context **out)
{
    if (!dims || !out) return LYM_ERR_ARGUMENT;
    *out = nullptr;
    for (int mu = 0; mu < 4; ++mu)
        if (dims[mu] < 2) return LYM_ERR_ARGUMENT;
    if (dims[3] % 2) return LYM_ERR_UNSUPPORTED;  // the even-odd half-site index needs an even L_t
    if (rep != LYM_REP_SU3_FUNDAMENTAL && rep != LYM_REP_SU2_ADJOINT) return LYM_ERR_ARGUMENT;
    const long long V = (long long)dims[0] * dims[1] * dims[2] * dims[3];
    if (V > (1ll << 30)) return LYM_ERR_UNSUPPORTED;
    lym_context *c = new lym_context();
    c->device = device;
    c->rep = rep;
    for (int mu = 0; mu < 4; ++mu) c->g.L[mu] = dims[mu];
    c->g.V = (int)V;
    c->g.Vh = (int)(V / 2);
    c->g.stride = (c->g.Vh + 63) / 64 * 64;
    int rc = guarded(c, [&]() {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
        c->partials = (double *)dev_alloc(c, (size_t)kBlasGridMax * kMaxRed * sizeof(double));
        c->bpartials = (double *)dev_alloc(c, (size_t)kBlasGridMax * kMaxBatch * kBatchMaxRed * sizeof(double));
        c->spartials = (double *)dev_alloc(c, ((size_t)c->g.Vh + 127) / 128 * sizeof(double));
        c->nbr = (int *)dev_alloc(c, (size_t)16 * c->g.stride * sizeof(int));
        launch_nbr_table(c->g, c->nbr, c->st);
        c->counter = (unsigned int *)dev_alloc(c, 64);
        c->d_err = (int *)dev_alloc(c, 64);
        CK(cudaMemsetAsync(c->d_err, 0, 64, c->st));
        c->d_state = dev_alloc(c, kStateBytes);
        c->d_scal = (double *)dev_alloc(c, 64 * sizeof(double));
        CK(cudaHostAlloc(&c->h_state, kStateBytes, cudaHostAllocDefault));
        CK(cudaHostAlloc((void **)&c->h_scal, 64 * sizeof(double), cudaHostAllocDefault));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        CK(cudaStreamSynchronize(c->st));
        return LYM_OK;
    });
    if (rc != LYM_OK) {
        lym_context_destroy(c);
        return rc;
    }
    *out = c;
    return LYM_OK;
}

void lym_context_destroy(lym_context *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->st_copy) cudaStreamSynchronize(c->st_copy);
    for (auto &kv : c->ops)
        for (int p = 0; p < 3; ++p) {
            cudaFree(kv.second.clover.T[p]);
            cudaFree(kv.second.clover.Tinv[p]);
        }
    for (auto &kv : c->gauges) {
        cudaFree(kv.second.dev.d64);
        cudaFree(kv.second.dev.f32);
        cudaFree(kv.second.dev.h16);
        cudaFree(kv.second.dev.sign);
        cudaFree(kv.second.dev.f32r8);
        cudaFree(kv.second.dev.f32r18);
    }
    for (auto &s : c->pool) cudaFree(s.v);
    for (auto &b : c->blocks) cudaFree(b.second);
    for (int k = 0; k < 3; ++k) cudaFree(c->aos[k]);
    cudaFree(c->partials);
    cudaFree(c->spartials);
    cudaFree(c->bpartials);
    cudaFree(c->nbr);
    for (auto &kv : c->orders) cudaFree(kv.second);
    cudaFree(c->counter);
    cudaFree(c->d_err);
    cudaFree(c->d_state);
    cudaFree(c->d_scal);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_scal) cudaFreeHost(c->h_scal);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->st) cudaStreamDestroy(c->st);
    if (c->st_copy) cudaStreamDestroy(c->st_copy);
    delete c;
}

const char *lym_last_error(lym_context *c) { return c ? c->err.c_str() : "no context"; }

int lym_context_volume(lym_context *c) { return c ? c->g.V : 0; }

size_t lym_context_device_bytes(lym_context *c) { return c ? c->bytes : 0; }

int lym_context_trim(lym_context *c)
{
    return guarded(c, [&]() {
        trim_pool(c);
        return LYM_OK;
    });
}

int lym_synchronize(lym_context *c)
{
    return guarded(c, [&]() {
        CK(cudaStreamSynchronize(c->st));
        return LYM_OK;
    });
}

static int gauge_store(lym_context *c, int id, const double *links, bool device_ptr)
{
    const Geom &g = c->g;
    GaugeEntry *ge;
    auto it = c->gauges.find(id);
    if (it == c->gauges.end()) {
        GaugeEntry e;
        e.dev.rep = c->rep;
        const size_t s = g.stride;
        const size_t d64 = c->rep == REP_SU3 ? 2 * 4 * 9 * s * sizeof(double2) : 2 * 4 * 9 * s * sizeof(double);
        const size_t f32 = c->rep == REP_SU3 ? 2 * 4 * 3 * s * sizeof(float4) : 2 * 4 * 3 * s * sizeof(float2);
        const size_t h16 = c->rep == REP_SU3 ? 2 * 4 * 3 * s * sizeof(uint2) : 2 * 4 * 3 * s * sizeof(__half2);
        e.dev.d64 = dev_alloc(c, d64);
        e.dev.f32 = dev_alloc(c, f32);
        e.dev.h16 = dev_alloc(c, h16);
        e.dev.sign = (uint8_t *)dev_alloc(c, 2 * s);
        e.dev.f32r8 = dev_alloc(c, 2 * 4 * 2 * s * sizeof(float4));  // written for SU(3) only
        if (c->rep == REP_SU3) e.dev.f32r18 = dev_alloc(c, 2 * 4 * 5 * s * sizeof(float4));
        e.dev.link_reals = c->link_reals;
        ge = &(c->gauges[id] = e);
    } else {
        ge = &it->second;
    }
    const size_t per = c->rep == REP_SU3 ? 18 : 9;
    const size_t bytes = (size_t)g.V * 4 * per * sizeof(double);
    if (!device_ptr) {
        double *buf = (double *)dev_alloc(c, bytes);
        CK(cudaMemcpyAsync(buf, links, bytes, cudaMemcpyHostToDevice, c->st));
        launch_upload_gauge(g, c->rep, buf, ge->dev, c->st);
        CK(cudaStreamSynchronize(c->st));
        dev_free(c, buf, bytes);
    } else {
        launch_upload_gauge(g, c->rep, links, ge->dev, c->st);
    }
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
    launch_compress_gauge(g, ge->dev, c->d_err, c->st);
    CK(cudaMemcpyAsync(c->h_scal, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    memcpy(&ge->recon_err, c->h_scal, sizeof(int));
    ge->dev.recon_ok = ge->recon_err == 0;
    // operators on this gauge field need a new clover term
    for (auto &kv : c->ops)
        if (kv.second.gauge_id == id) kv.second.clover_ok = false;
    return LYM_OK;
}

int lym_gauge_upload(lym_context *c, int id, const double *links)
{
    if (!links) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() { return gauge_store(c, id, links, false); });
}

int lym_gauge_upload_device(lym_context *c, int id, const double *links)
{
    if (!links) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() { return gauge_store(c, id, links, true); });
}

int lym_gauge_upload_fundamental(lym_context *c, int id, const double *gauge_links, int boundary)
{
    if (!gauge_links || (boundary != LYM_BC_PERIODIC && boundary != LYM_BC_ANTIPERIODIC)) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const Geom &g = c->g;
        const size_t in_per = c->rep == REP_SU3 ? 18 : 8, out_per = c->rep == REP_SU3 ? 18 : 9;
        const size_t bin = (size_t)g.V * 4 * in_per * sizeof(double), bout = (size_t)g.V * 4 * out_per * sizeof(double);
        double *din = (double *)dev_alloc(c, bin), *dout = (double *)dev_alloc(c, bout);
        CK(cudaMemcpyAsync(din, gauge_links, bin, cudaMemcpyHostToDevice, c->st));
        launch_fundamental_to_fermion(g, c->rep, boundary, din, dout, c->st);
        int rc = gauge_store(c, id, dout, true);
        CK(cudaStreamSynchronize(c->st));
        dev_free(c, din, bin);
        dev_free(c, dout, bout);
        return rc;
    });
}

int lym_gauge_evict(lym_context *c, int id)
{
    return guarded(c, [&]() {
        auto it = c->gauges.find(id);
        if (it == c->gauges.end()) fail(c, LYM_ERR_NOT_FOUND, "gauge field %d is not resident", id);
        for (auto &kv : c->ops)
            if (kv.second.gauge_id == id) fail(c, LYM_ERR_ARGUMENT, "gauge field %d is used by operator %d", id, kv.first);
        CK(cudaStreamSynchronize(c->st));
        const size_t s = c->g.stride;
        const bool su3 = c->rep == REP_SU3;
        dev_free(c, it->second.dev.d64, su3 ? 2 * 4 * 9 * s * sizeof(double2) : 2 * 4 * 9 * s * sizeof(double));
        dev_free(c, it->second.dev.f32, su3 ? 2 * 4 * 3 * s * sizeof(float4) : 2 * 4 * 3 * s * sizeof(float2));
        dev_free(c, it->second.dev.h16, su3 ? 2 * 4 * 3 * s * sizeof(uint2) : 2 * 4 * 3 * s * sizeof(__half2));
        dev_free(c, it->second.dev.sign, 2 * s);
        dev_free(c, it->second.dev.f32r8, 2 * 4 * 2 * s * sizeof(float4));
        if (su3) dev_free(c, it->second.dev.f32r18, 2 * 4 * 5 * s * sizeof(float4));
        c->gauges.erase(it);
        return LYM_OK;
    });
}

int lym_operator_create(lym_context *c, int gauge_id, int kind, double kappa, double csw, int gamma5, int *op_id)
{
    if (!op_id || kind < 0 || kind > 5) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        gauge_of(c, gauge_id);
        if (is_even_odd(kind) && c->rep != REP_SU3 && c->rep != REP_SU2ADJ)
            fail(c, LYM_ERR_UNSUPPORTED, "even-odd operator needs diracVectorLength 3");
        OpEntry e;
        e.gauge_id = gauge_id;
        e.kind = kind;
        e.kappa = kappa;
        e.csw = kind_has_clover(kind) ? csw : 0.0;
        e.gamma5 = gamma5 ? 1 : 0;
        const int id = c->next_op++;
        c->ops[id] = e;
        *op_id = id;
        return LYM_OK;
    });
}

int lym_operator_set_gamma5(lym_context *c, int op_id, int gamma5)
{
    return guarded(c, [&]() {
        op_of(c, op_id).gamma5 = gamma5 ? 1 : 0;
        return LYM_OK;
    });
}

int lym_operator_set_kappa(lym_context *c, int op_id, double kappa)
{
    return guarded(c, [&]() {
        OpEntry &o = op_of(c, op_id);
        if (o.kappa != kappa) o.clover_ok = false;
        o.kappa = kappa;
        return LYM_OK;
    });
}

int lym_operator_set_csw(lym_context *c, int op_id, double csw)
{
    return guarded(c, [&]() {
        OpEntry &o = op_of(c, op_id);
        if (o.csw != csw) o.clover_ok = false;
        o.csw = kind_has_clover(o.kind) ? csw : 0.0;
        return LYM_OK;
    });
}

int lym_operator_set_gauge(lym_context *c, int op_id, int gauge_id)
{
    return guarded(c, [&]() {
        gauge_of(c, gauge_id);
        OpEntry &o = op_of(c, op_id);
        o.gauge_id = gauge_id;
        o.clover_ok = false;
        return LYM_OK;
    });
}

int lym_operator_destroy(lym_context *c, int op_id)
{
    return guarded(c, [&]() {
        OpEntry &o = op_of(c, op_id);
        CK(cudaStreamSynchronize(c->st));
        free_clover(c, o);
        c->ops.erase(op_id);
        return LYM_OK;
    });
}

static int do_multiply(lym_context *c, int op_id, int prec, double *out, const double *v1, const double *v2,
                       double2 alpha, bool device_ptr)
{
    if (!out || !v1) return LYM_ERR_ARGUMENT;
    if (prec < PREC_D || prec > PREC_H) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        Vec a(c, prec, 2), o(c, prec, 2);
        Vec *w = nullptr;
        upload_vec(c, *a, v1, device_ptr, 0);
        if (v2) {
            w = new Vec(c, prec, 2);
            upload_vec(c, **w, v2, device_ptr, 1);
        }
        try {
            op_apply(c, op, prec, *o, *a, w ? &**w : nullptr, alpha);
        } catch (...) {
            delete w;
            throw;
        }
        delete w;
        download_vec(c, out, *o, device_ptr, 2);
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        return LYM_OK;
    });
}

int lym_multiply(lym_context *c, int op_id, double *out, const double *in)
{
    return do_multiply(c, op_id, PREC_D, out, in, nullptr, C2(0.0), false);
}

int lym_multiply_add(lym_context *c, int op_id, double *out, const double *v1, const double *v2, double are, double aim)
{
    if (!v2) return LYM_ERR_ARGUMENT;
    return do_multiply(c, op_id, PREC_D, out, v1, v2, C2(are, aim), false);
}

int lym_multiply_device(lym_context *c, int op_id, double *out, const double *in)
{
    return do_multiply(c, op_id, PREC_D, out, in, nullptr, C2(0.0), true);
}

int lym_multiply_add_device(lym_context *c, int op_id, double *out, const double *v1, const double *v2, double are,
                            double aim)
{
    if (!v2) return LYM_ERR_ARGUMENT;
    return do_multiply(c, op_id, PREC_D, out, v1, v2, C2(are, aim), true);
}

int lym_multiply_precision(lym_context *c, int op_id, int prec, double *out, const double *in)
{
    return do_multiply(c, op_id, prec, out, in, nullptr, C2(0.0), false);
}

int lym_field_strength(lym_context *c, int op_id, double *F)
{
    if (!F) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        const size_t b = (size_t)c->g.V * 6 * 9 * 2 * sizeof(double);
        double *d = (double *)dev_alloc(c, b);
        OpEntry tmp = op;
        tmp.clover = CloverDev();
        tmp.clover_ok = false;
        try {
            ensure_clover(c, tmp, d);
        } catch (...) {
            free_clover(c, tmp);
            dev_free(c, d, b);
            throw;
        }
        CK(cudaMemcpyAsync(F, d, b, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        free_clover(c, tmp);
        dev_free(c, d, b);
        if (c->rep == REP_SU2ADJ) {
            // adjoint F is real: compact to the reference's real 3x3 layout
            const size_t n = (size_t)c->g.V * 6 * 9;
            for (size_t k = 0; k < n; ++k) F[k] = F[2 * k];
        }
        return LYM_OK;
    });
}

static int do_solve(lym_context *c, int op_id, int solver, double precision, int max_steps, const double *source,
                    double *solution, const double *guess, lym_solve_stats *stats, bool device_ptr, bool shifted,
                    double2 shift)
{
    if (!source || !solution || max_steps < 0) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        lym_solve_stats local;
        memset(&local, 0, sizeof(local));
        Vec b(c, PREC_D, 2), x(c, PREC_D, 2);
        Vec *gs = nullptr;
        upload_vec(c, *b, source, device_ptr, 0);
        if (guess) {
            gs = new Vec(c, PREC_D, 2);
            upload_vec(c, **gs, guess, device_ptr, 1);
        }
        const Spinor *gp = gs ? &**gs : nullptr;
        CK(cudaEventRecord(c->ev0, c->st));
        int rc = LYM_OK;
        // a source or guess with a non-finite entry: not converged at once (the reference
        // iterates on its non-finite residuals until max_steps and returns false)
        const double bb = norm2_now(c, *b), gg = gp ? norm2_now(c, *gp) : 0.0;
        const bool finite_inputs = std::isfinite(bb) && std::isfinite(gg);
        try {
            if (!finite_inputs) {
                zero(c, *x);
                local.last_error = local.true_residual = std::numeric_limits<double>::quiet_NaN();
                c->err = "the source or the initial guess has non-finite entries";
                rc = LYM_NOT_CONVERGED;
            } else if (shifted) {
                auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
                    op_apply(c, op, PREC_D, out, in, &in, shift, skip);
                };
                rc = bicgstab_solve(c, mv, 2, *b, *x, gp, precision, max_steps, 0.0, &local);
            } else {
                switch (solver) {
                case LYM_SOLVER_CG: {
                    auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
                        op_apply(c, op, PREC_D, out, in, nullptr, C2(0.0), skip);
                    };
                    rc = cg_solve(c, mv, 2, *b, *x, gp, precision, max_steps, &local);
                    break;
                }
                case LYM_SOLVER_BICGSTAB: {
                    auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
                        op_apply(c, op, PREC_D, out, in, nullptr, C2(0.0), skip);
                    };
                    rc = bicgstab_solve(c, mv, 2, *b, *x, gp, precision, max_steps, 0.0, &local);
                    break;
                }
                case LYM_SOLVER_EO_BICGSTAB: rc = eo_bicgstab(c, op, *b, *x, gp, precision, max_steps, &local); break;
                case LYM_SOLVER_EO_CG:
                case LYM_SOLVER_EO_CG_MIXED_SINGLE:
                case LYM_SOLVER_EO_CG_MIXED_HALF: {
                    if (op.kind != LYM_OP_IMPROVED && op.kind != LYM_OP_DIRAC_WILSON)
                        fail(c, LYM_ERR_UNSUPPORTED, "even-odd CG solves D x = b for a DiracWilson/Improved operator");
                    const int sp = solver == LYM_SOLVER_EO_CG ? PREC_D
                                   : solver == LYM_SOLVER_EO_CG_MIXED_SINGLE ? PREC_F : PREC_H;
                    const double tol = precision <= 0.0 ? (precision == 0.0 ? 1e-10 : -precision)
                                                        : std::sqrt(precision);
                    rc = eo_cg(c, op, sp, *b, *x, gp, tol, max_steps, &local);
                    local.true_residual = true_residual(c, op, *b, *x);
                    break;
                }
                case LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE:
                case LYM_SOLVER_EO_BICGSTAB_MIXED_HALF: {
                    if (op.kind != LYM_OP_IMPROVED && op.kind != LYM_OP_DIRAC_WILSON)
                        fail(c, LYM_ERR_UNSUPPORTED, "even-odd BiCGStab solves D x = b for a DiracWilson/Improved operator");
                    if (gp) fail(c, LYM_ERR_UNSUPPORTED, "the mixed-precision BiCGStab starts from x = 0 (no guess)");
                    const int sp = solver == LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE ? PREC_F : PREC_H;
                    const double tol = precision <= 0.0 ? (precision == 0.0 ? 1e-10 : -precision)
                                                        : std::sqrt(precision);
                    // the block engine with one busy slot (the batched stencil's smallest width)
                    bool gave_up = false;
                    {
                        BlockEngine engine(c, sp, 2, ALGO_BICGSTAB);
                        engine.add(0, op, *b, *x, tol, max_steps, 0);
                        while (engine.working()) engine.advance();
                        engine.advance();
                        const auto &s = engine.info(0);
                        local.iterations = local.steps = s.iters;
                        local.reliable_updates = s.updates;
                        local.converged = s.converged;
                        gave_up = s.gave_up;
                        rc = s.converged ? LYM_OK : LYM_NOT_CONVERGED;
                    }
                    if (gave_up) {  // BiCGStab breaks down on this source: CG on (gamma5 S)^2
                        const int its = local.iterations, ups = local.reliable_updates;
                        rc = eo_cg(c, op, sp, *b, *x, nullptr, tol, max_steps, &local);
                        local.iterations += its;
                        local.steps = local.iterations;
                        local.reliable_updates += ups;
                    }
                    local.true_residual = true_residual(c, op, *b, *x);
                    break;
                }
                default: fail(c, LYM_ERR_ARGUMENT, "unknown solver %d", solver);
                }
            }
        } catch (...) {
            delete gs;
            throw;
        }
        delete gs;
        CK(cudaEventRecord(c->ev1, c->st));
        download_vec(c, solution, *x, device_ptr, 2);
        CK(cudaStreamSynchronize(c->st));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        local.seconds = ms * 1e-3;
        if (stats) *stats = local;
        CK(cudaGetLastError());
        return rc;
    });
}

int lym_solve(lym_context *c, int op_id, int solver, double precision, int max_steps, const double *source,
              double *solution, const double *guess, lym_solve_stats *stats)
{
    return do_solve(c, op_id, solver, precision, max_steps, source, solution, guess, stats, false, false, C2(0.0));
}

int lym_solve_device(lym_context *c, int op_id, int solver, double precision, int max_steps, const double *source,
                     double *solution, const double *guess, lym_solve_stats *stats)
{
    return do_solve(c, op_id, solver, precision, max_steps, source, solution, guess, stats, true, false, C2(0.0));
}

// Solves the sources listed in `tags` with one block engine, refilling its slots as they
// finish (continuous batching).  Sources on which BiCGStab gave up (breakdown or no
// progress) are returned in gave_up, without statistics.
static int run_block(lym_context *c, OpEntry &op, int sp, int algo, double tol, int max_steps,
                     const std::vector<int> &tags, const double *const *sources, double *const *solutions, int width,
                     lym_solve_stats *stats, bool device_ptr, std::vector<int> &gave_up)
{
    BlockEngine engine(c, sp, width, algo);
    std::vector<Vec *> bufs;  // two full FP64 spinors per slot
    int rc_all = LYM_OK;
    auto now = []() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    std::vector<double> t_start(tags.size(), 0.0);
    // host buffers: the sources' H2D copies run ahead on the copy stream through a ring of
    // K device staging buffers, and every solution's D2H copy runs there while the solves go
    // on, through a ring of KD: as many as the engine has slots, so that collecting a whole
    // wave of finished slots never waits on an earlier download (the host thread would hold
    // back the engine's next launches meanwhile)
    const size_t vb = (size_t)c->g.V * 24 * sizeof(double);
    const int K = device_ptr ? 0 : (int)std::min<size_t>(4, tags.size());
    const int KD = device_ptr ? 0 : (int)std::min<size_t>((size_t)width, tags.size());
    std::vector<std::unique_ptr<DevBuf>> up, down;
    struct Events {
        std::vector<cudaEvent_t> e;
        ~Events()
        {
            for (auto x : e) cudaEventDestroy(x);
        }
        cudaEvent_t make()
        {
            cudaEvent_t x;
            cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
            e.push_back(x);
            return x;
        }
    } events;
    std::vector<cudaEvent_t> ev_up(K), ev_used(K), ev_unpacked(KD), ev_down(KD);
    for (int r = 0; r < K; ++r) {
        up.emplace_back(new DevBuf(c, vb));
        ev_up[r] = events.make();
        ev_used[r] = events.make();
    }
    for (int r = 0; r < KD; ++r) {
        down.emplace_back(new DevBuf(c, vb));
        ev_unpacked[r] = events.make();
        ev_down[r] = events.make();
    }
    auto issue_up = [&](size_t k) {
        const int r = (int)(k % K);
        if (k >= (size_t)K) CK(cudaStreamWaitEvent(c->st_copy, ev_used[r], 0));
        CK(cudaMemcpyAsync(up[r]->p, sources[tags[k]], vb, cudaMemcpyHostToDevice, c->st_copy));
        CK(cudaEventRecord(ev_up[r], c->st_copy));
    };
    size_t ndown = 0;
    struct CopyDrain {
        lym_context *c;
        ~CopyDrain() { cudaStreamSynchronize(c->st_copy); }
    } drain{c};
    if (K > 0) {
        // the staging buffers are zeroed on the context's stream when they are handed out:
        // the copy stream starts its first uploads only after that (and after the engine's
        // own set-up), so that no zeroing lands on a source that has already arrived
        cudaEvent_t ready = events.make();
        CK(cudaEventRecord(ready, c->st));
        CK(cudaStreamWaitEvent(c->st_copy, ready, 0));
    }
    for (int k = 0; k < K; ++k) issue_up(k);
    auto collect = [&](int f) {
        const double t_collect = now();
        const auto &s = engine.info(f);
        const int tag = tags[s.tag];
        if (s.gave_up) {
            gave_up.push_back(tag);
        } else {
            if (device_ptr) {
                download_vec(c, solutions[tag], s.X, true, 2);
            } else {
                const int r = (int)(ndown % KD);
                if (ndown >= (size_t)KD) CK(cudaEventSynchronize(ev_down[r]));  // the buffer's last copy is done
                launch_unpack(c->g, s.X, (double *)down[r]->p, c->st);
                CK(cudaEventRecord(ev_unpacked[r], c->st));
                CK(cudaStreamWaitEvent(c->st_copy, ev_unpacked[r], 0));
                CK(cudaMemcpyAsync(solutions[tag], down[r]->p, vb, cudaMemcpyDeviceToHost, c->st_copy));
                CK(cudaEventRecord(ev_down[r], c->st_copy));
                ++ndown;
            }
            if (stats) {
                stats[tag].iterations = stats[tag].steps = s.iters;
                stats[tag].reliable_updates = s.updates;
                stats[tag].converged = s.converged;
                stats[tag].true_residual = true_residual(c, *s.op, s.B, s.X);
                stats[tag].seconds = now() - t_start[s.tag];
            }
            if (!s.converged) rc_all = LYM_NOT_CONVERGED;
        }
        engine.release(f);
        c->engine_stats[3] += now() - t_collect;
    };
    try {
        for (int j = 0; j < 2 * width; ++j) bufs.push_back(new Vec(c, PREC_D, 2));
        size_t next = 0;
        for (;;) {
            int j;
            while (next < tags.size() && (j = engine.free_slot()) >= 0) {
                const Spinor B = **bufs[2 * j], X = **bufs[2 * j + 1];
                if (device_ptr) {
                    upload_vec(c, B, sources[tags[next]], true, 0);
                } else {
                    const int r = (int)(next % K);
                    CK(cudaStreamWaitEvent(c->st, ev_up[r], 0));
                    launch_pack(c->g, (const double *)up[r]->p, B, c->st);
                    CK(cudaEventRecord(ev_used[r], c->st));
                    if (next + K < tags.size()) issue_up(next + K);
                }
                t_start[next] = now();
                const double t0 = now();
                engine.add(j, op, B, X, tol, max_steps, (long long)next);
                c->engine_stats[2] += now() - t0;
                ++next;
            }
            for (int f : engine.advance()) collect(f);
            if (!engine.working() && next >= tags.size()) {
                for (int f : engine.advance()) collect(f);
                if (!engine.working()) break;
            }
        }
    } catch (...) {
        cudaStreamSynchronize(c->st_copy);
        for (auto v : bufs) delete v;
        throw;
    }
    CK(cudaStreamSynchronize(c->st_copy));
    for (auto v : bufs) delete v;
    return rc_all;
}

static int do_solve_block(lym_context *c, int op_id, int solver, double precision, int max_steps, int nrhs,
                          const double *const *sources, double *const *solutions, int batch, lym_solve_stats *stats,
                          bool device_ptr)
{
    if (!sources || !solutions || nrhs < 1 || max_steps < 0) return LYM_ERR_ARGUMENT;
    if (batch == 0) batch = 16;
    if (batch < 1 || batch > kMaxBatch || (batch & (batch - 1))) return LYM_ERR_ARGUMENT;
    for (int j = 0; j < nrhs; ++j)
        if (!sources[j] || !solutions[j]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        if (op.kind != LYM_OP_IMPROVED && op.kind != LYM_OP_DIRAC_WILSON)
            fail(c, LYM_ERR_UNSUPPORTED, "block solves solve D x = b for a DiracWilson/Improved operator");
        if (solver != LYM_SOLVER_EO_CG_MIXED_SINGLE && solver != LYM_SOLVER_EO_CG_MIXED_HALF &&
            solver != LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE && solver != LYM_SOLVER_EO_BICGSTAB_MIXED_HALF)
            fail(c, LYM_ERR_UNSUPPORTED, "block solves use the mixed-precision even-odd CG or BiCGStab solvers");
        const int sp = (solver == LYM_SOLVER_EO_CG_MIXED_SINGLE || solver == LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE)
                           ? PREC_F
                           : PREC_H;
        const int algo = (solver == LYM_SOLVER_EO_BICGSTAB_MIXED_SINGLE || solver == LYM_SOLVER_EO_BICGSTAB_MIXED_HALF)
                             ? ALGO_BICGSTAB
                             : ALGO_CG;
        const double tol = precision <= 0.0 ? (precision == 0.0 ? 1e-10 : -precision) : std::sqrt(precision);
        const int width = std::max(2, std::min(batch, 1 << (int)std::ceil(std::log2((double)nrhs))));
        std::vector<int> tags(nrhs), gave_up;
        for (int j = 0; j < nrhs; ++j) tags[j] = j;
        int rc = run_block(c, op, sp, algo, tol, max_steps, tags, sources, solutions, width, stats, device_ptr, gave_up);
        if (!gave_up.empty()) {
            // BiCGStab broke down or stopped making progress on these sources (an indefinite
            // Schur operator): they are solved again with CG on (gamma5 S)^2
            std::vector<int> again;
            const int w2 = std::max(2, std::min(width, 1 << (int)std::ceil(std::log2((double)gave_up.size()))));
            const int rc2 = run_block(c, op, sp, ALGO_CG, tol, max_steps, gave_up, sources, solutions, w2, stats,
                                      device_ptr, again);
            if (rc2 != LYM_OK) rc = rc2;
        }
        CK(cudaGetLastError());
        return rc;
    });
}

int lym_solve_block(lym_context *c, int op_id, int solver, double precision, int max_steps, int nrhs,
                    const double *const *sources, double *const *solutions, int batch, lym_solve_stats *stats)
{
    return do_solve_block(c, op_id, solver, precision, max_steps, nrhs, sources, solutions, batch, stats, false);
}

int lym_solve_block_device(lym_context *c, int op_id, int solver, double precision, int max_steps, int nrhs,
                           const double *const *sources, double *const *solutions, int batch, lym_solve_stats *stats)
{
    return do_solve_block(c, op_id, solver, precision, max_steps, nrhs, sources, solutions, batch, stats, true);
}

int lym_solve_shifted(lym_context *c, int op_id, double sre, double sim, double precision, int max_steps,
                      const double *source, double *solution, const double *guess, lym_solve_stats *stats)
{
    return do_solve(c, op_id, LYM_SOLVER_BICGSTAB, precision, max_steps, source, solution, guess, stats, false, true,
                    C2(sre, sim));
}

int lym_solve_bicgstab_l(lym_context *c, int op_id, int l, double precision, int max_steps, const double *source,
                         double *solution, const double *guess, lym_solve_stats *stats)
{
    if (!source || !solution || max_steps < 0 || l < 1 || l > 16) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        return solve_framed(c, source, solution, guess, stats,
                            [&](const Spinor &b, const Spinor &x, const Spinor *g, lym_solve_stats *st) {
                                return bicgstab_l_solve(c, op, l, b, x, g, precision, max_steps, st);
                            });
    });
}

int lym_solve_preconditioned(lym_context *c, int op_id, int preconditioner_op_id, double precision, int max_steps,
                             const double *source, double *solution, const double *guess, lym_solve_stats *stats)
{
    if (!source || !solution || max_steps < 0) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        OpEntry &pre = op_of(c, preconditioner_op_id);
        if (pre.gauge_id != op.gauge_id)
            fail(c, LYM_ERR_ARGUMENT, "the preconditioner must act on the operator's gauge field");
        return solve_framed(c, source, solution, guess, stats,
                            [&](const Spinor &b, const Spinor &x, const Spinor *g, lym_solve_stats *st) {
                                return bicgstab_precond_solve(c, op, pre, b, x, g, precision, max_steps, st);
                            });
    });
}

// The multishift solvers on device spinors: xv[i] receives (A + shifts[i])^{-1} b.  For the
// chronological solver xv[i] (i >= 1) holds the guess of shift i on entry.
static int run_multishift(lym_context *c, OpEntry &op, int algorithm, int nshift, const double *shifts,
                          double precision, int max_steps, const Spinor &b, std::vector<Spinor> &xv,
                          lym_solve_stats &local)
{
    int rc = LYM_OK;
    if (algorithm == LYM_MULTISHIFT_CG) {
        rc = multishift_cg(c, op, nshift, shifts, precision, max_steps, b, xv, &local);
    } else if (algorithm == LYM_MULTISHIFT_ME) {
        // MEMultishiftSolver::solve: CG per shift, warm-started from the previous shift
        int total = 0;
        bool ok = true;
        for (int i = 0; i < nshift; ++i) {
            const double sh = shifts[i];
            auto mv = [&](const Spinor &out, const Spinor &in, const int *skip) {
                op_apply(c, op, PREC_D, out, in, &in, C2(sh), skip);
            };
            lym_solve_stats s1;
            memset(&s1, 0, sizeof(s1));
            if (i == 0) {
                Vec z(c, PREC_D, 2);
                zero(c, *z);
                rc = cg_solve(c, mv, 2, b, xv[0], &*z, precision, max_steps, &s1);
            } else {
                rc = cg_solve(c, mv, 2, b, xv[i], &xv[i - 1], precision, max_steps, &s1);
            }
            ok = ok && rc == LYM_OK;
            total += s1.iterations;
        }
        local.iterations = total;
        local.steps = total;
        local.converged = ok;
        rc = ok ? LYM_OK : LYM_NOT_CONVERGED;
    } else if (algorithm == LYM_MULTISHIFT_MMMR) {
        rc = multishift_mmmr(c, op, nshift, shifts, precision, max_steps, b, xv, &local);
    } else if (algorithm == LYM_MULTISHIFT_CG_MIXED_SINGLE || algorithm == LYM_MULTISHIFT_CG_MIXED_HALF) {
        // the shared Krylov space runs in FP32 for both: the precision of its operator
        // bounds the accuracy of every shifted solution (FP16 leaves them near 1e-3, FP32
        // near 1e-7), and the refinement from there is what the storage choice saves on
        const int rp = algorithm == LYM_MULTISHIFT_CG_MIXED_SINGLE ? PREC_F : PREC_H;
        rc = multishift_cg_mixed(c, op, rp, nshift, shifts, precision, max_steps, b, xv, &local);
    } else if (algorithm == LYM_MULTISHIFT_CHRONOLOGICAL) {
        rc = multishift_chrono(c, op, nshift, shifts, precision, max_steps, b, xv, &local);
    } else {
        fail(c, LYM_ERR_UNSUPPORTED, "multishift algorithm %d", algorithm);
    }
    return rc;
}

// Device spinors owned for the length of one call.
struct VecSet {
    std::vector<Vec *> v;
    std::vector<Spinor> s;
    VecSet(lym_context *c, int n, int prec, int nparity)
    {
        for (int i = 0; i < n; ++i) {
            v.push_back(new Vec(c, prec, nparity));
            s.push_back(**v.back());
        }
    }
    ~VecSet()
    {
        for (auto p : v) delete p;
    }
};

static int do_multishift(lym_context *c, int op_id, int algorithm, int nshift, const double *shifts, double precision,
                         int max_steps, const double *source, double **solutions, lym_solve_stats *stats,
                         bool device_ptr)
{
    if (!shifts || !source || !solutions || nshift < 1 || nshift > kMaxShifts) return LYM_ERR_ARGUMENT;
    for (int i = 0; i < nshift; ++i)
        if (!solutions[i]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        lym_solve_stats local;
        memset(&local, 0, sizeof(local));
        Vec b(c, PREC_D, 2);
        upload_vec(c, *b, source, device_ptr, 0);
        VecSet xs(c, nshift, PREC_D, 2);
        CK(cudaEventRecord(c->ev0, c->st));
        // solutions[i] (i >= 1) hold the chronological guesses on entry
        if (algorithm == LYM_MULTISHIFT_CHRONOLOGICAL)
            for (int i = 1; i < nshift; ++i) upload_vec(c, xs.s[i], solutions[i], device_ptr, 1);
        const int rc = run_multishift(c, op, algorithm, nshift, shifts, precision, max_steps, *b, xs.s, local);
        CK(cudaEventRecord(c->ev1, c->st));
        for (int i = 0; i < nshift; ++i) download_vec(c, solutions[i], xs.s[i], device_ptr, 2), CK(cudaStreamSynchronize(c->st));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        local.seconds = ms * 1e-3;
        if (stats) *stats = local;
        CK(cudaGetLastError());
        return rc;
    });
}

// RationalApproximation::evaluate (dirac_functions/RationalApproximation.cpp:18-42):
// output = sum_i alphas[i] (A + betas[i])^{-1} input, everything on the device.
static int do_rational(lym_context *c, int op_id, int algorithm, int n, const double *alphas, const double *betas,
                       double precision, int max_steps, const double *input, double *output, lym_solve_stats *stats,
                       bool device_ptr)
{
    if (!alphas || !betas || !input || !output || n < 1 || n > kMaxShifts) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        lym_solve_stats local;
        memset(&local, 0, sizeof(local));
        Vec b(c, PREC_D, 2), out(c, PREC_D, 2);
        upload_vec(c, *b, input, device_ptr, 0);
        VecSet xs(c, n, PREC_D, 2);
        for (int i = 1; i < n; ++i) zero(c, xs.s[i]);  // no chronological history
        CK(cudaEventRecord(c->ev0, c->st));
        const int rc = run_multishift(c, op, algorithm, n, betas, precision, max_steps, *b, xs.s, local);
        zero(c, *out);
        for (int i = 0; i < n; ++i) axpby(c, xs.s[i], *out, C2(alphas[i]), C2(1.0));
        CK(cudaEventRecord(c->ev1, c->st));
        download_vec(c, output, *out, device_ptr, 2);
        CK(cudaStreamSynchronize(c->st));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        local.seconds = ms * 1e-3;
        if (stats) *stats = local;
        CK(cudaGetLastError());
        return rc;
    });
}

// The solves of NFlavorFermionAction::updateForce (actions/NFlavorFermionAction.cpp:76-96)
// for one pseudofermion: x_i = (A + betas[i])^{-1} phi with the multishift on square_op_id,
// then y_i = D x_i with dirac_op_id (DiracOperator::multiply), on the device.
static int do_rhmc_force_solves(lym_context *c, int square_op_id, int dirac_op_id, int algorithm, int n,
                                const double *betas, double precision, int max_steps, const double *phi, double **x,
                                double **y, lym_solve_stats *stats, bool device_ptr)
{
    if (!betas || !phi || !x || !y || n < 1 || n > kMaxShifts) return LYM_ERR_ARGUMENT;
    for (int i = 0; i < n; ++i)
        if (!x[i] || !y[i]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &sq = op_of(c, square_op_id);
        OpEntry &dop = op_of(c, dirac_op_id);
        if (dop.gauge_id != sq.gauge_id)
            fail(c, LYM_ERR_ARGUMENT, "the Dirac and squared operators act on different gauge fields");
        lym_solve_stats local;
        memset(&local, 0, sizeof(local));
        Vec b(c, PREC_D, 2), yv(c, PREC_D, 2);
        upload_vec(c, *b, phi, device_ptr, 0);
        VecSet xs(c, n, PREC_D, 2);
        for (int i = 1; i < n; ++i) zero(c, xs.s[i]);
        CK(cudaEventRecord(c->ev0, c->st));
        const int rc = run_multishift(c, sq, algorithm, n, betas, precision, max_steps, *b, xs.s, local);
        for (int i = 0; i < n; ++i) {
            op_apply(c, dop, PREC_D, *yv, xs.s[i], nullptr, C2(0.0));
            download_vec(c, x[i], xs.s[i], device_ptr, 2);
            CK(cudaStreamSynchronize(c->st));
            download_vec(c, y[i], *yv, device_ptr, 2);
            CK(cudaStreamSynchronize(c->st));
        }
        CK(cudaEventRecord(c->ev1, c->st));
        float ms = 0.f;
        CK(cudaEventSynchronize(c->ev1));
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        local.seconds = ms * 1e-3;
        if (stats) *stats = local;
        CK(cudaGetLastError());
        return rc;
    });
}

int lym_multishift(lym_context *c, int op_id, int algorithm, int nshift, const double *shifts, double precision,
                   int max_steps, const double *source, double **solutions, lym_solve_stats *stats)
{
    return do_multishift(c, op_id, algorithm, nshift, shifts, precision, max_steps, source, solutions, stats, false);
}

int lym_multishift_device(lym_context *c, int op_id, int algorithm, int nshift, const double *shifts, double precision,
                          int max_steps, const double *source, double **solutions, lym_solve_stats *stats)
{
    return do_multishift(c, op_id, algorithm, nshift, shifts, precision, max_steps, source, solutions, stats, true);
}

int lym_rational_evaluate(lym_context *c, int op_id, int algorithm, int n, const double *alphas, const double *betas,
                          double precision, int max_steps, const double *input, double *output, lym_solve_stats *stats)
{
    return do_rational(c, op_id, algorithm, n, alphas, betas, precision, max_steps, input, output, stats, false);
}

int lym_rational_evaluate_device(lym_context *c, int op_id, int algorithm, int n, const double *alphas,
                                 const double *betas, double precision, int max_steps, const double *input,
                                 double *output, lym_solve_stats *stats)
{
    return do_rational(c, op_id, algorithm, n, alphas, betas, precision, max_steps, input, output, stats, true);
}

int lym_rhmc_force_solves(lym_context *c, int square_op_id, int dirac_op_id, int algorithm, int n, const double *betas,
                          double precision, int max_steps, const double *phi, double **x, double **y,
                          lym_solve_stats *stats)
{
    return do_rhmc_force_solves(c, square_op_id, dirac_op_id, algorithm, n, betas, precision, max_steps, phi, x, y,
                                stats, false);
}

int lym_rhmc_force_solves_device(lym_context *c, int square_op_id, int dirac_op_id, int algorithm, int n,
                                 const double *betas, double precision, int max_steps, const double *phi, double **x,
                                 double **y, lym_solve_stats *stats)
{
    return do_rhmc_force_solves(c, square_op_id, dirac_op_id, algorithm, n, betas, precision, max_steps, phi, x, y,
                                stats, true);
}


static int do_meson(lym_context *c, const double *const *props, double *pion, double *scalar, double *ps,
                    bool device_ptr)
{
    if (!props || !pion || !scalar || !ps) return LYM_ERR_ARGUMENT;
    for (int k = 0; k < 12; ++k)
        if (!props[k]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const size_t vb = (size_t)c->g.V * 24 * sizeof(double);
        const int Lt = c->g.L[3];
        MesonProps P;
        std::vector<std::unique_ptr<DevBuf>> staged;
        for (int k = 0; k < 12; ++k) {
            if (device_ptr) {
                P.p[k] = (const double2 *)props[k];
            } else {
                staged.emplace_back(new DevBuf(c, vb));
                CK(cudaMemcpyAsync(staged.back()->p, props[k], vb, cudaMemcpyHostToDevice, c->st));
                P.p[k] = (const double2 *)staged.back()->p;
            }
        }
        DevBuf scratch(c, meson_scratch_bytes(c->g)), res(c, 3 * (size_t)Lt * sizeof(double));
        launch_meson_contractions(c->g, P, (double *)scratch.p, (double *)res.p, c->st);
        count(c, 2);
        std::vector<double> h(3 * (size_t)Lt);
        CK(cudaMemcpyAsync(h.data(), res.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        for (int t = 0; t < Lt; ++t) {
            pion[t] = h[t];
            scalar[t] = h[Lt + t];
            ps[t] = h[2 * Lt + t];
        }
        return LYM_OK;
    });
}

int lym_meson_contractions(lym_context *c, const double *const *propagators, double *pion, double *scalar, double *ps)
{
    return do_meson(c, propagators, pion, scalar, ps, false);
}

int lym_meson_contractions_device(lym_context *c, const double *const *propagators, double *pion, double *scalar,
                                  double *ps)
{
    return do_meson(c, propagators, pion, scalar, ps, true);
}

int lym_dots_device(lym_context *c, int n, const double *const *a, const double *const *b, int gamma5, double *out)
{
    if (n < 0 || (n > 0 && (!a || !b || !out))) return LYM_ERR_ARGUMENT;
    for (int k = 0; k < n; ++k)
        if (!a[k] || !b[k]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const int nblk = dot_blocks(c->g);
        DevBuf partials(c, (size_t)kMaxDots * nblk * sizeof(double2)), res(c, (size_t)kMaxDots * sizeof(double2));
        for (int k0 = 0; k0 < n; k0 += kMaxDots) {
            const int m = std::min(kMaxDots, n - k0);
            DotPairs D;
            for (int k = 0; k < m; ++k) {
                D.a[k] = (const double2 *)a[k0 + k];
                D.b[k] = (const double2 *)b[k0 + k];
            }
            launch_dots(c->g, D, m, gamma5 ? 1 : 0, (double2 *)partials.p, (double2 *)res.p, c->st);
            count(c, 2);
            CK(cudaMemcpyAsync(out + 2 * (size_t)k0, res.p, m * sizeof(double2), cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
        }
        CK(cudaGetLastError());
        return LYM_OK;
    });
}

int lym_noise_z2_device(lym_context *c, unsigned long long seed, unsigned long long stream, double *out)
{
    if (!out) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        launch_z2_noise(c->g, out, seed, stream, c->st);
        count(c, 1);
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        return LYM_OK;
    });
}

// MesonCorrelator::execute (correlators/MesonCorrelator.cpp:22-157) on the device: the 12
// point sources (StochasticEstimator.cpp:100-112), their block solve, the contractions.
int lym_meson_correlator(lym_context *c, int op_id, int solver, double precision, int max_steps, int batch,
                         double *pion, double *scalar, double *ps, lym_solve_stats *stats)
{
    if (!pion || !scalar || !ps) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const size_t vb = (size_t)c->g.V * 24 * sizeof(double);
        std::vector<std::unique_ptr<DevBuf>> bufs;
        std::vector<const double *> src(12);
        std::vector<double *> sol(12);
        const double2 one = make_double2(1.0, 0.0);
        for (int k = 0; k < 12; ++k) {
            const int alpha = k % 4, col = k / 4;
            bufs.emplace_back(new DevBuf(c, vb));
            CK(cudaMemsetAsync(bufs.back()->p, 0, vb, c->st));
            CK(cudaMemcpyAsync((double2 *)bufs.back()->p + alpha * 3 + col, &one, sizeof(one), cudaMemcpyHostToDevice,
                               c->st));
            src[k] = (const double *)bufs.back()->p;
            bufs.emplace_back(new DevBuf(c, vb));
            sol[k] = (double *)bufs.back()->p;
        }
        CK(cudaStreamSynchronize(c->st));
        const int rc = do_solve_block(c, op_id, solver, precision, max_steps, 12, src.data(), sol.data(), batch,
                                      stats, true);
        if (rc < 0) return rc;
        const int rm = do_meson(c, sol.data(), pion, scalar, ps, true);
        return rm < 0 ? rm : rc;
    });
}

// ChiralCondensate::execute (fermion_measurements/ChiralCondensate.cpp:84-118) on the
// device: n real Z2 noise vectors eta_k (lym_noise_z2_device streams 0..n-1 of `seed`), the
// block solve D x_k = eta_k and, with `connected`, D y_k = x_k; per estimator k, out[8k..8k+7]
// = <eta,x>/V, <eta,g5 x>/V, <x,x>/V, <eta,y>/V as (re, im) pairs (0 without `connected`).
int lym_chiral_condensate(lym_context *c, int op_id, int solver, double precision, int max_steps, int batch,
                          int n, unsigned long long seed, int connected, double *out, lym_solve_stats *stats)
{
    if (n < 1 || !out) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const size_t vb = (size_t)c->g.V * 24 * sizeof(double);
        std::vector<std::unique_ptr<DevBuf>> bufs;
        std::vector<const double *> eta(n), xc(n);
        std::vector<double *> x(n), y(connected ? n : 0);
        for (int k = 0; k < n; ++k) {
            bufs.emplace_back(new DevBuf(c, vb));
            launch_z2_noise(c->g, (double *)bufs.back()->p, seed, (unsigned long long)k, c->st);
            count(c, 1);
            eta[k] = (const double *)bufs.back()->p;
            bufs.emplace_back(new DevBuf(c, vb));
            x[k] = (double *)bufs.back()->p;
            xc[k] = x[k];
            if (connected) {
                bufs.emplace_back(new DevBuf(c, vb));
                y[k] = (double *)bufs.back()->p;
            }
        }
        CK(cudaStreamSynchronize(c->st));
        int rc = do_solve_block(c, op_id, solver, precision, max_steps, n, eta.data(), x.data(), batch, stats, true);
        if (rc < 0) return rc;
        if (connected) {
            const int rc2 = do_solve_block(c, op_id, solver, precision, max_steps, n, xc.data(), y.data(), batch,
                                           stats ? stats + n : nullptr, true);
            if (rc2 < 0) return rc2;
            if (rc2 != LYM_OK) rc = rc2;
        }
        std::vector<double> d(2 * (size_t)n);
        const double V = (double)c->g.V;
        auto put = [&](int slot) {
            for (int k = 0; k < n; ++k) {
                out[8 * (size_t)k + 2 * slot] = d[2 * k] / V;
                out[8 * (size_t)k + 2 * slot + 1] = d[2 * k + 1] / V;
            }
        };
        int r;
        if ((r = lym_dots_device(c, n, eta.data(), xc.data(), 0, d.data())) < 0) return r;
        put(0);
        if ((r = lym_dots_device(c, n, eta.data(), xc.data(), 1, d.data())) < 0) return r;
        put(1);
        if ((r = lym_dots_device(c, n, xc.data(), xc.data(), 0, d.data())) < 0) return r;
        put(2);
        if (connected) {
            std::vector<const double *> yc(y.begin(), y.end());
            if ((r = lym_dots_device(c, n, eta.data(), yc.data(), 0, d.data())) < 0) return r;
            put(3);
        } else {
            for (int k = 0; k < n; ++k) out[8 * (size_t)k + 6] = out[8 * (size_t)k + 7] = 0.0;
        }
        return rc;
    });
}

int lym_gauge_read(lym_context *c, int gauge_id, int format, const char *directory, const char *name, int number,
                   int boundary, double *plaquette)
{
    if (!c) return LYM_ERR_ARGUMENT;
    const int nc = c->rep == REP_SU3 ? 3 : 2;
    std::vector<double> links;
    try {
        links.resize((size_t)c->g.V * 4 * nc * nc * 2);
    } catch (const std::bad_alloc &) {
        return LYM_ERR_MEMORY;
    }
    const int rc = lym_gauge_file_read(format, c->g.L, nc, directory, name, number, links.data(), plaquette);
    if (rc != LYM_OK) {
        c->err = "gauge configuration file could not be read";
        return rc;
    }
    return lym_gauge_upload_fundamental(c, gauge_id, links.data(), boundary);
}

// FermionForce::derivative (hmc_forces/FermionForce.cpp:11-20) of the operator's force for n
// weighted pairs: ImprovedFermionForce for the kinds with the clover term,
// DiracWilsonFermionForce otherwise
static int do_fermion_force(lym_context *c, int op_id, int n, const double *const *X, const double *const *Y,
                            const double *weights, double *force, bool device_ptr)
{
    if (n < 1 || !X || !Y || !weights || !force) return LYM_ERR_ARGUMENT;
    for (int i = 0; i < n; ++i)
        if (!X[i] || !Y[i]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        GaugeEntry &ge = gauge_of(c, op.gauge_id);
        const size_t vb = (size_t)c->g.V * 24 * sizeof(double), fb = (size_t)c->g.V * 4 * 9 * sizeof(double2);
        std::vector<std::unique_ptr<DevBuf>> bufs;
        std::vector<const double2 *> hx(n), hy(n);
        double *dF = force;
        for (int i = 0; i < n; ++i) {
            if (device_ptr) {
                hx[i] = (const double2 *)X[i];
                hy[i] = (const double2 *)Y[i];
                continue;
            }
            bufs.emplace_back(new DevBuf(c, vb));
            CK(cudaMemcpyAsync(bufs.back()->p, X[i], vb, cudaMemcpyHostToDevice, c->st));
            hx[i] = (const double2 *)bufs.back()->p;
            bufs.emplace_back(new DevBuf(c, vb));
            CK(cudaMemcpyAsync(bufs.back()->p, Y[i], vb, cudaMemcpyHostToDevice, c->st));
            hy[i] = (const double2 *)bufs.back()->p;
        }
        if (!device_ptr) {
            bufs.emplace_back(new DevBuf(c, fb));
            CK(cudaMemcpyAsync(bufs.back()->p, force, fb, cudaMemcpyHostToDevice, c->st));
            dF = (double *)bufs.back()->p;
        }
        DevBuf tab(c, (size_t)n * (2 * sizeof(void *) + sizeof(double)));
        char *t = (char *)tab.p;
        CK(cudaMemcpyAsync(t, hx.data(), n * sizeof(void *), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(t + n * sizeof(void *), hy.data(), n * sizeof(void *), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(t + 2 * n * sizeof(void *), weights, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
        const int clover = kind_has_clover(op.kind) ? 1 : 0;
        std::unique_ptr<DevBuf> scratch;
        if (clover) scratch.reset(new DevBuf(c, fermion_force_scratch_bytes(c->g)));
        launch_fermion_force(c->g, ge.dev, n, (const double2 *const *)t, (const double2 *const *)(t + n * sizeof(void *)),
                             (const double *)(t + 2 * n * sizeof(void *)), op.kappa, op.csw, clover, (double2 *)dF,
                             clover ? (double2 *)scratch->p : nullptr, c->st);
        count(c, 1 + clover);
        if (!device_ptr) CK(cudaMemcpyAsync(force, dF, fb, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        return LYM_OK;
    });
}

int lym_fermion_force(lym_context *c, int op_id, const double *X, const double *Y, double weight, double *force)
{
    return do_fermion_force(c, op_id, 1, &X, &Y, &weight, force, false);
}

int lym_fermion_force_device(lym_context *c, int op_id, const double *X, const double *Y, double weight,
                             double *force)
{
    return do_fermion_force(c, op_id, 1, &X, &Y, &weight, force, true);
}

int lym_fermion_force_multi(lym_context *c, int op_id, int n, const double *const *X, const double *const *Y,
                            const double *weights, double *force)
{
    return do_fermion_force(c, op_id, n, X, Y, weights, force, false);
}

int lym_fermion_force_multi_device(lym_context *c, int op_id, int n, const double *const *X, const double *const *Y,
                                   const double *weights, double *force)
{
    return do_fermion_force(c, op_id, n, X, Y, weights, force, true);
}

int lym_neighbour_tables(lym_context *c, int *sup, int *sdn)
{
    if (!sup || !sdn) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const size_t b = (size_t)c->g.V * 4 * sizeof(int);
        int *d = (int *)dev_alloc(c, 2 * b);
        launch_neighbour_tables(c->g, d, d + (size_t)c->g.V * 4, c->st);
        CK(cudaMemcpyAsync(sup, d, b, cudaMemcpyDeviceToHost, c->st));
        CK(cudaMemcpyAsync(sdn, d + (size_t)c->g.V * 4, b, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        dev_free(c, d, 2 * b);
        return LYM_OK;
    });
}

int lym_stencil_indices(lym_context *c, int *out)
{
    if (!out) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        const size_t b = (size_t)c->g.V * 9 * sizeof(int);
        int *d = (int *)dev_alloc(c, b);
        launch_stencil_index_probe(c->g, d, c->st);
        CK(cudaMemcpyAsync(out, d, b, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        dev_free(c, d, b);
        return LYM_OK;
    });
}

unsigned long long lym_context_kernel_launches(lym_context *c) { return c ? c->launches : 0ull; }

int lym_context_engine_stats(lym_context *c, double *out, int n)
{
    if (!c || !out || n < 0) return LYM_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> g(c->mu);
    for (int k = 0; k < n && k < 9; ++k) out[k] = c->engine_stats[k];
    return LYM_OK;
}

int lym_time_stencil(lym_context *c, int op_id, int prec, int which, int iters, double *ms_per_launch)
{
    if (!ms_per_launch || iters < 1 || prec < PREC_D || prec > PREC_H || which < 0 || which > 1)
        return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        GaugeEntry &ge = gauge_of(c, op.gauge_id);
        const bool clov = kind_has_clover(op.kind);
        if (clov) ensure_clover(c, op);
        require_recon(c, ge, prec);
        Vec a(c, prec, 1), b(c, prec, 1), y(c, prec, 1);
        DslashParams P;
        P.g = c->g;
        P.prec = prec;
        P.rep = c->rep;
        P.U = &ge.dev;
        if (which == 0) {  // out_o = T_oo y_o - kappa^2 H_oe a_e  (second half of the Schur operator)
            P.epi = EPI_XPAY_;
            P.parity = 1;
            P.clover = clov ? op.clover.T[prec] : nullptr;
            P.b = -op.kappa * op.kappa;
        } else {           // out_e = Tinv_ee H_eo a_o             (first half)
            P.epi = clov ? EPI_CLOVINV_ : EPI_SCALE_;
            P.parity = 0;
            P.clover = clov ? op.clover.Tinv[prec] : nullptr;
        }
        P.in = *a;
        P.out = *b;
        P.y = *y;
        P.v2 = *y;
        for (int k = 0; k < 3; ++k) launch_dslash(P, c->st);
        CK(cudaEventRecord(c->ev0, c->st));
        for (int k = 0; k < iters; ++k) launch_dslash(P, c->st);
        CK(cudaEventRecord(c->ev1, c->st));
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        count(c, iters + 3);
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        *ms_per_launch = (double)ms / iters;
        return LYM_OK;
    });
}

int lym_time_stencil_batch(lym_context *c, int op_id, int prec, int which, int batch, int iters,
                           double *ms_per_launch)
{
    if (!ms_per_launch || iters < 1 || (prec != PREC_F && prec != PREC_H) || which < 0 || which > 1 ||
        batch < 2 || batch > kMaxBatch || (batch & (batch - 1)))
        return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        OpEntry &op = op_of(c, op_id);
        GaugeEntry &ge = gauge_of(c, op.gauge_id);
        const bool clov = kind_has_clover(op.kind);
        if (clov) ensure_clover(c, op);
        BVec a(c, prec, batch), b(c, prec, batch), y(c, prec, batch);
        for (BVec *v : {&a, &b, &y}) CK(cudaMemsetAsync(v->s.v, 0, v->bytes, c->st));
        SlotTables tab(c, std::vector<const OpEntry *>(batch, &op));  // every slot on this operator
        const BatchTile tile = tune_batch(c, ge.dev, clov, prec, b.s, a.s, y.s, tab.b, tab.T, tab.Ti, tab.uniform);
        DslashBatchParams P;
        P.g = c->g;
        P.prec = prec;
        P.rep = c->rep;
        P.U = &ge.dev;
        P.nbr = c->nbr;
        P.order = order_table(c, tile.by, tile.bz);
        P.err = c->d_err + 1;  // the copy-wait word of the bulk-copy variant
        P.walk_by = tile.by;
        P.walk_bz = tile.bz;
        P.minb = tile.minb;
        P.has_clover = clov;
        P.uniform = tab.uniform;
        if (which == 0) {
            P.epi = EPI_XPAY_;
            P.parity = 1;
            P.clover_slot = clov ? tab.T : nullptr;
            P.b_slot = tab.b;
        } else {
            P.epi = clov ? EPI_CLOVINV_ : EPI_SCALE_;
            P.parity = 0;
            P.clover_slot = clov ? tab.Ti : nullptr;
        }
        P.in = a.s;
        P.out = b.s;
        P.y = y.s;
        for (int k = 0; k < 3; ++k) launch_dslash_batch(P, c->st);
        CK(cudaEventRecord(c->ev0, c->st));
        for (int k = 0; k < iters; ++k) launch_dslash_batch(P, c->st);
        CK(cudaEventRecord(c->ev1, c->st));
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
        check_copy_waits(c, tile);
        count(c, iters + 3);
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        *ms_per_launch = (double)ms / iters;
        return LYM_OK;
    });
}

int lym_multiply_batch(lym_context *c, int prec, int nrhs, const int *op_ids, const double *const *in,
                       double *const *out)
{
    if (!op_ids || !in || !out || nrhs < 1 || nrhs > kMaxBatch || (prec != PREC_F && prec != PREC_H))
        return LYM_ERR_ARGUMENT;
    for (int j = 0; j < nrhs; ++j)
        if (!in[j] || !out[j]) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        std::vector<const OpEntry *> ops;
        for (int j = 0; j < nrhs; ++j) {
            OpEntry &op = op_of(c, op_ids[j]);
            if (op.kind != LYM_OP_EVEN_ODD_IMPROVED)
                fail(c, LYM_ERR_UNSUPPORTED, "lym_multiply_batch applies EvenOddImproved operators");
            if (j && (op.gauge_id != ops[0]->gauge_id || op.gamma5 != ops[0]->gamma5))
                fail(c, LYM_ERR_ARGUMENT, "the operators of one batch share the gauge field and the gamma5 flag");
            ensure_clover(c, op);
            ops.push_back(&op);
        }
        int nb = 2;
        while (nb < nrhs) nb *= 2;
        BVec bin(c, prec, nb), btmp(c, prec, nb), bout(c, prec, nb);
        for (BVec *v : {&bin, &btmp, &bout}) CK(cudaMemsetAsync(v->s.v, 0, v->bytes, c->st));
        std::vector<const OpEntry *> slot_ops(nb, ops[0]);  // unused slots borrow the first operator
        for (int j = 0; j < nrhs; ++j) slot_ops[j] = ops[j];
        SlotTables tab(c, slot_ops);
        Vec full(c, PREC_D, 2);
        for (int j = 0; j < nrhs; ++j) {
            upload_vec(c, *full, in[j], false, 0);
            if (prec == PREC_F) axpby_views(c, (*full).parity(1).d(), bin.f().slot(j), C2(1.0), C2(0.0));
            else axpby_views(c, (*full).parity(1).d(), bin.h().slot(j), C2(1.0), C2(0.0));
        }
        const GaugeDev &U = gauge_of(c, ops[0]->gauge_id).dev;
        const BatchTile tile = tune_batch(c, U, true, prec, btmp.s, bin.s, bout.s, tab.b, tab.T, tab.Ti, tab.uniform);
        apply_schur_batch(c, U, true, prec, bout.s, bin.s, btmp.s, ops[0]->gamma5, nullptr, nullptr, tab.b, tab.T,
                          tab.Ti, tile, tab.uniform);
        for (int j = 0; j < nrhs; ++j) {
            upload_vec(c, *full, in[j], false, 0);  // the even parity passes through
            if (prec == PREC_F) axpby_views(c, bout.f().slot(j), (*full).parity(1).d(), C2(1.0), C2(0.0));
            else axpby_views(c, bout.h().slot(j), (*full).parity(1).d(), C2(1.0), C2(0.0));
            download_vec(c, out[j], *full, false, 0);
            CK(cudaStreamSynchronize(c->st));
        }
        CK(cudaGetLastError());
        check_copy_waits(c, tile);
        return LYM_OK;
    });
}

int lym_set_batch_tile(lym_context *c, int by, int bz, int minb)
{
    return guarded(c, [&]() {
        if (by < 0) {
            c->tile_forced = false;
            return LYM_OK;
        }
        bool known = false;
        for (int k = 0; k < kBatchMinBlocksCount; ++k) known |= kBatchMinBlocks[k] == minb;
        const Geom &g = c->g;
        if (!known || (by != 0 && (g.L[1] % by || bz < 1 || g.L[2] % bz)))
            fail(c, LYM_ERR_ARGUMENT, "batch tile (%d, %d, %d) does not fit the lattice or the compiled variants", by,
                 bz, minb);
        c->forced_tile = BatchTile{by, by ? bz : 0, minb};
        c->tile_forced = true;
        return LYM_OK;
    });
}

int lym_get_batch_tile(lym_context *c, int prec, int batch, int has_clover, int *by, int *bz, int *minb)
{
    if (!by || !bz || !minb) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        BatchTile t;
        if (c->tile_forced) {
            t = c->forced_tile;
        } else {
            auto it = c->tiles.find((prec * 64 + batch) * 2 + (has_clover ? 1 : 0));
            if (it == c->tiles.end()) fail(c, LYM_ERR_NOT_FOUND, "no tuned batch configuration for this key yet");
            t = it->second;
        }
        *by = t.by;
        *bz = t.bz;
        *minb = t.minb;
        return LYM_OK;
    });
}

int lym_set_link_format(lym_context *c, int reals)
{
    return guarded(c, [&]() {
        if (reals != 12 && reals != 8) fail(c, LYM_ERR_ARGUMENT, "link format: 12 or 8 reals");
        if (reals == 8 && c->rep != REP_SU3)
            fail(c, LYM_ERR_UNSUPPORTED, "the 8-real link format is for SU(3) fundamental links");
        c->link_reals = reals;
        for (auto &kv : c->gauges) kv.second.dev.link_reals = reals;
        return LYM_OK;
    });
}

int lym_context_inject_alloc_failures(lym_context *c, int n)
{
    if (n < 0) return LYM_ERR_ARGUMENT;
    return guarded(c, [&]() {
        c->inject_alloc_failures = n;
        return LYM_OK;
    });
}

int lym_context_inject_copy_wait_timeout(lym_context *c)
{
    return guarded(c, [&]() {
        c->inject_copy_wait = true;
        return LYM_OK;
    });
}

void *lym_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void lym_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

}  // extern "C"

// ------------------------------------------------- allocation-free variant --
extern "C" int lym_multiply_device_noalloc(lym_context *c, int op_id, double *out, const double *in)
{
    return guarded(c, [&]() {
        if (!out || !in || out == in)
            fail(c, LYM_ERR_ARGUMENT, "lym_multiply_device_noalloc: out and in must be distinct device vectors");
        OpEntry &op = op_of(c, op_id);
        if (op.kind != LYM_OP_EVEN_ODD_IMPROVED)
            fail(c, LYM_ERR_UNSUPPORTED, "lym_multiply_device_noalloc applies EvenOddImproved operators only");
        if (c->g.Vh > kNoallocMaxHalfSites)
            fail(c, LYM_ERR_ARGUMENT, "lym_multiply_device_noalloc: volume %d exceeds its maximum of %d sites",
                 c->g.V, 2 * kNoallocMaxHalfSites);
        if (!op.clover_ok)
            fail(c, LYM_ERR_ARGUMENT,
                 "lym_multiply_device_noalloc: the operator's clover term is not built yet (building it allocates); "
                 "apply the operator once through lym_multiply or lym_multiply_device first");
        GaugeEntry &ge = gauge_of(c, op.gauge_id);
        cudaError_t ce = cudaSuccess;
        const int rc =
            noalloc_schur(c->g, c->rep, c->device, c->st, ge.dev, &op.clover, op.kappa, op.gamma5, out, in, &ce);
        if (rc != LYM_OK)
            fail(c, rc, "lym_multiply_device_noalloc: CUDA error %s", cudaGetErrorString(ce));
        CK(cudaStreamSynchronize(c->st));
        count(c, 2);
        return LYM_OK;
    });
}

#include "lym_server.inc"
