// Multi-right-hand-side (batched) fields and kernels.
//
// A batch of nb right-hand sides (nb a power of two <= 32) is stored interleaved with
// the RHS index innermost: word k of RHS r at half-site h is v[(k*stride + h)*nb + r].
// One thread handles one (h, r) pair with r fastest, so the nb lanes of a site load the
// same neighbour-index, link and clover words (one broadcast transaction) while their
// spinor words are nb consecutive vectors (fully coalesced).  Link, clover and index
// traffic per site is therefore shared by the whole batch, which is why this path reads
// uncompressed 18-real links and a neighbour table instead of recomputing them per lane.
#pragma once

#include "lym_blas.cuh"
#include "lym_dslash.cuh"

namespace lym {

constexpr int kMaxBatch = 32;

// ------------------------------------------------------------ batch views --
struct SpinorFBr {  // FP32, one RHS of a batch
    float4 *v;
    int stride, lognb, r;
    LYM_HD SpinorFBr par(int) const { return *this; }  // one parity per batch view
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float4 w = __ldg(v + (((size_t)k * stride + h) << lognb) + r);
            s[2 * k] = cx<R>{(R)w.x, (R)w.y};
            s[2 * k + 1] = cx<R>{(R)w.z, (R)w.w};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 6; ++k)
            v[(((size_t)k * stride + h) << lognb) + r] =
                make_float4((float)s[2 * k].re, (float)s[2 * k].im, (float)s[2 * k + 1].re, (float)s[2 * k + 1].im);
    }
};

struct SpinorFB {
    float4 *v;
    int stride, lognb;
    LYM_HD SpinorFB par(int p) const { return SpinorFB{v + ((size_t)p * 6 * stride << lognb), stride, lognb}; }
    LYM_HD SpinorFBr bind(int r) const { return SpinorFBr{v, stride, lognb, r}; }
};

struct SpinorHBr {  // FP16 with a per-(site, RHS) norm, one RHS of a batch
    int4 *v;
    float *norm;
    int stride, lognb, r;
    LYM_HD SpinorHBr par(int) const { return *this; }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
        const float nrm = __ldg(norm + ((size_t)h << lognb) + r);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int4 w = __ldg(v + (((size_t)k * stride + h) << lognb) + r);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&w);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 f = __half22float2(hp[j]);
                s[4 * k + j] = cx<R>{(R)(f.x * nrm), (R)(f.y * nrm)};
            }
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < 12; ++k) m = fmaxf(m, fmaxf(fabsf((float)s[k].re), fabsf((float)s[k].im)));
        const float inv = m > 0.f ? 1.0f / m : 0.f;
        norm[((size_t)h << lognb) + r] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int4 w;
            __half2 *hp = reinterpret_cast<__half2 *>(&w);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                hp[j] = __floats2half2_rn((float)s[4 * k + j].re * inv, (float)s[4 * k + j].im * inv);
            v[(((size_t)k * stride + h) << lognb) + r] = w;
        }
    }
};

struct SpinorHB {
    int4 *v;
    float *norm;
    int stride, lognb;
    LYM_HD SpinorHB par(int p) const
    {
        return SpinorHB{v + ((size_t)p * 3 * stride << lognb), norm + ((size_t)p * stride << lognb), stride, lognb};
    }
    LYM_HD SpinorHBr bind(int r) const { return SpinorHBr{v, norm, stride, lognb, r}; }
};

// ---------------------------------------------------------- batch stencil --
template <class SB, class GaugeT, class CloverT> struct DslashBatchArg {
    Geom g;
    SB in, out, y;
    GaugeT U;
    CloverT T;
    int parity, gamma5, has_clover, lognb;
    double a, b;
    NbrTable nbr;        // precomputed neighbour half-site indices
    const int *skip_if;  // skip the launch when *skip_if != 0
    const int *active;   // per-RHS mask (nullptr: all active)
    // per-RHS operator (nullptr: the shared a/b and T above): slots of one batch share the
    // gauge field but may carry different kappa, hence different b and clover terms
    const double *b_slot;
    const void *const *clover_slot;
};

// out_r = a H in_r (EPI_SCALE), Tinv (a H in_r) (EPI_CLOVINV) or
// G5^g (T y_r + b H in_r) (EPI_XPAY), for every active RHS r
template <typename R, int EPI, class SB, class GaugeT, class CloverT>
__global__ void __launch_bounds__(128) dslash_batch_kernel(const DslashBatchArg<SB, GaugeT, CloverT> arg)
{
    if (arg.skip_if && *arg.skip_if) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int h = tid >> arg.lognb, r = tid & ((1 << arg.lognb) - 1);
    if (h >= arg.g.Vh) return;
    if (arg.active && !arg.active[r]) return;
    const auto in = arg.in.bind(r);
    CloverT T = arg.T;
    if (arg.clover_slot) T.c = (decltype(T.c))arg.clover_slot[r];
    cx<R> acc[12], res[12];
    hopping_table<R>(arg.nbr, in, arg.U, arg.parity, h, acc);
    if (EPI == EPI_SCALE) {
#pragma unroll
        for (int k = 0; k < 12; ++k) res[k] = (R)arg.a * acc[k];
    } else if (EPI == EPI_CLOVINV) {
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = (R)arg.a * acc[k];
        clover_apply<R>(T, arg.parity, h, acc, res);
    } else {
        cx<R> yv[12];
        arg.y.bind(r).template load<R>(h, yv);
        if (arg.has_clover) {
            clover_apply<R>(T, arg.parity, h, yv, res);
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) res[k] = yv[k];
        }
        const R b = arg.b_slot ? (R)arg.b_slot[r] : (R)arg.b;
#pragma unroll
        for (int k = 0; k < 12; ++k) fma_r(res[k], b, acc[k]);
        if (arg.gamma5) {
#pragma unroll
            for (int k = 6; k < 12; ++k) res[k] = -res[k];
        }
    }
    arg.out.bind(r).template store<R>(h, res);
}

// --------------------------------------------------- batch site kernels ----
// Like site_kernel, over (h, r) pairs; each thread keeps one r (the grid stride is a
// multiple of nb), reductions are per RHS: partials[block][r][k], and the last block
// runs Op::finalize(r, totals) for every r in parallel (thread r).
template <class Op>
__global__ void __launch_bounds__(kBlasThreads) site_batch_kernel(Op op, int vh, int lognb, double *partials,
                                                                  unsigned int *counter, Gate gate)
{
    if (gate.closed()) return;
    constexpr int NR = Op::NRED > 0 ? Op::NRED : 1;
    const int nb = 1 << lognb;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = tid & (nb - 1);
    double acc[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) acc[k] = 0.0;
    const long total = (long)vh << lognb;
    for (long i = tid; i < total; i += (long)gridDim.x * blockDim.x) op.site((int)(i >> lognb), r, acc);
    if constexpr (Op::NRED > 0) {
        __shared__ double smem[kBlasThreads / 32][kMaxBatch][NR];
        __shared__ bool last;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            double x = acc[k];
            for (int o = 16; o >= nb; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            acc[k] = x;
        }
        if (lane < nb)
#pragma unroll
            for (int k = 0; k < NR; ++k) smem[warp][lane][k] = acc[k];
        __syncthreads();
        if (threadIdx.x < nb) {
            for (int k = 0; k < NR; ++k) {
                double s = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += smem[w][threadIdx.x][k];
                partials[((size_t)blockIdx.x * kMaxBatch + threadIdx.x) * NR + k] = s;
            }
            __threadfence();  // every writer makes its partial sums visible device-wide
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned int ticket = atomicAdd(counter, 1u);
            last = (ticket == gridDim.x - 1);
        }
        __syncthreads();
        if (last) {
            __threadfence();
            if (threadIdx.x < nb) {
                double tot[NR];
                for (int k = 0; k < NR; ++k) {
                    double s = 0.0;
                    for (int b = 0; b < (int)gridDim.x; ++b)
                        s += ((volatile double *)partials)[((size_t)b * kMaxBatch + threadIdx.x) * NR + k];
                    tot[k] = s;
                }
                op.finalize(threadIdx.x, tot);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                op.finalize_all();
                *counter = 0u;
            }
        }
    }
}

// ------------------------------------------------------ batched CG state ---
struct BatchCGState {
    int pause;                 // gates every captured kernel
    int iter, max_iter, nb;
    double delta2;
    double rr[kMaxBatch], rr_prev[kMaxBatch], rr_max[kMaxBatch], eps[kMaxBatch], beta[kMaxBatch];
    double2 alpha[kMaxBatch];
    int active[kMaxBatch];     // 0: converged and frozen
    int converged[kMaxBatch];  // the recursion's residual reached eps
    int need_update[kMaxBatch];
    int failed;
};

template <class SP, class SAp> struct OpBAlpha {
    static constexpr int NRED = 2;
    SP p;
    SAp ap;
    BatchCGState *s;
    LYM_D void site(int h, int r, double *acc) const
    {
        if (!s->active[r]) return;
        cx<double> x[12], y[12];
        p.bind(r).template load<double>(h, x);
        ap.bind(r).template load<double>(h, y);
        dotc(x, y, acc[0], acc[1]);
    }
    LYM_D void finalize(int r, const double *t) const
    {
        if (s->active[r]) s->alpha[r] = cdiv(make_double2(s->rr[r], 0.0), make_double2(t[0], t[1]));
    }
    LYM_D void finalize_all() const {}
};

template <class SX, class SP, class SR, class SAp> struct OpBUpdate {
    static constexpr int NRED = 1;
    SX x;
    SP p;
    SR rv;
    SAp ap;
    BatchCGState *s;
    LYM_D void site(int h, int r, double *acc) const
    {
        if (!s->active[r]) return;
        const cx<double> al = {s->alpha[r].x, s->alpha[r].y};
        cx<double> xv[12], pv[12], res[12], av[12];
        x.bind(r).template load<double>(h, xv);
        p.bind(r).template load<double>(h, pv);
        rv.bind(r).template load<double>(h, res);
        ap.bind(r).template load<double>(h, av);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            fma_c(xv[k], al, pv[k]);
            res[k] = res[k] - al * av[k];
        }
        acc[0] += norm2(res);
        x.bind(r).template store<double>(h, xv);
        rv.bind(r).template store<double>(h, res);
    }
    LYM_D void finalize(int r, const double *t) const
    {
        if (!s->active[r]) return;
        const double rr_new = t[0];
        s->rr_prev[r] = s->rr[r];
        s->beta[r] = rr_new / s->rr[r];
        s->rr[r] = rr_new;
        if (rr_new > s->rr_max[r]) s->rr_max[r] = rr_new;
        if (!(rr_new == rr_new)) {
            s->failed = 1;
            s->pause = 1;
        } else if (rr_new < s->eps[r]) {
            s->converged[r] = 1;
            s->need_update[r] = 1;
            s->pause = 1;
        } else if (rr_new < s->delta2 * s->rr_max[r]) {
            s->need_update[r] = 1;
            s->pause = 1;
        }
    }
    LYM_D void finalize_all() const
    {
        s->iter += 1;
        if (s->iter >= s->max_iter) s->pause = 1;
    }
};

template <class SP, class SR> struct OpBDirection {
    static constexpr int NRED = 0;
    SP p;
    SR rv;
    BatchCGState *s;
    LYM_D void site(int h, int r, double *) const
    {
        if (!s->active[r] || s->need_update[r]) return;
        const double b = s->beta[r];
        cx<double> pv[12], res[12];
        p.bind(r).template load<double>(h, pv);
        rv.bind(r).template load<double>(h, res);
#pragma unroll
        for (int k = 0; k < 12; ++k) pv[k] = res[k] + b * pv[k];
        p.bind(r).template store<double>(h, pv);
    }
    LYM_D void finalize(int, const double *) const {}
    LYM_D void finalize_all() const {}
};

}  // namespace lym
