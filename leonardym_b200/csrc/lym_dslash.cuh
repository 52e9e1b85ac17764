// Wilson hopping stencil and its fused epilogues.
//
// H x(s) = sum_mu [ U_mu(s) (1 - g_mu) x(s+mu) + U_mu(s-mu)^+ (1 + g_mu) x(s-mu) ]
// in the chiral basis of the reference, written through its half-spinor
// projections (dirac_operators/DiracWilsonOperator.cpp:25-190):
//   h_k(minus, from s-mu) = x_k + c[mu][k] x_{p[mu][k]},
//   h_k(plus,  from s+mu) = x_k - c[mu][k] x_{p[mu][k]},  k = 0, 1
//   upper spin k   += W_minus + W_plus
//   lower spin p   += conj(c) (W_minus - W_plus)
// with c = {(-i,-i), (-1,+1), (-i,+i), (+1,+1)}, p = {(3,2), (3,2), (2,3), (2,3)}.
#pragma once

#include "lym_common.cuh"

namespace lym {

// c codes: 0 -> +1, 1 -> -1, 2 -> +i, 3 -> -i
template <typename R> LYM_D cx<R> mul_code(int code, cx<R> z)
{
    switch (code) {
    case 0: return z;
    case 1: return -z;
    case 2: return times_i(z);
    default: return times_mi(z);
    }
}
LYM_D int conj_code(int code) { return code < 2 ? code : (code ^ 1); }

constexpr int proj_code(int mu, int k)
{
    return (mu == 0) ? 3 : (mu == 1) ? (k == 0 ? 1 : 0) : (mu == 2) ? (k == 0 ? 3 : 2) : 0;
}
constexpr int proj_partner(int mu, int k) { return (mu < 2) ? (k == 0 ? 3 : 2) : (k == 0 ? 2 : 3); }

// Accumulate H x at half-site h of output parity p.  `in` addresses the other parity.
template <typename R, class SpinorT, class GaugeT>
LYM_D void hopping(const Geom &g, const SpinorT &in, const GaugeT &U, int p, int h, cx<R> acc[12])
{
    int c[4];
    site_coords(g, h, p, c);
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = cx<R>{0, 0};
    const int q = 1 - p;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        {  // forward neighbour: U_mu(s) (1 - g_mu) x(s + mu)
            const int hf = neighbour_h(g, c, mu, +1);
            cx<R> x[12];
            in.template load<R>(hf, x);
            typename GaugeT::Link L;
            U.load(p, mu, h, L);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int code = proj_code(mu, k), pk = proj_partner(mu, k);
                cx<R> hv[3], w[3];
#pragma unroll
                for (int m = 0; m < 3; ++m) hv[m] = x[3 * k + m] - mul_code(code, x[3 * pk + m]);
                mul_u(L, hv, w);
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    acc[3 * k + m] = acc[3 * k + m] + w[m];
                    acc[3 * pk + m] = acc[3 * pk + m] - mul_code(conj_code(code), w[m]);
                }
            }
        }
        {  // backward neighbour: U_mu(s - mu)^+ (1 + g_mu) x(s - mu)
            const int hb = neighbour_h(g, c, mu, -1);
            cx<R> x[12];
            in.template load<R>(hb, x);
            typename GaugeT::Link L;
            U.load(q, mu, hb, L);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int code = proj_code(mu, k), pk = proj_partner(mu, k);
                cx<R> hv[3], w[3];
#pragma unroll
                for (int m = 0; m < 3; ++m) hv[m] = x[3 * k + m] + mul_code(code, x[3 * pk + m]);
                mul_ud(L, hv, w);
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    acc[3 * k + m] = acc[3 * k + m] + w[m];
                    acc[3 * pk + m] = acc[3 * pk + m] + mul_code(conj_code(code), w[m]);
                }
            }
        }
    }
}

// The same accumulation with the neighbour indices read from a table.
template <typename R, class SpinorT, class GaugeT>
LYM_D void hopping_table(const NbrTable &nbr, const SpinorT &in, const GaugeT &U, int p, int h, cx<R> acc[12])
{
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = cx<R>{0, 0};
    const int q = 1 - p;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        {
            const int hf = nbr.get(p, mu, 0, h);
            cx<R> x[12];
            in.template load<R>(hf, x);
            typename GaugeT::Link L;
            U.load(p, mu, h, L);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int code = proj_code(mu, k), pk = proj_partner(mu, k);
                cx<R> hv[3], w[3];
#pragma unroll
                for (int m = 0; m < 3; ++m) hv[m] = x[3 * k + m] - mul_code(code, x[3 * pk + m]);
                mul_u(L, hv, w);
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    acc[3 * k + m] = acc[3 * k + m] + w[m];
                    acc[3 * pk + m] = acc[3 * pk + m] - mul_code(conj_code(code), w[m]);
                }
            }
        }
        {
            const int hb = nbr.get(p, mu, 1, h);
            cx<R> x[12];
            in.template load<R>(hb, x);
            typename GaugeT::Link L;
            U.load(q, mu, hb, L);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int code = proj_code(mu, k), pk = proj_partner(mu, k);
                cx<R> hv[3], w[3];
#pragma unroll
                for (int m = 0; m < 3; ++m) hv[m] = x[3 * k + m] + mul_code(code, x[3 * pk + m]);
                mul_ud(L, hv, w);
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    acc[3 * k + m] = acc[3 * k + m] + w[m];
                    acc[3 * pk + m] = acc[3 * pk + m] + mul_code(conj_code(code), w[m]);
                }
            }
        }
    }
}

template <typename R, class CloverT>
LYM_D void clover_apply(const CloverT &T, int p, int h, const cx<R> x[12], cx<R> y[12])
{
    R d[6];
    cx<R> o[15];
    T.template load_block<R>(p, 0, h, d, o);
    hermitian6_apply(d, o, x, y);
    T.template load_block<R>(p, 1, h, d, o);
    hermitian6_apply(d, o, x + 6, y + 6);
}

// Epilogue kinds
enum Epilogue : int {
    EPI_SCALE = 0,      // out = a * Hx
    EPI_CLOVINV = 1,    // out = Tinv (a * Hx)        (Tinv of the output parity)
    EPI_XPAY = 2,       // out = G5^g (T y + b Hx) + alpha v2   (T = 1 without clover)
    EPI_XPAY_INV = 3,   // out = Tinv (y + b Hx)
    EPI_XPAY_RES = 4,   // EPI_XPAY, then s = r - alpha out per RHS (batched BiCGStab)
    EPI_XPAY_OMEGA = 5, // EPI_XPAY, then the BiCGStab omega sums of out, y and rhat per RHS
};

template <class SpinorT, class GaugeT, class CloverT>
struct DslashArg {
    Geom g;
    SpinorT in;    // input, other parity (half-vector view)
    SpinorT out;   // output parity view
    SpinorT y;     // EPI_XPAY: same-parity input
    SpinorT v2;    // EPI_XPAY: optional added vector
    GaugeT U;
    CloverT T;     // T (EPI_XPAY with clover) or Tinv (EPI_CLOVINV)
    int parity;    // output parity
    int gamma5;    // EPI_XPAY: negate lower spins of (T y + b Hx)
    int has_v2;
    int has_clover;
    double a, b, alpha_re, alpha_im;
    const int *skip_if;  // optional: skip when *skip_if != 0
};

template <typename R, int EPI, class SpinorT, class GaugeT, class CloverT>
__global__ void __launch_bounds__(128) dslash_kernel(const DslashArg<SpinorT, GaugeT, CloverT> arg)
{
    if (arg.skip_if && *arg.skip_if) return;
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= arg.g.Vh) return;
    cx<R> acc[12];
    hopping<R>(arg.g, arg.in, arg.U, arg.parity, h, acc);
    cx<R> res[12];
    if (EPI == EPI_SCALE) {
#pragma unroll
        for (int k = 0; k < 12; ++k) res[k] = (R)arg.a * acc[k];
    } else if (EPI == EPI_CLOVINV) {
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = (R)arg.a * acc[k];
        clover_apply<R>(arg.T, arg.parity, h, acc, res);
    } else if (EPI == EPI_XPAY_INV) {
        cx<R> yv[12];
        arg.y.template load<R>(h, yv);
        const R b = (R)arg.b;
#pragma unroll
        for (int k = 0; k < 12; ++k) fma_r(yv[k], b, acc[k]);
        clover_apply<R>(arg.T, arg.parity, h, yv, res);
    } else {
        cx<R> yv[12];
        arg.y.template load<R>(h, yv);
        if (arg.has_clover) {
            clover_apply<R>(arg.T, arg.parity, h, yv, res);
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) res[k] = yv[k];
        }
        const R b = (R)arg.b;
#pragma unroll
        for (int k = 0; k < 12; ++k) fma_r(res[k], b, acc[k]);
        if (arg.gamma5) {
#pragma unroll
            for (int k = 6; k < 12; ++k) res[k] = -res[k];
        }
        if (arg.has_v2) {
            cx<R> v[12];
            arg.v2.template load<R>(h, v);
            const cx<R> al = {(R)arg.alpha_re, (R)arg.alpha_im};
#pragma unroll
            for (int k = 0; k < 12; ++k) fma_c(res[k], al, v[k]);
        }
    }
    arg.out.template store<R>(h, res);
}

// The second launch of a Schur product inside the even-odd CG on (gamma5 S)^2 (the CG of
// ConjugateGradient.cpp:10-74 run on the normal equations of the Schur system), with the
// CG's vector work in the epilogue.  Q = gamma5 S is Hermitian, so with A = Q Q,
// <p, A p> = |Q p|^2:
//   CG_NORM:   q = G5 (T y + b H x) (y = p) is stored and |q|^2 is reduced; fin(|q|^2) sets
//              alpha = |r|^2 / <p, A p> (so no pass over p and A p is needed for alpha);
//   CG_UPDATE: A p = G5 (T y + b H x) (y = q) stays in registers: x += alpha p (p read from
//              v2), r -= alpha A p, and |r|^2 is reduced; fin(|r|^2) runs the CG step's
//              scalar recursion (beta, stop and reliable-update tests).  A p is never written.
// The per-block sums go to fixed slots; the last block (atomic ticket) adds them in a fixed
// order, so the result is the same on every run.
enum CGFuseMode : int { CG_NORM = 0, CG_UPDATE = 1 };

template <class SX, class SR, class Fin> struct CGEpilogue {
    SX x;
    SR r;
    const double2 *alpha;    // CG_UPDATE: the state's alpha
    Fin fin;
    double *partials;        // [gridDim.x]
    unsigned int *counter;   // zero between launches
};

template <typename R, int MODE, class SpinorT, class GaugeT, class CloverT, class SX, class SR, class Fin>
__global__ void __launch_bounds__(128)
    dslash_cg_kernel(const DslashArg<SpinorT, GaugeT, CloverT> arg, const CGEpilogue<SX, SR, Fin> f)
{
    if (arg.skip_if && *arg.skip_if) return;  // the whole grid: the CG state is paused
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (h < arg.g.Vh) {
        cx<R> acc[12], yv[12], res[12];
        hopping<R>(arg.g, arg.in, arg.U, arg.parity, h, acc);
        arg.y.template load<R>(h, yv);
        if (arg.has_clover) {
            clover_apply<R>(arg.T, arg.parity, h, yv, res);
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) res[k] = yv[k];
        }
        const R b = (R)arg.b;
#pragma unroll
        for (int k = 0; k < 12; ++k) fma_r(res[k], b, acc[k]);
#pragma unroll
        for (int k = 6; k < 12; ++k) res[k] = -res[k];  // gamma5
        if (MODE == CG_NORM) {
            arg.out.template store<R>(h, res);
#pragma unroll
            for (int k = 0; k < 12; ++k) part += (double)res[k].re * res[k].re + (double)res[k].im * res[k].im;
        } else {
            const double2 a = *f.alpha;
            const cx<double> al = {a.x, a.y};
            cx<double> xv[12], pv[12], rv[12];
            f.x.template load<double>(h, xv);
            arg.v2.template load<double>(h, pv);
            f.r.template load<double>(h, rv);
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                fma_c(xv[k], al, pv[k]);
                const cx<double> ap = {(double)res[k].re, (double)res[k].im};
                rv[k] = rv[k] - al * ap;
                part += rv[k].re * rv[k].re + rv[k].im * rv[k].im;
            }
            f.x.template store<double>(h, xv);
            f.r.template store<double>(h, rv);
        }
    }
    // fixed-order reduction: warps, then the block's 4 warps, then the blocks in order
    __shared__ double wsum[4];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        f.partials[blockIdx.x] = (wsum[0] + wsum[1]) + (wsum[2] + wsum[3]);
        __threadfence();
        last = atomicAdd(f.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t += ((volatile double *)f.partials)[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        f.fin((wsum[0] + wsum[1]) + (wsum[2] + wsum[3]));
        *f.counter = 0u;
    }
}

// Stand-alone clover application: out = G5^g (T x) on one parity (no hopping).
template <typename R, class SpinorT, class CloverT>
__global__ void clover_kernel(Geom g, SpinorT out, SpinorT in, CloverT T, int parity, int gamma5)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    cx<R> x[12], y[12];
    in.template load<R>(h, x);
    clover_apply<R>(T, parity, h, x, y);
    if (gamma5) {
#pragma unroll
        for (int k = 6; k < 12; ++k) y[k] = -y[k];
    }
    out.template store<R>(h, y);
}

}  // namespace lym
