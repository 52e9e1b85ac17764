// Fused per-site vector kernels with deterministic global reductions.
//
// Every solver step is one launch of site_kernel<Op>: Op::site() updates the 12
// complex components of one half-site (any storage precision, through the spinor
// views) and adds its contribution to up to NRED FP64 partial sums.  Partial
// sums of each block land in a fixed slot; the last block to finish sums the
// slots in a fixed order and calls Op::finalize() with the totals, which runs the
// scalar recurrences of the solver (FP64) in device memory.  No atomics touch
// the sums, so results are bitwise reproducible run to run.
#pragma once

#include "lym_common.cuh"

namespace lym {

constexpr int kBlasThreads = 256;
constexpr int kMaxRed = 8;

struct RedBuf {
    double *partials;        // [gridDim.x][kMaxRed]
    unsigned int *counter;   // zero between launches
};

template <int N>
LYM_D void block_sum(double v[N], double *smem /* [kBlasThreads/32][N] */)
{
#pragma unroll
    for (int k = 0; k < N; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        v[k] = x;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) smem[warp * N + k] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double x = lane < nw ? smem[lane * N + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

// Skip gates: a kernel does nothing when *skip_if != 0 or (run_if && *run_if == 0).
struct Gate {
    const int *skip_if;
    const int *run_if;
    LYM_D bool closed() const { return (skip_if && *skip_if) || (run_if && !*run_if); }
};

template <class Op>
__global__ void __launch_bounds__(kBlasThreads) site_kernel(Op op, int vh, int nparity, RedBuf rb, Gate gate)
{
    if (gate.closed()) return;
    double acc[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int k = 0; k < (Op::NRED > 0 ? Op::NRED : 1); ++k) acc[k] = 0.0;
    for (int p = 0; p < nparity; ++p)
        for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < vh; h += gridDim.x * blockDim.x) op.site(p, h, acc);
    if constexpr (Op::NRED > 0) {
        __shared__ double smem[(kBlasThreads / 32) * kMaxRed];
        __shared__ bool last;
        block_sum<Op::NRED>(acc, smem);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < Op::NRED; ++k) rb.partials[blockIdx.x * kMaxRed + k] = acc[k];
            __threadfence();
            unsigned int ticket = atomicAdd(rb.counter, 1u);
            last = (ticket == gridDim.x - 1);
        }
        __syncthreads();
        if (last) {
            __threadfence();
            double tot[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
            for (int k = 0; k < Op::NRED; ++k) tot[k] = 0.0;
            for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
                for (int k = 0; k < Op::NRED; ++k) tot[k] += ((volatile double *)rb.partials)[b * kMaxRed + k];
            block_sum<Op::NRED>(tot, smem);
            if (threadIdx.x == 0) {
                op.finalize(tot);
                *rb.counter = 0u;
            }
        }
    } else {
        (void)rb;
    }
}

// ------------------------------------------------------------------ helpers --
template <typename R> LYM_D double norm2(const cx<R> v[12])
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 12; ++k) s += (double)v[k].re * (double)v[k].re + (double)v[k].im * (double)v[k].im;
    return s;
}
// sum conj(a) b
template <typename R> LYM_D void dotc(const cx<R> a[12], const cx<R> b[12], double &re, double &im)
{
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        re += (double)a[k].re * (double)b[k].re + (double)a[k].im * (double)b[k].im;
        im += (double)a[k].re * (double)b[k].im - (double)a[k].im * (double)b[k].re;
    }
}

LYM_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
LYM_HD double2 cdiv(double2 a, double2 b)
{
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
LYM_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
LYM_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
LYM_HD double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

}  // namespace lym
