// Dispatcher over the batched stencil instantiations (lym_batch.cuh) and the traversal
// tables the autotuner chooses between.
#include "lym_batch.cuh"
#include "lym_internal.h"

namespace lym {

// Compiled variants of the batched stencil: the register budget the compiler is held to
// (__launch_bounds__(128, minb)) for the direct-load kernel (codes 1, 3, 4), the same for
// the kernel that stages neighbour spinors in shared memory with per-thread cp.async
// (codes 16 + minb: 19, 20), the same reading SU(3) links in all 18 reals (codes 64 + 19,
// 20: 83, 84; as 19, 20 for the adjoint representation) and the one that stages the
// spinors with bulk copies completing on mbarriers (codes 32 + minb: 35, 36; FP32 batches,
// else as 19, 20).  The autotuner times the first kBatchTunedCount; the bulk-copy kernel is
// selected only by lym_set_batch_tile (on 24^3 x 48 with 16 right-hand sides it takes 829
// us per launch against 434 us for the cp.async kernel: one 16 np-byte copy per spinor
// component costs more to issue than the per-thread 16-byte copies it replaces).
const int kBatchMinBlocks[] = {1, 3, 4, 19, 20, 83, 84, 35, 36};
const int kBatchMinBlocksCount = 9;
const int kBatchTunedCount = 7;

template <int EPI, int MINB, bool BULK = false, class SB, class G>
static void launch_staged(const DslashBatchArg<SB, G> &a, int nblk, cudaStream_t st)
{
    constexpr bool BK = BULK && std::is_same<SB, BatchF>::value;  // FP16 batches: the cp.async kernel
    static bool attr = false;  // the shared-memory limit above 48 KB, once per instantiation
    const int bytes = staged_smem_bytes(a.lognp);
    if (!attr) {
        cudaFuncSetAttribute(dslash_batch_staged_kernel<EPI, MINB, BK, SB, G>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, staged_smem_bytes(0));
        attr = true;
    }
    dslash_batch_staged_kernel<EPI, MINB, BK><<<nblk, kStagedThreads, bytes, st>>>(a);
}

static BatchF fview(const SpinorBatch &s) { return BatchF{(float4 *)s.v, s.stride, s.lognb - 1}; }
static BatchH hview(const SpinorBatch &s) { return BatchH{(int4 *)s.v, (float2 *)s.norm, s.stride, s.lognb - 1}; }
static void view_as(const SpinorBatch &s, BatchF &v) { v = s.v ? fview(s) : BatchF{}; }
static void view_as(const SpinorBatch &s, BatchH &v) { v = s.v ? hview(s) : BatchH{}; }

template <int EPI, class SB, class G>
static void launch_minb(const DslashBatchParams &P, const DslashBatchArg<SB, G> &a, cudaStream_t st)
{
    const long threads = (long)P.g.Vh << a.lognp;
    const int nb = (int)((threads + 127) / 128);
    switch (P.minb) {
    case 3: dslash_batch_kernel<EPI, 3><<<nb, 128, 0, st>>>(a); break;
    case 4: dslash_batch_kernel<EPI, 4><<<nb, 128, 0, st>>>(a); break;
    case 19: launch_staged<EPI, 3>(a, nb, st); break;
    case 20: launch_staged<EPI, 4>(a, nb, st); break;
    case 35: launch_staged<EPI, 3, true>(a, nb, st); break;
    case 36: launch_staged<EPI, 4, true>(a, nb, st); break;
    default: dslash_batch_kernel<EPI, 1><<<nb, 128, 0, st>>>(a); break;
    }
}

static unsigned walk_magic(int d) { return d == 1 ? 0u : (unsigned)(((1ull << 32) + d - 1) / d); }

// the arithmetic walk of the traversal (by, bz) when its divisions are exact (ColumnWalk)
ColumnWalk column_walk(const Geom &g, int by, int bz)
{
    ColumnWalk w{};
    if (by == 0) {  // h order: one column of Ly x Lz
        by = g.L[1];
        bz = g.L[2];
    }
    if (bz < 1 || by < 1 || g.L[1] % by || g.L[2] % bz || g.L[3] % 2 || g.Vh >= (1 << 24)) return w;
    const int div[5] = {g.L[3] / 2, bz, by, g.L[0], g.L[2] / bz};
    for (int d : div)
        if (d < 1 || d > 256) return w;
    for (int k = 0; k < 4; ++k) w.L[k] = g.L[k];
    w.lth = div[0];
    w.bz = bz;
    w.by = by;
    w.nzb = div[4];
    w.m_lth = walk_magic(div[0]);
    w.m_bz = walk_magic(bz);
    w.m_by = walk_magic(by);
    w.m_lx = walk_magic(g.L[0]);
    w.m_nzb = walk_magic(div[4]);
    w.on = 1;
    return w;
}

template <class SB, class G>
static void run(const DslashBatchParams &P, const SB &in, const SB &out, const SB &y, const G &U, cudaStream_t st)
{
    SB res_s;
    view_as(P.res_s, res_s);
    DslashBatchArg<SB, G> a{P.g,       in,          out,       y,         U,
                            P.parity,  P.gamma5,    P.has_clover, in.lognp, (float)P.a,
                            (float)P.b, NbrTable{P.nbr, P.g.stride}, P.order, P.skip_if, P.active,
                            P.b_slot,  P.clover_slot, P.uniform, P.res_r.v ? fview(P.res_r) : BatchF{},
                            res_s,     P.res_alpha, P.om_rhat.v ? fview(P.om_rhat) : BatchF{}, P.om_partials,
                            column_walk(P.g, P.walk_by, P.walk_bz), P.err};
    switch (P.epi) {
    case EPI_SCALE_: launch_minb<EPI_SCALE>(P, a, st); break;
    case EPI_CLOVINV_: launch_minb<EPI_CLOVINV>(P, a, st); break;
    case EPI_XPAY_RES_: launch_minb<EPI_XPAY_RES>(P, a, st); break;
    case EPI_XPAY_OMEGA_: {  // staged variants only (batch_omega_fusable)
        const int nblk = (int)batch_stencil_blocks(P.g, in.lognp + 1);
        switch (P.minb) {
        case 19: launch_staged<EPI_XPAY_OMEGA, 3>(a, nblk, st); break;
        case 35: launch_staged<EPI_XPAY_OMEGA, 3, true>(a, nblk, st); break;
        case 36: launch_staged<EPI_XPAY_OMEGA, 4, true>(a, nblk, st); break;
        default: launch_staged<EPI_XPAY_OMEGA, 4>(a, nblk, st); break;
        }
        break;
    }
    default: launch_minb<EPI_XPAY>(P, a, st); break;
    }
}

// The omega sums of the staged stencil's blocks (EPI_XPAY_OMEGA), [block][nb][7], added in a
// fixed order: kOmegaChunks blocks each add a fixed range of stencil blocks, then one block per
// RHS adds the chunk sums and applies omega_finalize.
constexpr int kOmegaThreads = 256;
constexpr int kOmegaChunks = 256;
__global__ void __launch_bounds__(kOmegaThreads) omega_chunk_kernel(const double *partials, int nblk, int nb,
                                                                    double *chunks, const BatchCGState *S)
{
    if (S->pause) return;
    const int w = nb * 7, j = threadIdx.x;
    if (j >= w) return;
    const long per = (nblk + kOmegaChunks - 1) / kOmegaChunks;
    const long b0 = blockIdx.x * per, b1 = min((long)nblk, b0 + per);
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    long b = b0;
    for (; b + 4 <= b1; b += 4) {
        t0 += __ldcg(partials + b * w + j);
        t1 += __ldcg(partials + (b + 1) * w + j);
        t2 += __ldcg(partials + (b + 2) * w + j);
        t3 += __ldcg(partials + (b + 3) * w + j);
    }
    for (; b < b1; ++b) t0 += __ldcg(partials + b * w + j);
    chunks[(long)blockIdx.x * w + j] = (t0 + t1) + (t2 + t3);
}

__global__ void __launch_bounds__(kOmegaThreads) omega_finalize_kernel(const double *chunks, int nb, BatchCGState *S)
{
    if (S->pause) return;
    __shared__ double sm[kOmegaThreads][7];
    const int r = blockIdx.x, w = nb * 7;
    double t[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < kOmegaChunks; b += blockDim.x)
#pragma unroll
        for (int j = 0; j < 7; ++j) t[j] += chunks[(long)b * w + r * 7 + j];
#pragma unroll
    for (int j = 0; j < 7; ++j) sm[threadIdx.x][j] = t[j];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
#pragma unroll
            for (int j = 0; j < 7; ++j) sm[threadIdx.x][j] += sm[threadIdx.x + o][j];
        __syncthreads();
    }
    if (threadIdx.x == 0) omega_finalize(S, r, sm[0]);
}

bool batch_omega_fusable(int minb, int prec)
{
    const int m = minb & ~64;
    return prec == PREC_F && (m == 19 || m == 20 || m == 35 || m == 36);
}

long omega_scratch_doubles(const Geom &g, int lognb)
{
    return (batch_stencil_blocks(g, lognb) + kOmegaChunks) * (7L << lognb);
}

void launch_omega_finalize(double *scratch, const Geom &g, int lognb, void *state, cudaStream_t st)
{
    const long nblk = batch_stencil_blocks(g, lognb);
    const int nb = 1 << lognb;
    double *chunks = scratch + nblk * 7 * nb;
    omega_chunk_kernel<<<kOmegaChunks, kOmegaThreads, 0, st>>>(scratch, (int)nblk, nb, chunks, (BatchCGState *)state);
    omega_finalize_kernel<<<nb, kOmegaThreads, 0, st>>>(chunks, nb, (BatchCGState *)state);
}

void launch_dslash_batch(const DslashBatchParams &P0, cudaStream_t st)
{
    // variant bit 64: SU(3) links read in all 18 reals; the kernel variant is the code without it
    DslashBatchParams P = P0;
    const bool f18 = (P.minb & 64) && P.rep == REP_SU3 && P.U->f32r18;
    P.minb &= ~64;
    const GaugeDev &U = *P.U;
    const int s = P.g.stride;
    const GaugeC12P c12{(const float4 *)U.f32, U.sign, s};
    const GaugeF18P l18{(const float4 *)U.f32r18, s};
    const GaugeR6P r6{(const float2 *)U.f32, U.sign, s};
    if (P.prec == PREC_F) {
        if (P.rep != REP_SU3) run(P, fview(P.in), fview(P.out), fview(P.y), r6, st);
        else if (f18) run(P, fview(P.in), fview(P.out), fview(P.y), l18, st);
        else run(P, fview(P.in), fview(P.out), fview(P.y), c12, st);
    } else {
        if (P.rep != REP_SU3) run(P, hview(P.in), hview(P.out), hview(P.y), r6, st);
        else if (f18) run(P, hview(P.in), hview(P.out), hview(P.y), l18, st);
        else run(P, hview(P.in), hview(P.out), hview(P.y), c12, st);
    }
}

// Work item w -> half-site h for a column (by, bz): the lattice is walked in columns of
// by * bz sites of the (y, z) plane, each column with x, then y, z inside the column
// and t fastest, i.e. in the order (y block, z block, x, y, z, t / 2).  Consecutive
// items are consecutive half-sites along t (coalesced), and the x neighbours of a site
// are by * bz * Lt / 2 items away, so they are still in L2 when they are read again.
// The half-site index h = t / 2 + Lt / 2 * (z + Lz * (y + Ly * x)) does not depend on
// the parity, so one table serves both.
__global__ void order_table_kernel(Geom g, int by, int bz, int *order)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= g.Vh) return;
    const int lth = g.L[3] / 2;
    int u = w;
    const int th = u % lth;
    u /= lth;
    const int zi = u % bz;
    u /= bz;
    const int yi = u % by;
    u /= by;
    const int x = u % g.L[0];
    u /= g.L[0];
    const int nzb = g.L[2] / bz;
    const int zb = u % nzb, yb = u / nzb;
    const int y = yb * by + yi, z = zb * bz + zi;
    order[w] = th + lth * (z + g.L[2] * (y + g.L[1] * x));
}

void launch_order_table(const Geom &g, int by, int bz, int *order, cudaStream_t st)
{
    order_table_kernel<<<(g.Vh + 127) / 128, 128, 0, st>>>(g, by, bz, order);
}

}  // namespace lym
