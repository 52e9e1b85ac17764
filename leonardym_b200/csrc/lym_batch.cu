// Dispatcher over the batched stencil instantiations (lym_batch.cuh).  The batched path
// reads FP32 links without reconstruction whatever the spinor storage (FP32 or FP16):
// link bytes are shared by the batch.
#include "lym_batch.cuh"
#include "lym_internal.h"

namespace lym {

static SpinorFB fview(const SpinorBatch &s) { return SpinorFB{(float4 *)s.v, s.stride, s.lognb}; }
static SpinorHB hview(const SpinorBatch &s) { return SpinorHB{(int4 *)s.v, s.norm, s.stride, s.lognb}; }

template <typename R, class SB, class G, class C>
static void run(const DslashBatchParams &P, const SB &in, const SB &out, const SB &y, const G &U, const C &T,
                cudaStream_t st)
{
    DslashBatchArg<SB, G, C> a{P.g,       in,        out,       y,          U,         T,       P.parity, P.gamma5,
                               P.clover != nullptr,  in.lognb,  P.a,        P.b,       NbrTable{P.nbr, P.g.stride},
                               P.skip_if, P.active,  P.b_slot,  P.clover_slot};
    const long threads = (long)P.g.Vh << in.lognb;
    const int nb = (int)((threads + 127) / 128);
    switch (P.epi) {
    case EPI_SCALE_: dslash_batch_kernel<R, EPI_SCALE><<<nb, 128, 0, st>>>(a); break;
    case EPI_CLOVINV_: dslash_batch_kernel<R, EPI_CLOVINV><<<nb, 128, 0, st>>>(a); break;
    default: dslash_batch_kernel<R, EPI_XPAY><<<nb, 128, 0, st>>>(a); break;
    }
}

void launch_dslash_batch(const DslashBatchParams &P, cudaStream_t st)
{
    const GaugeDev &U = *P.U;
    const int s = P.g.stride;
    if (P.prec == PREC_F) {
        CloverF T{(const float4 *)P.clover, s};
        if (P.rep == REP_SU3)
            run<float>(P, fview(P.in), fview(P.out), fview(P.y), GaugeF18{(const float2 *)U.f32full, s}, T, st);
        else
            run<float>(P, fview(P.in), fview(P.out), fview(P.y), GaugeF9{(const float *)U.f32full, s}, T, st);
    } else {
        CloverH T{(const uint2 *)P.clover, s};
        if (P.rep == REP_SU3)
            run<float>(P, hview(P.in), hview(P.out), hview(P.y), GaugeF18{(const float2 *)U.f32full, s}, T, st);
        else
            run<float>(P, hview(P.in), hview(P.out), hview(P.y), GaugeF9{(const float *)U.f32full, s}, T, st);
    }
}

}  // namespace lym
