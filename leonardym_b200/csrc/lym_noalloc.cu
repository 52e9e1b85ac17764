// Even-odd operator application that allocates no device memory.
//
// Some callers cannot call cudaMalloc: processes that hand all of their device memory
// to one arena or framework allocator up front (a solve server that has reserved its
// HBM budget and accounts every byte of it), and code on a latency-critical path that
// must not add cudaMalloc / cudaFree calls, which synchronise the whole device.  For
// them lym_multiply_device_noalloc applies EvenOddImprovedDiracWilsonOperator::multiply
// (EvenOddImprovedDiracWilsonOperator.cpp:26-47) to caller-owned device vectors in the
// reference's layout; its one intermediate vector, the even-site half spinor
// T_ee^-1 H_eo x_o, lives in the file-scope array below instead of memory the library
// allocates.  The array is kNoallocMaxHalfSites (lym_internal.h) half-sites of FP64
// (12 MiB), held by every GPU that loads the library until the process exits.
#include <mutex>

#include "../../include/lym_b200.h"
#include "lym_dslash.cuh"
#include "lym_internal.h"

namespace lym {

static __device__ __align__(256) double2 g_noalloc_half_spinor[12 * kNoallocMaxHalfSites];

// A spinor of one parity read from / written to the reference's AoS layout
// (double[V][4][3][2]): half-site h of parity p is lexicographic site
// s = 2h + ((p + x + y + z) & 1), because s is even at t = 0 and t is the fastest index.
struct SpinorAoS {
    double2 *base;
    Geom g;
    int parity;
    LYM_D int site(int h) const
    {
        int r = (2 * h) / g.L[3];
        const int z = r % g.L[2];
        r /= g.L[2];
        const int y = r % g.L[1], x = r / g.L[1];
        return 2 * h + ((parity + x + y + z) & 1);
    }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
        const double2 *v = base + (size_t)site(h) * 12;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double2 w = __ldg(v + k);
            s[k] = cx<R>{(R)w.x, (R)w.y};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
        double2 *v = base + (size_t)site(h) * 12;
#pragma unroll
        for (int k = 0; k < 12; ++k) v[k] = make_double2((double)s[k].re, (double)s[k].im);
    }
};

// tmp = T_ee^-1 H_eo x_o, and the even sites of the output are those of the input
// (EvenOddImprovedDiracWilsonOperator.cpp:38-41), copied by the same threads
template <class GaugeT>
__global__ void noalloc_schur_even(Geom g, SpinorAoS in_odd, SpinorAoS in_even, SpinorAoS out_even, SpinorD tmp,
                                   GaugeT U, CloverD Tinv, int clover)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    cx<double> acc[12], res[12];
    in_even.load<double>(h, res);
    out_even.store<double>(h, res);
    hopping<double>(g, in_odd, U, 0, h, acc);
    if (clover) clover_apply<double>(Tinv, 0, h, acc, res);
    else
#pragma unroll
        for (int k = 0; k < 12; ++k) res[k] = acc[k];
    tmp.store<double>(h, res);
}

template <class GaugeT>
__global__ void noalloc_schur_odd(Geom g, SpinorD tmp, SpinorAoS in_odd, SpinorAoS out_odd, GaugeT U, CloverD T,
                                  int clover, double kappa2, int gamma5)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    cx<double> acc[12], y[12], res[12];
    hopping<double>(g, tmp, U, 1, h, acc);
    in_odd.load<double>(h, y);
    if (clover) clover_apply<double>(T, 1, h, y, res);
    else
#pragma unroll
        for (int k = 0; k < 12; ++k) res[k] = y[k];
#pragma unroll
    for (int k = 0; k < 12; ++k) fma_r(res[k], -kappa2, acc[k]);
    if (gamma5)
#pragma unroll
        for (int k = 6; k < 12; ++k) res[k] = -res[k];
    out_odd.store<double>(h, res);
}

// Device address of the scratch array on the current device, looked up once per device.
static double2 *scratch_address(int device, cudaError_t *err)
{
    static std::mutex mu;
    static double2 *addr[64] = {nullptr};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    if (!addr[device]) {
        void *p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_half_spinor);
        if (*err != cudaSuccess) return nullptr;
        addr[device] = (double2 *)p;
    }
    *err = cudaSuccess;
    return addr[device];
}

int noalloc_schur(const Geom &g, int rep, int device, cudaStream_t st, const GaugeDev &U, const CloverDev *C,
                  double kappa, int gamma5, double *out, const double *in, cudaError_t *cuda_err)
{
    *cuda_err = cudaSuccess;
    if (g.Vh > kNoallocMaxHalfSites) return LYM_ERR_ARGUMENT;
    double2 *scratch = scratch_address(device, cuda_err);
    if (!scratch) return LYM_ERR_CUDA;
    SpinorAoS in_odd{(double2 *)in, g, 1}, out_odd{(double2 *)out, g, 1};
    SpinorAoS in_even{(double2 *)in, g, 0}, out_even{(double2 *)out, g, 0};
    SpinorD tmp{scratch, kNoallocMaxHalfSites};
    const int clover = C != nullptr;
    CloverD T{clover ? (const double2 *)C->T[PREC_D] : nullptr, g.stride};
    CloverD Ti{clover ? (const double2 *)C->Tinv[PREC_D] : nullptr, g.stride};
    const int nb = (g.Vh + 127) / 128;
    if (rep == REP_SU3) {
        GaugeD18 G{(const double2 *)U.d64, g.stride};
        noalloc_schur_even<<<nb, 128, 0, st>>>(g, in_odd, in_even, out_even, tmp, G, Ti, clover);
        noalloc_schur_odd<<<nb, 128, 0, st>>>(g, tmp, in_odd, out_odd, G, T, clover, kappa * kappa, gamma5);
    } else {
        GaugeD9 G{(const double *)U.d64, g.stride};
        noalloc_schur_even<<<nb, 128, 0, st>>>(g, in_odd, in_even, out_even, tmp, G, Ti, clover);
        noalloc_schur_odd<<<nb, 128, 0, st>>>(g, tmp, in_odd, out_odd, G, T, clover, kappa * kappa, gamma5);
    }
    *cuda_err = cudaGetLastError();
    return *cuda_err == cudaSuccess ? LYM_OK : LYM_ERR_CUDA;
}

}  // namespace lym
