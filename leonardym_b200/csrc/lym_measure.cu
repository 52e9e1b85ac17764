// Consumers of the propagator solves, on the device: the connected meson contractions of
// MesonCorrelator::execute (correlators/MesonCorrelator.cpp:98-157) and the noise dot
// products of ChiralCondensate::execute (fermion_measurements/ChiralCondensate.cpp:92-105).
// Inputs are spinors in the reference's AoS layout (double2[V][4][3], site
// t + Lt (z + Lz (y + Ly x))) already in device memory, e.g. the solutions of
// lym_solve_block_device.  Every sum is reduced in a fixed order (per-site or per-block
// values first, then one block per output), so results do not depend on scheduling.
#include <algorithm>

#include "../../include/lym_b200.h"
#include "lym_internal.h"

namespace lym {

namespace {

constexpr int kMeasThreads = 256;

// gamma_t and gamma5 gamma_t of the chiral basis (the basis of the projections in
// DiracWilsonOperator.cpp:25-190): gamma_t = [[0, 1], [1, 0]], gamma5 = diag(1, -1) in
// 2x2 spin blocks.  Both are signed permutations: row a has its one entry in column a ^ 2,
// 1 for gamma_t, +1 (a < 2) or -1 (a >= 2) for gamma5 gamma_t.
__host__ __device__ constexpr int spin_perm(int a) { return a ^ 2; }
__host__ __device__ constexpr double sign_g5gt(int a) { return a < 2 ? 1.0 : -1.0; }

__device__ __forceinline__ double re_conj_mul(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

// one site: pion = sum_k |S_k|^2; scalar = sum Re g5gt(mu,nu) g5gt(a,b) conj(S_{ca}[mu]) S_{cb}[nu];
// ps = sum Re gt(a,b) (conj(S_{cmu}[a]) S_{cmu}[b] - conj(S_{ca}[mu]) S_{cb}[mu]); S_{ca} the
// propagator of the point source with spin a, colour c (index c * 4 + a)
__global__ void __launch_bounds__(kMeasThreads) meson_site_kernel(MesonProps P, int V, double *out)
{
    const int site = blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= V) return;
    double pion = 0.0, sc = 0.0, ps = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll 1
        for (int d = 0; d < 3; ++d) {
            double2 S[4][4];  // [source spin a][sink spin mu] of colour component d
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double2 *p = P.p[c * 4 + a] + (size_t)site * 12 + d;
#pragma unroll
                for (int mu = 0; mu < 4; ++mu) S[a][mu] = __ldg(p + 3 * mu);
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) {
#pragma unroll
                for (int mu = 0; mu < 4; ++mu) {
                    pion += re_conj_mul(S[a][mu], S[a][mu]);
                    sc += sign_g5gt(a) * sign_g5gt(mu) * re_conj_mul(S[a][mu], S[spin_perm(a)][spin_perm(mu)]);
                    ps += re_conj_mul(S[mu][a], S[mu][spin_perm(a)]) - re_conj_mul(S[a][mu], S[spin_perm(a)][mu]);
                }
            }
        }
    }
    out[3 * (size_t)site + 0] = pion;
    out[3 * (size_t)site + 1] = sc;
    out[3 * (size_t)site + 2] = ps;
}

// per time slice: block t sums the per-site values of the sites with t(site) = t (site % Lt)
__global__ void __launch_bounds__(kMeasThreads) time_slice_sum_kernel(const double *per_site, int V, int Lt,
                                                                      int nval, double *result)
{
    __shared__ double red[kMeasThreads];
    const int t = blockIdx.x;
    const int n = V / Lt;
    for (int k = 0; k < nval; ++k) {
        double s = 0.0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) s += per_site[((size_t)j * Lt + t) * nval + k];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) result[(size_t)k * Lt + t] = red[0];
        __syncthreads();
    }
}

// <a_k, b_k> (gamma5 = 0) or <a_k, gamma5 b_k> (gamma5 = 1) over full AoS spinors: blocks of
// grid.x sites for vector k = blockIdx.y write partial sums; dot_finish_kernel adds them
__global__ void __launch_bounds__(kMeasThreads) dot_partial_kernel(DotPairs D, int V, int gamma5, double2 *partials)
{
    __shared__ double2 red[kMeasThreads];
    const int k = blockIdx.y;
    const double2 *a = D.a[k], *b = D.b[k];
    double2 acc = make_double2(0.0, 0.0);
    const long n = (long)V * 12;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double2 x = __ldg(a + i), y = __ldg(b + i);
        const double sgn = (gamma5 && ((i % 12) >= 6)) ? -1.0 : 1.0;  // spins 2, 3
        acc.x += sgn * (x.x * y.x + x.y * y.y);
        acc.y += sgn * (x.x * y.y - x.y * y.x);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            red[threadIdx.x].x += red[threadIdx.x + o].x;
            red[threadIdx.x].y += red[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[(size_t)k * gridDim.x + blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kMeasThreads) dot_finish_kernel(const double2 *partials, int nblk, double2 *out)
{
    __shared__ double2 red[kMeasThreads];
    const int k = blockIdx.x;
    double2 s = make_double2(0.0, 0.0);
    for (int j = threadIdx.x; j < nblk; j += blockDim.x) {
        s.x += partials[(size_t)k * nblk + j].x;
        s.y += partials[(size_t)k * nblk + j].y;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            red[threadIdx.x].x += red[threadIdx.x + o].x;
            red[threadIdx.x].y += red[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = red[0];
}

// Real Z2 noise (entries +-1, imaginary part 0) for every spin-colour component, as
// StochasticEstimator::generateRandomNoise (StochasticEstimator.h:16-31) draws it, from a
// counter-based generator instead of a time-seeded one: component j of noise vector
// `stream` is the sign bit of splitmix64(seed + golden * (stream * 12 V + j + 1)) (Steele,
// Lea and Flood's SplitMix64 finaliser), so every (seed, stream) gives the same vector.
__device__ __forceinline__ unsigned long long splitmix64_mix(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(kMeasThreads) z2_noise_kernel(double2 *out, long n, unsigned long long seed,
                                                                unsigned long long stream)
{
    for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
        const unsigned long long z =
            splitmix64_mix(seed + 0x9E3779B97F4A7C15ull * (stream * (unsigned long long)n + (unsigned long long)j + 1ull));
        out[j] = make_double2((z >> 63) ? 1.0 : -1.0, 0.0);
    }
}

}  // namespace

void launch_z2_noise(const Geom &g, double *out, unsigned long long seed, unsigned long long stream, cudaStream_t st)
{
    const long n = (long)g.V * 12;
    const int grid = (int)std::min<long>((n + kMeasThreads - 1) / kMeasThreads, 8 * 148);
    z2_noise_kernel<<<grid, kMeasThreads, 0, st>>>((double2 *)out, n, seed, stream);
}

size_t meson_scratch_bytes(const Geom &g) { return (size_t)g.V * 3 * sizeof(double); }

void launch_meson_contractions(const Geom &g, const MesonProps &P, double *scratch, double *result, cudaStream_t st)
{
    meson_site_kernel<<<(g.V + kMeasThreads - 1) / kMeasThreads, kMeasThreads, 0, st>>>(P, g.V, scratch);
    time_slice_sum_kernel<<<g.L[3], kMeasThreads, 0, st>>>(scratch, g.V, g.L[3], 3, result);
}

int dot_blocks(const Geom &g) { return std::min((g.V * 12 + kMeasThreads - 1) / kMeasThreads, 2 * 148); }

void launch_dots(const Geom &g, const DotPairs &D, int n, int gamma5, double2 *partials, double2 *out,
                 cudaStream_t st)
{
    const int nblk = dot_blocks(g);
    dot_partial_kernel<<<dim3(nblk, n), kMeasThreads, 0, st>>>(D, g.V, gamma5, partials);
    dot_finish_kernel<<<n, kMeasThreads, 0, st>>>(partials, nblk, out);
}

}  // namespace lym
