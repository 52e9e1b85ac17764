// Common device types for the B200 Wilson-clover library.
//
// Data layout in HBM (one lattice geometry per context):
//   * sites are split by parity p = (x+y+z+t) & 1; inside a parity the half-site
//     index is h = s >> 1, where s = t + Lt*(z + Lz*(y + Ly*x)) is the reference's
//     lexicographic index (MPILattice/LocalLayout.h:149-163).  This requires Lt even.
//   * every field is struct-of-arrays over h with a padded stride, so a warp's
//     32 consecutive half-sites read 32 consecutive vector words (coalesced).
//   * a full-lattice spinor is [parity][word][stride]; a half spinor is one parity.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define LYM_HD __host__ __device__ __forceinline__
#define LYM_D __device__ __forceinline__

namespace lym {

// ---------------------------------------------------------------- complex --
template <typename R>
struct cx {
    R re, im;
};

template <typename R> LYM_HD cx<R> mk(R a, R b) { return cx<R>{a, b}; }
template <typename R> LYM_HD cx<R> operator+(cx<R> a, cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> LYM_HD cx<R> operator-(cx<R> a, cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R> LYM_HD cx<R> operator-(cx<R> a) { return {-a.re, -a.im}; }
template <typename R> LYM_HD cx<R> operator*(cx<R> a, cx<R> b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> LYM_HD cx<R> operator*(R s, cx<R> a) { return {s * a.re, s * a.im}; }
template <typename R> LYM_HD cx<R> operator*(cx<R> a, R s) { return {s * a.re, s * a.im}; }
template <typename R> LYM_HD cx<R> conj(cx<R> a) { return {a.re, -a.im}; }
template <typename R> LYM_HD cx<R> times_i(cx<R> a) { return {-a.im, a.re}; }
template <typename R> LYM_HD cx<R> times_mi(cx<R> a) { return {a.im, -a.re}; }
// a += b * c
template <typename R> LYM_HD void fma_c(cx<R> &a, cx<R> b, cx<R> c)
{
    a.re = fma(b.re, c.re, a.re);
    a.re = fma(-b.im, c.im, a.re);
    a.im = fma(b.re, c.im, a.im);
    a.im = fma(b.im, c.re, a.im);
}
// a += conj(b) * c
template <typename R> LYM_HD void fma_cc(cx<R> &a, cx<R> b, cx<R> c)
{
    a.re = fma(b.re, c.re, a.re);
    a.re = fma(b.im, c.im, a.re);
    a.im = fma(b.re, c.im, a.im);
    a.im = fma(-b.im, c.re, a.im);
}
// a += s * c for real s
template <typename R> LYM_HD void fma_r(cx<R> &a, R s, cx<R> c)
{
    a.re = fma(s, c.re, a.re);
    a.im = fma(s, c.im, a.im);
}

// --------------------------------------------------------------- geometry --
struct Geom {
    int L[4];      // x, y, z, t extents
    int V;         // volume
    int Vh;        // V / 2
    int stride;    // padded Vh (multiple of 64)
};

// coordinates of half-site h of parity p
LYM_D void site_coords(const Geom &g, int h, int p, int c[4])
{
    int s0 = 2 * h;
    int t0 = s0 % g.L[3];
    int r = s0 / g.L[3];
    c[2] = r % g.L[2];
    r /= g.L[2];
    c[1] = r % g.L[1];
    c[0] = r / g.L[1];
    c[3] = t0 + ((p + c[0] + c[1] + c[2]) & 1);
}

LYM_HD int lex_of(const Geom &g, int x, int y, int z, int t)
{
    return g.L[3] * (g.L[2] * (g.L[1] * x + y) + z) + t;
}

// half-site index of the neighbour in direction mu (dir = +1 / -1)
LYM_D int neighbour_h(const Geom &g, const int c[4], int mu, int dir)
{
    int n[4] = {c[0], c[1], c[2], c[3]};
    int v = n[mu] + dir;
    if (v == g.L[mu]) v = 0;
    if (v < 0) v = g.L[mu] - 1;
    n[mu] = v;
    return lex_of(g, n[0], n[1], n[2], n[3]) >> 1;
}

// ---------------------------------------------------------- spinor fields --
// Three storage precisions; all expose load(h, cx<R>[12]) / store(h, cx<R>[12])
// where component k = spin * 3 + colour.

struct SpinorD {  // FP64: 12 x double2 words
    double2 *v;
    int stride;
    static constexpr int kWords = 12;
    LYM_HD SpinorD par(int p) const { return SpinorD{v + (size_t)p * 12 * stride, stride}; }
    // component k of half-site h (vector steps that stream one component at a time)
    LYM_D cx<double> get(int k, int h) const
    {
        const double2 w = __ldg(v + (size_t)k * stride + h);
        return cx<double>{w.x, w.y};
    }
    LYM_D void put(int k, int h, cx<double> s) const { v[(size_t)k * stride + h] = make_double2(s.re, s.im); }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            double2 w = __ldg(v + (size_t)k * stride + h);
            s[k] = cx<R>{(R)w.x, (R)w.y};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 12; ++k) v[(size_t)k * stride + h] = make_double2((double)s[k].re, (double)s[k].im);
    }
};

struct SpinorF {  // FP32: 6 x float4 words (two complex per word)
    float4 *v;
    int stride;
    static constexpr int kWords = 6;
    LYM_HD SpinorF par(int p) const { return SpinorF{v + (size_t)p * 6 * stride, stride}; }
    // component k of half-site h (vector steps that stream one component at a time)
    LYM_D cx<double> get(int k, int h) const
    {
        const float2 w = __ldg(reinterpret_cast<const float2 *>(v + (size_t)(k >> 1) * stride + h) + (k & 1));
        return cx<double>{w.x, w.y};
    }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float4 w = __ldg(v + (size_t)k * stride + h);
            s[2 * k] = cx<R>{(R)w.x, (R)w.y};
            s[2 * k + 1] = cx<R>{(R)w.z, (R)w.w};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
#pragma unroll
        for (int k = 0; k < 6; ++k)
            v[(size_t)k * stride + h] =
                make_float4((float)s[2 * k].re, (float)s[2 * k].im, (float)s[2 * k + 1].re, (float)s[2 * k + 1].im);
    }
};

// FP16 spinor with one FP32 norm per site: value = half * norm
// v / m for the FP16 storage of a site whose largest magnitude is m (|v| <= m): 1 / m
// overflows FP32 when m is subnormal (the far tail of a point-source solve on a large
// lattice), so such a site is first scaled by 2^64, exactly.
struct HalfScale {
    float pre, inv;
    LYM_D explicit HalfScale(float m)
    {
        pre = (m > 0.f && m < 1.17549435e-38f) ? 18446744073709551616.f : 1.f;
        inv = m > 0.f ? 1.0f / (m * pre) : 0.f;
    }
    LYM_D float operator()(float v) const { return (v * pre) * inv; }
};

struct SpinorH {
    int4 *v;       // 3 words of 8 halves
    float *norm;
    int stride;
    static constexpr int kWords = 3;
    LYM_HD SpinorH par(int p) const { return SpinorH{v + (size_t)p * 3 * stride, norm + (size_t)p * stride, stride}; }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
        const float nrm = __ldg(norm + h);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int4 w = __ldg(v + (size_t)k * stride + h);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&w);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float2 f = __half22float2(hp[j]);
                s[4 * k + j] = cx<R>{(R)(f.x * nrm), (R)(f.y * nrm)};
            }
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < 12; ++k) m = fmaxf(m, fmaxf(fabsf((float)s[k].re), fabsf((float)s[k].im)));
        const HalfScale sc(m);
        norm[h] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int4 w;
            __half2 *hp = reinterpret_cast<__half2 *>(&w);
#pragma unroll
            for (int j = 0; j < 4; ++j) hp[j] = __floats2half2_rn(sc((float)s[4 * k + j].re), sc((float)s[4 * k + j].im));
            v[(size_t)k * stride + h] = w;
        }
    }
};

// ------------------------------------------------------------ link fields --
// A link is held in registers as a 3x3 matrix of cx<R> (fundamental SU(3)) or R
// (adjoint SU(2): real orthogonal).  u[i][j] = U(i, j).

template <typename R> struct LinkC {
    cx<R> u[3][3];
};
template <typename R> struct LinkR {
    R u[3][3];
};

// y = U x  and  y = U^dagger x for the two link kinds
template <typename R> LYM_D void mul_u(const LinkC<R> &U, const cx<R> x[3], cx<R> y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cx<R> a = {0, 0};
#pragma unroll
        for (int j = 0; j < 3; ++j) fma_c(a, U.u[i][j], x[j]);
        y[i] = a;
    }
}
template <typename R> LYM_D void mul_ud(const LinkC<R> &U, const cx<R> x[3], cx<R> y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cx<R> a = {0, 0};
#pragma unroll
        for (int j = 0; j < 3; ++j) fma_cc(a, U.u[j][i], x[j]);
        y[i] = a;
    }
}
template <typename R> LYM_D void mul_u(const LinkR<R> &U, const cx<R> x[3], cx<R> y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cx<R> a = {0, 0};
#pragma unroll
        for (int j = 0; j < 3; ++j) fma_r(a, U.u[i][j], x[j]);
        y[i] = a;
    }
}
template <typename R> LYM_D void mul_ud(const LinkR<R> &U, const cx<R> x[3], cx<R> y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cx<R> a = {0, 0};
#pragma unroll
        for (int j = 0; j < 3; ++j) fma_r(a, U.u[j][i], x[j]);
        y[i] = a;
    }
}

// Gauge storage: [parity][mu][word][stride].  Parity p, direction mu, half-site h
// holds U_mu(x) for the site x = (p, h).  Reconstructed formats keep a sign byte
// per site (bit mu set: the link is -V with V in SU(3) / SO(3)), which is how the
// antiperiodic boundary condition folded into the links survives compression.

// FP64 complex, 18 reals (no reconstruction)
struct GaugeD18 {
    typedef LinkC<double> Link;
    const double2 *u;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const double2 *b = u + ((size_t)(p * 4 + mu) * 9) * stride + h;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            double2 w = __ldg(b + (size_t)k * stride);
            U.u[k / 3][k % 3] = cx<double>{w.x, w.y};
        }
    }
};

// FP64 real, 9 reals (adjoint, no reconstruction)
struct GaugeD9 {
    typedef LinkR<double> Link;
    const double *u;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const double *b = u + ((size_t)(p * 4 + mu) * 9) * stride + h;
#pragma unroll
        for (int k = 0; k < 9; ++k) U.u[k / 3][k % 3] = __ldg(b + (size_t)k * stride);
    }
};

// FP32 complex, 18 reals (no reconstruction; the batched stencil)
struct GaugeF18 {
    typedef LinkC<float> Link;
    const float2 *u;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const float2 *b = u + ((size_t)(p * 4 + mu) * 9) * stride + h;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const float2 w = __ldg(b + (size_t)k * stride);
            U.u[k / 3][k % 3] = cx<float>{w.x, w.y};
        }
    }
};

// FP32 real, 9 reals (adjoint, no reconstruction; the batched stencil)
struct GaugeF9 {
    typedef LinkR<float> Link;
    const float *u;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const float *b = u + ((size_t)(p * 4 + mu) * 9) * stride + h;
#pragma unroll
        for (int k = 0; k < 9; ++k) U.u[k / 3][k % 3] = __ldg(b + (size_t)k * stride);
    }
};

// Precomputed half-site indices of the 8 neighbours: nbr[(p*8 + 2 mu + dir)*stride + h],
// dir 0 = +mu, 1 = -mu (the same values neighbour_h computes; tested bit-exact).
struct NbrTable {
    const int *n;
    int stride;
    LYM_D int get(int p, int mu, int dir, int h) const { return __ldg(n + ((unsigned)(p * 8 + 2 * mu + dir) * stride + h)); }
};

// FP32 complex, 12 reals: rows 0 and 1; row 2 = sign * conj(row0 x row1)
struct GaugeF12 {
    typedef LinkC<float> Link;
    const float4 *u;
    const uint8_t *sign;  // [parity][stride]
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const float4 *b = u + ((size_t)(p * 4 + mu) * 3) * stride + h;
        float4 w0 = __ldg(b), w1 = __ldg(b + stride), w2 = __ldg(b + 2 * (size_t)stride);
        U.u[0][0] = {w0.x, w0.y};
        U.u[0][1] = {w0.z, w0.w};
        U.u[0][2] = {w1.x, w1.y};
        U.u[1][0] = {w1.z, w1.w};
        U.u[1][1] = {w2.x, w2.y};
        U.u[1][2] = {w2.z, w2.w};
        const float s = ((__ldg(sign + (size_t)p * stride + h) >> mu) & 1) ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            cx<float> v = U.u[0][a] * U.u[1][c] - U.u[0][c] * U.u[1][a];
            U.u[2][j] = s * conj(v);
        }
    }
};

// FP32 complex, 8 reals (SU(3) only): for V = s U in SU(3) (s from the sign table), the
// words (a2, a3) and (b1, arg a1, arg c1), with a, b, c the rows of V.  Rebuilt from the
// unitarity of V: |a1|^2 = 1 - |a2|^2 - |a3|^2 = 1 - N (row a), |c1|^2 = N - |b1|^2
// (column 1), and with a = conj(b x c) and the orthogonality of columns 1, 2 and 1, 3 the
// 2 x 2 systems for (b2, c2) and (b3, c3), whose determinants are -N and N:
//   b2 = -(conj(c1 a3) + conj(a1) a2 b1) / N,   c2 = (conj(b1 a3) - conj(a1) a2 c1) / N,
//   b3 =  (conj(c1 a2) - conj(a1) a3 b1) / N,   c3 = -(conj(b1 a2) + conj(a1) a3 c1) / N.
// N is 1 - |a1|^2, so the rounding of the rebuilt entries grows as |a1| nears 1.
struct GaugeF8 {
    typedef LinkC<float> Link;
    const float4 *u;      // [parity][mu][2][stride]
    const uint8_t *sign;  // [parity][stride]
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const float4 *b = u + ((size_t)(p * 4 + mu) * 2) * stride + h;
        const float4 w0 = __ldg(b), w1 = __ldg(b + stride);
        const cx<float> a2 = {w0.x, w0.y}, a3 = {w0.z, w0.w}, b1 = {w1.x, w1.y};
        const float N = w0.x * w0.x + w0.y * w0.y + w0.z * w0.z + w0.w * w0.w;
        float sa, ca, sc, cc;
        sincosf(w1.z, &sa, &ca);
        sincosf(w1.w, &sc, &cc);
        const float ra = sqrtf(fmaxf(1.f - N, 0.f)), rc = sqrtf(fmaxf(N - (b1.re * b1.re + b1.im * b1.im), 0.f));
        const cx<float> a1 = {ra * ca, ra * sa}, c1 = {rc * cc, rc * sc};
        const float inv = 1.f / N;
        const cx<float> t2 = conj(a1) * a2, t3 = conj(a1) * a3;
        const float s = ((__ldg(sign + (size_t)p * stride + h) >> mu) & 1) ? -1.f : 1.f;
        const float si = s * inv;
        U.u[0][0] = s * a1;
        U.u[0][1] = s * a2;
        U.u[0][2] = s * a3;
        U.u[1][0] = s * b1;
        U.u[2][0] = s * c1;
        U.u[1][1] = -si * (conj(c1 * a3) + t2 * b1);
        U.u[1][2] = si * (conj(c1 * a2) - t3 * b1);
        U.u[2][1] = si * (conj(b1 * a3) - t2 * c1);
        U.u[2][2] = -si * (conj(b1 * a2) + t3 * c1);
    }
};

// FP32 real, 6 reals (adjoint): rows 0 and 1; row 2 = sign * (row0 x row1)
struct GaugeF6 {
    typedef LinkR<float> Link;
    const float2 *u;
    const uint8_t *sign;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const float2 *b = u + ((size_t)(p * 4 + mu) * 3) * stride + h;
        float2 w0 = __ldg(b), w1 = __ldg(b + stride), w2 = __ldg(b + 2 * (size_t)stride);
        U.u[0][0] = w0.x;
        U.u[0][1] = w0.y;
        U.u[0][2] = w1.x;
        U.u[1][0] = w1.y;
        U.u[1][1] = w2.x;
        U.u[1][2] = w2.y;
        const float s = ((__ldg(sign + (size_t)p * stride + h) >> mu) & 1) ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            U.u[2][j] = s * (U.u[0][a] * U.u[1][c] - U.u[0][c] * U.u[1][a]);
        }
    }
};

// FP16 complex, 12 reals (|U_ij| <= 1, no norm needed)
struct GaugeH12 {
    typedef LinkC<float> Link;
    const uint2 *u;  // 3 words of 4 halves (rows 0 and 1)
    const uint8_t *sign;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const uint2 *b = u + ((size_t)(p * 4 + mu) * 3) * stride + h;
        float v[12];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            uint2 w = __ldg(b + (size_t)k * stride);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&w);
            float2 a = __half22float2(hp[0]), c = __half22float2(hp[1]);
            v[4 * k] = a.x;
            v[4 * k + 1] = a.y;
            v[4 * k + 2] = c.x;
            v[4 * k + 3] = c.y;
        }
        U.u[0][0] = {v[0], v[1]};
        U.u[0][1] = {v[2], v[3]};
        U.u[0][2] = {v[4], v[5]};
        U.u[1][0] = {v[6], v[7]};
        U.u[1][1] = {v[8], v[9]};
        U.u[1][2] = {v[10], v[11]};
        const float s = ((__ldg(sign + (size_t)p * stride + h) >> mu) & 1) ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            cx<float> w = U.u[0][a] * U.u[1][c] - U.u[0][c] * U.u[1][a];
            U.u[2][j] = s * conj(w);
        }
    }
};

// FP16 real, 6 reals (adjoint)
struct GaugeH6 {
    typedef LinkR<float> Link;
    const __half2 *u;  // 3 words of 2 halves
    const uint8_t *sign;
    int stride;
    LYM_D void load(int p, int mu, int h, Link &U) const
    {
        const __half2 *b = u + ((size_t)(p * 4 + mu) * 3) * stride + h;
        float2 w0 = __half22float2(b[0]), w1 = __half22float2(b[stride]), w2 = __half22float2(b[2 * (size_t)stride]);
        U.u[0][0] = w0.x;
        U.u[0][1] = w0.y;
        U.u[0][2] = w1.x;
        U.u[1][0] = w1.y;
        U.u[1][1] = w2.x;
        U.u[1][2] = w2.y;
        const float s = ((__ldg(sign + (size_t)p * stride + h) >> mu) & 1) ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            U.u[2][j] = s * (U.u[0][a] * U.u[1][c] - U.u[0][c] * U.u[1][a]);
        }
    }
};

// ---------------------------------------------------------- clover fields --
// T = 1 + kappa csw gamma5 C is block diagonal in the chiral basis: two Hermitian
// 6x6 blocks (spins 0,1 and spins 2,3).  Packed per block as 6 real diagonal
// entries followed by the 15 complex entries below the diagonal, row-major:
// (1,0) (2,0) (2,1) (3,0) ... (5,4).  36 reals per block, 72 per site.

LYM_HD int tri_index(int i, int j)  // i > j
{
    return i * (i - 1) / 2 + j;
}

template <typename R>
LYM_D void hermitian6_apply(const R diag[6], const cx<R> off[15], const cx<R> x[6], cx<R> y[6])
{
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = diag[i] * x[i];
#pragma unroll
    for (int i = 1; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < i; ++j) {
            const cx<R> a = off[tri_index(i, j)];
            fma_c(y[i], a, x[j]);
            fma_cc(y[j], a, x[i]);
        }
}

struct CloverD {  // FP64: per block 18 double2 words: 3 for the diagonal, 15 off-diagonal
    const double2 *c;  // [parity][2 blocks][18][stride]
    int stride;
    template <typename R> LYM_D void load_block(int p, int b, int h, R diag[6], cx<R> off[15]) const
    {
        const double2 *base = c + ((size_t)(p * 2 + b) * 18) * stride + h;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double2 w = __ldg(base + (size_t)k * stride);
            diag[2 * k] = (R)w.x;
            diag[2 * k + 1] = (R)w.y;
        }
#pragma unroll
        for (int k = 0; k < 15; ++k) {
            double2 w = __ldg(base + (size_t)(3 + k) * stride);
            off[k] = cx<R>{(R)w.x, (R)w.y};
        }
    }
};

struct CloverF {  // FP32: per block 9 float4 words
    const float4 *c;  // [parity][2][9][stride]
    int stride;
    template <typename R> LYM_D void load_block(int p, int b, int h, R diag[6], cx<R> off[15]) const
    {
        const float4 *base = c + ((size_t)(p * 2 + b) * 9) * stride + h;
        float v[36];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            float4 w = __ldg(base + (size_t)k * stride);
            v[4 * k] = w.x;
            v[4 * k + 1] = w.y;
            v[4 * k + 2] = w.z;
            v[4 * k + 3] = w.w;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) diag[k] = (R)v[k];
#pragma unroll
        for (int k = 0; k < 15; ++k) off[k] = cx<R>{(R)v[6 + 2 * k], (R)v[7 + 2 * k]};
    }
};

struct CloverH {  // FP16: per block 36 halves = 4.5 int4 -> stored as 9 words of 4 halves (uint2)
    const uint2 *c;  // [parity][2][9][stride]
    int stride;
    template <typename R> LYM_D void load_block(int p, int b, int h, R diag[6], cx<R> off[15]) const
    {
        const uint2 *base = c + ((size_t)(p * 2 + b) * 9) * stride + h;
        float v[36];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            uint2 w = __ldg(base + (size_t)k * stride);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&w);
            float2 a = __half22float2(hp[0]), c2 = __half22float2(hp[1]);
            v[4 * k] = a.x;
            v[4 * k + 1] = a.y;
            v[4 * k + 2] = c2.x;
            v[4 * k + 3] = c2.y;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) diag[k] = (R)v[k];
#pragma unroll
        for (int k = 0; k < 15; ++k) off[k] = cx<R>{(R)v[6 + 2 * k], (R)v[7 + 2 * k]};
    }
};

struct NoClover {
    template <typename R> LYM_D void load_block(int, int, int, R *, cx<R> *) const {}
};

}  // namespace lym
