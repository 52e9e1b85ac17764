// Device kernels: layout conversion, gauge upload / compression, clover build,
// and the dispatcher over the stencil instantiations.
#include "lym_blas.cuh"
#include "lym_dslash.cuh"
#include "lym_internal.h"
#include "lym_solver_ops.cuh"

namespace lym {

size_t Spinor::bytes_per_parity() const
{
    switch (prec) {
    case PREC_D: return (size_t)12 * stride * sizeof(double2);
    case PREC_F: return (size_t)6 * stride * sizeof(float4);
    default: return (size_t)3 * stride * sizeof(int4);
    }
}

Spinor Spinor::parity(int p) const
{
    Spinor s = *this;
    s.owned = false;
    s.nparity = 1;
    s.v = (char *)v + (size_t)p * bytes_per_parity();
    if (norm) s.norm = norm + (size_t)p * stride;
    return s;
}

static inline int nblocks(int n, int t) { return (n + t - 1) / t; }

// ----------------------------------------------------------------- layout --
LYM_D void lex_coords(const Geom &g, int s, int c[4])
{
    c[3] = s % g.L[3];
    int r = s / g.L[3];
    c[2] = r % g.L[2];
    r /= g.L[2];
    c[1] = r % g.L[1];
    c[0] = r / g.L[1];
}

template <class View>
__global__ void pack_kernel(Geom g, const double *aos, View v0, View v1)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    lex_coords(g, s, c);
    const int p = (c[0] + c[1] + c[2] + c[3]) & 1;
    cx<double> x[12];
    const double2 *src = reinterpret_cast<const double2 *>(aos) + (size_t)s * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        double2 w = src[k];
        x[k] = {w.x, w.y};
    }
    (p ? v1 : v0).template store<double>(s >> 1, x);
}

template <class View>
__global__ void unpack_kernel(Geom g, View v0, View v1, double *aos)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    lex_coords(g, s, c);
    const int p = (c[0] + c[1] + c[2] + c[3]) & 1;
    cx<double> x[12];
    (p ? v1 : v0).template load<double>(s >> 1, x);
    double2 *dst = reinterpret_cast<double2 *>(aos) + (size_t)s * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) dst[k] = make_double2(x[k].re, x[k].im);
}

void launch_pack(const Geom &g, const double *aos, const Spinor &full, cudaStream_t st)
{
    const int nb = nblocks(g.V, 128);
    if (full.prec == PREC_D) pack_kernel<<<nb, 128, 0, st>>>(g, aos, full.d(0), full.d(1));
    else if (full.prec == PREC_F) pack_kernel<<<nb, 128, 0, st>>>(g, aos, full.f(0), full.f(1));
    else pack_kernel<<<nb, 128, 0, st>>>(g, aos, full.h(0), full.h(1));
}

void launch_unpack(const Geom &g, const Spinor &full, double *aos, cudaStream_t st)
{
    const int nb = nblocks(g.V, 128);
    if (full.prec == PREC_D) unpack_kernel<<<nb, 128, 0, st>>>(g, full.d(0), full.d(1), aos);
    else if (full.prec == PREC_F) unpack_kernel<<<nb, 128, 0, st>>>(g, full.f(0), full.f(1), aos);
    else unpack_kernel<<<nb, 128, 0, st>>>(g, full.h(0), full.h(1), aos);
}

template <class Dst, class Src>
__global__ void convert_kernel(int vh, Dst d, Src s)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= vh) return;
    cx<double> x[12];
    s.template load<double>(h, x);
    d.template store<double>(h, x);
}

template <class Dst>
static void convert_from(const Geom &g, const Dst &d, const Spinor &src, int p, cudaStream_t st)
{
    const int nb = nblocks(g.Vh, 128);
    if (src.prec == PREC_D) convert_kernel<<<nb, 128, 0, st>>>(g.Vh, d, src.d(p));
    else if (src.prec == PREC_F) convert_kernel<<<nb, 128, 0, st>>>(g.Vh, d, src.f(p));
    else convert_kernel<<<nb, 128, 0, st>>>(g.Vh, d, src.h(p));
}

void launch_convert(const Geom &g, const Spinor &dst, const Spinor &src, cudaStream_t st)
{
    const int np = dst.nparity < src.nparity ? dst.nparity : src.nparity;
    for (int p = 0; p < np; ++p) {
        if (dst.prec == PREC_D) convert_from(g, dst.d(p), src, p, st);
        else if (dst.prec == PREC_F) convert_from(g, dst.f(p), src, p, st);
        else convert_from(g, dst.h(p), src, p, st);
    }
}

// ------------------------------------------------------------------ gauge --
// AoS input: per site 4 links, each N x N column-major (complex or real).
__global__ void upload_gauge_kernel(Geom g, int rep, const double *aos, void *d64)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    lex_coords(g, s, c);
    const int p = (c[0] + c[1] + c[2] + c[3]) & 1, h = s >> 1;
    for (int mu = 0; mu < 4; ++mu) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const size_t word = ((size_t)(p * 4 + mu) * 9 + i * 3 + j) * g.stride + h;
                if (rep == REP_SU3) {
                    const double2 *src = reinterpret_cast<const double2 *>(aos) + ((size_t)s * 4 + mu) * 9;
                    ((double2 *)d64)[word] = src[j * 3 + i];
                } else {
                    const double *src = aos + ((size_t)s * 4 + mu) * 9;
                    ((double *)d64)[word] = src[j * 3 + i];
                }
            }
    }
}

void launch_upload_gauge(const Geom &g, int rep, const double *aos, GaugeDev &U, cudaStream_t st)
{
    upload_gauge_kernel<<<nblocks(g.V, 128), 128, 0, st>>>(g, rep, aos, U.d64);
}

LYM_D void load_link_d(const Geom &g, int rep, const void *d64, int p, int mu, int h, cx<double> u[3][3])
{
    for (int k = 0; k < 9; ++k) {
        const size_t word = ((size_t)(p * 4 + mu) * 9 + k) * g.stride + h;
        if (rep == REP_SU3) {
            double2 w = ((const double2 *)d64)[word];
            u[k / 3][k % 3] = {w.x, w.y};
        } else {
            u[k / 3][k % 3] = {((const double *)d64)[word], 0.0};
        }
    }
}

// Compress the FP64 links to the reconstructed FP32 / FP16 formats.  A link is
// accepted when it is +-V with V special unitary (SU(3)) or special orthogonal
// (adjoint); the sign goes to the sign table.
__global__ void compress_gauge_kernel(Geom g, int rep, const void *d64, void *f32, void *h16, uint8_t *sign, int *err,
                                      float4 *f32r8, float4 *f32r18)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (h >= g.Vh) return;
    uint8_t bits = 0;
    for (int mu = 0; mu < 4; ++mu) {
        cx<double> u[3][3];
        load_link_d(g, rep, d64, p, mu, h, u);
        // unitarity: max |U U^+ - 1|
        double dev = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                cx<double> a = {i == j ? -1.0 : 0.0, 0.0};
                for (int k = 0; k < 3; ++k) fma_c(a, u[i][k], conj(u[j][k]));
                dev = fmax(dev, fabs(a.re) + fabs(a.im));
            }
        cx<double> det = u[0][0] * (u[1][1] * u[2][2] - u[1][2] * u[2][1]) -
                         u[0][1] * (u[1][0] * u[2][2] - u[1][2] * u[2][0]) +
                         u[0][2] * (u[1][0] * u[2][1] - u[1][1] * u[2][0]);
        int neg = 0;
        if (fabs(det.re - 1.0) + fabs(det.im) < 1e-8) neg = 0;
        else if (fabs(det.re + 1.0) + fabs(det.im) < 1e-8) neg = 1;
        else atomicOr(err, 1);
        if (dev > 1e-8) atomicOr(err, 2);
        bits |= (uint8_t)(neg << mu);
        const size_t w0 = (size_t)(p * 4 + mu) * 3 * g.stride + h;
        if (rep == REP_SU3) {
            float4 *F = (float4 *)f32;
            F[w0] = make_float4(u[0][0].re, u[0][0].im, u[0][1].re, u[0][1].im);
            F[w0 + g.stride] = make_float4(u[0][2].re, u[0][2].im, u[1][0].re, u[1][0].im);
            F[w0 + 2 * (size_t)g.stride] = make_float4(u[1][1].re, u[1][1].im, u[1][2].re, u[1][2].im);
            // 8 reals of V = s U (GaugeF8): (a2, a3), (b1, arg a1, arg c1)
            const double sg = neg ? -1.0 : 1.0;
            const size_t w8 = (size_t)(p * 4 + mu) * 2 * g.stride + h;
            f32r8[w8] = make_float4(sg * u[0][1].re, sg * u[0][1].im, sg * u[0][2].re, sg * u[0][2].im);
            f32r8[w8 + g.stride] = make_float4(sg * u[1][0].re, sg * u[1][0].im, atan2(sg * u[0][0].im, sg * u[0][0].re),
                                               atan2(sg * u[2][0].im, sg * u[2][0].re));
            // all 18 reals (GaugeF18P): entries row-major, two per word, the last word half used
            const size_t w18 = (size_t)(p * 4 + mu) * 5 * g.stride + h;
            for (int k = 0; k < 5; ++k) {
                const cx<double> a = u[(2 * k) / 3][(2 * k) % 3];
                const cx<double> b = k < 4 ? u[(2 * k + 1) / 3][(2 * k + 1) % 3] : cx<double>{0.0, 0.0};
                f32r18[w18 + (size_t)k * g.stride] = make_float4(a.re, a.im, b.re, b.im);
            }
            uint2 *H = (uint2 *)h16;
            double v[12] = {u[0][0].re, u[0][0].im, u[0][1].re, u[0][1].im, u[0][2].re, u[0][2].im,
                            u[1][0].re, u[1][0].im, u[1][1].re, u[1][1].im, u[1][2].re, u[1][2].im};
            for (int k = 0; k < 3; ++k) {
                uint2 w;
                __half2 *hp = reinterpret_cast<__half2 *>(&w);
                hp[0] = __floats2half2_rn((float)v[4 * k], (float)v[4 * k + 1]);
                hp[1] = __floats2half2_rn((float)v[4 * k + 2], (float)v[4 * k + 3]);
                H[w0 + (size_t)k * g.stride] = w;
            }
        } else {
            float2 *F = (float2 *)f32;
            F[w0] = make_float2(u[0][0].re, u[0][1].re);
            F[w0 + g.stride] = make_float2(u[0][2].re, u[1][0].re);
            F[w0 + 2 * (size_t)g.stride] = make_float2(u[1][1].re, u[1][2].re);
            __half2 *H = (__half2 *)h16;
            H[w0] = __floats2half2_rn((float)u[0][0].re, (float)u[0][1].re);
            H[w0 + g.stride] = __floats2half2_rn((float)u[0][2].re, (float)u[1][0].re);
            H[w0 + 2 * (size_t)g.stride] = __floats2half2_rn((float)u[1][1].re, (float)u[1][2].re);
        }
    }
    sign[(size_t)p * g.stride + h] = bits;
}

void launch_compress_gauge(const Geom &g, GaugeDev &U, int *err, cudaStream_t st)
{
    dim3 grid(nblocks(g.Vh, 128), 2);
    compress_gauge_kernel<<<grid, 128, 0, st>>>(g, U.rep, U.d64, U.f32, U.h16, U.sign, err, (float4 *)U.f32r8,
                                                (float4 *)U.f32r18);
}

// Fundamental gauge links -> fermion links: the adjoint map for SU(2)
// (utils/ConvertLattice.h:24-34,100-105) and the boundary condition folded into the
// links (LatticeBoundaryConditions.h:8-14).  In/out are host-layout AoS arrays.
__global__ void fundamental_to_fermion_kernel(Geom g, int rep, int bc, const double *gauge, double *fermion)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    lex_coords(g, s, c);
    for (int mu = 0; mu < 4; ++mu) {
        const double sgn = (bc == 1 && mu == 3 && c[3] == g.L[3] - 1) ? -1.0 : 1.0;
        if (rep == REP_SU3) {
            const double *src = gauge + ((size_t)s * 4 + mu) * 18;
            double *dst = fermion + ((size_t)s * 4 + mu) * 18;
            for (int k = 0; k < 18; ++k) dst[k] = sgn * src[k];
        } else {
            // SU(2) column-major complex 2x2 -> real 3x3 adj(a,b) = 2 Re tr(T_a U T_b U^+)
            const double2 *u2 = reinterpret_cast<const double2 *>(gauge) + ((size_t)s * 4 + mu) * 4;
            cx<double> U[2][2] = {{{u2[0].x, u2[0].y}, {u2[2].x, u2[2].y}}, {{u2[1].x, u2[1].y}, {u2[3].x, u2[3].y}}};
            const cx<double> Tm[3][2][2] = {{{{0, 0}, {0.5, 0}}, {{0.5, 0}, {0, 0}}},
                                            {{{0, 0}, {0, -0.5}}, {{0, 0.5}, {0, 0}}},
                                            {{{0.5, 0}, {0, 0}}, {{0, 0}, {-0.5, 0}}}};
            double *dst = fermion + ((size_t)s * 4 + mu) * 9;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    cx<double> A[2][2], B[2][2];
                    for (int i = 0; i < 2; ++i)
                        for (int j = 0; j < 2; ++j) {
                            A[i][j] = {0, 0};
                            for (int k = 0; k < 2; ++k) fma_c(A[i][j], Tm[a][i][k], U[k][j]);
                        }
                    for (int i = 0; i < 2; ++i)
                        for (int j = 0; j < 2; ++j) {
                            B[i][j] = {0, 0};
                            for (int k = 0; k < 2; ++k) fma_c(B[i][j], A[i][k], Tm[b][k][j]);
                        }
                    double tr = 0.0;
                    for (int i = 0; i < 2; ++i)
                        for (int k = 0; k < 2; ++k) {
                            cx<double> t = B[i][k] * conj(U[i][k]);  // (B U^+)_ii = sum_k B_ik conj(U_ik)
                            tr += t.re;
                        }
                    dst[b * 3 + a] = sgn * 2.0 * tr;
                }
        }
    }
}

void launch_fundamental_to_fermion(const Geom &g, int rep, int bc, const double *gauge_aos, double *fermion_aos,
                                   cudaStream_t st)
{
    fundamental_to_fermion_kernel<<<nblocks(g.V, 128), 128, 0, st>>>(g, rep, bc, gauge_aos, fermion_aos);
}

// ----------------------------------------------------------------- clover --
LYM_D void load_link_at(const Geom &g, int rep, const void *d64, int x, int y, int z, int t, int mu,
                        cx<double> u[3][3])
{
    x = (x + g.L[0]) % g.L[0];
    y = (y + g.L[1]) % g.L[1];
    z = (z + g.L[2]) % g.L[2];
    t = (t + g.L[3]) % g.L[3];
    const int s = lex_of(g, x, y, z, t);
    load_link_d(g, rep, d64, (x + y + z + t) & 1, mu, s >> 1, u);
}

LYM_D void m3_mul(const cx<double> a[3][3], const cx<double> b[3][3], cx<double> c[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cx<double> s = {0, 0};
            for (int k = 0; k < 3; ++k) fma_c(s, a[i][k], b[k][j]);
            c[i][j] = s;
        }
}
LYM_D void m3_dag(const cx<double> a[3][3], cx<double> c[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i][j] = conj(a[j][i]);
}

// Gauss-Jordan inverse with partial pivoting of a 6x6 complex matrix (row-major).
LYM_D int invert6(cx<double> m[6][6], cx<double> inv[6][6])
{
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) inv[i][j] = {i == j ? 1.0 : 0.0, 0.0};
    for (int col = 0; col < 6; ++col) {
        int piv = col;
        double best = hypot(m[col][col].re, m[col][col].im);
        for (int r = col + 1; r < 6; ++r) {
            const double a = hypot(m[r][col].re, m[r][col].im);
            if (a > best) {
                best = a;
                piv = r;
            }
        }
        if (best == 0.0) return 1;
        if (piv != col)
            for (int j = 0; j < 6; ++j) {
                cx<double> t = m[col][j];
                m[col][j] = m[piv][j];
                m[piv][j] = t;
                t = inv[col][j];
                inv[col][j] = inv[piv][j];
                inv[piv][j] = t;
            }
        const cx<double> d = m[col][col];
        const double dn = d.re * d.re + d.im * d.im;
        const cx<double> r = {d.re / dn, -d.im / dn};
        for (int j = 0; j < 6; ++j) {
            m[col][j] = m[col][j] * r;
            inv[col][j] = inv[col][j] * r;
        }
        for (int rr = 0; rr < 6; ++rr) {
            if (rr == col) continue;
            const cx<double> f = m[rr][col];
            for (int j = 0; j < 6; ++j) {
                m[rr][j] = m[rr][j] - f * m[col][j];
                inv[rr][j] = inv[rr][j] - f * inv[col][j];
            }
        }
    }
    return 0;
}

LYM_D void store_block_d(double2 *base, int stride, int h, const cx<double> m[6][6], bool symmetrize)
{
    for (int k = 0; k < 3; ++k) base[(size_t)k * stride + h] = make_double2(m[2 * k][2 * k].re, m[2 * k + 1][2 * k + 1].re);
    for (int i = 1; i < 6; ++i)
        for (int j = 0; j < i; ++j) {
            cx<double> a = m[i][j];
            if (symmetrize) a = 0.5 * (a + conj(m[j][i]));
            base[(size_t)(3 + tri_index(i, j)) * stride + h] = make_double2(a.re, a.im);
        }
}

// Field strength F_{mu nu} (ImprovedDiracWilsonOperator.cpp:502-523) and the two
// Hermitian blocks of T = 1 + kappa csw gamma5 C with their inverses
// (EvenOddImprovedDiracWilsonOperator.cpp:285-317).  One thread per site.
__global__ void clover_build_kernel(Geom g, int rep, const void *d64, double kc, double2 *T, double2 *Tinv,
                                    double *Fout, int *err)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (h >= g.Vh) return;
    int c[4];
    site_coords(g, h, p, c);
    const int planes[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    cx<double> F[6][3][3];
    for (int pl = 0; pl < 6; ++pl) {
        const int mu = planes[pl][0], nu = planes[pl][1];
        int e[4][4] = {{0}};
        e[mu][mu] = 1;
        e[nu][nu] = 1;
        const int *m = e[mu], *n = e[nu];
        cx<double> Q[3][3], A[3][3], B[3][3], C[3][3], D[3][3], t1[3][3], t2[3][3], t3[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Q[i][j] = {0, 0};
#define LINK(dx, dir, out) load_link_at(g, rep, d64, c[0] + (dx)[0], c[1] + (dx)[1], c[2] + (dx)[2], c[3] + (dx)[3], dir, out)
        int o_m[4], o_n[4], o_mn[4], o_nm[4], o0[4] = {0, 0, 0, 0}, o_pm[4], o_pn[4], o_mpn[4];
        for (int k = 0; k < 4; ++k) {
            o_m[k] = -m[k];            // x - mu
            o_n[k] = -n[k];            // x - nu
            o_mn[k] = -m[k] - n[k];    // x - mu - nu
            o_pm[k] = m[k];            // x + mu
            o_pn[k] = n[k];            // x + nu
            o_nm[k] = -n[k] + m[k];    // x - nu + mu
            o_mpn[k] = -m[k] + n[k];   // x - mu + nu
        }
        // leaf 1: U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
        LINK(o_m, mu, t1); m3_dag(t1, A);
        LINK(o_mn, nu, t1); m3_dag(t1, B);
        LINK(o_mn, mu, C);
        LINK(o_n, nu, D);
        m3_mul(A, B, t1); m3_mul(t1, C, t2); m3_mul(t2, D, t3);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = Q[i][j] + t3[i][j];
        // leaf 2: U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+
        LINK(o_n, nu, t1); m3_dag(t1, A);
        LINK(o_n, mu, B);
        LINK(o_nm, nu, C);
        LINK(o0, mu, t1); m3_dag(t1, D);
        m3_mul(A, B, t1); m3_mul(t1, C, t2); m3_mul(t2, D, t3);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = Q[i][j] + t3[i][j];
        // leaf 3: U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
        LINK(o0, mu, A);
        LINK(o_pm, nu, B);
        LINK(o_pn, mu, t1); m3_dag(t1, C);
        LINK(o0, nu, t1); m3_dag(t1, D);
        m3_mul(A, B, t1); m3_mul(t1, C, t2); m3_mul(t2, D, t3);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = Q[i][j] + t3[i][j];
        // leaf 4: U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
        LINK(o0, nu, A);
        LINK(o_mpn, mu, t1); m3_dag(t1, B);
        LINK(o_m, nu, t1); m3_dag(t1, C);
        LINK(o_m, mu, D);
        m3_mul(A, B, t1); m3_mul(t1, C, t2); m3_mul(t2, D, t3);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = Q[i][j] + t3[i][j];
#undef LINK
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) F[pl][i][j] = 0.125 * (Q[i][j] - conj(Q[j][i]));
    }
    if (Fout) {
        const int s = lex_of(g, c[0], c[1], c[2], c[3]);
        for (int pl = 0; pl < 6; ++pl)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const size_t at = (((size_t)s * 6 + pl) * 9 + j * 3 + i) * 2;
                    Fout[at] = F[pl][i][j].re;
                    Fout[at + 1] = F[pl][i][j].im;
                }
    }
    for (int blk = 0; blk < 2; ++blk) {
        // local spin a, b in {0,1}; component r = a*3 + i
        cx<double> M[6][6], Mi[6][6];
        const double sg = blk == 0 ? 1.0 : -1.0;  // gamma5 sign of the block
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const cx<double> F0 = F[0][i][j], F1 = F[1][i][j], F2 = F[2][i][j];
                const cx<double> F3 = F[3][i][j], F4 = F[4][i][j], F5 = F[5][i][j];
                cx<double> a00, a11, a01, a10;
                if (blk == 0) {
                    a00 = times_i(F5 - F0);
                    a11 = times_i(F0 - F5);
                    a01 = F1 + F4 + times_i(F2 - F3);
                    a10 = -F1 - F4 + times_i(F2 - F3);
                } else {
                    a00 = times_i(F0 + F5);
                    a11 = times_i(-F0 - F5);
                    a01 = -F1 + F4 + times_i(F2 + F3);
                    a10 = F1 - F4 + times_i(F2 + F3);
                }
                M[i][j] = (sg * kc) * a00;
                M[3 + i][3 + j] = (sg * kc) * a11;
                M[i][3 + j] = (sg * kc) * a01;
                M[3 + i][j] = (sg * kc) * a10;
            }
        for (int k = 0; k < 6; ++k) M[k][k].re += 1.0;
        double2 *Tb = T + (size_t)(p * 2 + blk) * 18 * g.stride;
        store_block_d(Tb, g.stride, h, M, false);
        if (invert6(M, Mi)) atomicOr(err, 4);
        double2 *Ib = Tinv + (size_t)(p * 2 + blk) * 18 * g.stride;
        store_block_d(Ib, g.stride, h, Mi, true);
    }
}

void launch_clover_build(const Geom &g, const GaugeDev &U, double kc, CloverDev &C, double *F_aos, int *err,
                         cudaStream_t st)
{
    dim3 grid(nblocks(g.Vh, 64), 2);
    clover_build_kernel<<<grid, 64, 0, st>>>(g, U.rep, U.d64, kc, (double2 *)C.T[PREC_D], (double2 *)C.Tinv[PREC_D],
                                             F_aos, err);
}

__global__ void clover_compress_kernel(Geom g, const double2 *src, float4 *f32, uint2 *h16)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int pb = blockIdx.y;  // parity * 2 + block
    if (h >= g.Vh) return;
    double v[36];
    const double2 *base = src + (size_t)pb * 18 * g.stride + h;
    for (int k = 0; k < 18; ++k) {
        double2 w = base[(size_t)k * g.stride];
        v[2 * k] = w.x;
        v[2 * k + 1] = w.y;
    }
    float4 *fb = f32 + (size_t)pb * 9 * g.stride + h;
    uint2 *hb = h16 + (size_t)pb * 9 * g.stride + h;
    for (int k = 0; k < 9; ++k) {
        fb[(size_t)k * g.stride] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        uint2 w;
        __half2 *hp = reinterpret_cast<__half2 *>(&w);
        hp[0] = __floats2half2_rn((float)v[4 * k], (float)v[4 * k + 1]);
        hp[1] = __floats2half2_rn((float)v[4 * k + 2], (float)v[4 * k + 3]);
        hb[(size_t)k * g.stride] = w;
    }
}

void launch_clover_compress(const Geom &g, CloverDev &C, cudaStream_t st)
{
    dim3 grid(nblocks(g.Vh, 128), 4);
    clover_compress_kernel<<<grid, 128, 0, st>>>(g, (const double2 *)C.T[PREC_D], (float4 *)C.T[PREC_F],
                                                 (uint2 *)C.T[PREC_H]);
    clover_compress_kernel<<<grid, 128, 0, st>>>(g, (const double2 *)C.Tinv[PREC_D], (float4 *)C.Tinv[PREC_F],
                                                 (uint2 *)C.Tinv[PREC_H]);
}

// --------------------------------------------------------- index checking --
// Reference-order neighbour tables (LocalLayout.h:34-110), for layout tests.
__global__ void neighbour_tables_kernel(Geom g, int *sup, int *sdn)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    lex_coords(g, s, c);
    for (int mu = 0; mu < 4; ++mu) {
        int a[4] = {c[0], c[1], c[2], c[3]}, b[4] = {c[0], c[1], c[2], c[3]};
        a[mu] = (a[mu] + 1) % g.L[mu];
        b[mu] = (b[mu] - 1 + g.L[mu]) % g.L[mu];
        sup[s * 4 + mu] = lex_of(g, a[0], a[1], a[2], a[3]);
        sdn[s * 4 + mu] = lex_of(g, b[0], b[1], b[2], b[3]);
    }
}

void launch_neighbour_tables(const Geom &g, int *sup, int *sdn, cudaStream_t st)
{
    neighbour_tables_kernel<<<nblocks(g.V, 128), 128, 0, st>>>(g, sup, sdn);
}

// What the stencil computes for every (parity, h): its own lexicographic index and
// the half-site indices of its 8 neighbours, out[(p*Vh + h)*9 + k].
__global__ void stencil_index_probe_kernel(Geom g, int *out)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (h >= g.Vh) return;
    int c[4];
    site_coords(g, h, p, c);
    int *o = out + ((size_t)p * g.Vh + h) * 9;
    o[0] = lex_of(g, c[0], c[1], c[2], c[3]);
    for (int mu = 0; mu < 4; ++mu) {
        o[1 + 2 * mu] = neighbour_h(g, c, mu, +1);
        o[2 + 2 * mu] = neighbour_h(g, c, mu, -1);
    }
}

__global__ void nbr_table_kernel(Geom g, int *nbr)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (h >= g.Vh) return;
    int c[4];
    site_coords(g, h, p, c);
    for (int mu = 0; mu < 4; ++mu) {
        nbr[(size_t)(p * 8 + 2 * mu) * g.stride + h] = neighbour_h(g, c, mu, +1);
        nbr[(size_t)(p * 8 + 2 * mu + 1) * g.stride + h] = neighbour_h(g, c, mu, -1);
    }
}

void launch_nbr_table(const Geom &g, int *nbr, cudaStream_t st)
{
    dim3 grid(nblocks(g.Vh, 128), 2);
    nbr_table_kernel<<<grid, 128, 0, st>>>(g, nbr);
}

void launch_stencil_index_probe(const Geom &g, int *out, cudaStream_t st)
{
    dim3 grid(nblocks(g.Vh, 128), 2);
    stencil_index_probe_kernel<<<grid, 128, 0, st>>>(g, out);
}

// ----------------------------------------------------------------- dslash --
template <typename R, class S, class G, class C>
static void run_dslash(const DslashParams &P, const S &in, const S &out, const S &y, const S &v2, const G &U,
                       const C &T, cudaStream_t st)
{
    DslashArg<S, G, C> a;
    a.g = P.g;
    a.in = in;
    a.out = out;
    a.y = y;
    a.v2 = v2;
    a.U = U;
    a.T = T;
    a.parity = P.parity;
    a.gamma5 = P.gamma5;
    a.has_v2 = P.has_v2;
    a.has_clover = P.clover != nullptr;
    a.a = P.a;
    a.b = P.b;
    a.alpha_re = P.alpha_re;
    a.alpha_im = P.alpha_im;
    a.skip_if = P.skip_if;
    const int nb = nblocks(P.g.Vh, 128);
    switch (P.epi) {
    case EPI_SCALE_: dslash_kernel<R, EPI_SCALE><<<nb, 128, 0, st>>>(a); break;
    case EPI_CLOVINV_: dslash_kernel<R, EPI_CLOVINV><<<nb, 128, 0, st>>>(a); break;
    case EPI_XPAY_: dslash_kernel<R, EPI_XPAY><<<nb, 128, 0, st>>>(a); break;
    default: dslash_kernel<R, EPI_XPAY_INV><<<nb, 128, 0, st>>>(a); break;
    }
}

void launch_dslash(const DslashParams &P, cudaStream_t st)
{
    const GaugeDev &U = *P.U;
    const int s = P.g.stride;
    if (P.prec == PREC_D) {
        CloverD T{(const double2 *)P.clover, s};
        if (P.rep == REP_SU3)
            run_dslash<double>(P, P.in.d(), P.out.d(), P.y.d(), P.v2.d(), GaugeD18{(const double2 *)U.d64, s}, T, st);
        else
            run_dslash<double>(P, P.in.d(), P.out.d(), P.y.d(), P.v2.d(), GaugeD9{(const double *)U.d64, s}, T, st);
    } else if (P.prec == PREC_F) {
        CloverF T{(const float4 *)P.clover, s};
        if (P.rep == REP_SU3 && U.link_reals == 8)
            run_dslash<float>(P, P.in.f(), P.out.f(), P.y.f(), P.v2.f(), GaugeF8{(const float4 *)U.f32r8, U.sign, s}, T,
                              st);
        else if (P.rep == REP_SU3)
            run_dslash<float>(P, P.in.f(), P.out.f(), P.y.f(), P.v2.f(), GaugeF12{(const float4 *)U.f32, U.sign, s}, T,
                              st);
        else
            run_dslash<float>(P, P.in.f(), P.out.f(), P.y.f(), P.v2.f(), GaugeF6{(const float2 *)U.f32, U.sign, s}, T,
                              st);
    } else {
        CloverH T{(const uint2 *)P.clover, s};
        if (P.rep == REP_SU3)
            run_dslash<float>(P, P.in.h(), P.out.h(), P.y.h(), P.v2.h(), GaugeH12{(const uint2 *)U.h16, U.sign, s}, T,
                              st);
        else
            run_dslash<float>(P, P.in.h(), P.out.h(), P.y.h(), P.v2.h(), GaugeH6{(const __half2 *)U.h16, U.sign, s}, T,
                              st);
    }
}

// ---------------------------------------------------- stencil + CG epilogue --
struct CGAlphaFromNorm {  // alpha = |r|^2 / <p, A p> with <p, A p> = |Q p|^2
    CGState *s;
    LYM_D void operator()(double qq) const { s->alpha = make_double2(s->rr / qq, 0.0); }
};
template <class Upd> struct CGUpdateFin {  // the scalar step of OpCGUpdate
    Upd u;
    LYM_D void operator()(double rr) const
    {
        const double t[1] = {rr};
        u.finalize(t);
    }
};

template <typename R, class S, class SX, class SR, class G, class C>
static void run_dslash_cg(const DslashParams &P, int mode, const S &in, const S &out, const S &y, const S &p,
                          const SX &x, const SR &r, const G &U, const C &T, void *state, double *partials,
                          unsigned int *counter, cudaStream_t st)
{
    DslashArg<S, G, C> a;
    a.g = P.g;
    a.in = in;
    a.out = out;
    a.y = y;
    a.v2 = p;
    a.U = U;
    a.T = T;
    a.parity = P.parity;
    a.gamma5 = 1;
    a.has_v2 = 0;
    a.has_clover = P.clover != nullptr;
    a.a = P.a;
    a.b = P.b;
    a.alpha_re = a.alpha_im = 0.0;
    a.skip_if = P.skip_if;
    CGState *cs = (CGState *)state;
    const int nb = nblocks(P.g.Vh, 128);
    if (mode == CG_NORM) {
        CGEpilogue<SX, SR, CGAlphaFromNorm> f{x, r, &cs->alpha, CGAlphaFromNorm{cs}, partials, counter};
        dslash_cg_kernel<R, CG_NORM><<<nb, 128, 0, st>>>(a, f);
    } else {
        typedef OpCGUpdate<SX, S, SR, S> Upd;
        CGEpilogue<SX, SR, CGUpdateFin<Upd>> f{x, r, &cs->alpha, CGUpdateFin<Upd>{Upd{x, p, r, p, cs}}, partials,
                                                counter};
        dslash_cg_kernel<R, CG_UPDATE><<<nb, 128, 0, st>>>(a, f);
    }
}

void launch_dslash_cg(const DslashParams &P, int mode, const Spinor &p, const Spinor &x, const Spinor &r, void *state,
                      double *partials, unsigned int *counter, cudaStream_t st)
{
    const GaugeDev &U = *P.U;
    const int s = P.g.stride;
    if (P.prec == PREC_D) {
        CloverD T{(const double2 *)P.clover, s};
        if (P.rep == REP_SU3)
            run_dslash_cg<double>(P, mode, P.in.d(), P.out.d(), P.y.d(), p.d(), x.d(), r.d(),
                                  GaugeD18{(const double2 *)U.d64, s}, T, state, partials, counter, st);
        else
            run_dslash_cg<double>(P, mode, P.in.d(), P.out.d(), P.y.d(), p.d(), x.d(), r.d(),
                                  GaugeD9{(const double *)U.d64, s}, T, state, partials, counter, st);
    } else if (P.prec == PREC_F) {
        CloverF T{(const float4 *)P.clover, s};
        if (P.rep == REP_SU3 && U.link_reals == 8)
            run_dslash_cg<float>(P, mode, P.in.f(), P.out.f(), P.y.f(), p.f(), x.f(), r.f(),
                                 GaugeF8{(const float4 *)U.f32r8, U.sign, s}, T, state, partials, counter, st);
        else if (P.rep == REP_SU3)
            run_dslash_cg<float>(P, mode, P.in.f(), P.out.f(), P.y.f(), p.f(), x.f(), r.f(),
                                 GaugeF12{(const float4 *)U.f32, U.sign, s}, T, state, partials, counter, st);
        else
            run_dslash_cg<float>(P, mode, P.in.f(), P.out.f(), P.y.f(), p.f(), x.f(), r.f(),
                                 GaugeF6{(const float2 *)U.f32, U.sign, s}, T, state, partials, counter, st);
    } else {
        CloverH T{(const uint2 *)P.clover, s};
        if (P.rep == REP_SU3)
            run_dslash_cg<float>(P, mode, P.in.h(), P.out.h(), P.y.h(), p.h(), x.f(), r.f(),
                                 GaugeH12{(const uint2 *)U.h16, U.sign, s}, T, state, partials, counter, st);
        else
            run_dslash_cg<float>(P, mode, P.in.h(), P.out.h(), P.y.h(), p.h(), x.f(), r.f(),
                                 GaugeH6{(const __half2 *)U.h16, U.sign, s}, T, state, partials, counter, st);
    }
}

template <typename R, class S, class C>
static void run_clover(const Geom &g, const S &out, const S &in, const C &T, int parity, int gamma5, cudaStream_t st)
{
    clover_kernel<R><<<nblocks(g.Vh, 128), 128, 0, st>>>(g, out, in, T, parity, gamma5);
}

void launch_clover(const Geom &g, int prec, const Spinor &out, const Spinor &in, const void *clover, int parity,
                   int gamma5, cudaStream_t st)
{
    if (prec == PREC_D) run_clover<double>(g, out.d(), in.d(), CloverD{(const double2 *)clover, g.stride}, parity, gamma5, st);
    else if (prec == PREC_F) run_clover<float>(g, out.f(), in.f(), CloverF{(const float4 *)clover, g.stride}, parity, gamma5, st);
    else run_clover<float>(g, out.h(), in.h(), CloverH{(const uint2 *)clover, g.stride}, parity, gamma5, st);
}

}  // namespace lym
