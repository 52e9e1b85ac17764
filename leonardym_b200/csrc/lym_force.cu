// Fermion force of the Wilson and Wilson-clover operators on the device:
// FermionForce::derivative (hmc_forces/FermionForce.cpp:11-20) with the per-link matrices of
// DiracWilsonFermionForce::derivative (hmc_forces/DiracWilsonFermionForce.cpp:10-53) and
// ImprovedFermionForce::derivative (hmc_forces/ImprovedFermionForce.cpp:11-223, the eight
// clover-leaf terms with the link products of its setLattice, :225-268, formed on the fly):
//   force[x][mu] -= weight * F_mu(x),  F = clover / 4 + Wilson.
// X, Y and the force field are in the reference's AoS layout: spinors double2[V][4][3], force
// matrices double2[V][4][3][3] column-major ([site][mu][j][i] = F(i, j)).  One thread per
// (site, mu), everything in FP64.
#include <cmath>
#include <complex>

#include "lym_common.cuh"
#include "lym_internal.h"

namespace lym {

namespace {

typedef cx<double> C;

struct M3 {
    C a[3][3];  // a[i][j] = M(i, j)
};

// (gamma5 (1 - gamma_mu))_{ab}, (gamma5 (1 + gamma_mu))_{ab}, (gamma5 sigma_{mu nu})_{ab} of
// the chiral basis: gamma_k = [[0, -i s_k], [i s_k, 0]] (k = x, y, z), gamma_t = [[0, 1], [1, 0]],
// gamma5 = diag(1, 1, -1, -1), sigma_{mu nu} = (i/2) [gamma_mu, gamma_nu] (the reference's
// Gamma / Sigma tables, utils/Gamma.cpp)
struct ForceTables {
    C mg[4][4][4];
    C pg[4][4][4];
    C g5s[4][4][4][4];
};
__constant__ ForceTables c_ft;

LYM_D M3 mul(const M3 &A, const M3 &B)
{
    M3 R;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            C s{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 3; ++k) fma_c(s, A.a[i][k], B.a[k][j]);
            R.a[i][j] = s;
        }
    return R;
}
LYM_D M3 dag(const M3 &A)
{
    M3 R;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) R.a[i][j] = conj(A.a[j][i]);
    return R;
}
LYM_D void mv(const M3 &A, const C x[3], C y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        C s{0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 3; ++k) fma_c(s, A.a[i][k], x[k]);
        y[i] = s;
    }
}
// F += s * tensor(x, y), tensor(x, y)(i, j) = y[i] conj(x[j])  (FermionForce.cpp:22-31)
LYM_D void add_tensor(M3 &F, double s, const C x[3], const C y[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            C t{0.0, 0.0};
            fma_cc(t, x[j], y[i]);
            F.a[i][j] = F.a[i][j] + s * t;
        }
}

struct ForceArg {
    Geom g;
    const void *links;  // FP64 fermion links [2][4][9][stride] (complex, or real for the adjoint)
    int rep;
    const double2 *X, *Y;
    double2 *force;
    double kappa, csw, weight;
    int clover;
};

template <class Gauge> struct Ctx {
    const ForceArg &a;
    Gauge U;
    LYM_D int coord_site(const int c[4]) const
    {
        return c[3] + a.g.L[3] * (c[2] + a.g.L[2] * (c[1] + a.g.L[1] * c[0]));
    }
    LYM_D void coords(int s, int c[4]) const
    {
        c[3] = s % a.g.L[3];
        int r = s / a.g.L[3];
        c[2] = r % a.g.L[2];
        r /= a.g.L[2];
        c[1] = r % a.g.L[1];
        c[0] = r / a.g.L[1];
    }
    // site + d1 e_m1 + d2 e_m2 (periodic in the index)
    LYM_D int shift(int s, int m1, int d1, int m2 = 0, int d2 = 0) const
    {
        int c[4];
        coords(s, c);
        c[m1] = (c[m1] + d1 + a.g.L[m1]) % a.g.L[m1];
        if (d2) c[m2] = (c[m2] + d2 + a.g.L[m2]) % a.g.L[m2];
        return coord_site(c);
    }
    LYM_D M3 link(int s, int mu) const
    {
        int c[4];
        coords(s, c);
        const int p = (c[0] + c[1] + c[2] + c[3]) & 1;
        typename Gauge::Link L;
        U.load(p, mu, s >> 1, L);
        M3 M;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) M.a[i][j] = as_c(L.u[i][j]);
        return M;
    }
    LYM_D static C as_c(cx<double> z) { return z; }
    LYM_D static C as_c(double z) { return C{z, 0.0}; }
    LYM_D void spinor(const double2 *V, int s, C v[4][3]) const
    {
#pragma unroll
        for (int al = 0; al < 4; ++al)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double2 w = __ldg(V + (size_t)s * 12 + al * 3 + d);
                v[al][d] = C{w.x, w.y};
            }
    }
};

// sum over beta of coef * T[alpha][beta] * v[beta] for one alpha
LYM_D void spin_comb(const C T[4][4], int al, C coef, const C v[4][3], C out[3])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = C{0.0, 0.0};
#pragma unroll
    for (int be = 0; be < 4; ++be) {
        const C w = coef * T[al][be];
        if (w.re == 0.0 && w.im == 0.0) continue;
#pragma unroll
        for (int d = 0; d < 3; ++d) fma_c(out[d], w, v[be][d]);
    }
}

template <class Gauge> __global__ void __launch_bounds__(128) fermion_force_kernel(ForceArg a, Gauge U)
{
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 4L * a.g.V) return;
    const int site = (int)(tid >> 2), mu = (int)(tid & 3);
    const Ctx<Gauge> cx_{a, U};
    M3 F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) F.a[i][j] = C{0.0, 0.0};
    const C mk{-a.kappa, 0.0};
    const int xp = cx_.shift(site, mu, +1);
    {
        // DiracWilsonFermionForce::derivative
        C Xs[4][3], Ys[4][3], Xp[4][3], Yp[4][3];
        cx_.spinor(a.X, site, Xs);
        cx_.spinor(a.Y, site, Ys);
        cx_.spinor(a.X, xp, Xp);
        cx_.spinor(a.Y, xp, Yp);
        const M3 Um = cx_.link(site, mu), Ud = dag(Um);
        C UdXs[4][3], UdYs[4][3];
#pragma unroll
        for (int al = 0; al < 4; ++al) {
            mv(Ud, Xs[al], UdXs[al]);
            mv(Ud, Ys[al], UdYs[al]);
        }
#pragma unroll 1
        for (int al = 0; al < 4; ++al) {
            C t[3], u[3];
            spin_comb(c_ft.mg[mu], al, mk, Yp, t);
            add_tensor(F, 1.0, Xs[al], t);
            spin_comb(c_ft.pg[mu], al, mk, UdYs, t);
            mv(Um, Xp[al], u);
            add_tensor(F, -1.0, u, t);
            spin_comb(c_ft.mg[mu], al, mk, Xp, t);
            add_tensor(F, 1.0, Ys[al], t);
            spin_comb(c_ft.pg[mu], al, mk, UdXs, t);
            mv(Um, Yp[al], u);
            add_tensor(F, -1.0, u, t);
        }
    }
    if (a.clover) {
        // ImprovedFermionForce::derivative, terms 1-8 for every nu != mu
        M3 Fc;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Fc.a[i][j] = C{0.0, 0.0};
        const C ikc{0.0, a.kappa * a.csw};
        const M3 Umu_x = cx_.link(site, mu);
#pragma unroll 1
        for (int nu = 0; nu < 4; ++nu) {
            if (nu == mu) continue;
            const int xpn = cx_.shift(site, nu, +1), xmn = cx_.shift(site, nu, -1);
            const int xpm_mn = cx_.shift(site, mu, +1, nu, -1), xpm_pn = cx_.shift(site, mu, +1, nu, +1);
            const M3 Unu_x = cx_.link(site, nu), Unu_xpm = cx_.link(xp, nu), Umu_xpn = cx_.link(xpn, mu);
            const M3 Unu_xpm_mn = cx_.link(xpm_mn, nu), Umu_xmn = cx_.link(xmn, mu), Unu_xmn = cx_.link(xmn, nu);
            const M3 Umu_xd = dag(Umu_x);
#pragma unroll 1
            for (int term = 0; term < 8; ++term) {
                M3 L, R;
                bool hasL = true, hasR = true;
                int ps;
                switch (term) {
                case 0:  // L = U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
                    L = mul(mul(Unu_xpm, dag(Umu_xpn)), dag(Unu_x));
                    hasR = false;
                    ps = site;
                    break;
                case 1:  // L = U_mu(x)^+, R = U_mu(x) U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
                    L = Umu_xd;
                    R = mul(mul(mul(Umu_x, dag(Unu_xpm_mn)), dag(Umu_xmn)), Unu_xmn);
                    ps = site;
                    break;
                case 2:  // L = U_nu(x+mu) U_mu(x+nu)^+, R = U_nu(x)
                    L = mul(Unu_xpm, dag(Umu_xpn));
                    R = Unu_x;
                    ps = xpn;
                    break;
                case 3:  // L = U_mu(x)^+ U_nu(x-nu)^+, R = U_mu(x) U_nu(x+mu-nu)^+ U_mu(x-nu)^+
                    L = mul(Umu_xd, dag(Unu_xmn));
                    R = mul(mul(Umu_x, dag(Unu_xpm_mn)), dag(Umu_xmn));
                    ps = xmn;
                    break;
                case 4:  // R = U_nu(x) U_mu(x+nu) U_nu(x+mu)^+
                    hasL = false;
                    R = mul(mul(Unu_x, Umu_xpn), dag(Unu_xpm));
                    ps = xp;
                    break;
                case 5:  // L = U_mu(x)^+ U_nu(x-nu)^+ U_mu(x-nu) U_nu(x+mu-nu), R = U_mu(x)
                    L = mul(mul(mul(Umu_xd, dag(Unu_xmn)), Umu_xmn), Unu_xpm_mn);
                    R = Umu_x;
                    ps = xp;
                    break;
                case 6:  // L = U_nu(x+mu), R = U_nu(x) U_mu(x+nu)
                    L = Unu_xpm;
                    R = mul(Unu_x, Umu_xpn);
                    ps = xpm_pn;
                    break;
                default:  // L = U_mu(x)^+ U_nu(x-nu)^+ U_mu(x-nu), R = U_mu(x) U_nu(x+mu-nu)^+
                    L = mul(mul(Umu_xd, dag(Unu_xmn)), Umu_xmn);
                    R = mul(Umu_x, dag(Unu_xpm_mn));
                    ps = xpm_mn;
                    break;
                }
                const double sg = (term & 1) ? -1.0 : 1.0;
                C Xq[4][3], Yq[4][3];
                cx_.spinor(a.X, ps, Xq);
                cx_.spinor(a.Y, ps, Yq);
#pragma unroll 1
                for (int al = 0; al < 4; ++al) {
                    C pX[3], pY[3], lX[3], lY[3], rX[3], rY[3];
                    spin_comb(c_ft.g5s[mu][nu], al, ikc, Xq, pX);
                    spin_comb(c_ft.g5s[mu][nu], al, ikc, Yq, pY);
                    if (hasL) {
                        mv(L, pY, lY);
                        mv(L, pX, lX);
                    } else {
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            lY[d] = pY[d];
                            lX[d] = pX[d];
                        }
                    }
                    if (hasR) {
                        mv(R, Xq[al], rX);
                        mv(R, Yq[al], rY);
                    } else {
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            rX[d] = Xq[al][d];
                            rY[d] = Yq[al][d];
                        }
                    }
                    add_tensor(Fc, sg, rX, lY);
                    add_tensor(Fc, sg, rY, lX);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) F.a[i][j] = 0.25 * Fc.a[i][j] + F.a[i][j];
    }
    double2 *out = a.force + ((size_t)site * 4 + mu) * 9;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double2 w = out[j * 3 + i];
            w.x -= a.weight * F.a[i][j].re;
            w.y -= a.weight * F.a[i][j].im;
            out[j * 3 + i] = w;
        }
}

void upload_tables(cudaStream_t st)
{
    typedef std::complex<double> Z;
    const Z I(0.0, 1.0);
    Z g[4][4][4] = {}, g5[4][4] = {};
    // gamma_k = [[0, -i s_k], [i s_k, 0]] for k = x, y, z; gamma_t = [[0, 1], [1, 0]]
    const Z s[3][2][2] = {{{0.0, 1.0}, {1.0, 0.0}}, {{0.0, -I}, {I, 0.0}}, {{1.0, 0.0}, {0.0, -1.0}}};
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                g[k][i][2 + j] = -I * s[k][i][j];
                g[k][2 + i][j] = I * s[k][i][j];
            }
    for (int i = 0; i < 2; ++i) {
        g[3][i][2 + i] = 1.0;
        g[3][2 + i][i] = 1.0;
    }
    for (int i = 0; i < 4; ++i) g5[i][i] = i < 2 ? 1.0 : -1.0;
    ForceTables T;
    for (int m = 0; m < 4; ++m)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                // gamma5 (1 -+ gamma_mu) = g5[a][a] (delta_ab -+ g[m][a][b])
                const Z d = a == b ? 1.0 : 0.0;
                const Z mgz = g5[a][a] * (d - g[m][a][b]), pgz = g5[a][a] * (d + g[m][a][b]);
                T.mg[m][a][b] = C{mgz.real(), mgz.imag()};
                T.pg[m][a][b] = C{pgz.real(), pgz.imag()};
            }
    for (int m = 0; m < 4; ++m)
        for (int n = 0; n < 4; ++n)
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) {
                    Z c = 0.0;
                    for (int k = 0; k < 4; ++k) c += g[m][a][k] * g[n][k][b] - g[n][a][k] * g[m][k][b];
                    const Z v = g5[a][a] * 0.5 * I * c;
                    T.g5s[m][n][a][b] = C{v.real(), v.imag()};
                }
    cudaMemcpyToSymbolAsync(c_ft, &T, sizeof(T), 0, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);  // T is a host local
}

}  // namespace

void launch_fermion_force(const Geom &g, const GaugeDev &U, const double2 *X, const double2 *Y, double kappa,
                          double csw, int clover, double weight, double2 *force, cudaStream_t st)
{
    upload_tables(st);
    ForceArg a{g, U.d64, U.rep, X, Y, force, kappa, csw, weight, clover};
    const long n = 4L * g.V;
    const int grid = (int)((n + 127) / 128);
    if (U.rep == REP_SU3)
        fermion_force_kernel<GaugeD18><<<grid, 128, 0, st>>>(a, GaugeD18{(const double2 *)U.d64, g.stride});
    else
        fermion_force_kernel<GaugeD9><<<grid, 128, 0, st>>>(a, GaugeD9{(const double *)U.d64, g.stride});
}

}  // namespace lym
