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
    int n;                     // pairs (x_i, y_i) with weights w_i
    const double2 *const *X;   // device array [n] of AoS spinors
    const double2 *const *Y;
    const double *w;           // device array [n]
    double2 *force;
    const double2 *N;  // [V][6][3][3] plane matrices (clover only)
    double kappa, csw;
    int clover;
};

// planes (mu < nu): 01 02 03 12 13 23
LYM_D int plane_index(int mu, int nu)
{
    const int a = mu < nu ? mu : nu, b = mu < nu ? nu : mu;
    return a == 0 ? b - 1 : (a == 1 ? b + 1 : 5);
}
LYM_D M3 load_plane(const double2 *N, int site, int plane)
{
    M3 M;
    const double2 *b = N + ((size_t)site * 6 + plane) * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double2 w = __ldg(b + k);
        M.a[k / 3][k % 3] = C{w.x, w.y};
    }
    return M;
}

// N^{mu nu}(x) = i kappa c_sw sum_i w_i sum_{ab} (gamma5 sigma_{mu nu})_{ab} (Y_b X_a^+ + X_b Y_a^+) at
// every site, for the six planes mu < nu: the spinor part of ImprovedFermionForce's terms, whose
// term k is then sign_k L_k N(x_k) R_k^+ (tensor(R X_a, L P_Y[a]) + tensor(R Y_a, L P_X[a]) summed
// over a)
__global__ void __launch_bounds__(128) clover_outer_kernel(ForceArg a, double2 *N)
{
    // one thread per (site, plane): the six threads of a site are neighbours in the warp, so
    // each spinor word comes from DRAM once and from L1 for the other five
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 6L * a.g.V) return;
    const int site = (int)(tid / 6), p = (int)(tid % 6);
    {
        const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2), nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
        M3 acc;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc.a[i][j] = C{0.0, 0.0};
#pragma unroll 1
        for (int k = 0; k < a.n; ++k) {
            const double2 *Xp = a.X[k] + (size_t)site * 12, *Yp = a.Y[k] + (size_t)site * 12;
            const C ikc{0.0, a.kappa * a.csw * a.w[k]};
#pragma unroll 1
            for (int al = 0; al < 4; ++al) {
                C xa[3], ya[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double2 x = __ldg(Xp + al * 3 + d), y = __ldg(Yp + al * 3 + d);
                    xa[d] = C{x.x, x.y};
                    ya[d] = C{y.x, y.y};
                }
#pragma unroll 1
                for (int be = 0; be < 4; ++be) {
                    const C g = c_ft.g5s[mu][nu][al][be];
                    if (g.re == 0.0 && g.im == 0.0) continue;
                    const C c = ikc * g;
                    C xb[3], yb[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double2 x = __ldg(Xp + be * 3 + d), y = __ldg(Yp + be * 3 + d);
                        xb[d] = C{x.x, x.y};
                        yb[d] = C{y.x, y.y};
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            C t{0.0, 0.0};
                            fma_cc(t, xa[j], yb[i]);
                            fma_cc(t, ya[j], xb[i]);
                            fma_c(acc.a[i][j], c, t);
                        }
                }
            }
        }
        double2 *o = N + ((size_t)site * 6 + p) * 9;
#pragma unroll
        for (int k = 0; k < 9; ++k) o[k] = make_double2(acc.a[k / 3][k % 3].re, acc.a[k / 3][k % 3].im);
    }
}

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
    LYM_D static void colour(const double2 *V, int s, int al, C v[3])
    {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double2 w = __ldg(V + (size_t)s * 12 + al * 3 + d);
            v[d] = C{w.x, w.y};
        }
    }
};

// out = coef * sum_beta T[al][beta] V(s, beta), the non-zero entries only
LYM_D void spin_comb(const C T[4][4], int al, C coef, const double2 *V, int s, C out[3])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = C{0.0, 0.0};
#pragma unroll 1
    for (int be = 0; be < 4; ++be) {
        const C w = coef * T[al][be];
        if (w.re == 0.0 && w.im == 0.0) continue;
        C v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double2 z = __ldg(V + (size_t)s * 12 + be * 3 + d);
            v[d] = C{z.x, z.y};
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) fma_c(out[d], w, v[d]);
    }
}
// the same of U^+ V(s, beta)
LYM_D void spin_comb_dag(const C T[4][4], int al, C coef, const M3 &U, const double2 *V, int s, C out[3])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = C{0.0, 0.0};
#pragma unroll 1
    for (int be = 0; be < 4; ++be) {
        const C w = coef * T[al][be];
        if (w.re == 0.0 && w.im == 0.0) continue;
        C v[3], u[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double2 z = __ldg(V + (size_t)s * 12 + be * 3 + d);
            v[d] = C{z.x, z.y};
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            C t{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 3; ++k) fma_cc(t, U.a[k][i], v[k]);
            u[i] = t;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) fma_c(out[d], w, u[d]);
    }
}

template <class Gauge> __global__ void __launch_bounds__(128) fermion_force_kernel(ForceArg a, Gauge U)
{
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 4L * a.g.V) return;
    const int site = (int)(tid >> 2), mu = (int)(tid & 3);
    const Ctx<Gauge> cx_{a, U};
    M3 F;  // sum_i w_i F_i, Wilson part first
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) F.a[i][j] = C{0.0, 0.0};
    const int xp = cx_.shift(site, mu, +1);
    const M3 Um = cx_.link(site, mu);
    // DiracWilsonFermionForce::derivative
#pragma unroll 1
    for (int i = 0; i < a.n; ++i) {
        const double2 *X = a.X[i], *Y = a.Y[i];
        const C mk{-a.kappa * a.w[i], 0.0};
#pragma unroll 1
        for (int pass = 0; pass < 2; ++pass) {  // (X, Y), then X and Y exchanged
            const double2 *A = pass ? Y : X, *B = pass ? X : Y;
#pragma unroll 1
            for (int al = 0; al < 4; ++al) {
                C t[3], u[3], v[3];
                spin_comb(c_ft.mg[mu], al, mk, B, xp, t);
                Ctx<Gauge>::colour(A, site, al, v);
                add_tensor(F, 1.0, v, t);
                spin_comb_dag(c_ft.pg[mu], al, mk, Um, B, site, t);
                Ctx<Gauge>::colour(A, xp, al, v);
                mv(Um, v, u);
                add_tensor(F, -1.0, u, t);
            }
        }
    }
    if (a.clover) {
        // ImprovedFermionForce::derivative: term k of plane (mu, nu) adds sign_k L_k N^{mu nu}(x_k) R_k^+
        // (N from clover_outer_kernel: the spin traces of both pair orders, weights included);
        // the clover sum / 4
        M3 Fc;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Fc.a[i][j] = C{0.0, 0.0};
#pragma unroll 1
        for (int nu = 0; nu < 4; ++nu) {
            if (nu == mu) continue;
            const int plane = plane_index(mu, nu);
            const double sgn = mu < nu ? 1.0 : -1.0;  // N^{nu mu} = -N^{mu nu}
            const int xpn = cx_.shift(site, nu, +1), xmn = cx_.shift(site, nu, -1);
            const int xpm_mn = cx_.shift(site, mu, +1, nu, -1), xpm_pn = cx_.shift(site, mu, +1, nu, +1);
            auto add = [&](double sg, const M3 &M) {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) Fc.a[i][j] = Fc.a[i][j] + (sg * sgn) * M.a[i][j];
            };
            // the terms in an order that shares their link products (k = term of
            // ImprovedFermionForce.cpp; L_k, R_k its matrices): A = U_nu(x+mu) U_mu(x+nu)^+
            {
                const M3 Unu_x = cx_.link(site, nu);
                const M3 A = mul(cx_.link(xp, nu), dag(cx_.link(xpn, mu)));
                add(+1.0, mul(mul(A, load_plane(a.N, xpn, plane)), dag(Unu_x)));  // k=2: L=A, R=U_nu(x)
                add(+1.0, mul(mul(A, dag(Unu_x)), load_plane(a.N, site, plane)));  // k=0: L=A U_nu(x)^+
            }
            {
                // D = U_nu(x) U_mu(x+nu)
                const M3 Unu_xpm = cx_.link(xp, nu);
                const M3 D = mul(cx_.link(site, nu), cx_.link(xpn, mu));
                add(+1.0, mul(mul(Unu_xpm, load_plane(a.N, xpm_pn, plane)), dag(D)));  // k=6: L=U_nu(x+mu), R=D
                add(+1.0, mul(load_plane(a.N, xp, plane), dag(mul(D, dag(Unu_xpm)))));  // k=4: R=D U_nu(x+mu)^+
            }
            {
                // C = U_mu(x)^+ U_nu(x-nu)^+, R7 = U_mu(x) U_nu(x+mu-nu)^+, B = R7 U_mu(x-nu)^+
                const M3 Umu_xmn = cx_.link(xmn, mu), Unu_xmn = cx_.link(xmn, nu), Unu_xpm_mn = cx_.link(xpm_mn, nu);
                const M3 C = mul(dag(Um), dag(Unu_xmn));
                const M3 R7 = mul(Um, dag(Unu_xpm_mn));
                const M3 L7 = mul(C, Umu_xmn);
                add(-1.0, mul(mul(L7, load_plane(a.N, xpm_mn, plane)), dag(R7)));  // k=7
                add(-1.0, mul(mul(mul(L7, Unu_xpm_mn), load_plane(a.N, xp, plane)), dag(Um)));  // k=5: L=L7 U_nu(x+mu-nu), R=U_mu(x)
                const M3 B = mul(R7, dag(Umu_xmn));
                add(-1.0, mul(mul(C, load_plane(a.N, xmn, plane)), dag(B)));  // k=3: L=C, R=B
                add(-1.0, mul(mul(dag(Um), load_plane(a.N, site, plane)), dag(mul(B, Unu_xmn))));  // k=1: L=U_mu(x)^+, R=B U_nu(x-nu)
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
            w.x -= F.a[i][j].re;
            w.y -= F.a[i][j].im;
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

size_t fermion_force_scratch_bytes(const Geom &g) { return (size_t)g.V * 6 * 9 * sizeof(double2); }

void launch_fermion_force(const Geom &g, const GaugeDev &U, int n, const double2 *const *X, const double2 *const *Y,
                          const double *weights, double kappa, double csw, int clover, double2 *force,
                          double2 *scratch, cudaStream_t st)
{
    upload_tables(st);
    ForceArg a{g, n, X, Y, weights, force, scratch, kappa, csw, clover};
    if (clover) clover_outer_kernel<<<(int)((6L * g.V + 127) / 128), 128, 0, st>>>(a, scratch);
    const long threads = 4L * g.V;
    const int grid = (int)((threads + 127) / 128);
    if (U.rep == REP_SU3)
        fermion_force_kernel<GaugeD18><<<grid, 128, 0, st>>>(a, GaugeD18{(const double2 *)U.d64, g.stride});
    else
        fermion_force_kernel<GaugeD9><<<grid, 128, 0, st>>>(a, GaugeD9{(const double *)U.d64, g.stride});
}

}  // namespace lym
