// Fused vector steps of the Krylov solvers.  Each functor is run by site_kernel
// (lym_blas.cuh); finalize() runs once, in the last block, with the global sums
// and advances the solver's FP64 scalar state held in device memory.
#pragma once

#include "lym_blas.cuh"

namespace lym {

// ------------------------------------------------------------------ state --
struct CGState {
    double rr;         // |r|^2 of the recursion
    double rr_prev;    // |r|^2 before the last update (reliable-update beta)
    double rr_max;     // max |r|^2 since the last reliable update
    double eps;        // stop: rr < eps
    double delta2;     // reliable update when rr < delta2 * rr_max (0: never)
    double2 alpha;
    double beta;
    int iter;
    int max_iter;
    int pause;         // gates every captured kernel
    int converged;
    int need_update;
    int failed;
};

struct BiCGState {
    double2 rho;       // rho_{k-1}
    double2 rho_next;
    double2 alpha;
    double2 omega;
    double2 beta;
    double norm;       // |r|^2
    double precision;
    double last_error;
    int step;
    int max_steps;
    int pause;
    int converged;
    int breakdown;     // rho == 0 (BiConjugateGradient.cpp:381-384)
    int degenerate;    // (t,t) == 0: solution = source (BiConjugateGradient.cpp:455-464)
};

// ------------------------------------------------------------ simple ops ---
template <class SA, class SB> struct OpDot {  // sum conj(a) b -> out[0..1]
    static constexpr int NRED = 2;
    SA a;
    SB b;
    double *out;
    LYM_D void site(int p, int h, double *acc) const
    {
        cx<double> x[12], y[12];
        a.par(p).template load<double>(h, x);
        b.par(p).template load<double>(h, y);
        dotc(x, y, acc[0], acc[1]);
    }
    LYM_D void finalize(const double *t) const
    {
        out[0] = t[0];
        out[1] = t[1];
    }
};

// x += a, a = 0: a reduced-precision solution accumulator folded into the FP64 solution
template <class SA, class SX> struct OpFoldClear {
    static constexpr int NRED = 0;
    SA a;
    SX x;
    LYM_D void site(int p, int h, double *) const  // one component at a time
    {
        const SA ap = a.par(p);
        const SX xp = x.par(p);
#pragma unroll 4
        for (int k = 0; k < 12; ++k) {
            const cx<double> av = ap.get(k, h);
            xp.put(k, h, xp.get(k, h) + av);
            ap.put(k, h, cx<double>{0.0, 0.0});
        }
    }
};

// BiCGStab going on after a reliable update with the true residual rt in place of the
// recursive r: p += rt - r, r = rt; out = (<rh, rt>, <w, p>) with p as stored
template <class SR, class SP, class ST, class SH, class SW> struct OpBiContinue {
    static constexpr int NRED = 4;
    SR r;
    SP p;
    ST rt;
    SH rh;
    SW w;
    double *out;
    LYM_D void site(int q, int h, double *acc) const
    {
        if constexpr (SP::kPerComponent) {
            // FP32 direction (pair-layout r and p): two components at a time, every load of
            // both issued before their stores; r and p are read and written as whole 16-byte
            // words, the pair mate's lane written back as read (the batched loop is paused
            // during a reliable update, so nothing else writes those words).  The stored
            // direction is pn rounded to FP32, formed in registers.
#pragma unroll
            for (int k0 = 0; k0 < 12; k0 += 2) {
                float4 rw[2], pw[2];
                cx<double> tv[2], hv[2], wv[2];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    rw[i] = r.par(q).word(k0 + i, h);
                    pw[i] = p.par(q).word(k0 + i, h);
                    tv[i] = rt.par(q).get(k0 + i, h);
                    hv[i] = rh.par(q).get(k0 + i, h);
                    wv[i] = w.par(q).get(k0 + i, h);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const cx<double> rv = r.lane(rw[i]);
                    const cx<double> pn = p.lane(pw[i]) + tv[i] - rv;
                    p.par(q).put_word(k0 + i, h, p.with(pw[i], pn));
                    r.par(q).put_word(k0 + i, h, r.with(rw[i], tv[i]));
                    const cx<double> ps{(double)(float)pn.re, (double)(float)pn.im};
                    acc[0] += hv[i].re * tv[i].re + hv[i].im * tv[i].im;
                    acc[1] += hv[i].re * tv[i].im - hv[i].im * tv[i].re;
                    acc[2] += wv[i].re * ps.re + wv[i].im * ps.im;
                    acc[3] += wv[i].re * ps.im - wv[i].im * ps.re;
                }
            }
            return;
        }
        cx<double> rv[12], pv[12], tv[12];
        r.par(q).template load<double>(h, rv);
        p.par(q).template load<double>(h, pv);
        rt.par(q).template load<double>(h, tv);
#pragma unroll
        for (int k = 0; k < 12; ++k) pv[k] = pv[k] + tv[k] - rv[k];
        p.par(q).template store<double>(h, pv);
        r.par(q).template store<double>(h, tv);
        p.par(q).template load<double>(h, pv);  // the stored direction
        rh.par(q).template load<double>(h, rv);
        dotc(rv, tv, acc[0], acc[1]);
        w.par(q).template load<double>(h, rv);
        dotc(rv, pv, acc[2], acc[3]);
    }
    LYM_D void finalize(const double *t) const
    {
        for (int k = 0; k < 4; ++k) out[k] = t[k];
    }
};

// CG going on after a reliable update: r = rt, p = rt + b p
template <class SR, class SP, class ST> struct OpCGContinue {
    static constexpr int NRED = 0;
    SR r;
    SP p;
    ST rt;
    double b;
    LYM_D void site(int q, int h, double *) const
    {
        cx<double> pv[12], tv[12];
        p.par(q).template load<double>(h, pv);
        rt.par(q).template load<double>(h, tv);
#pragma unroll
        for (int k = 0; k < 12; ++k) pv[k] = tv[k] + b * pv[k];
        p.par(q).template store<double>(h, pv);
        r.par(q).template store<double>(h, tv);
    }
};

template <class SA> struct OpNorm {
    static constexpr int NRED = 1;
    SA a;
    double *out;
    LYM_D void site(int p, int h, double *acc) const
    {
        cx<double> x[12];
        a.par(p).template load<double>(h, x);
        acc[0] += norm2(x);
    }
    LYM_D void finalize(const double *t) const { out[0] = t[0]; }
};

// y = a x + b y   (complex a, b from host constants)
template <class SX, class SY> struct OpAxpby {
    static constexpr int NRED = 0;
    SX x;
    SY y;
    double2 a, b;
    LYM_D void site(int p, int h, double *) const
    {
        // a term with a zero coefficient is not read: y = a x overwrites y whatever it held
        const bool use_x = a.x != 0.0 || a.y != 0.0, use_y = b.x != 0.0 || b.y != 0.0;
        cx<double> u[12], v[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) u[k] = v[k] = cx<double>{0.0, 0.0};
        if (use_x) x.par(p).template load<double>(h, u);
        if (use_y) y.par(p).template load<double>(h, v);
        const cx<double> A = {a.x, a.y}, B = {b.x, b.y};
#pragma unroll
        for (int k = 0; k < 12; ++k) v[k] = (use_x ? A * u[k] : cx<double>{0.0, 0.0}) + (use_y ? B * v[k] : cx<double>{0.0, 0.0});
        y.par(p).template store<double>(h, v);
    }
    LYM_D void finalize(const double *) const {}
};

// z = x - y,  out = |z|^2
template <class SX, class SY, class SZ> struct OpSubNorm {
    static constexpr int NRED = 1;
    SX x;
    SY y;
    SZ z;
    double *out;
    LYM_D void site(int p, int h, double *acc) const
    {
        cx<double> u[12], v[12];
        x.par(p).template load<double>(h, u);
        y.par(p).template load<double>(h, v);
#pragma unroll
        for (int k = 0; k < 12; ++k) u[k] = u[k] - v[k];
        acc[0] += norm2(u);
        z.par(p).template store<double>(h, u);
    }
    LYM_D void finalize(const double *t) const { out[0] = t[0]; }
};

// gamma5 in place on one view (lower spins negated)
template <class SX> struct OpGamma5 {
    static constexpr int NRED = 0;
    SX x;
    LYM_D void site(int p, int h, double *) const
    {
        cx<double> u[12];
        x.par(p).template load<double>(h, u);
#pragma unroll
        for (int k = 6; k < 12; ++k) u[k] = -u[k];
        x.par(p).template store<double>(h, u);
    }
    LYM_D void finalize(const double *) const {}
};

// ------------------------------------------------------------------- CG ----
// alpha = rr / <p, Ap>  (ConjugateGradient.cpp:44-45)
template <class SP, class SAp> struct OpCGAlpha {
    static constexpr int NRED = 2;
    SP p;
    SAp ap;
    CGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> x[12], y[12];
        p.par(q).template load<double>(h, x);
        ap.par(q).template load<double>(h, y);
        dotc(x, y, acc[0], acc[1]);
    }
    LYM_D void finalize(const double *t) const { s->alpha = cdiv(make_double2(s->rr, 0.0), make_double2(t[0], t[1])); }
};

// x += alpha p ; r -= alpha Ap ; rr_new = |r|^2 (ConjugateGradient.cpp:47-68)
template <class SX, class SP, class SR, class SAp> struct OpCGUpdate {
    static constexpr int NRED = 1;
    SX x;
    SP p;
    SR r;
    SAp ap;
    CGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        const cx<double> al = {s->alpha.x, s->alpha.y};
        cx<double> xv[12], pv[12], rv[12], av[12];
        x.par(q).template load<double>(h, xv);
        p.par(q).template load<double>(h, pv);
        r.par(q).template load<double>(h, rv);
        ap.par(q).template load<double>(h, av);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            fma_c(xv[k], al, pv[k]);
            rv[k] = rv[k] - al * av[k];
        }
        acc[0] += norm2(rv);
        x.par(q).template store<double>(h, xv);
        r.par(q).template store<double>(h, rv);
    }
    LYM_D void finalize(const double *t) const
    {
        const double rr_new = t[0];
        s->iter += 1;
        s->rr_prev = s->rr;
        s->beta = rr_new / s->rr;
        s->rr = rr_new;
        if (rr_new > s->rr_max) s->rr_max = rr_new;
        if (!(rr_new == rr_new)) {  // NaN
            s->failed = 1;
            s->pause = 1;
        } else if (rr_new < s->eps) {
            s->converged = 1;
            s->need_update = 1;
            s->pause = 1;
        } else if (s->delta2 > 0.0 && rr_new < s->delta2 * s->rr_max) {
            s->need_update = 1;
            s->pause = 1;
        } else if (s->iter >= s->max_iter) {
            s->pause = 1;
        }
    }
};

// p = r + beta p
template <class SP, class SR> struct OpCGDirection {
    static constexpr int NRED = 0;
    SP p;
    SR r;
    CGState *s;
    LYM_D void site(int q, int h, double *) const
    {
        const double b = s->beta;
        cx<double> pv[12], rv[12];
        p.par(q).template load<double>(h, pv);
        r.par(q).template load<double>(h, rv);
#pragma unroll
        for (int k = 0; k < 12; ++k) pv[k] = rv[k] + b * pv[k];
        p.par(q).template store<double>(h, pv);
    }
    LYM_D void finalize(const double *) const {}
};

// ------------------------------------------------------------- BiCGStab ----
// rho_next = <rhat, r>; beta = (rho_next / rho)(alpha / omega)  (BiConjugateGradient.cpp:359-387)
template <class SH, class SR> struct OpBiRho {
    static constexpr int NRED = 2;
    SH rhat;
    SR r;
    BiCGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> a[12], b[12];
        rhat.par(q).template load<double>(h, a);
        r.par(q).template load<double>(h, b);
        dotc(a, b, acc[0], acc[1]);
    }
    LYM_D void finalize(const double *t) const
    {
        const double2 rn = make_double2(t[0], t[1]);
        s->rho_next = rn;
        if (rn.x * rn.x + rn.y * rn.y == 0.0) {
            s->breakdown = 1;
            s->pause = 1;
            return;
        }
        s->beta = cmul(cdiv(rn, s->rho), cdiv(s->alpha, s->omega));
    }
};

// p = r + beta (p - omega nu)
template <class SP, class SR, class SN> struct OpBiDirection {
    static constexpr int NRED = 0;
    SP p;
    SR r;
    SN nu;
    BiCGState *s;
    LYM_D void site(int q, int h, double *) const
    {
        const cx<double> be = {s->beta.x, s->beta.y}, om = {s->omega.x, s->omega.y};
        cx<double> pv[12], rv[12], nv[12];
        p.par(q).template load<double>(h, pv);
        r.par(q).template load<double>(h, rv);
        nu.par(q).template load<double>(h, nv);
#pragma unroll
        for (int k = 0; k < 12; ++k) pv[k] = rv[k] + be * (pv[k] - om * nv[k]);
        p.par(q).template store<double>(h, pv);
    }
    LYM_D void finalize(const double *) const {}
};

// alpha = rho_next / <rhat, nu>
template <class SH, class SN> struct OpBiAlpha {
    static constexpr int NRED = 2;
    SH rhat;
    SN nu;
    BiCGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> a[12], b[12];
        rhat.par(q).template load<double>(h, a);
        nu.par(q).template load<double>(h, b);
        dotc(a, b, acc[0], acc[1]);
    }
    LYM_D void finalize(const double *t) const { s->alpha = cdiv(s->rho_next, make_double2(t[0], t[1])); }
};

// s = r - alpha nu
template <class SS, class SR, class SN> struct OpBiS {
    static constexpr int NRED = 0;
    SS sv;
    SR r;
    SN nu;
    BiCGState *s;
    LYM_D void site(int q, int h, double *) const
    {
        const cx<double> al = {s->alpha.x, s->alpha.y};
        cx<double> rv[12], nv[12];
        r.par(q).template load<double>(h, rv);
        nu.par(q).template load<double>(h, nv);
#pragma unroll
        for (int k = 0; k < 12; ++k) rv[k] = rv[k] - al * nv[k];
        sv.par(q).template store<double>(h, rv);
    }
    LYM_D void finalize(const double *) const {}
};

// omega = <t,s>/<t,t>
template <class ST, class SS> struct OpBiOmega {
    static constexpr int NRED = 4;
    ST t;
    SS sv;
    BiCGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> a[12], b[12];
        t.par(q).template load<double>(h, a);
        sv.par(q).template load<double>(h, b);
        dotc(a, b, acc[0], acc[1]);
        dotc(a, a, acc[2], acc[3]);
    }
    LYM_D void finalize(const double *t2) const
    {
        s->omega = cdiv(make_double2(t2[0], t2[1]), make_double2(t2[2], t2[3]));
        if (t2[2] == 0.0) {
            s->degenerate = 1;
            s->converged = 1;
            s->pause = 1;
        }
    }
};

// x += alpha p + omega s ; r = s - omega t ; norm = |r|^2 ; rho_next = <rhat, r> of the next step
template <class SX, class SP, class SS, class ST, class SR, class SH> struct OpBiUpdate {
    static constexpr int NRED = 3;
    SX x;
    SP p;
    SS sv;
    ST t;
    SR r;
    SH rhat;
    BiCGState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        const cx<double> al = {s->alpha.x, s->alpha.y}, om = {s->omega.x, s->omega.y};
        cx<double> xv[12], pv[12], sv_[12], tv[12], hv[12];
        x.par(q).template load<double>(h, xv);
        p.par(q).template load<double>(h, pv);
        sv.par(q).template load<double>(h, sv_);
        t.par(q).template load<double>(h, tv);
        rhat.par(q).template load<double>(h, hv);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            xv[k] = xv[k] + (al * pv[k] + om * sv_[k]);
            tv[k] = sv_[k] - om * tv[k];  // new residual
        }
        acc[0] += norm2(tv);
        dotc(hv, tv, acc[1], acc[2]);
        x.par(q).template store<double>(h, xv);
        r.par(q).template store<double>(h, tv);
    }
    LYM_D void finalize(const double *t3) const
    {
        const double norm = t3[0];
        s->norm = norm;
        if (!(norm == norm)) {
            s->breakdown = 1;
            s->pause = 1;
            return;
        }
        if (norm < s->precision) {
            s->converged = 1;
            s->pause = 1;
            s->last_error = norm;
            return;
        }
        s->rho = s->rho_next;
        s->last_error = norm;
        s->step += 1;
        if (s->step >= s->max_steps) {
            s->pause = 1;
            return;
        }
        // next step's rho_next and beta (fused OpBiRho)
        const double2 rn = make_double2(t3[1], t3[2]);
        s->rho_next = rn;
        if (rn.x * rn.x + rn.y * rn.y == 0.0) {
            s->breakdown = 1;
            s->pause = 1;
            return;
        }
        s->beta = cmul(cdiv(rn, s->rho), cdiv(s->alpha, s->omega));
    }
};

// ------------------------------------------------------ multishift CG ------
constexpr int kMaxShifts = 32;
constexpr int kMsWin = 8;  // steps per windowed update of the shifted x_i and p_i

struct MultishiftState {
    int pause;                    // first word: gates every captured kernel
    double sigma[kMaxShifts];     // shift relative to the base system: sigma_i - sigma_0
    double zeta[kMaxShifts];      // zeta_k
    double zeta_prev[kMaxShifts]; // zeta_{k-1}
    double alpha_s[kMaxShifts];
    double beta_s[kMaxShifts];
    int active[kMaxShifts];
    int nshift;
    int base;                     // index of the base system (smallest shift)
    double rr, rr_prev;
    double alpha, alpha_prev, beta;
    double eps;                   // per-shift stop: zeta_i^2 rr < eps
    int iter, max_iter, converged, stop;
    // mixed precision: reliable update of the base system when rr < delta2 * rr_max
    // (0: never); the step that sets need_update updates x but not the directions
    double delta2, rr_max;
    int need_update, failed;
    // windowed updates: the step within the window and, per shift, the coefficients of
    // x_i - x_i(window start) and of p_i on P_i (p_i at the window start, slot 0) and on
    // the window's residuals R_0..R_{win-1} (slots 1..win)
    int win;
    int xupd[kMaxShifts], pupd[kMaxShifts];
    double cx[kMaxShifts][kMsWin + 1], cp[kMaxShifts][kMsWin + 1];
};

// base alpha = rr / <p, Ap>, then the shifted coefficients (Jegerlehner recursions)
template <class SP, class SAp> struct OpMsAlpha {
    static constexpr int NRED = 2;
    SP p;
    SAp ap;
    MultishiftState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> x[12], y[12];
        p.par(q).template load<double>(h, x);
        ap.par(q).template load<double>(h, y);
        dotc(x, y, acc[0], acc[1]);
    }
    // On entry s->alpha = alpha_{k-1}, s->beta = beta_k (p_k = r_k + beta_k p_{k-1}),
    // zeta = zeta_k, zeta_prev = zeta_{k-1}.  For (A + sigma) with residuals
    // r^sigma_k = zeta_k r_k the three-term recurrences give
    //   zeta_{k+1} = zeta_k zeta_{k-1} a_{k-1} /
    //                (zeta_{k-1} a_{k-1} (1 + sigma a_k) + a_k b_k (zeta_{k-1} - zeta_k))
    //   a^sigma_k  = a_k zeta_{k+1} / zeta_k.
    LYM_D void finalize(const double *t) const
    {
        const double a = s->rr / t[0];
        const double am1 = s->alpha;
        for (int i = 0; i < s->nshift; ++i) {
            if (s->active[i] == 2) s->active[i] = 0;  // converged at the previous step
            if (!s->active[i]) continue;
            const double z = s->zeta[i], zp = s->zeta_prev[i];
            const double den = zp * am1 * (1.0 + s->sigma[i] * a) + a * s->beta * (zp - z);
            const double zn = (z * zp * am1) / den;
            s->alpha_s[i] = a * zn / z;
            s->zeta_prev[i] = z;
            s->zeta[i] = zn;
        }
        s->alpha_prev = am1;
        s->alpha = a;
    }
};

// After r_{k+1}: beta, the shifted betas, per-shift convergence, reliable-update and stop
// flags.  False when the residual is not finite (the state is paused).
LYM_D bool ms_residual_step(MultishiftState *s, double rr_new)
{
    s->iter += 1;
    s->beta = rr_new / s->rr;
    s->rr_prev = s->rr;
    s->rr = rr_new;
    if (rr_new > s->rr_max) s->rr_max = rr_new;
    if (!(rr_new == rr_new)) {  // NaN: stop before the update
        s->failed = 1;
        s->stop = 1;
        s->pause = 1;
        return false;
    }
    int any = 0;
    for (int i = 0; i < s->nshift; ++i) {
        if (!s->active[i]) continue;
        // residual of shift i after this step: zeta_{k+1} r_{k+1}
        const double zr = s->zeta[i] * s->zeta[i] * rr_new;
        s->beta_s[i] = s->beta * (s->zeta[i] / s->zeta_prev[i]) * (s->zeta[i] / s->zeta_prev[i]);
        // converged: this step's x update still runs, then the shift is frozen.
        // The base system (sigma 0, index base) keeps its direction p, which
        // drives the recursion of all the others.
        if (zr < s->eps && i != s->base) s->active[i] = 2;
        else if (zr >= s->eps) any = 1;
    }
    // the x / p update of this step (OpMsUpdate) still runs; it turns stop into pause
    if (!any) {
        s->converged = 1;
        s->stop = 1;
        s->need_update = s->delta2 > 0.0;
    } else if (s->delta2 > 0.0 && rr_new < s->delta2 * s->rr_max) {
        s->need_update = 1;
        s->stop = 1;
    } else if (s->iter >= s->max_iter) {
        s->stop = 1;
    }
    return true;
}

// x_i += alpha_i p_i ; r -= alpha Ap ; rr_new
template <class SR, class SAp> struct OpMsResidual {
    static constexpr int NRED = 1;
    SR r;
    SAp ap;
    MultishiftState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        const double a = s->alpha;
        cx<double> rv[12], av[12];
        r.par(q).template load<double>(h, rv);
        ap.par(q).template load<double>(h, av);
#pragma unroll
        for (int k = 0; k < 12; ++k) rv[k] = rv[k] - a * av[k];
        acc[0] += norm2(rv);
        r.par(q).template store<double>(h, rv);
    }
    LYM_D void finalize(const double *t) const { ms_residual_step(s, t[0]); }
};

// Windowed form of OpMsUpdate's step: x_i += alpha_i p_i and p_i = zeta_i R_m + beta_i p_i
// applied to the coefficients of x_i and p_i (same conditions as OpMsUpdate), R_m = r_{k+1}.
LYM_D void ms_window_step(MultishiftState *s)
{
    const int m = s->win;
    const bool dir = !s->need_update;
    for (int i = 0; i < s->nshift; ++i) {
        const int act = s->active[i];
        if (!act) continue;
        const double a = s->alpha_s[i];
        for (int j = 0; j <= m; ++j) s->cx[i][j] += a * s->cp[i][j];
        s->xupd[i] = 1;
        if (act == 1 && dir) {
            const double b = s->beta_s[i];
            for (int j = 0; j <= m; ++j) s->cp[i][j] *= b;
            s->cp[i][m + 1] = s->zeta[i];
            s->pupd[i] = 1;
        }
    }
    s->win = m + 1;
}

// r_{k+1} = r_k - alpha Ap with the residuals in a ring of kMsWin + 1 FP32 slots (r_k in
// slot k mod (kMsWin + 1)), |r_{k+1}|^2, then the step's scalars and window coefficients.
template <class SAp> struct OpMsResidualRing {
    static constexpr int NRED = 1;
    const SpinorF *ring;
    SAp ap;
    MultishiftState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        const int k = s->iter;
        const SpinorF rin = ring[k % (kMsWin + 1)], rout = ring[(k + 1) % (kMsWin + 1)];
        const double a = s->alpha;
        cx<double> rv[12], av[12];
        rin.par(q).template load<double>(h, rv);
        ap.par(q).template load<double>(h, av);
#pragma unroll
        for (int c = 0; c < 12; ++c) rv[c] = rv[c] - a * av[c];
        acc[0] += norm2(rv);
        rout.par(q).template store<double>(h, rv);
    }
    LYM_D void finalize(const double *t) const
    {
        if (ms_residual_step(s, t[0])) ms_window_step(s);
    }
};

// the base system's direction, materialised every step for the operator: p = r_{k+1} + beta p
// (not after a step that asks for a reliable update: the host rebuilds it from the true residual)
template <class SP> struct OpMsBaseDirection {
    static constexpr int NRED = 1;  // no sum; finalize ends the step
    const SpinorF *ring;
    SP p;
    MultishiftState *s;
    LYM_D void site(int q, int h, double *) const
    {
        if (s->need_update || s->active[s->base] != 1) return;
        const double b = s->beta;
        cx<double> rv[12], pv[12];
        ring[s->iter % (kMsWin + 1)].par(q).template load<double>(h, rv);
        p.par(q).template load<double>(h, pv);
#pragma unroll
        for (int c = 0; c < 12; ++c) pv[c] = rv[c] + b * pv[c];
        p.par(q).template store<double>(h, pv);
    }
    LYM_D void finalize(const double *) const
    {
        if (s->stop) s->pause = 1;
    }
};

// Window flush: per shift x_i += cx_i0 P_i + sum_j cx_i(j+1) R_j and (running shifts)
// P_i = cp_i0 P_i + sum_j cp_i(j+1) R_j, R_j = r_{k0+1+j}: one pass over x_i and P_i
// per window instead of one per step.  FP32 words streamed one at a time; coefficients in
// shared memory.  Runs whether or not the state is paused (a pause ends the window early).
struct MsFlushArg {
    const SpinorF *ring;  // kMsWin + 1 residual slots
    const SpinorF *x;     // per-shift FP32 solution accumulators
    const SpinorF *p;     // per-shift directions
    MultishiftState *s;
    int nshift;
    int vh;
};

constexpr int kMsFlushThreads = 256;

static __global__ void __launch_bounds__(kMsFlushThreads) ms_flush_kernel(MsFlushArg a)
{
    __shared__ float cxs[kMaxShifts][kMsWin + 1], cps[kMaxShifts][kMsWin + 1];
    __shared__ int fl[kMaxShifts];
    __shared__ float4 *xp[kMaxShifts], *pp[kMaxShifts], *rp[kMsWin];
    const MultishiftState *s = a.s;
    const int m = s->win;
    if (m == 0) return;
    const int k0 = s->iter - m;
    for (int t = threadIdx.x; t < a.nshift * (kMsWin + 1); t += blockDim.x) {
        const int i = t / (kMsWin + 1), j = t % (kMsWin + 1);
        cxs[i][j] = (float)s->cx[i][j];
        cps[i][j] = (float)s->cp[i][j];
    }
    for (int i = threadIdx.x; i < a.nshift; i += blockDim.x) {
        fl[i] = (s->xupd[i] ? 1 : 0) | ((s->pupd[i] && s->active[i] == 1) ? 2 : 0);
        xp[i] = a.x[i].v;
        pp[i] = a.p[i].v;
    }
    for (int j = threadIdx.x; j < m; j += blockDim.x) rp[j] = a.ring[(k0 + 1 + j) % (kMsWin + 1)].v;
    __syncthreads();
    const int stride = a.ring[0].stride;
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < a.vh; h += gridDim.x * blockDim.x) {
        for (int w = 0; w < 6; ++w) {
            const size_t o = (size_t)w * stride + h;
            float4 R[kMsWin];
#pragma unroll
            for (int j = 0; j < kMsWin; ++j)
                if (j < m) R[j] = rp[j][o];
            for (int i = 0; i < a.nshift; ++i) {
                const int f = fl[i];
                if (!f) continue;
                const float4 P = pp[i][o];
                float4 X = xp[i][o], Q;
                const float c0 = cxs[i][0], d0 = cps[i][0];
                X.x += c0 * P.x; X.y += c0 * P.y; X.z += c0 * P.z; X.w += c0 * P.w;
                Q.x = d0 * P.x; Q.y = d0 * P.y; Q.z = d0 * P.z; Q.w = d0 * P.w;
#pragma unroll
                for (int j = 0; j < kMsWin; ++j) {
                    if (j < m) {
                        const float c = cxs[i][j + 1], d = cps[i][j + 1];
                        X.x += c * R[j].x; X.y += c * R[j].y; X.z += c * R[j].z; X.w += c * R[j].w;
                        Q.x += d * R[j].x; Q.y += d * R[j].y; Q.z += d * R[j].z; Q.w += d * R[j].w;
                    }
                }
                xp[i][o] = X;
                if (f & 2) pp[i][o] = Q;
            }
        }
    }
}

// start a new window (after the flush)
static __global__ void ms_window_reset_kernel(MultishiftState *s, int nshift)
{
    const int i = threadIdx.x;
    if (i < nshift) {
        s->xupd[i] = s->pupd[i] = 0;
        for (int j = 0; j <= kMsWin; ++j) s->cx[i][j] = s->cp[i][j] = 0.0;
        s->cp[i][0] = 1.0;
    }
    if (i == 0) s->win = 0;
}

// per shift: x_i += alpha_i p_i ; p_i = zeta_i r + beta_i p_i  (one launch over all shifts;
// a step that asks for a reliable update leaves the directions to OpMsDirection)
template <class SX, class SP = SX, class SR = SX> struct OpMsUpdate {
    static constexpr int NRED = 1;  // no sum; finalize ends the step
    SX *x;   // device array of nshift views
    SP *ps;
    SR r;
    MultishiftState *s;
    int nshift;
    LYM_D void site(int q, int h, double *) const
    {
        cx<double> rv[12];
        const bool dir = !s->need_update;
        if (dir) r.par(q).template load<double>(h, rv);
        for (int i = 0; i < nshift; ++i) {
            const int act = s->active[i];
            if (!act) continue;
            cx<double> xv[12], pv[12];
            x[i].par(q).template load<double>(h, xv);
            ps[i].par(q).template load<double>(h, pv);
            const double ai = s->alpha_s[i];
#pragma unroll
            for (int k = 0; k < 12; ++k) fma_r(xv[k], ai, pv[k]);
            x[i].par(q).template store<double>(h, xv);
            if (act == 1 && dir) {
                const double z = s->zeta[i], b = s->beta_s[i];
#pragma unroll
                for (int k = 0; k < 12; ++k) pv[k] = z * rv[k] + b * pv[k];
                ps[i].par(q).template store<double>(h, pv);
            }
        }
    }
    LYM_D void finalize(const double *) const
    {
        if (s->stop) s->pause = 1;
    }
};

// p_i = zeta_i r + beta_i p_i for the running shifts (after a reliable update of r)
template <class SP, class SR> struct OpMsDirection {
    static constexpr int NRED = 0;
    SP *ps;
    SR r;
    MultishiftState *s;
    int nshift;
    LYM_D void site(int q, int h, double *) const
    {
        cx<double> rv[12];
        r.par(q).template load<double>(h, rv);
        for (int i = 0; i < nshift; ++i) {
            if (s->active[i] != 1) continue;
            cx<double> pv[12];
            ps[i].par(q).template load<double>(h, pv);
            const double z = s->zeta[i], b = s->beta_s[i];
#pragma unroll
            for (int k = 0; k < 12; ++k) pv[k] = z * rv[k] + b * pv[k];
            ps[i].par(q).template store<double>(h, pv);
        }
    }
};

// --------------------------------------------- multishift minimal residual --
// MMMRMultishiftSolver::solve, non-ALIGNED_OPT branch (inverters/MMMRMultishiftSolver.cpp:123-198)
struct MMMRState {
    int pause;
    int nshift, first, iter, max_iter, converged;
    double sigma[kMaxShifts];   // shifts[i] - shifts.back()
    double2 f[kMaxShifts];
    double2 coef[kMaxShifts];   // x_i += coef_i r
    double2 alpha;
    double omega;               // over-relaxation 0.95 (MMMRMultishiftSolver.cpp:37)
    double eps;
    double rr;
};

// alpha = omega <p,r>/<p,p>; f_i = f_i / (1 + (s_i - s_last) alpha)
template <class SP, class SR> struct OpMMMRAlpha {
    static constexpr int NRED = 4;
    SP p;
    SR r;
    MMMRState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> a[12], b[12];
        p.par(q).template load<double>(h, a);
        r.par(q).template load<double>(h, b);
        dotc(a, b, acc[0], acc[1]);
        dotc(a, a, acc[2], acc[3]);
    }
    LYM_D void finalize(const double *t) const
    {
        const double2 al = cscale(s->omega, cdiv(make_double2(t[0], t[1]), make_double2(t[2], t[3])));
        s->alpha = al;
        const int last = s->nshift - 1;
        s->coef[last] = al;
        for (int i = s->first; i < last; ++i) {
            s->f[i] = cdiv(s->f[i], cadd(make_double2(1.0, 0.0), cscale(s->sigma[i], al)));
            s->coef[i] = cmul(s->f[i], al);
        }
    }
};

// x_i += coef_i r (i >= first) ; r -= alpha p ; error = |r|^2
template <class SV> struct OpMMMRUpdate {
    static constexpr int NRED = 1;
    SV *x;
    SV r;
    SV p;
    MMMRState *s;
    LYM_D void site(int q, int h, double *acc) const
    {
        cx<double> rv[12], pv[12];
        r.par(q).template load<double>(h, rv);
        p.par(q).template load<double>(h, pv);
        for (int i = s->first; i < s->nshift; ++i) {
            cx<double> xv[12];
            x[i].par(q).template load<double>(h, xv);
            const cx<double> cf = {s->coef[i].x, s->coef[i].y};
#pragma unroll
            for (int k = 0; k < 12; ++k) fma_c(xv[k], cf, rv[k]);
            x[i].par(q).template store<double>(h, xv);
        }
        const cx<double> al = {s->alpha.x, s->alpha.y};
#pragma unroll
        for (int k = 0; k < 12; ++k) rv[k] = rv[k] - al * pv[k];
        acc[0] += norm2(rv);
        r.par(q).template store<double>(h, rv);
    }
    LYM_D void finalize(const double *t) const
    {
        s->rr = t[0];
        s->iter += 1;
        if (t[0] < s->eps) {
            s->converged = 1;
            s->pause = 1;
        } else if (s->iter >= s->max_iter || !(t[0] == t[0])) {
            s->pause = 1;
        }
    }
};

}  // namespace lym
