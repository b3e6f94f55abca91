/*
 * FP64 discrete adjoint of the step -- TEST INFRASTRUCTURE ONLY (see
 * lbm_oracle.h: never linked into or called from the product library).
 *
 * The reference has no adjoint (nor gray LBM).  This file states, in double
 * precision and in the parity-free "logical" form, the forward step the
 * oracle's ora_step performs for the features the adjoint supports, and its
 * discrete adjoint:
 *
 *   forward   x^t(n,i) = C(x^{t-1}(n - c_i))_i     if n - c_i is fluid
 *                      = C(x^{t-1}(n))_{opp i}      otherwise (half-way bounce-back)
 *   adjoint   mu(m,k)  = lambda^t(m + c_k, k)      if m + c_k is fluid
 *                      = lambda^t(m, opp k)          otherwise
 *             lambda^{t-1}(m,.) = [dC/dx (x^{t-1}(m,.))]^T mu(m,.)
 *             dJ/dn_s(m) += mu(m,.) . dC/dn_s,   dJ/dtau += mu(m,.) . dC/dtau
 *
 * x^t are the populations a cell gathers at step t+1 (what ora_logical
 * returns after t steps) and C is the per-cell collision of lbm_oracle_body.inc
 * (BGK esoteric_pull.hpp:408-432 or TRT one_step_pull.hpp:187-204, Guo
 * forcing esoteric_pull.hpp:55-70) followed by gray-LBM partial bounce-back
 * C_i = (1 - n_s) f*_i + n_s x_{opp i} (Walsh, Burwinkle & Saar 2009).
 *
 * Jacobian of C at x (rho = sum x, u~ = j / rho, u = u~ + a/2, F = rho a):
 *   dC_i/dx_k = (1 - n_s) [A_ik + dG_i/drho + dG_i/du . (c_k - u~) / rho] + n_s delta(opp i, k)
 *   A_ik = delta_ik (1 - (w+ + w-)/2) - delta(opp i, k) (w+ - w-)/2
 *   G_i  = w+ feq+_i + w- feq-_i + (1 - w+/2) F+_i + (1 - w-/2) F-_i
 * (w+-: relaxation rates; +/-: parts even/odd in c).  Every G_i is linear in
 * rho at fixed u, so sum_i mu_i dG_i/drho = sum_i mu_i G_i / rho, and both
 * contractions reduce to the moments m0 = sum w mu, m = sum w mu c,
 * M = sum w mu c c^T.  Smagorinsky LES and moving walls are outside the
 * adjoint's scope (rejected).
 *
 * All forward states are kept in memory: the oracle's lattices are small.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const int a_cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
static const int a_cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
static const int a_cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};

typedef struct {
    int q;
    double w[27];
    int opp[27];
    double wp, wm, gp, gm; /* relaxation rates and Guo prefactors */
    double dwp, dwm;       /* d(omega+)/dtau, d(omega-)/dtau */
} adj_lattice;

static int adj_setup(const ora_cfg* c, adj_lattice* L) {
    if (!c || (c->q != 19 && c->q != 27)) return 1;
    if (!(c->tau > 0.5) || c->les_k != 0.0) return 1;
    if (c->flags) {
        const size_t N = c->nx * c->ny * c->nz;
        for (size_t n = 0; n < N; ++n)
            if (c->flags[n] > ORA_WALL) return 1; /* moving walls: not in the adjoint's scope */
    }
    L->q = c->q;
    for (int d = 0; d < c->q; ++d) {
        const int len2 = a_cx[d] * a_cx[d] + a_cy[d] * a_cy[d] + a_cz[d] * a_cz[d];
        if (c->q == 19)
            L->w[d] = len2 == 0 ? 1.0 / 3.0 : (len2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
        else
            L->w[d] = len2 == 0 ? 8.0 / 27.0 : (len2 == 1 ? 2.0 / 27.0 : (len2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
        L->opp[d] = d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1);
    }
    const double tau = c->tau;
    L->wp = 1.0 / tau;
    L->dwp = -L->wp * L->wp;
    if (c->collision == ORA_BGK) {
        L->wm = L->wp;
        L->dwm = L->dwp;
    } else if (c->tau_minus > 0.0) {
        L->wm = 1.0 / c->tau_minus;
        L->dwm = 0.0;
    } else {
        const double taum = 0.5 + c->trt_magic / (tau - 0.5);
        L->wm = 1.0 / taum;
        L->dwm = L->wm * L->wm * c->trt_magic / ((tau - 0.5) * (tau - 0.5));
    }
    L->gp = 1.0 - 0.5 * L->wp;
    L->gm = 1.0 - 0.5 * L->wm;
    return 0;
}

static size_t adj_wrap(size_t c, int d, size_t e) {
    if (d > 0) return c + 1U == e ? 0U : c + 1U;
    if (d < 0) return c == 0U ? e - 1U : c - 1U;
    return c;
}

/* n + s * c_d with periodic wrap. */
static size_t adj_nbr(const ora_cfg* c, size_t n, int d, int s) {
    const size_t x = n % c->nx, y = (n / c->nx) % c->ny, z = n / (c->nx * c->ny);
    const size_t xn = adj_wrap(x, s * a_cx[d], c->nx);
    const size_t yn = adj_wrap(y, s * a_cy[d], c->ny);
    const size_t zn = adj_wrap(z, s * a_cz[d], c->nz);
    return (zn * c->ny + yn) * c->nx + xn;
}

static int adj_fluid(const ora_cfg* c, size_t n) { return !c->flags || c->flags[n] == ORA_FLUID; }

typedef struct {
    double rho, ut[3], u[3], a[3], F[3];
    double feq[27], Fi[27]; /* equilibrium and Guo source (c - u) . F, 9 (c.u)(c.F) terms */
    double fstar[27];       /* post-TRT, before gray mixing */
    double ns;
} adj_cell;

static void adj_collide(const adj_lattice* L, const ora_cfg* c, size_t n, const double* x, double* out,
                        adj_cell* s) {
    const size_t N = c->nx * c->ny * c->nz;
    double rho = 0.0, j[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < L->q; ++d) {
        rho += x[d];
        j[0] += a_cx[d] * x[d];
        j[1] += a_cy[d] * x[d];
        j[2] += a_cz[d] * x[d];
    }
    s->rho = rho;
    s->a[0] = c->ax + (c->local_a ? (double)c->local_a[n] : 0.0);
    s->a[1] = c->ay + (c->local_a ? (double)c->local_a[N + n] : 0.0);
    s->a[2] = c->az + (c->local_a ? (double)c->local_a[2 * N + n] : 0.0);
    for (int b = 0; b < 3; ++b) {
        s->ut[b] = j[b] / rho;
        s->u[b] = s->ut[b] + 0.5 * s->a[b];
        s->F[b] = rho * s->a[b];
    }
    const double* u = s->u;
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double uF = u[0] * s->F[0] + u[1] * s->F[1] + u[2] * s->F[2];
    for (int d = 0; d < L->q; ++d) {
        const double cu = a_cx[d] * u[0] + a_cy[d] * u[1] + a_cz[d] * u[2];
        const double cF = a_cx[d] * s->F[0] + a_cy[d] * s->F[1] + a_cz[d] * s->F[2];
        s->feq[d] = L->w[d] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
        s->Fi[d] = L->w[d] * (3.0 * (cF - uF) + 9.0 * cu * cF);
    }
    for (int d = 0; d < L->q; ++d) {
        const int o = L->opp[d];
        const double even = 0.5 * ((x[d] - s->feq[d]) + (x[o] - s->feq[o]));
        const double oddp = 0.5 * ((x[d] - s->feq[d]) - (x[o] - s->feq[o]));
        const double fe = 0.5 * (s->Fi[d] + s->Fi[o]), fo = 0.5 * (s->Fi[d] - s->Fi[o]);
        s->fstar[d] = x[d] - L->wp * even - L->wm * oddp + L->gp * fe + L->gm * fo;
    }
    s->ns = c->solid_fraction ? (double)c->solid_fraction[n] : 0.0;
    for (int d = 0; d < L->q; ++d) out[d] = (1.0 - s->ns) * s->fstar[d] + s->ns * x[L->opp[d]];
}

/* One logical forward step: x (q*N, [d][n]) -> y. */
static void adj_forward_step(const adj_lattice* L, const ora_cfg* c, const double* x, double* y) {
    const size_t N = c->nx * c->ny * c->nz;
    double xi[27], out[27];
    adj_cell s;
    memset(y, 0, sizeof(double) * (size_t)L->q * N);
    for (size_t m = 0; m < N; ++m) {
        if (!adj_fluid(c, m)) continue;
        for (int d = 0; d < L->q; ++d) xi[d] = x[(size_t)d * N + m];
        adj_collide(L, c, m, xi, out, &s);
        for (int k = 0; k < L->q; ++k) {
            const size_t dst = adj_nbr(c, m, k, +1);
            if (adj_fluid(c, dst))
                y[(size_t)k * N + dst] = out[k];
            else
                y[(size_t)L->opp[k] * N + m] = out[k];
        }
    }
}

int ora_adjoint_forward(const ora_cfg* c, const double* x0, uint64_t steps, double* x_end) {
    adj_lattice L;
    if (adj_setup(c, &L)) return 1;
    const size_t N = c->nx * c->ny * c->nz, bytes = sizeof(double) * (size_t)c->q * N;
    double* a = (double*)malloc(bytes);
    double* b = (double*)malloc(bytes);
    if (!a || !b) {
        free(a);
        free(b);
        return 2;
    }
    memcpy(a, x0, bytes);
    for (uint64_t t = 0; t < steps; ++t) {
        adj_forward_step(&L, c, a, b);
        double* tmp = a;
        a = b;
        b = tmp;
    }
    memcpy(x_end, a, bytes);
    free(a);
    free(b);
    return 0;
}

/* lambda = [dC/dx]^T mu at the cell state s (computed by adj_collide at x);
 * also the n_s and tau derivatives of mu . C. */
static void adj_cell_transpose(const adj_lattice* L, const double* x, const adj_cell* s, const double* mu,
                               double* lam, double* g_ns, double* g_tau) {
    const int q = L->q;
    const double* u = s->u;
    const double* ut = s->ut;
    const double* a = s->a;
    double m0 = 0.0, m[3] = {0, 0, 0}, M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int d = 0; d < q; ++d) {
        const double wm = L->w[d] * mu[d];
        const double e[3] = {(double)a_cx[d], (double)a_cy[d], (double)a_cz[d]};
        m0 += wm;
        for (int p = 0; p < 3; ++p) {
            m[p] += wm * e[p];
            for (int r = 0; r < 3; ++r) M[p][r] += wm * e[p] * e[r];
        }
    }
    double Mu[3], Ma[3];
    for (int p = 0; p < 3; ++p) {
        Mu[p] = M[p][0] * u[0] + M[p][1] * u[1] + M[p][2] * u[2];
        Ma[p] = M[p][0] * a[0] + M[p][1] * a[1] + M[p][2] * a[2];
    }
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double ua = u[0] * a[0] + u[1] * a[1] + u[2] * a[2];
    const double uMu = u[0] * Mu[0] + u[1] * Mu[1] + u[2] * Mu[2];
    const double uMa = u[0] * Ma[0] + u[1] * Ma[1] + u[2] * Ma[2];
    const double mu_ = m[0] * u[0] + m[1] * u[1] + m[2] * u[2];
    const double ma = m[0] * a[0] + m[1] * a[1] + m[2] * a[2];
    const double P = L->wp * (m0 * (1.0 - 1.5 * uu) + 4.5 * uMu) + 3.0 * L->wm * mu_ +
                     L->gp * (9.0 * uMa - 3.0 * m0 * ua) + 3.0 * L->gm * ma;
    double V[3];
    for (int p = 0; p < 3; ++p) {
        const double v = L->wp * u[p] + L->gp * a[p];
        V[p] = s->rho * (9.0 * (L->wp * Mu[p] + L->gp * Ma[p]) - 3.0 * m0 * v + 3.0 * L->wm * m[p]);
    }
    const double ns = s->ns;
    for (int k = 0; k < q; ++k) {
        const int o = L->opp[k];
        const double ck[3] = {a_cx[k] - ut[0], a_cy[k] - ut[1], a_cz[k] - ut[2]};
        const double jac = mu[k] * (1.0 - 0.5 * (L->wp + L->wm)) - mu[o] * 0.5 * (L->wp - L->wm) + P +
                           (V[0] * ck[0] + V[1] * ck[1] + V[2] * ck[2]) / s->rho;
        lam[k] = (1.0 - ns) * jac + ns * mu[o];
    }
    double gn = 0.0, gt = 0.0;
    for (int k = 0; k < q; ++k) {
        const int o = L->opp[k];
        gn += mu[k] * (x[o] - s->fstar[k]);
        const double even = 0.5 * ((x[k] - s->feq[k]) + (x[o] - s->feq[o]));
        const double oddp = 0.5 * ((x[k] - s->feq[k]) - (x[o] - s->feq[o]));
        const double fe = 0.5 * (s->Fi[k] + s->Fi[o]), fo = 0.5 * (s->Fi[k] - s->Fi[o]);
        gt += mu[k] * (L->dwp * (-even - 0.5 * fe) + L->dwm * (-oddp - 0.5 * fo));
    }
    *g_ns = gn;
    *g_tau = (1.0 - ns) * gt;
}

int ora_adjoint(const ora_cfg* c, const double* x0, uint64_t steps, const double* g_rho, const double* g_u,
                double* grad_ns, double* grad_tau) {
    adj_lattice L;
    if (adj_setup(c, &L) || steps == 0) return 1;
    const int q = c->q;
    const size_t N = c->nx * c->ny * c->nz, QN = (size_t)q * N;
    double* xs = (double*)malloc(sizeof(double) * QN * (size_t)(steps + 1));
    double* lam = (double*)calloc(QN, sizeof(double));
    double* nxt = (double*)calloc(QN, sizeof(double));
    if (!xs || !lam || !nxt) {
        free(xs);
        free(lam);
        free(nxt);
        return 2;
    }
    memcpy(xs, x0, sizeof(double) * QN);
    for (uint64_t t = 1; t <= steps; ++t) adj_forward_step(&L, c, xs + (t - 1) * QN, xs + t * QN);

    /* lambda^T = dJ/dx^T from dJ/d(rho, u) of the final state */
    const double* xT = xs + steps * QN;
    for (size_t n = 0; n < N; ++n) {
        if (!adj_fluid(c, n)) continue;
        double rho = 0.0, j[3] = {0, 0, 0};
        for (int d = 0; d < q; ++d) {
            const double v = xT[(size_t)d * N + n];
            rho += v;
            j[0] += a_cx[d] * v;
            j[1] += a_cy[d] * v;
            j[2] += a_cz[d] * v;
        }
        for (int d = 0; d < q; ++d) {
            double v = g_rho ? g_rho[n] : 0.0;
            v += (g_u[n] * (a_cx[d] - j[0] / rho) + g_u[N + n] * (a_cy[d] - j[1] / rho) +
                  g_u[2 * N + n] * (a_cz[d] - j[2] / rho)) / rho;
            lam[(size_t)d * N + n] = v;
        }
    }
    for (size_t n = 0; n < N; ++n) grad_ns[n] = 0.0;
    double gtau = 0.0;
    double xi[27], out[27], mu[27], li[27];
    adj_cell s;
    for (uint64_t t = steps; t >= 1; --t) {
        const double* xp = xs + (t - 1) * QN;
        memset(nxt, 0, sizeof(double) * QN);
        for (size_t m = 0; m < N; ++m) {
            if (!adj_fluid(c, m)) continue;
            for (int k = 0; k < q; ++k) {
                const size_t dst = adj_nbr(c, m, k, +1);
                mu[k] = adj_fluid(c, dst) ? lam[(size_t)k * N + dst] : lam[(size_t)L.opp[k] * N + m];
                xi[k] = xp[(size_t)k * N + m];
            }
            adj_collide(&L, c, m, xi, out, &s);
            double gn, gt;
            adj_cell_transpose(&L, xi, &s, mu, li, &gn, &gt);
            for (int k = 0; k < q; ++k) nxt[(size_t)k * N + m] = li[k];
            grad_ns[m] += gn;
            gtau += gt;
        }
        double* tmp = lam;
        lam = nxt;
        nxt = tmp;
    }
    *grad_tau = gtau;
    free(xs);
    free(lam);
    free(nxt);
    return 0;
}
