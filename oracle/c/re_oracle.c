/*
 * CPU oracle / CPU baseline (test infrastructure; not part of the product).
 *
 * A float64 C restatement, parallelised with OpenMP, of the same Roe-Exner step as the
 * NumPy oracle (oracle/roe_exner.py), following PyExner's
 *   src/PyExner/solvers/kernels/roe_exner.py   (roe_solver 312-533, roe_solve_2D 535-612,
 *       momentum_corrections 14-62, compute_G 85-130, compute_n 64-73, _get_lambda 163-209,
 *       compute_dt 211-255, compute_dt_2D 257-310, exner_solver 614-663, exner_solve_2D 665-717)
 *   src/PyExner/solvers/roe_exner_solver.py     (init 58-78, step 80-116, dt 118-122)
 *   src/PyExner/domain/boundaries/roeexner_{reflective,transmissive,transmissivebed,constantinflux}.py
 *   src/PyExner/integrators/forwardeuler.py:37-49 and SSPRK2.py:30-51 (intended form).
 * Expressions keep the reference's operation order; build with -ffp-contract=off so that
 * no product is fused.  Used by bench.py as the multi-threaded CPU baseline and by the
 * tests as a second, independent restatement of the oracle.
 */
#include <math.h>
#include <tgmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Arithmetic type of the state and of every operation: double by default; built with
 * -DOC_REAL=float for the float32 variant (the reference's own state is float32), in
 * which every literal below is a float32 constant and <tgmath.h> picks the float32
 * math functions. */
#ifndef OC_REAL
#define OC_REAL double
#endif
typedef OC_REAL real_t;
#define R(x) ((real_t)(x))
#define G_ACC R(9.81)
#define DRY_TOL R(1e-4)
#define SED_TOL R(1e-5)
#define VEL_TOL R(1e-6)

typedef struct {
    int32_t kind, count;
    const int64_t* cells;  /* flat row*nx + col */
    const int64_t* donors;
    double nx, ny, hu_const, hv_const;
} oc_handler;

enum { K_REFL = 1, K_TRANS = 2, K_TBED = 3, K_INFLUX = 4 };

typedef struct {
    int ny, nx, mpm, nsed;
    double dx;
    const double* seds; /* 7 x nsed, row-major */
    const uint8_t* nodata;
    const oc_handler* hs;
    int nh;
} oc_case;

typedef struct {
    real_t *h, *hu, *hv, *z, *zb, *n, *nb, *G;
} oc_state;

static real_t maxd(real_t a, real_t b) { return (a < b || b != b) ? b : a; } /* jnp.maximum */

/* ---------------------------------------------------------------- boundary handlers */
static void bc_apply(const oc_case* C, oc_state* s) {
    real_t* f[6] = {s->h, s->hu, s->hv, s->zb, s->n, s->G};
    for (int k = 0; k < C->nh; ++k) {
        const oc_handler* H = &C->hs[k];
        const int m = H->count;
        real_t* t = (real_t*)malloc(sizeof(real_t) * 6 * (size_t)(m > 0 ? m : 1));
        for (int p = 0; p < m; ++p) {
            const int64_t d = H->donors[p];
            switch (H->kind) {
                case K_REFL: {
                    const real_t hu = f[1][d], hv = f[2][d];
                    const real_t nxr = (real_t)H->nx, nyr = (real_t)H->ny;
                    const real_t mn = hu * nxr + hv * nyr, mt = -hu * nyr + hv * nxr, mr = -mn;
                    t[0 * m + p] = f[0][d];
                    t[1 * m + p] = mr * nxr - mt * nyr;
                    t[2 * m + p] = mr * nyr + mt * nxr;
                    t[3 * m + p] = f[3][d];
                    t[4 * m + p] = f[4][d];
                    t[5 * m + p] = f[5][d];
                    break;
                }
                case K_TRANS:
                    t[0 * m + p] = f[0][d];
                    t[1 * m + p] = f[1][d];
                    t[2 * m + p] = f[2][d];
                    break;
                case K_TBED:
                    t[3 * m + p] = f[3][d];
                    break;
                case K_INFLUX:
                    t[1 * m + p] = H->hu_const;
                    t[2 * m + p] = H->hv_const;
                    break;
            }
        }
        unsigned fm = H->kind == K_REFL ? 0x3f : H->kind == K_TRANS ? 0x07 : H->kind == K_TBED ? 0x08 : 0x06;
        for (int p = 0; p < m; ++p)
            for (int q = 0; q < 6; ++q)
                if ((fm >> q) & 1u) f[q][H->cells[p]] = t[q * m + p];
        free(t);
    }
}

/* ---------------------------------------------------------------- Roe-Exner face */
static void roe_face(const real_t* si, const real_t* sj, int yf, real_t dx, real_t P[3], real_t M[3]) {
    real_t hi = maxd(si[0], DRY_TOL), hj = maxd(sj[0], DRY_TOL);
    const real_t ui = hi > DRY_TOL ? si[1] / hi : R(0.0), vi = hi > DRY_TOL ? si[2] / hi : R(0.0);
    const real_t uj = hj > DRY_TOL ? sj[1] / hj : R(0.0), vj = hj > DRY_TOL ? sj[2] / hj : R(0.0);
    const real_t uhi = yf ? -vi : ui, vhi = yf ? ui : vi, uhj = yf ? -vj : uj, vhj = yf ? uj : vj;
    const real_t sqi = sqrt(hi), sqj = sqrt(hj), den = sqi + sqj;
    const real_t ht = R(0.5) * (hi + hj), ct = sqrt(G_ACC * ht);
    const real_t ut = (uhi * sqi + uhj * sqj) / den, vt = (vhi * sqi + vhj * sqj) / den;
    const real_t l1r = ut - ct, l2 = ut, l3r = ut + ct;
    real_t ei = uhi - sqrt(G_ACC * hi), ej = uhj - sqrt(G_ACC * hj);
    const int m1 = (ei < R(0.0)) && (ej > R(0.0));
    const real_t lE1 = m1 ? l1r - ei * (ej - l1r) / (ej - ei) : R(0.0);
    const real_t l1 = m1 ? ei * (ej - l1r) / (ej - ei) : l1r;
    ei = uhi + sqrt(G_ACC * hi);
    ej = uhj + sqrt(G_ACC * hj);
    const int m3 = (ei < R(0.0)) && (ej > R(0.0));
    const real_t lE3 = m3 ? l3r - ej * (l3r - ei) / (ej - ei) : R(0.0);
    const real_t l3 = m3 ? ej * (l3r - ei) / ((ej - ei) + VEL_TOL) : l3r;
    const real_t dh = hj - hi, dhu = hj * uhj - hi * uhi, dhv = hj * vhj - hi * vhi;
    const real_t den2 = -R(2.0) * ct;
    const real_t a1 = (-l3r * dh + dhu) / den2, a2 = (-vt * dh + dhv) / ct, a3 = (l1r * dh - dhu) / den2;
    const real_t zbi = si[3] > SED_TOL ? si[3] : SED_TOL * R(0.01), zbj = sj[3] > SED_TOL ? sj[3] : SED_TOL * R(0.01);
    const real_t dz = (sj[4] + zbj) - (si[4] + zbi);
    const real_t thrust = -G_ACC * ht * dz;
    const real_t nt = R(0.5) * (si[5] + sj[5]);
    const real_t sf = (nt * nt * sqrt(ut * ut + vt * vt) * ut) / (maxd(DRY_TOL, pow(ht, R(4.0) / R(3.0))));
    const real_t tau = G_ACC * ht * sf * dx;
    const real_t b1 = (thrust - tau) / den2, b3 = -b1;
    const real_t lam[3] = {l1, l2, l3}, alp[3] = {a1, a2, a3}, bet[3] = {b1, R(0.0), b3};
    const real_t Pc[3][3] = {{R(1.0), l1, vt}, {R(0.0), R(0.0), ct}, {R(1.0), l3, vt}};
    real_t pos[3] = {0, 0, 0}, neg[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        const real_t w = lam[k] * alp[k] - bet[k];
        for (int r = 0; r < 3; ++r) {
            const real_t fl = w * Pc[k][r];
            pos[r] = pos[r] + (lam[k] > R(0.0) ? fl : R(0.0));
            neg[r] = neg[r] + (lam[k] <= R(0.0) ? fl : R(0.0));
        }
    }
    const real_t lE[3] = {lE1, R(0.0), lE3};
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) {
            const real_t fl = lE[k] * alp[k] * Pc[k][r];
            pos[r] = pos[r] + (lE[k] > R(0.0) ? fl : R(0.0));
            neg[r] = neg[r] + (lE[k] <= R(0.0) ? fl : R(0.0));
        }
    if (yf) {
        P[0] = pos[0]; P[1] = pos[2]; P[2] = -pos[1];
        M[0] = neg[0]; M[1] = neg[2]; M[2] = -neg[1];
    } else {
        P[0] = pos[0]; P[1] = pos[1]; P[2] = pos[2];
        M[0] = neg[0]; M[1] = neg[1]; M[2] = neg[2];
    }
}

static int nodata(const oc_case* C, int64_t i) { return C->nodata ? C->nodata[i] != 0 : 0; }

/* ---------------------------------------------------------------- grass factor */
static real_t grass(const oc_case* C, real_t h, real_t hu, real_t hv, int m0, real_t Gin) {
    if (!C->mpm) {
        real_t G = m0 ? R(0.0) : Gin;
        return h > DRY_TOL ? G : R(0.0);
    }
    const real_t hc = maxd(h, DRY_TOL), u = hu / hc, v = hv / hc, vel2 = u * u + v * v;
    const int ns = C->nsed;
    const double* S = C->seds;
    real_t G = R(0.0), por = R(0.0);
    for (int k = 0; k < ns; ++k) {
        const real_t frac = (real_t)S[0 * ns + k], d50 = (real_t)S[1 * ns + k], s = (real_t)S[2 * ns + k] / R(1000.0),
                     thc = (real_t)S[5 * ns + k];
        const real_t np_ = pow(d50, R(1.0) / R(6.0)) / R(21.1);
        real_t th = (np_ * np_ * vel2) / ((s - R(1.0)) * d50 * cbrt(hc));
        th = maxd(th, R(0.0));
        const real_t dth = maxd(th - thc, R(0.0));
        const real_t g1 = np_ * (np_ * np_) * sqrt(G_ACC) / ((s - R(1.0)) * sqrt(hc));
        const real_t g2 = R(8.0) * sqrt(dth) / (pow(th, R(1.5)) + R(1e-5));
        const real_t c = frac * g1 * g2 * dth;
        G = k == 0 ? c : G + c;
        por += (real_t)S[6 * ns + k];
    }
    G = G / (R(1.0) - por / ns);
    if (m0) G = R(0.0);
    return hc > DRY_TOL ? G : R(0.0);
}

/* ---------------------------------------------------------------- Exner face */
static real_t exner_face(const real_t* si, const real_t* sj, int yf) {
    const real_t hi = si[0] > DRY_TOL ? si[0] : DRY_TOL * R(0.01), hj = sj[0] > DRY_TOL ? sj[0] : DRY_TOL * R(0.01);
    const real_t zbi = si[3] > SED_TOL ? si[3] : SED_TOL * R(0.01), zbj = sj[3] > SED_TOL ? sj[3] : SED_TOL * R(0.01);
    const real_t sqi = sqrt(hi), sqj = sqrt(hj);
    const real_t ui = hi > DRY_TOL ? si[1] / hi : R(0.0), vi = hi > DRY_TOL ? si[2] / hi : R(0.0);
    const real_t uj = hj > DRY_TOL ? sj[1] / hj : R(0.0), vj = hj > DRY_TOL ? sj[2] / hj : R(0.0);
    const real_t uhi = yf ? -vi : ui, uhj = yf ? -vj : uj;
    const real_t ut = (uhi * sqi + uhj * sqj) / (sqi + sqj);
    const real_t umi = ui * ui + vi * vi, umj = uj * uj + vj * vj;
    const real_t gi = si[5], gj = sj[5];
    const real_t qi = gi * umi * uhi, qj = gj * umj * uhj;
    const real_t gt = R(0.5) * (gi + gj), dz = zbj - zbi;
    const real_t dq = gt * umj * uhj - gt * umi * uhi;
    const real_t lam4 = fabs(dz) > SED_TOL ? dq / dz : ut;
    const real_t qbi = qi + (gt - gi) * umi * uhi, qbj = qj + (gt - gj) * umj * uhj;
    return lam4 >= 0 ? qbi : qbj;
}

/* ---------------------------------------------------------------- wave speeds */
static real_t face_dt(const real_t* si, const real_t* sj, int yf, real_t dx) {
    const real_t hi = maxd(si[0], DRY_TOL), hj = maxd(sj[0], DRY_TOL);
    const real_t sqi = sqrt(hi), sqj = sqrt(hj), den = sqi + sqj;
    const real_t ui = si[1] / hi, vi = si[2] / hi, uj = sj[1] / hj, vj = sj[2] / hj;
    const real_t uhi = yf ? -vi : ui, vhi = yf ? ui : vi, uhj = yf ? -vj : uj, vhj = yf ? uj : vj;
    const real_t ht = R(0.5) * (hi + hj);
    const real_t ut = (uhi * sqi + uhj * sqj) / den, ct = sqrt(G_ACC * ht);
    const real_t gt = R(0.5) * (si[3] + sj[3]);
    const real_t at = gt * (uhi * uhi + uhi * uhj + uhj * uhj + vhi * vhj) / (sqi * sqj);
    const real_t l1 = ut - ct, l3 = ut + ct;
    real_t lmin, lmax;
    if (at < R(1e-5)) {
        lmin = ut - ct;
        lmax = ut + ct;
    } else {
        const real_t b = -2 * ut, c = (1 + at) * (ct * ct) - ut * ut, d = -(ct * ct) * at * ut;
        const real_t p = (-3 * c - b * b) / R(3.0);
        const real_t q = (2 * (b * (b * b)) - (-9 * b) * c + 27 * d) / -R(27.0);
        real_t x = (3 * q) / (2 * p) * sqrt(-3 / p);
        x = x < -R(1.0) ? -R(1.0) : (x > R(1.0) ? R(1.0) : x);
        const real_t th = acos(x), sq = 2 * sqrt(-p / 3), shift = -b / -R(3.0);
        lmax = sq * cos(th / 3) + shift;
        lmin = sq * cos((th + R(6.283185307179586)) / 3) + shift;
    }
    const real_t roe = maxd(fabs(lmin), fabs(lmax)), swe = maxd(fabs(l1), fabs(l3));
    return roe < VEL_TOL ? dx / swe : dx / roe;
}

real_t oc_re_cfl(const oc_case* C, const oc_state* s, real_t cfl) {
    const int ny = C->ny, nx = C->nx;
    real_t best = INFINITY;
#pragma omp parallel for reduction(min : best) schedule(static)
    for (int r = 0; r < ny; ++r) {
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const real_t si[4] = {s->h[i], s->hu[i], s->hv[i], s->G[i]};
            if (c + 1 < nx) {
                const int64_t j = i + 1;
                if ((s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j))) {
                    const real_t sj[4] = {s->h[j], s->hu[j], s->hv[j], s->G[j]};
                    const real_t d = face_dt(si, sj, 0, (real_t)C->dx);
                    if (d < best || d != d) best = d;
                }
            }
            if (r + 1 < ny) {
                const int64_t j = i + nx;
                if ((s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j))) {
                    const real_t sj[4] = {s->h[j], s->hu[j], s->hv[j], s->G[j]};
                    const real_t d = face_dt(si, sj, 1, (real_t)C->dx);
                    if (d < best || d != d) best = d;
                }
            }
        }
    }
    return maxd(cfl * best, R(1e-6));
}

/* one stage: s -> o (o's planes are overwritten, n included: boundary handlers write it;
   z and nb are shared and read only) */
void oc_re_stage(const oc_case* C, const oc_state* s, oc_state* o, real_t dt, real_t* work) {
    const int ny = C->ny, nx = C->nx;
    const int64_t N = (int64_t)ny * nx;
    real_t* Fx = work;            /* 6 per x-face: P, M */
    real_t* Fy = work + 6 * N;    /* 6 per y-face */
    const real_t dx = (real_t)C->dx;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const real_t si[6] = {s->h[i], s->hu[i], s->hv[i], s->zb[i], s->z[i], s->nb[i]};
            if (c + 1 < nx) {
                const int64_t j = i + 1;
                const real_t sj[6] = {s->h[j], s->hu[j], s->hv[j], s->zb[j], s->z[j], s->nb[j]};
                real_t P[3], M[3];
                roe_face(si, sj, 0, dx, P, M);
                const int act = (s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j));
                for (int k = 0; k < 3; ++k) {
                    Fx[6 * i + k] = act ? P[k] : R(0.0);
                    Fx[6 * i + 3 + k] = act ? M[k] : R(0.0);
                }
            }
            if (r + 1 < ny) {
                const int64_t j = i + nx;
                const real_t sj[6] = {s->h[j], s->hu[j], s->hv[j], s->zb[j], s->z[j], s->nb[j]};
                real_t P[3], M[3];
                roe_face(si, sj, 1, dx, P, M);
                const int act = (s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j));
                for (int k = 0; k < 3; ++k) {
                    Fy[6 * i + k] = act ? P[k] : R(0.0);
                    Fy[6 * i + 3 + k] = act ? M[k] : R(0.0);
                }
            }
        }
    /* update in the scatter order of roe_exner.py:597-602 */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            real_t f[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                if (c + 1 < nx) f[k] += Fx[6 * i + 3 + k];
                if (c >= 1) f[k] += Fx[6 * (i - 1) + k];
                if (r + 1 < ny) f[k] += Fy[6 * i + 3 + k];
                if (r >= 1) f[k] += Fy[6 * (i - nx) + k];
            }
            o->h[i] = s->h[i] - dt * f[0] / dx;
            o->hu[i] = s->hu[i] - dt * f[1] / dx;
            o->hv[i] = s->hv[i] - dt * f[2] / dx;
            o->zb[i] = s->zb[i];
            o->G[i] = s->G[i];
            o->n[i] = s->n[i];
        }
    /* momentum corrections on the interior (roe_exner.py:14-62), in place: they read h only */
#pragma omp parallel for schedule(static)
    for (int r = 1; r < ny - 1; ++r)
        for (int c = 1; c < nx - 1; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const real_t eta = o->h[i] + (s->z[i] + s->zb[i]);
            const int64_t E = i + 1, W = i - 1, Nn = i - nx, S = i + nx;
            const int stop_u = ((eta < s->z[E] + s->zb[E]) && (o->h[E] < DRY_TOL)) ||
                               ((eta < s->z[W] + s->zb[W]) && (o->h[W] < DRY_TOL)) || nodata(C, E) || nodata(C, W);
            const int stop_v = ((eta < s->z[Nn] + s->zb[Nn]) && (o->h[Nn] < DRY_TOL)) ||
                               ((eta < s->z[S] + s->zb[S]) && (o->h[S] < DRY_TOL)) || nodata(C, Nn) || nodata(C, S);
            const int active = (o->h[i] > DRY_TOL) && !nodata(C, i);
            if (!(active && !stop_u)) o->hu[i] = R(0.0);
            if (!(active && !stop_v)) o->hv[i] = R(0.0);
        }
    oc_state t = *o;
    bc_apply(C, &t);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) o->G[i] = grass(C, o->h[i], o->hu[i], o->hv[i], nodata(C, i), o->G[i]);
    /* Exner faces (roe_exner.py:665-717) */
    real_t* Ex = work;       /* 1 per x-face */
    real_t* Ey = work + N;   /* 1 per y-face */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const real_t si[6] = {o->h[i], o->hu[i], o->hv[i], o->zb[i], s->z[i], o->G[i]};
            for (int yf = 0; yf < 2; ++yf) {
                if (yf ? (r + 1 >= ny) : (c + 1 >= nx)) continue;
                const int64_t j = yf ? i + nx : i + 1;
                const real_t sj[6] = {o->h[j], o->hu[j], o->hv[j], o->zb[j], s->z[j], o->G[j]};
                const int stop = (nodata(C, i) || nodata(C, j)) || ((o->zb[i] < SED_TOL) && (o->zb[j] < SED_TOL));
                const int depth = (o->h[i] > DRY_TOL) || (o->h[j] > DRY_TOL);
                const real_t F = (depth && !stop) ? exner_face(si, sj, yf) : R(0.0);
                (yf ? Ey : Ex)[i] = F;
            }
        }
    real_t* zn = work + 2 * N;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            real_t f = R(0.0);
            if (c >= 1) f += -Ex[i - 1];
            if (c + 1 < nx) f += Ex[i];
            if (r >= 1) f += -Ey[i - nx];
            if (r + 1 < ny) f += Ey[i];
            zn[i] = o->zb[i] - dt * f / dx;
        }
    memcpy(o->zb, zn, sizeof(real_t) * (size_t)N);
    bc_apply(C, &t);
}

void oc_re_init(const oc_case* C, oc_state* s) {
    const int64_t N = (int64_t)C->ny * C->nx;
    real_t d50f = R(0.0);
    for (int k = 0; k < C->nsed && C->mpm; ++k) d50f += (real_t)C->seds[1 * C->nsed + k] * (real_t)C->seds[0 * C->nsed + k];
    const real_t np_mix = C->mpm ? pow(d50f / C->nsed, R(1.0) / R(6.0)) / R(21.1) : R(0.0);
    for (int64_t i = 0; i < N; ++i) {
        s->nb[i] = C->mpm ? (s->zb[i] > SED_TOL ? np_mix : s->n[i]) : s->n[i];
        s->G[i] = grass(C, s->h[i], s->hu[i], s->hv[i], nodata(C, i), s->G[i]);
    }
    bc_apply(C, s);
}

/* nsteps Forward-Euler (scheme 0) or SSPRK2 (scheme 1) steps in place; dts[nsteps] out */
int oc_re_run(const oc_case* C, oc_state* s, int nsteps, int scheme, double cfl_in, double* dts) {
    const real_t cfl = (real_t)cfl_in;
    const int64_t N = (int64_t)C->ny * C->nx;
    real_t* buf = (real_t*)malloc(sizeof(real_t) * (size_t)(N * 6 + N * 12));
    if (!buf) return 1;
    oc_state a = *s, b = *s;
    b.h = buf;
    b.hu = buf + N;
    b.hv = buf + 2 * N;
    b.zb = buf + 3 * N;
    b.G = buf + 4 * N;
    b.n = buf + 5 * N;
    real_t* work = buf + 6 * N;
    for (int k = 0; k < nsteps; ++k) {
        const real_t dt = oc_re_cfl(C, &a, cfl);
        if (dts) dts[k] = dt;
        oc_re_stage(C, &a, &b, dt, work);
        if (scheme == 1) {
            oc_state c2 = b;
            real_t* tmp = (real_t*)malloc(sizeof(real_t) * (size_t)(N * 6));
            c2.h = tmp;
            c2.hu = tmp + N;
            c2.hv = tmp + 2 * N;
            c2.zb = tmp + 3 * N;
            c2.G = tmp + 4 * N;
            c2.n = tmp + 5 * N;
            oc_re_stage(C, &b, &c2, dt, work);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) {
                a.h[i] = R(0.5) * a.h[i] + R(0.5) * c2.h[i];
                a.hu[i] = R(0.5) * a.hu[i] + R(0.5) * c2.hu[i];
                a.hv[i] = R(0.5) * a.hv[i] + R(0.5) * c2.hv[i];
                a.zb[i] = R(0.5) * a.zb[i] + R(0.5) * c2.zb[i];
                a.G[i] = R(0.5) * a.G[i] + R(0.5) * c2.G[i];
                a.n[i] = R(0.5) * a.n[i] + R(0.5) * c2.n[i];
            }
            free(tmp);
        } else {
            memcpy(a.h, b.h, sizeof(real_t) * (size_t)N);
            memcpy(a.hu, b.hu, sizeof(real_t) * (size_t)N);
            memcpy(a.hv, b.hv, sizeof(real_t) * (size_t)N);
            memcpy(a.zb, b.zb, sizeof(real_t) * (size_t)N);
            memcpy(a.G, b.G, sizeof(real_t) * (size_t)N);
            memcpy(a.n, b.n, sizeof(real_t) * (size_t)N);
        }
    }
    free(buf);
    return 0;
}
