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
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define G_ACC 9.81
#define DRY_TOL 1e-4
#define SED_TOL 1e-5
#define VEL_TOL 1e-6

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
    double *h, *hu, *hv, *z, *zb, *n, *nb, *G;
} oc_state;

static double maxd(double a, double b) { return (a < b || b != b) ? b : a; } /* jnp.maximum */

/* ---------------------------------------------------------------- boundary handlers */
static void bc_apply(const oc_case* C, oc_state* s) {
    double* f[6] = {s->h, s->hu, s->hv, s->zb, s->n, s->G};
    for (int k = 0; k < C->nh; ++k) {
        const oc_handler* H = &C->hs[k];
        const int m = H->count;
        double* t = (double*)malloc(sizeof(double) * 6 * (size_t)(m > 0 ? m : 1));
        for (int p = 0; p < m; ++p) {
            const int64_t d = H->donors[p];
            switch (H->kind) {
                case K_REFL: {
                    const double hu = f[1][d], hv = f[2][d];
                    const double mn = hu * H->nx + hv * H->ny, mt = -hu * H->ny + hv * H->nx, mr = -mn;
                    t[0 * m + p] = f[0][d];
                    t[1 * m + p] = mr * H->nx - mt * H->ny;
                    t[2 * m + p] = mr * H->ny + mt * H->nx;
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
static void roe_face(const double* si, const double* sj, int yf, double dx, double P[3], double M[3]) {
    double hi = maxd(si[0], DRY_TOL), hj = maxd(sj[0], DRY_TOL);
    const double ui = hi > DRY_TOL ? si[1] / hi : 0.0, vi = hi > DRY_TOL ? si[2] / hi : 0.0;
    const double uj = hj > DRY_TOL ? sj[1] / hj : 0.0, vj = hj > DRY_TOL ? sj[2] / hj : 0.0;
    const double uhi = yf ? -vi : ui, vhi = yf ? ui : vi, uhj = yf ? -vj : uj, vhj = yf ? uj : vj;
    const double sqi = sqrt(hi), sqj = sqrt(hj), den = sqi + sqj;
    const double ht = 0.5 * (hi + hj), ct = sqrt(G_ACC * ht);
    const double ut = (uhi * sqi + uhj * sqj) / den, vt = (vhi * sqi + vhj * sqj) / den;
    const double l1r = ut - ct, l2 = ut, l3r = ut + ct;
    double ei = uhi - sqrt(G_ACC * hi), ej = uhj - sqrt(G_ACC * hj);
    const int m1 = (ei < 0.0) && (ej > 0.0);
    const double lE1 = m1 ? l1r - ei * (ej - l1r) / (ej - ei) : 0.0;
    const double l1 = m1 ? ei * (ej - l1r) / (ej - ei) : l1r;
    ei = uhi + sqrt(G_ACC * hi);
    ej = uhj + sqrt(G_ACC * hj);
    const int m3 = (ei < 0.0) && (ej > 0.0);
    const double lE3 = m3 ? l3r - ej * (l3r - ei) / (ej - ei) : 0.0;
    const double l3 = m3 ? ej * (l3r - ei) / ((ej - ei) + VEL_TOL) : l3r;
    const double dh = hj - hi, dhu = hj * uhj - hi * uhi, dhv = hj * vhj - hi * vhi;
    const double den2 = -2.0 * ct;
    const double a1 = (-l3r * dh + dhu) / den2, a2 = (-vt * dh + dhv) / ct, a3 = (l1r * dh - dhu) / den2;
    const double zbi = si[3] > SED_TOL ? si[3] : SED_TOL * 0.01, zbj = sj[3] > SED_TOL ? sj[3] : SED_TOL * 0.01;
    const double dz = (sj[4] + zbj) - (si[4] + zbi);
    const double thrust = -G_ACC * ht * dz;
    const double nt = 0.5 * (si[5] + sj[5]);
    const double sf = (nt * nt * sqrt(ut * ut + vt * vt) * ut) / (maxd(DRY_TOL, pow(ht, 4.0 / 3.0)));
    const double tau = G_ACC * ht * sf * dx;
    const double b1 = (thrust - tau) / den2, b3 = -b1;
    const double lam[3] = {l1, l2, l3}, alp[3] = {a1, a2, a3}, bet[3] = {b1, 0.0, b3};
    const double Pc[3][3] = {{1.0, l1, vt}, {0.0, 0.0, ct}, {1.0, l3, vt}};
    double pos[3] = {0, 0, 0}, neg[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        const double w = lam[k] * alp[k] - bet[k];
        for (int r = 0; r < 3; ++r) {
            const double fl = w * Pc[k][r];
            pos[r] = pos[r] + (lam[k] > 0.0 ? fl : 0.0);
            neg[r] = neg[r] + (lam[k] <= 0.0 ? fl : 0.0);
        }
    }
    const double lE[3] = {lE1, 0.0, lE3};
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) {
            const double fl = lE[k] * alp[k] * Pc[k][r];
            pos[r] = pos[r] + (lE[k] > 0.0 ? fl : 0.0);
            neg[r] = neg[r] + (lE[k] <= 0.0 ? fl : 0.0);
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
static double grass(const oc_case* C, double h, double hu, double hv, int m0, double Gin) {
    if (!C->mpm) {
        double G = m0 ? 0.0 : Gin;
        return h > DRY_TOL ? G : 0.0;
    }
    const double hc = maxd(h, DRY_TOL), u = hu / hc, v = hv / hc, vel2 = u * u + v * v;
    const int ns = C->nsed;
    const double* S = C->seds;
    double G = 0.0, por = 0.0;
    for (int k = 0; k < ns; ++k) {
        const double frac = S[0 * ns + k], d50 = S[1 * ns + k], s = S[2 * ns + k] / 1000.0, thc = S[5 * ns + k];
        const double np_ = pow(d50, 1.0 / 6.0) / 21.1;
        double th = (np_ * np_ * vel2) / ((s - 1.0) * d50 * cbrt(hc));
        th = maxd(th, 0.0);
        const double dth = maxd(th - thc, 0.0);
        const double g1 = np_ * (np_ * np_) * sqrt(G_ACC) / ((s - 1.0) * sqrt(hc));
        const double g2 = 8.0 * sqrt(dth) / (pow(th, 1.5) + 1e-5);
        const double c = frac * g1 * g2 * dth;
        G = k == 0 ? c : G + c;
        por += S[6 * ns + k];
    }
    G = G / (1.0 - por / ns);
    if (m0) G = 0.0;
    return hc > DRY_TOL ? G : 0.0;
}

/* ---------------------------------------------------------------- Exner face */
static double exner_face(const double* si, const double* sj, int yf) {
    const double hi = si[0] > DRY_TOL ? si[0] : DRY_TOL * 0.01, hj = sj[0] > DRY_TOL ? sj[0] : DRY_TOL * 0.01;
    const double zbi = si[3] > SED_TOL ? si[3] : SED_TOL * 0.01, zbj = sj[3] > SED_TOL ? sj[3] : SED_TOL * 0.01;
    const double sqi = sqrt(hi), sqj = sqrt(hj);
    const double ui = hi > DRY_TOL ? si[1] / hi : 0.0, vi = hi > DRY_TOL ? si[2] / hi : 0.0;
    const double uj = hj > DRY_TOL ? sj[1] / hj : 0.0, vj = hj > DRY_TOL ? sj[2] / hj : 0.0;
    const double uhi = yf ? -vi : ui, uhj = yf ? -vj : uj;
    const double ut = (uhi * sqi + uhj * sqj) / (sqi + sqj);
    const double umi = ui * ui + vi * vi, umj = uj * uj + vj * vj;
    const double gi = si[5], gj = sj[5];
    const double qi = gi * umi * uhi, qj = gj * umj * uhj;
    const double gt = 0.5 * (gi + gj), dz = zbj - zbi;
    const double dq = gt * umj * uhj - gt * umi * uhi;
    const double lam4 = fabs(dz) > SED_TOL ? dq / dz : ut;
    const double qbi = qi + (gt - gi) * umi * uhi, qbj = qj + (gt - gj) * umj * uhj;
    return lam4 >= 0 ? qbi : qbj;
}

/* ---------------------------------------------------------------- wave speeds */
static double face_dt(const double* si, const double* sj, int yf, double dx) {
    const double hi = maxd(si[0], DRY_TOL), hj = maxd(sj[0], DRY_TOL);
    const double sqi = sqrt(hi), sqj = sqrt(hj), den = sqi + sqj;
    const double ui = si[1] / hi, vi = si[2] / hi, uj = sj[1] / hj, vj = sj[2] / hj;
    const double uhi = yf ? -vi : ui, vhi = yf ? ui : vi, uhj = yf ? -vj : uj, vhj = yf ? uj : vj;
    const double ht = 0.5 * (hi + hj);
    const double ut = (uhi * sqi + uhj * sqj) / den, ct = sqrt(G_ACC * ht);
    const double gt = 0.5 * (si[3] + sj[3]);
    const double at = gt * (uhi * uhi + uhi * uhj + uhj * uhj + vhi * vhj) / (sqi * sqj);
    const double l1 = ut - ct, l3 = ut + ct;
    double lmin, lmax;
    if (at < 1e-5) {
        lmin = ut - ct;
        lmax = ut + ct;
    } else {
        const double b = -2 * ut, c = (1 + at) * (ct * ct) - ut * ut, d = -(ct * ct) * at * ut;
        const double p = (-3 * c - b * b) / 3.0;
        const double q = (2 * (b * (b * b)) - (-9 * b) * c + 27 * d) / -27.0;
        double x = (3 * q) / (2 * p) * sqrt(-3 / p);
        x = x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x);
        const double th = acos(x), sq = 2 * sqrt(-p / 3), shift = -b / -3.0;
        lmax = sq * cos(th / 3) + shift;
        lmin = sq * cos((th + 6.283185307179586) / 3) + shift;
    }
    const double roe = maxd(fabs(lmin), fabs(lmax)), swe = maxd(fabs(l1), fabs(l3));
    return roe < VEL_TOL ? dx / swe : dx / roe;
}

double oc_re_cfl(const oc_case* C, const oc_state* s, double cfl) {
    const int ny = C->ny, nx = C->nx;
    double best = INFINITY;
#pragma omp parallel for reduction(min : best) schedule(static)
    for (int r = 0; r < ny; ++r) {
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const double si[4] = {s->h[i], s->hu[i], s->hv[i], s->G[i]};
            if (c + 1 < nx) {
                const int64_t j = i + 1;
                if ((s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j))) {
                    const double sj[4] = {s->h[j], s->hu[j], s->hv[j], s->G[j]};
                    const double d = face_dt(si, sj, 0, C->dx);
                    if (d < best || d != d) best = d;
                }
            }
            if (r + 1 < ny) {
                const int64_t j = i + nx;
                if ((s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j))) {
                    const double sj[4] = {s->h[j], s->hu[j], s->hv[j], s->G[j]};
                    const double d = face_dt(si, sj, 1, C->dx);
                    if (d < best || d != d) best = d;
                }
            }
        }
    }
    return maxd(cfl * best, 1e-6);
}

/* one stage: s -> o (o's planes are overwritten, n included: boundary handlers write it;
   z and nb are shared and read only) */
void oc_re_stage(const oc_case* C, const oc_state* s, oc_state* o, double dt, double* work) {
    const int ny = C->ny, nx = C->nx;
    const int64_t N = (int64_t)ny * nx;
    double* Fx = work;            /* 6 per x-face: P, M */
    double* Fy = work + 6 * N;    /* 6 per y-face */
    const double dx = C->dx;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const double si[6] = {s->h[i], s->hu[i], s->hv[i], s->zb[i], s->z[i], s->nb[i]};
            if (c + 1 < nx) {
                const int64_t j = i + 1;
                const double sj[6] = {s->h[j], s->hu[j], s->hv[j], s->zb[j], s->z[j], s->nb[j]};
                double P[3], M[3];
                roe_face(si, sj, 0, dx, P, M);
                const int act = (s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j));
                for (int k = 0; k < 3; ++k) {
                    Fx[6 * i + k] = act ? P[k] : 0.0;
                    Fx[6 * i + 3 + k] = act ? M[k] : 0.0;
                }
            }
            if (r + 1 < ny) {
                const int64_t j = i + nx;
                const double sj[6] = {s->h[j], s->hu[j], s->hv[j], s->zb[j], s->z[j], s->nb[j]};
                double P[3], M[3];
                roe_face(si, sj, 1, dx, P, M);
                const int act = (s->h[i] > DRY_TOL || s->h[j] > DRY_TOL) && !(nodata(C, i) || nodata(C, j));
                for (int k = 0; k < 3; ++k) {
                    Fy[6 * i + k] = act ? P[k] : 0.0;
                    Fy[6 * i + 3 + k] = act ? M[k] : 0.0;
                }
            }
        }
    /* update in the scatter order of roe_exner.py:597-602 */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            double f[3] = {0, 0, 0};
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
            const double eta = o->h[i] + (s->z[i] + s->zb[i]);
            const int64_t E = i + 1, W = i - 1, Nn = i - nx, S = i + nx;
            const int stop_u = ((eta < s->z[E] + s->zb[E]) && (o->h[E] < DRY_TOL)) ||
                               ((eta < s->z[W] + s->zb[W]) && (o->h[W] < DRY_TOL)) || nodata(C, E) || nodata(C, W);
            const int stop_v = ((eta < s->z[Nn] + s->zb[Nn]) && (o->h[Nn] < DRY_TOL)) ||
                               ((eta < s->z[S] + s->zb[S]) && (o->h[S] < DRY_TOL)) || nodata(C, Nn) || nodata(C, S);
            const int active = (o->h[i] > DRY_TOL) && !nodata(C, i);
            if (!(active && !stop_u)) o->hu[i] = 0.0;
            if (!(active && !stop_v)) o->hv[i] = 0.0;
        }
    oc_state t = *o;
    bc_apply(C, &t);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) o->G[i] = grass(C, o->h[i], o->hu[i], o->hv[i], nodata(C, i), o->G[i]);
    /* Exner faces (roe_exner.py:665-717) */
    double* Ex = work;       /* 1 per x-face */
    double* Ey = work + N;   /* 1 per y-face */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            const double si[6] = {o->h[i], o->hu[i], o->hv[i], o->zb[i], s->z[i], o->G[i]};
            for (int yf = 0; yf < 2; ++yf) {
                if (yf ? (r + 1 >= ny) : (c + 1 >= nx)) continue;
                const int64_t j = yf ? i + nx : i + 1;
                const double sj[6] = {o->h[j], o->hu[j], o->hv[j], o->zb[j], s->z[j], o->G[j]};
                const int stop = (nodata(C, i) || nodata(C, j)) || ((o->zb[i] < SED_TOL) && (o->zb[j] < SED_TOL));
                const int depth = (o->h[i] > DRY_TOL) || (o->h[j] > DRY_TOL);
                const double F = (depth && !stop) ? exner_face(si, sj, yf) : 0.0;
                (yf ? Ey : Ex)[i] = F;
            }
        }
    double* zn = work + 2 * N;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const int64_t i = (int64_t)r * nx + c;
            double f = 0.0;
            if (c >= 1) f += -Ex[i - 1];
            if (c + 1 < nx) f += Ex[i];
            if (r >= 1) f += -Ey[i - nx];
            if (r + 1 < ny) f += Ey[i];
            zn[i] = o->zb[i] - dt * f / dx;
        }
    memcpy(o->zb, zn, sizeof(double) * (size_t)N);
    bc_apply(C, &t);
}

void oc_re_init(const oc_case* C, oc_state* s) {
    const int64_t N = (int64_t)C->ny * C->nx;
    double d50f = 0.0;
    for (int k = 0; k < C->nsed && C->mpm; ++k) d50f += C->seds[1 * C->nsed + k] * C->seds[0 * C->nsed + k];
    const double np_mix = C->mpm ? pow(d50f / C->nsed, 1.0 / 6.0) / 21.1 : 0.0;
    for (int64_t i = 0; i < N; ++i) {
        s->nb[i] = C->mpm ? (s->zb[i] > SED_TOL ? np_mix : s->n[i]) : s->n[i];
        s->G[i] = grass(C, s->h[i], s->hu[i], s->hv[i], nodata(C, i), s->G[i]);
    }
    bc_apply(C, s);
}

/* nsteps Forward-Euler (scheme 0) or SSPRK2 (scheme 1) steps in place; dts[nsteps] out */
int oc_re_run(const oc_case* C, oc_state* s, int nsteps, int scheme, double cfl, double* dts) {
    const int64_t N = (int64_t)C->ny * C->nx;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(N * 6 + N * 12));
    if (!buf) return 1;
    oc_state a = *s, b = *s;
    b.h = buf;
    b.hu = buf + N;
    b.hv = buf + 2 * N;
    b.zb = buf + 3 * N;
    b.G = buf + 4 * N;
    b.n = buf + 5 * N;
    double* work = buf + 6 * N;
    for (int k = 0; k < nsteps; ++k) {
        const double dt = oc_re_cfl(C, &a, cfl);
        if (dts) dts[k] = dt;
        oc_re_stage(C, &a, &b, dt, work);
        if (scheme == 1) {
            oc_state c2 = b;
            double* tmp = (double*)malloc(sizeof(double) * (size_t)(N * 6));
            c2.h = tmp;
            c2.hu = tmp + N;
            c2.hv = tmp + 2 * N;
            c2.zb = tmp + 3 * N;
            c2.G = tmp + 4 * N;
            c2.n = tmp + 5 * N;
            oc_re_stage(C, &b, &c2, dt, work);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) {
                a.h[i] = 0.5 * a.h[i] + 0.5 * c2.h[i];
                a.hu[i] = 0.5 * a.hu[i] + 0.5 * c2.hu[i];
                a.hv[i] = 0.5 * a.hv[i] + 0.5 * c2.hv[i];
                a.zb[i] = 0.5 * a.zb[i] + 0.5 * c2.zb[i];
                a.G[i] = 0.5 * a.G[i] + 0.5 * c2.G[i];
                a.n[i] = 0.5 * a.n[i] + 0.5 * c2.n[i];
            }
            free(tmp);
        } else {
            memcpy(a.h, b.h, sizeof(double) * (size_t)N);
            memcpy(a.hu, b.hu, sizeof(double) * (size_t)N);
            memcpy(a.hv, b.hv, sizeof(double) * (size_t)N);
            memcpy(a.zb, b.zb, sizeof(double) * (size_t)N);
            memcpy(a.G, b.G, sizeof(double) * (size_t)N);
            memcpy(a.n, b.n, sizeof(double) * (size_t)N);
        }
    }
    free(buf);
    return 0;
}
