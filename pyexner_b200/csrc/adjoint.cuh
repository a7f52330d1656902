// Reverse-mode (adjoint) kernels of the float64 Roe-Exner stage and of the CFL step.
//
// A stage is, in the reference's order (roe_exner_solver.py:80-116):
//   U1 = U - dt/dx * sum of face fluctuations(U)          hydro (roe_exner.py:535-612)
//   momentum corrections (zeroing masks)                    (:14-62)
//   handlers                                                (boundary_registry.py:183-187)
//   G = grass(h, hu, hv) or the constant pass-through      (:85-140)
//   zb2 = zb1 - dt/dx * sum of Exner face fluxes            (:665-717)
//   handlers
// and the SSPRK2 average for the second stage.  The adjoint runs these backwards.  Each
// cell gathers the contributions of its faces: the derivatives of a face's outputs with
// respect to the cell's own inputs come from one evaluation of the same face formula on
// DualN numbers seeded with those inputs (the neighbour held constant), so no face
// arithmetic is written twice.  Masks and branches (wet/dry, activity, upwinding, the
// correction zeroing) are taken from the forward values and carry no derivative.
// Handlers are linear in the state for every kind except ConstantOutflux (refused):
// their adjoint moves the boundary cells' adjoints to the donors (scatter-add).
#pragma once
// pxb_device.cuh first: its templates must see the standard fabs at their definition;
// the dual types bring their own overloads through argument-dependent lookup.
#include "pxb_device.cuh"
#include "init_bc.cuh"
#include "adjoint_args.cuh"
#include "dualn.cuh"

namespace pxb {


__device__ __forceinline__ bool adj_cell(int ny, int nx, long long pitch, int& r, int& c, long long& i) {
    c = blockIdx.x * blockDim.x + threadIdx.x;
    r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= ny || c >= nx) return false;
    i = (long long)r * pitch + c;
    return true;
}

__device__ __forceinline__ bool adj_nodata(const uint8_t* m, long long i) { return m ? m[i] != 0 : false; }

// warp sum then one atomic per warp (every lane of the warp calls this)
__device__ __forceinline__ void adj_dt_add(double* dst, double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

// SSPRK2 average / plain store: S = scale * out_adj; with `avg`, avg_adj = 0.5 * out_adj.
__global__ void adj_store_kernel(int ny, int nx, long long pitch, double scale, const double* oh, const double* ohu,
                                 const double* ohv, const double* ozb, const double* oG, double* Sh, double* Shu,
                                 double* Shv, double* Szb, double* SG, double* Ah, double* Ahu, double* Ahv, double* Azb,
                                 double* AG) {
    int r, c;
    long long i;
    if (!adj_cell(ny, nx, pitch, r, c, i)) return;
    const double a[5] = {oh[i], ohu[i], ohv[i], ozb[i], oG[i]};
    Sh[i] = scale * a[0];
    Shu[i] = scale * a[1];
    Shv[i] = scale * a[2];
    Szb[i] = scale * a[3];
    SG[i] = scale * a[4];
    if (Ah) {
        Ah[i] = 0.5 * a[0];
        Ahu[i] = 0.5 * a[1];
        Ahv[i] = 0.5 * a[2];
        Azb[i] = 0.5 * a[3];
        AG[i] = 0.5 * a[4];
    }
}

// Exner update backwards: T = S (identity paths) + face terms; dt adjoint.
__global__ void __launch_bounds__(256) adj_exner_kernel(const AdjArgs a) {
    int r, c;
    long long i;
    const bool in = adj_cell(a.ny, a.nx, a.pitch, r, c, i);
    double add_dt = 0.0;
    if (in) {
        using D = DualN<5>;
        const double dt = *a.dt, dx = a.dx;
        auto ecell = [&](long long k) { return make_ecell(a.sh[k], a.shu[k], a.shv[k], a.szb[k], a.sG[k]); };
        const ECell<double> C = ecell(i);
        const ECell<D> Cd = make_ecell(D::seed(a.sh[i], 0), D::seed(a.shu[i], 1), D::seed(a.shv[i], 2),
                                       D::seed(a.szb[i], 3), D::seed(a.sG[i], 4));
        auto econst = [&](long long k) {
            return make_ecell(D(a.sh[k]), D(a.shu[k]), D(a.shv[k]), D(a.szb[k]), D(a.sG[k]));
        };
        const bool mC = adj_nodata(a.nodata, i);
        double g[5] = {0, 0, 0, 0, 0};
        double acc = 0.0;  // sum of the signed face fluxes of this cell (forward values)
        // face (I|J) with flux F: zb2[I] -= dt/dx F, zb2[J] += dt/dx F
        auto face = [&](long long k, bool cell_is_I, bool yf) {
            const ECell<double> N = ecell(k);
            const bool mk = adj_nodata(a.nodata, k);
            const bool act = cell_is_I ? exner_active(C, N, mC, mk) : exner_active(N, C, mk, mC);
            if (!act) return;
            const ECell<D> Nd = econst(k);
            D F;
            if (yf) F = cell_is_I ? exner_face<D, true>(Cd, Nd) : exner_face<D, true>(Nd, Cd);
            else F = cell_is_I ? exner_face<D, false>(Cd, Nd) : exner_face<D, false>(Nd, Cd);
            const double zI = cell_is_I ? a.Szb[i] : a.Szb[k], zJ = cell_is_I ? a.Szb[k] : a.Szb[i];
            const double Fbar = -dt / dx * (zI - zJ);
            for (int q = 0; q < 5; ++q) g[q] += Fbar * F.d[q];
            acc += cell_is_I ? F.v : -F.v;
        };
        if (c >= 1) face(i - 1, false, false);
        if (c + 1 < a.nx) face(i + 1, true, false);
        if (r >= 1) face(i - a.pitch, false, true);
        if (r + 1 < a.ny) face(i + a.pitch, true, true);
        (void)C;
        a.Th[i] = a.Sh[i] + g[0];
        a.Thu[i] = a.Shu[i] + g[1];
        a.Thv[i] = a.Shv[i] + g[2];
        a.Tzb[i] = a.Szb[i] + g[3];
        a.TG[i] = a.SG[i] + g[4];
        add_dt = a.Szb[i] * (-acc / dx);
    }
    adj_dt_add(a.dtbar, add_dt);
}

// warp sum of each of N values, one atomic per value and warp (every lane calls this)
template <int N>
__device__ __forceinline__ void adj_sum_add(double* dst, const double (&v)[N]) {
#pragma unroll
    for (int q = 0; q < N; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
        if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(dst + q, x);
    }
}

// grass factor backwards, in place on T (G of the state after handlers 1 -> h, hu, hv);
// PAR: also the adjoint of the MPM constants of the single sediment class (a.tbar), from
// one evaluation on dual numbers seeded in the cell's h, hu, hv and in those constants
template <bool PAR>
__global__ void __launch_bounds__(256) adj_grass_kernel(const AdjArgs a) {
    int r, c;
    long long i;
    const bool in = adj_cell(a.ny, a.nx, a.pitch, r, c, i);
    if constexpr (PAR) {
        double tb[7] = {0, 0, 0, 0, 0, 0, 0};
        if (in && a.mpm) {
            using D = DualN<10>;
            const bool m = adj_nodata(a.nodata, i);
            SedTable<D> sd;
            sd.n = 1;
            sd.s[0].np2 = D::seed(a.sed.s[0].np2, 3);
            sd.s[0].sm1d = D::seed(a.sed.s[0].sm1d, 4);
            sd.s[0].thc = D::seed(a.sed.s[0].thc, 5);
            sd.s[0].np3sg = D::seed(a.sed.s[0].np3sg, 6);
            sd.s[0].sm1 = D::seed(a.sed.s[0].sm1, 7);
            sd.s[0].frac = D::seed(a.sed.s[0].frac, 8);
            sd.one_minus_por = D::seed(a.sed.one_minus_por, 9);
            const D G = mpm_grass(D::seed(a.sh[i], 0), D::seed(a.shu[i], 1), D::seed(a.shv[i], 2), m, sd);
            const double gbar = a.TG[i];
            a.Th[i] += gbar * G.d[0];
            a.Thu[i] += gbar * G.d[1];
            a.Thv[i] += gbar * G.d[2];
            a.TG[i] = 0.0;
#pragma unroll
            for (int q = 0; q < 7; ++q) tb[q] = gbar * G.d[3 + q];
        } else if (in) {
            a.TG[i] = (!adj_nodata(a.nodata, i) && a.sh[i] > DRY_TOL) ? a.TG[i] : 0.0;
        }
        adj_sum_add<7>(a.tbar, tb);
        return;
    }
    if (!in) return;
    const bool m = adj_nodata(a.nodata, i);
    const double gbar = a.TG[i];
    if (a.mpm) {
        using D = DualN<3>;
        SedTable<D> sd;  // the sediment constants as (constant) dual numbers
        sd.n = a.sed.n;
        for (int k = 0; k < a.sed.n; ++k) {
            sd.s[k].np2 = a.sed.s[k].np2;
            sd.s[k].sm1d = a.sed.s[k].sm1d;
            sd.s[k].thc = a.sed.s[k].thc;
            sd.s[k].np3sg = a.sed.s[k].np3sg;
            sd.s[k].sm1 = a.sed.s[k].sm1;
            sd.s[k].frac = a.sed.s[k].frac;
        }
        sd.one_minus_por = a.sed.one_minus_por;
        const D G = mpm_grass(D::seed(a.sh[i], 0), D::seed(a.shu[i], 1), D::seed(a.shv[i], 2), m, sd);
        a.Th[i] += gbar * G.d[0];
        a.Thu[i] += gbar * G.d[1];
        a.Thv[i] += gbar * G.d[2];
        a.TG[i] = 0.0;  // MPM recomputes G: the incoming G has no influence
    } else {
        a.TG[i] = (!m && a.sh[i] > DRY_TOL) ? gbar : 0.0;
    }
}

// momentum corrections backwards, in place on T (interior cells)
__global__ void adj_corr_kernel(const AdjArgs a) {
    int r, c;
    long long i;
    if (!adj_cell(a.ny, a.nx, a.pitch, r, c, i)) return;
    if (r < 1 || r > a.ny - 2 || c < 1 || c > a.nx - 2) return;
    const double DRY = DRY_TOL;
    const long long E = i + 1, W = i - 1, N = i - a.pitch, S = i + a.pitch;
    const double eta = a.h1[i] + (a.z[i] + a.zb[i]);
    const bool stop_u = ((eta < a.z[E] + a.zb[E]) && (a.h1[E] < DRY)) || ((eta < a.z[W] + a.zb[W]) && (a.h1[W] < DRY)) ||
                        adj_nodata(a.nodata, E) || adj_nodata(a.nodata, W);
    const bool stop_v = ((eta < a.z[N] + a.zb[N]) && (a.h1[N] < DRY)) || ((eta < a.z[S] + a.zb[S]) && (a.h1[S] < DRY)) ||
                        adj_nodata(a.nodata, N) || adj_nodata(a.nodata, S);
    const bool active = (a.h1[i] > DRY) && !adj_nodata(a.nodata, i);
    if (!(active && !stop_u)) a.Thu[i] = 0.0;
    if (!(active && !stop_v)) a.Thv[i] = 0.0;
}

// hydro update backwards: I += T (identity paths) + face terms; dt adjoint.  NB: a fifth
// tangent in the cell's n_b (Manning friction of its faces) adds its adjoint to a.nbbar.
template <bool NB>
__global__ void __launch_bounds__(256) adj_hydro_kernel(const AdjArgs a) {
    int r, c;
    long long i;
    const bool in = adj_cell(a.ny, a.nx, a.pitch, r, c, i);
    double add_dt = 0.0;
    if (in) {
        using D = DualN<NB ? 5 : 4>;
        const double dt = *a.dt, dx = a.dx, DRY = DRY_TOL;
        const HCell<D> Cd = make_hcell(D::seed(a.h[i], 0), D::seed(a.hu[i], 1), D::seed(a.hv[i], 2),
                                       D::seed(a.zb[i], 3), D(a.z[i]), NB ? D::seed(a.nb[i], NB ? 4 : 0) : D(a.nb[i]));
        auto hconst = [&](long long k) {
            return make_hcell(D(a.h[k]), D(a.hu[k]), D(a.hv[k]), D(a.zb[k]), D(a.z[k]), D(a.nb[k]));
        };
        const bool mC = adj_nodata(a.nodata, i);
        const double k_ = -dt / dx;
        double g[NB ? 5 : 4] = {};
        double f[3] = {0, 0, 0};  // forward fluctuation sum of this cell
        // face (I|J): M goes to I, P to J
        auto face = [&](long long k, bool cell_is_I, bool yf) {
            const bool mk = adj_nodata(a.nodata, k);
            if (!(((a.h[i] > DRY) || (a.h[k] > DRY)) && !(mC || mk))) return;
            const HCell<D> Nd = hconst(k);
            D P[3], M[3];
            if (yf) {
                if (cell_is_I) roe_exner_face<D, true>(Cd, Nd, D(dx), P, M);
                else roe_exner_face<D, true>(Nd, Cd, D(dx), P, M);
            } else {
                if (cell_is_I) roe_exner_face<D, false>(Cd, Nd, D(dx), P, M);
                else roe_exner_face<D, false>(Nd, Cd, D(dx), P, M);
            }
            const long long I = cell_is_I ? i : k, J = cell_is_I ? k : i;
            const double aI[3] = {a.Th[I], a.Thu[I], a.Thv[I]}, aJ[3] = {a.Th[J], a.Thu[J], a.Thv[J]};
            for (int q = 0; q < (NB ? 5 : 4); ++q)
                for (int m = 0; m < 3; ++m) g[q] += k_ * (aI[m] * M[m].d[q] + aJ[m] * P[m].d[q]);
            for (int m = 0; m < 3; ++m) f[m] += cell_is_I ? M[m].v : P[m].v;
        };
        if (c + 1 < a.nx) face(i + 1, true, false);
        if (c >= 1) face(i - 1, false, false);
        if (r + 1 < a.ny) face(i + a.pitch, true, true);
        if (r >= 1) face(i - a.pitch, false, true);
        a.Ih[i] += a.Th[i] + g[0];
        a.Ihu[i] += a.Thu[i] + g[1];
        a.Ihv[i] += a.Thv[i] + g[2];
        a.Izb[i] += a.Tzb[i] + g[3];
        a.IG[i] += a.TG[i];
        if constexpr (NB) a.nbbar[i] += g[NB ? 4 : 0];
        add_dt = -(a.Th[i] * f[0] + a.Thu[i] * f[1] + a.Thv[i] * f[2]) / dx;
    }
    adj_dt_add(a.dtbar, add_dt);
}

// ---------------------------------------------------------------- handlers backwards

// pass 1: the boundary cells' adjoints of the fields the handler writes
__global__ void adj_bc_read_kernel(const AdjBcArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const unsigned fm = bc_field_mask(a.kind);
    const long long b = a.cells[k];
    for (int s = 0; s < 6; ++s) a.tmp[s * a.count + k] = ((fm >> s) & 1u) && a.f[s] ? a.f[s][b] : 0.0;
}

// pass 2: the overwritten fields of the boundary cells lose their adjoint
__global__ void adj_bc_zero_kernel(const AdjBcArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const unsigned fm = bc_field_mask(a.kind);
    const long long b = a.cells[k];
    for (int s = 0; s < 6; ++s)
        if (((fm >> s) & 1u) && a.f[s]) a.f[s][b] = 0.0;
}

// pass 3: donors receive the transposed Jacobian of the handler times the saved adjoints
__global__ void adj_bc_scatter_kernel(const AdjBcArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const long long d = a.donors[k];
    const double* t = a.tmp;
    const int n = a.count;
    auto add = [&](int s, double v) {
        if (a.f[s] && v != 0.0) atomicAdd(a.f[s] + d, v);
    };
    switch (a.kind) {
        case PXB_BC_RE_REFLECTIVE: {  // hu' = (-nx^2 + ny^2) hu - 2 nx ny hv, hv' = -2 nx ny hu + (nx^2 - ny^2) hv
            const double nx = a.nx, ny = a.ny;
            // forward: mom_n = hu nx + hv ny, mom_t = -hu ny + hv nx, hu' = -mom_n nx - mom_t ny,
            // hv' = -mom_n ny + mom_t nx
            const double bu = t[1 * n + k], bv = t[2 * n + k];
            const double bmn = -bu * nx - bv * ny, bmt = -bu * ny + bv * nx;
            add(0, t[0 * n + k]);
            add(1, bmn * nx - bmt * ny);
            add(2, bmn * ny + bmt * nx);
            add(3, t[3 * n + k]);
            add(5, t[5 * n + k]);
            break;
        }
        case PXB_BC_RE_TRANSMISSIVE:
            add(0, t[0 * n + k]);
            add(1, t[1 * n + k]);
            add(2, t[2 * n + k]);
            break;
        case PXB_BC_RE_TRANSMISSIVEBED:
        case PXB_BC_RE_STEEPFALL:
            add(3, t[3 * n + k]);
            break;
        case PXB_BC_RE_NORMALFLOWDEPTH:  // hu, hv copied; h and z_b prescribed
            add(1, t[1 * n + k]);
            add(2, t[2 * n + k]);
            break;
        case PXB_BC_RE_ZEROMOMENTUM:  // NaN values keep the cell's own momentum (its donor)
            if (a.c0 != a.c0) add(1, t[1 * n + k]);
            if (a.c1 != a.c1) add(2, t[2 * n + k]);
            break;
        case PXB_BC_RE_CONSTANTINFLUX:  // prescribed hu = q values[1], hv = q values[2]: the adjoint of q
            if (a.qbar) {
                const double v = t[1 * n + k] * a.vx + t[2 * n + k] * a.vy;
                if (v != 0.0) atomicAdd(a.qbar, v);
            }
            break;
        default:  // Berthon: prescribed values
            break;
    }
}

// compute_n of the initialisation backwards (roe_exner.py:64-73): n_b = n_p_mix where the
// raw z_b > SED_TOL (MPM), the raw n elsewhere (and everywhere with a constant grass
// factor).  The n_b adjoint moves to n (when nbar is set) or to n_p_mix (summed into
// *npbar); n_b's own value before the initialisation has no influence.
__global__ void __launch_bounds__(256) adj_compute_n_kernel(int ny, int nx, long long pitch, int mpm,
                                                            const double* zb, double* nbbar, double* nbar,
                                                            double* npbar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    double v[1] = {0.0};
    if (r < ny && c < nx) {
        const long long i = (long long)r * pitch + c;
        const double b = nbbar[i];
        if (mpm && zb[i] > SED_TOL) v[0] = b;
        else if (nbar) nbar[i] += b;
        nbbar[i] = 0.0;
    }
    adj_sum_add<1>(npbar, v);
}

// ---------------------------------------------------------------- dt backwards

__device__ __forceinline__ bool adj_face_speed(const AdjCflArgs& a, int r, int c, bool yf, double& s) {
    if (yf ? (r + 1 >= a.ny) : (c + 1 >= a.nx)) return false;
    const long long i = (long long)r * a.pitch + c, j = yf ? i + a.pitch : i + 1;
    if (!(((a.h[i] > DRY_TOL) || (a.h[j] > DRY_TOL)) && !(adj_nodata(a.nodata, i) || adj_nodata(a.nodata, j))))
        return false;
    const CCell<double> I = make_ccell(a.h[i], a.hu[i], a.hv[i], a.G[i]);
    const CCell<double> J = make_ccell(a.h[j], a.hu[j], a.hv[j], a.G[j]);
    s = yf ? face_speed<double, true>(I, J) : face_speed<double, false>(I, J);
    return true;
}

// pass 1: maximum speed (bits); pass 2: number of faces at it
__global__ void __launch_bounds__(256) adj_cfl_max_kernel(const AdjCflArgs a, int pass) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long best = 0ull;
    unsigned int ties = 0;
    if (r < a.ny && c < a.nx) {
        for (int yf = 0; yf < 2; ++yf) {
            double s;
            if (adj_face_speed(a, r, c, yf != 0, s)) {
                const unsigned long long b = speed_bits(s);
                if (pass == 0) best = b > best ? b : best;
                else ties += (b == *a.maxbits) ? 1u : 0u;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(FULL, best, o);
        best = ob > best ? ob : best;
        ties += __shfl_xor_sync(FULL, ties, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (pass == 0 && best != 0ull) atomicMax(a.maxbits, best);
        if (pass == 1 && ties) atomicAdd(a.nties, ties);
    }
}

// pass 3: d(dt)/d(s_max) spread over the tying faces, through their speeds' local Jacobians
__global__ void __launch_bounds__(256) adj_cfl_grad_kernel(const AdjCflArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= a.ny || c >= a.nx) return;
    const unsigned long long m = *a.maxbits;
    const double smax = bits_speed(m, 0.0);
    const double dt = a.cfl * (a.dx / smax);
    if (!(dt >= a.floor_dt) || *a.nties == 0u) return;  // the floor (or no face): dt does not depend on the state
    const double sbar = *a.dtbar * (-a.cfl * a.dx / (smax * smax)) / (double)*a.nties;
    for (int yf = 0; yf < 2; ++yf) {
        double s;
        if (!adj_face_speed(a, r, c, yf != 0, s) || speed_bits(s) != m) continue;
        using D = DualN<8>;
        const long long i = (long long)r * a.pitch + c, j = yf ? i + a.pitch : i + 1;
        const CCell<D> I = make_ccell(D::seed(a.h[i], 0), D::seed(a.hu[i], 1), D::seed(a.hv[i], 2), D::seed(a.G[i], 3));
        const CCell<D> J = make_ccell(D::seed(a.h[j], 4), D::seed(a.hu[j], 5), D::seed(a.hv[j], 6), D::seed(a.G[j], 7));
        const D sd = yf ? face_speed<D, true>(I, J) : face_speed<D, false>(I, J);
        atomicAdd(a.Ah + i, sbar * sd.d[0]);
        atomicAdd(a.Ahu + i, sbar * sd.d[1]);
        atomicAdd(a.Ahv + i, sbar * sd.d[2]);
        atomicAdd(a.AG + i, sbar * sd.d[3]);
        atomicAdd(a.Ah + j, sbar * sd.d[4]);
        atomicAdd(a.Ahu + j, sbar * sd.d[5]);
        atomicAdd(a.Ahv + j, sbar * sd.d[6]);
        atomicAdd(a.AG + j, sbar * sd.d[7]);
    }
}

}  // namespace pxb
