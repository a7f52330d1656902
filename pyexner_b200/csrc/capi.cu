// extern "C" boundary of the library (declared in include/pyexner_b200.h).
//
// Host-side responsibilities:
//   * validate arguments and layouts, and report errors through status codes plus a
//     thread-local message;
//   * resolve the ordered boundary handlers into per-ring-cell recipes (the symbolic
//     equivalent of applying PyExner's handlers one after another,
//     src/PyExner/domain/boundary_registry.py:183-187) and upload them once; layouts that
//     do not resolve run on the general stage path (re_general.cuh), which applies the
//     handlers one after another on the device;
//   * turn the sediment matrix into per-class constants;
//   * size the warp strips / row bands of the stage and CFL kernels to the device;
//   * capture the fixed-step integrator loops into CUDA graphs and replay them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "adjoint_args.cuh"
#include "pxb_launch.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define PXB_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(PXB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ recipe resolution
// Expression of one field group of one cell after some handlers: the value of that
// group at cell `src` before the whole application, mapped by `m` (momentum only),
// or a constant pair (momentum of ConstantInflux).
struct GroupExpr {
    long long src = -1;  // -1: identity (the cell itself)
    bool is_const = false;
    double m[4] = {1, 0, 0, 1};
    bool set = false;
};
struct CellExpr {
    GroupExpr h, mom, zb, g, n, z;
};

struct Resolved {
    std::vector<pxb_ring_recipe> ring;  // 2*nx + 2*ny
    std::string error;
};

GroupExpr ident(long long cell) {
    GroupExpr e;
    e.src = cell;
    return e;
}

GroupExpr get(const std::unordered_map<long long, CellExpr>& mp, long long cell, GroupExpr CellExpr::*grp) {
    auto it = mp.find(cell);
    if (it == mp.end() || !((it->second).*grp).set) return ident(cell);
    return (it->second).*grp;
}

GroupExpr map_mom(const GroupExpr& e, const double a[4]) {
    GroupExpr o = e;
    if (e.is_const) {
        o.m[0] = a[0] * e.m[0] + a[1] * e.m[1];
        o.m[1] = a[2] * e.m[0] + a[3] * e.m[1];
        o.m[2] = o.m[3] = 0;
    } else {
        o.m[0] = a[0] * e.m[0] + a[1] * e.m[2];
        o.m[1] = a[0] * e.m[1] + a[1] * e.m[3];
        o.m[2] = a[2] * e.m[0] + a[3] * e.m[2];
        o.m[3] = a[2] * e.m[1] + a[3] * e.m[3];
    }
    return o;
}

bool is_ring(long long r, long long c, long long ny, long long nx) {
    return r == 0 || r == ny - 1 || c == 0 || c == nx - 1;
}

// Apply the handler sequence symbolically; flat cell ids are row*nx + col.
Resolved resolve(const pxb_bc_handler* hs, int nh, int ny, int nx, long long pitch, bool roe, bool need_idempotent) {
    Resolved R;
    std::unordered_map<long long, CellExpr> mp;
    for (int k = 0; k < nh; ++k) {
        const pxb_bc_handler& H = hs[k];
        std::vector<std::pair<long long, CellExpr>> upd;
        upd.reserve(H.count);
        for (int p = 0; p < H.count; ++p) {
            const long long bc = H.cells[p], dc = H.donors[p];
            const long long b = (bc / pitch) * nx + (bc % pitch);
            const long long d = (dc / pitch) * nx + (dc % pitch);
            auto it = mp.find(b);
            CellExpr ne = (it == mp.end()) ? CellExpr() : it->second;
            auto setg = [](GroupExpr& dst, GroupExpr v) { v.set = true; dst = v; };
            const double nxv = H.nx, nyv = H.ny;
            switch (H.kind) {
                case PXB_BC_RE_REFLECTIVE: {
                    const double a[4] = {nyv * nyv - nxv * nxv, -2 * nxv * nyv, -2 * nxv * nyv, nxv * nxv - nyv * nyv};
                    setg(ne.h, get(mp, d, &CellExpr::h));
                    setg(ne.zb, get(mp, d, &CellExpr::zb));
                    setg(ne.n, get(mp, d, &CellExpr::n));
                    setg(ne.g, get(mp, d, &CellExpr::g));
                    setg(ne.mom, map_mom(get(mp, d, &CellExpr::mom), a));
                    break;
                }
                case PXB_BC_RE_TRANSMISSIVE:
                    setg(ne.h, get(mp, d, &CellExpr::h));
                    setg(ne.mom, get(mp, d, &CellExpr::mom));
                    break;
                case PXB_BC_RE_TRANSMISSIVEBED:
                    setg(ne.zb, get(mp, d, &CellExpr::zb));
                    break;
                case PXB_BC_RE_CONSTANTINFLUX: {
                    GroupExpr e;
                    e.is_const = true;
                    e.m[0] = H.hu_const;
                    e.m[1] = H.hv_const;
                    e.m[2] = e.m[3] = 0;
                    setg(ne.mom, e);
                    break;
                }
                case PXB_BC_ROE_REFLECTIVE: {
                    const double a[4] = {1 - 2 * nxv * nxv, 0, 0, 1 - 2 * nyv * nyv};
                    setg(ne.h, get(mp, d, &CellExpr::h));
                    setg(ne.z, get(mp, d, &CellExpr::z));
                    setg(ne.n, get(mp, d, &CellExpr::n));
                    setg(ne.mom, map_mom(get(mp, d, &CellExpr::mom), a));
                    break;
                }
                case PXB_BC_ROE_TRANSMISSIVE:
                    setg(ne.h, get(mp, d, &CellExpr::h));
                    setg(ne.z, get(mp, d, &CellExpr::z));
                    setg(ne.n, get(mp, d, &CellExpr::n));
                    setg(ne.mom, get(mp, d, &CellExpr::mom));
                    break;
                case PXB_BC_RE_CONSTANTOUTFLUX:
                case PXB_BC_RE_BERTHON:
                case PXB_BC_RE_NORMALFLOWDEPTH:
                case PXB_BC_RE_STEEPFALL:
                case PXB_BC_RE_ZEROMOMENTUM:
                    R.error = "boundary kind " + std::to_string(H.kind) +
                              " computes its values from the time or from donor values; it runs on the general "
                              "stage path only";
                    return R;
                default:
                    R.error = "unknown boundary kind " + std::to_string(H.kind);
                    return R;
            }
            upd.emplace_back(b, ne);
        }
        for (auto& u : upd) mp[u.first] = u.second;  // scatter after the gather
    }
    R.ring.assign((size_t)(2 * nx + 2 * ny), pxb_ring_recipe{});
    for (auto& kv : mp) {
        const long long cell = kv.first;
        const long long r = cell / nx, c = cell % nx;
        if (!is_ring(r, c, ny, nx)) {
            R.error = "boundary cell (" + std::to_string(r) + "," + std::to_string(c) +
                      ") is off the outer ring; the stage kernels support ring boundaries only";
            return R;
        }
        const CellExpr& e = kv.second;
        pxb_ring_recipe rc{};
        auto off = [&](const GroupExpr& g, int8_t& dy, int8_t& dx) -> bool {
            if (!g.set || g.is_const) return true;
            const long long sr = g.src / nx, sc = g.src % nx;
            const long long oy = sr - r, ox = sc - c;
            if (oy < -1 || oy > 1 || ox < -1 || ox > 1) return false;
            if (oy != 0 && !((r == 0 && oy > 0) || (r == ny - 1 && oy < 0))) return false;
            if (ox != 0 && !((c == 0 && ox > 0) || (c == nx - 1 && ox < 0))) return false;
            dy = (int8_t)oy;
            dx = (int8_t)ox;
            return true;
        };
        bool ok = off(e.h, rc.h_dy, rc.h_dx) && off(e.mom, rc.m_dy, rc.m_dx) && off(e.zb, rc.zb_dy, rc.zb_dx) &&
                  off(e.g, rc.g_dy, rc.g_dx);
        if (roe && ok) {
            // Roe handlers write h, z and n together: their donors coincide.
            if (e.z.set && e.z.src != e.h.src) ok = false;
            if (e.n.set && e.n.src != e.h.src) ok = false;
        }
        if (!ok) {
            R.error = "boundary cell (" + std::to_string(r) + "," + std::to_string(c) +
                      ") takes its value from a cell the stage kernels cannot reach (donor must be an adjacent cell "
                      "toward the interior)";
            return R;
        }
        if (e.h.set) rc.flags |= 1u;
        if (e.mom.set) {
            rc.flags |= 2u;
            if (e.mom.is_const) rc.flags |= 4u;
            for (int q = 0; q < 4; ++q) rc.m[q] = e.mom.m[q];
        }
        if (e.zb.set) rc.flags |= 8u;
        if (e.g.set) rc.flags |= 16u;
        if (r == 0) R.ring[(size_t)c] = rc;
        if (r == ny - 1) R.ring[(size_t)(nx + c)] = rc;
        if (c == 0) R.ring[(size_t)(2 * nx + r)] = rc;
        if (c == nx - 1) R.ring[(size_t)(2 * nx + ny + r)] = rc;
    }
    if (need_idempotent) {
        // The Roe-Exner stage stores h, hu, hv after the first application; that is
        // exact when a second application would not change them, i.e. when no donor
        // of a hydro recipe carries a hydro recipe itself.
        for (auto& kv : mp) {
            const long long cell = kv.first;
            const CellExpr& e = kv.second;
            // The kernel evaluates the second pass in registers from first-pass values of
            // donors in the same row (the cell itself included); a donor in another row
            // must not be a hydro boundary cell, so that its value is the same in both passes.
            auto bad = [&](const GroupExpr& g, GroupExpr CellExpr::*grp) {
                if (!g.set || g.is_const || g.src / nx == cell / nx) return false;
                auto it = mp.find(g.src);
                return it != mp.end() && ((it->second).*grp).set;
            };
            if (bad(e.h, &CellExpr::h) || bad(e.mom, &CellExpr::mom)) {
                const long long r = cell / nx, c = cell % nx;
                R.error = "boundary cell (" + std::to_string(r) + "," + std::to_string(c) +
                          ") copies a depth or momentum from a boundary cell in another row; the stage kernel "
                          "cannot apply the second boundary pass to it";
                return R;
            }
            // The fused kernel never writes n: the n left by the set-up application must be
            // a fixed point of the handlers, i.e. no cell copies n from a cell whose own n
            // comes from somewhere else.
            if (e.n.set && e.n.src != cell) {
                auto it = mp.find(e.n.src);
                if (it != mp.end() && it->second.n.set && it->second.n.src != e.n.src) {
                    const long long r = cell / nx, c = cell % nx;
                    R.error = "boundary cell (" + std::to_string(r) + "," + std::to_string(c) +
                              ") copies n from a boundary cell whose n changes with every application; the fused "
                              "stage kernel keeps n fixed";
                    return R;
                }
            }
        }
    }
    return R;
}

// ------------------------------------------------------------------ shared plan bits
struct DevHandler {
    int kind = 0, count = 0;
    long long* cells = nullptr;
    long long* donors = nullptr;
    double nx = 0, ny = 0, c0 = 0, c1 = 0;
    double q = 0, vx = 0, vy = 0, hb = 0;  // ConstantOutflux, NormalFlowDepth; vx, vy also ConstantInflux
    float neg_alpha = 0, zb0 = 0;          // Berthon, NormalFlowDepth
    double c0_dot = 0, c1_dot = 0;         // tangents of c0, c1 (tangent-linear runs only)
};

// A handler constant of the arithmetic type T; dual numbers also carry its tangent.
template <class T>
T make_val(double v, double) {
    return T(v);
}
template <>
pxb::Dual make_val<pxb::Dual>(double v, double d) {
    return pxb::Dual(v, d);
}

// Constants of the Berthon analytic inlet / outlet, in float32 like the reference's
// float32 values (roeexner_berthon.py:40-52, roeexner_normalflowdepth.py:34-41):
//   u = ((alpha x + beta) / A)^(1/3),  zb0 = -(u^3 + 2 g q) / (2 g max(u, 1e-12)) + gamma,
//   h = q / u.  u^3 is u * (u * u) (jax integer_pow); the cube root is the correctly
// rounded float32 power, taken in double precision and rounded once.
void berthon_constants(const double* v, DevHandler& d) {
    const float q = (float)v[0], A = (float)v[1], alpha = (float)v[2], beta = (float)v[3];
    const float gamma = (float)v[4], x = (float)v[5];
    const float ax = alpha * x;
    const float w = (ax + beta) / A;
    const float third = 1.0f / 3.0f;
    const float u = (float)std::pow((double)w, (double)third);
    const float g2 = (float)(2.0 * 9.81);
    const float u3 = u * (u * u);
    const float num = u3 + g2 * q;
    const float tiny = (float)1e-12;
    const float umax = (u != u) ? u : (u < tiny ? tiny : u);  // jnp.maximum (NaN propagates)
    const float den = g2 * umax;
    d.zb0 = -num / den + gamma;
    d.neg_alpha = -alpha;
    d.hb = (double)(q / u);
    d.q = q;
}

struct Geometry {
    int band_rows = 0, nstrips = 0, nbands = 0, grid = 0;
};

// Tallest band of the stage kernel's default geometry (tuning knob; float32 Gaussian bed:
// 160 and 192 measured alike at 8192^2, 160 ahead of 192 at 4096^2)
#ifndef PXB_STAGE_MAX_ROWS
#define PXB_STAGE_MAX_ROWS 176
#endif
// CFL work items per resident warp and the shortest band that rule may give (tuning knobs;
// 4 and 64 against 2 and 32: the same at 2048^2, 10 % faster CFL at 8192^2 with bedload
// everywhere, where the cubic's cost varies from item to item)
#ifndef PXB_CFL_ITEMS_PER_WARP
#define PXB_CFL_ITEMS_PER_WARP 4
#endif
#ifndef PXB_CFL_MIN_ROWS
#define PXB_CFL_MIN_ROWS 64
#endif

Geometry stage_geometry(int ny, int nx, int esize, int resident_warps, int want_rows) {
    Geometry g;
    const int sout = pxb_stage_strip_out(esize);
    g.nstrips = std::max(1, (nx - 3 + sout - 1) / sout);
    int rows = want_rows;
    if (rows <= 0) {
        // k rounds of items, each with about one item per resident warp (the work queue
        // hands out the items beyond the first), for the smallest k whose bands are at most
        // PXB_STAGE_MAX_ROWS tall: a whole number of rounds leaves no partial last round
        // with idle SMs, and on large grids several rounds of shorter bands keep the
        // concurrently active items close together in memory (halos shared through L2)
        const int ipb = pxb_stage_items_per_band(g.nstrips), span = ny - 1;
        int k = 1, bands = std::max(1, resident_warps / ipb);
        while ((span + bands - 1) / bands > PXB_STAGE_MAX_ROWS) bands = std::max(1, ++k * resident_warps / ipb);
        rows = std::max(8, (span + bands - 1) / bands);
    }
    g.band_rows = rows;
    g.nbands = std::max(1, (ny - 1 + rows - 1) / rows);
    const int items = pxb_stage_items_per_band(g.nstrips) * g.nbands;
    // Unless the grid is small, launch exactly the resident capacity: every SM then holds
    // the same number of blocks (a grid a little below capacity is spread unevenly by the
    // block scheduler), and the kernel's work queue hands out the items beyond one per warp.
    const int need = std::max(1, (items + 3) / 4), cap = std::max(1, resident_warps / 4);
    g.grid = need >= cap / 4 ? cap : need;
    return g;
}

Geometry cfl_geometry(int ny, int nx, int resident_warps) {
    Geometry g;
    g.nstrips = std::max(1, (nx + 30) / 31);
    // about PXB_CFL_ITEMS_PER_WARP items per resident warp, handed out by the kernel's queue
    // so that the SMs finish together; where that would make bands shorter than
    // PXB_CFL_MIN_ROWS rows (each band re-reads one row for its first y-faces) one item per
    // warp is faster
    const int target_bands = std::max(1, PXB_CFL_ITEMS_PER_WARP * resident_warps / g.nstrips);
    g.band_rows = (ny + target_bands - 1) / target_bands;
    if (g.band_rows < PXB_CFL_MIN_ROWS) {
        const int one = std::max(1, resident_warps / g.nstrips);
        g.band_rows = std::max(8, (ny + one - 1) / one);
    }
    g.nbands = std::max(1, (ny + g.band_rows - 1) / g.band_rows);
    const int items = g.nstrips * g.nbands;
    const int need = std::max(1, (items + 7) / 8), cap = std::max(1, resident_warps / 8);
    g.grid = need >= cap / 4 ? std::min(need, cap) : need;
    return g;
}

// Device memory of a plan: cudaMalloc'd (no arena), carved from a caller's workspace, or
// only counted (the size query of pxb_re_plan_workspace_size).  Carved blocks start on
// 256-byte boundaries.
struct DevArena {
    char* base = nullptr;  // the caller's workspace (carving), null when counting
    size_t cap = 0, used = 0;
    bool counting = false;
};

int arena_alloc(DevArena* A, void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (!A) {
        const cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return fail(PXB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return PXB_OK;
    }
    const size_t at = (A->used + 255) & ~(size_t)255;
    A->used = at + bytes;
    if (A->counting) return PXB_OK;
    if (A->used > A->cap) return fail(PXB_ERR_ARG, std::string("workspace too small (") + what + ")");
    *p = A->base + at;
    return PXB_OK;
}

// Host -> device copy unless the arena only counts.
int arena_copy(DevArena* A, void* dst, const void* src, size_t bytes) {
    if (A && A->counting) return PXB_OK;
    PXB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return PXB_OK;
}

int upload_handlers(const pxb_bc_handler* hs, int nh, long long max_index, std::vector<DevHandler>& out,
                    int& maxcount, DevArena* A = nullptr) {
    maxcount = 0;
    for (int k = 0; k < nh; ++k) {
        const pxb_bc_handler& H = hs[k];
        if (H.count < 0 || (H.count > 0 && (!H.cells || !H.donors)))
            return fail(PXB_ERR_ARG, "boundary handler " + std::to_string(k) + " has no index arrays");
        for (int p = 0; p < H.count; ++p)
            if (H.cells[p] < 0 || H.cells[p] >= max_index || H.donors[p] < 0 || H.donors[p] >= max_index)
                return fail(PXB_ERR_ARG, "boundary handler " + std::to_string(k) + " indexes outside the grid");
        DevHandler d;
        d.kind = H.kind;
        d.count = H.count;
        d.nx = H.nx;
        d.ny = H.ny;
        d.c0 = H.hu_const;
        d.c1 = H.hv_const;
        const double* v = H.values;
        switch (H.kind) {
            case PXB_BC_RE_CONSTANTOUTFLUX: {  // float32 values, float32 momenta (roeexner_constantoutflux.py:29-64)
                const float q = (float)v[0], vx = (float)v[1], vy = (float)v[2];
                d.q = q;
                d.vx = vx;
                d.vy = vy;
                d.c0 = (double)(q * vx);
                d.c1 = (double)(q * vy);
                break;
            }
            case PXB_BC_RE_BERTHON:
            case PXB_BC_RE_NORMALFLOWDEPTH:
                berthon_constants(v, d);
                break;
            case PXB_BC_RE_CONSTANTINFLUX:  // direction of the discharge, for its tangent
                d.vx = (float)v[1];
                d.vy = (float)v[2];
                break;
            case PXB_BC_RE_ZEROMOMENTUM:  // values[1] * normal (roeexner_zeromomentum.py:26-27)
                d.c0 = (double)(float)v[1] * H.nx;
                d.c1 = (double)(float)v[1] * H.ny;
                break;
            default:
                break;
        }
        if (H.count > 0) {
            const size_t nb = sizeof(long long) * H.count;
            int st = arena_alloc(A, (void**)&d.cells, nb, "boundary cells");
            if (st == PXB_OK) st = arena_alloc(A, (void**)&d.donors, nb, "boundary donors");
            if (st == PXB_OK) st = arena_copy(A, d.cells, H.cells, nb);
            if (st == PXB_OK) st = arena_copy(A, d.donors, H.donors, nb);
            if (st != PXB_OK) {
                out.push_back(d);  // released with the plan
                return st;
            }
        }
        maxcount = std::max(maxcount, H.count);
        out.push_back(d);
    }
    return PXB_OK;
}

// The float64 sediment constants of fill_sed with their tangents for a tangent of the
// sediment matrix (same operations on the values, so the values are fill_sed's bits).
void fill_sed_dual(pxb::SedTable<pxb::Dual>& S, const double* seds, const double* dseds, int nsed) {
    using pxb::Dual;
    auto at = [&](int row, int k) { return Dual(seds[row * nsed + k], dseds ? dseds[row * nsed + k] : 0.0); };
    S = pxb::SedTable<Dual>();
    S.n = nsed;
    Dual por_sum = 0.0, d50f_sum = 0.0;
    for (int k = 0; k < nsed; ++k) {
        const Dual frac = at(0, k), d50 = at(1, k), dens = at(2, k), thc = at(5, k), por = at(6, k);
        const Dual s = dens / Dual(1000.0);
        const Dual np_ = pxb::hpow(d50, 1.0 / 6.0) / Dual(21.1);
        S.s[k].np2 = np_ * np_;
        S.s[k].sm1d = (s - Dual(1.0)) * d50;
        S.s[k].thc = thc;
        S.s[k].np3sg = np_ * (np_ * np_) * Dual(std::sqrt(9.81));
        S.s[k].sm1 = s - Dual(1.0);
        S.s[k].frac = frac;
        por_sum = por_sum + por;
        d50f_sum = d50f_sum + d50 * frac;
    }
    S.one_minus_por = Dual(1.0) - por_sum / Dual((double)nsed);
    S.inv_one_minus_por = Dual(1.0) / (Dual(1.0) - por_sum / Dual((double)nsed));
    S.n_p_mix = pxb::hpow(d50f_sum / Dual((double)nsed), 1.0 / 6.0) / Dual(21.1);
}

template <class T>
void fill_sed(pxb::SedTable<T>& S, const double* seds, int nsed) {
    std::memset(&S, 0, sizeof(S));
    S.n = nsed;
    double por_sum = 0, d50f_sum = 0;
    for (int k = 0; k < nsed; ++k) {
        const double frac = seds[0 * nsed + k], d50 = seds[1 * nsed + k], dens = seds[2 * nsed + k];
        const double thc = seds[5 * nsed + k], por = seds[6 * nsed + k];
        const double s = dens / 1000.0;
        const double np_ = std::pow(d50, 1.0 / 6.0) / 21.1;
        S.s[k].np2 = (T)(np_ * np_);
        S.s[k].sm1d = (T)((s - 1.0) * d50);
        S.s[k].thc = (T)thc;
        S.s[k].np3sg = (T)(np_ * (np_ * np_) * std::sqrt(9.81));  // n_p**3 as jax integer_pow
        S.s[k].sm1 = (T)(s - 1.0);
        S.s[k].frac = (T)frac;
        por_sum += por;
        d50f_sum += d50 * frac;
    }
    S.one_minus_por = (T)(1.0 - por_sum / nsed);
    S.inv_one_minus_por = (T)(1.0 / (1.0 - por_sum / nsed));
    S.n_p_mix = (T)(std::pow(d50f_sum / nsed, 1.0 / 6.0) / 21.1);
    for (int k = 0; k < nsed; ++k) {
        const double frac = seds[0 * nsed + k], d50 = seds[1 * nsed + k], dens = seds[2 * nsed + k];
        const double s = dens / 1000.0;
        const double np_ = std::pow(d50, 1.0 / 6.0) / 21.1;
        S.k_theta[k] = (T)(np_ * np_ / ((s - 1.0) * d50));
        S.k_g1[k] = (T)(8.0 * frac * (np_ * (np_ * np_)) * std::sqrt(9.81) / (s - 1.0));
    }
}

struct PlanCommon {
    int ny = 0, nx = 0;
    long long pitch = 0;
    int dtype = 0;
    double dx = 0;
    int sm_count = 0;
    std::vector<DevHandler> handlers;
    pxb_ring_recipe* ring = nullptr;
    void* bc_tmp = nullptr;
    pxb::CflScratch* scr = nullptr;
    void* dt_dev = nullptr;
    cudaStream_t cap = nullptr;  // capture stream of the graph cache, created on first use
    bool ws = false;             // device memory carved from the caller's workspace
    Geometry cfl;
    // graph cache
    struct Cached {
        std::vector<const void*> key;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<Cached> graphs;

    size_t esize() const { return dtype == PXB_F64 ? 8 : 4; }

    void release() {
        for (auto& h : handlers) {
            if (!ws) cudaFree(h.cells);
            if (!ws) cudaFree(h.donors);
        }
        handlers.clear();
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        if (!ws) {
            cudaFree(ring);
            cudaFree(bc_tmp);
            cudaFree(scr);
            cudaFree(dt_dev);
        }
        if (cap) cudaStreamDestroy(cap);
        ring = nullptr;
        bc_tmp = nullptr;
        scr = nullptr;
        dt_dev = nullptr;
        cap = nullptr;
    }
};

// Boundary kinds a plan accepts: the "Roe Exner" handlers or the "Roe" handlers.
bool kind_ok(int kind, bool roe) {
    if (roe) return kind == PXB_BC_ROE_REFLECTIVE || kind == PXB_BC_ROE_TRANSMISSIVE;
    return (kind >= PXB_BC_RE_REFLECTIVE && kind <= PXB_BC_RE_CONSTANTINFLUX) ||
           (kind >= PXB_BC_RE_CONSTANTOUTFLUX && kind <= PXB_BC_RE_ZEROMOMENTUM);
}

// want_path: PXB_PATH_AUTO / _FUSED / _GENERAL (Roe plans: fused only); path: the result.
int common_setup(PlanCommon& P, int ny, int nx, long long pitch, int dtype, double dx, const pxb_bc_handler* hs,
                 int nh, bool roe, int want_path, int& path, DevArena* A = nullptr) {
    if (ny < 3 || nx < 3) return fail(PXB_ERR_ARG, "grid must be at least 3 x 3 cells including the ring");
    if (pitch < nx) return fail(PXB_ERR_ARG, "pitch smaller than nx");
    if ((long long)ny * pitch >= (1LL << 31)) return fail(PXB_ERR_ARG, "planes of 2^31 elements or more are not supported");
    if (dtype != PXB_F32 && dtype != PXB_F64) return fail(PXB_ERR_ARG, "dtype must be PXB_F32 or PXB_F64");
    if (!(dx > 0) || !std::isfinite(dx)) return fail(PXB_ERR_ARG, "dx must be positive and finite");
    if (nh < 0 || (nh > 0 && !hs)) return fail(PXB_ERR_ARG, "handlers pointer is null");
    P.ny = ny;
    P.nx = nx;
    P.pitch = pitch;
    P.dtype = dtype;
    P.dx = dx;
    int dev = 0;
    PXB_CUDA(cudaGetDevice(&dev));
    PXB_CUDA(cudaDeviceGetAttribute(&P.sm_count, cudaDevAttrMultiProcessorCount, dev));
    if (want_path < PXB_PATH_AUTO || want_path > PXB_PATH_GENERAL || (roe && want_path == PXB_PATH_GENERAL))
        return fail(PXB_ERR_ARG, "unknown stage path");
    for (int k = 0; k < nh; ++k)
        if (!kind_ok(hs[k].kind, roe))
            return fail(PXB_ERR_ARG, "boundary handler " + std::to_string(k) + " has kind " + std::to_string(hs[k].kind) +
                                         (roe ? ", not a \"Roe\" handler" : ", not a \"Roe Exner\" handler"));
    path = want_path == PXB_PATH_GENERAL ? PXB_PATH_GENERAL : PXB_PATH_FUSED;
    P.ws = A != nullptr;
    if (nh > 0) {
        int maxcount = 0;
        int st = upload_handlers(hs, nh, (long long)(ny - 1) * pitch + nx, P.handlers, maxcount, A);
        if (st != PXB_OK) return st;
        st = arena_alloc(A, &P.bc_tmp, 6 * (size_t)std::max(1, maxcount) * P.esize(), "boundary scratch");
        if (st != PXB_OK) return st;
        if (path == PXB_PATH_FUSED) {
            Resolved R = resolve(hs, nh, ny, nx, pitch, roe, !roe);
            if (!R.error.empty()) {
                if (want_path == PXB_PATH_FUSED || roe) return fail(PXB_ERR_UNSUPPORTED, R.error);
                path = PXB_PATH_GENERAL;
            } else {
                const size_t nb = sizeof(pxb_ring_recipe) * R.ring.size();
                st = arena_alloc(A, (void**)&P.ring, nb, "ring recipes");
                if (st == PXB_OK) st = arena_copy(A, P.ring, R.ring.data(), nb);
                if (st != PXB_OK) return st;
            }
        }
    }
    int st = arena_alloc(A, (void**)&P.scr, sizeof(pxb::CflScratch), "scratch");
    if (st == PXB_OK) st = arena_alloc(A, &P.dt_dev, 8, "time step");
    if (st != PXB_OK) return st;
    if (!(A && A->counting)) {
        PXB_CUDA(cudaMemset(P.scr, 0, sizeof(pxb::CflScratch)));
        PXB_CUDA(cudaMemset(P.dt_dev, 0, 8));
    }
    return PXB_OK;
}

int check_plan_error(PlanCommon& P, cudaStream_t s) {
    pxb::CflScratch h{};
    PXB_CUDA(cudaMemcpyAsync(&h, P.scr, sizeof(h), cudaMemcpyDeviceToHost, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    if (h.err != 0) {
        PXB_CUDA(cudaMemsetAsync(&P.scr->err, 0, sizeof(int), s));
        PXB_CUDA(cudaStreamSynchronize(s));
        return fail(PXB_ERR_NONFINITE, (h.err & 2) ? "non-finite time step (dry domain or NaN state)"
                                                   : "non-finite value in the updated state");
    }
    return PXB_OK;
}

// Run `body` captured into a graph (cached per key) and launch it `reps` times on `s`.
template <class F>
int run_graph(PlanCommon& P, const std::vector<const void*>& key, int reps, cudaStream_t s, F body) {
    cudaGraphExec_t exec = nullptr;
    for (auto& g : P.graphs)
        if (g.key == key) exec = g.exec;
    if (!exec) {
        cudaGraph_t graph;
        if (!P.cap) PXB_CUDA(cudaStreamCreateWithFlags(&P.cap, cudaStreamNonBlocking));
        PXB_CUDA(cudaStreamBeginCapture(P.cap, cudaStreamCaptureModeThreadLocal));
        const int st = body(P.cap);
        cudaGraph_t tmp = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(P.cap, &tmp);
        if (st != PXB_OK) {
            if (tmp) cudaGraphDestroy(tmp);
            return st;
        }
        if (ec != cudaSuccess) return fail(PXB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
        graph = tmp;
        PXB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        cudaGraphDestroy(graph);
        PlanCommon::Cached c;
        c.key = key;
        c.exec = exec;
        P.graphs.push_back(c);
    }
    for (int i = 0; i < reps; ++i) PXB_CUDA(cudaGraphLaunch(exec, s));
    return PXB_OK;
}

}  // namespace

namespace pxb {
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace pxb

// =====================================================================================
struct pxb_re_plan {
    PlanCommon c;
    int path = PXB_PATH_FUSED;
    void* gen = nullptr;  // general path: 7 scratch planes (h, hu, hv, z_b, G, n, z_b after Exner)
    // tangent-linear model (float64 plans): dual planes and scratch, allocated on first use
    void* jvp = nullptr;
    pxb::DualScratch* dscr = nullptr;
    void* jvp_tmp = nullptr;
    pxb::SedTable<pxb::Dual> sedD;
    std::vector<double> seds;  // the sediment matrix (7 x nsed), for the tangent tables
    int nsed = 0;
    int mpm = 0;
    const uint8_t* nodata = nullptr;
    Geometry stage[8];  // by (mpm, mask, avg) variant: band geometry from its occupancy
    int want_rows = 0;
    pxb::SedTable<float> sedf;
    pxb::SedTable<double> sedd;
    // volume budget (pxb_re_set_budget / pxb_re_volume): per-item outflow partials of the
    // stage kernel, the caller's accumulator, and the volume reduction's scratch
    double* bud_part = nullptr;
    long long bud_items = 0;
    pxb::BudgetAcc* bud_acc = nullptr;
    double* vol_scr = nullptr;
};

struct pxb_roe_plan {
    PlanCommon c;
};

// One member of a ragged ensemble.
struct EnsMember {
    int ny = 0, nx = 0;
    long long pitch = 0;
    double dx = 0;
    pxb_re_fields a{}, b{};
    const uint8_t* nodata = nullptr;
    pxb_ring_recipe* ring = nullptr;  // device, null without handlers
    std::vector<DevHandler> handlers;
};

struct pxb_re_ens {
    int dtype = 0, mpm = 0, nm = 0;
    int band_rows = 0;
    int sm_count = 0;
    int bps[2] = {1, 1};  // resident stage blocks per SM: plain, averaged
    bool has_mask = false;
    std::vector<EnsMember> m;
    std::vector<void*> owned;           // zero nodata planes of members without one
    void* bc_tmp = nullptr;
    pxb::SedTable<float> sedf;
    pxb::SedTable<double> sedd;
    pxb::CflScratch* scr = nullptr;     // one per member
    void* dt = nullptr;                 // one dt per member (dtype)
    // argument tables on the device: stage 0 a->b, 1 b->a, 2 b->a averaged with a, 3 a->b without G;
    // CFL 0 on a, 1 on b
    void* st_args[4] = {nullptr, nullptr, nullptr, nullptr};
    void* cfl_args[2] = {nullptr, nullptr};
    int* st_base = nullptr;
    int* cfl_base = nullptr;
    int st_total = 0, cfl_total = 0;
    double cfl_value = -1;
    const void* cfl_log = nullptr;
    cudaStream_t cap = nullptr;
    struct Cached {
        std::vector<const void*> key;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<Cached> graphs;

    size_t esize() const { return dtype == PXB_F64 ? 8 : 4; }
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    void release() {
        drop_graphs();
        for (auto& mb : m) {
            for (auto& h : mb.handlers) {
                cudaFree(h.cells);
                cudaFree(h.donors);
            }
            cudaFree(mb.ring);
        }
        m.clear();
        for (void* p : owned) cudaFree(p);
        owned.clear();
        for (auto& p : st_args) cudaFree(p), p = nullptr;
        for (auto& p : cfl_args) cudaFree(p), p = nullptr;
        cudaFree(st_base);
        cudaFree(cfl_base);
        cudaFree(bc_tmp);
        cudaFree(scr);
        cudaFree(dt);
        if (cap) cudaStreamDestroy(cap);
        st_base = cfl_base = nullptr;
        bc_tmp = nullptr;
        scr = nullptr;
        dt = nullptr;
        cap = nullptr;
    }
};

namespace {

template <class T>
const pxb::SedTable<T>& sed_of(const pxb_re_plan* p);
template <>
const pxb::SedTable<float>& sed_of<float>(const pxb_re_plan* p) { return p->sedf; }
template <>
const pxb::SedTable<double>& sed_of<double>(const pxb_re_plan* p) { return p->sedd; }
template <>
const pxb::SedTable<pxb::Dual>& sed_of<pxb::Dual>(const pxb_re_plan* p) { return p->sedD; }


int check_fields(const pxb_re_fields* f, bool need_g) {
    if (!f) return fail(PXB_ERR_ARG, "fields pointer is null");
    if (!f->h || !f->hu || !f->hv || !f->z_b) return fail(PXB_ERR_ARG, "h, hu, hv and z_b must be set");
    if (need_g && !f->G) return fail(PXB_ERR_ARG, "G must be set");
    return PXB_OK;
}

template <class T>
int re_cfl_impl(pxb_re_plan* P, const pxb_re_fields* f, double cfl, void* dt_out, void* dt_log, cudaStream_t s) {
    pxb::CflArgs<T> a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.h = (const T*)f->h;
    a.hu = (const T*)f->hu;
    a.hv = (const T*)f->hv;
    a.G = (const T*)f->G;
    a.nodata = P->nodata;
    a.dx = (T)P->c.dx;
    a.cfl = (T)cfl;
    a.floor_dt = (T)pxb::DT_FLOOR;
    a.scr = P->c.scr;
    a.dt_out = (T*)dt_out;
    a.dt_log = (T*)dt_log;
    a.band_rows = P->c.cfl.band_rows;
    a.nstrips = P->c.cfl.nstrips;
    a.nbands = P->c.cfl.nbands;
    PXB_CUDA(pxb::launch_re_cfl<T>(a, P->nodata != nullptr, P->c.cfl.grid, s));
    return PXB_OK;
}

template <class T>
int re_stage_impl(pxb_re_plan* P, const pxb_re_fields* in, const pxb_re_fields* out, const pxb_re_fields* avg,
                  const void* dt, cudaStream_t s, double bud_w = 0.0) {
    pxb::REStageArgs<T> a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.dx = (T)P->c.dx;
    a.h = (const T*)in->h;
    a.hu = (const T*)in->hu;
    a.hv = (const T*)in->hv;
    a.zb = (const T*)in->z_b;
    a.z = (const T*)in->z;
    a.nb = (const T*)in->n_b;
    a.G = (const T*)in->G;
    a.nodata = P->nodata;
    a.oh = (T*)out->h;
    a.ohu = (T*)out->hu;
    a.ohv = (T*)out->hv;
    a.ozb = (T*)out->z_b;
    a.oG = (T*)out->G;
    if (avg) {
        a.ah = (const T*)avg->h;
        a.ahu = (const T*)avg->hu;
        a.ahv = (const T*)avg->hv;
        a.azb = (const T*)avg->z_b;
        a.aG = (const T*)avg->G;
    }
    a.dt = (const T*)dt;
    a.ring = P->c.ring;
    a.sed = sed_of<T>(P);
    const int v = (P->mpm ? 4 : 0) | (P->nodata ? 2 : 0) | (avg ? 1 : 0);
    const Geometry& g = P->stage[v];
    a.band_rows = g.band_rows;
    a.nstrips = g.nstrips;
    a.nbands = g.nbands;
    a.err = &P->c.scr->err;
    a.queue = P->c.scr->queue;
    const long long nitems = (long long)pxb_stage_items_per_band(g.nstrips) * g.nbands;
    const bool bud = bud_w > 0.0 && P->bud_acc && P->bud_part;
    if (bud && nitems > P->bud_items) return fail(PXB_ERR_ARG, "budget partials smaller than the band geometry");
    if (bud) a.bud = P->bud_part;
    PXB_CUDA(pxb::launch_re_stage<T>(a, P->mpm != 0, P->nodata != nullptr, avg != nullptr, g.grid, s));
    if (bud)
        PXB_CUDA(pxb::launch_budget_stage<T>(P->bud_part, (int)nitems, (const T*)dt, bud_w * P->c.dx, P->bud_acc, s));
    return PXB_OK;
}

// Every handler in order on the field slots f (h, hu, hv, z_b, n, G), at the time *tptr
// (device) or tval.
template <class T>
int apply_handlers(const std::vector<DevHandler>& hs, void* bc_tmp, T* const f[6], const double* tptr, double tval,
                   cudaStream_t s) {
    for (auto& h : hs) {
        pxb::BcArgs<T> b{};
        for (int k = 0; k < 6; ++k) b.f[k] = f[k];
        b.cells = h.cells;
        b.donors = h.donors;
        b.count = h.count;
        b.kind = h.kind;
        b.nx = (T)h.nx;
        b.ny = (T)h.ny;
        b.c0 = make_val<T>(h.c0, h.c0_dot);
        b.c1 = make_val<T>(h.c1, h.c1_dot);
        b.q = (T)h.q;
        b.vx = (T)h.vx;
        b.vy = (T)h.vy;
        b.neg_alpha = h.neg_alpha;
        b.zb0 = h.zb0;
        b.hb = (T)h.hb;
        b.tptr = tptr;
        b.tval = tval;
        b.tmp = (T*)bc_tmp;
        PXB_CUDA(pxb::launch_bc<T>(b, s));
    }
    return PXB_OK;
}

template <class T>
int apply_handlers(PlanCommon& C, T* const f[6], const double* tptr, double tval, cudaStream_t s) {
    return apply_handlers<T>(C.handlers, C.bc_tmp, f, tptr, tval, s);
}

// init_fn_roeexner on one grid: n_b and G, then the handlers at t = 0.
template <class T>
int init_fields(int ny, int nx, long long pitch, const pxb_re_fields* f, const uint8_t* nodata, int mpm,
                const pxb::SedTable<T>& sed, const std::vector<DevHandler>& hs, void* bc_tmp, cudaStream_t s) {
    pxb::InitArgs<T> a{};
    a.ny = ny;
    a.nx = nx;
    a.pitch = pitch;
    a.h = (const T*)f->h;
    a.hu = (const T*)f->hu;
    a.hv = (const T*)f->hv;
    a.zb = (const T*)f->z_b;
    a.n = (const T*)f->n;
    a.nb = (T*)f->n_b;
    a.G = (T*)f->G;
    a.nodata = nodata;
    a.mpm = mpm;
    a.sed = sed;
    PXB_CUDA(pxb::launch_re_init<T>(a, s));
    T* const fs[6] = {(T*)f->h, (T*)f->hu, (T*)f->hv, (T*)f->z_b, (T*)f->n, (T*)f->G};
    return apply_handlers<T>(hs, bc_tmp, fs, nullptr, 0.0, s);
}

// One stage on the general path (re_general.cuh).
template <class T>
int re_general_impl(pxb_re_plan* P, const pxb_re_fields* in, const pxb_re_fields* out, const pxb_re_fields* avg,
                    const void* dt, const double* tptr, double tval, cudaStream_t s, void* scratch = nullptr,
                    void* bc_tmp = nullptr) {
    const size_t plane = (size_t)P->c.ny * (size_t)P->c.pitch;
    T* S = (T*)(scratch ? scratch : P->gen);
    void* tmp = bc_tmp ? bc_tmp : P->c.bc_tmp;
    pxb::GenArgs<T> a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.dx = (T)P->c.dx;
    a.h = (const T*)in->h;
    a.hu = (const T*)in->hu;
    a.hv = (const T*)in->hv;
    a.zb = (const T*)in->z_b;
    a.z = (const T*)in->z;
    a.nb = (const T*)in->n_b;
    a.G = (const T*)in->G;
    a.n = (const T*)in->n;
    a.sh = S;
    a.shu = S + plane;
    a.shv = S + 2 * plane;
    a.szb = S + 3 * plane;
    a.sG = S + 4 * plane;
    a.sn = S + 5 * plane;
    a.szb2 = S + 6 * plane;
    a.nodata = P->nodata;
    a.dt = (const T*)dt;
    a.sed = sed_of<T>(P);
    a.mpm = P->mpm;
    a.oh = (T*)out->h;
    a.ohu = (T*)out->hu;
    a.ohv = (T*)out->hv;
    a.ozb = (T*)out->z_b;
    a.oG = (T*)out->G;
    // n is carried when the input has it (and the partner too, for an averaged stage)
    a.on = (in->n && (!avg || avg->n)) ? (T*)out->n : nullptr;
    if (avg) {
        a.ah = (const T*)avg->h;
        a.ahu = (const T*)avg->hu;
        a.ahv = (const T*)avg->hv;
        a.azb = (const T*)avg->z_b;
        a.aG = (const T*)avg->G;
        a.an = (const T*)avg->n;
    }
    a.err = &P->c.scr->err;
    PXB_CUDA(pxb::launch_re_general<T>(a, pxb::GEN_HYDRO, s));
    PXB_CUDA(pxb::launch_re_general<T>(a, pxb::GEN_CORR, s));
    T* const f1[6] = {a.sh, a.shu, a.shv, a.szb, a.sn, a.sG};
    int st = apply_handlers<T>(P->c.handlers, tmp, f1, tptr, tval, s);
    if (st != PXB_OK) return st;
    PXB_CUDA(pxb::launch_re_general<T>(a, pxb::GEN_GRASS, s));
    PXB_CUDA(pxb::launch_re_general<T>(a, pxb::GEN_EXNER, s));
    T* const f2[6] = {a.sh, a.shu, a.shv, a.szb2, a.sn, a.sG};
    st = apply_handlers<T>(P->c.handlers, tmp, f2, tptr, tval, s);
    if (st != PXB_OK) return st;
    PXB_CUDA(pxb::launch_re_general<T>(a, pxb::GEN_STORE, s));
    return PXB_OK;
}

template <class T>
int re_init_impl(pxb_re_plan* P, const pxb_re_fields* f, cudaStream_t s) {
    return init_fields<T>(P->c.ny, P->c.nx, P->c.pitch, f, P->nodata, P->mpm, sed_of<T>(P), P->c.handlers,
                          P->c.bc_tmp, s);
}

// Band heights of the fused stage kernel timed on this state (stage a -> b, plain and
// averaged with a; a is not written); the fastest is kept for every variant.
template <class T>
int re_autotune_impl(pxb_re_plan* P, const pxb_re_fields* A, const pxb_re_fields* B, cudaStream_t s, int32_t* out) {
    const bool f64 = P->c.dtype == PXB_F64;
    auto set_rows = [&](int rows) {
        for (int v = 0; v < 8; ++v) {
            const bool mpm = v & 4, hm = v & 2, avg = v & 1;
            const int bps = f64 ? pxb::re_stage_blocks_per_sm<double>(mpm, hm, avg)
                                : pxb::re_stage_blocks_per_sm<float>(mpm, hm, avg);
            P->stage[v] = stage_geometry(P->c.ny, P->c.nx, f64 ? 8 : 4, std::max(1, bps) * 4 * P->c.sm_count, rows);
        }
    };
    set_rows(0);
    const int r0 = P->stage[(P->mpm ? 4 : 0) | (P->nodata ? 2 : 0)].band_rows;
    std::vector<int> cand = {r0, 2 * r0, 3 * r0, 4 * r0, 8, 16, 24, 32, 48, 64, 96, 128, 192, 256};
    std::vector<int> uniq;
    for (int c : cand)
        if (c >= 8 && c <= std::max(8, P->c.ny) && std::find(uniq.begin(), uniq.end(), c) == uniq.end())
            uniq.push_back(c);
    pxb_re_fields Bs = *B;
    Bs.z = A->z;
    Bs.n_b = A->n_b;
    int st = re_cfl_impl<T>(P, A, 0.5, P->c.dt_dev, nullptr, s);  // a dt for the timed stages
    if (st != PXB_OK) return st;
    cudaEvent_t e0, e1;
    PXB_CUDA(cudaEventCreate(&e0));
    PXB_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    int best = r0;
    for (int rows : uniq) {
        set_rows(rows);
        float ms = 1e30f;
        for (int rep = 0; rep < 4 && st == PXB_OK; ++rep) {  // the first repetition warms up
            cudaEventRecord(e0, s);
            st = re_stage_impl<T>(P, A, &Bs, nullptr, P->c.dt_dev, s);
            if (st == PXB_OK) st = re_stage_impl<T>(P, A, &Bs, A, P->c.dt_dev, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) ms = std::min(ms, t);
        }
        if (st != PXB_OK) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = rows;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != PXB_OK) return st;
    P->want_rows = best;
    set_rows(best);
    for (auto& g : P->c.graphs) cudaGraphExecDestroy(g.exec);  // captured with the old geometry
    P->c.graphs.clear();
    if (out) *out = best;
    return PXB_OK;
}

// One stage on the plan's path; the general path reads the time from *tptr or tval.
int re_stage_any(pxb_re_plan* P, const pxb_re_fields* in, const pxb_re_fields* out, const pxb_re_fields* avg,
                 const void* dt, const double* tptr, double tval, cudaStream_t s, double bud_w = 0.0) {
    const bool f64 = P->c.dtype == PXB_F64;
    if (P->path == PXB_PATH_GENERAL)
        return f64 ? re_general_impl<double>(P, in, out, avg, dt, tptr, tval, s)
                   : re_general_impl<float>(P, in, out, avg, dt, tptr, tval, s);
    return f64 ? re_stage_impl<double>(P, in, out, avg, dt, s, bud_w)
               : re_stage_impl<float>(P, in, out, avg, dt, s, bud_w);
}

int re_steps(pxb_re_plan* P, const pxb_re_fields* A, const pxb_re_fields* B, int nsteps, int scheme, double cfl,
             double t0, void* dt_log, cudaStream_t s) {
    const bool f64 = P->c.dtype == PXB_F64;
    const bool general = P->path == PXB_PATH_GENERAL;
    auto cfl_call = [&](const pxb_re_fields* f, cudaStream_t st) {
        return f64 ? re_cfl_impl<double>(P, f, cfl, P->c.dt_dev, dt_log, st)
                   : re_cfl_impl<float>(P, f, cfl, P->c.dt_dev, dt_log, st);
    };
    // the time of the step is the one the CFL launch before the stage recorded
    const double* tdev = &P->c.scr->t_step;
    // with a budget accumulator set, every stage adds its boundary outflow weighted by the
    // integrator: u^{n+1} - u^n = -dt R(u^n) (Forward Euler), -dt/2 (R(u^n) + R(u^(1))) (SSPRK2)
    const double bud_w = (P->bud_acc && !general) ? (scheme == PXB_SSPRK2 ? 0.5 : 1.0) : 0.0;
    auto stage_call = [&](const pxb_re_fields* in, const pxb_re_fields* out, const pxb_re_fields* avg,
                          cudaStream_t st) { return re_stage_any(P, in, out, avg, P->c.dt_dev, tdev, 0.0, st, bud_w); };
    // static planes of b are those of a; the general path carries n in b as well
    pxb_re_fields Bs = *B;
    Bs.z = A->z;
    Bs.n_b = A->n_b;
    if (general) {
        if (A->n && (!B->n || B->n == A->n))
            return fail(PXB_ERR_ARG, "the general stage path needs b->n distinct from a->n");
    } else {
        Bs.n = A->n;
    }
    const double cfl_d = cfl;
    std::vector<const void*> key = {A->h, A->hu, A->hv, A->z_b, A->G, A->z, A->n_b, A->n, B->h, B->hu, B->hv,
                                    B->z_b, B->G, Bs.n, dt_log, (const void*)(intptr_t)scheme};
    key.push_back(*(const void* const*)&cfl_d);
    key.push_back((const void*)P->bud_acc);
    PXB_CUDA(cudaMemsetAsync(&P->c.scr->step, 0, sizeof(unsigned int), s));
    // only the general path has handlers that read the time
    if (general)
        PXB_CUDA(f64 ? pxb::launch_set_time<double>(P->c.scr, t0, s) : pxb::launch_set_time<float>(P->c.scr, t0, s));
    if (scheme == PXB_SSPRK2) {
        pxb_re_fields B1 = Bs;
        if (P->mpm) B1.G = nullptr;  // stage-1 G is recomputed by stage 2
        return run_graph(P->c, key, nsteps, s, [&](cudaStream_t st) {
            int r = cfl_call(A, st);
            if (r == PXB_OK) r = stage_call(A, &B1, nullptr, st);
            if (r == PXB_OK) r = stage_call(&Bs, A, A, st);
            return r;
        });
    }
    // Forward Euler: a -> b -> a pairs, then one odd step and a copy back.
    int r = run_graph(P->c, key, nsteps / 2, s, [&](cudaStream_t st) {
        int q = cfl_call(A, st);
        if (q == PXB_OK) q = stage_call(A, &Bs, nullptr, st);
        if (q == PXB_OK) q = cfl_call(&Bs, st);
        if (q == PXB_OK) q = stage_call(&Bs, A, nullptr, st);
        return q;
    });
    if (r != PXB_OK || (nsteps & 1) == 0) return r;
    r = cfl_call(A, s);
    if (r == PXB_OK) r = stage_call(A, &Bs, nullptr, s);
    if (r != PXB_OK) return r;
    const size_t es = P->c.esize();
    const void* src[6] = {Bs.h, Bs.hu, Bs.hv, Bs.z_b, Bs.G, Bs.n};
    void* dst[6] = {A->h, A->hu, A->hv, A->z_b, A->G, A->n};
    const int ncopy = (general && A->n) ? 6 : 5;
    for (int k = 0; k < ncopy; ++k)
        PXB_CUDA(cudaMemcpy2DAsync(dst[k], P->c.pitch * es, src[k], P->c.pitch * es, P->c.nx * es, P->c.ny,
                                   cudaMemcpyDeviceToDevice, s));
    return PXB_OK;
}

// ------------------------------------------------------------------ plain Roe
template <class T>
int roe_cfl_impl(pxb_roe_plan* P, const pxb_roe_fields* f, double cfl, void* dt_out, void* dt_log, cudaStream_t s) {
    pxb::CflArgs<T> a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.h = (const T*)f->h;
    a.hu = (const T*)f->hu;
    a.hv = (const T*)f->hv;
    a.dx = (T)P->c.dx;
    a.cfl = (T)cfl;
    a.floor_dt = T(0);
    a.scr = P->c.scr;
    a.dt_out = (T*)dt_out;
    a.dt_log = (T*)dt_log;
    const long long cells = (long long)P->c.ny * P->c.nx;
    const int grid = (int)std::max(1LL, std::min<long long>((cells + 255) / 256, 4LL * P->c.sm_count));
    PXB_CUDA(pxb::launch_roe_cfl<T>(a, grid, s));
    return PXB_OK;
}

template <class T>
int roe_stage_impl(pxb_roe_plan* P, const pxb_roe_fields* in, const pxb_roe_fields* out, const pxb_roe_fields* avg,
                   const void* dt, cudaStream_t s) {
    pxb::RoeArgs<T> a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.dx = (T)P->c.dx;
    a.h = (const T*)in->h;
    a.hu = (const T*)in->hu;
    a.hv = (const T*)in->hv;
    a.z = (const T*)in->z;
    a.n = (const T*)in->n;
    a.oh = (T*)out->h;
    a.ohu = (T*)out->hu;
    a.ohv = (T*)out->hv;
    a.oz = (T*)out->z;
    a.on = (T*)out->n;
    if (avg) {
        a.ah = (const T*)avg->h;
        a.ahu = (const T*)avg->hu;
        a.ahv = (const T*)avg->hv;
        a.az = (const T*)avg->z;
        a.an = (const T*)avg->n;
    }
    a.dt = (const T*)dt;
    a.ring = P->c.ring;
    a.err = &P->c.scr->err;
    PXB_CUDA(pxb::launch_roe_stage<T>(a, avg != nullptr, s));
    return PXB_OK;
}

int check_roe_fields(const pxb_roe_fields* f) {
    if (!f || !f->h || !f->hu || !f->hv || !f->z || !f->n) return fail(PXB_ERR_ARG, "h, hu, hv, z and n must be set");
    return PXB_OK;
}

// ------------------------------------------------------------------ ragged ensembles
template <class T>
const pxb::SedTable<T>& ens_sed(const pxb_re_ens* E);
template <>
const pxb::SedTable<float>& ens_sed<float>(const pxb_re_ens* E) { return E->sedf; }
template <>
const pxb::SedTable<double>& ens_sed<double>(const pxb_re_ens* E) { return E->sedd; }

constexpr int ENS_CFL_ROWS = 32;  // rows per CFL work item

template <class T>
pxb::REStageArgs<T> ens_stage_args(const pxb_re_ens* E, int k, const pxb_re_fields* in, const pxb_re_fields* out,
                                   const pxb_re_fields* avg, const pxb_re_fields* statics) {
    const EnsMember& mb = E->m[(size_t)k];
    pxb::REStageArgs<T> a{};
    a.ny = mb.ny;
    a.nx = mb.nx;
    a.pitch = mb.pitch;
    a.dx = (T)mb.dx;
    a.h = (const T*)in->h;
    a.hu = (const T*)in->hu;
    a.hv = (const T*)in->hv;
    a.zb = (const T*)in->z_b;
    a.z = (const T*)statics->z;
    a.nb = (const T*)statics->n_b;
    a.G = (const T*)in->G;
    a.nodata = mb.nodata;
    a.oh = (T*)out->h;
    a.ohu = (T*)out->hu;
    a.ohv = (T*)out->hv;
    a.ozb = (T*)out->z_b;
    a.oG = (T*)out->G;
    if (avg) {
        a.ah = (const T*)avg->h;
        a.ahu = (const T*)avg->hu;
        a.ahv = (const T*)avg->hv;
        a.azb = (const T*)avg->z_b;
        a.aG = (const T*)avg->G;
    }
    a.dt = (const T*)E->dt + k;
    a.ring = mb.ring;
    a.sed = ens_sed<T>(E);
    a.band_rows = E->band_rows;
    const int sout = pxb_stage_strip_out((int)sizeof(T));
    a.nstrips = std::max(1, (mb.nx - 3 + sout - 1) / sout);
    a.nbands = std::max(1, (mb.ny - 1 + E->band_rows - 1) / E->band_rows);
    a.err = &E->scr[k].err;
    return a;
}

// Stage argument tables and item offsets for the current band height.
template <class T>
int ens_build_stage_tables(pxb_re_ens* E) {
    std::vector<pxb::REStageArgs<T>> t[4];
    std::vector<int> base(1, 0);
    for (int k = 0; k < E->nm; ++k) {
        const EnsMember& mb = E->m[(size_t)k];
        pxb_re_fields b_noG = mb.b;  // SSPRK2 stage 1 in MPM mode: G is recomputed by stage 2
        b_noG.G = nullptr;
        t[0].push_back(ens_stage_args<T>(E, k, &mb.a, &mb.b, nullptr, &mb.a));
        t[1].push_back(ens_stage_args<T>(E, k, &mb.b, &mb.a, nullptr, &mb.a));
        t[2].push_back(ens_stage_args<T>(E, k, &mb.b, &mb.a, &mb.a, &mb.a));
        t[3].push_back(ens_stage_args<T>(E, k, &mb.a, &b_noG, nullptr, &mb.a));
        const pxb::REStageArgs<T>& a = t[0].back();
        base.push_back(base.back() + pxb_stage_items_per_band(a.nstrips) * a.nbands);
    }
    for (int v = 0; v < 4; ++v) {
        if (!E->st_args[v]) PXB_CUDA(cudaMalloc(&E->st_args[v], sizeof(pxb::REStageArgs<T>) * E->nm));
        PXB_CUDA(cudaMemcpy(E->st_args[v], t[v].data(), sizeof(pxb::REStageArgs<T>) * E->nm, cudaMemcpyHostToDevice));
    }
    if (!E->st_base) PXB_CUDA(cudaMalloc(&E->st_base, sizeof(int) * (E->nm + 1)));
    PXB_CUDA(cudaMemcpy(E->st_base, base.data(), sizeof(int) * (E->nm + 1), cudaMemcpyHostToDevice));
    E->st_total = base.back();
    E->drop_graphs();
    return PXB_OK;
}

// CFL argument tables for a cfl number and a dt log.
template <class T>
int ens_build_cfl_tables(pxb_re_ens* E, double cfl, void* dt_log) {
    std::vector<pxb::CflArgs<T>> t[2];
    std::vector<int> base(1, 0);
    for (int k = 0; k < E->nm; ++k) {
        const EnsMember& mb = E->m[(size_t)k];
        for (int v = 0; v < 2; ++v) {
            const pxb_re_fields& f = v == 0 ? mb.a : mb.b;
            pxb::CflArgs<T> a{};
            a.ny = mb.ny;
            a.nx = mb.nx;
            a.pitch = mb.pitch;
            a.h = (const T*)f.h;
            a.hu = (const T*)f.hu;
            a.hv = (const T*)f.hv;
            a.G = (const T*)f.G;
            a.nodata = mb.nodata;
            a.dx = (T)mb.dx;
            a.cfl = (T)cfl;
            a.floor_dt = (T)pxb::DT_FLOOR;
            a.scr = E->scr + k;
            a.dt_out = (T*)E->dt + k;
            a.dt_log = (T*)dt_log;
            a.band_rows = ENS_CFL_ROWS;
            a.nstrips = std::max(1, (mb.nx + 30) / 31);
            a.nbands = std::max(1, (mb.ny + ENS_CFL_ROWS - 1) / ENS_CFL_ROWS);
            t[v].push_back(a);
        }
        base.push_back(base.back() + t[0].back().nstrips * t[0].back().nbands);
    }
    for (int v = 0; v < 2; ++v) {
        if (!E->cfl_args[v]) PXB_CUDA(cudaMalloc(&E->cfl_args[v], sizeof(pxb::CflArgs<T>) * E->nm));
        PXB_CUDA(cudaMemcpy(E->cfl_args[v], t[v].data(), sizeof(pxb::CflArgs<T>) * E->nm, cudaMemcpyHostToDevice));
    }
    if (!E->cfl_base) PXB_CUDA(cudaMalloc(&E->cfl_base, sizeof(int) * (E->nm + 1)));
    PXB_CUDA(cudaMemcpy(E->cfl_base, base.data(), sizeof(int) * (E->nm + 1), cudaMemcpyHostToDevice));
    E->cfl_total = base.back();
    E->cfl_value = cfl;
    E->cfl_log = dt_log;
    E->drop_graphs();
    return PXB_OK;
}

template <class T>
int ens_stage_launch(pxb_re_ens* E, int v, cudaStream_t s) {
    pxb::EnsStageArgs<T> a{};
    a.args = (const pxb::REStageArgs<T>*)E->st_args[v];
    a.base = E->st_base;
    a.nmembers = E->nm;
    a.queue = E->scr[0].queue;
    const bool avg = v == 2;
    const int grid = std::max(1, std::min((E->st_total + 3) / 4, std::max(1, E->bps[avg ? 1 : 0]) * E->sm_count));
    PXB_CUDA(pxb::launch_ens_stage<T>(a, E->mpm != 0, E->has_mask, avg, grid, s));
    return PXB_OK;
}

template <class T>
int ens_cfl_launch(pxb_re_ens* E, int v, cudaStream_t s) {
    pxb::EnsCflArgs<T> a{};
    a.args = (const pxb::CflArgs<T>*)E->cfl_args[v];
    a.base = E->cfl_base;
    a.nmembers = E->nm;
    a.log_stride = E->nm;
    const int grid = std::max(1, std::min((E->cfl_total + 7) / 8, 8 * E->sm_count));
    PXB_CUDA(pxb::launch_ens_cfl<T>(a, E->has_mask, grid, s));
    return PXB_OK;
}

template <class T>
int ens_run_impl(pxb_re_ens* E, int nsteps, int scheme, double cfl, void* dt_log, cudaStream_t s) {
    if (cfl != E->cfl_value || dt_log != E->cfl_log) {
        const int st = ens_build_cfl_tables<T>(E, cfl, dt_log);
        if (st != PXB_OK) return st;
    }
    // the dt log restarts at row 0
    PXB_CUDA(cudaMemset2DAsync(&E->scr[0].step, sizeof(pxb::CflScratch), 0, sizeof(unsigned int), E->nm, s));
    std::vector<const void*> key = {(const void*)(intptr_t)scheme, (const void*)(intptr_t)E->band_rows};
    auto body_rk = [&](cudaStream_t st) {
        int r = ens_cfl_launch<T>(E, 0, st);
        if (r == PXB_OK) r = ens_stage_launch<T>(E, E->mpm ? 3 : 0, st);
        if (r == PXB_OK) r = ens_stage_launch<T>(E, 2, st);
        return r;
    };
    auto body_fe2 = [&](cudaStream_t st) {
        int r = ens_cfl_launch<T>(E, 0, st);
        if (r == PXB_OK) r = ens_stage_launch<T>(E, 0, st);
        if (r == PXB_OK) r = ens_cfl_launch<T>(E, 1, st);
        if (r == PXB_OK) r = ens_stage_launch<T>(E, 1, st);
        return r;
    };
    const int reps = scheme == PXB_SSPRK2 ? nsteps : nsteps / 2;
    if (reps > 0) {
        cudaGraphExec_t exec = nullptr;
        for (auto& g : E->graphs)
            if (g.key == key) exec = g.exec;
        if (!exec) {
            PXB_CUDA(cudaStreamBeginCapture(E->cap, cudaStreamCaptureModeThreadLocal));
            const int st = scheme == PXB_SSPRK2 ? body_rk(E->cap) : body_fe2(E->cap);
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(E->cap, &graph);
            if (st != PXB_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ec != cudaSuccess) return fail(PXB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
            const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) return fail(PXB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
            pxb_re_ens::Cached c;
            c.key = key;
            c.exec = exec;
            E->graphs.push_back(c);
        }
        for (int i = 0; i < reps; ++i) PXB_CUDA(cudaGraphLaunch(exec, s));
    }
    if (scheme == PXB_SSPRK2 || (nsteps & 1) == 0) return PXB_OK;
    // odd Forward-Euler step: a -> b, then b back into a
    int r = ens_cfl_launch<T>(E, 0, s);
    if (r == PXB_OK) r = ens_stage_launch<T>(E, 0, s);
    if (r != PXB_OK) return r;
    const size_t es = E->esize();
    for (const EnsMember& mb : E->m) {
        const void* src[5] = {mb.b.h, mb.b.hu, mb.b.hv, mb.b.z_b, mb.b.G};
        void* dst[5] = {mb.a.h, mb.a.hu, mb.a.hv, mb.a.z_b, mb.a.G};
        for (int k = 0; k < 5; ++k)
            PXB_CUDA(cudaMemcpy2DAsync(dst[k], mb.pitch * es, src[k], mb.pitch * es, mb.nx * es, mb.ny,
                                       cudaMemcpyDeviceToDevice, s));
    }
    return PXB_OK;
}

// Candidate band heights timed on stage 1 (a -> b) of the current states; keeps the fastest.
template <class T>
int ens_autotune_impl(pxb_re_ens* E, cudaStream_t s, int32_t* out) {
    static const int cand[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 160, 192, 256};
    int st = ens_build_cfl_tables<T>(E, 0.5, nullptr);
    if (st != PXB_OK) return st;
    st = ens_cfl_launch<T>(E, 0, s);  // a dt to run the stage with (the states are not touched)
    if (st != PXB_OK) return st;
    cudaEvent_t e0, e1;
    PXB_CUDA(cudaEventCreate(&e0));
    PXB_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    int best = E->band_rows;
    for (int rows : cand) {
        E->band_rows = rows;
        st = ens_build_stage_tables<T>(E);
        if (st == PXB_OK) st = ens_stage_launch<T>(E, 0, s);  // warm-up
        float ms = 1e30f;
        for (int rep = 0; rep < 3 && st == PXB_OK; ++rep) {
            cudaEventRecord(e0, s);
            st = ens_stage_launch<T>(E, 0, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        if (st != PXB_OK) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = rows;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != PXB_OK) return st;
    E->band_rows = best;
    st = ens_build_stage_tables<T>(E);
    if (st != PXB_OK) return st;
    PXB_CUDA(cudaMemset2DAsync(&E->scr[0].step, sizeof(pxb::CflScratch), 0, sizeof(unsigned int), E->nm, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    if (out) *out = best;
    return PXB_OK;
}

// ------------------------------------------------------------------ tangent-linear model
// Dual planes: state A (h, hu, hv, z, z_b, n, n_b, G), state B (same layout; its z and
// n_b are A's) and the 7 scratch planes of the general path, plus one dual dt.
int jvp_buffers(pxb_re_plan* P) {
    if (P->jvp) return PXB_OK;
    const size_t plane = (size_t)P->c.ny * (size_t)P->c.pitch;
    PXB_CUDA(cudaMalloc(&P->jvp, sizeof(pxb::Dual) * (plane * 23 + 1)));
    PXB_CUDA(cudaMalloc(&P->dscr, sizeof(pxb::DualScratch)));
    PXB_CUDA(cudaMemset(P->dscr, 0, sizeof(pxb::DualScratch)));
    int maxcount = 1;
    for (auto& h : P->c.handlers) maxcount = std::max(maxcount, h.count);
    PXB_CUDA(cudaMalloc(&P->jvp_tmp, sizeof(pxb::Dual) * 6 * (size_t)maxcount));
    return PXB_OK;
}

pxb_re_fields dual_state(pxb_re_plan* P, int which) {
    const size_t plane = (size_t)P->c.ny * (size_t)P->c.pitch;
    pxb::Dual* b = (pxb::Dual*)P->jvp + (size_t)which * 8 * plane;
    pxb_re_fields f{};
    f.h = b;
    f.hu = b + plane;
    f.hv = b + 2 * plane;
    f.z = b + 3 * plane;
    f.z_b = b + 4 * plane;
    f.n = b + 5 * plane;
    f.n_b = b + 6 * plane;
    f.G = b + 7 * plane;
    return f;
}

void field_slots(const pxb_re_fields* f, void* out[8]) {
    out[0] = f->h;
    out[1] = f->hu;
    out[2] = f->hv;
    out[3] = f->z;
    out[4] = f->z_b;
    out[5] = f->n;
    out[6] = f->n_b;
    out[7] = f->G;
}

int jvp_pack(pxb_re_plan* P, const pxb_re_fields* v, const pxb_re_fields* t, const pxb_re_fields* D, cudaStream_t s) {
    void *vs[8], *ts[8], *ds[8];
    field_slots(v, vs);
    field_slots(t, ts);
    field_slots(D, ds);
    for (int k = 0; k < 8; ++k)
        PXB_CUDA(pxb::launch_dual_pack(P->c.ny, P->c.nx, P->c.pitch, (const double*)vs[k], (const double*)ts[k],
                                       (pxb::Dual*)ds[k], s));
    return PXB_OK;
}

int jvp_unpack(pxb_re_plan* P, const pxb_re_fields* D, const pxb_re_fields* v, const pxb_re_fields* t, cudaStream_t s) {
    void *vs[8], *ts[8], *ds[8];
    field_slots(v, vs);
    field_slots(t, ts);
    field_slots(D, ds);
    for (int k = 0; k < 8; ++k)
        PXB_CUDA(pxb::launch_dual_unpack(P->c.ny, P->c.nx, P->c.pitch, (const pxb::Dual*)ds[k], (double*)vs[k],
                                         (double*)ts[k], s));
    return PXB_OK;
}

int check_tangent_fields(const pxb_re_fields* f, const char* what) {
    if (!f || !f->h || !f->hu || !f->hv || !f->z || !f->z_b || !f->n || !f->n_b || !f->G)
        return fail(PXB_ERR_ARG, std::string(what) + ": every plane (h, hu, hv, z, z_b, n, n_b, G) must be set");
    return PXB_OK;
}

// Tangents of the run's parameters: the sediment matrix (MPM constants) and the discharge
// of ConstantInflux handlers (hu = q * values[1], hv = q * values[2]).
void jvp_params(pxb_re_plan* P, const pxb_re_tangent_params* tp) {
    if (P->mpm) fill_sed_dual(P->sedD, P->seds.data(), tp ? tp->seds_dot : nullptr, P->nsed);
    for (size_t k = 0; k < P->c.handlers.size(); ++k) {
        DevHandler& h = P->c.handlers[k];
        const double qd = (tp && tp->values0_dot && h.kind == PXB_BC_RE_CONSTANTINFLUX) ? tp->values0_dot[k] : 0.0;
        h.c0_dot = qd * h.vx;
        h.c1_dot = qd * h.vy;
    }
}

int jvp_init_impl(pxb_re_plan* P, const pxb_re_fields* f, const pxb_re_fields* fd, cudaStream_t s) {
    int st = jvp_buffers(P);
    if (st != PXB_OK) return st;
    const pxb_re_fields DA = dual_state(P, 0);
    st = jvp_pack(P, f, fd, &DA, s);
    if (st == PXB_OK)
        st = init_fields<pxb::Dual>(P->c.ny, P->c.nx, P->c.pitch, &DA, P->nodata, P->mpm, P->sedD, P->c.handlers,
                                    P->jvp_tmp, s);
    if (st == PXB_OK) st = jvp_unpack(P, &DA, f, fd, s);
    return st;
}

int jvp_run_impl(pxb_re_plan* P, const pxb_re_fields* a, const pxb_re_fields* ad, int nsteps, int scheme, double cfl,
                 double t0, double* dt_log, double* dt_dot_log, cudaStream_t s) {
    int st = jvp_buffers(P);
    if (st != PXB_OK) return st;
    const size_t plane = (size_t)P->c.ny * (size_t)P->c.pitch;
    pxb_re_fields DA = dual_state(P, 0), DB = dual_state(P, 1);
    DB.z = DA.z;
    DB.n_b = DA.n_b;
    void* gscr = (pxb::Dual*)P->jvp + 16 * plane;
    pxb::Dual* dtd = (pxb::Dual*)P->jvp + 23 * plane;
    st = jvp_pack(P, a, ad, &DA, s);
    if (st != PXB_OK) return st;
    pxb::DualScratch init{};
    init.t_step = t0;
    init.t_next = t0;
    PXB_CUDA(cudaMemcpyAsync(P->dscr, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    PXB_CUDA(cudaStreamSynchronize(s));  // `init` lives on this stack frame
    const double* tdev = &P->dscr->t_step;
    pxb_re_fields* cur = &DA;
    pxb_re_fields* nxt = &DB;
    for (int k = 0; k < nsteps && st == PXB_OK; ++k) {
        pxb::DualCflArgs c{};
        c.ny = P->c.ny;
        c.nx = P->c.nx;
        c.pitch = P->c.pitch;
        c.h = (const pxb::Dual*)cur->h;
        c.hu = (const pxb::Dual*)cur->hu;
        c.hv = (const pxb::Dual*)cur->hv;
        c.G = (const pxb::Dual*)cur->G;
        c.nodata = P->nodata;
        c.dx = P->c.dx;
        c.cfl = cfl;
        c.floor_dt = pxb::DT_FLOOR;
        c.scr = P->dscr;
        c.dt_out = dtd;
        c.dt_log = dt_log;
        c.dt_dot_log = dt_dot_log;
        c.err = &P->c.scr->err;
        PXB_CUDA(pxb::launch_dual_cfl(c, s));
        if (scheme == PXB_SSPRK2) {
            st = re_general_impl<pxb::Dual>(P, cur, nxt, nullptr, dtd, tdev, 0.0, s, gscr, P->jvp_tmp);
            if (st == PXB_OK) st = re_general_impl<pxb::Dual>(P, nxt, cur, cur, dtd, tdev, 0.0, s, gscr, P->jvp_tmp);
        } else {
            st = re_general_impl<pxb::Dual>(P, cur, nxt, nullptr, dtd, tdev, 0.0, s, gscr, P->jvp_tmp);
            std::swap(cur, nxt);
        }
    }
    if (st != PXB_OK) return st;
    return jvp_unpack(P, cur, a, ad, s);
}

// ------------------------------------------------------------------ reverse mode
// State planes carried by the adjoint: h, hu, hv, z_b, G (z, n_b static; n has no effect).
struct Planes5 {
    double* p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

Planes5 planes_of(double* base, size_t plane, int k) {
    Planes5 q;
    for (int f = 0; f < 5; ++f) q.p[f] = base + ((size_t)k * 5 + f) * plane;
    return q;
}

pxb_re_fields fields_of(const Planes5& q, const pxb_re_fields* statics) {
    pxb_re_fields f{};
    f.h = q.p[0];
    f.hu = q.p[1];
    f.hv = q.p[2];
    f.z_b = q.p[3];
    f.G = q.p[4];
    f.z = statics->z;
    f.n_b = statics->n_b;
    f.n = nullptr;
    return f;
}

int copy5(PlanCommon& C, const Planes5& dst, const Planes5& src, cudaStream_t s) {
    for (int f = 0; f < 5; ++f)
        PXB_CUDA(cudaMemcpyAsync(dst.p[f], src.p[f], sizeof(double) * (size_t)C.ny * C.pitch, cudaMemcpyDeviceToDevice, s));
    return PXB_OK;
}

int zero5(PlanCommon& C, const Planes5& q, cudaStream_t s) {
    for (int f = 0; f < 5; ++f) PXB_CUDA(cudaMemsetAsync(q.p[f], 0, sizeof(double) * (size_t)C.ny * C.pitch, s));
    return PXB_OK;
}

// Handlers backwards (last to first) on adjoint planes (slots h, hu, hv, z_b, -, G);
// qbar (device, one per handler, or null) accumulates the adjoints of the ConstantInflux
// discharges values[0].
int adj_handlers(PlanCommon& C, double* const f[6], double* tmp, cudaStream_t s, double* qbar = nullptr) {
    for (size_t q = C.handlers.size(); q-- > 0;) {
        const DevHandler& h = C.handlers[q];
        pxb::AdjBcArgs b{};
        b.vx = h.vx;
        b.vy = h.vy;
        b.qbar = qbar ? qbar + q : nullptr;
        for (int k = 0; k < 6; ++k) b.f[k] = f[k];
        b.cells = h.cells;
        b.donors = h.donors;
        b.count = h.count;
        b.kind = h.kind;
        b.nx = h.nx;
        b.ny = h.ny;
        b.c0 = h.c0;
        b.c1 = h.c1;
        b.tmp = tmp;
        PXB_CUDA(pxb::launch_adj_bc(b, s));
    }
    return PXB_OK;
}

struct AdjWork {
    double* base = nullptr;  // all planes
    size_t plane = 0;
    int nck = 0, K = 0;
    Planes5 u1, aS, aT, aCur, aNext, aU1;
    double* h1 = nullptr;
    double* gscr = nullptr;  // 7 planes for the general stage
    double* dev = nullptr;   // dt, dtbar, times (checkpoints then segment)
    unsigned long long* maxbits = nullptr;
    unsigned int* nties = nullptr;
    double* bctmp = nullptr;
    // parameter adjoints (null: not requested): per handler the ConstantInflux discharge,
    // then the MPM table of the sediment class; the n_b adjoint plane
    double* qbar = nullptr;
    double* tbar = nullptr;
    double* nbbar = nullptr;
    Planes5 ck(int k) const { return planes_of(base, plane, k); }                  // checkpoint k
    Planes5 seg(int k) const { return planes_of(base, plane, nck + k); }           // segment state k
    void release() {
        cudaFree(base);
        cudaFree(dev);
        cudaFree(maxbits);
        cudaFree(bctmp);
        base = dev = nullptr;
        maxbits = nullptr;
        bctmp = nullptr;
    }
};

// The stage input's adjoint += the reverse of one stage, given the adjoint of its output in
// W.aS (overwritten).  The stage internals are recomputed from the input first.
int adj_stage(pxb_re_plan* P, AdjWork& W, const pxb_re_fields* in, const Planes5& aIn, const double* dt,
              const double* tptr, cudaStream_t s) {
    const size_t plane = W.plane;
    double* S = W.gscr;
    // forward recompute: hydro, corrections, handlers 1, grass (as re_general_impl)
    pxb::GenArgs<double> g{};
    g.ny = P->c.ny;
    g.nx = P->c.nx;
    g.pitch = P->c.pitch;
    g.dx = P->c.dx;
    g.h = (const double*)in->h;
    g.hu = (const double*)in->hu;
    g.hv = (const double*)in->hv;
    g.zb = (const double*)in->z_b;
    g.z = (const double*)in->z;
    g.nb = (const double*)in->n_b;
    g.G = (const double*)in->G;
    g.n = nullptr;
    g.sh = S;
    g.shu = S + plane;
    g.shv = S + 2 * plane;
    g.szb = S + 3 * plane;
    g.sG = S + 4 * plane;
    g.sn = S + 5 * plane;
    g.szb2 = S + 6 * plane;
    g.nodata = P->nodata;
    g.dt = dt;
    g.sed = P->sedd;
    g.mpm = P->mpm;
    g.err = &P->c.scr->err;
    PXB_CUDA(pxb::launch_re_general<double>(g, pxb::GEN_HYDRO, s));
    PXB_CUDA(pxb::launch_re_general<double>(g, pxb::GEN_CORR, s));
    PXB_CUDA(cudaMemcpyAsync(W.h1, g.sh, sizeof(double) * plane, cudaMemcpyDeviceToDevice, s));
    double* const f1[6] = {g.sh, g.shu, g.shv, g.szb, g.sn, g.sG};
    int st = apply_handlers<double>(P->c.handlers, P->c.bc_tmp, f1, tptr, 0.0, s);
    if (st != PXB_OK) return st;
    PXB_CUDA(pxb::launch_re_general<double>(g, pxb::GEN_GRASS, s));
    // backwards
    pxb::AdjArgs a{};
    a.ny = P->c.ny;
    a.nx = P->c.nx;
    a.pitch = P->c.pitch;
    a.dx = P->c.dx;
    a.h = g.h;
    a.hu = g.hu;
    a.hv = g.hv;
    a.zb = g.zb;
    a.z = g.z;
    a.nb = g.nb;
    a.G = g.G;
    a.h1 = W.h1;
    a.sh = g.sh;
    a.shu = g.shu;
    a.shv = g.shv;
    a.szb = g.szb;
    a.sG = g.sG;
    a.nodata = P->nodata;
    a.dt = dt;
    a.sed = P->sedd;
    a.mpm = P->mpm;
    a.Sh = W.aS.p[0];
    a.Shu = W.aS.p[1];
    a.Shv = W.aS.p[2];
    a.Szb = W.aS.p[3];
    a.SG = W.aS.p[4];
    a.Th = W.aT.p[0];
    a.Thu = W.aT.p[1];
    a.Thv = W.aT.p[2];
    a.Tzb = W.aT.p[3];
    a.TG = W.aT.p[4];
    a.Ih = aIn.p[0];
    a.Ihu = aIn.p[1];
    a.Ihv = aIn.p[2];
    a.Izb = aIn.p[3];
    a.IG = aIn.p[4];
    a.dtbar = W.dev + 1;
    a.nbbar = W.nbbar;
    a.tbar = W.tbar;
    double* const fS[6] = {W.aS.p[0], W.aS.p[1], W.aS.p[2], W.aS.p[3], nullptr, W.aS.p[4]};
    st = adj_handlers(P->c, fS, W.bctmp, s, W.qbar);  // handlers 2
    if (st != PXB_OK) return st;
    PXB_CUDA(pxb::launch_adj_stage(a, 0, s));  // Exner
    PXB_CUDA(pxb::launch_adj_stage(a, 1, s));  // grass
    double* const fT[6] = {W.aT.p[0], W.aT.p[1], W.aT.p[2], W.aT.p[3], nullptr, W.aT.p[4]};
    st = adj_handlers(P->c, fT, W.bctmp, s, W.qbar);  // handlers 1
    if (st != PXB_OK) return st;
    PXB_CUDA(pxb::launch_adj_stage(a, 2, s));  // corrections
    PXB_CUDA(pxb::launch_adj_stage(a, 3, s));  // hydro
    return PXB_OK;
}

// One forward stage on the general kernels (float64) into `out`.
int adj_fwd_stage(pxb_re_plan* P, AdjWork& W, const pxb_re_fields* in, const pxb_re_fields* out,
                  const pxb_re_fields* avg, const double* dt, const double* tptr, cudaStream_t s) {
    return re_general_impl<double>(P, in, out, avg, dt, tptr, 0.0, s, W.gscr, P->c.bc_tmp);
}

int adj_step_fwd(pxb_re_plan* P, AdjWork& W, const Planes5& u, const Planes5& next, int scheme,
                 const pxb_re_fields* statics, double cfl, cudaStream_t s) {
    double* dt = W.dev;
    const pxb_re_fields F = fields_of(u, statics), U1 = fields_of(W.u1, statics), N = fields_of(next, statics);
    int st = re_cfl_impl<double>(P, &F, cfl, dt, nullptr, s);
    if (st != PXB_OK) return st;
    const double* tptr = &P->c.scr->t_step;
    st = adj_fwd_stage(P, W, &F, &U1, nullptr, dt, tptr, s);
    if (st != PXB_OK) return st;
    if (scheme == PXB_SSPRK2) return adj_fwd_stage(P, W, &U1, &N, &F, dt, tptr, s);
    return copy5(P->c, next, W.u1, s);
}

// Device array of the parameter adjoints of one reverse-mode call: nh handler discharges,
// then the 7 MPM table entries of the sediment class and the adjoint of n_p_mix.
int param_adjoint_buffer(pxb_re_plan* P, const pxb_re_param_adjoints* pa, double** out) {
    *out = nullptr;
    if (!pa || (!pa->seds_bar && !pa->values0_bar)) return PXB_OK;
    if (pa->seds_bar && P->mpm && P->nsed != 1)
        return fail(PXB_ERR_UNSUPPORTED, "sediment-matrix adjoints are built for one sediment class");
    const size_t n = P->c.handlers.size() + 8;
    PXB_CUDA(cudaMalloc(out, sizeof(double) * n));
    PXB_CUDA(cudaMemset(*out, 0, sizeof(double) * n));
    return PXB_OK;
}

// The accumulated parameter adjoints into the caller's host arrays: discharges directly;
// the MPM table (and n_p_mix) to the sediment matrix through the derivatives of the
// table with respect to each matrix entry (fill_sed_dual, the tangent model's table).
int apply_param_adjoints(pxb_re_plan* P, const double* dev, const pxb_re_param_adjoints* pa, cudaStream_t s) {
    if (!dev) return PXB_OK;
    const size_t nh = P->c.handlers.size();
    std::vector<double> h(nh + 8);
    PXB_CUDA(cudaMemcpyAsync(h.data(), dev, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    if (pa->values0_bar)
        for (size_t k = 0; k < nh; ++k)
            if (P->c.handlers[k].kind == PXB_BC_RE_CONSTANTINFLUX) pa->values0_bar[k] += h[k];
    if (pa->seds_bar && P->mpm) {
        const double* tb = h.data() + nh;  // np2, sm1d, thc, np3sg, sm1, frac, 1 - porosity, n_p_mix
        const int ns = P->nsed;
        std::vector<double> unit(7 * (size_t)ns, 0.0);
        for (int e = 0; e < 7 * ns; ++e) {
            unit[e] = 1.0;
            pxb::SedTable<pxb::Dual> S;
            fill_sed_dual(S, P->seds.data(), unit.data(), ns);
            unit[e] = 0.0;
            const pxb::SedT<pxb::Dual>& c = S.s[0];
            pa->seds_bar[e] += tb[0] * c.np2.d + tb[1] * c.sm1d.d + tb[2] * c.thc.d + tb[3] * c.np3sg.d +
                               tb[4] * c.sm1.d + tb[5] * c.frac.d + tb[6] * S.one_minus_por.d + tb[7] * S.n_p_mix.d;
        }
    }
    return PXB_OK;
}

int vjp_run_impl(pxb_re_plan* P, const pxb_re_fields* a0, int nsteps, int scheme, double cfl, double t0, int every,
                 const pxb_re_fields* abar, const pxb_re_param_adjoints* pa, cudaStream_t s) {
    for (auto& h : P->c.handlers)
        if (h.kind == PXB_BC_RE_CONSTANTOUTFLUX)
            return fail(PXB_ERR_UNSUPPORTED, "the reverse mode does not cover ConstantOutflux handlers (nonlinear)");
    double* pdev = nullptr;
    {
        const int pst = param_adjoint_buffer(P, pa, &pdev);
        if (pst != PXB_OK) return pst;
    }
    AdjWork W;
    if (pdev) {
        W.qbar = pdev;
        if (pa->seds_bar && P->mpm) W.tbar = pdev + P->c.handlers.size();
        if (pa->seds_bar && abar->n_b) W.nbbar = (double*)abar->n_b;
    }
    W.K = every > 0 ? every : 32;
    W.nck = (nsteps + W.K - 1) / W.K;
    W.plane = (size_t)P->c.ny * (size_t)P->c.pitch;
    // checkpoints, segment states (K + 1), u1, aS, aT, aCur, aNext, aU1 (5 planes each), h1, 7 scratch
    const size_t nplanes = (size_t)5 * (W.nck + W.K + 1 + 6) + 1 + 7;
    int maxcount = 1;
    for (auto& h : P->c.handlers) maxcount = std::max(maxcount, h.count);
    auto bail = [&](int code) {
        cudaStreamSynchronize(s);
        W.release();
        cudaFree(pdev);
        return code;
    };
    if (cudaMalloc(&W.base, sizeof(double) * nplanes * W.plane) != cudaSuccess ||
        cudaMalloc(&W.dev, sizeof(double) * (2 + W.nck + W.K)) != cudaSuccess ||
        cudaMalloc(&W.maxbits, 16) != cudaSuccess ||
        cudaMalloc(&W.bctmp, sizeof(double) * 6 * (size_t)maxcount) != cudaSuccess)
        return bail(fail(PXB_ERR_CUDA, "reverse-mode buffers"));
    W.nties = (unsigned int*)(W.maxbits + 1);
    const int o = W.nck + W.K + 1;
    W.u1 = planes_of(W.base, W.plane, o);
    W.aS = planes_of(W.base, W.plane, o + 1);
    W.aT = planes_of(W.base, W.plane, o + 2);
    W.aCur = planes_of(W.base, W.plane, o + 3);
    W.aNext = planes_of(W.base, W.plane, o + 4);
    W.aU1 = planes_of(W.base, W.plane, o + 5);
    W.h1 = W.base + (size_t)5 * (o + 6) * W.plane;
    W.gscr = W.h1 + W.plane;
    double* tck = W.dev + 2;
    double* tseg = tck + W.nck;
    Planes5 A0;
    A0.p[0] = (double*)a0->h;
    A0.p[1] = (double*)a0->hu;
    A0.p[2] = (double*)a0->hv;
    A0.p[3] = (double*)a0->z_b;
    A0.p[4] = (double*)a0->G;
    int st = PXB_OK;
    auto chk = [&](int r) {
        if (st == PXB_OK) st = r;
        return st == PXB_OK;
    };
    // forward sweep with checkpoints
    chk(copy5(P->c, W.ck(0), A0, s));
    if (st == PXB_OK && pxb::launch_set_time<double>(P->c.scr, t0, s) != cudaSuccess) st = fail(PXB_ERR_CUDA, "time");
    for (int n = 0; n < nsteps && st == PXB_OK; ++n) {
        const int k = n / W.K;
        if (n % W.K == 0) {
            if (n > 0) chk(copy5(P->c, W.ck(k), W.seg(0), s));
            if (cudaMemcpyAsync(tck + k, &P->c.scr->t_next, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                st = fail(PXB_ERR_CUDA, "checkpoint time");
            if (n == 0) chk(copy5(P->c, W.seg(0), A0, s));
        }
        if (st == PXB_OK) chk(adj_step_fwd(P, W, W.seg(0), W.seg(0), scheme, a0, cfl, s));
    }
    // backward sweep
    const pxb_re_fields* statics = a0;
    Planes5 AB;
    AB.p[0] = (double*)abar->h;
    AB.p[1] = (double*)abar->hu;
    AB.p[2] = (double*)abar->hv;
    AB.p[3] = (double*)abar->z_b;
    AB.p[4] = (double*)abar->G;
    if (st == PXB_OK) chk(copy5(P->c, W.aNext, AB, s));
    for (int k = W.nck - 1; k >= 0 && st == PXB_OK; --k) {
        const int n0 = k * W.K, n1 = std::min(nsteps, n0 + W.K);
        chk(copy5(P->c, W.seg(0), W.ck(k), s));
        if (st == PXB_OK && cudaMemcpyAsync(&P->c.scr->t_next, tck + k, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = fail(PXB_ERR_CUDA, "segment time");
        for (int j = 0; j < n1 - n0 - 1 && st == PXB_OK; ++j) {
            if (cudaMemcpyAsync(tseg + j, &P->c.scr->t_next, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                st = fail(PXB_ERR_CUDA, "step time");
            else chk(adj_step_fwd(P, W, W.seg(j), W.seg(j + 1), scheme, statics, cfl, s));
        }
        if (st == PXB_OK && n1 - n0 - 1 >= 0 &&
            cudaMemcpyAsync(tseg + (n1 - n0 - 1), &P->c.scr->t_next, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = fail(PXB_ERR_CUDA, "step time");
        for (int j = n1 - n0 - 1; j >= 0 && st == PXB_OK; --j) {
            const Planes5 u = W.seg(j);
            const pxb_re_fields F = fields_of(u, statics), U1 = fields_of(W.u1, statics);
            double* dt = W.dev;
            // the step's time and dt again (the CFL kernel moves t_next into t_step)
            if (cudaMemcpyAsync(&P->c.scr->t_next, tseg + j, 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                cudaMemsetAsync(W.dev + 1, 0, sizeof(double), s) != cudaSuccess) {
                st = fail(PXB_ERR_CUDA, "step state");
                break;
            }
            if (!chk(re_cfl_impl<double>(P, &F, cfl, dt, nullptr, s))) break;
            const double* tptr = &P->c.scr->t_step;
            if (!chk(zero5(P->c, W.aCur, s))) break;
            if (scheme == PXB_SSPRK2) {
                const double* o5[5] = {W.aNext.p[0], W.aNext.p[1], W.aNext.p[2], W.aNext.p[3], W.aNext.p[4]};
                if (!chk(adj_fwd_stage(P, W, &F, &U1, nullptr, dt, tptr, s))) break;
                if (pxb::launch_adj_store(P->c.ny, P->c.nx, P->c.pitch, 0.5, o5, W.aS.p, W.aCur.p, s) != cudaSuccess) {
                    st = fail(PXB_ERR_CUDA, "adjoint store");
                    break;
                }
                if (!chk(zero5(P->c, W.aU1, s))) break;
                if (!chk(adj_stage(P, W, &U1, W.aU1, dt, tptr, s))) break;
                const double* o1[5] = {W.aU1.p[0], W.aU1.p[1], W.aU1.p[2], W.aU1.p[3], W.aU1.p[4]};
                if (pxb::launch_adj_store(P->c.ny, P->c.nx, P->c.pitch, 1.0, o1, W.aS.p, nullptr, s) != cudaSuccess) {
                    st = fail(PXB_ERR_CUDA, "adjoint store");
                    break;
                }
                if (!chk(adj_stage(P, W, &F, W.aCur, dt, tptr, s))) break;
            } else {
                const double* o5[5] = {W.aNext.p[0], W.aNext.p[1], W.aNext.p[2], W.aNext.p[3], W.aNext.p[4]};
                if (pxb::launch_adj_store(P->c.ny, P->c.nx, P->c.pitch, 1.0, o5, W.aS.p, nullptr, s) != cudaSuccess) {
                    st = fail(PXB_ERR_CUDA, "adjoint store");
                    break;
                }
                if (!chk(adj_stage(P, W, &F, W.aCur, dt, tptr, s))) break;
            }
            // dt depends on the step's input through the fastest face
            pxb::AdjCflArgs c{};
            c.ny = P->c.ny;
            c.nx = P->c.nx;
            c.pitch = P->c.pitch;
            c.h = (const double*)F.h;
            c.hu = (const double*)F.hu;
            c.hv = (const double*)F.hv;
            c.G = (const double*)F.G;
            c.nodata = P->nodata;
            c.dx = P->c.dx;
            c.cfl = cfl;
            c.floor_dt = pxb::DT_FLOOR;
            c.maxbits = W.maxbits;
            c.nties = W.nties;
            c.dtbar = W.dev + 1;
            c.Ah = W.aCur.p[0];
            c.Ahu = W.aCur.p[1];
            c.Ahv = W.aCur.p[2];
            c.AG = W.aCur.p[4];
            if (cudaMemsetAsync(W.maxbits, 0, 16, s) != cudaSuccess || pxb::launch_adj_cfl(c, s) != cudaSuccess) {
                st = fail(PXB_ERR_CUDA, "adjoint of dt");
                break;
            }
            std::swap(W.aCur, W.aNext);
        }
    }
    if (st == PXB_OK) chk(copy5(P->c, AB, W.aNext, s));
    if (st == PXB_OK) chk(apply_param_adjoints(P, pdev, pa, s));
    cudaStreamSynchronize(s);
    W.release();
    cudaFree(pdev);
    return st;
}

// init_fn_roeexner backwards: handlers (t = 0), then the grass factor from the raw state.
int vjp_init_impl(pxb_re_plan* P, const pxb_re_fields* f, const pxb_re_fields* fbar, const pxb_re_param_adjoints* pa,
                  cudaStream_t s) {
    for (auto& h : P->c.handlers)
        if (h.kind == PXB_BC_RE_CONSTANTOUTFLUX)
            return fail(PXB_ERR_UNSUPPORTED, "the reverse mode does not cover ConstantOutflux handlers (nonlinear)");
    double* pdev = nullptr;
    {
        const int pst = param_adjoint_buffer(P, pa, &pdev);
        if (pst != PXB_OK) return pst;
    }
    int maxcount = 1;
    for (auto& h : P->c.handlers) maxcount = std::max(maxcount, h.count);
    double* tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(double) * 6 * (size_t)maxcount) != cudaSuccess) {
        cudaFree(pdev);
        return fail(PXB_ERR_CUDA, "reverse-mode handler buffer");
    }
    double* const fb[6] = {(double*)fbar->h, (double*)fbar->hu, (double*)fbar->hv, (double*)fbar->z_b, nullptr,
                           (double*)fbar->G};
    int st = adj_handlers(P->c, fb, tmp, s, pdev);
    if (st == PXB_OK) {
        pxb::AdjArgs a{};
        a.ny = P->c.ny;
        a.nx = P->c.nx;
        a.pitch = P->c.pitch;
        a.dx = P->c.dx;
        a.sh = (const double*)f->h;
        a.shu = (const double*)f->hu;
        a.shv = (const double*)f->hv;
        a.nodata = P->nodata;
        a.sed = P->sedd;
        a.mpm = P->mpm;
        a.Th = fb[0];
        a.Thu = fb[1];
        a.Thv = fb[2];
        a.TG = fb[5];
        if (pdev && pa->seds_bar && P->mpm) a.tbar = pdev + P->c.handlers.size();
        if (pxb::launch_adj_stage(a, 1, s) != cudaSuccess) st = fail(PXB_ERR_CUDA, "adjoint of the grass factor");
    }
    // compute_n: the n_b adjoint to the raw n and to n_p_mix (the sediment matrix)
    if (st == PXB_OK && pdev && pa->seds_bar && fbar->n_b &&
        pxb::launch_adj_compute_n(P->c.ny, P->c.nx, P->c.pitch, P->mpm, (const double*)f->z_b, (double*)fbar->n_b,
                                  (double*)fbar->n, pdev + P->c.handlers.size() + 7, s) != cudaSuccess)
        st = fail(PXB_ERR_CUDA, "adjoint of compute_n");
    if (st == PXB_OK) st = apply_param_adjoints(P, pdev, pa, s);
    cudaStreamSynchronize(s);
    cudaFree(tmp);
    cudaFree(pdev);
    return st;
}

}  // namespace

// ===================================================================== C entry points
extern "C" {

const char* pxb_last_error(void) { return g_err.c_str(); }

int pxb_label_polygons(int32_t ny, int32_t nx, const double* xc, const double* yc, const double* verts,
                       int32_t npoly, int32_t nverts, int64_t* counts, int64_t* cells, int64_t cells_cap,
                       void* stream) {
    if (ny < 1 || nx < 1 || npoly < 1 || nverts < 1) return fail(PXB_ERR_ARG, "empty grid or polygon set");
    if (!xc || !yc || !verts || !counts) return fail(PXB_ERR_ARG, "null coordinate, vertex or count array");
    if ((long long)npoly * ny * nx >= (1LL << 40)) return fail(PXB_ERR_ARG, "label planes too large");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t rows = (size_t)npoly * ny;
    double *dx = nullptr, *dy = nullptr, *dv = nullptr;
    uint8_t* lab = nullptr;
    long long *cnt = nullptr, *off = nullptr, *dcells = nullptr;
    std::vector<long long> hc(rows), ho(rows);
    int code = PXB_OK;
    std::string msg;
    auto ok = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && code == PXB_OK) {
            code = PXB_ERR_CUDA;
            msg = std::string(what) + ": " + cudaGetErrorString(e);
        }
        return code == PXB_OK;
    };
    if (ok(cudaMalloc(&dx, sizeof(double) * nx), "coordinates") && ok(cudaMalloc(&dy, sizeof(double) * ny), "coordinates") &&
        ok(cudaMalloc(&dv, sizeof(double) * 2 * (size_t)npoly * nverts), "vertices") &&
        ok(cudaMalloc(&lab, rows * (size_t)nx), "labels") && ok(cudaMalloc(&cnt, sizeof(long long) * rows), "counts") &&
        ok(cudaMemcpyAsync(dx, xc, sizeof(double) * nx, cudaMemcpyHostToDevice, s), "copy") &&
        ok(cudaMemcpyAsync(dy, yc, sizeof(double) * ny, cudaMemcpyHostToDevice, s), "copy") &&
        ok(cudaMemcpyAsync(dv, verts, sizeof(double) * 2 * (size_t)npoly * nverts, cudaMemcpyHostToDevice, s), "copy") &&
        ok(pxb::launch_label(ny, nx, dx, dy, dv, npoly, nverts, lab, s), "label kernel") &&
        ok(pxb::launch_label_count(ny, nx, npoly, lab, cnt, s), "count kernel") &&
        ok(cudaMemcpyAsync(hc.data(), cnt, sizeof(long long) * rows, cudaMemcpyDeviceToHost, s), "copy") &&
        ok(cudaStreamSynchronize(s), "synchronise")) {
        long long total = 0;
        for (int p = 0; p < npoly; ++p) {
            long long n = 0;
            for (int r = 0; r < ny; ++r) {
                ho[(size_t)p * ny + r] = total + n;
                n += hc[(size_t)p * ny + r];
            }
            counts[p] = n;
            total += n;
        }
        if (cells) {
            if (total > cells_cap) {
                code = PXB_ERR_ARG;
                msg = "cells capacity " + std::to_string(cells_cap) + " < " + std::to_string(total) + " labelled cells";
            } else if (total > 0 &&
                       ok(cudaMalloc(&off, sizeof(long long) * rows), "offsets") &&
                       ok(cudaMalloc(&dcells, sizeof(long long) * (size_t)total), "cells") &&
                       ok(cudaMemcpyAsync(off, ho.data(), sizeof(long long) * rows, cudaMemcpyHostToDevice, s), "copy") &&
                       ok(pxb::launch_label_fill(ny, nx, npoly, lab, off, dcells, s), "fill kernel") &&
                       ok(cudaMemcpyAsync(cells, dcells, sizeof(long long) * (size_t)total, cudaMemcpyDeviceToHost, s),
                          "copy")) {
                ok(cudaStreamSynchronize(s), "synchronise");
            }
        }
    }
    cudaStreamSynchronize(s);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dv);
    cudaFree(lab);
    cudaFree(cnt);
    cudaFree(off);
    cudaFree(dcells);
    return code == PXB_OK ? PXB_OK : fail(code, msg);
}
int pxb_version(void) { return 1; }

namespace {
// Roe-Exner plan on cudaMalloc'd memory (A null), on the caller's workspace, or only
// counting the workspace's size (A->counting; the plan is then discarded).
int re_plan_create(const pxb_re_config* cfg, DevArena* A, pxb_re_plan** out) {
    if (!cfg || !out) return fail(PXB_ERR_ARG, "null config or output pointer");
    *out = nullptr;
    if (cfg->mpm && (!cfg->seds || cfg->nsed < 1 || cfg->nsed > PXB_MAX_SED))
        return fail(PXB_ERR_ARG, "MPM needs 1..8 sediment classes");
    pxb_re_plan* P = new pxb_re_plan();
    int st = common_setup(P->c, cfg->ny, cfg->nx, cfg->pitch, cfg->dtype, cfg->dx, cfg->handlers, cfg->nhandlers, false,
                          cfg->stage_path, P->path, A);
    if (st == PXB_OK && P->path == PXB_PATH_GENERAL)
        st = arena_alloc(A, &P->gen, 7 * (size_t)cfg->ny * (size_t)cfg->pitch * P->c.esize(), "scratch planes");
    if (st == PXB_OK && A)  // the volume reduction's block partials (allocated on first use otherwise)
        st = arena_alloc(A, (void**)&P->vol_scr, sizeof(double) * (4 * (size_t)(4 * P->c.sm_count) + 2),
                         "volume scratch");
    if (st != PXB_OK || (A && A->counting)) {
        if (!P->c.ws) cudaFree(P->gen);
        P->c.release();
        delete P;
        return st;
    }
    P->mpm = cfg->mpm;
    P->nodata = cfg->nodata;
    P->want_rows = cfg->band_rows;
    if (cfg->mpm) {
        fill_sed(P->sedf, cfg->seds, cfg->nsed);
        fill_sed(P->sedd, cfg->seds, cfg->nsed);
        P->seds.assign(cfg->seds, cfg->seds + 7 * cfg->nsed);
        P->nsed = cfg->nsed;
        fill_sed_dual(P->sedD, P->seds.data(), nullptr, P->nsed);
    }
    const bool f64 = cfg->dtype == PXB_F64;
    for (int v = 0; v < 8; ++v) {
        const bool mpm = v & 4, hm = v & 2, avg = v & 1;
        const int bps = f64 ? pxb::re_stage_blocks_per_sm<double>(mpm, hm, avg)
                            : pxb::re_stage_blocks_per_sm<float>(mpm, hm, avg);
        P->stage[v] = stage_geometry(cfg->ny, cfg->nx, f64 ? 8 : 4, std::max(1, bps) * 4 * P->c.sm_count, cfg->band_rows);
    }
    const int cb = f64 ? pxb::re_cfl_blocks_per_sm<double>(cfg->nodata != nullptr)
                       : pxb::re_cfl_blocks_per_sm<float>(cfg->nodata != nullptr);
    P->c.cfl = cfl_geometry(cfg->ny, cfg->nx, std::max(1, cb) * 8 * P->c.sm_count);
    *out = P;
    return PXB_OK;
}

// Entry points that allocate device tables on first use refuse a workspace plan.
int refuse_ws(const pxb_re_plan* P, const char* what) {
    if (P && P->c.ws)
        return fail(PXB_ERR_UNSUPPORTED, std::string(what) + " allocates device memory: not on a workspace plan");
    return PXB_OK;
}
}  // namespace

int pxb_re_plan_create(const pxb_re_config* cfg, pxb_re_plan** out) { return re_plan_create(cfg, nullptr, out); }

int pxb_re_plan_workspace_size(const pxb_re_config* cfg, size_t* bytes) {
    if (!bytes) return fail(PXB_ERR_ARG, "null output pointer");
    *bytes = 0;
    DevArena A;
    A.counting = true;
    pxb_re_plan* P = nullptr;
    const int st = re_plan_create(cfg, &A, &P);
    if (st != PXB_OK) return st;
    *bytes = A.used;
    return PXB_OK;
}

int pxb_re_plan_create_in(const pxb_re_config* cfg, void* workspace, size_t bytes, pxb_re_plan** out) {
    if (!workspace || ((uintptr_t)workspace & 255u)) return fail(PXB_ERR_ARG, "workspace must be 256-byte aligned");
    DevArena A;
    A.base = (char*)workspace;
    A.cap = bytes;
    return re_plan_create(cfg, &A, out);
}

int pxb_re_plan_destroy(pxb_re_plan* plan) {
    if (!plan) return PXB_OK;
    cudaDeviceSynchronize();
    plan->c.release();
    if (!plan->c.ws) {
        cudaFree(plan->gen);
        cudaFree(plan->vol_scr);
    }
    cudaFree(plan->jvp);
    cudaFree(plan->dscr);
    cudaFree(plan->jvp_tmp);
    cudaFree(plan->bud_part);
    delete plan;
    return PXB_OK;
}

int pxb_re_plan_path(const pxb_re_plan* plan) { return plan ? plan->path : 0; }

int pxb_re_autotune(pxb_re_plan* P, const pxb_re_fields* a, const pxb_re_fields* b, void* stream, int32_t* band_rows) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_fields(a, true);
    if (st) return st;
    st = check_fields(b, true);
    if (st) return st;
    if (!a->z || !a->n_b) return fail(PXB_ERR_ARG, "z and n_b must be set");
    if (a->h == b->h || a->z_b == b->z_b) return fail(PXB_ERR_ARG, "b must not alias a");
    if (P->path != PXB_PATH_FUSED) {  // the general path has no band geometry
        if (band_rows) *band_rows = 0;
        return PXB_OK;
    }
    cudaStream_t s = (cudaStream_t)stream;
    return P->c.dtype == PXB_F64 ? re_autotune_impl<double>(P, a, b, s, band_rows)
                                 : re_autotune_impl<float>(P, a, b, s, band_rows);
}

int pxb_re_init(pxb_re_plan* P, const pxb_re_fields* f, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_fields(f, true);
    if (st) return st;
    if (!f->n || !f->n_b) return fail(PXB_ERR_ARG, "n and n_b must be set");
    cudaStream_t s = (cudaStream_t)stream;
    return P->c.dtype == PXB_F64 ? re_init_impl<double>(P, f, s) : re_init_impl<float>(P, f, s);
}

int pxb_re_cfl(pxb_re_plan* P, const pxb_re_fields* f, double cfl, void* dt_dev, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_fields(f, true);
    if (st) return st;
    if (!dt_dev) return fail(PXB_ERR_ARG, "dt_dev is null");
    cudaStream_t s = (cudaStream_t)stream;
    return P->c.dtype == PXB_F64 ? re_cfl_impl<double>(P, f, cfl, dt_dev, nullptr, s)
                                 : re_cfl_impl<float>(P, f, cfl, dt_dev, nullptr, s);
}

int pxb_re_stage(pxb_re_plan* P, const pxb_re_fields* in, const pxb_re_fields* out, const pxb_re_fields* avg,
                 const void* dt_dev, double time, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_fields(in, !P->mpm);
    if (st) return st;
    st = check_fields(out, !P->mpm);
    if (st) return st;
    if (!in->z || !in->n_b) return fail(PXB_ERR_ARG, "input z and n_b must be set");
    if (avg && (st = check_fields(avg, out->G != nullptr))) return st;
    if (!dt_dev) return fail(PXB_ERR_ARG, "dt_dev is null");
    if (in->h == out->h || in->hu == out->hu || in->hv == out->hv || in->z_b == out->z_b)
        return fail(PXB_ERR_ARG, "stage output must not alias its input");
    if (P->path == PXB_PATH_GENERAL && in->n && out->n == in->n)
        return fail(PXB_ERR_ARG, "stage output n must not alias its input on the general path");
    return re_stage_any(P, in, out, avg, dt_dev, nullptr, time, (cudaStream_t)stream);
}

int pxb_re_run(pxb_re_plan* P, const pxb_re_fields* a, const pxb_re_fields* b, int32_t nsteps, int32_t scheme,
               double cfl, double t0, void* dt_log, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_fields(a, true);
    if (st) return st;
    st = check_fields(b, true);
    if (st) return st;
    if (!a->z || !a->n_b) return fail(PXB_ERR_ARG, "z and n_b must be set");
    if (nsteps < 0) return fail(PXB_ERR_ARG, "nsteps < 0");
    if (scheme != PXB_FE && scheme != PXB_SSPRK2) return fail(PXB_ERR_ARG, "scheme must be PXB_FE or PXB_SSPRK2");
    if (nsteps == 0) return PXB_OK;
    return re_steps(P, a, b, nsteps, scheme, cfl, t0, dt_log, (cudaStream_t)stream);
}

int pxb_re_set_budget(pxb_re_plan* P, double* acc_dev) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (acc_dev && !P->bud_part) {
        const int st = refuse_ws(P, "the volume budget");
        if (st != PXB_OK) return st;
    }
    if (acc_dev && P->path != PXB_PATH_FUSED)
        return fail(PXB_ERR_UNSUPPORTED, "the volume budget is built into the fused stage path only");
    if (acc_dev && ((uintptr_t)acc_dev & 7u)) return fail(PXB_ERR_ARG, "acc_dev must be 8-byte aligned");
    if (acc_dev && !P->bud_part) {
        // every band geometry the plan can take: bands of one row at least
        const int nstrips = std::max(1, (P->c.nx - 3 + pxb_stage_strip_out((int)P->c.esize()) - 1) /
                                            pxb_stage_strip_out((int)P->c.esize()));
        const long long items = (long long)pxb_stage_items_per_band(nstrips) * P->c.ny;
        PXB_CUDA(cudaMalloc(&P->bud_part, sizeof(double) * 2 * (size_t)items));
        P->bud_items = items;
    }
    P->bud_acc = (pxb::BudgetAcc*)acc_dev;
    return PXB_OK;
}

int pxb_re_volume(pxb_re_plan* P, const pxb_re_fields* f, double* volumes, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (!f || !f->h || !f->z_b) return fail(PXB_ERR_ARG, "h and z_b must be set");
    if (!volumes) return fail(PXB_ERR_ARG, "volumes is null");
    const int nblocks = std::max(1, std::min(P->c.ny - 2, 4 * P->c.sm_count));
    if (!P->vol_scr) PXB_CUDA(cudaMalloc(&P->vol_scr, sizeof(double) * (4 * (size_t)(4 * P->c.sm_count) + 2)));
    cudaStream_t s = (cudaStream_t)stream;
    double* out = P->vol_scr + 4 * (size_t)(4 * P->c.sm_count);
    const double dx2 = P->c.dx * P->c.dx;
    if (P->c.dtype == PXB_F64)
        PXB_CUDA(pxb::launch_volume<double>(P->c.ny, P->c.nx, P->c.pitch, (const double*)f->h, (const double*)f->z_b,
                                            P->nodata, P->vol_scr, nblocks, dx2, out, s));
    else
        PXB_CUDA(pxb::launch_volume<float>(P->c.ny, P->c.nx, P->c.pitch, (const float*)f->h, (const float*)f->z_b,
                                           P->nodata, P->vol_scr, nblocks, dx2, out, s));
    PXB_CUDA(cudaMemcpyAsync(volumes, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    return PXB_OK;
}

int pxb_re_jvp_init(pxb_re_plan* P, const pxb_re_fields* f, const pxb_re_fields* f_dot,
                    const pxb_re_tangent_params* tp, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (refuse_ws(P, "the tangent-linear model") != PXB_OK) return PXB_ERR_UNSUPPORTED;
    if (P->c.dtype != PXB_F64) return fail(PXB_ERR_ARG, "the tangent-linear model runs on float64 plans");
    int st = check_tangent_fields(f, "state");
    if (st == PXB_OK) st = check_tangent_fields(f_dot, "tangent");
    if (st != PXB_OK) return st;
    jvp_params(P, tp);
    st = jvp_init_impl(P, f, f_dot, (cudaStream_t)stream);
    jvp_params(P, nullptr);
    return st;
}

int pxb_re_jvp_run(pxb_re_plan* P, const pxb_re_fields* a, const pxb_re_fields* a_dot, int32_t nsteps, int32_t scheme,
                   double cfl, double t0, const pxb_re_tangent_params* tp, void* dt_log, void* dt_dot_log,
                   void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (refuse_ws(P, "the tangent-linear model") != PXB_OK) return PXB_ERR_UNSUPPORTED;
    if (P->c.dtype != PXB_F64) return fail(PXB_ERR_ARG, "the tangent-linear model runs on float64 plans");
    int st = check_tangent_fields(a, "state");
    if (st == PXB_OK) st = check_tangent_fields(a_dot, "tangent");
    if (st != PXB_OK) return st;
    if (nsteps < 0) return fail(PXB_ERR_ARG, "nsteps < 0");
    if (scheme != PXB_FE && scheme != PXB_SSPRK2) return fail(PXB_ERR_ARG, "scheme must be PXB_FE or PXB_SSPRK2");
    if (nsteps == 0) return PXB_OK;
    jvp_params(P, tp);
    st = jvp_run_impl(P, a, a_dot, nsteps, scheme, cfl, t0, (double*)dt_log, (double*)dt_dot_log,
                      (cudaStream_t)stream);
    jvp_params(P, nullptr);
    return st;
}

int pxb_re_vjp_init_params(pxb_re_plan* P, const pxb_re_fields* f, const pxb_re_fields* fbar,
                           const pxb_re_param_adjoints* pbar, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (refuse_ws(P, "the reverse mode") != PXB_OK) return PXB_ERR_UNSUPPORTED;
    if (P->c.dtype != PXB_F64) return fail(PXB_ERR_ARG, "the reverse mode runs on float64 plans");
    if (!f || !f->h || !f->hu || !f->hv) return fail(PXB_ERR_ARG, "state: h, hu and hv must be set");
    if (!fbar || !fbar->h || !fbar->hu || !fbar->hv || !fbar->z_b || !fbar->G)
        return fail(PXB_ERR_ARG, "adjoint: h, hu, hv, z_b and G must be set");
    if (pbar && pbar->seds_bar && fbar->n_b && !f->z_b) return fail(PXB_ERR_ARG, "state: z_b must be set");
    return vjp_init_impl(P, f, fbar, pbar, (cudaStream_t)stream);
}

int pxb_re_vjp_init(pxb_re_plan* P, const pxb_re_fields* f, const pxb_re_fields* fbar, void* stream) {
    return pxb_re_vjp_init_params(P, f, fbar, nullptr, stream);
}

int pxb_re_vjp_run(pxb_re_plan* P, const pxb_re_fields* a0, int32_t nsteps, int32_t scheme, double cfl, double t0,
                   int32_t checkpoint_every, const pxb_re_fields* abar, void* stream) {
    return pxb_re_vjp_run_params(P, a0, nsteps, scheme, cfl, t0, checkpoint_every, abar, nullptr, stream);
}

int pxb_re_vjp_run_params(pxb_re_plan* P, const pxb_re_fields* a0, int32_t nsteps, int32_t scheme, double cfl,
                          double t0, int32_t checkpoint_every, const pxb_re_fields* abar,
                          const pxb_re_param_adjoints* pbar, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    if (refuse_ws(P, "the reverse mode") != PXB_OK) return PXB_ERR_UNSUPPORTED;
    if (P->c.dtype != PXB_F64) return fail(PXB_ERR_ARG, "the reverse mode runs on float64 plans");
    if (!a0 || !a0->h || !a0->hu || !a0->hv || !a0->z || !a0->z_b || !a0->n_b || !a0->G)
        return fail(PXB_ERR_ARG, "state: h, hu, hv, z, z_b, n_b and G must be set");
    if (!abar || !abar->h || !abar->hu || !abar->hv || !abar->z_b || !abar->G)
        return fail(PXB_ERR_ARG, "adjoint: h, hu, hv, z_b and G must be set");
    if (nsteps < 0) return fail(PXB_ERR_ARG, "nsteps < 0");
    if (scheme != PXB_FE && scheme != PXB_SSPRK2) return fail(PXB_ERR_ARG, "scheme must be PXB_FE or PXB_SSPRK2");
    if (nsteps == 0) return PXB_OK;
    return vjp_run_impl(P, a0, nsteps, scheme, cfl, t0, checkpoint_every, abar, pbar, (cudaStream_t)stream);
}

int pxb_re_check(pxb_re_plan* P, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    return check_plan_error(P->c, (cudaStream_t)stream);
}

int pxb_re_ens_create(const pxb_re_ens_config* cfg, pxb_re_ens** out) {
    if (!cfg || !out) return fail(PXB_ERR_ARG, "null config or output pointer");
    *out = nullptr;
    if (cfg->nmembers < 1 || !cfg->members) return fail(PXB_ERR_ARG, "an ensemble needs at least one member");
    if (cfg->dtype != PXB_F32 && cfg->dtype != PXB_F64) return fail(PXB_ERR_ARG, "dtype must be PXB_F32 or PXB_F64");
    if (cfg->mpm && (!cfg->seds || cfg->nsed < 1 || cfg->nsed > PXB_MAX_SED))
        return fail(PXB_ERR_ARG, "MPM needs 1..8 sediment classes");
    if (cfg->band_rows < 0) return fail(PXB_ERR_ARG, "band_rows < 0");
    pxb_re_ens* E = new pxb_re_ens();
    auto bail = [&](int code) {
        E->release();
        delete E;
        return code;
    };
    E->dtype = cfg->dtype;
    E->mpm = cfg->mpm;
    E->nm = cfg->nmembers;
    E->band_rows = cfg->band_rows > 0 ? cfg->band_rows : 64;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&E->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return bail(fail(PXB_ERR_CUDA, "no CUDA device"));
    if (cfg->mpm) {
        fill_sed(E->sedf, cfg->seds, cfg->nsed);
        fill_sed(E->sedd, cfg->seds, cfg->nsed);
    }
    const size_t es = E->esize();
    int maxcount = 0;
    for (int k = 0; k < E->nm; ++k) {
        const pxb_re_member& M = cfg->members[k];
        const std::string who = "member " + std::to_string(k) + ": ";
        if (M.ny < 3 || M.nx < 3) return bail(fail(PXB_ERR_ARG, who + "grid must be at least 3 x 3 cells"));
        if (M.pitch < M.nx) return bail(fail(PXB_ERR_ARG, who + "pitch smaller than nx"));
        if ((long long)M.ny * M.pitch >= (1LL << 31)) return bail(fail(PXB_ERR_ARG, who + "plane of 2^31 elements or more"));
        if (!(M.dx > 0) || !std::isfinite(M.dx)) return bail(fail(PXB_ERR_ARG, who + "dx must be positive and finite"));
        if (!M.a.h || !M.a.hu || !M.a.hv || !M.a.z || !M.a.z_b || !M.a.n || !M.a.n_b || !M.a.G)
            return bail(fail(PXB_ERR_ARG, who + "every plane of a must be set"));
        if (!M.b.h || !M.b.hu || !M.b.hv || !M.b.z_b || !M.b.G)
            return bail(fail(PXB_ERR_ARG, who + "b needs h, hu, hv, z_b and G"));
        if (M.nhandlers < 0 || (M.nhandlers > 0 && !M.handlers)) return bail(fail(PXB_ERR_ARG, who + "null handlers"));
        EnsMember mb;
        mb.ny = M.ny;
        mb.nx = M.nx;
        mb.pitch = M.pitch;
        mb.dx = M.dx;
        mb.a = M.a;
        mb.b = M.b;
        mb.nodata = M.nodata;
        E->has_mask = E->has_mask || M.nodata != nullptr;
        for (int q = 0; q < M.nhandlers; ++q)
            if (!kind_ok(M.handlers[q].kind, false))
                return bail(fail(PXB_ERR_ARG, who + "handler " + std::to_string(q) + " is not a \"Roe Exner\" handler"));
        if (M.nhandlers > 0) {
            Resolved R = resolve(M.handlers, M.nhandlers, M.ny, M.nx, M.pitch, false, true);
            if (!R.error.empty()) return bail(fail(PXB_ERR_UNSUPPORTED, who + R.error));
            int mc = 0;
            const int st = upload_handlers(M.handlers, M.nhandlers, (long long)(M.ny - 1) * M.pitch + M.nx, mb.handlers, mc);
            E->m.push_back(mb);  // owned from here on (released with the ensemble)
            if (st != PXB_OK) return bail(st);
            maxcount = std::max(maxcount, mc);
            EnsMember& me = E->m.back();
            if (cudaMalloc(&me.ring, sizeof(pxb_ring_recipe) * R.ring.size()) != cudaSuccess ||
                cudaMemcpy(me.ring, R.ring.data(), sizeof(pxb_ring_recipe) * R.ring.size(), cudaMemcpyHostToDevice) !=
                    cudaSuccess)
                return bail(fail(PXB_ERR_CUDA, who + "ring recipes"));
        } else {
            E->m.push_back(mb);
        }
    }
    if (E->has_mask) {  // members without a mask read a zero plane
        for (auto& mb : E->m) {
            if (mb.nodata) continue;
            void* p = nullptr;
            const size_t bytes = (size_t)mb.ny * (size_t)mb.pitch;
            if (cudaMalloc(&p, bytes) != cudaSuccess || cudaMemset(p, 0, bytes) != cudaSuccess)
                return bail(fail(PXB_ERR_CUDA, "nodata plane"));
            E->owned.push_back(p);
            mb.nodata = (const uint8_t*)p;
        }
    }
    if (cudaMalloc(&E->bc_tmp, 6 * (size_t)std::max(1, maxcount) * es) != cudaSuccess ||
        cudaMalloc(&E->scr, sizeof(pxb::CflScratch) * E->nm) != cudaSuccess ||
        cudaMemset(E->scr, 0, sizeof(pxb::CflScratch) * E->nm) != cudaSuccess ||
        cudaMalloc(&E->dt, es * E->nm) != cudaSuccess || cudaMemset(E->dt, 0, es * E->nm) != cudaSuccess ||
        cudaStreamCreateWithFlags(&E->cap, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PXB_ERR_CUDA, "ensemble scratch"));
    for (int v = 0; v < 2; ++v)
        E->bps[v] = E->dtype == PXB_F64 ? pxb::ens_stage_blocks_per_sm<double>(E->mpm != 0, E->has_mask, v == 1)
                                        : pxb::ens_stage_blocks_per_sm<float>(E->mpm != 0, E->has_mask, v == 1);
    int st = E->dtype == PXB_F64 ? ens_build_stage_tables<double>(E) : ens_build_stage_tables<float>(E);
    if (st != PXB_OK) return bail(st);
    *out = E;
    return PXB_OK;
}

int pxb_re_ens_destroy(pxb_re_ens* E) {
    if (!E) return PXB_OK;
    cudaDeviceSynchronize();
    E->release();
    delete E;
    return PXB_OK;
}

int pxb_re_ens_init(pxb_re_ens* E, void* stream) {
    if (!E) return fail(PXB_ERR_ARG, "null ensemble");
    cudaStream_t s = (cudaStream_t)stream;
    for (const EnsMember& mb : E->m) {
        const int st = E->dtype == PXB_F64
                           ? init_fields<double>(mb.ny, mb.nx, mb.pitch, &mb.a, mb.nodata, E->mpm, E->sedd, mb.handlers,
                                                 E->bc_tmp, s)
                           : init_fields<float>(mb.ny, mb.nx, mb.pitch, &mb.a, mb.nodata, E->mpm, E->sedf, mb.handlers,
                                                E->bc_tmp, s);
        if (st != PXB_OK) return st;
    }
    return PXB_OK;
}

int pxb_re_ens_autotune(pxb_re_ens* E, void* stream, int32_t* band_rows) {
    if (!E) return fail(PXB_ERR_ARG, "null ensemble");
    cudaStream_t s = (cudaStream_t)stream;
    return E->dtype == PXB_F64 ? ens_autotune_impl<double>(E, s, band_rows) : ens_autotune_impl<float>(E, s, band_rows);
}

int pxb_re_ens_run(pxb_re_ens* E, int32_t nsteps, int32_t scheme, double cfl, void* dt_log, void* stream) {
    if (!E) return fail(PXB_ERR_ARG, "null ensemble");
    if (nsteps < 0) return fail(PXB_ERR_ARG, "nsteps < 0");
    if (scheme != PXB_FE && scheme != PXB_SSPRK2) return fail(PXB_ERR_ARG, "scheme must be PXB_FE or PXB_SSPRK2");
    if (nsteps == 0) return PXB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    return E->dtype == PXB_F64 ? ens_run_impl<double>(E, nsteps, scheme, cfl, dt_log, s)
                               : ens_run_impl<float>(E, nsteps, scheme, cfl, dt_log, s);
}

int pxb_re_ens_check(pxb_re_ens* E, void* stream, int32_t* first_bad) {
    if (!E) return fail(PXB_ERR_ARG, "null ensemble");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<pxb::CflScratch> h((size_t)E->nm);
    PXB_CUDA(cudaMemcpyAsync(h.data(), E->scr, sizeof(pxb::CflScratch) * E->nm, cudaMemcpyDeviceToHost, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    int bad = -1, code = 0;
    for (int k = 0; k < E->nm; ++k)
        if (h[(size_t)k].err != 0 && bad < 0) {
            bad = k;
            code = h[(size_t)k].err;
        }
    if (first_bad) *first_bad = bad;
    if (bad < 0) return PXB_OK;
    PXB_CUDA(cudaMemset2DAsync(&E->scr[0].err, sizeof(pxb::CflScratch), 0, sizeof(int), E->nm, s));
    PXB_CUDA(cudaStreamSynchronize(s));
    return fail(PXB_ERR_NONFINITE, "member " + std::to_string(bad) +
                                       ((code & 2) ? ": non-finite time step" : ": non-finite value in the updated state"));
}

int pxb_roe_plan_create(const pxb_roe_config* cfg, pxb_roe_plan** out) {
    if (!cfg || !out) return fail(PXB_ERR_ARG, "null config or output pointer");
    *out = nullptr;
    pxb_roe_plan* P = new pxb_roe_plan();
    int path = 0;
    int st = common_setup(P->c, cfg->ny, cfg->nx, cfg->pitch, cfg->dtype, cfg->dx, cfg->handlers, cfg->nhandlers, true,
                          PXB_PATH_FUSED, path);
    if (st != PXB_OK) {
        P->c.release();
        delete P;
        return st;
    }
    *out = P;
    return PXB_OK;
}

int pxb_roe_plan_destroy(pxb_roe_plan* plan) {
    if (!plan) return PXB_OK;
    cudaDeviceSynchronize();
    plan->c.release();
    delete plan;
    return PXB_OK;
}

int pxb_roe_cfl(pxb_roe_plan* P, const pxb_roe_fields* f, double cfl, void* dt_dev, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_roe_fields(f);
    if (st) return st;
    if (!dt_dev) return fail(PXB_ERR_ARG, "dt_dev is null");
    cudaStream_t s = (cudaStream_t)stream;
    return P->c.dtype == PXB_F64 ? roe_cfl_impl<double>(P, f, cfl, dt_dev, nullptr, s)
                                 : roe_cfl_impl<float>(P, f, cfl, dt_dev, nullptr, s);
}

int pxb_roe_stage(pxb_roe_plan* P, const pxb_roe_fields* in, const pxb_roe_fields* out, const pxb_roe_fields* avg,
                  const void* dt_dev, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_roe_fields(in);
    if (st) return st;
    st = check_roe_fields(out);
    if (st) return st;
    if (avg && (st = check_roe_fields(avg))) return st;
    if (!dt_dev) return fail(PXB_ERR_ARG, "dt_dev is null");
    if (in->h == out->h || in->hu == out->hu || in->hv == out->hv)
        return fail(PXB_ERR_ARG, "stage output must not alias its input");
    cudaStream_t s = (cudaStream_t)stream;
    return P->c.dtype == PXB_F64 ? roe_stage_impl<double>(P, in, out, avg, dt_dev, s)
                                 : roe_stage_impl<float>(P, in, out, avg, dt_dev, s);
}

int pxb_roe_run(pxb_roe_plan* P, const pxb_roe_fields* A, const pxb_roe_fields* B, int32_t nsteps, int32_t scheme,
                double cfl, void* dt_log, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    int st = check_roe_fields(A);
    if (st) return st;
    st = check_roe_fields(B);
    if (st) return st;
    if (nsteps < 0) return fail(PXB_ERR_ARG, "nsteps < 0");
    if (scheme != PXB_FE && scheme != PXB_SSPRK2) return fail(PXB_ERR_ARG, "scheme must be PXB_FE or PXB_SSPRK2");
    if (nsteps == 0) return PXB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const bool f64 = P->c.dtype == PXB_F64;
    const size_t es = P->c.esize();
    // b's z and n start as copies of a's (only ring cells are rewritten by a stage)
    PXB_CUDA(cudaMemcpy2DAsync(B->z, P->c.pitch * es, A->z, P->c.pitch * es, P->c.nx * es, P->c.ny,
                               cudaMemcpyDeviceToDevice, s));
    PXB_CUDA(cudaMemcpy2DAsync(B->n, P->c.pitch * es, A->n, P->c.pitch * es, P->c.nx * es, P->c.ny,
                               cudaMemcpyDeviceToDevice, s));
    PXB_CUDA(cudaMemsetAsync(&P->c.scr->step, 0, sizeof(unsigned int), s));
    auto cfl_call = [&](const pxb_roe_fields* f, cudaStream_t st2) {
        return f64 ? roe_cfl_impl<double>(P, f, cfl, P->c.dt_dev, dt_log, st2)
                   : roe_cfl_impl<float>(P, f, cfl, P->c.dt_dev, dt_log, st2);
    };
    auto stage_call = [&](const pxb_roe_fields* in, const pxb_roe_fields* out, const pxb_roe_fields* avg,
                          cudaStream_t st2) {
        return f64 ? roe_stage_impl<double>(P, in, out, avg, P->c.dt_dev, st2)
                   : roe_stage_impl<float>(P, in, out, avg, P->c.dt_dev, st2);
    };
    const double cfl_d = cfl;
    std::vector<const void*> key = {A->h, A->hu, A->hv, A->z, A->n, B->h, B->hu, B->hv, B->z, B->n, dt_log,
                                    (const void*)(intptr_t)scheme};
    key.push_back(*(const void* const*)&cfl_d);
    if (scheme == PXB_SSPRK2) {
        return run_graph(P->c, key, nsteps, s, [&](cudaStream_t st2) {
            int r = cfl_call(A, st2);
            if (r == PXB_OK) r = stage_call(A, B, nullptr, st2);
            if (r == PXB_OK) r = stage_call(B, A, A, st2);
            return r;
        });
    }
    int r = run_graph(P->c, key, nsteps / 2, s, [&](cudaStream_t st2) {
        int q = cfl_call(A, st2);
        if (q == PXB_OK) q = stage_call(A, B, nullptr, st2);
        if (q == PXB_OK) q = cfl_call(B, st2);
        if (q == PXB_OK) q = stage_call(B, A, nullptr, st2);
        return q;
    });
    if (r != PXB_OK || (nsteps & 1) == 0) return r;
    r = cfl_call(A, s);
    if (r == PXB_OK) r = stage_call(A, B, nullptr, s);
    if (r != PXB_OK) return r;
    const void* src[5] = {B->h, B->hu, B->hv, B->z, B->n};
    void* dst[5] = {A->h, A->hu, A->hv, A->z, A->n};
    for (int k = 0; k < 5; ++k)
        PXB_CUDA(cudaMemcpy2DAsync(dst[k], P->c.pitch * es, src[k], P->c.pitch * es, P->c.nx * es, P->c.ny,
                                   cudaMemcpyDeviceToDevice, s));
    return PXB_OK;
}

int pxb_roe_check(pxb_roe_plan* P, void* stream) {
    if (!P) return fail(PXB_ERR_ARG, "null plan");
    return check_plan_error(P->c, (cudaStream_t)stream);
}

}  // extern "C"
