// Tangent-linear model of the float64 Roe-Exner step: the CFL reduction on dual numbers
// and the conversions between (value plane, tangent plane) pairs and dual planes.  The
// stage itself is the general path's kernel chain (re_general.cuh) instantiated on Dual.
//
// dt = max(cfl * dx / s_max, 1e-6) (roe_exner_solver.py:118-122) depends on the state
// through the fastest face: ds_max is the tangent of the face whose speed equals s_max (a
// second pass finds it by the value's bits), averaged over the faces that tie for the
// maximum as JAX's min/max reductions do (mirror-image faces at reflective walls tie
// exactly), then d(dt) = -cfl * dx * ds_max / s_max^2, and 0 where the floor is active.
// The tie sum is accumulated with atomics, so with ties the tangent's last bits may vary
// from run to run.
#pragma once
#include "dual.cuh"
#include "pxb_device.cuh"

namespace pxb {

__device__ __forceinline__ bool dual_face(const DualCflArgs& a, int r, int c, bool yf, Dual& s) {
    if (yf ? (r + 1 >= a.ny) : (c + 1 >= a.nx)) return false;
    const long long i = (long long)r * a.pitch + c;
    const long long j = yf ? i + a.pitch : i + 1;
    const bool mi = a.nodata ? a.nodata[i] != 0 : false, mj = a.nodata ? a.nodata[j] != 0 : false;
    const double DRY = DRY_TOL;
    if (!(((a.h[i].v > DRY) || (a.h[j].v > DRY)) && !(mi || mj))) return false;
    const CCell<Dual> I = make_ccell(a.h[i], a.hu[i], a.hv[i], a.G[i]);
    const CCell<Dual> J = make_ccell(a.h[j], a.hu[j], a.hv[j], a.G[j]);
    s = yf ? face_speed<Dual, true>(I, J) : face_speed<Dual, false>(I, J);
    return true;
}

// pass 1: maximum of the face speeds' values (bits, as re_cfl_kernel)
__global__ void __launch_bounds__(256) dual_cfl_max_kernel(const DualCflArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long best = 0ull;
    if (r < a.ny && c < a.nx) {
        for (int yf = 0; yf < 2; ++yf) {
            Dual s;
            if (dual_face(a, r, c, yf != 0, s)) {
                const unsigned long long b = speed_bits(s.v);
                best = b > best ? b : best;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(FULL, best, o);
        best = other > best ? other : best;
    }
    if ((threadIdx.x & 31) == 0 && best != 0ull) atomicMax(&a.scr->maxbits, best);
}

// pass 2: the tangent of a face whose speed is the maximum
__global__ void __launch_bounds__(256) dual_cfl_arg_kernel(const DualCflArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= a.ny || c >= a.nx) return;
    const unsigned long long m = a.scr->maxbits;
    for (int yf = 0; yf < 2; ++yf) {
        Dual s;
        if (dual_face(a, r, c, yf != 0, s) && speed_bits(s.v) == m) {
            atomicAdd(&a.scr->dsum, s.d);
            atomicAdd(&a.scr->nties, 1u);
        }
    }
}

__global__ void dual_cfl_finalize_kernel(const DualCflArgs a) {
    DualScratch* scr = a.scr;
    const Dual smax(bits_speed(scr->maxbits, 0.0), scr->nties > 0 ? scr->dsum / scr->nties : 0.0);
    Dual dt = Dual(a.cfl) * (Dual(a.dx) / smax);
    if (dt.v < a.floor_dt) dt = Dual(a.floor_dt);
    *a.dt_out = dt;
    if (a.dt_log) a.dt_log[scr->step] = dt.v;
    if (a.dt_dot_log) a.dt_dot_log[scr->step] = dt.d;
    scr->step += 1;
    scr->t_step = scr->t_next;
    scr->t_next = scr->t_next + dt.v;
    if (!isfinite(dt.v)) *a.err |= 2;
    scr->maxbits = 0ull;
    scr->dsum = 0.0;
    scr->nties = 0u;
}

// (value, tangent) planes -> dual plane; a null tangent plane is zero
__global__ void dual_pack_kernel(int ny, int nx, long long pitch, const double* v, const double* t, Dual* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= ny || c >= nx) return;
    const long long i = (long long)r * pitch + c;
    out[i] = Dual(v[i], t ? t[i] : 0.0);
}

__global__ void dual_unpack_kernel(int ny, int nx, long long pitch, const Dual* in, double* v, double* t) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= ny || c >= nx) return;
    const long long i = (long long)r * pitch + c;
    v[i] = in[i].v;
    if (t) t[i] = in[i].d;
}

}  // namespace pxb
