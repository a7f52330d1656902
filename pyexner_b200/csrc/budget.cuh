// Water and sediment volume budget of the Roe-Exner step.
//
// The reference updates every cell by flux differences: the hydro fluctuations of each
// face are scattered to its two cells and U -= dt/dx F (roe_exner.py:597-606), and the
// Exner face fluxes enter z_b with opposite signs on the two sides (roe_exner.py:708-715).
// Summed over the physical cells the interior faces telescope, so the change of the water
// volume sum(h) dx^2 and of the erodible-bed volume sum(z_b) dx^2 over a step equals
// minus dt dx times the flux through the outer boundary of the physical cells, up to
// rounding.  The stage kernel leaves the boundary flux sum of every work item in a
// partial array; budget_stage_kernel adds one stage's total, weighted by the integrator
// (1 for Forward Euler, 1/2 per stage for SSPRK2) and by dt dx, into a float64 outflow
// accumulator with Neumaier compensation; volume_kernel sums the two volumes of a state
// the same way.  Every sum runs in a fixed order, so the results do not depend on how the
// GPU scheduled the work.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pxb {

// Outflow volumes (m^3) through the boundary of the physical cells since the accumulator
// was zeroed, each with its Neumaier compensation term: the total is sum + comp.
struct BudgetAcc {
    double water, water_comp, sed, sed_comp;
};

// Neumaier's compensated summation step: s + c carries the sum of every x added.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    const double t = s + x;
    c += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
    s = t;
}

// One block of 256 threads: the item partials of one stage (2 per item: water, sediment)
// summed in a fixed order, times w * dt * dx, added to the accumulator.
template <class T>
__global__ void __launch_bounds__(256) budget_stage_kernel(const double* part, int nitems, const T* dt, double w_dx,
                                                           BudgetAcc* acc) {
    __shared__ double sh[4][256];
    double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
    for (int k = threadIdx.x; k < nitems; k += blockDim.x) {
        neumaier_add(s0, c0, part[2 * k]);
        neumaier_add(s1, c1, part[2 * k + 1]);
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = c0;
    sh[2][threadIdx.x] = s1;
    sh[3][threadIdx.x] = c1;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double S0 = 0.0, C0 = 0.0, S1 = 0.0, C1 = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
        neumaier_add(S0, C0, sh[0][t]);
        C0 += sh[1][t];
        neumaier_add(S1, C1, sh[2][t]);
        C1 += sh[3][t];
    }
    const double scale = w_dx * (double)(*dt);
    neumaier_add(acc->water, acc->water_comp, (S0 + C0) * scale);
    neumaier_add(acc->sed, acc->sed_comp, (S1 + C1) * scale);
}

// Partial sums of h and z_b over the physical cells (rows and columns 1 .. n-2 that are
// not nodata): block b writes part[4b .. 4b+3] = (sum h, comp, sum z_b, comp).  Rows are
// spread over the blocks, columns over the threads, each in a fixed order.
template <class T>
__global__ void __launch_bounds__(256) volume_kernel(int ny, int nx, long long pitch, const T* h, const T* zb,
                                                     const uint8_t* nodata, double* part) {
    __shared__ double sh[4][256];
    double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
    for (int r = 1 + blockIdx.x; r <= ny - 2; r += gridDim.x) {
        const long long row = (long long)r * pitch;
        for (int c = 1 + threadIdx.x; c <= nx - 2; c += blockDim.x) {
            if (nodata && nodata[row + c]) continue;
            neumaier_add(s0, c0, (double)h[row + c]);
            neumaier_add(s1, c1, (double)zb[row + c]);
        }
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = c0;
    sh[2][threadIdx.x] = s1;
    sh[3][threadIdx.x] = c1;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double S0 = 0.0, C0 = 0.0, S1 = 0.0, C1 = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
        neumaier_add(S0, C0, sh[0][t]);
        C0 += sh[1][t];
        neumaier_add(S1, C1, sh[2][t]);
        C1 += sh[3][t];
    }
    part[4 * blockIdx.x] = S0;
    part[4 * blockIdx.x + 1] = C0;
    part[4 * blockIdx.x + 2] = S1;
    part[4 * blockIdx.x + 3] = C1;
}

// The block partials of volume_kernel in block order, times dx^2: out = (water, bed) in m^3.
static __global__ void volume_final_kernel(const double* part, int nblocks, double dx2, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double S0 = 0.0, C0 = 0.0, S1 = 0.0, C1 = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        neumaier_add(S0, C0, part[4 * b]);
        C0 += part[4 * b + 1];
        neumaier_add(S1, C1, part[4 * b + 2]);
        C1 += part[4 * b + 3];
    }
    out[0] = (S0 + C0) * dx2;
    out[1] = (S1 + C1) * dx2;
}

}  // namespace pxb
