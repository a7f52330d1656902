// Boundary set-up on the device: the even-odd polygon test of every cell centre and the
// raster-order list of each polygon's cells (PyExner src/PyExner/domain/boundary_registry.py:
// point_in_polygon 19-44, compute_label_mask 46-59, the argwhere of
// compute_reflective_indices 61-82).  Off the clock; it replaces the host test for large
// grids, where the vectorised host version needs (cells x vertices) temporaries.
//
// Compiled with --fmad=false: the crossing abscissa tx = xi + (xj - xi) * (y - yi) / (yj - yi)
// rounds every operation on its own, as NumPy / XLA CPU do, so the labels are the host's bits.
#include <cuda_runtime.h>

#include <cstdint>

#include "pxb_launch.h"

namespace pxb {

// labels[p][r][c] = 1 when the centre (xc[c], yc[r]) is inside polygon p (even-odd rule,
// edge k from vertex k-1 to vertex k, the vertex list zero-padded to nv as the reference
// pads it; a point on a right-hand edge counts within 1e-8).
__global__ void label_kernel(int ny, int nx, const double* __restrict__ xc, const double* __restrict__ yc,
                             const double* __restrict__ verts, int npoly, int nv, uint8_t* __restrict__ labels) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= ny || c >= nx) return;
    const double x = xc[c], y = yc[r];
    for (int p = 0; p < npoly; ++p) {
        const double* v = verts + (size_t)p * nv * 2;
        int hits = 0;
        for (int k = 0; k < nv; ++k) {
            const int j = k == 0 ? nv - 1 : k - 1;
            const double xi = v[2 * k], yi = v[2 * k + 1], xj = v[2 * j], yj = v[2 * j + 1];
            const bool crosses = (yi > y) != (yj > y);
            const double den = crosses ? (yj - yi) : 1.0;
            const double tx = xi + (xj - xi) * (y - yi) / den;
            hits += (crosses && (x <= tx + 1e-8)) ? 1 : 0;
        }
        labels[((size_t)p * ny + r) * nx + c] = (uint8_t)(hits & 1);
    }
}

// One warp per (polygon, row): number of labelled cells.
__global__ void label_count_kernel(int ny, int nx, int npoly, const uint8_t* __restrict__ labels,
                                   long long* __restrict__ counts) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= npoly * ny) return;
    const uint8_t* row = labels + (size_t)w * nx;
    long long n = 0;
    for (int c0 = 0; c0 < nx; c0 += 32) {
        const int c = c0 + lane;
        const unsigned b = __ballot_sync(0xffffffffu, c < nx && row[c] != 0);
        n += __popc(b);
    }
    if (lane == 0) counts[w] = n;
}

// One warp per (polygon, row): flat indices r * nx + c of the labelled cells, in raster
// order, from the row's offset.
__global__ void label_fill_kernel(int ny, int nx, int npoly, const uint8_t* __restrict__ labels,
                                  const long long* __restrict__ offsets, long long* __restrict__ cells) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= npoly * ny) return;
    const int r = w % ny;
    const uint8_t* row = labels + (size_t)w * nx;
    long long off = offsets[w];
    for (int c0 = 0; c0 < nx; c0 += 32) {
        const int c = c0 + lane;
        const bool on = c < nx && row[c] != 0;
        const unsigned b = __ballot_sync(0xffffffffu, on);
        if (on) cells[off + __popc(b & ((1u << lane) - 1u))] = (long long)r * nx + c;
        off += __popc(b);
    }
}

cudaError_t launch_label(int ny, int nx, const double* xc, const double* yc, const double* verts, int npoly, int nv,
                         uint8_t* labels, cudaStream_t s) {
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
    label_kernel<<<g, b, 0, s>>>(ny, nx, xc, yc, verts, npoly, nv, labels);
    return cudaGetLastError();
}

cudaError_t launch_label_count(int ny, int nx, int npoly, const uint8_t* labels, long long* counts, cudaStream_t s) {
    const long long warps = (long long)npoly * ny;
    label_count_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(ny, nx, npoly, labels, counts);
    return cudaGetLastError();
}

cudaError_t launch_label_fill(int ny, int nx, int npoly, const uint8_t* labels, const long long* offsets,
                              long long* cells, cudaStream_t s) {
    const long long warps = (long long)npoly * ny;
    label_fill_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(ny, nx, npoly, labels, offsets, cells);
    return cudaGetLastError();
}

}  // namespace pxb
