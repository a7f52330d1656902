// Launch entry points implemented per precision (kernels_f32.cu, kernels_f64.cu).
#pragma once
#include <cuda_runtime.h>

#include "budget.cuh"
#include "ens.cuh"
#include "init_bc.cuh"
#include "re_cfl.cuh"
#include "re_general.cuh"
#include "re_stage.cuh"
#include "roe_plain.cuh"
#include "dual.cuh"

#include <string>

namespace pxb {

// Records the message returned by pxb_last_error() on this thread; returns `code`.
int set_error(int code, const std::string& msg);

// Boundary set-up on the device (setup_f64.cu).
cudaError_t launch_label(int ny, int nx, const double* xc, const double* yc, const double* verts, int npoly, int nv,
                         uint8_t* labels, cudaStream_t s);
cudaError_t launch_label_count(int ny, int nx, int npoly, const uint8_t* labels, long long* counts, cudaStream_t s);
cudaError_t launch_label_fill(int ny, int nx, int npoly, const uint8_t* labels, const long long* offsets,
                              long long* cells, cudaStream_t s);

template <class T>
cudaError_t launch_re_stage(const REStageArgs<T>& a, bool mpm, bool has_mask, bool avg, int grid, cudaStream_t s);
template <class T>
int re_stage_blocks_per_sm(bool mpm, bool has_mask, bool avg);
template <class T>
cudaError_t launch_re_cfl(const CflArgs<T>& a, bool has_mask, int grid, cudaStream_t s);
template <class T>
int re_cfl_blocks_per_sm(bool has_mask);
// Volume budget (budget.cuh): one stage's boundary outflow into the accumulator; the
// water and bed volumes of a state into out[2] (device).
template <class T>
cudaError_t launch_budget_stage(const double* part, int nitems, const T* dt, double w_dx, BudgetAcc* acc,
                                cudaStream_t s);
template <class T>
cudaError_t launch_volume(int ny, int nx, long long pitch, const T* h, const T* zb, const uint8_t* nodata,
                          double* part, int nblocks, double dx2, double* out, cudaStream_t s);
template <class T>
cudaError_t launch_re_init(const InitArgs<T>& a, cudaStream_t s);
template <class T>
cudaError_t launch_bc(const BcArgs<T>& a, cudaStream_t s);
// Phases of the general stage path (re_general.cuh).
enum GenPhase { GEN_HYDRO = 0, GEN_CORR = 1, GEN_GRASS = 2, GEN_EXNER = 3, GEN_STORE = 4 };
template <class T>
cudaError_t launch_re_general(const GenArgs<T>& a, int phase, cudaStream_t s);
template <class T>
cudaError_t launch_set_time(CflScratch* scr, double t0, cudaStream_t s);

// Reverse mode (kernels_adj.cu); the argument structs are in adjoint_args.cuh.
struct AdjArgs;
struct AdjBcArgs;
struct AdjCflArgs;
cudaError_t launch_adj_store(int ny, int nx, long long pitch, double scale, const double* const o[5], double* const S[5],
                             double* const A[5], cudaStream_t s);
cudaError_t launch_adj_stage(const AdjArgs& a, int phase, cudaStream_t s);
cudaError_t launch_adj_bc(const AdjBcArgs& a, cudaStream_t s);
cudaError_t launch_adj_cfl(const AdjCflArgs& a, cudaStream_t s);
cudaError_t launch_adj_compute_n(int ny, int nx, long long pitch, int mpm, const double* zb, double* nbbar,
                                 double* nbar, double* npbar, cudaStream_t s);

// Tangent-linear model (kernels_dual.cu).
cudaError_t launch_dual_cfl(const DualCflArgs& a, cudaStream_t s);
cudaError_t launch_dual_pack(int ny, int nx, long long pitch, const double* v, const double* t, Dual* out,
                             cudaStream_t s);
cudaError_t launch_dual_unpack(int ny, int nx, long long pitch, const Dual* in, double* v, double* t, cudaStream_t s);
template <class T>
cudaError_t launch_ens_stage(const EnsStageArgs<T>& a, bool mpm, bool has_mask, bool avg, int grid, cudaStream_t s);
template <class T>
int ens_stage_blocks_per_sm(bool mpm, bool has_mask, bool avg);
template <class T>
cudaError_t launch_ens_cfl(const EnsCflArgs<T>& a, bool has_mask, int grid, cudaStream_t s);
template <class T>
cudaError_t launch_roe_stage(const RoeArgs<T>& a, bool avg, cudaStream_t s);
template <class T>
cudaError_t launch_roe_cfl(const CflArgs<T>& a, int grid, cudaStream_t s);

}  // namespace pxb
