/*
 * pyexner_b200 — C ABI of the B200 (sm_100a) explicit finite-volume step of PyExner.
 *
 * This boundary replaces the jitted JAX calls that PyExner's integrators make on its
 * solver bundles (PyExner src/PyExner/solvers/registry.py:18-38):
 *
 *   step_fn(state, time, dt, mask, config) -> state        roe_exner_solver.py:80-116, roe_solver.py:40-54
 *   compute_dt_fn(state, cfl, mask, config) -> dt           roe_exner_solver.py:118-122, roe_solver.py:56-60
 *   init_fn(state, mask, config) -> state                  roe_exner_solver.py:58-78
 *
 * and the device loops of the integrators that drive them
 * (src/PyExner/integrators/forwardeuler.py:37-49, src/PyExner/integrators/SSPRK2.py:30-51).
 *
 * Conventions
 *   - Every plane is a row-major (ny, nx) array INCLUDING the one-cell ring, with a
 *     row pitch given in elements.  Row index grows toward -y: y-faces carry the normal
 *     (0,-1) (roe_exner.py:577).  All planes of one call share ny, nx, pitch and dtype.
 *   - dtype PXB_F32 or PXB_F64 selects the arithmetic of every kernel of a plan.
 *   - Device pointers are owned by the caller.  A plan allocates its small tables
 *     (boundary recipes, the CFL reduction word, the error word) once, in
 *     pxb_*_plan_create; no call after that allocates.
 *   - Every call is stream-ordered on the given cudaStream_t (may be 0) and returns a
 *     status code; pxb_last_error() gives the message of the last failure on the
 *     calling thread.
 */
#ifndef PYEXNER_B200_H
#define PYEXNER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PXB_OK 0
#define PXB_ERR_ARG 1        /* bad argument (null pointer, size, dtype, layout)      */
#define PXB_ERR_CUDA 2       /* a CUDA call failed                                     */
#define PXB_ERR_NONFINITE 3  /* the device flagged a non-finite dt or state value      */
#define PXB_ERR_UNSUPPORTED 4/* boundary layout the requested stage path does not cover */

#define PXB_F32 0
#define PXB_F64 1

#define PXB_FE 0     /* Forward Euler, forwardeuler.py:37-49        */
#define PXB_SSPRK2 1 /* SSPRK2 (intended form), SSPRK2.py:30-51     */

/* Boundary handler kinds (PyExner BOUNDARY_REGISTRY names, "<flux_scheme> <type>"). */
#define PXB_BC_RE_REFLECTIVE 1       /* "Roe Exner Reflective"      roeexner_reflective.py:17-63      */
#define PXB_BC_RE_TRANSMISSIVE 2     /* "Roe Exner Transmissive"    roeexner_transmissive.py:17-31    */
#define PXB_BC_RE_TRANSMISSIVEBED 3  /* "Roe Exner TransmissiveBed" roeexner_transmissivebed.py:17-27 */
#define PXB_BC_RE_CONSTANTINFLUX 4   /* "Roe Exner ConstantInflux"  roeexner_constantinflux.py:18-48  */
#define PXB_BC_ROE_REFLECTIVE 5      /* "Roe Reflective"            roe_reflective.py:18-44           */
#define PXB_BC_ROE_TRANSMISSIVE 6    /* "Roe Transmissive"          roe_transmissive.py:17-43         */
#define PXB_BC_RE_CONSTANTOUTFLUX 7  /* "Roe Exner ConstantOutflux" roeexner_constantoutflux.py:18-73 */
#define PXB_BC_RE_BERTHON 8          /* "Roe Exner Berthon"         roeexner_berthon.py:19-56         */
#define PXB_BC_RE_NORMALFLOWDEPTH 9  /* "Roe Exner NormalFlowDepth" roeexner_normalflowdepth.py:19-51 */
#define PXB_BC_RE_STEEPFALL 10       /* "Roe Exner SteepFall"       roeexner_steepfall.py:17-26       */
#define PXB_BC_RE_ZEROMOMENTUM 11    /* "Roe Exner ZeroMomentum"    roeexner_zeromomentum.py:16-31    */

/* Stage paths of a Roe-Exner plan (pxb_re_config.stage_path). */
#define PXB_PATH_AUTO 0     /* fused when the boundary layout allows it, else general          */
#define PXB_PATH_FUSED 1    /* one fused kernel per stage; ring layouts of kinds 1-4 only       */
#define PXB_PATH_GENERAL 2  /* cell-parallel kernel chain; any handler layout and kind          */

/* One boundary handler: cells by (flat row*pitch+col) index, donors alike.
 * Replaces a handler object built by BoundaryManager (boundary_registry.py:132-171)
 * with the index maps of compute_reflective_indices (boundary_registry.py:61-82).
 * ZeroMomentum handlers carry the cells of their mask and use each cell as its own donor.
 * values: the YAML values as the reference parses them (float32, NaN allowed,
 * boundary_registry.py:107-110), zero-padded to 8:
 *   ConstantOutflux  [q, nx, ny]                  Newton depth on the outgoing invariant
 *   Berthon          [q, A, alpha, beta, gamma, x] z_b = -alpha*t + zb0(q, A, alpha, beta, gamma, x)
 *   NormalFlowDepth  [q, A, alpha, beta, gamma, x] as Berthon, and h = q/u
 *   ZeroMomentum     [h, hu, hv, z]               hu = values[1]*nx, hv = values[1]*ny (NaN: keep) */
typedef struct pxb_bc_handler {
    int32_t kind;
    int32_t count;          /* number of (boundary, donor) pairs            */
    const int64_t* cells;   /* host array, `count` boundary cells           */
    const int64_t* donors;  /* host array, `count` donor (interior) cells   */
    double nx, ny;          /* outward normal as given in the YAML          */
    double hu_const, hv_const; /* ConstantInflux: float32(values[0]*values[1]), float32(values[0]*values[2]) */
    double values[8];
} pxb_bc_handler;

/* Per ring cell, the boundary result after all handlers, as a function of the
 * pre-boundary values of one donor cell per field group, resolved by the library from
 * the ordered handlers at plan creation (internal table; listed here because its
 * layout is part of the device-side contract).  dy/dx are donor offsets in rows/columns.
 * flags: 1 h, 2 momentum, 4 momentum is constant (m[0], m[1]), 8 z_b, 16 G.
 * momentum: hu' = m[0]*hu + m[1]*hv, hv' = m[2]*hu + m[3]*hv (donor values).
 * Table layout: top row [nx], bottom row [nx], left column [ny], right column [ny]. */
typedef struct pxb_ring_recipe {
    int8_t h_dy, h_dx, m_dy, m_dx, zb_dy, zb_dx, g_dy, g_dx;
    uint32_t flags;
    uint32_t pad;
    double m[4];
} pxb_ring_recipe;

/* Roe-Exner state planes (RoeExnerState, src/PyExner/state/roe_exner_state.py:8-48). */
typedef struct pxb_re_fields {
    void* h;
    void* hu;
    void* hv;
    void* z;    /* rigid bed (static)                         */
    void* z_b;  /* erodible layer                              */
    void* n;    /* Manning (only boundary handlers touch it)   */
    void* n_b;  /* Manning used in the flux (frozen after init) */
    void* G;    /* grass factor                                */
} pxb_re_fields;

/* Plain Roe state planes (RoeState, src/PyExner/state/roe_state.py:8-61). */
typedef struct pxb_roe_fields {
    void* h;
    void* hu;
    void* hv;
    void* z;
    void* n;
} pxb_roe_fields;

typedef struct pxb_re_plan pxb_re_plan;
typedef struct pxb_roe_plan pxb_roe_plan;

/* Configuration of a Roe-Exner plan.
 * mpm = 1: grass factor from Meyer-Peter & Mueller (roe_exner.py:85-130), erosion.grass_factor "MPM";
 * mpm = 0: constant grass factor read from the state (roe_exner.py:136-140).
 * seds: host pointer to the 7 x nsed matrix of src/PyExner/io/pnetcdf_reader.py:136-158
 *       (row-major: fraction, d50, density, k_d, k_e, theta_c, porosity), nsed <= 8.
 * nodata: device uint8 plane of mask[0] (roe_exner_solver.py:21-39) or NULL if all false. */
typedef struct pxb_re_config {
    int32_t ny, nx;
    int64_t pitch;
    int32_t dtype;
    int32_t mpm;
    double dx;
    const double* seds;
    int32_t nsed;
    const uint8_t* nodata;
    const pxb_bc_handler* handlers; /* in YAML order; resolved into ring recipes at plan creation */
    int32_t nhandlers;
    int32_t band_rows;              /* rows per warp band of the stage kernel; 0 = automatic   */
    int32_t stage_path;             /* PXB_PATH_AUTO / _FUSED / _GENERAL                       */
} pxb_re_config;

/* --- Roe-Exner ------------------------------------------------------------------ */
int pxb_re_plan_create(const pxb_re_config* cfg, pxb_re_plan** out);
int pxb_re_plan_destroy(pxb_re_plan* plan);

/* Caller-owned device memory (the workspace of the plan-and-buffers ownership model: the host
 * framework owns every device buffer, the library allocates none).  *bytes receives the device
 * bytes a plan for cfg needs: its boundary tables and scratch, and on the general stage path
 * its seven scratch planes.  pxb_re_plan_create_in builds the same plan inside `workspace` (a
 * device pointer, 256-byte aligned, at least that many bytes, untouched by the caller until
 * pxb_re_plan_destroy): its creation and its pxb_re_init, pxb_re_cfl, pxb_re_stage,
 * pxb_re_volume, pxb_re_autotune and pxb_re_check calls allocate no device memory.
 * pxb_re_run captures its step graph on first use, which the CUDA driver allocates for;
 * pxb_re_set_budget, the tangent-linear model (pxb_re_jvp_*) and the reverse mode
 * (pxb_re_vjp_*), which allocate their tables on first use, return PXB_ERR_UNSUPPORTED on
 * such a plan.  Replaces the plans' cudaMalloc of their tables (no counterpart in the
 * reference, whose JAX arrays are allocated by XLA: solvers/roe_exner_solver.py:58-122). */
int pxb_re_plan_workspace_size(const pxb_re_config* cfg, size_t* bytes);
int pxb_re_plan_create_in(const pxb_re_config* cfg, void* workspace, size_t bytes, pxb_re_plan** out);

/* init_fn_roeexner (roe_exner_solver.py:58-78): n_b, G, then the handlers at t = 0, in place. */
int pxb_re_init(pxb_re_plan* plan, const pxb_re_fields* f, void* stream);

/* The stage path the plan resolved to: PXB_PATH_FUSED or PXB_PATH_GENERAL. */
int pxb_re_plan_path(const pxb_re_plan* plan);

/* Autotuner of the fused stage kernel's band height (no counterpart in the reference):
 * times a set of heights on stage a -> b (plain and SSPRK2-averaged with a; `a` is not
 * written, `b` is scratch) and keeps the fastest for the plan; *band_rows (may be NULL)
 * receives it, 0 on the general path.  Synchronises `stream`. */
int pxb_re_autotune(pxb_re_plan* plan, const pxb_re_fields* a, const pxb_re_fields* b, void* stream,
                    int32_t* band_rows);

/* compute_dt_roeexner (roe_exner_solver.py:118-122): dt = max(cfl * min_faces dt_face, 1e-6)
 * written to dt_dev (one element of the plan dtype, device memory). */
int pxb_re_cfl(pxb_re_plan* plan, const pxb_re_fields* f, double cfl, void* dt_dev, void* stream);

/* step_fn_roeexner (roe_exner_solver.py:80-116): one stage from `in` to `out` with the
 * device scalar dt at simulation time `time` (read by time-dependent handlers).  If `avg`
 * is not NULL the result is 0.5*avg + 0.5*stage(in) on h, hu, hv, z_b, G (the SSPRK2
 * combination, SSPRK2.py:40); out may alias avg, never in.  out->G may be NULL when the
 * caller does not need G (it is recomputed in MPM mode).  The general path also carries
 * n through the handlers: it writes out->n when set (averaged with avg->n when both are
 * set); the fused path leaves n alone (its plans only accept layouts that keep n fixed). */
int pxb_re_stage(pxb_re_plan* plan, const pxb_re_fields* in, const pxb_re_fields* out,
                 const pxb_re_fields* avg, const void* dt_dev, double time, void* stream);

/* A fixed number of integrator steps (forwardeuler.py:37-49 / SSPRK2.py:30-51 without
 * output probes), starting at simulation time t0; the time of each step (the sum of the
 * dts before it, in float64) is kept on the device.  The state starts and ends in `a`;
 * `b` is scratch state of the same layout (h, hu, hv, z_b, G are written; n too on the
 * general path, which needs b->n distinct from a->n).  dt_log: device array of nsteps
 * dts or NULL.  The steps are captured once into a CUDA graph and replayed. */
int pxb_re_run(pxb_re_plan* plan, const pxb_re_fields* a, const pxb_re_fields* b, int32_t nsteps,
               int32_t scheme, double cfl, double t0, void* dt_log, void* stream);

/* Water and sediment volume budget.  The reference advances every cell by flux
 * differences (the fluctuation scatter and update of roe_exner.py:597-606, the Exner
 * update of roe_exner.py:708-715), so over the physical cells (rows and columns 1 .. n-2
 * that are not nodata) the interior faces telescope: the volumes change by the flux
 * through their outer boundary, up to rounding.
 *
 * pxb_re_volume: volumes[0] = sum h dx^2, volumes[1] = sum z_b dx^2 over the physical
 * cells (host array of 2), summed in float64 with Neumaier compensation in a fixed order.
 * Allocates a small scratch on its first call; synchronises `stream`.
 *
 * pxb_re_set_budget: acc_dev (device array of 4 doubles, zeroed by the caller) receives,
 * during every later pxb_re_run, the water and sediment volume that left the physical
 * cells through their boundary faces: acc[0] + acc[1] (water, m^3), acc[2] + acc[3]
 * (sediment, m^3), each pair a Neumaier sum and its compensation, accumulated in float64.
 * The face flux is the one the fluctuations telescope to: for a face with left (west or
 * north) cell I, h_I u_n,I + upwM_0 for water and the upwind Exner flux for sediment;
 * each stage adds dt dx times its boundary sum, times 1/2 under SSPRK2.  Then
 * volume(end) - volume(start) + outflow vanishes to rounding.  Fused stage path only
 * (PXB_ERR_UNSUPPORTED otherwise); acc_dev = NULL switches it off.  The first call with
 * an accumulator allocates the per-item partial array (16 bytes per work item of
 * one-row bands, the most items a band geometry can have). */
int pxb_re_volume(pxb_re_plan* plan, const pxb_re_fields* f, double* volumes, void* stream);
int pxb_re_set_budget(pxb_re_plan* plan, double* acc_dev);

/* Tangent-linear model (forward-mode derivative) of pxb_re_init / pxb_re_run, float64
 * plans only.  No counterpart in the reference's code (JAX would give it with jax.jvp).
 * The state planes and their tangents (every plane of both structs set) advance together:
 * values bit for bit as the float64 run, tangents by the chain rule through the step
 * including the state dependence of dt through the fastest face.  The stage runs the
 * general path's kernels on dual numbers (any boundary layout); the plan allocates its
 * dual planes on the first call.  Parameter tangents (may be NULL, or have NULL members):
 * seds_dot, 7 x nsed like pxb_re_config.seds (the MPM constants follow); values0_dot, one
 * per handler in plan order, the tangent of values[0] of ConstantInflux handlers (the
 * discharge; its momenta are q * values[1], q * values[2]).  dt_log / dt_dot_log: device
 * float64 arrays of nsteps values / tangents of dt, or NULL. */
typedef struct pxb_re_tangent_params {
    const double* seds_dot;
    const double* values0_dot;
} pxb_re_tangent_params;
int pxb_re_jvp_init(pxb_re_plan* plan, const pxb_re_fields* f, const pxb_re_fields* f_dot,
                    const pxb_re_tangent_params* params_dot, void* stream);
int pxb_re_jvp_run(pxb_re_plan* plan, const pxb_re_fields* a, const pxb_re_fields* a_dot, int32_t nsteps,
                   int32_t scheme, double cfl, double t0, const pxb_re_tangent_params* params_dot, void* dt_log,
                   void* dt_dot_log, void* stream);

/* Reverse mode (adjoint), float64 plans.  No counterpart in the reference's code (JAX
 * would give it with jax.vjp over a fixed-length loop).  pxb_re_vjp_run: `a0` is the state
 * after init (not modified); `abar` holds the adjoint of the state after nsteps steps
 * (dJ/du for h, hu, hv, z_b, G) and receives the adjoint of a0.  The steps are redone
 * forward with a checkpoint every `checkpoint_every` steps (0: 32) and undone segment by
 * segment: each stage backwards (handlers, Exner update, grass factor, corrections, hydro
 * update), with local Jacobians of the faces from multi-tangent dual numbers, and the
 * dependence of dt on the state through the fastest face.  pxb_re_vjp_init: `f` is the
 * state BEFORE init; `fbar` (in: adjoint after init, out: before) goes back through the
 * handlers and the grass factor.  Handlers of every kind but ConstantOutflux.  Allocates
 * its checkpoints for the call; synchronises `stream`. */
int pxb_re_vjp_init(pxb_re_plan* plan, const pxb_re_fields* f, const pxb_re_fields* fbar, void* stream);
int pxb_re_vjp_run(pxb_re_plan* plan, const pxb_re_fields* a0, int32_t nsteps, int32_t scheme, double cfl, double t0,
                   int32_t checkpoint_every, const pxb_re_fields* abar, void* stream);

/* Adjoints of the scalar parameters, the reverse-mode counterparts of
 * pxb_re_tangent_params (host arrays, ADDED to; either may be NULL):
 *   seds_bar[7 * nsed]   dJ/d(sediment matrix) of pnetcdf_reader.py:136-158 (row 1: the
 *                        grain diameter d50) through the MPM grass factor (roe_exner.py:85-130)
 *                        of every stage and the init, and through n_b = n_p_mix of compute_n
 *                        (roe_exner.py:64-73) in the friction of every Roe face; one sediment
 *                        class (PXB_ERR_UNSUPPORTED otherwise);
 *   values0_bar[nh]      dJ/d(values[0]) of each ConstantInflux handler (plan order), the
 *                        discharge of roeexner_constantinflux.py:29-30 (0 for other kinds).
 * pxb_re_vjp_run_params: as pxb_re_vjp_run; with seds_bar set, abar->n_b (when not NULL;
 * in: dJ/dn_b of the final state, n_b being constant) receives dJ/dn_b of a0.
 * pxb_re_vjp_init_params: as pxb_re_vjp_init; with seds_bar set, fbar->n_b (in: dJ/dn_b
 * after init) goes through compute_n to fbar->n (when set) and to the matrix, and leaves
 * zero.  The parameter sums use atomics, so their last bits can vary between runs. */
typedef struct pxb_re_param_adjoints {
    double* seds_bar;
    double* values0_bar;
} pxb_re_param_adjoints;
int pxb_re_vjp_init_params(pxb_re_plan* plan, const pxb_re_fields* f, const pxb_re_fields* fbar,
                           const pxb_re_param_adjoints* pbar, void* stream);
int pxb_re_vjp_run_params(pxb_re_plan* plan, const pxb_re_fields* a0, int32_t nsteps, int32_t scheme, double cfl,
                          double t0, int32_t checkpoint_every, const pxb_re_fields* abar,
                          const pxb_re_param_adjoints* pbar, void* stream);

/* Device error word of the plan (non-finite dt or state seen by a kernel): reads it
 * (synchronising `stream`), clears it, returns PXB_OK or PXB_ERR_NONFINITE. */
int pxb_re_check(pxb_re_plan* plan, void* stream);

/* --- plain Roe -------------------------------------------------------------------- */
typedef struct pxb_roe_config {
    int32_t ny, nx;
    int64_t pitch;
    int32_t dtype;
    double dx;
    const pxb_bc_handler* handlers;
    int32_t nhandlers;
} pxb_roe_config;

int pxb_roe_plan_create(const pxb_roe_config* cfg, pxb_roe_plan** out);
int pxb_roe_plan_destroy(pxb_roe_plan* plan);
/* compute_dt_roe (roe_solver.py:56-60, roe.py:13-30): cfl * min over all cells, no floor. */
int pxb_roe_cfl(pxb_roe_plan* plan, const pxb_roe_fields* f, double cfl, void* dt_dev, void* stream);
/* step_fn_roe (roe_solver.py:40-54); avg as in pxb_re_stage (h, hu, hv, z, n). */
int pxb_roe_stage(pxb_roe_plan* plan, const pxb_roe_fields* in, const pxb_roe_fields* out,
                  const pxb_roe_fields* avg, const void* dt_dev, void* stream);
int pxb_roe_run(pxb_roe_plan* plan, const pxb_roe_fields* a, const pxb_roe_fields* b, int32_t nsteps,
                int32_t scheme, double cfl, void* dt_log, void* stream);
int pxb_roe_check(pxb_roe_plan* plan, void* stream);

/* --- ragged ensembles ---------------------------------------------------------------- */
/* No counterpart in the reference (it runs one grid per process).  Many independent
 * Roe-Exner grids of different sizes advance together: each member has its own state,
 * boundary handlers and dt (as a separate run of forwardeuler.py:37-49 / SSPRK2.py:30-51
 * for a fixed step count would), and every phase is one launch for all members (CFL,
 * stage 1, stage 2), the steps captured into a CUDA graph.  Members run the fused stage
 * kernel, so their layouts must be ones it accepts (PXB_ERR_UNSUPPORTED otherwise).
 * All members share dtype, the grass-factor mode and the sediment table. */
typedef struct pxb_re_member {
    int32_t ny, nx;
    int64_t pitch;
    double dx;
    pxb_re_fields a;                 /* state, advanced in place                        */
    pxb_re_fields b;                 /* scratch state of the same layout (h, hu, hv, z_b, G) */
    const uint8_t* nodata;           /* device mask[0] plane or NULL                    */
    const pxb_bc_handler* handlers;  /* host array, YAML order                          */
    int32_t nhandlers;
} pxb_re_member;

typedef struct pxb_re_ens_config {
    int32_t dtype;
    int32_t mpm;
    const double* seds;              /* 7 x nsed, as pxb_re_config                      */
    int32_t nsed;
    const pxb_re_member* members;    /* host array                                      */
    int32_t nmembers;
    int32_t band_rows;               /* rows per band for every member; 0 = default     */
} pxb_re_ens_config;

typedef struct pxb_re_ens pxb_re_ens;

int pxb_re_ens_create(const pxb_re_ens_config* cfg, pxb_re_ens** out);
int pxb_re_ens_destroy(pxb_re_ens* ens);
/* init_fn_roeexner on every member's state a. */
int pxb_re_ens_init(pxb_re_ens* ens, void* stream);
/* Times the ensemble stage kernel for a set of band heights on the current states
 * (stage 1 from a into b; the states a are left unchanged), keeps the fastest and
 * returns it in *band_rows (may be NULL).  Synchronises `stream`. */
int pxb_re_ens_autotune(pxb_re_ens* ens, void* stream, int32_t* band_rows);
/* nsteps steps of every member (scheme PXB_FE / PXB_SSPRK2), states start and end in a.
 * dt_log: device array of nsteps x nmembers dts (member index fastest) or NULL. */
int pxb_re_ens_run(pxb_re_ens* ens, int32_t nsteps, int32_t scheme, double cfl, void* dt_log, void* stream);
/* Reads and clears the members' error words; *first_bad is the first member that saw a
 * non-finite dt or state (-1 if none).  Returns PXB_OK or PXB_ERR_NONFINITE. */
int pxb_re_ens_check(pxb_re_ens* ens, void* stream, int32_t* first_bad);

/* --- allocation-free time step ----------------------------------------------------- */
/* No counterpart in the reference: PyExner's JAX step never manages device memory
 * itself.  For callers that cannot allocate device memory when they need dt -- an XLA
 * custom call, which must work inside the buffers XLA has already allocated; a host
 * application whose policy forbids cudaMalloc after start-up.  Same result as
 * pxb_re_cfl, without a plan: dt = max(cfl * min over active faces of dx / speed, 1e-6),
 * written to dt_dev (one element of dtype).  nodata may be NULL.  Calls no
 * cudaMalloc/cudaFree: the reduction scratch is a fixed array of (8192 + 32) * 8 bytes in
 * device memory owned by the library, resident on every device that loads it until the
 * process exits.  Grids up to 31 * 8192 = 253952 columns wide (any height); wider grids
 * return PXB_ERR_ARG.  The first call on a device (and the first after cudaDeviceReset)
 * looks up the array's device address; make that first call before any stream capture.
 * All calls share the array: calls whose kernels can overlap on the GPU (unordered
 * streams, or several host threads on one device) race and must be serialised by the
 * caller. */
int pxb_re_cfl_noalloc(int32_t ny, int32_t nx, int64_t pitch, int32_t dtype, double dx, double cfl,
                       const void* h, const void* hu, const void* hv, const void* G, const uint8_t* nodata,
                       void* dt_dev, void* stream);

/* --- boundary set-up on the device ------------------------------------------------- */
/* The polygon labelling of BoundaryManager (boundary_registry.py:19-59) and the
 * raster-order cell lists its index maps start from (:61-82), for large grids.  Cell
 * centres are the outer product of xc[nx] (x of each column) and yc[ny] (y of each row),
 * host arrays; verts: host array npoly x nverts x 2 (x, y), each polygon zero-padded to
 * nverts as the reference pads it.  counts[npoly] (host) receives the number of cells
 * inside each polygon (even-odd rule, 1e-8 tolerance on the crossing abscissa); when
 * `cells` is not NULL it receives, polygon after polygon, the flat indices row*nx + col
 * of those cells in raster order (capacity cells_cap; PXB_ERR_ARG if too small, counts
 * still filled).  Allocates device scratch for the call; synchronises `stream`. */
int pxb_label_polygons(int32_t ny, int32_t nx, const double* xc, const double* yc, const double* verts,
                       int32_t npoly, int32_t nverts, int64_t* counts, int64_t* cells, int64_t cells_cap,
                       void* stream);

/* --- misc ------------------------------------------------------------------------- */
const char* pxb_last_error(void);
int pxb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PYEXNER_B200_H */
