/* xfp.h -- C ABI of the B200-native pressure projection (libxfp.so).
 *
 * Drop-in for xFluid's VariationalPressureSolver
 * (xFluid/xFluid/variationalpressure/variational_pressuresolver.h:30-44): the
 * same method -- the variational MAC-grid Poisson matrix, MIC(0)-preconditioned
 * CG in natural (lexicographic) order, and the pressure-gradient velocity
 * update -- computed by hand-written sm_100a CUDA kernels.
 *
 * Grid layout is xFluid's Array3d (xFluid/xFluid/array3d.h:143-146): flat index
 * k*ni*nj + j*ni + i.  Face arrays follow xFluid/xFluid/FluidSimulator.h:177-181:
 * u is (ni+1, nj, nk), v is (ni, nj+1, nk), w is (ni, nj, nk+1), each flattened
 * the same way with its own extents.  material holds xFluid's Material values
 * (xFluid/xFluid/material.h:4-8): 0 air, 1 fluid, 2 solid.
 *
 * Optional face weights wu/wv/ww (same shapes as u/v/w, values in [0,1]) are
 * open fractions that scale every face's contribution (fractional solids).
 * Pass NULL for all three to get exactly xFluid's matrix.
 *
 * Pointers are host memory unless xfp_options.device_pointers is set, in which
 * case they must be device memory on the context's device.  Calls on one
 * context are not re-entrant; use one context per host thread (each context
 * owns its stream and its scratch memory).
 *
 * Return codes: XFP_OK, XFP_NOT_CONVERGED (the last iterate is still written;
 * xFluid instead leaves the pressure grid unsized and applies it anyway,
 * variational_pressuresolver.cpp:80-86 with FluidSimulator.cpp:506-508), or a
 * negative XFP_ERR_* code; xfp_last_error() gives the message.
 */
#ifndef XFP_H
#define XFP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XFP_OK 0
#define XFP_NOT_CONVERGED 1
#define XFP_ERR_ARGS (-1)
#define XFP_ERR_CUDA (-2)
#define XFP_ERR_TIMEOUT (-3)
#define XFP_ERR_NOMEM (-4)
#define XFP_ERR_BREAKDOWN (-5)
#define XFP_ERR_UNSUPPORTED (-6)

/* Arithmetic used inside the solve (independent of the I/O type). */
#define XFP_PREC_F64 0   /* FP64 throughout, operation order of xFluid's solver */
#define XFP_PREC_F32 1   /* plain FP32: stencil, vectors, dots and factor in FP32 */
#define XFP_PREC_MIXED 2 /* FP32 stencil/vectors; FP64 dots, MIC(0) pivots and
                            iterative-refinement residual */

/* Pressure matrix (xfp_options.matrix).
 * VARIATIONAL: VariationalPressureSolver's (variational_pressuresolver.cpp:231-327), with optional face weights.
 * NORMAL: NormalPressureSolver's classic Poisson matrix (pressuresolver.cpp:220-347) -- diagonal = in-range
 *   non-solid neighbours, -1 to fluid neighbours, fluid rows only -- and its applyPressure (:109-212).  Face
 *   weights must be NULL; the batch and backward entry points return XFP_ERR_UNSUPPORTED for it. */
#define XFP_MATRIX_VARIATIONAL 0
#define XFP_MATRIX_NORMAL 1

typedef struct xfp_ctx xfp_ctx;

typedef struct xfp_options {
  double tol;            /* stop when |r|_inf <= tol*|b|_inf (pcg_solver.h:249-254,273) */
  int max_iter;          /* PCG iteration cap (pcg_solver.h:231 default 100) */
  double omega;          /* MIC(0) modification parameter (pcg_solver.h:87, 0.97) */
  double min_diag_ratio; /* MIC(0) pivot safeguard (pcg_solver.h:87, 0.25) */
  int precision;         /* XFP_PREC_* */
  int device_pointers;   /* 1: array arguments are device pointers */
  int device;            /* CUDA device ordinal */
  int check_every;       /* PCG iterations per host convergence read (0: 8) */
  double timeout_ms;     /* bound on any device-side wait (0: 2000 ms) */
  int max_refine;        /* mixed: iterative-refinement cycles (0: 20) */
  double inner_tol;      /* mixed: relative residual reduction per cycle (0: 1e-4) */
  int tile_k;            /* sweep tile height in k-lines: 8, 15 or 16; 0: timed on the first call per grid (or batch) shape and cached */
  void* stream;          /* cudaStream_t to run on; NULL: the context's own stream */
  int matrix;            /* XFP_MATRIX_*: which pressure matrix the solve/project/apply entry points use */
} xfp_options;

typedef struct xfp_stats {
  int status;            /* same as the return code */
  int iterations;        /* PCG iterations (summed over refinement cycles) */
  int refinements;       /* mixed precision: refinement cycles run */
  double residual;       /* final |b - A p|_inf (recursive residual for F64/F32) */
  double rel_residual;   /* residual / |b|_inf */
  double b_inf;          /* |b|_inf */
  long long rows;        /* unknown rows: fluid cells + solid cells next to fluid */
  long long stored;      /* cells in the line-compacted storage (rows + padding) */
  long long lines;       /* active x-lines */
  double ms_setup;       /* layout + assembly */
  double ms_factor;      /* MIC(0) factorisation */
  double ms_solve;       /* PCG */
  double ms_apply;       /* pressure scatter + velocity update */
  double ms_total;       /* whole call incl. host<->device copies */
  double bytes;          /* algorithmic bytes moved by the device kernels */
  double ms_sweeps;      /* device time of the timed MIC(0) triangular-solve sweeps (CUDA events on
                            the forward and backward solve of every N-th PCG iteration, with the
                            environment variable XFP_KERNEL_EVENTS=N at context creation; by
                            default none are timed and this is 0: an event between two launches
                            serialises them) */
  int sweeps;            /* triangular-solve sweep launches timed in ms_sweeps */
  long long launches;    /* device kernels launched by this call */
  int tile_k;            /* sweep tile height the call used (k-lines) */
  int graph;             /* 1: the PCG iterations ran as a CUDA graph; 0: launched one by one */
  double ms_vec[3];      /* device time of the PCG loop's vector kernels (CUDA events, sampled as
                            ms_sweeps is): SpMV + dot,
                            x/r update, s update -- launches after convergence excluded */
  int vec_launches[3];   /* launches timed in ms_vec, per kernel */
  long long h2d_bytes;   /* host-pointer mode: bytes this call moved host -> device */
  long long d2h_bytes;   /* host-pointer mode: bytes this call moved device -> host */
  int host_faces;        /* 1: only the faces that border fluid crossed PCIe (page-locked
                            velocity arrays, read and written in place); 0: whole arrays
                            were copied, or device pointers */
} xfp_stats;

/* Fills opt with defaults: tol 1e-5, max_iter 100, omega 0.97, ratio 0.25 --
 * PCGSolver's constructor defaults (pcg_solver.h:229-232) -- FP64, host
 * pointers, device 0. */
void xfp_default_options(xfp_options* opt);

/* Creates a context (device, stream, scratch pool).  Replaces constructing
 * VariationalPressureSolver (variational_pressuresolver.cpp:8-9). */
int xfp_create(xfp_ctx** ctx, const xfp_options* opt);
int xfp_destroy(xfp_ctx* ctx);
int xfp_set_options(xfp_ctx* ctx, const xfp_options* opt);
const char* xfp_last_error(const xfp_ctx* ctx);
const char* xfp_version(void);

/* Solve for pressure.  Replaces VariationalPressureSolver::solve
 * (variational_pressuresolver.cpp:50-118, with setSize/setVelocityField/
 * setMaterial at :11-28): assembles the variational system (:231-327), runs
 * MIC(0)-PCG (pcg_solver.h:243-285) and writes pressure for every cell
 * (0 in rows without an unknown, :86-101).  pressure is ni*nj*nk. */
int xfp_solve_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                  const double* u, const double* v, const double* w,
                  const double* wu, const double* wv, const double* ww,
                  double* pressure, xfp_stats* stats);
int xfp_solve_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                  const float* u, const float* v, const float* w,
                  const float* wu, const float* wv, const float* ww,
                  float* pressure, xfp_stats* stats);

/* Pressure-gradient update of u, v, w in place.  Replaces
 * VariationalPressureSolver::applyPressure (variational_pressuresolver.cpp:120-220). */
int xfp_apply_pressure_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                           const double* wu, const double* wv, const double* ww,
                           const double* pressure, double* u, double* v, double* w);
int xfp_apply_pressure_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                           const float* wu, const float* wv, const float* ww,
                           const float* pressure, float* u, float* v, float* w);

/* Solve and apply in one call, u/v/w updated in place: the pair
 * FluidSimulator::_solvePressure issues (FluidSimulator.cpp:501-509).
 * pressure may be NULL. */
int xfp_project_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                    double* u, double* v, double* w, const double* wu, const double* wv,
                    const double* ww, double* pressure, xfp_stats* stats);
int xfp_project_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                    float* u, float* v, float* w, const float* wu, const float* wv,
                    const float* ww, float* pressure, xfp_stats* stats);

/* Adjoint of the projection u_out = u - G A^{-1} D u (no reference
 * counterpart; xFluid is not differentiable).  Given g = dL/du_out (gu,gv,gw)
 * writes dL/du_in = g - D^T A^{-1} G^T g into (du,dv,dw): a second MIC(0)-PCG
 * solve with the same matrix plus the transposed gradient and divergence
 * kernels.  Outputs may alias inputs. */
int xfp_project_backward_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                             const double* wu, const double* wv, const double* ww,
                             const double* gu, const double* gv, const double* gw,
                             double* du, double* dv, double* dw, xfp_stats* stats);
int xfp_project_backward_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                             const float* wu, const float* wv, const float* ww,
                             const float* gu, const float* gv, const float* gw,
                             float* du, float* dv, float* dw, xfp_stats* stats);

/* One scene of a batch.  Arrays have the shapes and layout described at the top
 * of this header; the element type is float for xfp_project_batch_f32 and
 * double for xfp_project_batch_f64.  u, v, w are updated in place; wu/wv/ww
 * are optional (all three or none); pressure is optional output. */
typedef struct xfp_scene {
  int ni, nj, nk;
  const uint8_t* material;
  void* u;
  void* v;
  void* w;
  const void* wu;
  const void* wv;
  const void* ww;
  void* pressure;
} xfp_scene;

/* Projects n independent scenes of (possibly) different sizes together: each
 * scene is solved exactly as xfp_project_* solves it alone (its own
 * tolerance test, iteration count and PCG scalars), but the MIC(0) sweeps of
 * all scenes run in one persistent launch and the PCG iteration is replayed
 * as a CUDA graph.  No reference counterpart: xFluid projects one grid per
 * call (FluidSimulator.cpp:501-509).  With options.tile_k == 0 the sweep tile
 * height is picked per batch shape by timing the candidate heights on the
 * first call (cached in the context).  stats, if not NULL, receives n entries.  Returns
 * XFP_OK when every scene converged, XFP_NOT_CONVERGED when one did not. */
int xfp_project_batch_f32(xfp_ctx* ctx, int n, const xfp_scene* scenes, xfp_stats* stats);
int xfp_project_batch_f64(xfp_ctx* ctx, int n, const xfp_scene* scenes, xfp_stats* stats);

/* Differentiable rollouts (advect -> project, repeated; no reference
 * counterpart: xFluid moves velocity with particles, FluidSimulator.cpp:652-1085).
 * Semi-Lagrangian self-advection of the MAC velocity: each face value is
 * re-sampled (trilinear, lattice coordinates clamped to the grid) at its
 * departure point x_f - dt_over_dx * vel(x_f), vel sampled from u, v, w at
 * the face.  The backward form writes the exact adjoint (both the sampling
 * weights and the departure point's dependence on the velocity) of that map
 * at state (u,v,w): (du,dv,dw) = J^T (gu,gv,gw).  The box loss is the sum of
 * squared face values whose unit-cube position ((i,j+.5,k+.5)/(ni,nj,nk) for
 * u, etc.) lies in box = {x0,x1,y0,y1,z0,z1}; its gradient (2*value inside,
 * 0 outside) is written when gu/gv/gw are given; loss is a host double.
 * These entry points take device arrays only (options.device_pointers = 1);
 * box is host memory. */
int xfp_advect_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v,
                   const double* w, double* ou, double* ov, double* ow, double dt_over_dx);
int xfp_advect_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v,
                   const float* w, float* ou, float* ov, float* ow, double dt_over_dx);
int xfp_advect_backward_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v,
                            const double* w, const double* gu, const double* gv, const double* gw,
                            double* du, double* dv, double* dw, double dt_over_dx);
int xfp_advect_backward_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v,
                            const float* w, const float* gu, const float* gv, const float* gw,
                            float* du, float* dv, float* dw, double dt_over_dx);
int xfp_box_loss_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v,
                     const double* w, const double* box, double* loss, double* gu, double* gv,
                     double* gw);
int xfp_box_loss_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v,
                     const float* w, const double* box, double* loss, float* gu, float* gv, float* gw);

/* Failure-path diagnostic (no reference counterpart): the next MIC(0) sweep
 * launched on this context waits, at every tile hand-off, for a boundary word
 * that no producer writes.  Every such wait is bounded (options.timeout_ms):
 * the first to run out records where it gave up and raises the context's
 * error flag, every other wait then returns within a few hundred polls, and
 * the call returns XFP_ERR_TIMEOUT with the site in xfp_last_error().  The
 * context stays usable; nothing faults.  Needs a grid with more than one
 * sweep tile.  Used by the tests of the timeout path. */
int xfp_debug_expire_next_sweep(xfp_ctx* ctx);

/* ---- The simulator steps either side of the projection ----
 * FluidSimulator::timeStep applies the body forces (FluidSimulator.cpp:310), solves and
 * applies the pressure (:501-509) and then extrapolates the velocities (:322).
 *
 * xfp_apply_forces_*: FluidSimulator::_applyForces (FluidSimulator.cpp:429-499).  force is
 * the summed constant force (the sum of _forces); every face with a fluid cell on either side
 * gets force*dt, an axis with |force*dt| <= 1e-10 none.  u,v,w in place.
 * xfp_extrapolate_*: FluidSimulator::_expolateVelocity(layers, axis) for the three axes
 * (:521-650): layer by layer outward from the faces of fluid cells, each face of a layer takes
 * the average of its neighbours in the layer before.  The reference passes
 * layers = (int)(CFL number + 5) (:513).  0 <= layers <= 30000.  u,v,w in place.
 * xfp_project_step_*: both around one projection, in the reference's order: the force
 * enters inside the assembly and apply kernels (no separate pass over the velocities), then
 * the projection of xfp_project_*, then `layers` extrapolation layers on the projected
 * velocities (0: none).  Arrays as for xfp_project_*; pressure may be NULL. */
int xfp_apply_forces_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                         double* w, const double force[3], double dt);
int xfp_apply_forces_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                         float* w, const double force[3], double dt);
int xfp_extrapolate_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                        double* w, int layers);
int xfp_extrapolate_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                        float* w, int layers);
int xfp_project_step_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                         double* w, const double* wu, const double* wv, const double* ww, double* pressure,
                         const double force[3], double dt, int layers, xfp_stats* stats);
int xfp_project_step_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                         float* w, const float* wu, const float* wv, const float* ww, float* pressure,
                         const double force[3], double dt, int layers, xfp_stats* stats);

/* The reference solver's divergence diagnostic, VariationalPressureSolver::
 * _calculate_divergience (variationalpressure/variational_pressuresolver.cpp:
 * 526-597): for every fluid cell, +u(i)-u(i+1)+v(j)-v(j+1)+w(k)-w(k+1) over the
 * faces whose neighbour cell is not solid (outside the grid counts as solid),
 * unit weights; 0 for other cells.  div is ni*nj*nk in the cell layout.  The
 * projection zeroes the weighted form of this quantity (solid faces at 0.5),
 * which equals b - A p; this is the reference's unweighted diagnostic.  FP64
 * results are bit-identical to the reference. */
int xfp_divergence_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* u,
                       const double* v, const double* w, double* div);
int xfp_divergence_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const float* u,
                       const float* v, const float* w, float* div);

/* ---- Particle steps (FLIP/PIC) around the projection ----
 * One particle is xFluid's struct Particle {Vec3d p; Vec3d v;} (particle.h:5-15):
 * position then velocity, six doubles, so a std::vector<Particle>'s data()
 * is passed as it is.  Positions are in the simulator's units (cell width dx,
 * grid origin 0).  Grids, material and pointers follow the projection's rules
 * (host arrays, or device arrays with options.device_pointers).  All FP64.
 *
 * xfp_advect_particles_f64 replaces FluidSimulator::_advectParticles steps
 *   a-b (FluidSimulator.cpp:652-723): each particle's velocity becomes
 *   (1-ratio) PIC + ratio FLIP from the current faces (u,v,w) and those saved
 *   before the forces (_saveVelocity, :1095-1100); the particle moves by RK4
 *   through (u,v,w) over dt (:895-906), and a particle that would enter a solid
 *   cell is resolved as the reference does (collision.cpp:293-440).  As in the
 *   reference, whose six worker chunks of n/6 skip the remainder, the last
 *   n mod 6 particles are left unchanged.  Bit-identical to the reference,
 *   except where it reads outside its arrays: a collision point in a cell
 *   outside the grid leaves the particle in place.
 * xfp_particles_to_grid_f64 replaces _updateVelocityByParticles (:909-1085):
 *   every face of u,v,w becomes the kernel-weighted mean of the particles'
 *   velocity component (radius 1.5 dx), or 0 where the weight is <= 1e-7.
 *   The same contributions as the reference, summed in a fixed order other
 *   than its particle order: equal to FP64 rounding.
 * xfp_update_material replaces _updateMaterial (:402-427): non-solid cells
 *   become air, then every cell holding a particle becomes fluid.  Bit-identical.
 * xfp_distance_field_f64 replaces DirectedDistanceField::updateFeild
 *   (directeddistancefield.cpp:122-165): phi on the (ni*subdiv+1) x
 *   (nj*subdiv+1) x (nk*subdiv+1) vertex grid (may be NULL when only the
 *   material is wanted), and, when material is given, the material part of
 *   updateSurfaceInfo (:167-215): non-solid cells classified fluid or air by
 *   phi >= threshold.  phi equals the reference's to FP64 rounding (summation
 *   order); the classification follows phi exactly.  FluidSimulator uses
 *   subdiv 2, radius 3x its particle radius, threshold 0.4 (:207-213). */
typedef struct {
  double p[3];
  double v[3];
} xfp_particle;

int xfp_advect_particles_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, const uint8_t* material,
                             const double* u, const double* v, const double* w, const double* u_saved,
                             const double* v_saved, const double* w_saved, double ratio_flip, double dt,
                             long long n, xfp_particle* particles);
int xfp_particles_to_grid_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n,
                              const xfp_particle* particles, double* u, double* v, double* w);
/* Replaces FluidSimulator::_maxVelocity (FluidSimulator.cpp:387-400), the
 * speed frameStep divides the CFL distance by to pick each substep's dt
 * (:228-241): the square root of the largest v.v over the particles, v.v
 * rounded as the reference forms it (array3d.h:33-36), so the result -- and
 * the dt -- are the reference's bits.  0 for no particles.  Synchronous. */
int xfp_max_speed_f64(xfp_ctx* ctx, long long n, const xfp_particle* particles, double* max_speed);
int xfp_update_material(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n,
                        const xfp_particle* particles, uint8_t* material);
int xfp_distance_field_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, int subdiv, double radius,
                           double threshold, long long n, const xfp_particle* particles, double* phi,
                           uint8_t* material);

/* Diagnostics: runs the internal stages on one scene and returns them on the
 * dense grid (ni*nj*nk doubles each; any output may be NULL), in the
 * context's precision.  Exposes, for verification against the reference:
 *   diag/ax/ay/az/b  _calculate_coefficient (variational_pressuresolver.cpp:231-327);
 *                    ax[c]=A(c,c-1), ay[c]=A(c,c-ni), az[c]=A(c,c-ni*nj)
 *   inv/lx/ly/lz     factor_modified_incomplete_cholesky0 (pcg_solver.h:85-186);
 *                    lx[c]=L(c,c-1) etc.
 *   y = L^{-1} r     solve_lower (pcg_solver.h:192-204)
 *   z = M^{-1} r     solve_lower + solve_lower_transpose_in_place (pcg_solver.h:192-220)
 *   q = A r          multiply(FixedSparseMatrix) (sparse_matrix.h:264-276)
 * r is a dense input (rows without an unknown are ignored). */
int xfp_debug_stages(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material,
                     const double* u, const double* v, const double* w,
                     const double* wu, const double* wv, const double* ww,
                     const double* r, double* diag, double* ax, double* ay, double* az,
                     double* b, double* inv, double* lx, double* ly, double* lz,
                     double* y, double* z, double* q);

/* |b|_inf of the pressure system's right-hand side, computed without
 * allocating any device memory.  This entry point has no counterpart in the
 * reference.  It is for callers that must not call cudaMalloc/cudaFree: a
 * real-time loop that cannot afford cudaFree's device-wide synchronisation, or
 * an application whose own allocator has reserved the device's memory.  No
 * context is needed.
 *
 * b is the variational matrix's right-hand side with no body force: the value
 * equals, bit for bit, stats.b_inf of an FP64 solve or projection with
 * options.matrix = XFP_MATRIX_VARIATIONAL (xfp_solve_f64, xfp_project_f64).
 * It differs from the b of an XFP_MATRIX_NORMAL solve (which drops solid rows
 * and solid faces) and of xfp_project_step_* (which adds force*dt first).  A
 * NaN in the inputs that reaches b gives a NaN result.
 *
 * All arrays, including the output b_inf (one double), are device (or managed)
 * memory on the current device; host pointers are rejected.  The kernel runs
 * asynchronously on `stream` (NULL: the default stream); *b_inf is ready when
 * the stream's work completes.  Its only scratch is one fixed 128 KiB
 * __device__ array per GPU (held from the moment the library's device code is
 * loaded on that GPU until the process exits), so grids above 268,435,456
 * cells are rejected with XFP_ERR_ARGS.  Calls share that array: calls whose
 * kernels may overlap on the GPU (different streams or threads) race and must
 * be serialised by the caller.  Every call looks up the array's address in the
 * current context (so a context re-created by cudaDeviceReset is handled); the
 * first call on a device also loads the library's device code there, so make
 * that first call before any stream capture begins.  On error a message goes
 * to err (up to err_len bytes, may be NULL). */
int xfp_rhs_inf_noalloc_f64(int ni, int nj, int nk, const uint8_t* material,
                            const double* u, const double* v, const double* w,
                            const double* wu, const double* wv, const double* ww,
                            double* b_inf, void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* XFP_H */
