/* dgp -- B200-native explicit DG right-hand side and SSP-RK3 stepping.
 *
 * C ABI of libdgp.so.  Every function returns an int status (DGP_OK = 0,
 * negative on error; dgp_last_error() gives the message of the calling
 * thread's last failure).  Handles are opaque; one host thread per solver
 * handle; each solver owns one CUDA stream on the device that was current when
 * it was created.  State arrays crossing the ABI are FP64 in DG-Parallel's
 * layout: [cell][field][mode], cells in the order of the cell elements in the
 * mesh file (or of the `cells` array passed to dgp_mesh_from_arrays).
 *
 * Each entry point names the DG-Parallel interface it replaces.
 */
#ifndef DGP_H
#define DGP_H
#ifdef __cplusplus
extern "C" {
#endif

#define DGP_OK 0
#define DGP_ERR_INVALID (-1)     /* bad argument or handle */
#define DGP_ERR_IO (-2)          /* mesh file missing or malformed */
#define DGP_ERR_UNSUPPORTED (-3) /* law/flux/order/element combination not built */
#define DGP_ERR_CUDA (-4)        /* CUDA runtime error (message in dgp_last_error) */
#define DGP_ERR_NONPHYSICAL (-5) /* a stage produced a non-physical state */
#define DGP_ERR_NOMEM (-6)

/* conservation laws (ConservationLaw subclasses, ConservationLaw.h:12-60) */
#define DGP_LAW_SCALAR 0    /* ScalarLaw (ScalarLaw.cc), constant velocity field */
#define DGP_LAW_BURGERS2D 1 /* Burgers2D (Burgers2D.cc) */
#define DGP_LAW_EULER2D 2   /* Euler2d / Euler2dRoe (EulerLaw.cc) */
#define DGP_LAW_EULER3D 3   /* Euler3d (EulerLaw.cc) */
#define DGP_LAW_MAXWELL3D 4 /* 3D Maxwell on tets (no counterpart; Maxwell2d is 2D only) */
#define DGP_LAW_MAXWELL2D 5 /* Maxwell2d (MaxwellLaw.cc): fields Hx, Hy, Ez; its riemannSolver
                             * (MaxwellLaw.cc:137-195) whatever flux id is given */

/* numerical fluxes (ConservationLaw::riemannSolver overrides) */
#define DGP_FLUX_UPWIND 0  /* ScalarLaw::riemannSolver, Maxwell upwind */
#define DGP_FLUX_CENTRAL 1 /* Burgers2D::riemannSolver (maxIV = 0) */
#define DGP_FLUX_GODUNOV 2 /* Euler2d/Euler3d::riemannSolver: exact Riemann solver */
#define DGP_FLUX_ROE 3     /* Euler2dRoe::riemannSolver */
#define DGP_FLUX_LLF 4     /* local Lax-Friedrichs (no counterpart in DG-Parallel) */

/* analytic FieldEvaluator functors (FieldEvaluator.h:9-15) used as initial
 * condition, far field (ConservationLaw::getFarField) and exact solution.  A
 * host callback cannot run per GPU quadrature point, so evaluators are chosen
 * by id with parameters. */
#define DGP_FIELD_GAUSS 0   /* exp(-|x - c - a t|^2 / s), 2D */
#define DGP_FIELD_VORTEX 1  /* isentropic vortex, free stream (1,1,1,1), moving (1,1) */
#define DGP_FIELD_PULSE3D 2 /* Euler3d density pulse advected by velocity a, p = 1 */
#define DGP_FIELD_SINE 3    /* 0.5 + A sin(2 pi (x + y)) */
#define DGP_FIELD_GAUSS3D 4 /* exp(-|x - c - a t|^2 / s), 3D */
#define DGP_FIELD_TM110 5   /* TM110 mode of the PEC cube [0,L]^3 */
#define DGP_FIELD_TM2D 6    /* (Hx, Hy, Ez) of the mode Ez = sin(pi x/L) sin(pi y/L) cos(w t),
                             * w = pi sqrt(2)/L, of Maxwell2d's equations on [0,L]^2 */

/* law / field parameters: double[16]
 *  [0..2] advection velocity a   [3..5] centre c   [6] width s
 *  [7] gamma (default 1.4)       [8] vortex strength beta
 *  [9] amplitude A               [10] cavity side L */
#define DGP_NPARAMS 16

/* boundary conditions by classification id (ConservationLaw::boundaryFlux's
 * dispatch on BoundaryId, ConservationLaw.h:31-40; EulerLaw.cc:280-295,
 * MaxwellLaw.cc:113-131): */
#define DGP_BC_DEFAULT 0  /* the law's own rule for the id (40000 a wall, other ids the far field) */
#define DGP_BC_FARFIELD 1 /* the law's field through its boundary / Riemann flux */
#define DGP_BC_WALL 2     /* the law's wall: Euler slip mirror state, Maxwell2d reflection,
                           * Maxwell3d perfect conductor (not defined for the scalar laws) */
#define DGP_MAX_BC 8      /* ids a law can remap */

#define DGP_PRECISION_FP64 0  /* plain FP64 drop-in form */
#define DGP_PRECISION_MIXED 1 /* FP32 bulk arithmetic, FP64 geometry/totals/time */

#define DGP_RULE_REFERENCE 0
#define DGP_RULE_WORKLOAD 1
#define DGP_LIMITER_NONE 0
#define DGP_LIMITER_MOMENT 1
#define DGP_LIMITER_BARTH 2

typedef struct dgp_mesh_s* dgp_mesh;
typedef struct dgp_law_s* dgp_law;
typedef struct dgp_solver_s* dgp_solver;
typedef struct dgp_ensemble_s* dgp_ensemble;
typedef struct dgp_probe_s* dgp_probe;

const char* dgp_last_error(void);
int dgp_version(void);
/* the CUDA device of the calling thread for the solvers, meshes and ensembles
 * it creates afterwards (one process per GPU: each rank selects its own) */
int dgp_set_device(int device);

/* ---- mesh: replaces mImportExport::import (mImportExport.cc:57-170) and
 * mMesh::createCellBoundaries/createConnections (mMesh.cc:321-378) */
int dgp_mesh_from_msh(const char* path, dgp_mesh* out);
/* dim 2: cells are triangles (3 vertex indices), bfaces edges (2);
 * dim 3: tets (4) and triangles (3).  Indices are 0-based into xyz (nv x 3);
 * vertex_ids are the file ids used by DG-Parallel's entity ordering
 * (NULL -> 1..nv). */
int dgp_mesh_from_arrays(int dim, int nv, const double* xyz, const int* vertex_ids, int ncells,
                         const int* cells, int cell_tag, int nbfaces, const int* bfaces,
                         const int* btags, dgp_mesh* out);
/* The same with the face matching on the current CUDA device when gpu_faces
 * is nonzero (sort of packed face keys, left/right by the reference's entity
 * order, frames, orientations, normals; the faces, normals and measures equal
 * the host matching's, in another order); meshes whose vertex count does not
 * fit the packed keys (tets: 2^21 vertices), or no device, match on the host. */
int dgp_mesh_from_msh_ex(const char* path, int gpu_faces, dgp_mesh* out);
int dgp_mesh_from_arrays_ex(int dim, int nv, const double* xyz, const int* vertex_ids, int ncells,
                            const int* cells, int cell_tag, int nbfaces, const int* bfaces, const int* btags,
                            int gpu_faces, dgp_mesh* out);
int dgp_mesh_info(dgp_mesh m, int* dim, int* ncells, int* nfaces, int* nvertices);
/* per face: dim sorted vertex ids, left cell, right cell (-1: boundary),
 * local face on each side (-1), classification id; (dim + 5) ints per face.
 * Left/right follow DG-Parallel's upward-adjacency order
 * (DGBoundaryCell::check, DGCell.cc:355-391). */
int dgp_mesh_connectivity(dgp_mesh m, int* out);
/* per face: unit normal (outward from the left cell, 3 doubles) and measure */
int dgp_mesh_face_geometry(dgp_mesh m, double* out);
int dgp_mesh_destroy(dgp_mesh m);

/* ---- law: replaces the ConservationLaw + FieldEvaluator objects */
int dgp_law_create(int kind, int flux, int field, const double* params, dgp_law* out);
int dgp_law_destroy(dgp_law law);
/* Boundary condition of the faces classified boundary_id: bc_kind one of
 * DGP_BC_*.  Applies to solvers and ensembles created from the law afterwards;
 * periodic ids (510, 610) are paired edges, not boundary conditions.  At most
 * DGP_MAX_BC ids per law; DGP_ERR_UNSUPPORTED for a wall on a scalar law. */
int dgp_law_set_bc(dgp_law law, int boundary_id, int bc_kind);

/* ---- solver: DGAnalysis setup (DGAnalysis.cc:133-302) + TimeIntegrator */
int dgp_solver_create(dgp_mesh m, dgp_law law, int order, int precision, int limiter,
                      dgp_solver* out);
/* quadrature rule: DGP_RULE_REFERENCE (DG-Parallel's: volume degree 2p, tet
 * faces degree 2p + 1, edges p + 1 Gauss points) or DGP_RULE_WORKLOAD (at P2
 * the point counts the workloads state: triangles the 7-point volume rule of
 * degree 5, tets the 11-point volume and 6-point face rules of degree 4; built
 * for ScalarLaw on triangles and tets and 3D Maxwell on tets, 128-thread tiles;
 * DGP_ERR_UNSUPPORTED elsewhere).  dgp_solver_create uses the reference rule. */
int dgp_solver_create_ex(dgp_mesh m, dgp_law law, int order, int precision, int limiter, int rule,
                         dgp_solver* out);
int dgp_solver_destroy(dgp_solver s);
int dgp_solver_info(dgp_solver s, int* nfields, int* nmodes, int* ncells, int* nfaces);
/* DGCell::L2ProjInitial (DGCell.cc:1458-1483) of the law's field at time t */
int dgp_project(dgp_solver s, double t);
int dgp_set_state(dgp_solver s, const double* host_state);
int dgp_get_state(dgp_solver s, double* host_state);
/* device-resident variants (pointer to [cell][field][mode] FP64 in file order) */
int dgp_set_state_device(dgp_solver s, const double* dev_state);
int dgp_get_state_device(dgp_solver s, double* dev_state);
/* assembled theRightHandSide of every cell for the current state at time t:
 * TimeIntegrator::assembleVolume + assembleBoundary (TimeIntegrator.cc:1332-1412) */
int dgp_rhs(dgp_solver s, double t, double* host_rhs);
/* min over cells of DGCell::adaptTimeStep (DGCell.cc:1155-1207); times
 * 2^(bins - 1) with local time stepping (dgp_set_time_stepping) */
int dgp_cfl_dt(dgp_solver s, double cfl, double* dt);
/* RungeKuttaTVD3::advanceInTime(t, dt) (TimeIntegrator.cc:838-990), or
 * RungeKuttaTVD2adaptive::advanceInTime with local time stepping; resid may be NULL */
int dgp_step(dgp_solver s, double t, double dt, double* resid);
/* time loop of DGAnalysis::run (DGAnalysis.cc:480-731): CFL dt every step,
 * stretched to land on tend when tend > 0; at most max_steps when > 0.
 * Runs device-resident (CUDA graphs), no host sync per step. */
int dgp_run(dgp_solver s, double t0, double tend, double cfl, int max_steps, double* t_out,
            int* steps_out);
/* kernels one step of dgp_run launches (the fused stage kernel per stage and
 * the finalize of the last; or face/element kernels per stage with the P0
 * fallback's volume check and second face pass), limiter passes and the CFL
 * reduction; with
 * local time stepping the kernels of one advanceInTime, the step's end and the
 * CFL reduction) */
int dgp_launches_per_step(dgp_solver s, int* n);

/* ---- time stepping mode: DGAnalysis's timeSteppingMode (DGAnalysis.cc:229-242)
 * DGP_STEPPING_SSPRK3: RungeKuttaTVD3 (the default).
 * DGP_STEPPING_LOCAL: mode 5, local time stepping -- DGAnalysis::sortCellsBySize
 *   (DGAnalysis.cc:749-890) bins the cells by size (bin b: sizes in
 *   (max/2^(b+1), max/2^b], times 1.0001) and RungeKuttaTVD2adaptive
 *   (TimeIntegrator.cc:442-836) advances bin b with dt / 2^b, interface cells
 *   by the integrator's half steps.  dgp_step(t, dt) is then one
 *   advanceInTime(t, dt) (dt for bin 0; resid 0 as the reference returns),
 *   dgp_run and dgp_cfl_dt use the mode-5 step (CFL minimum times
 *   2^(bins - 1), DGAnalysis.cc:590).  The reference ships the range helpers
 *   this integrator calls (TimeIntegrator::assembleVolume/assembleBoundary(
 *   begin, end, t), TimeIntegrator.cc:1438-1487) with empty bodies, so its own
 *   mode 5 leaves the state unchanged; this library assembles what their
 *   whole-mesh versions assemble on each range.  FP64, no limiter, single
 *   solvers; meshes the reference rejects (fewer than 2 or more than 10 bins,
 *   a cell in no bin or on two interfaces, neighbours more than one bin apart)
 *   give DGP_ERR_INVALID; so does a solver whose P0 fallback is on
 *   (DGP_ERR_UNSUPPORTED: the local time stepping kernels have no P0 pass,
 *   turn it off first with dgp_set_p0_fallback(s, 0); non-physical states are
 *   still counted in dgp_status).  nbins (may be NULL) receives the number of
 *   bins.
 * dgp_lts_bins: per cell (file order) its bin and role (0 inner, 1 large on an
 *   interface, 2 small on an interface); either pointer may be NULL. */
#define DGP_STEPPING_SSPRK3 0
#define DGP_STEPPING_LOCAL 5
int dgp_set_time_stepping(dgp_solver s, int mode, int* nbins);
int dgp_lts_bins(dgp_solver s, int* bin, int* role);
/* Triangle moment limiter (DGP_LIMITER_MOMENT; replaces DGMomentLimiter::limit,
 * DGLimiter.cc:963-1133, which indexes the quadrilateral tensor basis and is
 * invalid on triangles).  The solver applies it after every SSP-RK3 stage
 * (TimeIntegrator::limit, TimeIntegrator.cc:1414-1434) and once after
 * dgp_project (DGAnalysis.cc:276-291).  dgp_limit applies it once to the
 * current state; triggers (may be NULL) receives per cell, in file order, the
 * lowest limited degree (0: untouched) -- the DGSensor trigger indicator.
 * dgp_limiter_triggers returns the triggers of the last application.
 * Barth limiter (DGP_LIMITER_BARTH; DGBarthLimiter::limit, DGLimiter.cc:184-287,
 * triangles and tets): per cell and field, the slope factor from the
 * neighbours' mean bounds at the face points scales the degree-1 modes and,
 * below 0.9, zeroes the higher ones, in place (the reference's
 * TimeIntegrator::limit would copy the unwritten second slot back over it);
 * applied at the same places; triggers are 1 where a factor is below 1. */
int dgp_limit(dgp_solver s, unsigned char* triggers);
int dgp_limiter_triggers(dgp_solver s, unsigned char* out);
/* P0 fallback of DGBoundaryCell::computeBoundaryContributions + DGCell::setToZero
 * (DGCell.cc:639-811): in every SSP-RK3 stage, cells with a non-physical trace
 * at a face point drop their modes k >= 1 and the stage is assembled again.
 * On by default for the Euler laws; 0 turns it off.  Turning it on while local
 * time stepping is on returns DGP_ERR_UNSUPPORTED. */
int dgp_set_p0_fallback(dgp_solver s, int on);
/* Mixed form: the volume contraction of the fused stage kernel on the
 * 5th-generation tensor cores (tcgen05.mma kind::tf32, operands split into
 * TF32 high and low parts, three products accumulated in FP32 in tensor
 * memory) instead of FP32 FMAs on the CUDA cores; off by default (it measured
 * slower on the P3 Euler vortex: a 128-row tile's MMA is too small to hide its
 * fixed latency).  DGP_ERR_UNSUPPORTED unless the solver is mixed, with
 * 128-thread tiles and at most 16 modes.  No counterpart in DG-Parallel. */
int dgp_set_tensor_cores(dgp_solver s, int on);
/* Rounding probe for the error decomposition of the mixed form: in the FP64
 * fused stage kernel, the terms selected by mask are rounded to FP32 (1 the
 * geometry: J^{-1}, |J| w, face normals, |J_f| w; 2 the face-point traces; 4
 * the volume-point values; 8 the volume flux products; 16 the face slots; 32
 * the contraction's result; 64 the reference tables); 0 turns it off.  Built
 * for the FP64 P3 Euler (Roe) solver with 128-thread tiles
 * (DGP_ERR_UNSUPPORTED elsewhere).  No counterpart in DG-Parallel. */
int dgp_set_rounding_probe(dgp_solver s, int mask);
/* Bound on the first wait of the fused stage kernel for its bulk copies, in
 * polls counted from the copies' issue (0 restores the default wait, about 4
 * million polls).  A CTA whose wait gives up waits again for its copies with
 * the full bound, writes nothing and returns; the next dgp_status returns
 * DGP_ERR_CUDA ("a bounded wait ... gave up") and that stage's output is
 * incomplete.  For testing the error path; no counterpart in DG-Parallel. */
int dgp_set_copy_wait_limit(dgp_solver s, int polls);
/* non-physical states seen since the last call (isPhysical, EulerLaw.cc:1398) */
int dgp_status(dgp_solver s, int* nonphysical, int* first_bad_cell);
/* L2 error of one field against the law's exact field (DGCell::densityErrorL2,
 * DGError.cc:805-826), FP64 reduction */
int dgp_l2_error(dgp_solver s, double t, int field, double* err);
/* Error norms against the exact field at time t, the family of DGError.cc
 * (DGCell::L1exact :549, LinfError :567, L1exactPressure :601,
 * entropyErrorL1_2D/3D :621-665, pressureErrorL2 :774, densityErrorL2 :805,
 * entropyErrorL2_2D :687; gamma 1.4 as there).  quantity >= 0: that field; -1:
 * pressure, -2: entropy deviation (p / p_ex) / (rho / rho_ex)^gamma - 1 (Euler
 * laws).  rule 0: the volume rule of degree 2p (as the L1 / Linf functions),
 * 1: degree 2(p+1) (as the L2 functions).  norms[3] = L1, L2, Linf. */
int dgp_error_norms(dgp_solver s, double t, int quantity, int rule, double* norms);

/* Point probes (DGPointSensor / DGLineSensor, DGSensor.cc:88-186; a line
 * sensor is a probe over points sampled along the segment).  The points (dim
 * doubles each) are located once on the host (a point takes the lowest-index
 * cell, in file order, that contains it, as DGCell::inCell tests it;
 * found[i] = 0 for points outside the mesh, whose values read NaN).
 * dgp_probe_eval: every field at every point of the current state, [n][M].
 * dgp_probe_record: during dgp_run, sample the state after every `every`-th
 * step into a device buffer of max_samples samples, inside the run's step
 * graph (no host round trip per sample); every = 0 stops recording.
 * dgp_probe_samples: the samples of the last run, times [k] and values
 * [k][n][M].  Destroy probes before their solver (a probe whose solver was
 * destroyed returns DGP_ERR_INVALID). */
int dgp_probe_create(dgp_solver s, int n, const double* points, dgp_probe* out, int* found);
int dgp_probe_destroy(dgp_probe p);
int dgp_probe_info(dgp_probe p, int* n, int* found);
int dgp_probe_eval(dgp_probe p, double* values);
int dgp_probe_record(dgp_probe p, int every, int max_samples);
int dgp_probe_samples(dgp_probe p, int* nsamples, double* times, double* values);

/* Checkpoints in the data format of DGAnalysis::write / read (DGPref.cc:712-766):
 * TACT, ITER, "dim cells faces", per cell its entity (type, geometric order,
 * vertex ids; mMesh::readMEntity, mMesh.cc:413-455) then the order and the
 * coefficients [field][mode] (DGCell::write, DGCell.cc:1523-1531), then the
 * face entities.  Written as readMEntity reads them (DGAnalysis::write leaves
 * out the geometric order); both layouts are read, cells matched by their
 * vertex ids.  Coefficients carry 17 significant digits (round trip exact). */
int dgp_checkpoint_write(dgp_solver s, const char* path, double t, int iter);
int dgp_checkpoint_read(dgp_solver s, const char* path, double* t, int* iter);
/* sum over cells of the cell integral of every field (conserved totals), FP64 */
int dgp_totals(dgp_solver s, double* totals);
int dgp_synchronize(dgp_solver s);
/* the solver's CUDA stream (cudaStream_t) for callers that order their own
 * work or record CUDA events against the solver's launches */
int dgp_solver_stream(dgp_solver s, void** stream);
/* mean device time (CUDA events on the solver's stream) over `iters` launches
 * each: ms[3] = the fused stage kernel of stage 1, of stage 2 and of the last
 * stage with the fused CFL reduction (solvers whose tiles' halos do not fit
 * the fused kernel: the face kernel, the element kernel of an inner stage and
 * of the last stage).  Leaves the state unchanged; resets the time control. */
int dgp_profile_kernels(dgp_solver s, int iters, float* ms);
/* *fused = 1 when each stage runs as one fused stage kernel (faces, volume,
 * lift and the SSP-RK3 update of a tile of cells), 0 when it runs as the face
 * and element kernels (a tile's halo too large for shared memory) */
int dgp_solver_fused(dgp_solver s, int* fused);
/* run the stages as the fused stage kernel (on = 1, the default where it is
 * built) or as the separate face and element kernels (on = 0; also turns off
 * the tensor-core contraction and the rounding probe, which only the fused
 * kernel has); DGP_ERR_UNSUPPORTED when on = 1 and the fused kernel is not
 * built for the solver */
int dgp_set_fused(dgp_solver s, int on);
/* Assembled right-hand side that allocates no device memory; no counterpart in
 * DG-Parallel.  For callers that cannot call cudaMalloc when they need a RHS
 * (device memory owned by another allocator, or no tolerance for the
 * synchronisation an allocation implies).  dev_state and dev_rhs are device
 * buffers, FP64 [cell][field][mode] in file order, like dgp_rhs's output.  The
 * intermediates (a state and a RHS copy in internal order; with the separate
 * stage form also the face slots and traces) live in a 32 MiB static device
 * array that every GPU loading the library holds until exit; meshes that need
 * more return DGP_ERR_INVALID.  The P0 fallback applies in the fused form (as
 * in dgp_rhs) and not in the separate form.
 * Calls share that array: calls that overlap on the GPU race.  The first call
 * on a device looks up the array's device address (host-side setup), so make
 * it before any stream capture.  Like dgp_rhs, the call resets the solver's
 * time control (time t, step 0).  A device reset (cudaDeviceReset) invalidates
 * every handle of this library on that device, the cached address of the
 * static array included.  Returns after the solver's stream is idle. */
int dgp_rhs_noalloc(dgp_solver s, const double* dev_state, double t, double* dev_rhs);

/* ---- ensembles (no counterpart in DG-Parallel, which runs one DGAnalysis per
 * process): n independent instances of uneven size, each with its own mesh,
 * law parameters and order, run batched on one GPU.  Instances with the same
 * (law, flux, element, order) share one set of kernels over a joined cell and
 * face index space; each keeps its own CFL step, end time and step count.  A
 * group's instances must share the law's gamma; field parameters (amplitude,
 * centre, ...) may differ.  Instance states use the layout of a single solver
 * on that instance's mesh. */
int dgp_ensemble_create(int n, const dgp_mesh* meshes, const dgp_law* laws, const int* orders, int precision,
                        int limiter, dgp_ensemble* out);
int dgp_ensemble_destroy(dgp_ensemble e);
/* group: index of the kernel group the instance runs in */
int dgp_ensemble_info(dgp_ensemble e, int i, int* nfields, int* nmodes, int* ncells, int* group);
int dgp_ensemble_project(dgp_ensemble e, double t);
int dgp_ensemble_get_state(dgp_ensemble e, int i, double* host_state);
int dgp_ensemble_set_state(dgp_ensemble e, int i, const double* host_state);
/* every instance from t0 to tend (or max_steps steps) at its own CFL step;
 * per-instance arrays (may be NULL): final time, steps taken, device time from
 * the common start to the instance's last step (ms); total_ms: the latest of
 * those.  Device-resident: CUDA graphs of 8 steps per group until all are done. */
int dgp_ensemble_run(dgp_ensemble e, double t0, double tend, double cfl, int max_steps, double* t_out,
                     int* steps_out, double* ms_out, double* total_ms);
/* conserved totals (FP64) and L2 error against the instance's exact field */
int dgp_ensemble_totals(dgp_ensemble e, int i, double* totals);
int dgp_ensemble_l2_error(dgp_ensemble e, int i, double t, int field, double* err);
int dgp_ensemble_launches_per_step(dgp_ensemble e, int* n);
/* ---- discrete adjoint (no counterpart in DG-Parallel): gradient with respect
 * to the initial coefficients of an objective of the state after nsteps
 * SSP-RK3 steps of fixed size dt, by checkpoint (every `every` steps) and
 * recompute.  The backward pass runs the transposed linearised operator
 * (transposed volume contraction and lift, Jacobians of the numerical and
 * boundary fluxes, reversed stage combination) on the device.  Built for every
 * flux (the exact Riemann solver differentiated through its Newton
 * iteration); meshes with periodic edges are refused.  With the Barth limiter
 * the limiter is linearised with its active set frozen: the forward pass
 * records each pass's slope factors per (cell, field), and the backward pass
 * applies that fixed linear map (degree 1 scaled, degrees >= 2 dropped below
 * 0.9) to the cotangents; the moment limiter is refused.
 * Receivers define J = sum_r (u_0(x_r, T) - observed_r)^2 on field 0 (the
 * density of the Euler laws); points are dim doubles each. */
int dgp_adjoint_set_receivers(dgp_solver s, int n, const double* points, const double* observed);
/* field 0 at the receivers for the current state (rho may be NULL) and J */
int dgp_receiver_values(dgp_solver s, double* rho, double* J);
/* from the current state at time t0; leaves the state at the final time; J may be NULL.
 * every > 0: checkpoint every `every` steps, the backward pass recomputes each
 * segment; every == 0: keep all 3 * nsteps stage states in device memory, the
 * backward pass recomputes nothing (DGP_ERR_NOMEM when they do not fit). */
int dgp_forward_checkpointed(dgp_solver s, double t0, double dt, int nsteps, int every, double* J);
/* on = 1: later forward passes (every == 0, the same nsteps) apply the Barth
 * slope factors recorded by the last such pass instead of computing them, i.e.
 * run the frozen map whose transpose the backward pass applies (a check of the
 * gradient by finite differences); on = 0 computes them again */
int dgp_adjoint_freeze_limiter(dgp_solver s, int on);
/* dJ/du0 (host, file order [cell][field][mode]) of the last forward pass; the
 * seed dJ/du_T is dJ_duT when not NULL, else the receiver objective's */
int dgp_backward(dgp_solver s, const double* dJ_duT, double* dJ_du0);
/* ---- autotuner: the tile shape (threads of the element and face kernels,
 * which sets the cells per element-kernel tile and the faces per face-kernel
 * CTA; 64, 128 or 256 where built) that runs fastest for a configuration at a
 * problem size.  Each candidate is timed over `iters` SSP-RK3 steps with CUDA
 * events; the winner is recorded in a process-wide table keyed by (law, flux,
 * element, order, precision, floor(log2 cells)) that dgp_solver_create and
 * dgp_ensemble_create consult (128 threads when nothing is recorded).  For
 * each shape both stage forms are timed where the fused stage kernel is built
 * (dgp_set_fused), and the faster is recorded with it (without a record, a
 * default measured on B200 decides: fused for the 2D Euler (Roe, LLF), scalar
 * and Maxwell laws at P2-P3, 2D Euler P1 and P1 on tets (scalar: P2); the
 * separate kernels for Burgers, the exact Godunov flux, 2D P4, the 3D Euler law
 * and tets of higher order).  ms_per_step[3] (may be NULL) gets each shape's best time, -1
 * where not built. */
int dgp_autotune(dgp_mesh m, dgp_law law, int order, int precision, int limiter, int iters, int* best_block,
                 float* ms_per_step);
/* the same for every (law, flux, element, order) group of an ensemble */
int dgp_autotune_ensemble(int n, const dgp_mesh* meshes, const dgp_law* laws, const int* orders, int precision,
                          int limiter, int iters);
/* records a tile shape by hand (as the autotuner would) for meshes of `cells` cells */
int dgp_tune_set(int law, int flux, int dim, int order, int precision, int cells, int block);
int dgp_solver_block(dgp_solver s, int* block, int* cells_per_tile);
int dgp_ensemble_group_block(dgp_ensemble e, int group, int* block, int* cells_per_tile);
#ifdef __cplusplus
}
#endif
#endif
