/* C restatement of DG-Parallel's explicit DG right-hand side and SSP-RK3 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the CPU oracle that the parity tests, the
 * smoke check and the bench's cpu_baseline leg compare the CUDA path against;
 * the product never links or calls it.  It restates, in plain FP64 C, the
 * reference algorithm of DGCell::computeVolumeContribution (DGCell.cc:184-249),
 * DGBoundaryCell::computeBoundaryContributions (DGCell.cc:639-732),
 * RungeKuttaTVD3::advanceInTime (TimeIntegrator.cc:838-990) and the CFL rule
 * of DGCell::adaptTimeStep (DGCell.cc:1155-1207), with DG-Parallel's face
 * left/right convention (std::set order keyed by the sum of glibc rand() over
 * vertex ids, mEntity.cc:173-200, Vertex.cc:26-31).  It also restates the
 * features the reference lacks (Lax-Friedrichs fluxes, 3D Maxwell on tets, the
 * isentropic vortex and TM110 cavity fields).
 */
#ifndef DG_ORACLE_H
#define DG_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { OR_SCALAR = 0, OR_BURGERS2D = 1, OR_EULER2D = 2, OR_EULER3D = 3, OR_MAXWELL3D = 4, OR_MAXWELL2D = 5 };
enum { OR_FLUX_UPWIND = 0, OR_FLUX_CENTRAL = 1, OR_FLUX_GODUNOV = 2, OR_FLUX_ROE = 3,
       OR_FLUX_LLF = 4 };
/* analytic fields used as initial condition, far field and exact solution */
enum { OR_FIELD_GAUSS = 0, OR_FIELD_VORTEX = 1, OR_FIELD_PULSE3D = 2, OR_FIELD_SINE = 3,
       OR_FIELD_GAUSS3D = 4, OR_FIELD_TM110 = 5, OR_FIELD_TM2D = 6 };

/* field parameters (16 doubles):
 *  [0..2] advection velocity a      [3..5] centre c       [6] width s
 *  [7] gamma   [8] vortex beta   [9] amplitude A   [10] cavity side L */
typedef struct or_solver or_solver;

or_solver* or_create(const char* msh_path, int law, int flux, int order, int field,
                     const double* params);
/* the same with a quadrature rule option: 0 DG-Parallel's, 1 the workloads'
 * point counts at P2 (the solver's DGP_RULE_WORKLOAD) */
or_solver* or_create_rule(const char* msh_path, int law, int flux, int order, int field,
                          const double* params, int rule);
void or_destroy(or_solver* s);
int or_num_cells(const or_solver* s);
int or_num_faces(const or_solver* s);
int or_num_fields(const or_solver* s);
int or_num_modes(const or_solver* s);
/* per face: nfv vertex ids (file ids, sorted ascending), eL, eR, lfL, lfR, bid;
 * nfv = 2 (edges) or 3 (tet faces); returns ints written. */
int or_connectivity(const or_solver* s, int* out);
void or_face_normals(const or_solver* s, double* out); /* per face n[3], measure */
void or_get_state(const or_solver* s, double* out);    /* [E][m][Np] file order */
void or_set_state(or_solver* s, const double* in);
void or_project(or_solver* s, double t);                /* L2 projection of the field */
void or_rhs(or_solver* s, double t, double* out);       /* assembled RHS, not scaled */
int or_rhs_p0(or_solver* s, double t, double* out);
double or_cfl_dt(const or_solver* s, double cfl);
double or_step(or_solver* s, double t, double dt);      /* SSP-RK3, returns resid */
double or_run(or_solver* s, double t0, double tend, double cfl, int nsteps, int* steps_done);
double or_l2_error(const or_solver* s, double t, int field_index); /* vs exact field */
/* L1, L2, Linf of a field (quantity >= 0), the pressure (-1) or the entropy
 * deviation (-2) against the exact field; rule 0: volume rule of degree 2p,
 * 1: degree 2(p+1) (definitions in dg_oracle.c); returns -1 if not defined */
int or_error_norms(const or_solver* s, double t, int quantity, int rule, double* out);
void or_field_eval(const or_solver* s, const double* x, double t, double* q);
unsigned int or_glibc_rand_first(unsigned int seed);   /* srand(seed); rand() */
/* limiters (definitions in dg_oracle.c), on = 1: triangle moment limiter,
 * on = 2: Barth limiter (triangles and tets), 0: off.  Applied after every
 * SSP-RK3 stage by or_step when enabled; or_limit applies it once to the
 * current state and writes the per-cell trigger (moment: lowest limited
 * degree, Barth: 1 where a slope factor is below 1; 0: untouched, file order)
 * when trig is not NULL; returns the number of triggered cells. */
void or_set_limiter(or_solver* s, int on);
int or_limit(or_solver* s, unsigned char* trig);
/* P0 fallback of DGCell::setToZero for cells with a non-physical face trace */
void or_set_p0_fallback(or_solver* s, int on);
void or_bad_cells(const or_solver* s, unsigned char* out); /* marks of the last stage */
void or_triggers(const or_solver* s, unsigned char* out);  /* of the last limiter pass */

/* local time stepping (RungeKuttaTVD2adaptive on the size bins of
 * DGAnalysis::sortCellsBySize; definitions in dg_oracle.c): or_lts_setup bins
 * the cells and returns the number of bins, or < 0 where the reference stops
 * (-1 fewer than 2 bins, -2 more than 10, -3 a cell in no bin, -4 a cell on
 * two interfaces, -5 neighbours more than one bin apart); or_lts_bins: bin
 * and role (0 inner, 1 large, 2 small on an interface) per cell, file order;
 * or_lts_step: one step of dt for bin 0; or_lts_dt: the mode-5 step. */
int or_lts_setup(or_solver* s);
void or_lts_bins(const or_solver* s, int* bin, int* role);
double or_lts_step(or_solver* s, double t, double dt);
double or_lts_dt(const or_solver* s, double cfl);

#ifdef __cplusplus
}
#endif
#endif
