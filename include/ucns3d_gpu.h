/*
 * ucns3d_gpu.h - C ABI of the B200 explicit residual engine.
 *
 * The engine replaces, for one GPU, the per-cell / per-face work of one
 * SSP-RK3 step of UCNS3D:
 *
 *   RUNGE_KUTTA3              src/time_p.f90:885-1027   -> ucg_rk3_step / ucg_step
 *   CALCULATE_CFL             src/time_p.f90:27-191     -> ucg_compute_dt
 *   CALL_FLUX_SUBROUTINES_3D  src/time_p.f90:2253-2497  -> ucg_residual
 *     LEAST_SQUARES / ALLGRADS_INNER/MIX   src/reconstruct_p.f90:2702, src/gradients.f90:10-706
 *     WENOWEIGHTS / CP_RECONSTRUCTION      src/reconstruct_p.f90:407-1250
 *     CHECKSOL / MUSCL / CHECKSOLX         src/reconstruct_p.f90:3126-3406, 2286-2352
 *     SOLUTIONTRIAV2                        src/reconstruct_p.f90:2358
 *     CALCULATE_FLUXESHI_CONVECTIVE         src/flux_p.f90:478-1030
 *     CALCULATE_FLUXESHI_DIFFUSIVE          src/flux_p.f90:1520-2107
 *   TGV kinetic energy sum     src/time_p.f90:4145-4198  -> ucg_reduce(UCG_REDUCE_KE)
 *
 * The Fortran driver keeps the mesh, the partitioning, UCNS3D.DAT and all
 * set-up (geometry, stencils, pseudo-inverses).  It packs the set-up tables
 * once (ucg_upload_geometry, ucg_upload_recon), then calls the engine from the
 * master thread in place of the SELECT CASE(RUNGEKUTTA) of TIME_MARCHING
 * (src/time_p.f90:4229-4263).
 *
 * Conventions
 *   - Every entry point returns 0 (UCG_OK) or a positive UCG_E* code; the
 *     engine never aborts.  ucg_last_error() gives the message.
 *   - Host pointers are borrowed for the duration of the call only.
 *   - Array shapes are written C-order, e.g. [n][5] is 5 contiguous doubles
 *     per cell, which is Fortran U(1:5, 1:n).  Cell and face indices are
 *     0-based.
 *   - A handle is not re-entrant: call it from one host thread.  All device
 *     work of a handle runs on one CUDA stream (ucg_get_stream).
 *   - There is no CPU fallback: without a usable sm_100 device ucg_create
 *     fails with UCG_ECUDA.
 */
#ifndef UCNS3D_GPU_H
#define UCNS3D_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UCG_NV 5          /* conserved variables rho, rho*u, rho*v, rho*w, E   */
#define UCG_MAX_FACES 6   /* hexahedra                                           */
#define UCG_MAX_QP 16     /* face quadrature points (4x4 Gauss on quadrilaterals) */

enum {
  UCG_OK = 0,
  UCG_EINVAL = 1,     /* bad argument or size                                    */
  UCG_ECUDA = 2,      /* CUDA runtime error (message has the CUDA error string)   */
  UCG_ENONPHYS = 3,   /* NaN, or non-positive density or pressure in the state    */
  UCG_ESTATE = 4,     /* call out of order (e.g. a step before the tables)        */
  UCG_ENOMEM = 5,     /* device allocation failed                                 */
  UCG_ETIMEOUT = 6    /* a bounded device wait gave up                            */
};

enum { UCG_FP64 = 0, UCG_MIXED = 1 };
enum { UCG_REDUCE_KE = 1, UCG_REDUCE_MASS = 2, UCG_REDUCE_ENERGY = 3, UCG_REDUCE_ENSTROPHY = 4 };

/* Scheme and fluid parameters.  Field names follow UCNS3D's module globals
 * (src/parameters.f90, src/declarations.f90).                               */
typedef struct ucg_config {
  int32_t governing;   /* 1 Navier-Stokes (ITESTCASE 4), 2 Euler (ITESTCASE 3)        */
  int32_t scheme;      /* 2 MUSCL (IWENO=-1), 3 WENO/CWENO (IWENO=1)                    */
  int32_t iorder;      /* reconstruction degree IORDER = spatialorder-1, 1..4           */
  int32_t ees;         /* 0 WENO, 5 CWENO (parameters.f90:1340-1372)                    */
  int32_t wenwrt;      /* 1 conserved-variable WENO, 2 characteristic-variable WENO
                          (WENO only; WENWRT, reconstruct_p.f90:445, 497-758)         */
  int32_t limiter;     /* MUSCL limiter code (SLOPE_LIMITERS): 1 Barth-Jespersen,
                          2/3/9 Michalak, 4/8 Venkatakrishnan blended, 5 van Albada,
                          6 van Leer, 7 Venkatakrishnan; the adjoint covers 7           */
  int32_t riemann;     /* iRiemann: 1 HLLC, 2 Rusanov, 3 Roe, 4 rotated Roe-HLL,
                          5 t-Roe, 9 HLL (flux_p.f90:587-660);
                          the adjoint covers HLLC                                      */
  int32_t precision;   /* UCG_FP64 or UCG_MIXED                                         */
  int32_t wenoz;       /* WENO-Z weights for CWENO (reconstruct_p.f90:1021-1029)         */
  int32_t ideg;        /* IDEGFREE: basis functions without the mean                    */
  int32_t imax;        /* cells of a full stencil without the cell itself               */
  int32_t admis_max;   /* stencil slots per cell (TYPESTEN)                             */
  int32_t ideg2;       /* CWENO directional stencils: IDEGFREE2 (0 otherwise)           */
  int32_t imax2;       /* CWENO directional stencils: NUMNEIGHBOURS2-1 (0 otherwise)    */
  int32_t nq_quad;     /* quadrature points on a quadrilateral face                     */
  int32_t nq_tri;      /* quadrature points on a triangular face                        */
  double gamma;        /* GAMMA                                                         */
  double prandtl;      /* PRANDTL                                                       */
  double visc;         /* VISC: free-stream dynamic viscosity (parameters.f90:1241)     */
  double r_gas;        /* R_gas (parameters.f90:1223-1227)                             */
  double pres;         /* PRES: free-stream pressure (Sutherland reference T0)          */
  double rres;         /* RRES: free-stream density                                    */
  double lwci;         /* wenocentralweight (LWCI1)                                     */
  double weno_eps;     /* DIVBYZERO of WENOWEIGHTS, 10E-12 (reconstruct_p.f90:437)       */
  double kappa_ven;    /* KAPPA_VEN of SLOPE_LIMITERS, 10 (reconstruct_p.f90:3436)       */
  double lamx;         /* jump damping of the viscous face gradient (LAMX, 1)           */
  double quad_w[UCG_MAX_QP];  /* face weights, summing to 1 (QUADRATUREQUAD3D)          */
  double tri_w[UCG_MAX_QP];   /* face weights, summing to 1 (QUADRATURETRIANG)          */
  double bc_state[UCG_NV];    /* free-stream primitive state rho,u,v,w,p for the BCs    */
  int32_t boundtype;   /* BOUNDTYPE (parameters.f90:253): 0 inflow faces take the free
                          stream and outflow faces their own state (supersonic);
                          1 the characteristic subsonic treatment where |u| < c
                          (BOUNDARYS, flow_operations.f90:2883-3012).  The far field
                          (code 6, :3230) does not depend on it                       */
  int32_t reorder;     /* 0 keep the caller's cell order on the device; 1 renumber the
                          cells internally by reverse Cuthill-McKee on the face-
                          neighbour graph at ucg_upload_geometry, so that the stencil
                          and face gathers of a mesh in partitioner or file order
                          touch nearby memory; kept only where it gathers from
                          fewer cache lines (ucg_cell_order).  Every [n][5] array
                          of the ABI stays
                          in the caller's order (permuted on the device), and each
                          face flux is still evaluated by the face side of the lower
                          caller index, so the results are bitwise those of
                          reorder 0 except for domain sums (ucg_reduce, ucg_force),
                          whose order of addition changes                         */
  int32_t mood;        /* 1: MOOD a posteriori limiting in every RK3 stage (MOOD = 1
                          when MOOD.DAT exists, parameters.f90:126-140;
                          RUNGE_KUTTA3_MOOD, time_p.f90:582-880; mood.f90).  WENO /
                          CWENO (scheme 3) and Euler only: the reference's MOOD
                          recomputes only the convective fluxes.  With MOOD the
                          CHECKSOL fall-back of a reconstruction runs only on the
                          cells the last MOOD pass recomputed (RECALC, initially 0,
                          memory.f90:1002-1010; reconstruct_p.f90:2310); the other
                          reduced cells keep their WENO values, then CHECKSOLX.  The
                          flags persist in the handle across stages and steps     */
  int32_t mood_mode;   /* MOOD_MODE: 1 relaxed (bounds widened by max(var1,
                          var2 * range)), 0 original                               */
  double mood_var[4];  /* MOOD_VAR1, MOOD_VAR2 (first cascade, to MUSCL), MOOD_VAR3,
                          MOOD_VAR4 (second cascade, to first order)               */
} ucg_config;

/* Per-cell geometry (IELEM(N,I) and the small parts of ILOCAL_RECON3(I),
 * src/declarations.f90:461-510, 644-704).  [n][F] arrays have UCG_MAX_FACES
 * entries per cell; unused faces are ignored.                                */
typedef struct ucg_geometry {
  int64_t ncells;
  const int32_t* nfaces;      /* [n]      IFCA                                          */
  const int32_t* face_type;   /* [n][F]   types_faces: 5 quadrilateral, 6 triangle      */
  const int32_t* neigh;       /* [n][F]   INEIGH, -1 on a physical boundary face        */
  const int32_t* neigh_face;  /* [n][F]   INEIGHN                                      */
  const int32_t* bc;          /* [n][F]   boundary code on faces with neigh = -1:
                                 1 inflow, 2 outflow, 3 symmetry, 4 wall (slip for
                                 Euler, no slip for Navier-Stokes,
                                 flow_operations.f90:3172-3186), 6 far field
                                 (BOUNDARYS, flow_operations.f90:2860-3375); 0
                                 elsewhere                                           */
  const int32_t* qperm;       /* [n][F][Q] quadrature point of the neighbour's face that
                                 coincides with this face's point q                     */
  const double* face_angle;   /* [n][F][2] FACEANGLEX, FACEANGLEY                       */
  const double* face_area;    /* [n][F]   SURF                                          */
  const double* dih;          /* [n][F]   DIH: centre-to-centre distance               */
  const double* qpoints;      /* [n][F][Q][3] QPOINTS in the cell's reference frame    */
  const double* volume;       /* [n]      TOTVOLUME                                     */
  const double* minedge;      /* [n]      MINEDGE                                       */
  const double* invccjac;     /* [n][3][3] INVCCJAC                                     */
  const double* basis_mean;   /* [n][ideg] INTEG_BASIS / VOLUME(1,1): basis cell means
                                 (NULL if ucg_build_recon forms them)                 */
  const int32_t* admis;       /* [n]      ADMIS                                         */
  const int32_t* full;        /* [n]      FULL                                          */
} ucg_geometry;

/* Reconstruction tables of cells [first, first+count): stencils and the
 * FP64 pseudo-inverses of PRESTORE_RECONSTRUCTION3 (src/prestore.f90:167-818)
 * and the smoothness matrices of INDICATORMATRIX (src/prestore.f90:1529-1673).
 * With table_id == NULL the matrices are given per cell (ntables ignored);
 * otherwise cell c uses matrix set table_id[c] out of ntables sets, which
 * lets meshes with repeated cell geometry upload each set once.             */
typedef struct ucg_recon {
  int64_t first, count;
  const int32_t* stencil;     /* [count][admis_max][imax+1] IHEXL, slot 0 = the cell,
                                 -1 = unused (only outside the rows 1..imax (imax2 for
                                 CWENO stencils ll > 0) of stencils ll < admis[c])     */
  int64_t ntables;
  const int32_t* table_id;    /* [count] or NULL                                        */
  const double* invmat;       /* [ntab][admis_max][imax][ideg] invmat_stencilt          */
  const double* invmat2;      /* [ntab][admis_max][imax2][ideg2] invmat_stenciltC (CWENO,
                                 slot 0 unused) or NULL                                 */
  const double* indicator;    /* [ntab][ideg][ideg] INDICATOR (WENO) or NULL           */
  const double* indicator2;   /* [ntab][ideg2][ideg2] INDICATORC (CWENO) or NULL       */
} ucg_recon;

/* Cell shapes for building the tables of ucg_recon on the device
 * (ucg_build_recon), in the caller's cell order.  Vertices are the cell's
 * nodes as seen from the cell (a periodic mesh gives each cell its own
 * unwrapped copy); the reference frame of cell c maps x to
 * INVCCJAC(c) (x - frame_origin(c)) and has Jacobian determinant
 * frame_det(c) (VEXT(1,:) and the determinant of the cell's mapping,
 * src/prestore.f90:167-260).                                                */
typedef struct ucg_shapes {
  int64_t ncells;
  const int32_t* shape;        /* [n]       ISHAPE: 1 hexahedron, 2 tetrahedron,
                                  3 pyramid, 4 prism                            */
  const double* vertices;      /* [n][8][3] nodes (hexahedron: hexaVOLUME order,
                                  src/grid_t.f90:662-669; prism: bottom 0-2, top
                                  3-5; pyramid: base 0-3, apex 4)             */
  const double* centre;        /* [n][3]    cell centres                        */
  const double* volume;        /* [n]       TOTVOLUME                           */
  const double* frame;         /* [n][3][3] INVCCJAC (as ucg_geometry.invccjac) */
  const double* frame_origin;  /* [n][3]                                        */
  const double* frame_det;     /* [n]                                           */
  double period[3];            /* box length of each periodic direction, 0 where
                                  the mesh is not periodic (stencil members are
                                  moved to the cell's periodic image)           */
} ucg_shapes;

typedef struct ucg_engine ucg_engine;

/* Create an engine on CUDA device `device` for meshes of `ncells` cells. */
int ucg_create(const ucg_config* cfg, int64_t ncells, int device, ucg_engine** out);
void ucg_destroy(ucg_engine* e);

/* Upload order: geometry first (ADMIS decides which stencil rows are
 * checked), then the reconstruction tables, in one or more cell ranges;
 * ucg_upload_recon before ucg_upload_geometry returns UCG_ESTATE. */
int ucg_upload_geometry(ucg_engine* e, const ucg_geometry* g);
int ucg_upload_recon(ucg_engine* e, const ucg_recon* r);
/* The reconstruction tables built on the device instead of uploaded:
 * the basis means of every cell, and per matrix set (r->table_id, as from
 * ucp_prepare_geometry, or one set per cell when NULL) the pseudo-inverses
 * of every stencil of the set's first cell (PRESTORE_RECONSTRUCTION3,
 * src/prestore.f90:167-818: moments of the stencil cells in the cell's
 * frame, the normal matrix, its inverse by Householder QR, QRDECOMPOSITION +
 * INVERT of src/matrix.f90:93-150) and its smoothness matrices
 * (INDICATORMATRIX, src/prestore.f90:1529-1673).  The quadrature, the
 * operations and their order are those of the host set-up library
 * (ucp_prepare), without fused multiply-adds on either side, so the tables
 * are ucp_prepare's bit for bit.  r: all cells (first 0, count n), stencil
 * and table_id / ntables as in ucg_recon; the matrix pointers are ignored.
 * Replaces ucg_upload_recon and the basis_mean of ucg_upload_geometry
 * (which may then be NULL).  Synchronous.  Device memory beyond the
 * handle's own while it runs: the shapes (about 300 bytes per cell) and a
 * staging buffer of at most 512 MiB.  UCG_EINVAL also when a normal matrix
 * is singular. */
int ucg_build_recon(ucg_engine* e, const ucg_shapes* s, const ucg_recon* r);

/* Conserved state U_C(I)%VAL(1,1:5), [n][5]. */
int ucg_set_state(ucg_engine* e, const double* u, int64_t n);
int ucg_get_state(ucg_engine* e, double* u, int64_t n);

/* CALCULATE_CFL: dt = min over cells, CCFL = cfl/3 (time_p.f90:46). */
int ucg_compute_dt(ucg_engine* e, double cfl, double* dt);

/* One CALL_FLUX_SUBROUTINES_3D on the current state; writes RHS(I)%VAL
 * (net outward flux, convective minus viscous) to rhs [n][5] if non-NULL. */
int ucg_residual(ucg_engine* e, double* rhs);

/* One RUNGE_KUTTA3 step with the given dt (asynchronous on the stream). */
int ucg_rk3_step(ucg_engine* e, double dt);

/* nsteps of (CALCULATE_CFL + RUNGE_KUTTA3), dt kept on the device; no host
 * synchronisation.  The dt of the last step is readable with ucg_last_dt.  */
int ucg_step(ucg_engine* e, double cfl, int32_t nsteps);
int ucg_last_dt(ucg_engine* e, double* dt);

/* Domain sums over cells: UCG_REDUCE_KE = sum V*rho*|u|^2/2 (time_p.f90:4145),
 * UCG_REDUCE_MASS = sum V*rho, UCG_REDUCE_ENERGY = sum V*E,
 * UCG_REDUCE_ENSTROPHY = sum V*rho*(rho*|grad u - grad u^T|_F^2/2)/2, the
 * TOTENS of a periodic (BOUNDTYPE 1) TGV run (ENSTROPHY_CALC,
 * flow_operations.f90:2718-2815; time_p.f90:4311-4320) with the cell-centre
 * velocity gradients of the viscous least squares; Navier-Stokes MUSCL
 * (IORDER 1) only, where those gradients are the linear polynomial's.     */
int ucg_reduce(ucg_engine* e, int32_t what, double* out);

/* Synchronise, then report UCG_ENONPHYS if a kernel met a NaN or a
 * non-positive density/pressure since the last call (and clear the flag). */
int ucg_check_health(ucg_engine* e);
int ucg_synchronize(ucg_engine* e);

/* Average device time of the stage kernels over `reps` residual
 * evaluations of the current state, measured with CUDA events on the
 * handle's stream, into ms[4]: ms[0] reconstruction, ms[1] face fluxes,
 * ms[2] time step (CALCULATE_CFL), ms[3] the stencil least-squares kernel
 * alone (part of ms[0]; all of it for MUSCL IORDER 1), after one untimed
 * evaluation.  For profiling; it leaves the state unchanged.               */
int ucg_time_kernels(ucg_engine* e, int32_t reps, double* ms);

/* Bounded device waits.  The opt-in least squares through the shared-memory
 * bulk-copy ring (UCG_LSQ_BULK=1 in the environment at ucg_create) waits on
 * each copy for at most `polls` polls (about 300 ns each; the default, about
 * 20 ms, is restored by polls < 0).  A wait that gives up makes its warp
 * finish the copies it has in flight (each with the default bound) and
 * return, and the next ucg_check_health reports UCG_ETIMEOUT; the handle
 * stays usable.  polls = 0 makes every such wait give up at once, which
 * exercises that path without a fault.  No counterpart in the reference. */
int ucg_set_wait_limit(ucg_engine* e, int64_t polls);

/* The cell numbering chosen at ucg_upload_geometry.  With cfg.reorder 1 the
 * engine computes reverse Cuthill-McKee and keeps it only if the face
 * neighbours of each 32-cell warp then span fewer 128-byte lines of the
 * state (by 5 %) than in the caller's order; *renumbered = 1 if it did.
 * n2o (optional, [n]) receives the caller's cell at each device position,
 * cost (optional, [2]) the mean lines per warp and face slot of the caller's
 * order and of reverse Cuthill-McKee (0 when reorder is 0).  No counterpart
 * in the reference, which takes the order of its grid reader and METIS. */
int ucg_cell_order(const ucg_engine* e, int32_t* renumbered, int32_t* n2o, double* cost);

/* `nsteps` implicit pseudo-time steps toward a steady state (RUNGEKUTTA =
 * 10: IMPLICIT_TIMEs, src/time_p.f90:2783-2905, RELAX = 1): each step forms
 * RHS, the local time steps DTL of CALCULATE_CFLL at CFL `cfl`
 * (src/time_p.f90:193-333), the first-order Jacobian of CALCULATE_JACOBIAN
 * (src/implicit_fluxes.f90:12-594: diagonal sum_f vpp_f area_f / 2 + V/DTL,
 * per face (J(U_R) n / 2 - vpp / 2) area with COMPUTE_JACOBIANSE), relaxes
 * du = D^-1 (-RHS - sum_f O_f du_f) `nsweeps` times from du = 0 (RELAXATION
 * takes 10) and adds du to the state.  Every sweep reads the previous
 * sweep's corrections (the reference's in-place OpenMP loop depends on the
 * thread schedule); the steady state is the same.  Euler and Navier-Stokes,
 * any reconstruction.  A non-finite correction raises UCG_ENONPHYS at the
 * next ucg_check_health.  Queued on the handle's stream. */
int ucg_implicit_step(ucg_engine* e, double cfl, int32_t nsteps, int32_t nsweeps);

/* One physical time step dt of the dual-time scheme (RUNGEKUTTA = 11:
 * DUAL_TIME, src/time_p.f90:3035-3243): BDF2 in physical time, implicit
 * inner iterations in pseudo time (local steps at `cfl`, `nsweeps` sweeps,
 * the diagonal V (1/DTL + 1.5/dt) + ...): the first without the time term
 * (ISCOUN 1), the others with -V (1.5 U - 2 U^n + 0.5 U^{n-1}) / dt added
 * to the right-hand side, each adding its correction to the state, until
 * the correction norm sum |du| V / TOTALVOLUME, relative to its largest
 * value in this step, is at most inner_tol (RESLIMIT) or max_inner
 * iterations (UPPERLIMIT) are done; *inner_iters (optional) receives their
 * number.  Then U^{n-1} <- U^n <- U.  The history (U^n, U^{n-1}) starts as
 * the state of the first call after ucg_set_state (IT = RESTART).
 * Synchronous (one 8-byte read per inner iteration). */
int ucg_dual_time_step(ucg_engine* e, double dt, double cfl, int32_t max_inner, double inner_tol, int32_t nsweeps,
                       int32_t* inner_iters);

/* MOOD state after the last RK3 stage (cfg.mood 1), in the caller's cell
 * order: order[c] = IELEM(N,I)%MOOD_O, 1 where the second cascade
 * recomputed the cell at first order, 2 where only the first cascade
 * recomputed it (MUSCL), IORDER + 1 elsewhere (time_p.f90:660-680,
 * mood.f90:375-384); recalc[c] = RECALC, the cells whose reconstruction
 * may fall back to MUSCL in the next stage.  Either may be NULL.  Waits for
 * the handle's stream.  UCG_EINVAL without MOOD. */
int ucg_mood_state(ucg_engine* e, int32_t* order, int32_t* recalc);

/* Explicit dual time: one physical step dt of BDF2 (DUAL_TIME_EX,
 * src/time_p.f90:3244-3436, RUNGEKUTTA = 12) by explicit pseudo-time
 * iterations (RELAXATION_EX, :3844-3888): local steps DTL at `cfl`
 * (CALCULATE_CFLL, with CFL/3 as everywhere) from the state at the start of
 * the step, then per iteration du = -(V/dt (1.5 U - 2 U^n + 0.5 U^{n-1}) +
 * RHS(U)) dtau with dtau = (DTL/V) / (1 + 1.5 DTL/dt), U += du, until the
 * volume-weighted norm of du relative to its largest value in the step is
 * at most inner_tol (RESLIMIT) or max_inner (UPPERLIMIT) iterations are
 * done (*inner_iters, may be NULL).  Afterwards U^{n-1} <- U^n <- U and the
 * state becomes 2 U^n - U^{n-1}, the next step's first iterate.  The history
 * is shared with ucg_dual_time_step and restarts at ucg_set_state. */
int ucg_dual_time_step_explicit(ucg_engine* e, double dt, double cfl, int32_t max_inner, double inner_tol,
                                int32_t* inner_iters);

/* ---------------------------------------------------------------- partitions
 * One engine per rank of a partitioned mesh.  The rank's mesh is its owned
 * cells plus a halo: their face neighbours, every stencil member of both,
 * and the neighbours' face neighbours, numbered in increasing global index
 * (so each face keeps its owning side), with the tables of the whole mesh
 * sliced to it.  The residual of an owned cell is then that of the whole
 * mesh once the halo holds the current states.  UCNS3D exchanges cell means
 * (EXCHANGE_HIGHER, src/communications.f90:1085-1246) and partition-face
 * quadrature values (EXHBOUNDHIGHER, :1745-1956) in each stage; here the
 * deeper halo is reconstructed locally and only cell states travel.
 *
 * ucg_rk3_stage: RK3 stage `stage` (1, 2, 3) of step size dt, the same
 *   launches as the corresponding third of ucg_rk3_step (which equals the
 *   three stages in order).  UCG_EINVAL with MOOD.
 * ucg_halo_set (after ucg_upload_geometry): the rows this rank sends (owned
 *   cells, repeated per peer, in the order the peers expect) and receives
 *   (halo cells, each once), as the caller's cell indices.
 * ucg_halo_pack / ucg_halo_unpack: gather the send rows of the input state
 *   of `stage` (1: U^n, 2: U^(1), 3: U^(2)) into a DEVICE buffer
 *   [nsend][5], or scatter a DEVICE buffer [nrecv][5] into the receive rows,
 *   asynchronously on the handle's stream; the caller orders its transfer
 *   (NCCL or a device copy) on that stream.  The step of a rank is:
 *   unpack(1) <- peers' pack(1); stage 1; the same for stages 2 and 3.
 * ucg_set_cell_roles (before ucg_upload_geometry; NULL clears): per cell
 *   (caller order) 0 owned: stepped; 1 ring 1 (a face neighbour of an owned
 *   cell): reconstructed, not stepped; 2 the rest of the halo: only read.
 *   The reconstruction then covers roles 0-1, the face fluxes the faces of
 *   owned cells, the residual and the update the owned cells; rows of roles
 *   1-2 of ucg_residual and of the stepped state are unspecified until the
 *   next unpack, and the domain sums of ucg_reduce run over every local cell
 *   (sum the owned rows on the host instead).  Without roles every cell is
 *   reconstructed and stepped.
 *   The adjoint, implicit steps and MOOD refuse an engine with roles.
 * No counterpart entry points in the reference (its exchange is MPI inside
 * the time loop, src/time_p.f90:885-1027).                                 */
int ucg_set_cell_roles(ucg_engine* e, const int8_t* roles);
int ucg_rk3_stage(ucg_engine* e, int32_t stage, double dt);
int ucg_halo_set(ucg_engine* e, const int32_t* send_cells, int64_t nsend, const int32_t* recv_cells, int64_t nrecv);
int ucg_halo_pack(ucg_engine* e, int32_t stage, double* send_buf);
int ucg_halo_unpack(ucg_engine* e, int32_t stage, const double* recv_buf);

/* The cudaStream_t of the handle, as an opaque pointer. */
void* ucg_get_stream(ucg_engine* e);
/* Kernel launches issued by the handle since creation. */
int64_t ucg_launch_count(const ucg_engine* e);
/* Device bytes held by the handle. */
int64_t ucg_device_bytes(const ucg_engine* e);

int ucg_last_error(const ucg_engine* e, char* buf, int32_t len);

/* Residual of a MUSCL configuration (scheme 2, iorder 1: Euler or
 * Navier-Stokes) that allocates no memory at all.  No counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc: code that only
 * receives buffers from its own caller (a plug-in inside a host application
 * that owns the device pool), runs where the allocator is locked or
 * unavailable, or must not grow the process's device footprint.  Such a
 * caller passes everything in device-accessible memory: `geo` and `rec`
 * hold device pointers to the arrays of the layouts documented above (all
 * cells, first = 0), `u` is the state [n][5] and `rhs` receives RHS(I)%VAL
 * [n][5]; the work is queued on `stream` (a cudaStream_t, NULL = the default
 * stream) and the call returns without synchronising.
 * Scratch: the face values (and, for Navier-Stokes, the face gradients) live
 * in one fixed 64 MiB device array inside this library, which every GPU that
 * loads the library holds until the process exits; meshes of more than
 * 279,620 cells (Euler) or 82,241 cells (Navier-Stokes) are rejected with
 * UCG_EINVAL.  Every call writes all the scratch it later reads, so nothing
 * needs clearing, but all calls in the process share the array: calls that
 * overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller.  The first call in each CUDA context (the
 * device's primary context, or a context the caller made current) looks up
 * the array's device address in that context (cudaGetSymbolAddress); make
 * that first call before any stream capture.  Indices, face types and
 * boundary codes read from `geo` and `rec` on the device are checked, not
 * followed: a cell with an index out of range, a face type other than 5/6,
 * a boundary code other than 1, 2, 3, 4, 6, or (Navier-Stokes) any physical
 * boundary face gets a NaN row in rhs (and so may its face neighbours)
 * rather than a plausible-looking residual.  Returns UCG_OK, UCG_EINVAL
 * (unsupported configuration, NULL argument or too many cells) or
 * UCG_ECUDA.                                                              */
int ucg_residual_muscl_static(const ucg_config* cfg, const ucg_geometry* geo, const ucg_recon* rec,
                              const double* u, double* rhs, void* stream);
/* ---------------------------------------------------------------- adjoint
 * Discrete adjoint (VJP) and tangent (JVP) for the FP64 form of a MUSCL
 * (scheme 2, IORDER 1, Venkatakrishnan, HLLC) Euler or Navier-Stokes
 * configuration (the adjoint workload is the bump channel; Navier-Stokes
 * adds the reverse of the viscous fluxes, of the viscous least squares and
 * of the no-slip wall ghost).  ucg_residual_vjp and ucg_residual_jvp also cover
 * conserved-variable WENO and CWENO (scheme 3, EES 0 or 5, CWENO with or
 * without WENO-Z, HLLC, Euler or Navier-Stokes, FP64 form): the
 * reverse/tangent of the nonlinear weights, smoothness indicators and
 * stencil least squares, and of the MUSCL fall-back of the cells that
 * FULL = 0 or CHECKSOL send there (central polynomial, FIND_BOUNDS,
 * Venkatakrishnan, CHECKSOLX), and with Navier-Stokes of the viscous
 * fluxes at every face point, the face-point gradients and the viscous
 * least squares; the wall force and the runs below cover the same WENO and
 * CWENO configurations.  p denotes the free-stream state bc_state[5] (primitive:
 * rho, u, v, w, pressure) used by the inflow, outflow and far-field ghost
 * states.  Host arrays; [n][5] as everywhere.  Other configurations return
 * UCG_EINVAL.
 *
 * ucg_force: integrated wall pressure force in x at the current state,
 *   J = sum over faces with BC code 4 of (sum_q w_q p(u_face,q) - pres) * area
 *   * n_x, with the reconstructed face values (COMPUTEFORCE, src/io.f90:18752,
 *   inviscid part).
 * ucg_force_vjp: dJ/dU at the current state.
 * ucg_residual_vjp: mu = (dR/dU)^T lambda and, if pbar != NULL,
 *   pbar = (dR/dp)^T lambda, R the residual of ucg_residual.
 * ucg_residual_jvp: drhs = (dR/dU) du + (dR/dp) dp (dp may be NULL).
 * ucg_adjoint_run: nsteps RK3 steps of fixed dt from the current state, J at
 *   the final state, and its gradients w.r.t. the initial state (dJdU0) and
 *   p (dJdp[5]) by reverse sweeps over segments of `every` steps, each
 *   segment recomputed from its checkpoint.  The handle's state becomes the
 *   final state.
 * ucg_tangent_run: the same steps with tangents dU0 (and dp), J and
 *   dJ = <dJ/dU0, dU0> + <dJ/dp, dp> by forward mode; state as above.    */
int ucg_force(ucg_engine* e, double* fx);
int ucg_force_vjp(ucg_engine* e, double* dJdU);
/* ucg_wall_loads: COMPUTEFORCE (src/io.f90:18752-19000) in full at the
 *   current state, any scheme and precision form (not MOOD):
 *   out[6] = FX, FY, FZ, MX, MY, MZ.  Per wall face (BC code 4),
 *   SSP = sum_q w_q p_q - pres adds SSP * area * n, and with Navier-Stokes
 *   the shear SS = -sum_q mu_q (n . tau_q) w_q adds SS * area, tau from the
 *   cell's own face-point velocity gradients (ULEFTV) and mu from SUTHERLAND
 *   at the face state.  The moments are those of the pressure part about
 *   the cell centres, as the reference takes them: `centre` [n][3] (host,
 *   the caller's cell order), or NULL for zero moments.  Lift and drag
 *   coefficients follow on the host from FX, FY, FZ, the angle of attack
 *   and the free stream.  With partition roles only the faces of the stepped
 *   cells count (the ranks' sums add up to the whole mesh's).             */
int ucg_wall_loads(ucg_engine* e, const double* centre, double* out);
int ucg_residual_vjp(ucg_engine* e, const double* lambda, double* mu, double* pbar);
int ucg_residual_jvp(ucg_engine* e, const double* du, const double* dp, double* drhs);
int ucg_adjoint_run(ucg_engine* e, int32_t nsteps, double dt, int32_t every, double* J, double* dJdU0,
                    double* dJdp);
int ucg_tangent_run(ucg_engine* e, int32_t nsteps, double dt, const double* dU0, const double* dp, double* J,
                    double* dJ);
/* The same runs with the scalar output chosen: UCG_OBJ_FORCE_X the wall
 * force above, UCG_OBJ_KE the domain kinetic energy
 * J = sum_c V_c |rho u|^2 / (2 rho) (the TGV sum of time_p.f90:4145-4198
 * without its normalisation).  With the conserved-variable WENO and CWENO
 * residuals the reverse sweeps run the WENO VJP (nonlinear weights,
 * smoothness indicators, least squares, MUSCL fall-back) at every
 * recomputed stage state, and the wall force sums its quadrature points.
 * ucg_adjoint_run/ucg_tangent_run are these with UCG_OBJ_FORCE_X.         */
enum { UCG_OBJ_FORCE_X = 1, UCG_OBJ_KE = 2 };
int ucg_adjoint_run_obj(ucg_engine* e, int32_t objective, int32_t nsteps, double dt, int32_t every, double* J,
                        double* dJdU0, double* dJdp);
int ucg_tangent_run_obj(ucg_engine* e, int32_t objective, int32_t nsteps, double dt, const double* dU0,
                        const double* dp, double* J, double* dJ);
/* Average device times over `reps` evaluations at the current state (CUDA
 * events on the handle's stream), after one untimed evaluation, into ms[3]:
 * ms[0] residual (reconstruction + fluxes), ms[1] residual VJP, ms[2]
 * residual JVP (MUSCL or WENO).                                            */
int ucg_time_adjoint(ucg_engine* e, int32_t reps, double* ms);

/* Message of the last failure of ucg_create (no handle exists then). */
const char* ucg_create_error(void);

#ifdef __cplusplus
}
#endif
#endif
