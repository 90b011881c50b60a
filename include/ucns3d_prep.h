/*
 * ucns3d_prep.h - host-side set-up for the explicit residual engine.
 *
 * In UCNS3D the set-up runs in Fortran before the time loop
 * (src/main.f90:151-767): neighbours (NEIGHBOURSS, src/grid_p.f90:1850),
 * geometry (GEOMETRY_CALC, src/grid_t.f90:1192), stencils (DETSTENX,
 * STENCIILSX, STENCILS, src/grid_p.f90:3435, 5544, 6452), reference frames
 * (LOCALISE_STEN2, src/local_pt.f90:935) and the reconstruction tables
 * (PRESTORE_1, src/prestore.f90:16-818, 1529-1673).  A driver that keeps that
 * code packs its tables into ucg_geometry / ucg_recon itself.  This library
 * is for callers without the Fortran set-up: it builds seeded synthetic
 * meshes and computes the same tables in FP64 on the host (OpenMP), and
 * evaluates cell-averaged initial conditions (INITIALISE, src/init_p.f90:14).
 */
#ifndef UCNS3D_PREP_H
#define UCNS3D_PREP_H

#include <stdint.h>
#include "ucns3d_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ucp_mesh ucp_mesh;

/* Boundary codes of UCNS3D (src/bc_p.f90): 1 inflow, 2 outflow,
 * 3 symmetry, 4 wall, 6 far field; periodic sides carry no code.
 * bc[6] = codes of the x-, x+, y-, y+, z-, z+ sides of a box.             */

/* nx*ny*nz hexahedra on the box origin + [0,L].                          */
ucp_mesh* ucp_box_hex(int32_t nx, int32_t ny, int32_t nz, const double L[3],
                      const double origin[3], const int32_t periodic[3],
                      const int32_t bc[6]);

/* The same box with every hexahedron split into 6 tetrahedra about its
 * main diagonal; vertices are moved by a seeded uniform +-jitter*h per
 * coordinate (vertices on non-periodic sides stay on their side).         */
ucp_mesh* ucp_box_tet(int32_t nx, int32_t ny, int32_t nz, const double L[3],
                      const double origin[3], const int32_t periodic[3],
                      const int32_t bc[6], double jitter, uint64_t seed);

/* Channel [0,3]x[0,1] with a sinusoidal bump of height `bump` on the lower
 * wall over x in [1,2]; nx*ny quadrilaterals, each split into 2 triangles
 * with probability split_frac (seeded), extruded `nlayers` layers of
 * thickness dz.  Codes: x- inflow 1, x+ outflow 2, y- and y+ wall 4,
 * z- and z+ symmetry 3.  Cells: hexahedra and triangular prisms.          */
ucp_mesh* ucp_bump_channel(int32_t nx, int32_t ny, int32_t nlayers, double bump,
                           double dz, double split_frac, uint64_t seed);

/* Periodic box n^3 on [0,L]^3: hexahedra for z < L/2; above, each z-layer
 * of hexahedra is split, by a seeded choice per layer, into 6 tetrahedra or
 * into 2 prisms per hexahedron; the layer just above the hexahedra is prisms
 * with quadrilateral top and bottom so that every face is conforming.     */
ucp_mesh* ucp_mixed_box(int32_t n, double L, uint64_t seed);

/* UCNS3D's ASCII grid files <prefix>GRID.vrt, GRID.cel, GRID.bnd (the
 * reader of OPEN_ARBITRARY / FIND_SHAPE / READ_BOUND, src/io.f90:4157-4304,
 * src/grid_p.f90:1652-1743, src/bc_p.f90:36-130): hexahedra, tetrahedra,
 * pyramids and prisms in the 8-node encoding with repeated nodes, boundary
 * faces with their codes.  Periodic faces (codes 5, 50) are paired as
 * APPLY_BOUNDARY does (src/bc_p.f90:499-620): a face whose centroid lies on
 * the low side of the nodes' bounding box in one axis pairs with the face of
 * the same shape on the high side whose centroid has the same other two
 * coordinates (within 1e-13 of the coordinates' size), the axis becomes
 * periodic with the box's extent as the period (XPER, YPER, ZPER of
 * src/io.f90:4977-4979), and the two faces meet like interior faces.  A
 * periodic face off the box's sides or without a partner is refused.  The
 * mesh is then prepared like any other; every other boundary face must
 * appear in GRID.bnd.  ucp_write_grid writes a prepared mesh in the same
 * format (coordinates with 17 significant digits, so a read-back prepares
 * to the same tables); on a periodic mesh the faces on the periodic sides
 * get code 5 and the nodes a cell sees across them image nodes of their
 * own, and a mesh whose periodic faces are off the box's sides (a jittered
 * periodic box) is refused with UCG_EINVAL.                               */
ucp_mesh* ucp_read_grid(const char* prefix);
int32_t ucp_write_grid(const ucp_mesh* m, const char* prefix);

typedef struct ucp_scheme {
  int32_t scheme;     /* 2 MUSCL, 3 WENO                                     */
  int32_t iorder;     /* 1..4                                                */
  int32_t ees;        /* 0 WENO, 5 CWENO                                     */
  int32_t nthreads;   /* OpenMP threads, 0 = default                         */
} ucp_scheme;

/* Connectivity, geometry, stencils and tables for the given scheme.        */
int32_t ucp_prepare(ucp_mesh* m, const ucp_scheme* s);
/* The same without the tables (basis means, pseudo-inverses, smoothness
 * matrices): ucp_geometry then gives basis_mean NULL and ucp_recon only
 * the stencils; the engine builds the tables with ucg_build_recon from
 * ucp_shapes.                                                              */
int32_t ucp_prepare_geometry(ucp_mesh* m, const ucp_scheme* s);
/* Pointers into the mesh for ucg_build_recon (valid until ucp_free).       */
int32_t ucp_shapes(const ucp_mesh* m, ucg_shapes* out);

int64_t ucp_ncells(const ucp_mesh* m);
/* Sizes and face weights to copy into ucg_config.                          */
int32_t ucp_fill_config(const ucp_mesh* m, ucg_config* cfg);
/* Pointers into arrays owned by the mesh (valid until ucp_free).           */
int32_t ucp_geometry(const ucp_mesh* m, ucg_geometry* g);
int32_t ucp_recon(const ucp_mesh* m, ucg_recon* r);
/* Number of distinct matrix sets found (cells with identical stencil
 * geometry share one).                                                     */
int64_t ucp_ntables(const ucp_mesh* m);

/* Cell centres [n][3].                                                     */
int32_t ucp_cell_centres(const ucp_mesh* m, double* xyz);

enum { UCP_IC_TGV = 95, UCP_IC_VORTEX = 201, UCP_IC_UNIFORM = 1 };
/* Cell averages of the conserved variables, [n][5], by volume quadrature.
 * UCP_IC_TGV      params: gamma, p0, rho0                (profile.f90:253)
 * UCP_IC_VORTEX   params: gamma, strength, u_inf, v_inf, w_inf, xc, yc, zc,
 *                 time, Lx, Ly, Lz (isentropic vortex about the z axis,
 *                 advected; periodic images summed over the box)
 * UCP_IC_UNIFORM  params: gamma, rho, u, v, w, p                            */
int32_t ucp_initial_condition(const ucp_mesh* m, int32_t kind, const double* params,
                              int32_t nparams, double* u);

const char* ucp_last_error(void);
void ucp_free(ucp_mesh* m);

#ifdef __cplusplus
}
#endif
#endif
