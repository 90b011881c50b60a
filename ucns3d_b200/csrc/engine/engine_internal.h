// Engine handle and host helpers shared by the translation units of the C
// ABI (engine.cu: handle, uploads, stage driver; adjoint.cu: discrete
// adjoint and tangent).  Not part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "device.cuh"
#include "ucns3d_gpu.h"

namespace ucg {
// the stencil least squares alone, FP64 tables (recon_f64.cu)
cudaError_t launch_lsq_f64(int iorder, const Problem& p, const double* U, cudaStream_t st);
}  // namespace ucg

namespace ucg_host {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Device layout of the per-cell table blocks (see Problem in device.cuh).
struct Layout {
  int64_t tstride = 0, istride = 0;
  int soff[8] = {0};
  int i2off = 0;
};

}  // namespace ucg_host

struct ucg_engine {
  ucg_config cfg;
  ucg_host::Layout layout;
  int64_t n = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool mixed = false;
  int QS = 1;
  std::string err;
  int64_t launches = 0;
  int64_t bytes = 0;
  bool have_geometry = false, have_state = false;
  int64_t recon_cells = 0;
  using DevBuf = ucg_host::DevBuf;
  // geometry
  DevBuf nfaces, ftype, neigh, nface, bc, qperm, rot, area, dih, vol, minedge, jinv, admis, full, qpts, bmean;
  // tables
  DevBuf sten, invmat, ind;
  // scratch and state
  DevBuf gbuf, isb, wflag, dul, ulv, fgrad, gv, prim, upad, rhs, Un, Ua, Ub, health, dt, partial, red, staging, own, fflux, vflux, qbuf;
  // MOOD (cfg.mood): RECALC, the cascade's flags and selections, MOOD_O, the candidate state
  DevBuf mprev, mflag, msel, mmus, mord, Um;
  // implicit steps (ucg_implicit_step): local time steps, inverse diagonals, face blocks, corrections
  DevBuf imp_dtl, imp_dinv, imp_off, imp_du;
  // dual time (ucg_dual_time_step): U^n and U^{n-1}, the norm's block sums
  DevBuf dual_hist, dual_part;
  bool dual_ready = false;  // the history holds the state of a step (reset by ucg_set_state)
  double totvol = 0.0;      // TOTALVOLUME
  int64_t nown = 0;
  int64_t nown_plain = 0;  // owned faces [0, nown_plain): interior and mirror; the rest other boundaries
  cudaEvent_t mark = nullptr;  // recorded after k_lsq while ucg_time_kernels runs
  bool lsq_bulk = false;       // UCG_LSQ_BULK=1 at ucg_create: k_lsq_tma instead of k_lsq
  bool wface = false;          // IORDER 4 conserved WENO: face values one warp per variable (k_wface)
  long lsq_wait = -1;          // polls of a k_lsq_tma stage wait (ucg_set_wait_limit; < 0 the default)
  std::vector<uint8_t> recon_done;  // per cell, for ucg_upload_recon chunks
  std::vector<int8_t> admis_h;      // ADMIS per cell, for the stencil checks of ucg_upload_recon
  std::vector<int32_t> neigh_h;     // [n][6] face neighbours (host copy, adjoint set-up)
  std::vector<int32_t> sten1_h;     // [n][IMAX+1] first stencil (host copy, MUSCL IORDER 1 only)
  // cell renumbering (cfg.reorder): device cell c holds the caller's cell
  // n2o[c]; o2n is the inverse.  Empty when the caller's order is kept.
  std::vector<int32_t> n2o, o2n;
  DevBuf d_n2o, permbuf;            // n2o on the device; [n][5] staging of permuted transfers
  // partition roles (ucg_set_cell_roles, caller order; empty: every cell
  // is stepped): the device order holds the stepped cells [0, n_update),
  // then the other reconstructed cells [n_update, n_recon), then the rest
  std::vector<int8_t> roles;
  int64_t n_recon = 0, n_update = 0;
  // halo lists of a partition (ucg_halo_set), in the engine's order
  DevBuf halo_send, halo_recv;
  DevBuf wl_buf;  // ucg_wall_loads: [6][nown] face columns, sums, cell centres
  int64_t halo_nsend = 0, halo_nrecv = 0;
  double cost_caller = 0.0, cost_rcm = 0.0;  // gather cost of both orders (reorder 1)
  // discrete adjoint / tangent (adjoint.cu)
  bool adj_ready = false;
  DevBuf adj_face, adj_contrib, adj_rptr, adj_rsrc, adj_lam, adj_mu, adj_pface, adj_tflux, adj_tdul, adj_tU,
      adj_fcell, adj_traj, adj_bar, adj_tmp, adj_fwd, adj_gadj, adj_tgr;
  // discrete adjoint of the WENO reconstruction (adjoint_weno.cu)
  bool adjw_ready = false;
  DevBuf adjw_face, adjw_gbar, adjw_scr, adjw_self, adjw_contrib, adjw_rptr, adjw_rsrc, adjw_lam, adjw_mu,
      adjw_pface, adjw_tmp, adjw_gpt, adjw_gvb, adjw_tfg;
};

namespace ucg_host {

#define CK(call)                                             \
  do {                                                       \
    cudaError_t st_ = (call);                                \
    if (st_ != cudaSuccess) return cuda_fail(e, st_, #call); \
  } while (0)

int fail(ucg_engine* e, int code, const std::string& msg);
int cuda_fail(ucg_engine* e, cudaError_t st, const char* where);
int alloc(ucg_engine* e, DevBuf& b, size_t bytes);
void release(DevBuf& b);
ucg::Problem make_problem(ucg_engine* e);
bool ready(ucg_engine* e);
int launch_recon(ucg_engine* e, const ucg::Problem& p, const double* U);
int launch_flux(ucg_engine* e, const ucg::Problem& p, int mode, const double* Uc, const double* Un, double* Uo,
                double dt, bool check = true);
// the face fluxes alone (k_face; with p.msel only the faces of the selected cells)
int launch_faces(ucg_engine* e, const ucg::Problem& p, const double* Uc);
int rk3(ucg_engine* e, double dt, bool dt_dev);
// [n][5] FP64 arrays between the caller's cell order on the host and the
// device order (a plain copy when the engine keeps the caller's order);
// both leave the copy queued on the handle's stream
int cells_in(ucg_engine* e, double* dev_dst, const double* host_src);
int cells_out(ucg_engine* e, double* host_dst, const double* dev_src);
// reconstruction tables (engine.cu): stencil upload, staged expansion of
// per-table FP64 blocks, bookkeeping; the device set-up (setup.cu) fills
// the staging buffer itself
int upload_stencils(ucg_engine* e, int64_t first, int64_t count, const int32_t* stencil, DevBuf& rowbuf,
                    const int32_t** d_rowmap);
int expand_tables(ucg_engine* e, int64_t first, int64_t count, int64_t ntab, const int32_t* d_tid,
                  const int32_t* d_rowmap, const std::function<int(int, int64_t, int64_t, double*)>& fill);
void mark_recon(ucg_engine* e, int64_t first, int64_t count);
// frees the adjoint buffers (adjoint.cu)
void adjoint_release(ucg_engine* e);
// reverse of the WENO post-processing and least squares (adjoint_weno.cu)
int launch_weno_adjoint(ucg_engine* e, const ucg::Problem& p, const double* U, const double* adjF, double* gbar,
                        double* scr, double* selfc, double* contrib);
// tangent of the WENO face values from the tangent stencil polynomials dG
int launch_weno_tangent(ucg_engine* e, const ucg::Problem& p, const double* U, const double* dU, const double* dG,
                        double* tdul);
// Navier-Stokes WENO: the face-point gradient adjoints gpt back through the
// viscous coefficients and least squares into the slots of contrib; the
// tangent of the face-point gradients (tfg, k_visc_facegrad's layout)
int launch_weno_visc_adjoint(ucg_engine* e, const ucg::Problem& p, const double* U, const double* gpt, double* gvb,
                             double* contrib);
int launch_weno_visc_tangent(ucg_engine* e, const ucg::Problem& p, const double* U, const double* dU, double* dgv,
                             double* tfg);

}  // namespace ucg_host
