// Stage-wise stepping and halo transfers for one partition of a larger mesh.
//
// UCNS3D runs each MPI rank on a METIS partition and, in every RK stage,
// exchanges the cell means of the halo (EXCHANGE_HIGHER,
// src/communications.f90:1085-1246) and the face-quadrature values of the
// partition boundary (EXHBOUNDHIGHER, :1745-1956) before the fluxes.  Here a
// rank's engine holds its owned cells, their face neighbours, every stencil
// member of both and the face neighbours of the neighbours, so that the face
// values on both sides of each owned face are reconstructed locally; only
// cell states cross between ranks, once per stage.  These entry points give
// the stage boundary (ucg_rk3_stage) and the device-side gather and scatter
// of the halo rows of a stage's input state (ucg_halo_pack / _unpack) on the
// engine's stream; the transfer itself (NCCL, or a copy between two handles
// on one device) is the caller's, ordered on that stream.
#include "engine_internal.h"

#include "device.cuh"

using namespace ucg_host;

namespace {

using ucg::NV;

// out[i][v] = U[idx[i]][v]; one thread per element, so the writes coalesce
__global__ void k_halo_pack(const double* __restrict__ U, const int32_t* __restrict__ idx, int64_t n,
                            double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * NV) return;
  const int64_t i = t / NV;
  const int v = (int)(t - i * NV);
  out[t] = U[(int64_t)idx[i] * NV + v];
}

// U[idx[i]][v] = in[i][v]
__global__ void k_halo_unpack(double* __restrict__ U, const int32_t* __restrict__ idx, int64_t n,
                              const double* __restrict__ in) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * NV) return;
  const int64_t i = t / NV;
  const int v = (int)(t - i * NV);
  U[(int64_t)idx[i] * NV + v] = in[t];
}

// the input state of RK stage `stage` (1: U^n, 2: U^(1), 3: U^(2))
double* stage_state(ucg_engine* e, int stage) {
  return (double*)(stage == 1 ? e->Un.p : stage == 2 ? e->Ua.p : e->Ub.p);
}

// caller cell indices -> the engine's order, checked against [0, n)
int map_cells(ucg_engine* e, const int32_t* cells, int64_t count, std::vector<int32_t>& out, const char* what) {
  out.resize((size_t)count);
  for (int64_t i = 0; i < count; ++i) {
    const int32_t c = cells[i];
    if (c < 0 || c >= e->n) return fail(e, UCG_EINVAL, std::string(what) + " cell index out of range");
    out[(size_t)i] = e->o2n.empty() ? c : e->o2n[(size_t)c];
  }
  return UCG_OK;
}

}  // namespace

extern "C" {

int ucg_set_cell_roles(ucg_engine* e, const int8_t* roles) {
  if (!e) return UCG_EINVAL;
  if (e->have_geometry) return fail(e, UCG_ESTATE, "the roles go before the geometry upload");
  if (!roles) {
    e->roles.clear();
    return UCG_OK;
  }
  if (e->cfg.mood) return fail(e, UCG_EINVAL, "partition roles and MOOD do not combine");
  int64_t stepped = 0;
  for (int64_t c = 0; c < e->n; ++c) {
    if (roles[c] < 0 || roles[c] > 2) return fail(e, UCG_EINVAL, "a role is 0, 1 or 2");
    stepped += roles[c] == 0;
  }
  if (!stepped) return fail(e, UCG_EINVAL, "no cell has role 0");
  e->roles.assign(roles, roles + e->n);
  return UCG_OK;
}

int ucg_rk3_stage(ucg_engine* e, int32_t stage, double dt) {
  if (!e || stage < 1 || stage > 3 || !(dt > 0)) return fail(e, UCG_EINVAL, "bad argument");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (e->cfg.mood)
    return fail(e, UCG_EINVAL, "stage-wise steps cover configurations without MOOD (its fix-up reaches two "
                               "neighbour layers past the stage's input)");
  cudaSetDevice(e->device);
  ucg::Problem p = make_problem(e);
  double* Un = (double*)e->Un.p;
  double* Ua = (double*)e->Ua.p;
  double* Ub = (double*)e->Ub.p;
  // the three calls of rk3(), one per stage
  double* in = stage_state(e, stage);
  double* out = stage == 1 ? Ua : stage == 2 ? Ub : Un;
  int rc = launch_recon(e, p, in);
  return rc ? rc : launch_flux(e, p, stage, in, Un, out, dt);
}

int ucg_halo_set(ucg_engine* e, const int32_t* send_cells, int64_t nsend, const int32_t* recv_cells, int64_t nrecv) {
  if (!e || nsend < 0 || nrecv < 0 || (nsend && !send_cells) || (nrecv && !recv_cells))
    return fail(e, UCG_EINVAL, "bad argument");
  if (!e->have_geometry)  // the engine's cell order, which the lists are mapped to, is fixed there
    return fail(e, UCG_ESTATE, "set the halo lists after ucg_upload_geometry");
  std::vector<int32_t> s, r;
  int rc = map_cells(e, send_cells, nsend, s, "send");
  rc = rc ? rc : map_cells(e, recv_cells, nrecv, r, "receive");
  if (rc) return rc;
  // a received row must have one source: duplicates in the receive list would
  // make the scatter's result depend on the order of its writes
  std::vector<uint8_t> seen((size_t)e->n, 0);
  for (int32_t c : r) {
    if (seen[(size_t)c]) return fail(e, UCG_EINVAL, "a cell appears twice in the receive list");
    seen[(size_t)c] = 1;
  }
  cudaSetDevice(e->device);
  release(e->halo_send);
  release(e->halo_recv);
  e->halo_nsend = e->halo_nrecv = 0;
  if (nsend) {
    if ((rc = alloc(e, e->halo_send, (size_t)nsend * 4))) return rc;
    CK(cudaMemcpyAsync(e->halo_send.p, s.data(), (size_t)nsend * 4, cudaMemcpyHostToDevice, e->stream));
  }
  if (nrecv) {
    if ((rc = alloc(e, e->halo_recv, (size_t)nrecv * 4))) return rc;
    CK(cudaMemcpyAsync(e->halo_recv.p, r.data(), (size_t)nrecv * 4, cudaMemcpyHostToDevice, e->stream));
  }
  CK(cudaStreamSynchronize(e->stream));  // the host lists go out of scope
  e->halo_nsend = nsend;
  e->halo_nrecv = nrecv;
  return UCG_OK;
}

int ucg_halo_pack(ucg_engine* e, int32_t stage, double* send_buf) {
  if (!e || stage < 1 || stage > 3 || (e->halo_nsend && !send_buf)) return fail(e, UCG_EINVAL, "bad argument");
  if (!e->have_state) return fail(e, UCG_ESTATE, "no state set");
  if (!e->halo_nsend) return UCG_OK;
  cudaSetDevice(e->device);
  const int64_t m = e->halo_nsend * NV;
  k_halo_pack<<<(unsigned)((m + 255) / 256), 256, 0, e->stream>>>(stage_state(e, stage),
                                                                  (const int32_t*)e->halo_send.p,
                                                                  e->halo_nsend, send_buf);
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}

int ucg_halo_unpack(ucg_engine* e, int32_t stage, const double* recv_buf) {
  if (!e || stage < 1 || stage > 3 || (e->halo_nrecv && !recv_buf)) return fail(e, UCG_EINVAL, "bad argument");
  if (!e->have_state) return fail(e, UCG_ESTATE, "no state set");
  if (!e->halo_nrecv) return UCG_OK;
  cudaSetDevice(e->device);
  const int64_t m = e->halo_nrecv * NV;
  k_halo_unpack<<<(unsigned)((m + 255) / 256), 256, 0, e->stream>>>(stage_state(e, stage),
                                                                    (const int32_t*)e->halo_recv.p,
                                                                    e->halo_nrecv, recv_buf);
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}

}  // extern "C"
