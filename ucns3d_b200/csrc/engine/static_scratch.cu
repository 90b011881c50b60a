// Allocation-free residual entry point (ucg_residual_muscl_static).
//
// For callers that cannot call cudaMalloc - code that runs where device
// allocation is forbidden or unavailable (inside a host library that only
// receives buffers from its caller, an allocator-less embedded runtime, or
// after a framework has locked the device pool) - but that can hand over
// inputs and outputs in device-accessible memory.  The only scratch the
// computation needs, the face values (and, for Navier-Stokes, the face
// gradients) of every cell, lives in a fixed file-scope device array below,
// which every GPU that loads this library holds until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "device.cuh"
#include "ucns3d_gpu.h"

using namespace ucg;

namespace {

// 64 MiB of scratch: 30 doubles per cell (Euler) or 102 (Navier-Stokes).
constexpr long long kScratchDoubles = 8LL * 1024 * 1024;
constexpr int kEulerPerCell = MF * NV;          // face values
constexpr int kNSPerCell = MF * NV + MF * 12;   // + face gradients of T,u,v,w

static __device__ __align__(256) double g_scratch[kScratchDoubles];

// Device address of g_scratch, looked up once per CUDA context.  In host
// code the name g_scratch is only a host-side stand-in, never a device
// address, and a __device__ variable's address belongs to a context, not to
// a device ordinal: a caller may make its own context current
// (cuCtxCreate/cuCtxSetCurrent), and a cudaDeviceReset replaces the primary
// context.  The cache is therefore keyed by the context's unique id
// (cuCtxGetId, reached through the runtime's driver entry points, so the
// library does not link libcuda itself).
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

struct ScratchAddr {
  unsigned long long ctx_id;
  double* addr;
};

std::mutex g_mu;
ScratchAddr g_addr[64];
int g_naddr = 0, g_next = 0;
PfnCtxGetCurrent g_get_current = nullptr;
PfnCtxGetId g_get_id = nullptr;
bool g_resolved = false;

bool current_context_id(unsigned long long* id) {
  CUcontext ctx = nullptr;
  if (g_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return g_get_id(ctx, id) == CUDA_SUCCESS;
}

int scratch_in_current_context(double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_resolved) {
    g_resolved = true;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&g_get_current, 12000, cudaEnableDefault, &q1) !=
            cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess)
      g_get_current = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&g_get_id, 12000, cudaEnableDefault, &q2) !=
            cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      g_get_id = nullptr;
    cudaGetLastError();
  }
  if (!g_get_current || !g_get_id) return UCG_ECUDA;
  unsigned long long id = 0;
  const bool have_ctx = current_context_id(&id);
  if (have_ctx)
    for (int i = 0; i < g_naddr; ++i)
      if (g_addr[i].ctx_id == id) {
        *out = g_addr[i].addr;
        return UCG_OK;
      }
  // first call in this context (which this lookup creates if the thread had
  // none): the symbol's address in the current context
  void* ptr = nullptr;
  cudaError_t st = cudaGetSymbolAddress(&ptr, g_scratch);
  if (st != cudaSuccess || !ptr) {
    cudaGetLastError();
    return UCG_ECUDA;
  }
  if (!have_ctx && !current_context_id(&id)) return UCG_ECUDA;
  ScratchAddr& slot = g_naddr < 64 ? g_addr[g_naddr++] : g_addr[g_next++ % 64];
  slot.ctx_id = id;
  slot.addr = (double*)ptr;
  *out = (double*)ptr;
  return UCG_OK;
}

// MUSCL (IORDER 1) face values of one cell from the ABI-layout arrays:
// LEAST_SQUARES (gradients.f90:253-497), FIND_BOUNDS + Venkatakrishnan
// (reconstruct_p.f90:1821, 3421), CHECKSOLX (3245); for Navier-Stokes the
// viscous LSQ and face gradients (gradients.f90:502-706, SOLUTIONTRIAV2).
template <bool NS>
__global__ void k_static_recon(Problem p, ucg_geometry g, ucg_recon r, const double* __restrict__ U,
                               double* __restrict__ scratch) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.ncells) return;
  const int IM = p.imax, W = IM + 1;
  // indices come from caller memory on the device: an index out of range
  // marks the cell bad (NaN face values) instead of being followed
  int nf = g.nfaces[c];
  bool bad = nf < 1 || nf > MF;
  nf = bad ? 0 : nf;
  double u0[NV], pm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  cons2prim(p.gamma, u0, pm);
  const double t0 = pm[4] / (pm[0] * p.r_gas);
  const int32_t* st = r.stencil + c * W;
  int64_t t = r.table_id ? r.table_id[c] : c;
  if (t < 0 || t >= (r.table_id ? r.ntables : g.ncells)) {
    bad = true;
    t = 0;
  }
  const double* M = r.invmat + t * IM * 3;
  double gg[3][NV] = {}, gv[3][4] = {};
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[k + 1];
    if (y < 0 || y >= g.ncells) {
      bad = true;
      continue;
    }
    double uy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uy[v] = U[y * NV + v];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int v = 0; v < NV; ++v) gg[d][v] += M[k * 3 + d] * (uy[v] - u0[v]);
    if (NS) {
      double py[NV];
      cons2prim(p.gamma, uy, py);
      double ds[4] = {py[4] / (py[0] * p.r_gas) - t0, py[1] - pm[1], py[2] - pm[2], py[3] - pm[3]};
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < 4; ++v) gv[d][v] += M[k * 3 + d] * ds[v];
    }
  }
  double umin[NV], umax[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) umin[v] = umax[v] = u0[v];
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = g.neigh[c * MF + f];
    if (nb >= g.ncells) bad = true;
    if (nb < 0 || nb >= g.ncells) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      umin[v] = fmin(umin[v], U[nb * NV + v]);
      umax[v] = fmax(umax[v], U[nb * NV + v]);
    }
  }
  const double e = p.kappa_ven * g.minedge[c];
  const double epsi2 = e * e * e;
  double dd[MF][NV], slope[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) slope[v] = TOLBIG;
  for (int f = 0; f < nf; ++f) {
    const double* xi = g.qpoints + ((c * MF + f) * MQ) * 3;
    double b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[d] = xi[d] - g.basis_mean[c * 3 + d];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double res = b[0] * gg[0][v] + b[1] * gg[1][v] + b[2] * gg[2][v];
      dd[f][v] = (u0[v] + res) - u0[v];
      slope[v] = fmin(slope[v], venkat(dd[f][v], umin[v] - u0[v], umax[v] - u0[v], epsi2));
    }
  }
  bool first = false;
  for (int f = 0; f < nf; ++f) {
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = u0[v] + dd[f][v] * slope[v];
    first = first || jump_bad(p.gamma, pm, uf, 0.95);
  }
  double* o = scratch + c * (NS ? kNSPerCell : kEulerPerCell);
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  for (int f = 0; f < MF; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v)
      o[f * NV + v] = bad ? nan : (f < nf && !first) ? u0[v] + dd[f][v] * slope[v] : u0[v];
  if (NS) {
    const double* J = g.invccjac + c * 9;
    double* og = o + MF * NV;
    for (int f = 0; f < MF; ++f)
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          og[f * 12 + v * 3 + k] = bad ? nan : J[k] * gv[0][v] + J[3 + k] * gv[1][v] + J[6 + k] * gv[2][v];
  }
}

// Face fluxes (HLLC + viscous) summed per cell in face order; eight lanes
// per cell (CALCULATE_FLUXESHI_CONVECTIVE / _DIFFUSIVE, flux_p.f90:478, 1520).
template <bool NS>
__global__ void k_static_flux(Problem p, ucg_geometry g, const double* __restrict__ scratch, double* __restrict__ rhs) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = gid >> 3;
  const int f = (int)(gid & 7);
  const int base = (threadIdx.x & 31) & ~7;
  const int per = NS ? kNSPerCell : kEulerPerCell;
  double god[NV] = {0, 0, 0, 0, 0}, gvis[NV] = {0, 0, 0, 0, 0};
  const int nfc = c < g.ncells ? g.nfaces[c] : 0;
  const int64_t nb = c < g.ncells && f < MF ? g.neigh[c * MF + f] : -1;
  const int nf = c < g.ncells && f < MF ? g.neigh_face[c * MF + f] : 0;
  const bool in = c < g.ncells, badn = in && (nfc < 1 || nfc > MF);
  const bool ok = in && !badn && f < nfc;
  const int ft = ok ? g.face_type[c * MF + f] : 5;
  const int code = ok && nb < 0 ? g.bc[c * MF + f] : 0;
  // a physical face this path does not treat: Navier-Stokes walls and
  // boundaries (the reference's CALCULATE_BOUNDED_VISCOUS) and codes other
  // than inflow 1, outflow 2, symmetry 3, wall 4 and far field 6
  const bool unsupported = ok && nb < 0 && (NS || !(code == 1 || code == 2 || code == 3 || code == 4 || code == 6));
  if ((badn && f == 0) || (ok && (nb >= g.ncells || (nb >= 0 && (nf < 0 || nf >= MF)))) ||
      (ok && ft != 5 && ft != 6) || unsupported) {
    // count, index or code out of range in caller memory, or a face this
    // path does not treat: NaN instead of a plausible-looking residual
#pragma unroll
    for (int v = 0; v < NV; ++v) god[v] = __longlong_as_double(0x7ff8000000000000LL);
  } else if (ok) {
    const double a1 = g.face_angle[(c * MF + f) * 2], a2 = g.face_angle[(c * MF + f) * 2 + 1];
    const double rt[4] = {cos(a1), sin(a1), cos(a2), sin(a2)};
    const double* cl = scratch + c * per + f * NV;
    double crb[NV];
    const double* cr;
    if (nb >= 0) {
      cr = scratch + nb * per + nf * NV;
    } else {
      boundary_ghost(p, code, rt, cl, crb);
      cr = crb;
    }
    double a[NV], b[NV], h[NV], fl[NV];
    rot_f(rt, cr, b);
    rot_f(rt, cl, a);
    hllc(p.gamma, a, b, h);
    rot_b(rt, h, fl);
    const double ws = (ft == 5 ? p.quad_w[0] : p.tri_w[0]) * g.face_area[c * MF + f];
#pragma unroll
    for (int v = 0; v < NV; ++v) god[v] = fl[v] * ws;
    if (NS && nb >= 0) {
      double fv[NV];
      viscous_flux(p, rt, g.dih[c * MF + f], cl, cr, scratch + c * per + MF * NV + f * 12,
                   scratch + nb * per + MF * NV + nf * 12, fv, p.lamx);
#pragma unroll
      for (int v = 0; v < NV; ++v) gvis[v] = fv[v] * ws;
    }
  }
  double R[NV] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < MF; ++k)
#pragma unroll
    for (int v = 0; v < NV; ++v) R[v] = R[v] + __shfl_sync(0xffffffffu, god[v], base + k);
  if (NS) {
#pragma unroll
    for (int k = 0; k < MF; ++k)
#pragma unroll
      for (int v = 0; v < NV; ++v) R[v] = R[v] - __shfl_sync(0xffffffffu, gvis[v], base + k);
  }
  if (f == 0 && c < g.ncells)
#pragma unroll
    for (int v = 0; v < NV; ++v) rhs[c * NV + v] = R[v];
}

}  // namespace

extern "C" int ucg_residual_muscl_static(const ucg_config* cfg, const ucg_geometry* geo, const ucg_recon* rec,
                                         const double* u, double* rhs, void* stream) {
  if (!cfg || !geo || !rec || !u || !rhs) return UCG_EINVAL;
  if (cfg->scheme != 2 || cfg->iorder != 1 || cfg->ideg != 3 || cfg->admis_max != 1 || cfg->nq_quad != 1 ||
      cfg->nq_tri != 1 || cfg->limiter != 7 || cfg->riemann != 1 || (cfg->governing != 1 && cfg->governing != 2) ||
      (cfg->boundtype != 0 && cfg->boundtype != 1) || cfg->mood != 0)
    return UCG_EINVAL;
  const int64_t n = geo->ncells;
  if (n <= 0 || rec->first != 0 || rec->count != n || !rec->stencil || !rec->invmat) return UCG_EINVAL;
  const bool ns = cfg->governing == 1;
  if ((long long)n * (ns ? kNSPerCell : kEulerPerCell) > kScratchDoubles) return UCG_EINVAL;  // beyond the fixed scratch
  double* scratch = nullptr;
  int rc = scratch_in_current_context(&scratch);
  if (rc) return rc;
  Problem p{};
  p.n = n;
  p.imax = cfg->imax;
  p.gamma = cfg->gamma;
  p.prandtl = cfg->prandtl;
  p.visc = cfg->visc;
  p.r_gas = cfg->r_gas;
  p.pres = cfg->pres;
  p.rres = cfg->rres;
  p.kappa_ven = cfg->kappa_ven;
  p.lamx = cfg->lamx;
  p.quad_w[0] = cfg->quad_w[0];
  p.tri_w[0] = cfg->tri_w[0];
  for (int v = 0; v < NV; ++v) p.bc_state[v] = cfg->bc_state[v];
  p.boundtype = cfg->boundtype;
  p.governing = cfg->governing;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned b1 = (unsigned)((n + 127) / 128), b2 = (unsigned)((n * 8 + 255) / 256);
  if (ns) {
    k_static_recon<true><<<b1, 128, 0, s>>>(p, *geo, *rec, u, scratch);
    k_static_flux<true><<<b2, 256, 0, s>>>(p, *geo, scratch, rhs);
  } else {
    k_static_recon<false><<<b1, 128, 0, s>>>(p, *geo, *rec, u, scratch);
    k_static_flux<false><<<b2, 256, 0, s>>>(p, *geo, scratch, rhs);
  }
  return cudaGetLastError() == cudaSuccess ? UCG_OK : UCG_ECUDA;
}
