// mhc_capi.cu -- C ABI of the MaHyCo B200 library.
//
// Every launch goes through an Engine: a set of cases, their device
// descriptors and one work list per (group, phase).  A case created with
// mhc_case_create runs on a private engine holding only itself; a batch
// (mhc_batch_*) runs many cases of uneven sizes through one persistent
// launch per phase.  Cases are grouped by everything that selects a kernel
// template: dimension, number of environments, remap on/off, the set of
// one-cell-thick axes and the current sweep rotation.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/mahyco_b200.h"
#include "mhc_engine.cuh"

namespace {
thread_local std::string g_err;
}  // namespace

int mhc::set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

namespace mhc {
// a node vector field's three component arrays interleaved (x, y, z per
// node) on the device, so that it comes back in one copy
__global__ void kb_interleave3(const double* __restrict__ a, const double* __restrict__ b,
                               const double* __restrict__ c, double* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    out[3 * i] = a[i];
    out[3 * i + 1] = b[i];
    out[3 * i + 2] = c[i];
  }
}
// NewHypoModel::initElasto (NewHypoModelService.cc:13-26) and the initial
// density the equations of state keep (MieGruneisenEOSService.cc:31 and the
// like): F = I, rho_0 = the density after the initialisation
__global__ void kb_hyper_init(double* __restrict__ hf, const double* __restrict__ rho, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 9; ++q) hf[q * n + i] = (q % 4 == 0) ? 1. : 0.;
    hf[9 * n + i] = rho[i];
  }
}
}  // namespace mhc

namespace {

int pinned_get(size_t bytes, void** out);
void pinned_put(void* p, size_t bytes);


bool case_elasto(const mhc_case* h) { return h->P.env[0].elasto_model != 0; }
bool case_hourglass(const mhc_case* h) { return !h->P.with_projection && h->P.coef_antiderive != 0.; }
bool case_cell_bcs(const mhc_case* h) {
  for (int b = 0; b < h->P.nb_bc; ++b)
    if (h->P.bc[b].kind >= MHC_BC_DENSITY && h->P.bc[b].kind <= MHC_BC_PRESSURE) return true;
  return false;
}

// -- list building -----------------------------------------------------------
int engine_rebuild(Engine* e) {
  if (!e->dirty) return MHC_OK;
  if (e->nsm == 0) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  const int nc = (int)e->cases.size();
  // descriptors
  if (nc > e->desc_cap) {
    if (e->d_desc) CK(cudaFreeAsync(e->d_desc, e->stream));
    e->desc_cap = std::max(nc, 2 * e->desc_cap);
    CK(cudaMallocAsync((void**)&e->d_desc, e->desc_cap * sizeof(CaseDesc), e->stream));
  }
  std::vector<CaseDesc> desc(nc);
  for (int i = 0; i < nc; ++i) {
    mhc_case* h = e->cases[i];
    h->slot = i;
    desc[i].M = h->M;
    desc[i].F = h->F;
    desc[i].P = h->d_params;
  }
  // groups
  std::map<std::tuple<int, int, int, int, int, int, int, int, int, int, int, int, int, int, int, int>, int> gidx;
  e->groups.clear();
  for (int i = 0; i < nc; ++i) {
    mhc_case* h = e->cases[i];
    // 0 Lagrangian, 1 Full Euler remap, 2 per-axis Euler remap
    const int es = h->P.is_euler_scheme;
    int euler = h->P.with_projection ? ((es >= MHC_EULER_X && es <= MHC_EULER_Z) ? 2 : 1) : 0;
    int sens = (int)((h->it_host - 1) % h->DIM);
    const int el = case_elasto(h) ? 1 : 0, hg = case_hourglass(h) ? 1 : 0;
    const int lim = node_sweep_mode(h->P), clim = cell_sweep_mode(h->P);
    int cols, tile, ncols, ntile;
    sweep_masks(h, e->cell_layout, false, cols, tile);
    sweep_masks(h, e->node_layout, true, ncols, ntile);
    const int cbc = case_cell_bcs(h) ? 1 : 0;
    const int adv = h->P.sans_lagrange ? 1 : 0, csts = (h->P.schema_csts && h->P.with_projection) ? 1 : 0;
    auto key = std::make_tuple(h->DIM, h->NE, euler, skip_mask(h), sens, el, hg, lim, clim, cols, ncols, cbc, tile, ntile,
                               adv, csts);
    auto it = gidx.find(key);
    if (it == gidx.end()) {
      Group g;
      g.DIM = h->DIM; g.NE = h->NE; g.EULER = euler; g.skip = skip_mask(h); g.it0 = h->it_host;
      g.EL = el; g.HG = hg; g.LIM = lim; g.CLIM = clim; g.COLS = cols; g.NCOLS = ncols; g.CBC = cbc; g.TILE = tile; g.NTILE = ntile;
      g.ADV = adv;
      g.CSTS = csts;
      gidx[key] = (int)e->groups.size();
      e->groups.push_back(g);
      it = gidx.find(key);
    }
    e->groups[it->second].members.push_back(i);
  }
  // per group: member case indices, then for every phase the prefix sums
  // of the members' virtual blocks
  std::vector<int> ints;
  for (Group& g : e->groups) {
    const size_t oc = ints.size();
    for (int c : g.members) ints.push_back(c);
    g.cases.off_cases = oc;
    g.cases.n = (int)g.members.size();
    auto phase = [&](DevList& L, int ph) -> bool {
      L.off_cases = oc;
      L.n = (int)g.members.size();
      L.off_start = ints.size();
      long long tot = 0;
      for (int c : g.members) {
        ints.push_back((int)tot);
        int gx, gy, gz;
        phase_grid(ph, e->cases[c]->M, gx, gy, gz);
        tot += (long long)gx * gy * gz;
      }
      L.total = (int)tot;
      return tot <= INT_MAX;
    };
    bool ok = phase(g.init_cells, PH_CELLS) && phase(g.init_nodes, PH_NODES) && phase(g.lag_cells, PH_CELLS) &&
              phase(g.fin_cells, PH_CELLS) && phase(g.fin_nodes, PH_NODES) && phase(g.dt, PH_CELLS) &&
              phase(g.lag_nodes, PH_NODES);
    for (int D = 0; D < g.DIM; ++D)
      ok = ok && phase(g.sw_cells[D], group_cell_phase(g.CLIM, g.COLS, g.TILE, D)) &&
           phase(g.sw_nodes[D], group_node_phase(g.LIM, g.NCOLS, g.NTILE, D));
    if (!ok) return set_err(MHC_ERR_ARG, "more than 2^31 blocks in one phase of a batch");
  }
  if (ints.size() > e->ints_cap) {
    if (e->d_ints) CK(cudaFreeAsync(e->d_ints, e->stream));
    e->ints_cap = std::max(ints.size(), 2 * e->ints_cap);
    CK(cudaMallocAsync((void**)&e->d_ints, e->ints_cap * sizeof(int), e->stream));
  }
  // upload through the page-locked staging block: the copies are truly
  // asynchronous, so the host does not wait for the work in flight; the
  // block is reused once the previous upload has landed
  const size_t db = nc * sizeof(CaseDesc), ib = ints.size() * sizeof(int);
  if (!e->stage_ev) CK(cudaEventCreateWithFlags(&e->stage_ev, cudaEventDisableTiming));
  else CK(cudaEventSynchronize(e->stage_ev));
  if (db + ib > e->stage_cap) {
    if (e->h_stage) pinned_put(e->h_stage, e->stage_cap);
    e->h_stage = nullptr;
    e->stage_cap = std::max(db + ib, 2 * e->stage_cap);
    if (int pr = pinned_get(e->stage_cap, (void**)&e->h_stage)) return pr;
  }
  if (db) {
    memcpy(e->h_stage, desc.data(), db);
    CK(cudaMemcpyAsync(e->d_desc, e->h_stage, db, cudaMemcpyHostToDevice, e->stream));
  }
  if (ib) {
    memcpy(e->h_stage + db, ints.data(), ib);
    CK(cudaMemcpyAsync(e->d_ints, e->h_stage + db, ib, cudaMemcpyHostToDevice, e->stream));
  }
  CK(cudaEventRecord(e->stage_ev, e->stream));
  e->dirty = false;
  e->cycles_since_build = 0;
  if (e->graph) {
    CK(cudaStreamSynchronize(e->stream));  // no replay of the old graph in flight
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  return MHC_OK;
}

// RIDER velocity fields (RIDERService.cc:141-172 and 255-285): evaluated on
// the host with the C library's sin, cos and atan2, the functions the
// reference's own initialisation calls (the device versions differ from
// them by an ulp here and there), and written over the node velocities and
// prescribed velocities kb_init_nodes left; stream-ordered after it.  Pi is
// TypesMahyco.h:42's 3.14159265359.
int rider_upload(mhc_case* h, cudaStream_t st) {
  const mhc_case_params& P = h->P;
  const Mesh& M = h->M;
  const long long NN = M.nnode;
  const double Pi = 3.14159265359;
  const int kind = (P.cas_test - MHC_TEST_MONO_RIDER_TX) % 8;  // Tx Ty T45 Rotation Vortex Deformation (+2 reverse)
  std::vector<double> v(3 * NN, 0.0);
  for (long long n = 0; n < NN; ++n) {
    const long long i = n % M.nnx, r = n / M.nnx, j = r % M.nny, k = r / M.nny;
    const double x = M.o[0] + i * M.h[0], y = M.o[1] + j * M.h[1], z = M.dim == 3 ? M.o[2] + k * M.h[2] : 0.;
    (void)z;
    double vx = 0.0, vy = 0.0;
    if (kind == 0) vx = 1.;
    if (kind == 1) vy = 1.;
    if (kind == 2) { vx = 1.0; vy = 1.0; }
    if (kind == 3) {
      const double ddx = x - 0.5, ddy = y - 0.5;
      const double theta = std::atan2(ddy, ddx);
      const double rr = std::sqrt(ddx * ddx + ddy * ddy);
      const double omega = 4. * Pi;
      vx = -rr * omega * std::sin(omega * 0. + theta);
      vy = rr * omega * std::cos(omega * 0. + theta);
    }
    if (kind == 4 || kind == 6) {
      vx = -2. * std::cos(Pi * y) * std::sin(Pi * y) * std::sin(Pi * x) * std::sin(Pi * x);
      vy = 2. * std::cos(Pi * x) * std::sin(Pi * x) * std::sin(Pi * y) * std::sin(Pi * y);
    }
    if (kind == 5 || kind == 7) {
      const double ddx = x + 0.5, ddy = y + 0.5;
      vx = std::sin(4. * Pi * ddx) * std::sin(4. * Pi * ddy);
      vy = std::cos(4. * Pi * ddx) * std::cos(4. * Pi * ddy);
    }
    v[n] = vx;
    v[NN + n] = vy;
  }
  // pageable sources: each copy is staged before the call returns
  const size_t b = NN * sizeof(double);
  CK(cudaMemcpyAsync(h->F.vx, v.data(), b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->F.vy, v.data() + NN, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->F.vz, v.data() + 2 * NN, b, cudaMemcpyHostToDevice, st));
  if (h->F.v0) CK(cudaMemcpyAsync(h->F.v0, v.data(), 3 * b, cudaMemcpyHostToDevice, st));
  return MHC_OK;
}

// -- phase launches -------------------------------------------------------------
void launch_init(Engine* e) {
  for (Group& g : e->groups) {
    DISPATCH_GROUP(g, (plaunch(e, kb_init_cells<DIM_, NE_>, CT, 0, g.init_cells)));
    if (!g.EULER && !g.ADV) {
      // the temperature of a Lagrangian run (initEOS)
      DISPATCH_GROUP(g, (plaunch(e, kb_eref_candidates<DIM_, NE_>, CT, 0, g.init_cells, -1)));
      DISPATCH_GROUP(g, (plaunch(e, kb_init_temperature<DIM_, NE_>, CT, 0, g.init_cells, -1)));
    }
    DISPATCH_GROUP(g, (plaunch(e, kb_init_nodes<DIM_>, CT, 0, g.init_nodes)));
  }
  for (mhc_case* h : e->cases)
    if (h->F.hf) kb_hyper_init<<<(unsigned)((h->M.ncell + 255) / 256), 256, 0, e->stream>>>(h->F.hf, h->F.rho, h->M.ncell);
}

template <int DIM, bool EL, bool HG, bool LAG, bool CSTS = false>
void lag_nodes_launch(Engine* e, Group& g) {
  plaunch(e, kb_lagrange_nodes<DIM, EL, HG, LAG, CSTS>, CT, 0, g.lag_nodes);
  if (HG) plaunch(e, kb_hourglass<DIM>, CT, 0, g.lag_nodes);
}

// elasto-plasticity and the anti-hourglass correction come with Lagrangian
// runs only (validated at creation)
template <int DIM>
void lag_nodes_dispatch(Engine* e, Group& g) {
  if (g.EULER && g.CSTS) {
    lag_nodes_launch<DIM, false, false, false, true>(e, g);
  } else if (g.EULER && g.EL) {
    lag_nodes_launch<DIM, true, false, false>(e, g);
  } else if (g.EULER) {
    lag_nodes_launch<DIM, false, false, false>(e, g);
  } else if (g.EL) {
    if (g.HG) lag_nodes_launch<DIM, true, true, true>(e, g);
    else lag_nodes_launch<DIM, true, false, true>(e, g);
  } else {
    if (g.HG) lag_nodes_launch<DIM, false, true, true>(e, g);
    else lag_nodes_launch<DIM, false, false, true>(e, g);
  }
}

void launch_lagrange_nodes(Engine* e) {
  StageTimer tm(e, MHC_STAGE_LAGRANGE_NODES);
  for (Group& g : e->groups) {
    if (g.ADV) {
      // sans-lagrange: prescribed velocities (validated without cell
      // boundary conditions)
      if (g.DIM == 2) plaunch(e, kb_advect_nodes<2>, CT, 0, g.lag_nodes);
      else plaunch(e, kb_advect_nodes<3>, CT, 0, g.lag_nodes);
      continue;
    }
    if (g.DIM == 2) lag_nodes_dispatch<2>(e, g);
    else lag_nodes_dispatch<3>(e, g);
    if (g.CBC) {
      // cell variables of the boundary conditions, after the node pass
      if (g.DIM == 2) {
        plaunch(e, kb_node_bcs<2>, CT, 0, g.lag_nodes);
        plaunch(e, kb_cell_bcs<2>, CT, 0, g.lag_cells);
      } else {
        plaunch(e, kb_node_bcs<3>, CT, 0, g.lag_nodes);
        plaunch(e, kb_cell_bcs<3>, CT, 0, g.lag_cells);
      }
    }
  }
}

void launch_lagrange_cells(Engine* e) {
  StageTimer tm(e, MHC_STAGE_LAGRANGE_CELLS);
  for (Group& g : e->groups) {
    if (g.EL && g.EULER) {
      // elasto cases with the remap: the deviator and plastic strains packed
      // among the projected variables
      if (g.DIM == 2) plaunch(e, kb_lagrange_cells<2, 1, true, true>, CT, 0, g.lag_cells);
      else plaunch(e, kb_lagrange_cells<3, 1, true, true>, CT, 0, g.lag_cells);
    } else if (g.EL) {
      // elasto cases: one environment (validated at creation)
      if (g.DIM == 2) plaunch(e, kb_lagrange_cells<2, 1, false, true>, CT, 0, g.lag_cells);
      else plaunch(e, kb_lagrange_cells<3, 1, false, true>, CT, 0, g.lag_cells);
    } else if (g.CSTS) {
      // CSTS: the cell pass computes the geometry itself (it reads the
      // corner normals at n first), then the forward velocity update
      DISPATCH_GROUP(g, (plaunch(e, kb_lagrange_cells<DIM_, NE_, true, false, true>, CT, 0, g.lag_cells)));
      if (g.DIM == 2) plaunch(e, kb_csts_forward<2>, CT, 0, g.lag_nodes);
      else plaunch(e, kb_csts_forward<3>, CT, 0, g.lag_nodes);
    } else {
      if (g.DIM == 2) plaunch(e, kb_lagrange_geom<2>, CT, 0, g.lag_cells);
      else plaunch(e, kb_lagrange_geom<3>, CT, 0, g.lag_cells);
      if (g.ADV) DISPATCH_GROUP(g, (plaunch(e, kb_advect_cells<DIM_, NE_>, CT, 0, g.lag_cells)));
      else if (g.EULER) DISPATCH_GROUP(g, (plaunch(e, kb_lagrange_cells<DIM_, NE_, true, false>, CT, 0, g.lag_cells)));
      else DISPATCH_GROUP(g, (plaunch(e, kb_lagrange_cells<DIM_, NE_, false, false>, CT, 0, g.lag_cells)));
    }
  }
}

// directions swept this cycle by the members of a group (host mirror of
// sweep_dirs in mhc_launch.cuh)
int group_dirs(Engine* e, const Group& g, int* dirs) {
  const int dim = g.DIM;
  const long long it = g.it0 + e->cycles_since_build;
  const int sens = (int)((it - 1) % dim);
  int n = 0;
  for (int i = 0; i < dim; ++i) {
    int d = (i + sens) % dim;
    if ((g.skip >> d) & 1) continue;
    dirs[n++] = d;
  }
  return n;
}

// RemapADIService::appliRemap (RemapADIService.cc:15-90) for every group:
// the direction sweeps (:23-56), then the Euler reset and remapVariables
// (:58-87)
void launch_remap_sweeps(Engine* e) {
  for (int k = 0; k < 3; ++k) {
    for (Group& g : e->groups) {
      if (!g.EULER) continue;
      int dirs[3];
      int nd = group_dirs(e, g, dirs);
      if (k >= nd) continue;
      sweep_step_any(e, g, dirs[k], k);
    }
  }
}

// the end of appliRemap: per-axis Euler volumes (computeVolumeEuler) and
// RemapADIService::remapVariables (RemapADIFinal.cc:21-346), then the
// per-axis coordinate reset
void launch_remap_variables(Engine* e) {
  for (Group& g : e->groups) {
    if (!g.EULER) continue;
    int dirs[3];
    int K = group_dirs(e, g, dirs);
    {
      StageTimer tm(e, MHC_STAGE_FINALIZE_CELLS);
      if (g.EULER == 2) {
        if (g.DIM == 2) plaunch(e, kb_euler_volume<2>, CT, 0, g.fin_cells);
        else plaunch(e, kb_euler_volume<3>, CT, 0, g.fin_cells);
      }
      if (g.ADV) DISPATCH_GROUP(g, (plaunch(e, kb_remap_finalize_cells<DIM_, NE_, true>, CT, 0, g.fin_cells, K)));
      else DISPATCH_GROUP(g, (plaunch(e, kb_remap_finalize_cells<DIM_, NE_>, CT, 0, g.fin_cells, K)));
    }
    {
      StageTimer tm(e, MHC_STAGE_FINALIZE_NODES);
      if (K > 0 && g.ADV) DISPATCH_GROUP(g, (plaunch(e, kb_remap_finalize_nodes<DIM_, false>, CT, 0, g.fin_nodes, K)));
      else if (K > 0) DISPATCH_GROUP(g, (plaunch(e, kb_remap_finalize_nodes<DIM_>, CT, 0, g.fin_nodes, K)));
      if (g.EULER == 2) plaunch(e, kb_euler_axis_reset, CT, 0, g.fin_nodes);
    }
  }
}

void launch_remap(Engine* e) {
  launch_remap_sweeps(e);
  launch_remap_variables(e);
}

// node speeds stored by the node finalize pass for computeDeltaT;
// MHC_NODE_SPEED=0 in the environment recomputes them per cell corner
bool spd_enabled() {
  static const bool v = [] {
    const char* s = getenv("MHC_NODE_SPEED");
    return !(s && *s == '0');
  }();
  return v;
}

void launch_dt(Engine* e) {
  StageTimer tm(e, MHC_STAGE_DELTA_T);
  for (Group& g : e->groups) {
    // sans-lagrange keeps deltat_init: no CFL reduction; a Full Euler group
    // whose remap ran reads the node speeds its node finalize pass stored
    int dirs[3];
    const bool spd = g.EULER == 1 && group_dirs(e, g, dirs) > 0 && spd_enabled();
    if (!g.ADV && spd) DISPATCH_GROUP(g, (plaunch(e, kb_delta_t<DIM_, true>, CT, 0, g.dt)));
    else if (!g.ADV) DISPATCH_GROUP(g, (plaunch(e, kb_delta_t<DIM_>, CT, 0, g.dt)));
    if (g.cases.n > 0) {
      kb_delta_t_finalize<<<cdiv(g.cases.n, 128), 128, 0, e->stream>>>(e->d_desc, e->d_ints + g.cases.off_cases, g.cases.n);
      ++e->launches;
    }
  }
}

void end_cycle(Engine* e) {
  e->cycles_since_build += 1;
  for (mhc_case* h : e->cases) h->it_host += 1;
}

void launch_cycle(Engine* e) {
  launch_lagrange_nodes(e);
  launch_lagrange_cells(e);
  launch_remap(e);
  launch_dt(e);
  end_cycle(e);
}

int engine_cycle(Engine* e, int n) {
  int r = engine_rebuild(e);
  if (r) return r;
  for (int it = 0; it < n; ++it) launch_cycle(e);
  CK(cudaGetLastError());
  return MHC_OK;
}

// CUDA graph of one rotation period: 6 iterations bring every 2D and 3D
// group back to the same sweep order, so the same graph replays
int engine_cycle_graph(Engine* e, int n) {
  int r = engine_rebuild(e);
  if (r) return r;
  const int period = 6;
  while (n > 0 && e->cycles_since_build % period != 0) {
    launch_cycle(e);
    --n;
  }
  // n = 0 on an aligned engine only captures (setup outside a timed loop)
  if ((n >= period || n == 0) && !e->graph && e->cycles_since_build % period == 0) {
    long long saved = e->cycles_since_build;
    std::vector<long long> its;
    for (mhc_case* h : e->cases) its.push_back(h->it_host);
    cudaGraph_t g = nullptr;
    const long long before = e->launches;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < period; ++it) launch_cycle(e);
    e->graph_launches = e->launches - before;
    // the captured iterations did not run: the loop state goes back to
    // where it was, whether or not the capture succeeded
    e->launches = before;
    e->cycles_since_build = saved;
    for (size_t i = 0; i < e->cases.size(); ++i) e->cases[i]->it_host = its[i];
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      e->graph = nullptr;
      e->dirty = true;  // rebuild the launch lists before the next cycle
      return set_err(MHC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    }
  }
  while (n >= period && e->graph) {
    CK(cudaGraphLaunch(e->graph, e->stream));
    e->launches += e->graph_launches;
    for (int it = 0; it < period; ++it) end_cycle(e);
    n -= period;
  }
  for (; n > 0; --n) launch_cycle(e);
  CK(cudaGetLastError());
  return MHC_OK;
}

// page-locked host blocks are slow to allocate and to free (the driver maps
// and unmaps them, and a free waits for the device): the small per-case and
// per-engine blocks are kept in a process-wide free list and reused
namespace {
std::mutex g_pinned_mu;
std::multimap<size_t, void*> g_pinned_free;
}  // namespace

int pinned_get(size_t bytes, void** out) {
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    auto it = g_pinned_free.lower_bound(bytes);
    if (it != g_pinned_free.end() && it->first <= 2 * bytes) {
      *out = it->second;
      g_pinned_free.erase(it);
      return MHC_OK;
    }
  }
  CK(cudaMallocHost(out, bytes));
  return MHC_OK;
}

void pinned_put(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  g_pinned_free.emplace(bytes, p);
}

int engine_create(cudaStream_t stream, Engine** out) {
  Engine* e = new Engine();
  if (stream) {
    e->stream = stream;
  } else {
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete e;
      cudaGetLastError();
      return set_err(MHC_ERR_CUDA, "stream creation failed (no CUDA device?)");
    }
    e->own_stream = true;
  }
  *out = e;
  return MHC_OK;
}

void engine_release(Engine* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->d_desc) cudaFreeAsync(e->d_desc, e->stream);
  if (e->d_ints) cudaFreeAsync(e->d_ints, e->stream);
  for (int i = 0; i < 2; ++i)
    if (e->ev[i]) cudaEventDestroy(e->ev[i]);
  if (e->d_gather) cudaFreeAsync(e->d_gather, e->stream);
  if (e->h_gather) { cudaStreamSynchronize(e->stream); pinned_put(e->h_gather, e->gather_cap * sizeof(Scalars)); }
  e->d_gather = nullptr; e->h_gather = nullptr; e->gather_cap = 0;
  if (e->stage_ev) { cudaEventSynchronize(e->stage_ev); cudaEventDestroy(e->stage_ev); }
  if (e->h_stage) pinned_put(e->h_stage, e->stage_cap);
  e->stage_ev = nullptr; e->h_stage = nullptr; e->stage_cap = 0;
  e->graph = nullptr; e->d_desc = nullptr; e->desc_cap = 0; e->d_ints = nullptr; e->ints_cap = 0;
  e->ev[0] = e->ev[1] = nullptr;
}

void engine_destroy(Engine* e) {
  if (!e) return;
  cudaStreamSynchronize(e->stream);
  engine_release(e);
  cudaStreamSynchronize(e->stream);
  if (e->own_stream) cudaStreamDestroy(e->stream);
  delete e;
}

int engine_timed(Engine* e, int n, double* stage_ms, long long* launches) {
  if (!e->ev[0]) {
    CK(cudaEventCreate(&e->ev[0]));
    CK(cudaEventCreate(&e->ev[1]));
  }
  for (int s = 0; s < MHC_NUM_STAGES; ++s) { e->stage_ms[s] = 0.; e->stage_launches[s] = 0; }
  e->timing = true;
  int r = engine_cycle(e, n);
  e->timing = false;
  for (int s = 0; s < MHC_NUM_STAGES; ++s) {
    stage_ms[s] = e->stage_ms[s];
    if (launches) launches[s] = e->stage_launches[s];
  }
  return r;
}

// -- cases ------------------------------------------------------------------------
long long count_doubles(const mhc_case_params* p, long long& ncell, long long& nnode) {
  int dim = p->dim;
  ncell = (long long)p->nx * p->ny * (dim == 3 ? p->nz : 1);
  nnode = (long long)(p->nx + 1) * (p->ny + 1) * (dim == 3 ? p->nz + 1 : 1);
  int ne = p->nb_env, nv = 3 * ne + 1 + ((p->env[0].elasto_model && p->with_projection) ? MHC_ELASTO_XV : 0);
  long long cells = 9 + (ne > 1 ? 8 * ne : 0) + 2 * nv + ne + (p->env[0].elasto_model ? 9 : 0) + (p->env[0].elasto_model == 2 ? 10 : 0) + (dim == 3 ? 24 : 8) +
                    (p->projection_pente_borne ? nv : 0) + 2;  // (+2: boundary-condition energy, pressure)
  const bool csts = p->schema_csts && p->with_projection;
  long long nodes = 4 + 6 + 10 + ((p->sans_lagrange || csts) ? 3 : 0) + (csts ? 3 : 0) + ((p->with_projection && p->is_euler_scheme == MHC_EULER_FULL && !p->sans_lagrange) ? 1 : 0);
  if (csts) cells += 1;
  if (!p->with_projection && !p->sans_lagrange) cells += 2 * ne;  // temperature
  return cells * ncell + nodes * nnode;
}

int validate(const mhc_case_params* p) {
  if (p->dim != 2 && p->dim != 3) return set_err(MHC_ERR_ARG, "dim must be 2 or 3");
  if (p->nx < 1 || p->ny < 1 || (p->dim == 3 && p->nz < 1)) return set_err(MHC_ERR_ARG, "mesh size");
  if (p->nb_env < 1 || p->nb_env > MHC_MAX_ENV) return set_err(MHC_ERR_ARG, "nb_env must be 1..4");
  if ((long long)(p->nx + 1) * (p->ny + 1) * (p->dim == 3 ? p->nz + 1 : 1) > INT_MAX)
    return set_err(MHC_ERR_ARG, "a case holds at most 2^31 - 1 nodes");
  if (p->nb_bc < 0 || p->nb_bc > MHC_MAX_BC) return set_err(MHC_ERR_ARG, "nb_bc");
  bool surfaces = false, cellvars = false;
  for (int b = 0; b < p->nb_bc; ++b) {
    const int kind = p->bc[b].kind;
    if (kind < MHC_BC_VX || kind > MHC_BC_ON_FILE_PRESSURE)
      return set_err(MHC_ERR_UNSUPPORTED, "boundary condition kind");
    const bool surface = kind == MHC_BC_GEOMETRIC_PRESSURE || kind == MHC_BC_LINEAR_PRESSURE ||
                         kind == MHC_BC_SUPER_GAUSSIAN_PRESSURE || kind == MHC_BC_CONTACT_HERZ_PRESSURE ||
                         kind == MHC_BC_ON_FILE_PRESSURE;
    if (surface && p->with_projection)
      return set_err(MHC_ERR_UNSUPPORTED, "pressure boundary conditions need a Lagrangian loop");
    surfaces = surfaces || surface;
    cellvars = cellvars || (kind >= MHC_BC_DENSITY && kind <= MHC_BC_PRESSURE);
  }
  if (p->pressure_table_n < 0 || p->pressure_table_n > MHC_MAX_PTABLE)
    return set_err(MHC_ERR_ARG, "pressure_table_n: 0..MHC_MAX_PTABLE");
  // the reference interleaves both kinds condition by condition on shared node masses
  if (surfaces && cellvars)
    return set_err(MHC_ERR_UNSUPPORTED, "cell-variable boundary conditions together with pressure surfaces");
  if (cellvars && p->with_projection && p->is_euler_scheme != MHC_EULER_FULL)
    return set_err(MHC_ERR_UNSUPPORTED, "cell-variable boundary conditions with a per-axis Euler remap");
  if (cellvars && p->with_newton)
    return set_err(MHC_ERR_UNSUPPORTED, "cell-variable boundary conditions with the Newton energy update");
  if (p->cas_model < MHC_CASE_SOD || p->cas_model > MHC_CASE_TRIPLE_POINT) return set_err(MHC_ERR_ARG, "cas-model");
  // the three regions read the initial states of three environments
  if (p->cas_model == MHC_CASE_TRIPLE_POINT &&
      (p->nb_env != 3 || (p->cas_test != MHC_TEST_MONO_TRIPLE_POINT && p->cas_test != MHC_TEST_BI_TRIPLE_POINT)))
    return set_err(MHC_ERR_ARG, "POINTTRIPLE needs three environments and cas_test 2 or 12");
  if (p->mesh_cell_order != 0 && !(p->mesh_cell_order == 1 && p->dim == 2))
    return set_err(MHC_ERR_ARG, "mesh_cell_order: 0, or 1 in 2D");
  if (p->cas_model == MHC_CASE_RIDER &&
      (p->cas_test < MHC_TEST_MONO_RIDER_TX || p->cas_test > MHC_TEST_RIDER_DEFORMATION_REVERSE || p->nb_env < 2 ||
       !p->sans_lagrange || !(p->rider_radius > 0.)))
    return set_err(MHC_ERR_ARG, "RIDER: cas-test 23..38, two environments or more, sans-lagrange, radius > 0");
  if (p->sans_lagrange) {
    // pure advection: the remap carries the cells; nothing of the
    // Lagrange phase (elasto-plasticity, cell-variable or pressure
    // boundary conditions) has a meaning without it
    if (!p->with_projection) return set_err(MHC_ERR_UNSUPPORTED, "sans-lagrange needs the remap");
    if (cellvars) return set_err(MHC_ERR_UNSUPPORTED, "cell-variable boundary conditions with sans-lagrange");
    // it returns the kinetic energy lost by the dual projection, which does
    // not run here
    if (p->conservation_energie_totale)
      return set_err(MHC_ERR_UNSUPPORTED, "conservation-energie-totale with sans-lagrange");
    if (p->schema_csts) return set_err(MHC_ERR_UNSUPPORTED, "schema-csts with sans-lagrange");
  }
  if (p->schema_csts) {
    // the CSTS Newton update starts from a pressure the reference never
    // sets (MahycoModule.cc:1596-1599); without the remap the scheme needs
    // the pseudo-viscosity at n-1, kept only there; the forward update
    // reads the cell pressure that the cell-variable conditions replace
    if (!p->with_projection) return set_err(MHC_ERR_UNSUPPORTED, "schema-csts needs the remap");
    if (p->with_newton) return set_err(MHC_ERR_UNSUPPORTED, "schema-csts with the Newton energy update");
    if (cellvars) return set_err(MHC_ERR_UNSUPPORTED, "schema-csts with cell-variable boundary conditions");
    if (p->is_euler_scheme != MHC_EULER_FULL) return set_err(MHC_ERR_UNSUPPORTED, "schema-csts with a per-axis Euler remap");
  }
  if (p->cas_model == MHC_CASE_BUBBLES && (p->nb_env != 2 || p->bubbles_n[0] < 0 || p->bubbles_n[1] < 0 ||
                                           p->bubbles_n[2] < 0 || !(p->bubbles_radius >= 0.)))
    return set_err(MHC_ERR_ARG, "bubble lattice: two environments, counts >= 0, radius >= 0");
  if (p->ordre_projection < 1 || p->ordre_projection > 3)
    return set_err(MHC_ERR_UNSUPPORTED, "ordre-projection must be 1, 2 or 3");
  if (p->projection_limiteur_id < 0 || p->projection_limiteur_id > 7)
    return set_err(MHC_ERR_UNSUPPORTED, "projection-limiteur-id must be 0..7 (TypesMahyco.h limiteur)");
  if (p->is_euler_scheme != MHC_EULER_FULL && p->is_euler_scheme != MHC_EULER_X && p->is_euler_scheme != MHC_EULER_Y &&
      !(p->is_euler_scheme == MHC_EULER_Z && p->dim == 3))
    return set_err(MHC_ERR_UNSUPPORTED, "is-euler-scheme must be Full, X, Y or (3D) Z");
  if (p->projection_simple_pente && !p->projection_pente_borne)
    return set_err(MHC_ERR_UNSUPPORTED, "projection-simple-pente needs projection-pente-borne (MahycoModule.cc:47-51)");
  if (p->projection_pente_borne && p->ordre_projection != 2)
    return set_err(MHC_ERR_UNSUPPORTED, "projection-pente-borne needs ordre-projection 2");
  if (p->projection_pente_borne_debar_fix < 0 || p->projection_pente_borne_debar_fix > 2)
    return set_err(MHC_ERR_UNSUPPORTED, "projection-pente-borne-debar-fix must be 0, 1 or 2");
  if (p->projection_limiteur_pure_id < 0 || p->projection_limiteur_pure_id > 7)
    return set_err(MHC_ERR_UNSUPPORTED, "projection-limiteur-pure-id must be 0..7");
  for (int e = 0; e < p->nb_env; ++e) {
    const mhc_env_params& o = p->env[e];
    if (o.elasto_model < 0 || o.elasto_model > 2)
      return set_err(MHC_ERR_UNSUPPORTED, "elasto-model must be NoModel, DefaultModel or NewHypoModel");
    if (o.elasto_model == 0) continue;
    if (p->nb_env != 1) return set_err(MHC_ERR_UNSUPPORTED, "elasto-plasticity needs one environment");
    // with the remap: the deviator and plastic strains ride along as seven
    // more projected variables, through the warp-per-line cell sweeps
    if (p->with_projection &&
        (p->is_euler_scheme != MHC_EULER_FULL || p->projection_pente_borne || p->ordre_projection > 2 ||
         p->projection_limiteur_id > MHC_VANLEER || p->schema_csts || p->sans_lagrange))
      return set_err(MHC_ERR_UNSUPPORTED,
                     "elasto-plasticity with the remap needs the Full Euler scheme, order 1 or 2, a classical "
                     "limiter, no pente-borne, no schema-csts");
    if (o.rotation_order != 1 && o.rotation_order != 2) return set_err(MHC_ERR_UNSUPPORTED, "ordre-rotation must be 1 or 2");
    if (!(o.shear_modulus > 0.) || !(o.yield_strength > 0.)) return set_err(MHC_ERR_ARG, "shear modulus and yield strength must be > 0");
  }
  for (int e = 0; e < p->nb_env; ++e) {
    if (p->env[e].depot_type < MHC_DEPOT_NONE || p->env[e].depot_type > MHC_DEPOT_SUPER_GAUSSIAN)
      return set_err(MHC_ERR_ARG, "energy deposit kind");
    if (p->env[e].density_damage_thresold != 0.0 || p->env[e].tension_damage_thresold > -1.e12)
      return set_err(MHC_ERR_UNSUPPORTED, "damage thresholds other than the defaults");
    if (p->env[e].eos < 0 || p->env[e].eos > MHC_EOS_FICTIF) return set_err(MHC_ERR_ARG, "eos kind");
    if (p->env[e].eos == MHC_EOS_FICTIF && !p->sans_lagrange)
      return set_err(MHC_ERR_UNSUPPORTED, "the Fictif equation of state with a Lagrange phase");
  }
  if (p->longueur_caracteristique == MHC_LENGTH_OPPOSITE_FACES && p->dim != 3)
    return set_err(MHC_ERR_UNSUPPORTED, "faces-opposees needs a 3D mesh");
  return MHC_OK;
}

void case_free(mhc_case* h) {
  if (!h) return;
  if (h->h_scal) { cudaStreamSynchronize(h->stream); pinned_put(h->h_scal, 2 * sizeof(Scalars)); h->h_scal = nullptr; }
  for (int i = 0; i < 2; ++i)
    if (h->scal_ev[i]) { cudaEventDestroy(h->scal_ev[i]); h->scal_ev[i] = nullptr; }
  if (h->solo) { engine_destroy(h->solo); h->solo = nullptr; }
  if (h->stream) {
    // stream-ordered frees: the work already queued that reads the case
    // runs first; only a private stream is waited for, before it goes
    for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
    if (h->own_stream) {
      cudaStreamSynchronize(h->stream);
      cudaStreamDestroy(h->stream);
    }
  }
  delete h;
}

// allocates the device state of one case on `stream` (stream-ordered pool);
// a null stream gives the case a private stream
// keep freed device memory in the stream-ordered pool of the current device
// instead of returning it at every synchronisation: cases come and go
// (serving, batches), and re-mapping their memory costs milliseconds
void keep_pool_memory() {
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done[dev] = true;
}

int case_alloc(const mhc_case_params* params, cudaStream_t stream, mhc_case** out) {
  *out = nullptr;
  int v = validate(params);
  if (v != MHC_OK) return v;
  keep_pool_memory();
  mhc_case* h = new mhc_case();
  h->P = *params;
  h->DIM = params->dim;
  h->NE = params->nb_env;
  // projected variables: volume, mass, energy per environment, the
  // pseudo-viscosity, then (elasto-plasticity with the remap) the deviator's
  // xx, yy, xy, yz, zx times the volume and the plastic strain rate and
  // strain times the mass (PrepareRemap.cc:121-128)
  h->NV = 3 * h->NE + 1 + ((h->P.env[0].elasto_model && h->P.with_projection) ? MHC_ELASTO_XV : 0);
  Mesh& M = h->M;
  M.dim = h->DIM;
  M.ncx = params->nx; M.ncy = params->ny; M.ncz = h->DIM == 3 ? params->nz : 1;
  M.nnx = M.ncx + 1; M.nny = M.ncy + 1; M.nnz = h->DIM == 3 ? M.ncz + 1 : 1;
  M.ncell = (long long)M.ncx * M.ncy * M.ncz;
  M.nnode = (long long)M.nnx * M.nny * M.nnz;
  M.o[0] = params->origin[0]; M.o[1] = params->origin[1]; M.o[2] = params->origin[2];
  M.h[0] = params->lx / params->nx;
  M.h[1] = params->ly / params->ny;
  M.h[2] = h->DIM == 3 ? params->lz / params->nz : 0.;
  if (stream) {
    h->stream = stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete h;
      return set_err(MHC_ERR_CUDA, "stream creation failed (no CUDA device?)");
    }
    h->own_stream = true;
  }
  const long long N = M.ncell, NN = M.nnode;
  bool ok = true;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok || cudaMallocAsync(&p, bytes, h->stream) != cudaSuccess) { ok = false; return nullptr; }
    h->allocs.push_back(p);
    h->alloc_bytes.push_back(bytes);
    return p;
  };
  auto dcell = [&]() { return (double*)alloc(N * sizeof(double)); };
  auto dnode = [&]() { return (double*)alloc(NN * sizeof(double)); };
  Fields& F = h->F;
  memset(&F, 0, sizeof(F));
  F.rho = dcell(); F.e = dcell(); F.p = dcell(); F.c = dcell(); F.q = dcell();
  F.m = dcell(); F.V = dcell(); F.l = dcell(); F.Veul = dcell();
  if (h->NE > 1) {
    auto denv = [&]() { return (double*)alloc(h->NE * N * sizeof(double)); };
    F.ef = denv(); F.emf = denv(); F.em = denv(); F.erho = denv();
    F.ee = denv(); F.ep = denv(); F.ec = denv(); F.eq = denv();
  }
  F.mask = (uint8_t*)alloc(N);
  F.vx = dnode(); F.vy = dnode(); F.vz = dnode(); F.mn = dnode();
  for (int b = 0; b < 2; ++b)
    for (int d = 0; d < 3; ++d) F.X[b][d] = dnode();
  for (int b = 0; b < 2; ++b) {
    F.U[b] = (double*)alloc(h->NV * N * sizeof(double));
    F.Ud[b] = (double*)alloc(5 * NN * sizeof(double));
  }
  F.mflux = (double*)alloc(h->NE * N * sizeof(double));
  if (h->P.env[0].elasto_model) {
    F.S = (double*)alloc(6 * N * sizeof(double));
    F.pl = (double*)alloc(3 * N * sizeof(double));
    if (h->P.env[0].elasto_model == 2) F.hf = (double*)alloc(10 * N * sizeof(double));
  }
  F.cqs = (double*)alloc((h->DIM == 3 ? 24 : 8) * N * sizeof(double));
  if (h->P.projection_pente_borne) F.phi_pb = (double*)alloc(h->NV * N * sizeof(double));
  const bool csts = h->P.schema_csts && h->P.with_projection;
  if (h->P.sans_lagrange || csts) F.v0 = (double*)alloc(3 * NN * sizeof(double));
  if (h->P.with_projection && h->P.is_euler_scheme == MHC_EULER_FULL && !h->P.sans_lagrange) F.spd = dnode();
  if (csts) {
    F.pq = dcell();
    for (int d = 0; d < 3; ++d) F.fv[d] = dnode();
  } else {
    F.fv[0] = F.vx; F.fv[1] = F.vy; F.fv[2] = F.vz;
  }
  if (case_cell_bcs(h)) {
    F.ebc = (double*)alloc(N * sizeof(double));
    F.pbc = (double*)alloc(N * sizeof(double));
  }
  if (!h->P.with_projection && !h->P.sans_lagrange) {
    // the temperature the EOS services advance, carried by Lagrangian runs
    F.T = (double*)alloc(h->NE * N * sizeof(double));
    F.Tn = (double*)alloc(h->NE * N * sizeof(double));
  }
  h->d_scal = (Scalars*)alloc(sizeof(Scalars));
  h->d_params = (mhc_case_params*)alloc(sizeof(mhc_case_params));
  F.s = h->d_scal;
  if (!ok) {
    cudaGetLastError();
    case_free(h);
    return set_err(MHC_ERR_NOMEM, "device allocation failed");
  }
  if (F.phi_pb && cudaMemsetAsync(F.phi_pb, 0, h->NV * N * sizeof(double), h->stream) != cudaSuccess) {
    case_free(h);
    return set_err(MHC_ERR_CUDA, "memset");
  }
  if ((F.S && cudaMemsetAsync(F.S, 0, 6 * N * sizeof(double), h->stream) != cudaSuccess) ||
      (F.pl && cudaMemsetAsync(F.pl, 0, 3 * N * sizeof(double), h->stream) != cudaSuccess)) {
    case_free(h);
    return set_err(MHC_ERR_CUDA, "memset");
  }
  if (h->NE > 1) {
    // env slots of cells that never hold the env read as zero
    double* arr[] = {F.ef, F.emf, F.em, F.erho, F.ee, F.ep, F.ec, F.eq};
    for (double* a : arr)
      if (cudaMemsetAsync(a, 0, h->NE * N * sizeof(double), h->stream) != cudaSuccess) {
        case_free(h);
        return set_err(MHC_ERR_CUDA, "memset");
      }
  }
  if (cudaMemcpyAsync(h->d_params, &h->P, sizeof(mhc_case_params), cudaMemcpyHostToDevice, h->stream) != cudaSuccess) {
    case_free(h);
    return set_err(MHC_ERR_CUDA, "params upload");
  }
  *out = h;
  return MHC_OK;
}

// scalars of a case at start-init (iteration 1 about to run)
int case_reset_scalars(mhc_case* h, long long iteration_limit) {
  Scalars s;
  memset(&s, 0, sizeof(s));
  s.t = h->P.deltat_init;  // global time of iteration 1
  s.dt = h->P.deltat_init;
  s.old_dt = 0.;
  s.iteration = 1;
  s.dt_min_bits = 0x7fefffffffffffffull;
  s.iteration_limit = iteration_limit;
  for (int q = 0; q < 4; ++q) s.eref_first[q] = 0xffffffffu;
  // a copy from pageable host memory is staged before the call returns, so
  // the stack source may go at once (no wait for the work in flight)
  CK(cudaMemcpyAsync(h->d_scal, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  h->it_host = 1;
  return MHC_OK;
}

int solo_engine(mhc_case* h) {
  if (h->solo) return MHC_OK;
  int r = engine_create(h->stream, &h->solo);
  if (r) return r;
  h->solo->cases.push_back(h);
  h->solo->dirty = true;
  return MHC_OK;
}

// device -> host copy of `bytes` after the work queued on `s`: through two
// page-locked staging chunks, so that the device copy of chunk i+1 runs
// while the host copies chunk i out (a pageable cudaMemcpy stages through
// the driver at a fraction of the link's bandwidth)
namespace {
constexpr size_t kStageChunk = 4u << 20;
struct Staging {
  std::mutex mu;
  char* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};  // events belong to one device
};
Staging g_stage[64];  // per device
}  // namespace

int fetch(cudaStream_t s, const void* dev, void* host, size_t bytes) {
  if (bytes == 0) return MHC_OK;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, host) == cudaSuccess && at.type == cudaMemoryTypeHost) {
    // a page-locked destination: one copy straight into it
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return MHC_OK;
  }
  cudaGetLastError();
  if (bytes <= 64 * 1024) {
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost));
    return MHC_OK;
  }
  int device = 0;
  CK(cudaGetDevice(&device));
  if (device < 0 || device >= 64) return set_err(MHC_ERR_ARG, "device index");
  Staging& g = g_stage[device];
  std::lock_guard<std::mutex> lk(g.mu);
  for (int b = 0; b < 2; ++b) {
    if (!g.buf[b]) CK(cudaMallocHost((void**)&g.buf[b], kStageChunk));
    if (!g.ev[b]) CK(cudaEventCreateWithFlags(&g.ev[b], cudaEventDisableTiming));
  }
  const char* src = static_cast<const char*>(dev);
  char* dst = static_cast<char*>(host);
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  auto issue = [&](size_t i) -> int {
    const size_t off = i * kStageChunk, len = std::min(kStageChunk, bytes - off);
    CK(cudaMemcpyAsync(g.buf[i & 1], src + off, len, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(g.ev[i & 1], s));
    return MHC_OK;
  };
  int r = issue(0);
  if (r) return r;
  for (size_t i = 0; i < nch; ++i) {
    if (i + 1 < nch && (r = issue(i + 1))) return r;
    CK(cudaEventSynchronize(g.ev[i & 1]));
    const size_t off = i * kStageChunk, len = std::min(kStageChunk, bytes - off);
    memcpy(dst + off, g.buf[i & 1], len);
  }
  return MHC_OK;
}

int read_scalars(mhc_case* h, cudaStream_t s, Scalars* out) {
  CK(cudaStreamSynchronize(s));
  CK(cudaMemcpy(out, h->d_scal, sizeof(Scalars), cudaMemcpyDeviceToHost));
  return MHC_OK;
}

long long case_get_field(mhc_case* h, cudaStream_t st, const char* name, int env, double* host, long long cap) {
  const long long N = h->M.ncell, NN = h->M.nnode;
  Fields& F = h->F;
  struct { const char* n; double* g; double* e; } cells[] = {
      {"Density", F.rho, F.erho}, {"Pressure", F.p, F.ep}, {"InternalEnergy", F.e, F.ee},
      {"SoundSpeed", F.c, F.ec}, {"PseudoViscosity", F.q, F.eq}, {"CellMass", F.m, F.em},
      {"CellVolume", F.V, nullptr}, {"FracVol", nullptr, F.ef}, {"MassFraction", nullptr, F.emf},
      {"CaracteristicLength", F.l, nullptr}, {"EulerVolume", F.Veul, nullptr}};
  if (env >= h->NE) return set_err(MHC_ERR_ARG, "env out of range");
  for (auto& c : cells) {
    if (strcmp(name, c.n)) continue;
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    int r;
    if (env < 0) {  // the cell (global) values straight into the caller's buffer
      if (!c.g) for (long long i = 0; i < N; ++i) host[i] = 1.;
      else if ((r = fetch(st, c.g, host, N * 8))) return r;
      return N;
    }
    std::vector<double> g(N, 0.), e;
    std::vector<uint8_t> mask(N);
    if ((r = fetch(st, F.mask, mask.data(), N))) return r;
    if (c.g) { if ((r = fetch(st, c.g, g.data(), N * 8))) return r; }
    if (h->NE > 1 && c.e) {
      e.resize(N);
      if ((r = fetch(st, c.e + env * N, e.data(), N * 8))) return r;
    }
    const bool volume = !strcmp(name, "CellVolume");
    std::vector<double> fr;
    if (volume && h->NE > 1) {
      fr.resize(N);
      if ((r = fetch(st, F.ef + env * N, fr.data(), N * 8))) return r;
    }
    const bool fracvol = !strcmp(name, "FracVol");
    for (long long i = 0; i < N; ++i) {
      bool in = (mask[i] >> env) & 1;
      bool pure = __builtin_popcount(mask[i]) == 1;
      if (!in) host[i] = 0.;
      else if (pure && fracvol && h->NE > 1) host[i] = e[i];  // the remap's normalised fraction
      else if (pure) host[i] = c.g ? g[i] : 1.;
      else if (volume) host[i] = fr[i] * g[i];
      else host[i] = c.e ? e[i] : 0.;
    }
    return N;
  }
  if (!strcmp(name, "Temperature")) {
    // env >= 0: the environment's temperature (0 where it is absent); env <
    // 0: the cell value, which is a pure cell's and 0 in a mixed cell (the
    // services write environment values only)
    if (!F.T) return set_err(MHC_ERR_UNSUPPORTED, "the temperature is carried by Lagrangian runs only");
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    std::vector<uint8_t> mask(N);
    std::vector<double> t((size_t)h->NE * N);
    int r;
    if ((r = fetch(st, F.mask, mask.data(), N)) || (r = fetch(st, F.T, t.data(), h->NE * N * 8))) return r;
    for (long long i = 0; i < N; ++i) {
      const bool pure = __builtin_popcount(mask[i]) == 1;
      if (env >= 0) host[i] = ((mask[i] >> env) & 1) ? t[env * N + i] : 0.;
      else host[i] = pure ? t[(__builtin_ffs(mask[i]) - 1) * N + i] : 0.;
    }
    return N;
  }
  if (!strcmp(name, "EnvMask")) {
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    std::vector<uint8_t> mask(N);
    int r = fetch(st, F.mask, mask.data(), N);
    if (r) return r;
    for (long long i = 0; i < N; ++i) host[i] = mask[i];
    return N;
  }
  // elasto output variables: plastic strain, its rate, the deviator's norm
  // (DefaultModelService.cc:211-224)
  static const char* kPlastic[] = {"PlasticDeformation", "PlasticDeformationVelocity", "StrainNorm"};
  for (int q = 0; q < 3; ++q) {
    if (strcmp(name, kPlastic[q])) continue;
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    if (!F.pl) {
      for (long long i = 0; i < N; ++i) host[i] = 0.;
      return N;
    }
    int r = fetch(st, F.pl + q * N, host, N * 8);
    return r ? r : N;
  }
  // elasto output variables: minus the deviator components
  // (DefaultModelService.cc:217-221)
  static const char* kStrain[] = {"StrainTensorXX", "StrainTensorYY", "StrainTensorZZ", "StrainTensorXY",
                                  "StrainTensorYZ", "StrainTensorXZ"};
  for (int q = 0; q < 6; ++q) {
    if (strcmp(name, kStrain[q])) continue;
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    if (!F.S) {
      for (long long i = 0; i < N; ++i) host[i] = 0.;
      return N;
    }
    int r = fetch(st, F.S + q * N, host, N * 8);
    if (r) return r;
    for (long long i = 0; i < N; ++i) host[i] = -host[i];
    return N;
  }
  if (!strcmp(name, "NodeMass")) {
    if (cap < NN) return set_err(MHC_ERR_ARG, "capacity too small");
    int r = fetch(st, F.mn, host, NN * 8);
    return r ? r : NN;
  }
  const bool vn = !strcmp(name, "VelocityN");
  if (vn && !F.v0) return set_err(MHC_ERR_ARG, "VelocityN is kept by sans-lagrange cases only");
  if (!strcmp(name, "Velocity") || !strcmp(name, "NodeCoord") || vn) {
    if (cap < 3 * NN) return set_err(MHC_ERR_ARG, "capacity too small");
    std::vector<double> a, b, c;
    const double *pa, *pb, *pc;
    if (vn) { pa = F.v0; pb = F.v0 + NN; pc = F.v0 + 2 * NN; }
    else if (name[0] == 'V') { pa = F.vx; pb = F.vy; pc = F.vz; }
    else {
      // last Lagrangian positions: X of the last completed iteration
      Scalars s;
      int r = read_scalars(h, st, &s);
      if (r) return r;
      int par = (int)(s.iteration_done & 1);
      pa = F.X[par][0]; pb = F.X[par][1]; pc = F.X[par][2];
    }
    int r;
    double* d = nullptr;
    if (cudaMallocAsync((void**)&d, 3 * NN * sizeof(double), st) == cudaSuccess) {
      // interleaved on the device, then one copy (straight into a
      // page-locked destination)
      const int blocks = (int)std::min<long long>((NN + 255) / 256, 148LL * 8);
      kb_interleave3<<<blocks, 256, 0, st>>>(pa, pb, pc, d, NN);
      r = fetch(st, d, host, 3 * NN * 8);
      cudaFreeAsync(d, st);
      return r ? r : 3 * NN;
    }
    cudaGetLastError();  // no device memory left: the three arrays, interleaved here
    a.resize(NN); b.resize(NN); c.resize(NN);
    if ((r = fetch(st, pa, a.data(), NN * 8)) || (r = fetch(st, pb, b.data(), NN * 8)) || (r = fetch(st, pc, c.data(), NN * 8)))
      return r;
    for (long long i = 0; i < NN; ++i) { host[3 * i] = a[i]; host[3 * i + 1] = b[i]; host[3 * i + 2] = c[i]; }
    return 3 * NN;
  }
  return set_err(MHC_ERR_ARG, std::string("unknown field ") + name);
}

int case_time_history(mhc_case* h, cudaStream_t st, double* out) {
  const long long N = h->M.ncell;
  Scalars s;
  int r = read_scalars(h, st, &s);
  if (r) return r;
  out[0] = s.t_done;
  std::vector<double> m(N), p(N), rho(N), e(N), V(N), env(N);
  if (case_get_field(h, st, "EnvMask", -1, env.data(), N) < 0) return MHC_ERR_CUDA;
  for (int q = 0; q < h->NE; ++q) {
    if (case_get_field(h, st, "CellMass", q, m.data(), N) < 0 || case_get_field(h, st, "Pressure", q, p.data(), N) < 0 ||
        case_get_field(h, st, "Density", q, rho.data(), N) < 0 ||
        case_get_field(h, st, "InternalEnergy", q, e.data(), N) < 0 ||
        case_get_field(h, st, "CellVolume", q, V.data(), N) < 0)
      return MHC_ERR_CUDA;
    long long cnt = 0;
    double sm = 0., sp = 0., rv = 0., vv = 0., em = 0., mm = 0.;
    // in the order of the reference's cell numbering (mesh_cell_order)
    const bool cm = h->DIM == 2 && h->P.mesh_cell_order == 1;
    const long long nx = h->M.ncx, ny = h->M.ncy;
    auto cell = [&](long long k) { return cm ? (k / ny) + nx * (k % ny) : k; };
    for (long long k = 0; k < N; ++k) {
      const long long c = cell(k);
      if (!(((int)env[c] >> q) & 1)) continue;
      ++cnt; sm += m[c]; sp += p[c];
    }
    for (long long k = 0; k < N; ++k) {
      const long long c = cell(k);
      if (!(((int)env[c] >> q) & 1)) continue;
      em += e[c] * m[c]; mm += m[c];
    }
    for (long long k = 0; k < N; ++k) {
      const long long c = cell(k);
      if (!(((int)env[c] >> q) & 1)) continue;
      rv += rho[c] * V[c]; vv += V[c];
    }
    out[1 + 5 * q] = sm / cnt;
    out[1 + 5 * q + 1] = sp / cnt;
    out[1 + 5 * q + 2] = rv / vv;
    out[1 + 5 * q + 3] = em / mm;
    out[1 + 5 * q + 4] = cnt > 0;
  }
  return MHC_OK;
}

}  // namespace

int mhc::engine_rebuild_shared(Engine* e) { return engine_rebuild(e); }
int mhc::solo_engine_shared(mhc_case* h) { return solo_engine(h); }
void mhc::launch_remap_sweeps_shared(Engine* e) { launch_remap_sweeps(e); }
void mhc::launch_remap_variables_shared(Engine* e) { launch_remap_variables(e); }
int mhc::fetch_shared(cudaStream_t s, const void* dev, void* host, size_t bytes) { return fetch(s, dev, host, bytes); }

// ===========================================================================
// C ABI (linkage from the declarations in mahyco_b200.h)
// ===========================================================================
const char* mhc_last_error(void) { return g_err.c_str(); }
const char* mhc_version(void) { return "mahyco_b200 0.2 (sm_100a, fp64, batched engine)"; }

long long mhc_case_device_bytes(const mhc_case_params* p) {
  if (!p) return -1;
  long long nc, nn;
  long long d = count_doubles(p, nc, nn);
  return d * 8 + nc + (long long)sizeof(Scalars) + (long long)sizeof(mhc_case_params);
}

int mhc_case_create(const mhc_case_params* params, mhc_case** out) {
  if (!params || !out) return set_err(MHC_ERR_ARG, "null argument");
  return case_alloc(params, nullptr, out);
}

void* mhc_case_stream(mhc_case* h) { return h ? (void*)h->stream : nullptr; }

int mhc_case_destroy(mhc_case* h) {
  case_free(h);
  return MHC_OK;
}

int mhc_hydro_start_init(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  int r = case_reset_scalars(h, LLONG_MAX);
  if (r) return r;
  if ((r = solo_engine(h))) return r;
  h->solo->dirty = true;
  if ((r = engine_rebuild(h->solo))) return r;
  launch_init(h->solo);
  if (h->P.cas_model == MHC_CASE_RIDER && (r = rider_upload(h, h->solo->stream))) return r;
  CK(cudaGetLastError());
  h->stage = S_IDLE;
  h->initialised = true;
  return MHC_OK;
}

static int expect(mhc_case* h, int from, int to) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != from) return set_err(MHC_ERR_ORDER, "entry point called out of time-loop order");
  h->stage = to;
  return MHC_OK;
}

int mhc_save_values_at_n(mhc_case* h) { return expect(h, S_IDLE, S_SAVED); }
int mhc_update_velocity(mhc_case* h) { return expect(h, S_SAVED, S_VELOCITY); }
int mhc_apply_boundary_condition(mhc_case* h) { return expect(h, S_VELOCITY, S_BC); }
int mhc_update_position(mhc_case* h) {
  int r = expect(h, S_BC, S_POSITION);
  if (r) return r;
  if ((r = engine_rebuild(h->solo))) return r;
  launch_lagrange_nodes(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}
int mhc_compute_geometric_values(mhc_case* h) { return expect(h, S_POSITION, S_GEOM); }
int mhc_update_density(mhc_case* h) { return expect(h, S_GEOM, S_DENSITY); }
int mhc_compute_artificial_viscosity(mhc_case* h) { return expect(h, S_DENSITY, S_VISCO); }
int mhc_update_elasticity_and_plasticity(mhc_case* h) { return expect(h, S_VISCO, S_ELASTO); }
int mhc_update_energy_and_pressure(mhc_case* h) {
  int r = expect(h, S_ELASTO, S_ENERGY);
  if (r) return r;
  launch_lagrange_cells(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}
int mhc_remap(mhc_case* h) {
  int r = expect(h, S_ENERGY, S_REMAP);
  if (r) return r;
  launch_remap(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}
int mhc_remap_apply(mhc_case* h) { return mhc_remap(h); }
int mhc_compute_delta_t(mhc_case* h) {
  int r = expect(h, S_REMAP, S_IDLE);
  if (r) return r;
  launch_dt(h->solo);
  end_cycle(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_cycle(mhc_case* h, int n) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != S_IDLE) return set_err(MHC_ERR_ORDER, "an iteration is in progress");
  return engine_cycle(h->solo, n);
}

int mhc_cycle_graph(mhc_case* h, int n) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != S_IDLE) return set_err(MHC_ERR_ORDER, "an iteration is in progress");
  return engine_cycle_graph(h->solo, n);
}

int mhc_cycle_timed(mhc_case* h, int n, double* stage_ms, long long* stage_launches) {
  if (!h || !stage_ms) return set_err(MHC_ERR_ARG, "null argument");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  return engine_timed(h->solo, n, stage_ms, stage_launches);
}

// -- checkpoint / restart (protection-reprise) --------------------------------
// A checkpoint is a header (magic, the case parameters, the host-side loop
// state, the size of every device allocation) followed by the bytes of
// every device allocation in creation order: the whole device state of the
// case, scalars included.
namespace {
struct CkptHeader {
  char magic[8];
  long long version;
  mhc_case_params params;
  long long it_host;
  int stage;
  int initialised;
  long long nalloc;
};
constexpr char kCkptMagic[8] = {'M', 'H', 'C', 'C', 'K', 'P', 'T', '1'};

long long ckpt_bytes(const mhc_case* h) {
  long long b = (long long)sizeof(CkptHeader) + (long long)(h->alloc_bytes.size() * sizeof(long long));
  for (size_t a : h->alloc_bytes) b += (long long)a;
  return b;
}

int ckpt_save(mhc_case* h, cudaStream_t st, void* host, long long capacity) {
  const long long need = ckpt_bytes(h);
  if (!host || capacity < need) return set_err(MHC_ERR_ARG, "checkpoint buffer smaller than mhc_case_checkpoint_bytes");
  CkptHeader hd;
  memset(&hd, 0, sizeof(hd));
  memcpy(hd.magic, kCkptMagic, 8);
  hd.version = 1;
  hd.params = h->P;
  hd.it_host = h->it_host;
  hd.stage = h->stage;
  hd.initialised = h->initialised ? 1 : 0;
  hd.nalloc = (long long)h->allocs.size();
  char* out = static_cast<char*>(host);
  memcpy(out, &hd, sizeof(hd));
  out += sizeof(hd);
  for (size_t a : h->alloc_bytes) {
    const long long b = (long long)a;
    memcpy(out, &b, sizeof(b));
    out += sizeof(b);
  }
  CK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < h->allocs.size(); ++i) {
    CK(cudaMemcpyAsync(out, h->allocs[i], h->alloc_bytes[i], cudaMemcpyDeviceToHost, st));
    out += h->alloc_bytes[i];
  }
  CK(cudaStreamSynchronize(st));
  return MHC_OK;
}

int ckpt_restore(mhc_case* h, cudaStream_t st, const void* host, long long size) {
  if (!host || size < (long long)sizeof(CkptHeader)) return set_err(MHC_ERR_ARG, "checkpoint too small");
  CkptHeader hd;
  memcpy(&hd, host, sizeof(hd));
  if (memcmp(hd.magic, kCkptMagic, 8) || hd.version != 1) return set_err(MHC_ERR_ARG, "not a checkpoint of this library");
  if (memcmp(&hd.params, &h->P, sizeof(mhc_case_params)))
    return set_err(MHC_ERR_ARG, "checkpoint of a case with other parameters");
  if (hd.nalloc != (long long)h->allocs.size() || size != ckpt_bytes(h))
    return set_err(MHC_ERR_ARG, "checkpoint layout does not match the case");
  const char* in = static_cast<const char*>(host) + sizeof(hd);
  for (size_t i = 0; i < h->alloc_bytes.size(); ++i) {
    long long b;
    memcpy(&b, in, sizeof(b));
    in += sizeof(b);
    if (b != (long long)h->alloc_bytes[i]) return set_err(MHC_ERR_ARG, "checkpoint layout does not match the case");
  }
  CK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < h->allocs.size(); ++i) {
    CK(cudaMemcpyAsync(h->allocs[i], in, h->alloc_bytes[i], cudaMemcpyHostToDevice, st));
    in += h->alloc_bytes[i];
  }
  CK(cudaStreamSynchronize(st));
  h->it_host = hd.it_host;
  h->stage = hd.stage;
  h->initialised = hd.initialised != 0;
  return MHC_OK;
}
}  // namespace

long long mhc_case_checkpoint_bytes(mhc_case* h) { return h ? ckpt_bytes(h) : set_err(MHC_ERR_ARG, "null case"); }

int mhc_case_checkpoint(mhc_case* h, void* host, long long capacity) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (h->stage != S_IDLE) return set_err(MHC_ERR_ORDER, "checkpoint between iterations only");
  return ckpt_save(h, h->stream, host, capacity);
}

int mhc_case_restore(mhc_case* h, const void* host, long long size) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (h->stage != S_IDLE) return set_err(MHC_ERR_ORDER, "restore between iterations only");
  int r = ckpt_restore(h, h->stream, host, size);
  if (r) return r;
  if (h->solo) h->solo->dirty = true;  // iteration-dependent work lists are rebuilt
  return MHC_OK;
}

int mhc_scalars_request(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->h_scal) {
    if (int r = pinned_get(2 * sizeof(Scalars), (void**)&h->h_scal)) return r;
    for (int i = 0; i < 2; ++i) CK(cudaEventCreateWithFlags(&h->scal_ev[i], cudaEventDisableTiming));
  }
  const int slot = h->scal_next;
  h->scal_next ^= 1;
  CK(cudaEventSynchronize(h->scal_ev[slot]));  // the slot's previous copy has landed
  CK(cudaMemcpyAsync(&h->h_scal[slot], h->d_scal, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaEventRecord(h->scal_ev[slot], h->stream));
  return slot;
}

int mhc_scalars_wait(mhc_case* h, int slot, double* time, double* deltat, long long* iteration, int* status) {
  if (!h || slot < 0 || slot > 1 || !h->h_scal) return set_err(MHC_ERR_ARG, "bad case or slot");
  CK(cudaEventSynchronize(h->scal_ev[slot]));
  const Scalars& s = h->h_scal[slot];
  if (time) *time = s.t_done;
  if (deltat) *deltat = s.dt;
  if (iteration) *iteration = s.iteration_done;
  if (status) *status = s.status;
  return MHC_OK;
}

int mhc_synchronize(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  Scalars s;
  int r = read_scalars(h, h->stream, &s);
  return r ? r : s.status;
}

int mhc_get_scalars(mhc_case* h, double* time, double* deltat, long long* iteration, int* status) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  Scalars s;
  int r = read_scalars(h, h->stream, &s);
  if (r) return r;
  if (time) *time = s.t_done;
  if (deltat) *deltat = s.dt;
  if (iteration) *iteration = s.iteration_done;
  if (status) *status = s.status;
  return MHC_OK;
}

long long mhc_get_field(mhc_case* h, const char* name, int env, double* host, long long cap) {
  if (!h || !name || !host) return set_err(MHC_ERR_ARG, "null argument");
  return case_get_field(h, h->stream, name, env, host, cap);
}

int mhc_eos_apply(mhc_case* h, int env) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (env < 0 || env >= h->NE) return set_err(MHC_ERR_ARG, "env out of range");
  int r = solo_engine(h);
  if (r || (r = engine_rebuild(h->solo))) return r;
  Engine* e = h->solo;
  for (Group& g : e->groups) {
    switch (g.NE) {
      case 1: plaunch(e, kb_eos_apply<1>, CT, 0, g.init_cells, env); break;
      case 2: plaunch(e, kb_eos_apply<2>, CT, 0, g.init_cells, env); break;
      case 3: plaunch(e, kb_eos_apply<3>, CT, 0, g.init_cells, env); break;
      default: plaunch(e, kb_eos_apply<4>, CT, 0, g.init_cells, env); break;
    }
  }
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_time_history(mhc_case* h, double* out) {
  if (!h || !out) return set_err(MHC_ERR_ARG, "null argument");
  return case_time_history(h, h->stream, out);
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
struct mhc_batch {
  Engine* e = nullptr;
  std::vector<mhc_case*> slots;   // case index -> case (nullptr once removed)
  std::vector<char> detached;     // slot kept resident but no longer advanced
  std::vector<Scalars> last;      // scalars read when the slot was detached
  // asynchronous polls, double-buffered: the gathered scalars of every case,
  // their page-locked copy, the event after the copy, and the engine index
  // of every slot when the poll was enqueued (-1: not in that poll)
  struct Poll {
    Scalars* d = nullptr;
    Scalars* h = nullptr;
    int cap = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
    std::vector<int> index;
  } poll[2];
  int poll_next = 0;
  std::vector<Scalars> polled;    // each slot's scalars from the last completed poll
  std::vector<char> polled_ok;
  // start-init engines of earlier mhc_batch_init calls, released once their
  // list upload has landed (their frees are stream-ordered)
  std::vector<Engine*> init_engines;
};

// releases the start-init engines whose uploads have landed (all of them,
// waiting, with wait = true); no stream-wide synchronisation
void reap_init_engines(mhc_batch* b, bool wait) {
  std::vector<Engine*> keep;
  for (Engine* e : b->init_engines) {
    const bool done = !e->stage_ev || wait || cudaEventQuery(e->stage_ev) == cudaSuccess;
    if (!done) { keep.push_back(e); continue; }
    engine_release(e);  // waits on its own upload event only
    delete e;
  }
  b->init_engines.swap(keep);
}

int mhc_batch_create(mhc_batch** out) {
  if (!out) return set_err(MHC_ERR_ARG, "null argument");
  mhc_batch* b = new mhc_batch();
  int r = engine_create(nullptr, &b->e);
  if (r) { delete b; return r; }
  *out = b;
  return MHC_OK;
}

int mhc_batch_create_on_stream(void* stream, mhc_batch** out) {
  if (!out || !stream) return set_err(MHC_ERR_ARG, "null argument");
  mhc_batch* b = new mhc_batch();
  int r = engine_create(static_cast<cudaStream_t>(stream), &b->e);
  if (r) { delete b; return r; }
  *out = b;
  return MHC_OK;
}

int mhc_batch_destroy(mhc_batch* b) {
  if (!b) return MHC_OK;
  cudaStreamSynchronize(b->e->stream);
  reap_init_engines(b, true);
  for (mhc_batch::Poll& P : b->poll) {
    if (P.d) cudaFreeAsync(P.d, b->e->stream);
    if (P.h) pinned_put(P.h, P.cap * sizeof(Scalars));
    if (P.ev) cudaEventDestroy(P.ev);
  }
  cudaStreamSynchronize(b->e->stream);
  for (mhc_case* h : b->slots) case_free(h);
  engine_destroy(b->e);
  delete b;
  return MHC_OK;
}

void* mhc_batch_stream(mhc_batch* b) { return b ? (void*)b->e->stream : nullptr; }

int mhc_batch_add(mhc_batch* b, const mhc_case_params* params, long long iteration_limit, int* index) {
  if (!b || !params || !index) return set_err(MHC_ERR_ARG, "null argument");
  mhc_case* h = nullptr;
  int r = case_alloc(params, b->e->stream, &h);
  if (r) return r;
  if ((r = case_reset_scalars(h, iteration_limit > 0 ? iteration_limit : LLONG_MAX))) { case_free(h); return r; }
  h->initialised = false;
  *index = (int)b->slots.size();
  b->slots.push_back(h);
  b->detached.push_back(0);
  b->last.push_back(Scalars{});
  b->polled.push_back(Scalars{});
  b->polled_ok.push_back(0);
  b->e->cases.push_back(h);
  b->e->dirty = true;
  return MHC_OK;
}

int mhc_batch_init(mhc_batch* b) {
  if (!b) return set_err(MHC_ERR_ARG, "null batch");
  // start-init of the cases that have not run yet, through a temporary
  // engine on the batch stream, released later without waiting for the
  // work in flight
  reap_init_engines(b, false);
  Engine* tmp = nullptr;
  int r = engine_create(b->e->stream, &tmp);
  if (r) return r;
  for (mhc_case* h : b->e->cases)
    if (!h->initialised) tmp->cases.push_back(h);
  if (!tmp->cases.empty()) {
    if ((r = engine_rebuild(tmp))) { engine_destroy(tmp); return r; }
    launch_init(tmp);
    for (mhc_case* h : tmp->cases) {
      if (h->P.cas_model == MHC_CASE_RIDER && (r = rider_upload(h, tmp->stream))) return r;
      h->initialised = true;
    }
  }
  cudaError_t ce = cudaGetLastError();
  b->init_engines.push_back(tmp);
  if (ce != cudaSuccess) return set_err(MHC_ERR_CUDA, cudaGetErrorString(ce));
  b->e->dirty = true;
  return MHC_OK;
}

int mhc_batch_remove(mhc_batch* b, int index) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  mhc_case* h = b->slots[index];
  auto& v = b->e->cases;
  v.erase(std::remove(v.begin(), v.end(), h), v.end());
  b->e->dirty = true;
  case_free(h);  // stream-ordered: after the batch's work already queued
  b->slots[index] = nullptr;
  b->detached[index] = 0;
  return MHC_OK;
}

long long mhc_batch_checkpoint_bytes(mhc_batch* b, int index) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  return ckpt_bytes(b->slots[index]);
}

int mhc_batch_checkpoint(mhc_batch* b, int index, void* host, long long capacity) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  return ckpt_save(b->slots[index], b->e->stream, host, capacity);
}

int mhc_batch_restore(mhc_batch* b, int index, const void* host, long long size) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  int r = ckpt_restore(b->slots[index], b->e->stream, host, size);
  if (r) return r;
  b->e->dirty = true;
  return MHC_OK;
}

int mhc_batch_detach(mhc_batch* b, int index) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  if (b->detached[index]) return MHC_OK;
  mhc_case* h = b->slots[index];
  // a case that a completed poll saw finished (stopped, failed or at its
  // iteration limit) no longer changes: keep those scalars without waiting
  // for the work in flight; otherwise read them after it
  const Scalars& ps = b->polled[index];
  if (b->polled_ok[index] && (ps.status != 0 || ps.iteration_done >= ps.iteration_limit)) {
    b->last[index] = ps;
  } else {
    int r = read_scalars(h, b->e->stream, &b->last[index]);
    if (r) return r;
  }
  auto& v = b->e->cases;
  v.erase(std::remove(v.begin(), v.end(), h), v.end());
  b->e->dirty = true;
  b->detached[index] = 1;
  return MHC_OK;
}

int mhc_batch_poll(mhc_batch* b, int capacity, long long* iteration, int* status, double* time) {
  if (!b || capacity < 0) return set_err(MHC_ERR_ARG, "bad argument");
  Engine* e = b->e;
  int r = engine_rebuild(e);
  if (r) return r;
  const int n = (int)e->cases.size();
  if (n > e->gather_cap) {
    if (e->d_gather) CK(cudaFreeAsync(e->d_gather, e->stream));
    if (e->h_gather) { CK(cudaStreamSynchronize(e->stream)); pinned_put(e->h_gather, e->gather_cap * sizeof(Scalars)); }
    e->h_gather = nullptr;
    e->gather_cap = std::max(n, 2 * e->gather_cap);
    CK(cudaMallocAsync((void**)&e->d_gather, e->gather_cap * sizeof(Scalars), e->stream));
    if (int r = pinned_get(e->gather_cap * sizeof(Scalars), (void**)&e->h_gather)) return r;
  }
  if (n > 0) {
    kb_gather_scalars<<<cdiv(n, 128), 128, 0, e->stream>>>(e->d_desc, n, e->d_gather);
    ++e->launches;
    CK(cudaMemcpyAsync(e->h_gather, e->d_gather, n * sizeof(Scalars), cudaMemcpyDeviceToHost, e->stream));
  }
  CK(cudaStreamSynchronize(e->stream));
  const int ns = (int)b->slots.size();
  for (int i = 0; i < ns && i < capacity; ++i) {
    mhc_case* h = b->slots[i];
    const Scalars* sc = nullptr;
    if (!h) { if (iteration) iteration[i] = -1; if (status) status[i] = -1; if (time) time[i] = 0.; continue; }
    sc = b->detached[i] ? &b->last[i] : &e->h_gather[h->slot];
    if (iteration) iteration[i] = sc->iteration_done;
    if (status) status[i] = sc->status;
    if (time) time[i] = sc->t_done;
  }
  return ns;
}

int mhc_batch_poll_request(mhc_batch* b) {
  if (!b) return set_err(MHC_ERR_ARG, "null batch");
  Engine* e = b->e;
  int r = engine_rebuild(e);
  if (r) return r;
  const int k = b->poll_next;
  mhc_batch::Poll& P = b->poll[k];
  if (P.pending) CK(cudaEventSynchronize(P.ev));  // its buffers are about to be reused
  P.pending = false;
  const int n = (int)e->cases.size();
  if (!P.ev) CK(cudaEventCreateWithFlags(&P.ev, cudaEventDisableTiming));
  if (n > P.cap) {
    if (P.d) CK(cudaFreeAsync(P.d, e->stream));
    if (P.h) pinned_put(P.h, P.cap * sizeof(Scalars));
    P.h = nullptr;
    P.cap = std::max(n, 2 * P.cap);
    CK(cudaMallocAsync((void**)&P.d, P.cap * sizeof(Scalars), e->stream));
    if ((r = pinned_get(P.cap * sizeof(Scalars), (void**)&P.h))) return r;
  }
  P.index.assign(b->slots.size(), -1);
  for (size_t i = 0; i < b->slots.size(); ++i)
    if (b->slots[i] && !b->detached[i]) P.index[i] = b->slots[i]->slot;
  if (n > 0) {
    kb_gather_scalars<<<cdiv(n, 128), 128, 0, e->stream>>>(e->d_desc, n, P.d);
    ++e->launches;
    CK(cudaMemcpyAsync(P.h, P.d, n * sizeof(Scalars), cudaMemcpyDeviceToHost, e->stream));
  }
  CK(cudaEventRecord(P.ev, e->stream));
  P.pending = true;
  b->poll_next ^= 1;
  return k;
}

int mhc_batch_poll_wait(mhc_batch* b, int request, int capacity, long long* iteration, int* status, double* time) {
  if (!b || request < 0 || request > 1 || capacity < 0) return set_err(MHC_ERR_ARG, "bad argument");
  mhc_batch::Poll& P = b->poll[request];
  if (!P.pending) return set_err(MHC_ERR_ORDER, "no poll pending under this request");
  CK(cudaEventSynchronize(P.ev));
  P.pending = false;
  const int ns = (int)b->slots.size();
  for (int i = 0; i < ns; ++i) {
    const int idx = i < (int)P.index.size() ? P.index[i] : -1;
    const Scalars* sc = nullptr;
    if (b->slots[i] && b->detached[i]) sc = &b->last[i];
    else if (b->slots[i] && idx >= 0) {
      sc = &P.h[idx];
      b->polled[i] = *sc;
      b->polled_ok[i] = 1;
    }
    if (i >= capacity) continue;
    if (!b->slots[i]) { if (iteration) iteration[i] = -1; if (status) status[i] = -1; if (time) time[i] = 0.; }
    else if (!sc) { if (iteration) iteration[i] = 0; if (status) status[i] = 0; if (time) time[i] = 0.; }  // added after the poll
    else {
      if (iteration) iteration[i] = sc->iteration_done;
      if (status) status[i] = sc->status;
      if (time) time[i] = sc->t_done;
    }
  }
  return ns;
}

int mhc_batch_cycle(mhc_batch* b, int n) {
  if (!b) return set_err(MHC_ERR_ARG, "null batch");
  return engine_cycle(b->e, n);
}

int mhc_batch_cycle_graph(mhc_batch* b, int n) {
  if (!b) return set_err(MHC_ERR_ARG, "null batch");
  return engine_cycle_graph(b->e, n);
}

int mhc_batch_cycle_timed(mhc_batch* b, int n, double* stage_ms, long long* stage_launches) {
  if (!b || !stage_ms) return set_err(MHC_ERR_ARG, "null argument");
  return engine_timed(b->e, n, stage_ms, stage_launches);
}

int mhc_batch_synchronize(mhc_batch* b) {
  if (!b) return set_err(MHC_ERR_ARG, "null batch");
  CK(cudaStreamSynchronize(b->e->stream));
  return MHC_OK;
}

int mhc_batch_set_grid_scale(mhc_batch* b, int scale) {
  if (!b || scale < 0 || scale > 64) return set_err(MHC_ERR_ARG, "grid scale must be 0..64");
  b->e->grid_scale = scale;
  if (b->e->graph) { cudaGraphExecDestroy(b->e->graph); b->e->graph = nullptr; }
  return MHC_OK;
}

long long mhc_batch_launches(mhc_batch* b) { return b ? b->e->launches : -1; }

long long mhc_case_launches(mhc_case* h) { return (h && h->solo) ? h->solo->launches : (h ? 0 : -1); }

int mhc_batch_set_sweep_layout(mhc_batch* b, int cell_layout, int node_layout) {
  if (!b || cell_layout < 0 || cell_layout > 3 || node_layout < 0 || node_layout > 3)
    return set_err(MHC_ERR_ARG, "layouts are 0..3");
  b->e->cell_layout = cell_layout;
  b->e->node_layout = node_layout;
  b->e->dirty = true;
  return MHC_OK;
}

int mhc_case_set_sweep_layout(mhc_case* h, int cell_layout, int node_layout) {
  if (!h || cell_layout < 0 || cell_layout > 3 || node_layout < 0 || node_layout > 3)
    return set_err(MHC_ERR_ARG, "layouts are 0..3");
  int r = solo_engine(h);
  if (r) return r;
  h->solo->cell_layout = cell_layout;
  h->solo->node_layout = node_layout;
  h->solo->dirty = true;
  return MHC_OK;
}

int mhc_case_set_stage_grid_scale(mhc_case* h, int stage, int scale) {
  if (!h || stage < 0 || stage >= MHC_NUM_STAGES || scale < -1) return set_err(MHC_ERR_ARG, "bad stage or scale");
  int r = solo_engine(h);
  if (r) return r;
  h->solo->stage_scale[stage] = scale;
  if (h->solo->graph) h->solo->dirty = true;  // a captured graph holds the old grids
  return MHC_OK;
}

int mhc_batch_set_stage_grid_scale(mhc_batch* b, int stage, int scale) {
  if (!b || stage < 0 || stage >= MHC_NUM_STAGES || scale < -1 || scale > 64)
    return set_err(MHC_ERR_ARG, "stage must be 0..MHC_NUM_STAGES-1 and scale -1..64");
  b->e->stage_scale[stage] = scale;
  if (b->e->graph) { cudaGraphExecDestroy(b->e->graph); b->e->graph = nullptr; }
  return MHC_OK;
}

int mhc_batch_get_scalars(mhc_batch* b, int index, double* time, double* deltat, long long* iteration, int* status) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index]) return set_err(MHC_ERR_ARG, "bad case index");
  Scalars s;
  int r = read_scalars(b->slots[index], b->e->stream, &s);
  if (r) return r;
  if (time) *time = s.t_done;
  if (deltat) *deltat = s.dt;
  if (iteration) *iteration = s.iteration_done;
  if (status) *status = s.status;
  return MHC_OK;
}

long long mhc_batch_get_field(mhc_batch* b, int index, const char* name, int env, double* host, long long cap) {
  if (!b || index < 0 || index >= (int)b->slots.size() || !b->slots[index] || !name || !host)
    return set_err(MHC_ERR_ARG, "bad argument");
  return case_get_field(b->slots[index], b->e->stream, name, env, host, cap);
}
