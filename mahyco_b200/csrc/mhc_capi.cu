// mhc_capi.cu -- C ABI of the MaHyCo B200 library: case lifecycle, module
// entry points (fused into kernel stages), fused cycles and field access.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mahyco_b200.h"
#include "mhc_kernels.cuh"
#include "mhc_sweep.cuh"

using namespace mhc;

namespace {
thread_local std::string g_err;
int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CK(x)                                                                 \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess)                                                    \
      return set_err(MHC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

enum Stage {
  S_IDLE = 0, S_SAVED, S_VELOCITY, S_BC, S_POSITION, S_GEOM, S_DENSITY, S_VISCO,
  S_ELASTO, S_ENERGY, S_REMAP
};
}  // namespace

struct mhc_case {
  mhc_case_params P;
  Mesh M;
  int DIM = 3, NE = 1, NV = 4;
  Fields F;
  Scalars* d_scal = nullptr;
  cudaStream_t stream = nullptr;
  int sens_projection = 0;
  int stage = S_IDLE;
  bool initialised = false;
  std::vector<void*> allocs;
  cudaGraphExec_t graph = nullptr;
  int graph_n = 0;
  size_t lagrange_smem = 0;
  // optional per-stage timing: events recorded around every kernel group
  bool timing = false;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double stage_ms[MHC_NUM_STAGES] = {0};
  long long stage_launches[MHC_NUM_STAGES] = {0};
};

// brackets one kernel group with events on the case stream and accumulates
// its device time (only when timing is enabled)
struct StageTimer {
  mhc_case* h;
  int stage;
  StageTimer(mhc_case* h_, int s) : h(h_), stage(s) {
    if (h->timing) cudaEventRecord(h->ev[0], h->stream);
  }
  ~StageTimer() {
    if (!h->timing) return;
    cudaEventRecord(h->ev[1], h->stream);
    cudaEventSynchronize(h->ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    h->stage_ms[stage] += ms;
    h->stage_launches[stage] += 1;
  }
};

static long long count_doubles(const mhc_case_params* p, long long& ncell, long long& nnode) {
  int dim = p->dim;
  ncell = (long long)p->nx * p->ny * (dim == 3 ? p->nz : 1);
  nnode = (long long)(p->nx + 1) * (p->ny + 1) * (dim == 3 ? p->nz + 1 : 1);
  int ne = p->nb_env, nv = 3 * ne + 1;
  long long cells = 9 + (ne > 1 ? 8 * ne : 0) + 2 * nv + ne;
  long long nodes = 4 + 6 + 10;
  return cells * ncell + nodes * nnode;
}

// the API functions take their C linkage from the declarations in mahyco_b200.h

const char* mhc_last_error(void) { return g_err.c_str(); }
const char* mhc_version(void) { return "mahyco_b200 0.1 (sm_100a, fp64)"; }

long long mhc_case_device_bytes(const mhc_case_params* p) {
  if (!p) return -1;
  long long nc, nn;
  long long d = count_doubles(p, nc, nn);
  return d * 8 + nc + (long long)sizeof(Scalars);
}

static int validate(const mhc_case_params* p) {
  if (p->dim != 2 && p->dim != 3) return set_err(MHC_ERR_ARG, "dim must be 2 or 3");
  if (p->nx < 1 || p->ny < 1 || (p->dim == 3 && p->nz < 1)) return set_err(MHC_ERR_ARG, "mesh size");
  if (p->nb_env < 1 || p->nb_env > MHC_MAX_ENV) return set_err(MHC_ERR_ARG, "nb_env must be 1..4");
  if (p->nb_bc < 0 || p->nb_bc > MHC_MAX_BC) return set_err(MHC_ERR_ARG, "nb_bc");
  if (p->with_newton) return set_err(MHC_ERR_UNSUPPORTED, "with-newton energy update is not implemented");
  if (p->ordre_projection < 1 || p->ordre_projection > 2)
    return set_err(MHC_ERR_UNSUPPORTED, "ordre-projection must be 1 or 2");
  if (p->projection_limiteur_id < 0 || p->projection_limiteur_id > 2)
    return set_err(MHC_ERR_UNSUPPORTED, "only the classical limiters (0 minmod, 1 superbee, 2 vanleer)");
  if (p->is_euler_scheme != MHC_EULER_FULL) return set_err(MHC_ERR_UNSUPPORTED, "is-euler-scheme must be Full");
  for (int e = 0; e < p->nb_env; ++e) {
    if (p->env[e].density_damage_thresold != 0.0 || p->env[e].tension_damage_thresold > -1.e12)
      return set_err(MHC_ERR_UNSUPPORTED, "damage thresholds other than the defaults");
    if (p->env[e].eos < 0 || p->env[e].eos > 2) return set_err(MHC_ERR_ARG, "eos kind");
  }
  if (p->longueur_caracteristique == MHC_LENGTH_OPPOSITE_FACES && p->dim != 3)
    return set_err(MHC_ERR_UNSUPPORTED, "faces-opposees needs a 3D mesh");
  return MHC_OK;
}

int mhc_case_create(const mhc_case_params* params, mhc_case** out) {
  if (!params || !out) return set_err(MHC_ERR_ARG, "null argument");
  *out = nullptr;
  int v = validate(params);
  if (v != MHC_OK) return v;
  mhc_case* h = new mhc_case();
  h->P = *params;
  h->DIM = params->dim;
  h->NE = params->nb_env;
  h->NV = 3 * h->NE + 1;
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
  auto fail = [&](int code) { mhc_case_destroy(h); return code; };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_err(MHC_ERR_CUDA, "stream creation failed"));
  const long long N = M.ncell, NN = M.nnode;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    h->allocs.push_back(p);
    return p;
  };
  bool ok = true;
  auto dcell = [&]() { double* p = (double*)alloc(N * sizeof(double)); ok = ok && p; return p; };
  auto dnode = [&]() { double* p = (double*)alloc(NN * sizeof(double)); ok = ok && p; return p; };
  Fields& F = h->F;
  memset(&F, 0, sizeof(F));
  F.rho = dcell(); F.e = dcell(); F.p = dcell(); F.c = dcell(); F.q = dcell();
  F.m = dcell(); F.V = dcell(); F.l = dcell(); F.Veul = dcell();
  if (h->NE > 1) {
    auto denv = [&]() { double* p = (double*)alloc(h->NE * N * sizeof(double)); ok = ok && p; return p; };
    F.ef = denv(); F.emf = denv(); F.em = denv(); F.erho = denv();
    F.ee = denv(); F.ep = denv(); F.ec = denv(); F.eq = denv();
  }
  F.mask = (uint8_t*)alloc(N);
  ok = ok && F.mask;
  F.vx = dnode(); F.vy = dnode(); F.vz = dnode(); F.mn = dnode();
  for (int d = 0; d < 3; ++d) { F.Xp[d] = dnode(); F.Xn[d] = dnode(); }
  for (int b = 0; b < 2; ++b) {
    F.U[b] = (double*)alloc(h->NV * N * sizeof(double));
    F.Ud[b] = (double*)alloc(5 * NN * sizeof(double));
    ok = ok && F.U[b] && F.Ud[b];
  }
  F.mflux = (double*)alloc(h->NE * N * sizeof(double));
  h->d_scal = (Scalars*)alloc(sizeof(Scalars));
  ok = ok && F.mflux && h->d_scal;
  F.s = h->d_scal;
  if (!ok) {
    cudaGetLastError();
    return fail(set_err(MHC_ERR_NOMEM, "device allocation failed"));
  }
  if (h->NE > 1) {
    // env slots of cells that never hold the env must read as zero
    double* arr[] = {F.ef, F.emf, F.em, F.erho, F.ee, F.ep, F.ec, F.eq};
    for (double* a : arr)
      if (cudaMemsetAsync(a, 0, h->NE * N * sizeof(double), h->stream) != cudaSuccess)
        return fail(set_err(MHC_ERR_CUDA, "memset"));
  }
  h->lagrange_smem = (size_t)(LTX + 1) * (LTY + 1) * ((h->DIM == 3 ? 8 : 4) * 3 * sizeof(double) + 1);
  *out = h;
  return MHC_OK;
}

void* mhc_case_stream(mhc_case* h) { return h ? (void*)h->stream : nullptr; }

int mhc_case_destroy(mhc_case* h) {
  if (!h) return MHC_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (int i = 0; i < 2; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  for (void* p : h->allocs) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MHC_OK;
}

// ---------------------------------------------------------------------------
// template dispatch
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

template <int DIM, int NE>
static int launch_init(mhc_case* h) {
  const int T = 256;
  k_init_cells<DIM, NE><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F);
  k_init_nodes<DIM><<<blocks_for(h->M.nnode, T), T, 0, h->stream>>>(h->M, h->P, h->F);
  CK(cudaGetLastError());
  return MHC_OK;
}

template <int DIM>
static int launch_lagrange_nodes(mhc_case* h) {
  StageTimer tm(h, MHC_STAGE_LAGRANGE_NODES);
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(k_lagrange_nodes<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->lagrange_smem));
    attr_set = true;
  }
  dim3 grid((h->M.nnx + LTX - 1) / LTX, (h->M.nny + LTY - 1) / LTY,
            DIM == 3 ? (h->M.nnz + LZCHUNK - 1) / LZCHUNK : 1);
  k_lagrange_nodes<DIM><<<grid, LTX * LTY, h->lagrange_smem, h->stream>>>(h->M, h->P, h->F, h->P.with_projection ? 1 : 0);
  CK(cudaGetLastError());
  return MHC_OK;
}

template <int DIM, int NE>
static int launch_lagrange_cells(mhc_case* h) {
  StageTimer tm(h, MHC_STAGE_LAGRANGE_CELLS);
  const int T = 256;
  if (h->P.with_projection)
    k_lagrange_cells<DIM, NE, true><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F);
  else
    k_lagrange_cells<DIM, NE, false><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F);
  CK(cudaGetLastError());
  return MHC_OK;
}

// grid of the sweep tiles (SweepTile<D>): lanes along x, tile along D
template <int D>
static dim3 sweep_grid(int nx, int ny, int nz) {
  using T = SweepTile<D>;
  if (D == 0) return dim3((nx + T::TD - 1) / T::TD, ny, nz);
  if (D == 1) return dim3((nx + T::TW - 1) / T::TW, (ny + T::TD - 1) / T::TD, nz);
  return dim3((nx + T::TW - 1) / T::TW, (nz + T::TD - 1) / T::TD, ny);
}

template <int DIM, int NE, int D>
static void launch_sweep_dir(mhc_case* h, SweepArgs sa, DualArgs da) {
  const Mesh& M = h->M;
  {
    StageTimer tm(h, MHC_STAGE_SWEEP_CELLS);
    k_sweep_cells<DIM, NE, D><<<sweep_grid<D>(M.ncx, M.ncy, M.ncz), SweepTile<D>::THREADS, 0, h->stream>>>(
        h->M, h->P, h->F, sa);
  }
  {
    StageTimer tm(h, MHC_STAGE_SWEEP_NODES);
    k_sweep_nodes<DIM, NE, D><<<sweep_grid<D>(M.nnx, M.nny, M.nnz), SweepTile<D>::THREADS, 0, h->stream>>>(
        h->M, h->P, h->F, da);
  }
}

template <int DIM, int NE>
static int launch_remap(mhc_case* h) {
  // RemapADIService::appliRemap (RemapADIService.cc:15-90)
  int ub = 0, udb = 0;
  bool first = true;
  int done = 0;
  for (int i = 0; i < DIM; ++i) {
    int d = (i + h->sens_projection) % DIM;
    int ncd = d == 0 ? h->M.ncx : (d == 1 ? h->M.ncy : h->M.ncz);
    if (ncd == 1) continue;
    SweepArgs sa;
    sa.Uin = h->F.U[ub];
    sa.Uout = h->F.U[1 - ub];
    sa.first = first ? 1 : 0;
    sa.order = h->P.ordre_projection;
    sa.limiter = h->P.projection_limiteur_id;
    DualArgs da;
    da.Uin = first ? nullptr : h->F.Ud[udb];
    da.Uout = h->F.Ud[first ? 0 : 1 - udb];
    da.order = h->P.ordre_projection;
    da.limiter = h->P.projection_limiteur_id;
    da.done_dirs = done;
    if (d == 0) launch_sweep_dir<DIM, NE, 0>(h, sa, da);
    else if (d == 1) launch_sweep_dir<DIM, NE, 1>(h, sa, da);
    else if (DIM == 3) launch_sweep_dir<DIM, NE, (DIM == 3 ? 2 : 1)>(h, sa, da);
    ub = 1 - ub;
    udb = first ? 0 : 1 - udb;
    first = false;
    done |= 1 << d;
  }
  h->sens_projection = (h->sens_projection + 1) % DIM;
  const double* Ufin = h->F.U[ub];
  const double* Udfin = first ? nullptr : h->F.Ud[udb];
  const int T = 256;
  {
    StageTimer tm(h, MHC_STAGE_FINALIZE_CELLS);
    k_remap_finalize_cells<DIM, NE><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F, Ufin);
  }
  if (Udfin) {
    StageTimer tm(h, MHC_STAGE_FINALIZE_NODES);
    k_remap_finalize_nodes<DIM><<<blocks_for(h->M.nnode, T), T, 0, h->stream>>>(h->M, h->F, Udfin);
  }
  CK(cudaGetLastError());
  return MHC_OK;
}

template <int DIM>
static int launch_dt(mhc_case* h) {
  StageTimer tm(h, MHC_STAGE_DELTA_T);
  const int T = 256;
  k_delta_t<DIM><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F);
  k_delta_t_finalize<<<1, 1, 0, h->stream>>>(h->P, h->F);
  CK(cudaGetLastError());
  return MHC_OK;
}

#define DISPATCH_DN(fn, h)                                          \
  ((h)->DIM == 2 ? ((h)->NE == 1 ? fn<2, 1>(h) : (h)->NE == 2 ? fn<2, 2>(h) \
                    : (h)->NE == 3 ? fn<2, 3>(h) : fn<2, 4>(h))      \
                 : ((h)->NE == 1 ? fn<3, 1>(h) : (h)->NE == 2 ? fn<3, 2>(h) \
                    : (h)->NE == 3 ? fn<3, 3>(h) : fn<3, 4>(h)))
#define DISPATCH_D(fn, h) ((h)->DIM == 2 ? fn<2>(h) : fn<3>(h))

int mhc_hydro_start_init(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  Scalars s;
  memset(&s, 0, sizeof(s));
  s.t = h->P.deltat_init;  // global time of iteration 1
  s.dt = h->P.deltat_init;
  s.old_dt = 0.;
  s.iteration = 1;
  s.dt_min_bits = 0x7fefffffffffffffull;
  CK(cudaMemcpyAsync(h->d_scal, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  int r = DISPATCH_DN(launch_init, h);
  if (r != MHC_OK) return r;
  h->sens_projection = 0;
  h->stage = S_IDLE;
  h->initialised = true;
  return MHC_OK;
}

static void swap_positions(mhc_case* h) {
  for (int d = 0; d < 3; ++d) std::swap(h->F.Xp[d], h->F.Xn[d]);
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
  return DISPATCH_D(launch_lagrange_nodes, h);
}
int mhc_compute_geometric_values(mhc_case* h) { return expect(h, S_POSITION, S_GEOM); }
int mhc_update_density(mhc_case* h) { return expect(h, S_GEOM, S_DENSITY); }
int mhc_compute_artificial_viscosity(mhc_case* h) { return expect(h, S_DENSITY, S_VISCO); }
int mhc_update_elasticity_and_plasticity(mhc_case* h) { return expect(h, S_VISCO, S_ELASTO); }
int mhc_update_energy_and_pressure(mhc_case* h) {
  int r = expect(h, S_ELASTO, S_ENERGY);
  if (r) return r;
  return DISPATCH_DN(launch_lagrange_cells, h);
}
int mhc_remap(mhc_case* h) {
  int r = expect(h, S_ENERGY, S_REMAP);
  if (r) return r;
  if (!h->P.with_projection) return MHC_OK;
  return DISPATCH_DN(launch_remap, h);
}
int mhc_remap_apply(mhc_case* h) { return mhc_remap(h); }
int mhc_compute_delta_t(mhc_case* h) {
  int r = expect(h, S_REMAP, S_IDLE);
  if (r) return r;
  r = DISPATCH_D(launch_dt, h);
  swap_positions(h);
  return r;
}

static int one_iteration(mhc_case* h) {
  int r;
  if ((r = mhc_save_values_at_n(h))) return r;
  if ((r = mhc_update_velocity(h))) return r;
  if ((r = mhc_apply_boundary_condition(h))) return r;
  if ((r = mhc_update_position(h))) return r;
  if ((r = mhc_compute_geometric_values(h))) return r;
  if ((r = mhc_update_density(h))) return r;
  if ((r = mhc_compute_artificial_viscosity(h))) return r;
  if ((r = mhc_update_elasticity_and_plasticity(h))) return r;
  if ((r = mhc_update_energy_and_pressure(h))) return r;
  if ((r = mhc_remap(h))) return r;
  return mhc_compute_delta_t(h);
}

int mhc_cycle(mhc_case* h, int n) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  for (int it = 0; it < n; ++it) {
    int r = one_iteration(h);
    if (r) return r;
  }
  return MHC_OK;
}

int mhc_cycle_graph(mhc_case* h, int n) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (n <= 0) return MHC_OK;
  // the captured sequence depends on the direction rotation and on the
  // position buffer parity; a graph of dim*2 iterations returns both to
  // their starting state, so only multiples of that period are replayed
  const int period = 2 * h->DIM;
  if (n % period != 0 || h->stage != S_IDLE) return mhc_cycle(h, n);
  if (!h->graph || h->graph_n != period) {
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    int sp = h->sens_projection;
    double* xp[3] = {h->F.Xp[0], h->F.Xp[1], h->F.Xp[2]};
    double* xn[3] = {h->F.Xn[0], h->F.Xn[1], h->F.Xn[2]};
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int r = mhc_cycle(h, period);
    cudaGraph_t gg;
    cudaError_t e = cudaStreamEndCapture(h->stream, &gg);
    if (r) return r;
    if (e != cudaSuccess) return set_err(MHC_ERR_CUDA, cudaGetErrorString(e));
    g = gg;
    CK(cudaGraphInstantiate(&h->graph, g, 0));
    cudaGraphDestroy(g);
    h->graph_n = period;
    // capture did not execute anything: restore the host-side state
    h->sens_projection = sp;
    for (int d = 0; d < 3; ++d) { h->F.Xp[d] = xp[d]; h->F.Xn[d] = xn[d]; }
  }
  for (int r = 0; r < n / period; ++r) CK(cudaGraphLaunch(h->graph, h->stream));
  // host mirror of the state advanced by the replayed iterations
  h->sens_projection = (h->sens_projection + n) % h->DIM;
  if ((n & 1) != 0) swap_positions(h);
  return MHC_OK;
}

int mhc_cycle_timed(mhc_case* h, int n, double* stage_ms, long long* stage_launches) {
  if (!h || !stage_ms) return set_err(MHC_ERR_ARG, "null argument");
  if (!h->ev[0]) {
    CK(cudaEventCreate(&h->ev[0]));
    CK(cudaEventCreate(&h->ev[1]));
  }
  for (int s = 0; s < MHC_NUM_STAGES; ++s) { h->stage_ms[s] = 0.; h->stage_launches[s] = 0; }
  h->timing = true;
  int r = mhc_cycle(h, n);
  h->timing = false;
  for (int s = 0; s < MHC_NUM_STAGES; ++s) {
    stage_ms[s] = h->stage_ms[s];
    if (stage_launches) stage_launches[s] = h->stage_launches[s];
  }
  return r;
}

int mhc_synchronize(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  CK(cudaStreamSynchronize(h->stream));
  Scalars s;
  CK(cudaMemcpy(&s, h->d_scal, sizeof(s), cudaMemcpyDeviceToHost));
  return s.status;
}

int mhc_get_scalars(mhc_case* h, double* time, double* deltat, long long* iteration, int* status) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  CK(cudaStreamSynchronize(h->stream));
  Scalars s;
  CK(cudaMemcpy(&s, h->d_scal, sizeof(s), cudaMemcpyDeviceToHost));
  if (time) *time = s.t_done;
  if (deltat) *deltat = s.dt;
  if (iteration) *iteration = s.iteration_done;
  if (status) *status = s.status;
  return MHC_OK;
}

static int fetch(mhc_case* h, const void* dev, void* host, size_t bytes) {
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost));
  return MHC_OK;
}

long long mhc_get_field(mhc_case* h, const char* name, int env, double* host, long long cap) {
  if (!h || !name || !host) return set_err(MHC_ERR_ARG, "null argument");
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
    std::vector<double> g(N, 0.), e;
    std::vector<uint8_t> mask(N);
    int r;
    if ((r = fetch(h, F.mask, mask.data(), N))) return r;
    if (c.g) { if ((r = fetch(h, c.g, g.data(), N * 8))) return r; }
    if (env < 0) {
      if (!c.g) {  // global fraction of a cell: 1 for pure cells, not defined for mixed ones
        for (long long i = 0; i < N; ++i) host[i] = 1.;
      } else {
        memcpy(host, g.data(), N * 8);
      }
      return N;
    }
    if (h->NE > 1 && c.e) {
      e.resize(N);
      if ((r = fetch(h, c.e + env * N, e.data(), N * 8))) return r;
    }
    const bool volume = !strcmp(name, "CellVolume");
    std::vector<double> fr;
    if (volume && h->NE > 1) {
      fr.resize(N);
      if ((r = fetch(h, F.ef + env * N, fr.data(), N * 8))) return r;
    }
    for (long long i = 0; i < N; ++i) {
      bool in = (mask[i] >> env) & 1;
      bool pure = __builtin_popcount(mask[i]) == 1;
      if (!in) host[i] = 0.;
      else if (pure) host[i] = c.g ? g[i] : 1.;
      else if (volume) host[i] = fr[i] * g[i];
      else host[i] = c.e ? e[i] : 0.;
    }
    return N;
  }
  if (!strcmp(name, "EnvMask")) {
    if (cap < N) return set_err(MHC_ERR_ARG, "capacity too small");
    std::vector<uint8_t> mask(N);
    int r = fetch(h, F.mask, mask.data(), N);
    if (r) return r;
    for (long long i = 0; i < N; ++i) host[i] = mask[i];
    return N;
  }
  if (!strcmp(name, "NodeMass")) {
    if (cap < NN) return set_err(MHC_ERR_ARG, "capacity too small");
    int r = fetch(h, F.mn, host, NN * 8);
    return r ? r : NN;
  }
  if (!strcmp(name, "Velocity") || !strcmp(name, "NodeCoord")) {
    if (cap < 3 * NN) return set_err(MHC_ERR_ARG, "capacity too small");
    std::vector<double> a(NN), b(NN), c(NN);
    const double *pa, *pb, *pc;
    if (name[0] == 'V') { pa = F.vx; pb = F.vy; pc = F.vz; }
    else { pa = F.Xp[0]; pb = F.Xp[1]; pc = F.Xp[2]; }  // last Lagrangian positions
    int r;
    if ((r = fetch(h, pa, a.data(), NN * 8)) || (r = fetch(h, pb, b.data(), NN * 8)) ||
        (r = fetch(h, pc, c.data(), NN * 8)))
      return r;
    for (long long i = 0; i < NN; ++i) { host[3 * i] = a[i]; host[3 * i + 1] = b[i]; host[3 * i + 2] = c[i]; }
    return 3 * NN;
  }
  return set_err(MHC_ERR_ARG, std::string("unknown field ") + name);
}

template <int NE>
static int launch_eos(mhc_case* h, int env) {
  const int T = 256;
  k_eos_apply<NE><<<blocks_for(h->M.ncell, T), T, 0, h->stream>>>(h->M, h->P, h->F, env);
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_eos_apply(mhc_case* h, int env) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (env < 0 || env >= h->NE) return set_err(MHC_ERR_ARG, "env out of range");
  switch (h->NE) {
    case 1: return launch_eos<1>(h, env);
    case 2: return launch_eos<2>(h, env);
    case 3: return launch_eos<3>(h, env);
    default: return launch_eos<4>(h, env);
  }
}

int mhc_time_history(mhc_case* h, double* out) {
  if (!h || !out) return set_err(MHC_ERR_ARG, "null argument");
  const long long N = h->M.ncell;
  const int NE = h->NE;
  double t;
  int r = mhc_get_scalars(h, &t, nullptr, nullptr, nullptr);
  if (r) return r;
  out[0] = t;
  std::vector<double> m(N), p(N), rho(N), e(N), V(N), env(N);
  for (int q = 0; q < NE; ++q) {
    if (mhc_get_field(h, "CellMass", q, m.data(), N) < 0) return MHC_ERR_CUDA;
    if (mhc_get_field(h, "Pressure", q, p.data(), N) < 0) return MHC_ERR_CUDA;
    if (mhc_get_field(h, "Density", q, rho.data(), N) < 0) return MHC_ERR_CUDA;
    if (mhc_get_field(h, "InternalEnergy", q, e.data(), N) < 0) return MHC_ERR_CUDA;
    if (mhc_get_field(h, "CellVolume", q, V.data(), N) < 0) return MHC_ERR_CUDA;
    if (mhc_get_field(h, "EnvMask", -1, env.data(), N) < 0) return MHC_ERR_CUDA;
    long long cnt = 0;
    double sm = 0., sp = 0., rv = 0., vv = 0., em = 0., mm = 0.;
    for (long long c = 0; c < N; ++c) {
      if (!(((int)env[c] >> q) & 1)) continue;
      ++cnt; sm += m[c]; sp += p[c];
    }
    for (long long c = 0; c < N; ++c) {
      if (!(((int)env[c] >> q) & 1)) continue;
      em += e[c] * m[c]; mm += m[c];
    }
    for (long long c = 0; c < N; ++c) {
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

