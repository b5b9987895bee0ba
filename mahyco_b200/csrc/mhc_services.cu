// mhc_services.cu -- the per-method surface of the reference's services on
// a case: field upload (the inverse of mhc_get_field), the IEquationOfState
// methods one by one, and the IRemap methods (appliRemap split into its
// direction sweeps and remapVariables, the option getters).
//
// The fused time loop (mhc_cycle) does not use these entry points; they let
// a host that keeps the reference's module structure call each service
// method where the reference calls it.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "mhc_engine.cuh"

namespace {

using namespace mhc;

// initEOS on the cells of environment env: (pressure, density) -> (internal
// energy, sound speed); the global slot holds the value of a cell where env
// is alone
template <int NE>
__global__ void __launch_bounds__(CT) kb_eos_init_env(const CaseDesc* __restrict__ C, PhaseList L, int env) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    const Fields F = C[wi.c].F;
    const long long N = C[wi.c].M.ncell;
    const long long c = wi.x * (long long)CT + threadIdx.x;
    if (c >= N) continue;
    const uint8_t mask = F.mask[c];
    if (!((mask >> env) & 1)) continue;
    const mhc_env_params& o = C[wi.c].P->env[env];
    double e, cs;
    if (NE == 1 || __popc(mask) == 1) {
      eos_init(o, F.p[c], F.rho[c], e, cs);
      F.e[c] = e;
      F.c[c] = cs;
    } else {
      eos_init(o, F.ep[env * N + c], F.erho[env * N + c], e, cs);
      F.ee[env * N + c] = e;
      F.ec[env * N + c] = cs;
    }
  }
}

// applyOneCellEOS on one cell: pressure and sound speed in place, dp/de out
// (Fictif, FictifEOSService.cc:82-104: the pressure of the time, the
// internal energy reset to 0)
__global__ void kb_eos_one_cell(Fields F, mhc_env_params o, long long N, long long c, int env, int pure,
                                double* dpde_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long k = pure ? c : env * N + c;
  const double rho = pure ? F.rho[k] : F.erho[k], e = pure ? F.e[k] : F.ee[k];
  double p, cs, p2, dpde;
  if (o.eos == MHC_EOS_FICTIF) {
    fictif_apply(o, F.s->t, pure ? F.p[k] : F.ep[k], p, cs);
    dpde = (o.adiabatic_cst - 1.) * rho;
    if (pure) F.e[k] = 0.;
    else F.ee[k] = 0.;
  } else {
    eos_apply(o, rho, e, p, cs);
    eos_one_cell(o, rho, e, p2, dpde);
  }
  if (pure) { F.p[k] = p; F.c[k] = cs; }
  else { F.ep[k] = p; F.ec[k] = cs; }
  *dpde_out = dpde;
}

// Endommagement: the services' damage test on the global values of the env
// cells (PerfectGasEOSService.cc:92-118, StiffenedGasEOSService.cc:87-113,
// MieGruneisenEOSService.cc:150-176).  With the default density threshold
// (0, the only one accepted) density / initial density < 0 reduces to a
// negative density, the initial density being positive; Mie-Gruneisen
// tests the pressure only.
__global__ void __launch_bounds__(CT) kb_eos_damage_test(const CaseDesc* __restrict__ C, PhaseList L, int env) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    const Fields F = C[wi.c].F;
    const long long N = C[wi.c].M.ncell;
    const long long c = wi.x * (long long)CT + threadIdx.x;
    if (c >= N || !((F.mask[c] >> env) & 1)) continue;
    const mhc_env_params& o = C[wi.c].P->env[env];
    if (o.eos == MHC_EOS_FICTIF) continue;  // FictifEOSService::Endommagement does nothing
    const bool density_test = o.eos != MHC_EOS_MIE_GRUNEISEN && F.rho[c] < 0.;
    if (F.p[c] < o.tension_damage_thresold || density_test) atomicOr(&F.s->status, MHC_ST_DAMAGE);
  }
}

int check_env(mhc_case* h, int env) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (env < 0 || env >= h->NE) return set_err(MHC_ERR_ARG, "env out of range");
  return MHC_OK;
}

// state-changing calls outside the fused loop: after HydroStartInit,
// between iterations
int check_between_iterations(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != S_IDLE) return set_err(MHC_ERR_ORDER, "an iteration is in progress");
  return MHC_OK;
}

int upload(cudaStream_t s, void* dev, const void* host, size_t bytes) {
  if (bytes == 0) return MHC_OK;
  CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // the host buffer may be pageable and reused
  return MHC_OK;
}

// the remap arguments of the reference, checked against the case
int check_remap_args(mhc_case* h, int dimension, int with_dual, int nvars, int nenv) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (dimension != h->DIM) return set_err(MHC_ERR_ARG, "dimension differs from the case's");
  if (nenv != h->NE) return set_err(MHC_ERR_ARG, "nb_env differs from the case's");
  // the module passes withDualProjection = 1, 0 without Lagrange phase (PrepareRemap.cc:211)
  if (with_dual != (h->P.sans_lagrange ? 0 : 1))
    return set_err(MHC_ERR_ARG, "withDualProjection must be 1 (0 with sans-lagrange)");
  if (nvars != 18 * nenv && nvars != 3 * nenv + 5)
    return set_err(MHC_ERR_ARG, "nb_vars_to_project must be 18 nb_env or 3 nb_env + 5");
  return MHC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// option defaults
// ---------------------------------------------------------------------------
long long mhc_case_params_size(void) { return (long long)sizeof(mhc_case_params); }

void mhc_case_params_default(mhc_case_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->dim = 3;
  p->nx = p->ny = p->nz = 1;
  p->lx = p->ly = p->lz = 1.;
  p->nb_env = 1;
  for (int i = 0; i < MHC_MAX_ENV; ++i) {
    mhc_env_params& e = p->env[i];
    e.eos = MHC_EOS_PERFECT_GAS;
    e.adiabatic_cst = 1.4;
    e.tension_damage_thresold = -1.e12;
    e.s1 = 1.4;
    e.gamma0 = 1.97; e.a = 0.48; e.c0 = 5240.;
    e.temperature_ref = 300.;
    e.linear_pseudo_coeff = 0.5; e.quadratic_pseudo_coeff = 1.2;
    e.pression_initiale = 1.e5;
    e.rotation_order = 1;
    e.shear_modulus = 2.94e10; e.yield_strength = 3.e8;
    e.depot_cutoff[0] = e.depot_cutoff[1] = 1000.;
    e.depot_tfin = 1000.;
    e.depot_power = 4.;
  }
  p->cas_model = MHC_CASE_SOD;
  p->cas_test = MHC_TEST_SOD_X;
  p->sedov_energy = 0.244816;
  p->interface_pos = 0.5;
  p->calcul_vitson_max = 1;
  p->cfl = 0.3; p->deltat_init = 1.e-5; p->deltat_min = 1.e-8; p->deltat_max = 1.e-2;
  p->final_time = 1.e30;
  p->threshold = 1.e-10;
  p->with_projection = 1;
  for (int b = 0; b < MHC_MAX_BC; ++b) {
    p->bc[b].cutoff[0] = p->bc[b].cutoff[1] = 1000.;
    p->bc[b].power = 4.;
  }
  p->ordre_projection = 2;
  p->projection_limiteur_id = MHC_MINMOD;
  p->is_euler_scheme = MHC_EULER_FULL;
  p->remap_threshold = 1.e-10;
  p->time_history_period = 10;
  p->rider_radius = 0.15;
}

// ---------------------------------------------------------------------------
// initial fields (before HydroStartInit)
// ---------------------------------------------------------------------------
long long mhc_case_set_initial_field(mhc_case* h, const char* name, const double* host, long long n) {
  if (!h || !name || !host) return set_err(MHC_ERR_ARG, "null argument");
  if (h->initialised) return set_err(MHC_ERR_ORDER, "initial fields go before HydroStartInit");
  const long long N = h->M.ncell, NN = h->M.nnode;
  Fields& F = h->F;
  cudaStream_t st = h->stream;
  auto grow = [&](double** p, size_t bytes) -> int {
    if (*p) return MHC_OK;
    void* d = nullptr;
    CK(cudaMallocAsync(&d, bytes, st));
    h->allocs.push_back(d);
    h->alloc_bytes.push_back(bytes);
    *p = (double*)d;
    return MHC_OK;
  };
  int r;
  if (!strcmp(name, "NodeCoord")) {
    // a mesh file's grid: the initial positions of a Lagrangian case (the
    // remap and the pressure surfaces go back to the cartesian grid)
    if (h->P.with_projection) return set_err(MHC_ERR_UNSUPPORTED, "mesh-file coordinates with the remap");
    if (n < 3 * NN) return set_err(MHC_ERR_ARG, "too few values");
    std::vector<double> x(3 * NN);
    for (long long i = 0; i < NN; ++i)
      for (int d = 0; d < 3; ++d) x[d * NN + i] = host[3 * i + d];
    if ((r = grow(&F.x0, 3 * NN * sizeof(double))) || (r = upload(st, F.x0, x.data(), 3 * NN * 8))) return r;
    return 3 * NN;
  }
  const int slot = !strcmp(name, "Materiau") ? 0 : !strcmp(name, "Density") ? 1 : !strcmp(name, "Pressure") ? 2 : -1;
  if (slot < 0) return set_err(MHC_ERR_ARG, std::string("unknown initial field ") + name);
  if (h->P.cas_model != MHC_CASE_EXTERNAL)
    return set_err(MHC_ERR_ARG, "Materiau / Density / Pressure initial fields are for the EXTERNAL case model");
  if (n < N) return set_err(MHC_ERR_ARG, "too few values");
  if (!F.init) {
    // the ones not given: environment 0 and its initial state
    std::vector<double> d(3 * N);
    for (long long i = 0; i < N; ++i) {
      d[i] = 0.;
      d[N + i] = h->P.env[0].densite_initiale;
      d[2 * N + i] = h->P.env[0].pression_initiale;
    }
    if ((r = grow(&F.init, 3 * N * sizeof(double))) || (r = upload(st, F.init, d.data(), 3 * N * 8))) return r;
  }
  if ((r = upload(st, F.init + slot * N, host, N * 8))) return r;
  return N;
}

// ---------------------------------------------------------------------------
// field upload
// ---------------------------------------------------------------------------
long long mhc_set_field(mhc_case* h, const char* name, int env, const double* host, long long n) {
  if (!h || !name || !host) return set_err(MHC_ERR_ARG, "null argument");
  int r = check_between_iterations(h);
  if (r) return r;
  if (env >= h->NE) return set_err(MHC_ERR_ARG, "env out of range");
  const long long N = h->M.ncell, NN = h->M.nnode;
  Fields& F = h->F;
  cudaStream_t st = h->stream;
  struct { const char* n; double* g; double* e; } cells[] = {
      {"Density", F.rho, F.erho}, {"Pressure", F.p, F.ep}, {"InternalEnergy", F.e, F.ee},
      {"SoundSpeed", F.c, F.ec}, {"PseudoViscosity", F.q, F.eq}, {"CellMass", F.m, F.em},
      {"CellVolume", F.V, nullptr}, {"FracVol", nullptr, F.ef}, {"MassFraction", nullptr, F.emf},
      {"CaracteristicLength", F.l, nullptr}, {"EulerVolume", F.Veul, nullptr}};
  for (auto& c : cells) {
    if (strcmp(name, c.n)) continue;
    if (n < N) return set_err(MHC_ERR_ARG, "too few values");
    if (env < 0) {
      if (!c.g) return set_err(MHC_ERR_ARG, std::string(name) + " is an environment field: give env >= 0");
      return (r = upload(st, c.g, host, N * 8)) ? r : N;
    }
    if (!strcmp(name, "CellVolume")) return set_err(MHC_ERR_ARG, "CellVolume takes env < 0 (the env volume is f V)");
    if (!c.e && !c.g) return set_err(MHC_ERR_ARG, "field");
    // cells where env is alone keep its value in the global slot; mixed
    // cells in the environment array
    std::vector<uint8_t> mask(N);
    if ((r = fetch_shared(st, F.mask, mask.data(), N))) return r;
    std::vector<double> g, e;
    if (c.g) {
      g.resize(N);
      if ((r = fetch_shared(st, c.g, g.data(), N * 8))) return r;
    }
    const bool env_array = c.e && h->NE > 1;
    if (env_array) {
      e.resize(N);
      if ((r = fetch_shared(st, c.e + env * N, e.data(), N * 8))) return r;
    }
    // a pure cell's volume fraction lives in its environment's slot
    const bool fracvol = !strcmp(name, "FracVol");
    for (long long i = 0; i < N; ++i) {
      if (!((mask[i] >> env) & 1)) continue;
      const bool pure = __builtin_popcount(mask[i]) == 1;
      if (pure && c.g) g[i] = host[i];
      else if ((!pure || fracvol) && env_array) e[i] = host[i];
    }
    if (c.g && (r = upload(st, c.g, g.data(), N * 8))) return r;
    if (env_array && (r = upload(st, c.e + env * N, e.data(), N * 8))) return r;
    return N;
  }
  if (!strcmp(name, "Temperature")) {
    // the environment's temperature where it is present (env >= 0), or
    // every present environment's of a pure cell (env < 0)
    if (!F.T) return set_err(MHC_ERR_UNSUPPORTED, "the temperature is carried by Lagrangian runs only");
    if (n < N) return set_err(MHC_ERR_ARG, "too few values");
    std::vector<uint8_t> mask(N);
    std::vector<double> t((size_t)h->NE * N);
    if ((r = fetch_shared(st, F.mask, mask.data(), N)) || (r = fetch_shared(st, F.T, t.data(), h->NE * N * 8)))
      return r;
    for (long long i = 0; i < N; ++i) {
      if (env >= 0) {
        if ((mask[i] >> env) & 1) t[env * N + i] = host[i];
      } else if (__builtin_popcount(mask[i]) == 1) {
        t[(__builtin_ffs(mask[i]) - 1) * N + i] = host[i];
      }
    }
    return (r = upload(st, F.T, t.data(), h->NE * N * 8)) ? r : N;
  }
  if (!strcmp(name, "EnvMask")) {
    if (n < N) return set_err(MHC_ERR_ARG, "too few values");
    std::vector<uint8_t> mask(N);
    for (long long i = 0; i < N; ++i) {
      const double v = host[i];
      if (!(v >= 1. && v < (double)(1 << h->NE)) || v != (double)(int)v)
        return set_err(MHC_ERR_ARG, "EnvMask values are environment bit sets 1 .. 2^nb_env - 1");
      mask[i] = (uint8_t)v;
    }
    return (r = upload(st, F.mask, mask.data(), N)) ? r : N;
  }
  static const char* kStrain[] = {"StrainTensorXX", "StrainTensorYY", "StrainTensorZZ", "StrainTensorXY",
                                  "StrainTensorYZ", "StrainTensorXZ"};
  for (int q = 0; q < 6; ++q) {
    if (strcmp(name, kStrain[q])) continue;
    if (!F.S) return set_err(MHC_ERR_ARG, "the case has no elasto-plastic model");
    if (n < N) return set_err(MHC_ERR_ARG, "too few values");
    std::vector<double> s(N);
    for (long long i = 0; i < N; ++i) s[i] = -host[i];  // the outputs are minus the deviator
    return (r = upload(st, F.S + q * N, s.data(), N * 8)) ? r : N;
  }
  if (!strcmp(name, "NodeMass")) {
    if (n < NN) return set_err(MHC_ERR_ARG, "too few values");
    return (r = upload(st, F.mn, host, NN * 8)) ? r : NN;
  }
  const bool vn = !strcmp(name, "VelocityN");
  if (vn && !F.v0) return set_err(MHC_ERR_ARG, "VelocityN is kept by sans-lagrange cases only");
  if (!strcmp(name, "Velocity") || vn) {
    // VelocityN: the velocities at n of a sans-lagrange case, which the
    // node pass prescribes every iteration (m_velocity_n)
    if (n < 3 * NN) return set_err(MHC_ERR_ARG, "too few values");
    std::vector<double> a(NN), b(NN), c(NN);
    for (long long i = 0; i < NN; ++i) { a[i] = host[3 * i]; b[i] = host[3 * i + 1]; c[i] = host[3 * i + 2]; }
    double* d[3] = {F.vx, F.vy, F.vz};
    if (vn) { d[0] = F.v0; d[1] = F.v0 + NN; d[2] = F.v0 + 2 * NN; }
    if ((r = upload(st, d[0], a.data(), NN * 8)) || (r = upload(st, d[1], b.data(), NN * 8)) ||
        (r = upload(st, d[2], c.data(), NN * 8)))
      return r;
    return 3 * NN;
  }
  if (!strcmp(name, "NodeCoord"))
    return set_err(MHC_ERR_ARG, "NodeCoord is read-only (derived geometry of the last Lagrangian mesh)");
  return set_err(MHC_ERR_ARG, std::string("unknown field ") + name);
}

// ---------------------------------------------------------------------------
// IEquationOfState
// ---------------------------------------------------------------------------
int mhc_eos_init(mhc_case* h, int env) {
  int r = check_env(h, env);
  if (r || (r = check_between_iterations(h))) return r;
  if ((r = engine_rebuild_shared(h->solo))) return r;
  Engine* e = h->solo;
  for (Group& g : e->groups) {
    switch (g.NE) {
      case 1: plaunch(e, kb_eos_init_env<1>, CT, 0, g.init_cells, env); break;
      case 2: plaunch(e, kb_eos_init_env<2>, CT, 0, g.init_cells, env); break;
      case 3: plaunch(e, kb_eos_init_env<3>, CT, 0, g.init_cells, env); break;
      default: plaunch(e, kb_eos_init_env<4>, CT, 0, g.init_cells, env); break;
    }
  }
  if (h->F.T) {
    // initEOS also sets the environment's temperature (Lagrangian runs)
    CK(cudaMemsetAsync(&h->d_scal->eref_first[env], 0xff, sizeof(unsigned int), h->stream));
    for (Group& g : e->groups) {
      DISPATCH_GROUP(g, (plaunch(e, kb_eref_candidates<DIM_, NE_>, CT, 0, g.init_cells, env)));
      DISPATCH_GROUP(g, (plaunch(e, kb_init_temperature<DIM_, NE_>, CT, 0, g.init_cells, env)));
    }
  }
  if (h->F.hf && env == 0) {
    // and the initial density NewHypoModel divides by (one environment)
    const long long N = h->M.ncell;
    CK(cudaMemcpyAsync(h->F.hf + 9 * N, h->F.rho, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_eos_reinit(mhc_case* h, int env) { return check_env(h, env); }

int mhc_eos_apply_one_cell(mhc_case* h, int env, long long cell, double* dpde) {
  int r = check_env(h, env);
  if (r || (r = check_between_iterations(h))) return r;
  const long long N = h->M.ncell;
  if (cell < 0 || cell >= N) return set_err(MHC_ERR_ARG, "cell out of range");
  uint8_t mask = 0;
  CK(cudaMemcpyAsync(&mask, h->F.mask + cell, 1, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (!((mask >> env) & 1)) return set_err(MHC_ERR_ARG, "the cell does not hold this environment");
  const int pure = __builtin_popcount(mask) == 1;
  double* d_out = nullptr;  // stream-ordered, from the case stream's pool
  CK(cudaMallocAsync((void**)&d_out, sizeof(double), h->stream));
  kb_eos_one_cell<<<1, 32, 0, h->stream>>>(h->F, h->P.env[env], N, cell, env, pure, d_out);
  cudaError_t le = cudaGetLastError();
  double v = 0.;
  if (le == cudaSuccess) le = cudaMemcpyAsync(&v, d_out, 8, cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(d_out, h->stream);
  if (le == cudaSuccess) le = cudaStreamSynchronize(h->stream);
  if (le != cudaSuccess) return set_err(MHC_ERR_CUDA, std::string("applyOneCellEOS: ") + cudaGetErrorString(le));
  if (dpde) *dpde = v;
  return MHC_OK;
}

int mhc_eos_endommagement(mhc_case* h, int env) {
  int r = check_env(h, env);
  if (r || (r = check_between_iterations(h))) return r;
  if ((r = engine_rebuild_shared(h->solo))) return r;
  Engine* e = h->solo;
  for (Group& g : e->groups) plaunch(e, kb_eos_damage_test, CT, 0, g.init_cells, env);
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_eos_get_adiabatic_cst(mhc_case* h, int env, double* out) {
  int r = check_env(h, env);
  if (r) return r;
  if (!out) return set_err(MHC_ERR_ARG, "null argument");
  *out = h->P.env[env].adiabatic_cst;
  return MHC_OK;
}

int mhc_eos_get_density_damage_thresold(mhc_case* h, int env, double* out) {
  int r = check_env(h, env);
  if (r) return r;
  if (!out) return set_err(MHC_ERR_ARG, "null argument");
  *out = h->P.env[env].density_damage_thresold;
  return MHC_OK;
}

// ---------------------------------------------------------------------------
// IRemap
// ---------------------------------------------------------------------------
int mhc_remap_appli_remap(mhc_case* h, int dimension, int with_dual_projection, int nb_vars_to_project, int nb_env) {
  int r = check_remap_args(h, dimension, with_dual_projection, nb_vars_to_project, nb_env);
  return r ? r : mhc_remap(h);
}

int mhc_remap_sweeps(mhc_case* h) {
  if (!h) return set_err(MHC_ERR_ARG, "null case");
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != S_ENERGY) return set_err(MHC_ERR_ORDER, "entry point called out of time-loop order");
  h->stage = S_SWEPT;
  launch_remap_sweeps_shared(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_remap_variables(mhc_case* h, int dimension, int with_dual_projection, int nb_vars_to_project, int nb_env) {
  int r = check_remap_args(h, dimension, with_dual_projection, nb_vars_to_project, nb_env);
  if (r) return r;
  if (!h->initialised) return set_err(MHC_ERR_ORDER, "HydroStartInit has not run");
  if (h->stage != S_SWEPT) return set_err(MHC_ERR_ORDER, "remapVariables needs the remap sweeps first");
  h->stage = S_REMAP;
  launch_remap_variables_shared(h->solo);
  CK(cudaGetLastError());
  return MHC_OK;
}

int mhc_remap_resize_remap_variables(mhc_case* h, int nb_vars_to_project, int nb_env) {
  return check_remap_args(h, h ? h->DIM : 0, 1, nb_vars_to_project, nb_env);
}

int mhc_remap_synchronize_uremap(mhc_case* h) { return h ? MHC_OK : set_err(MHC_ERR_ARG, "null case"); }

int mhc_remap_get_ordre_projection(mhc_case* h) { return h ? h->P.ordre_projection : set_err(MHC_ERR_ARG, "null case"); }
int mhc_remap_has_projection_pente_borne(mhc_case* h) {
  return h ? (h->P.projection_pente_borne != 0) : set_err(MHC_ERR_ARG, "null case");
}
int mhc_remap_has_projection_simple_pente(mhc_case* h) {
  return h ? (h->P.projection_simple_pente != 0) : set_err(MHC_ERR_ARG, "null case");
}
int mhc_remap_has_conservation_energie_totale(mhc_case* h) {
  return h ? (h->P.conservation_energie_totale != 0) : set_err(MHC_ERR_ARG, "null case");
}

int mhc_remap_is_euler(mhc_case* h, char* out, int capacity) {
  if (!h || !out) return set_err(MHC_ERR_ARG, "null argument");
  const char* v = "Full";
  switch (h->P.is_euler_scheme) {
    case MHC_EULER_X: v = "X"; break;
    case MHC_EULER_Y: v = "Y"; break;
    case MHC_EULER_Z: v = "Z"; break;
    case MHC_EULER_NONE: v = "NON"; break;
    default: break;
  }
  if (capacity < (int)strlen(v) + 1) return set_err(MHC_ERR_ARG, "capacity too small");
  strcpy(out, v);
  return MHC_OK;
}
