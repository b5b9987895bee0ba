// mhc_kernels.cuh -- sm_100a kernels of one MaHyCo hydro cycle.
//
// Data layout (structure of arrays, FP64, device resident):
//   cell globals    rho e p c q m V l Veul          [ncell]
//   env slots       ef emf em erho ee ep ec eq      [NE][ncell]  (mixed cells only)
//   env mask        mask                            [ncell] (bit e = cell holds env e)
//   nodes           vx vy vz mn                     [nnode]
//   Lagrangian pos  Xp[3] (previous cycle), Xn[3] (this cycle)
//   remap           U[2][NV][ncell] (NV = 3*NE+1: volumes, masses, energies, pseudo*V)
//                   mflux[NE][ncell] (cell mass flux of the current sweep)
//                   Ud[2][5][nnode] (node momentum x3, mass, kinetic energy)
// A cell holding exactly one environment keeps that environment's values in
// the global slot (Arcane's pure-cell storage); env slots are read and
// written only for mixed cells.
//
// Every kernel follows the operation order of the reference function it
// replaces (cited per kernel) so that results match the CPU oracle.
#pragma once
#include "mhc_device.cuh"
#include "../../include/mahyco_case.h"

namespace mhc {

enum : int { ST_NEG_VOLUME = 1, ST_DT_UNDERFLOW = 2, ST_NAN = 4, ST_STOP = 8 };

// time-loop scalars living on the device (so that whole cycles can be
// replayed from a CUDA graph without host round trips)
struct Scalars {
  double t;          // global time of the iteration in progress
  double dt;         // deltat of the iteration in progress
  double old_dt;     // old deltat seen by the iteration in progress
  double t_done;     // time of the last completed iteration
  double dt_next;    // deltat computed by the last computeDeltaT
  long long iteration;       // iteration in progress (1-based)
  long long iteration_done;  // last completed iteration
  unsigned long long dt_min_bits;  // running min of l/(c+vmax) as ordered bits
  int status;        // ST_* flags
  int pad;
};

struct Fields {
  double *rho, *e, *p, *c, *q, *m, *V, *l, *Veul;
  double *ef, *emf, *em, *erho, *ee, *ep, *ec, *eq;
  uint8_t* mask;
  double *vx, *vy, *vz, *mn;
  double *Xp[3], *Xn[3];
  double* U[2];
  double* mflux;
  double* Ud[2];
  Scalars* s;
};

// ---------------------------------------------------------------------------
// equations of state
// ---------------------------------------------------------------------------
// Mie-Gruneisen pressure (MieGruneisenEOSService.cc:55-64); powers with
// integer exponents are evaluated correctly rounded.
__device__ __forceinline__ double mg_pressure(const mhc_env_params& o, double density, double e) {
  double J = o.rho0 / density;
  double mu = 1. / J - 1.;
  if (mu > 0.) {
    double num = o.rho0 * (o.c0 * o.c0) * mu * (1 + (1. - o.gamma0 / 2.) * mu - o.a * (mu * mu) / 2.);
    double onepm = 1. + mu;
    double b = (1. - (o.s1 - 1.) * mu - o.s2 * (mu * mu) / (1 + mu) - o.s2 * cube_rn(mu) / (onepm * onepm));
    double den = b * b;
    return num / den + (o.gamma0 + o.a * mu) * e;
  }
  return o.rho0 * (o.c0 * o.c0) * mu + (o.gamma0 + o.a * mu) * e;
}

// IEquationOfState::applyEOS for one environment cell (PerfectGas 45-67,
// StiffenedGas 43-63, MieGruneisen 44-97)
__device__ __forceinline__ void eos_apply(const mhc_env_params& o, double rho, double e, double& p, double& c) {
  if (o.eos == MHC_EOS_PERFECT_GAS) {
    double g = o.adiabatic_cst;
    p = (g - 1.) * rho * e;
    c = sqrt(g * p / rho);
  } else if (o.eos == MHC_EOS_STIFFENED_GAS) {
    double g = o.adiabatic_cst, pinf = o.limit_tension;
    p = ((g - 1.) * rho * e) - (g * pinf);
    c = sqrt((g / rho) * (p + pinf));
  } else {
    p = mg_pressure(o, rho, e);
    double p1 = mg_pressure(o, rho - 1.e-7, e);
    double p2 = mg_pressure(o, rho + 1.e-7, e);
    c = ((p2 - p1) > 0.) ? sqrt((p2 - p1) / 2.e-7) : 1.e4;
  }
}

// IEquationOfState::initEOS for one environment cell: (p, rho) -> (e, c)
__device__ __forceinline__ void eos_init(const mhc_env_params& o, double p, double rho, double& e, double& c) {
  if (o.eos == MHC_EOS_PERFECT_GAS) {
    double g = o.adiabatic_cst;
    e = p / ((g - 1.) * rho);
    c = sqrt(g * p / rho);
  } else if (o.eos == MHC_EOS_STIFFENED_GAS) {
    double g = o.adiabatic_cst, pinf = o.limit_tension;
    e = (p + (g * pinf)) / ((g - 1.) * rho);
    c = sqrt((g / rho) * (p + pinf));
  } else {
    e = p / o.gamma0;
    c = o.c0;
  }
}

__device__ __forceinline__ double char_length(const mhc_case_params& P, int DIM, double V, const R3* coord) {
  int lc = P.longueur_caracteristique;
  if (lc == MHC_LENGTH_CUBE_ROOT_VOLUME) return DIM == 2 ? sqrt(V) : pow_one_third(V);
  if (lc == MHC_LENGTH_OPPOSITE_FACES) {
    R3 fc[6];
    hex_face_centres(coord, fc);
    double d1 = norm(fc[0] - fc[3]), d2 = norm(fc[2] - fc[5]), d3 = norm(fc[1] - fc[4]);
    return (d1 * d2 * d3) / (d1 * d2 + d1 * d3 + d2 * d3);
  }
  int d = lc - MHC_LENGTH_MONODIM_X;
  return fabs(comp(coord[2], d) - comp(coord[0], d));
}

// cell geometry: corner normals, volume (MahycoModule.cc:1097-1162)
template <int DIM>
__device__ __forceinline__ double cell_volume(const R3* coord, R3* cqs) {
  if (DIM == 3) {
    R3 fc[6];
    hex_face_centres(coord, fc);
    cqs3(coord, fc, cqs);
  } else {
    cqs2(coord, cqs);
  }
  double volume = 0.;
  for (int n = 0; n < (DIM == 3 ? 8 : 4); ++n) volume += dot(coord[n], cqs[n]);
  return volume / DIM;
}

__device__ __forceinline__ bool node_on_surface(const Mesh& M, int i, int j, int k, int surf) {
  switch (surf) {
    case MHC_XMIN: return i == 0;
    case MHC_XMAX: return i == M.nnx - 1;
    case MHC_YMIN: return j == 0;
    case MHC_YMAX: return j == M.nny - 1;
    // in 2D every face lies on z = zmin = zmax (PrepareFaceGroup)
    case MHC_ZMIN: return M.dim == 2 || k == 0;
    default: return M.dim == 2 || k == M.nnz - 1;
  }
}

// ---------------------------------------------------------------------------
// init: MahycoModule::hydroStartInit + computeCellMass (MahycoModule.cc:21-237)
// ---------------------------------------------------------------------------
template <int DIM, int NE>
__global__ void k_init_cells(Mesh M, mhc_case_params P, Fields F) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  const int NBN = DIM == 3 ? 8 : 4;
  R3 coord[8];
  R3 s = {0., 0., 0.};
  for (int l = 0; l < NBN; ++l) {
    int a, b, d;
    local_node_offset(l, a, b, d);
    coord[l] = node_x0(M, i + a, j + b, k + d);
    s = s + coord[l];
  }
  R3 cc = (DIM == 2 ? .25 : .125) * s;
  // materials (SODService::initMat, SEDOVService::initMat, MahycoAnnexe.cc:102-139)
  double mat = 0.;
  if (P.cas_model == MHC_CASE_SOD) {
    if (P.cas_test == MHC_TEST_BISOD_X || P.cas_test == MHC_TEST_BISOD_Y || P.cas_test == MHC_TEST_BISOD_Z)
      mat = (comp(cc, P.cas_test - MHC_TEST_BISOD_X) < 0.5) ? 0. : 1.;
  } else if (P.cas_model == MHC_CASE_TWO_STATE) {
    if (NE > 1) mat = (comp(cc, P.interface_dir) < P.interface_pos) ? 0. : 1.;
  } else if (P.cas_model == MHC_CASE_SEDOV && P.cas_test != MHC_TEST_SEDOV) {
    bool center = false;
    for (int l = 0; l < NBN; ++l) {
      R3 x = coord[l];
      if (sqrt(x.x * x.x + x.y * x.y + x.z * x.z) < 1.e-10) center = true;
    }
    mat = center ? 1. : 0.;
  }
  uint8_t mask;
  if (mat == 0.) mask = 1;
  else if (mat > 0. && mat < 1.) mask = 3;
  else if (mat == 1.) mask = 2;
  else if (mat > 1. && mat < 2.) mask = 6;
  else if (mat == 2.) mask = 4;
  else if (mat > 2. && mat < 3.) mask = 12;
  else if (mat == 3.) mask = 8;
  else mask = 15;
  mask &= (uint8_t)((1 << NE) - 1);
  const bool pure = __popc(mask) == 1;
  // geometry
  R3 cqs[8];
  double V = cell_volume<DIM>(coord, cqs);
  if (V < 0.) atomicOr(&F.s->status, ST_NEG_VOLUME);
  double l = char_length(P, DIM, V, coord);
  // state: globals g*, env slots *e[]
  double rho = 0., p = 0., e = 0., cs = 0.;
  double rhoe[NE], pe[NE], ee[NE], ce[NE];
  for (int q = 0; q < NE; ++q) { rhoe[q] = pe[q] = ee[q] = ce[q] = 0.; }
  if (P.cas_model == MHC_CASE_SOD) {
    bool mono = P.cas_test == MHC_TEST_SOD_X || P.cas_test == MHC_TEST_SOD_Y || P.cas_test == MHC_TEST_SOD_Z;
    if (mono) {
      double r = comp(cc, P.cas_test - MHC_TEST_SOD_X);
      if (r < 0.5) { p = P.env[0].pression_initiale; rho = P.env[0].densite_initiale; }
      else { p = P.env[0].pression_initiale / 10.; rho = P.env[0].densite_initiale / 8.; }
    } else {
      int st = (mat == 0) ? 0 : 1;
      rho = P.env[st].densite_initiale;
      p = P.env[st].pression_initiale;
      if (!pure)
        for (int q = 0; q < NE; ++q)
          if ((mask >> q) & 1) { rhoe[q] = P.env[st].densite_initiale; pe[q] = P.env[st].pression_initiale; }
    }
  } else if (P.cas_model == MHC_CASE_TWO_STATE) {
    int st = (comp(cc, P.interface_dir) < P.interface_pos) ? 0 : 1;
    rho = P.env[st].densite_initiale;
    p = P.env[st].pression_initiale;
  } else if (P.cas_model == MHC_CASE_SEDOV) {
    double rhoInit = P.env[0].densite_initiale, pInit = P.env[0].pression_initiale;
    if (P.cas_test == MHC_TEST_SEDOV) e = 0.244816e-5;
    rho = rhoInit;
    p = pInit;
    bool center = false;
    for (int l2 = 0; l2 < NBN; ++l2) {
      R3 x = coord[l2];
      double rn = DIM == 3 ? sqrt(x.x * x.x + x.y * x.y + x.z * x.z) : sqrt(x.x * x.x + x.y * x.y);
      if (rn < 1.e-10) center = true;
    }
    if (center) {
      e += P.sedov_energy / V;
      p = 0.4 * rhoInit * e;
    }
  }
  // EOS init per environment (aliased for pure cells)
  for (int q = 0; q < NE; ++q) {
    if (!((mask >> q) & 1)) continue;
    if (pure) eos_init(P.env[q], p, rho, e, cs);
    else eos_init(P.env[q], pe[q], rhoe[q], ee[q], ce[q]);
  }
  double fe[NE], mfe[NE];
  for (int q = 0; q < NE; ++q) { fe[q] = 1.0; mfe[q] = 1.0; }
  if (!pure) {
    e = 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((mask >> q) & 1)) continue;
      e += ee[q] * mfe[q];
      cs = smax(ce[q], cs);
      rho += rhoe[q] * fe[q];
      p += pe[q] * fe[q];
    }
  }
  double m = rho * V;
  double me[NE];
  for (int q = 0; q < NE; ++q) me[q] = mfe[q] * m;
  F.rho[c] = rho; F.e[c] = e; F.p[c] = p; F.c[c] = cs; F.q[c] = 0.;
  F.m[c] = pure ? 1.0 * m : m;
  F.V[c] = V; F.l[c] = l; F.Veul[c] = V;
  F.mask[c] = mask;
  if (NE > 1 && !pure) {
    for (int q = 0; q < NE; ++q) {
      F.ef[q * N + c] = fe[q]; F.emf[q * N + c] = mfe[q]; F.em[q * N + c] = me[q];
      F.erho[q * N + c] = rhoe[q]; F.ee[q * N + c] = ee[q]; F.ep[q * N + c] = pe[q];
      F.ec[q * N + c] = ce[q]; F.eq[q * N + c] = 0.;
    }
  }
}

// computeNodeMass (MahycoModule.cc:247-262): gather of 1/8 (1/4) cell masses in
// ascending cell id; also initial velocity and Lagrangian positions.
template <int DIM>
__device__ __forceinline__ double node_mass_gather(const Mesh& M, const double* cm, int i, int j, int k) {
  const double w = DIM == 2 ? .25 : .125;
  double s = 0.;
  for (int dk = (DIM == 3 ? -1 : 0); dk <= 0; ++dk) {
    int ck = k + dk;
    if (DIM == 3 && (ck < 0 || ck >= M.ncz)) continue;
    for (int dj = -1; dj <= 0; ++dj) {
      int cj = j + dj;
      if (cj < 0 || cj >= M.ncy) continue;
      for (int di = -1; di <= 0; ++di) {
        int ci = i + di;
        if (ci < 0 || ci >= M.ncx) continue;
        s += w * cm[cell_id(M, ci, cj, DIM == 3 ? ck : 0)];
      }
    }
  }
  return s;
}

template <int DIM>
__global__ void k_init_nodes(Mesh M, mhc_case_params P, Fields F) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= M.nnode) return;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  R3 x = node_x0(M, i, j, k);
  F.Xp[0][n] = x.x; F.Xp[1][n] = x.y; F.Xp[2][n] = x.z;
  double vx = 0., vy = 0., vz = 0.;
  if (P.cas_model == MHC_CASE_SOD) {
    vx = P.env[0].vitesse_initiale[0]; vy = P.env[0].vitesse_initiale[1]; vz = P.env[0].vitesse_initiale[2];
  }
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  F.mn[n] = node_mass_gather<DIM>(M, F.m, i, j, k);
}

// ---------------------------------------------------------------------------
// Lagrange, node pass: updateVelocity + applyBoundaryCondition + updatePosition
// (MahycoModule.cc:438-501, 756-807, 730-741).
//
// The force on a node is the sum over its <= 8 cells, in ascending cell id,
// of (p_n + q_n) * CQS_n where CQS_n are the corner normals of the previous
// Lagrangian mesh.  Blocks own a TX x TY tile of node columns and march along
// z: each step computes the corner forces of one cell layer into shared
// memory once, finishes the node plane below it and starts the one above,
// so every corner normal is computed once per (tile, layer) and no atomics
// are used.
// ---------------------------------------------------------------------------
constexpr int LTX = 16, LTY = 16;
constexpr int LZCHUNK = 16;

template <int DIM>
__global__ void __launch_bounds__(LTX * LTY) k_lagrange_nodes(Mesh M, mhc_case_params P, Fields F, int euler) {
  constexpr int CW = LTX + 1, CH = LTY + 1, NCL = CW * CH;
  extern __shared__ double smem_dyn[];
  double* corner = smem_dyn;  // [NCL][NBN][3] corner forces of one cell layer
  unsigned char* cvalid = reinterpret_cast<unsigned char*>(smem_dyn + NCL * (DIM == 3 ? 8 : 4) * 3);
  const int tx = threadIdx.x % LTX, ty = threadIdx.x / LTX;
  const int i0 = blockIdx.x * LTX, j0 = blockIdx.y * LTY;
  const int ni = i0 + tx, nj = j0 + ty;
  const bool node_ok = ni < M.nnx && nj < M.nny;
  const int NBN = DIM == 3 ? 8 : 4;
  const double dt = F.s->dt;
  const double dth = 0.5 * (F.s->old_dt + dt);
  const double t = F.s->t;
  int kz0 = 0, kz1 = 1;
  if (DIM == 3) {
    kz0 = blockIdx.z * LZCHUNK;
    kz1 = min(kz0 + LZCHUNK, M.nnz);
  }
  R3 S = {0., 0., 0.};
  for (int L = (DIM == 3 ? kz0 - 1 : 0); L < (DIM == 3 ? kz1 : 1); ++L) {
    // corner forces of cell layer L
    for (int cl = threadIdx.x; cl < NCL; cl += LTX * LTY) {
      int a = cl % CW, b = cl / CW;
      int ci = i0 - 1 + a, cj = j0 - 1 + b;
      bool ok = ci >= 0 && ci < M.ncx && cj >= 0 && cj < M.ncy && (DIM == 2 || (L >= 0 && L < M.ncz));
      cvalid[cl] = ok;
      if (!ok) continue;
      int ck = DIM == 3 ? L : 0;
      R3 coord[8];
      for (int l = 0; l < NBN; ++l) {
        int da, db, dc;
        local_node_offset(l, da, db, dc);
        long long nn = node_id(M, ci + da, cj + db, ck + dc);
        coord[l] = {F.Xp[0][nn], F.Xp[1][nn], F.Xp[2][nn]};
      }
      R3 cq[8];
      if (DIM == 3) {
        R3 fc[6];
        hex_face_centres(coord, fc);
        cqs3(coord, fc, cq);
      } else {
        cqs2(coord, cq);
      }
      long long cc = cell_id(M, ci, cj, ck);
      double pr = F.p[cc] + F.q[cc];
      double* dst = &corner[cl * NBN * 3];
      for (int l = 0; l < NBN; ++l) {
        R3 fv = pr * cq[l];
        dst[3 * l] = fv.x; dst[3 * l + 1] = fv.y; dst[3 * l + 2] = fv.z;
      }
    }
    __syncthreads();
    if (node_ok) {
      // cells around node (ni,nj): local index (a,b) = (tx + di, ty + dj), di,dj in {0,1}
      const int c00 = ty * CW + tx, c10 = ty * CW + tx + 1, c01 = (ty + 1) * CW + tx, c11 = (ty + 1) * CW + tx + 1;
      auto add = [&](R3& acc, int cl, int l) {
        if (!cvalid[cl]) return;
        const double* src = &corner[cl * NBN * 3 + 3 * l];
        acc.x = acc.x + src[0]; acc.y = acc.y + src[1]; acc.z = acc.z + src[2];
      };
      int kplane = DIM == 3 ? L : 0;
      if (DIM == 2 || L >= kz0) {
        // bottoms of layer L complete node plane L
        if (DIM == 3) { add(S, c00, 2); add(S, c10, 3); add(S, c01, 1); add(S, c11, 0); }
        else { add(S, c00, 2); add(S, c10, 3); add(S, c01, 1); add(S, c11, 0); }
        long long n = node_id(M, ni, nj, kplane);
        double mnode = F.mn[n];
        double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
        double f = dth / mnode;
        vx = vx + f * S.x; vy = vy + f * S.y; vz = vz + f * S.z;
        vx = vx + dth * P.gravity[0]; vy = vy + dth * P.gravity[1]; vz = vz + dth * P.gravity[2];
        const double eps = 1.e-8;
        for (int b = 0; b < P.nb_bc; ++b) {
          const mhc_bc& bc = P.bc[b];
          if ((t - dt * (1 - eps)) < bc.tdebut) continue;
          if ((t - dt * (1 - eps)) > bc.tfin) continue;
          if (!node_on_surface(M, ni, nj, kplane, bc.surface)) continue;
          if (bc.kind == MHC_BC_VX) vx = bc.value;
          else if (bc.kind == MHC_BC_VY) vy = bc.value;
          else if (bc.kind == MHC_BC_VZ) vz = bc.value;
        }
        R3 x = euler ? node_x0(M, ni, nj, kplane) : R3{F.Xp[0][n], F.Xp[1][n], F.Xp[2][n]};
        F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
        F.Xn[0][n] = x.x + dt * vx; F.Xn[1][n] = x.y + dt * vy; F.Xn[2][n] = x.z + dt * vz;
      }
      if (DIM == 3 && L + 1 < kz1) {
        // tops of layer L start node plane L+1
        S = {0., 0., 0.};
        add(S, c00, 6); add(S, c10, 7); add(S, c01, 5); add(S, c11, 4);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Lagrange, cell pass: computeGeometricValues + updateDensity +
// computeArtificialViscosity + updateEnergyAndPressure
// (MahycoModule.cc:1097-1316, 386-426, 1430-1502, 1623-1698, 1708-1735).
// EULER: the results are packed directly into the remap conserved variables
// (PrepareRemap.cc:94-193).  Otherwise the EOS is applied here
// (Lagrange-only time loop).
// ---------------------------------------------------------------------------
template <int DIM, int NE, bool EULER>
__global__ void __launch_bounds__(256) k_lagrange_cells(Mesh M, mhc_case_params P, Fields F) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  constexpr int NV = 3 * NE + 1;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  const int NBN = DIM == 3 ? 8 : 4;
  R3 coord[8];
  for (int l = 0; l < NBN; ++l) {
    int a, b, d;
    local_node_offset(l, a, b, d);
    long long nn = node_id(M, i + a, j + b, k + d);
    coord[l] = {F.Xn[0][nn], F.Xn[1][nn], F.Xn[2][nn]};
  }
  R3 cqs[8];
  const double V = cell_volume<DIM>(coord, cqs);
  if (V < 0.) atomicOr(&F.s->status, ST_NEG_VOLUME);
  const double l = char_length(P, DIM, V, coord);
  const uint8_t mask = F.mask[c];
  const bool pure = __popc(mask) == 1;
  const double dt = F.s->dt;
  // state at n (global slots) and env slots of mixed cells
  const double rho_n = F.rho[c], e_n = F.e[c], p_n = F.p[c], q_n = F.q[c], cs = F.c[c], m = F.m[c];
  double fe[NE], mfe[NE], me[NE], rhone[NE], ene[NE], pne[NE], qne[NE];
  for (int q = 0; q < NE; ++q) {
    if (NE > 1 && !pure && ((mask >> q) & 1)) {
      fe[q] = F.ef[q * N + c]; mfe[q] = F.emf[q * N + c]; me[q] = F.em[q * N + c];
      rhone[q] = F.erho[q * N + c]; ene[q] = F.ee[q * N + c]; pne[q] = F.ep[q * N + c]; qne[q] = F.eq[q * N + c];
    } else {
      fe[q] = mfe[q] = 1.; me[q] = m; rhone[q] = rho_n; ene[q] = e_n; pne[q] = p_n; qne[q] = q_n;
    }
  }
  // updateDensity
  double Ve[NE], rhoe[NE], taue[NE];
  for (int q = 0; q < NE; ++q) {
    if (!((mask >> q) & 1)) { Ve[q] = rhoe[q] = taue[q] = 0.; continue; }
    Ve[q] = pure ? V : fe[q] * V;
    rhoe[q] = me[q] / Ve[q];
    taue[q] = 0.5 * (1.0 / rhone[q] + 1.0 / rhoe[q]);
  }
  double rho = m / V;
  double tau = 0.5 * (1.0 / rho_n + 1.0 / rho);
  double divu = 1.0 / dt * (1.0 / rho - 1.0 / rho_n) / tau;
  if (pure) {
    for (int q = 0; q < NE; ++q)
      if ((mask >> q) & 1) { rhoe[q] = rho; taue[q] = tau; }
  }
  // computeArtificialViscosity
  double qe[NE];
  for (int q = 0; q < NE; ++q) {
    qe[q] = 0.;
    if (!((mask >> q) & 1)) continue;
    if (divu < 0.0) {
      double a1 = P.env[q].linear_pseudo_coeff, a2 = P.env[q].quadratic_pseudo_coeff;
      qe[q] = 1. / taue[q] * (-a1 * l * cs * divu + a2 * l * l * divu * divu);
    }
  }
  double qg = 0.;
  if (pure) {
    for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) qg = qe[q];
  } else {
    for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) qg += qe[q] * fe[q];
  }
  // updateEnergyAndPressure
  double ee_[NE], pe[NE], ce[NE];
  for (int q = 0; q < NE; ++q) {
    ee_[q] = pe[q] = ce[q] = 0.;
    if (!((mask >> q) & 1)) continue;
    double qq = pure ? qg : qe[q];
    double qn = qne[q];
    double r = rhoe[q], rn = rhone[q];
    if (P.pression_explicite) {
      ee_[q] = ene[q] - (pne[q] + qq) * (1.0 / r - 1.0 / rn);
      eos_apply(P.env[q], r, ee_[q], pe[q], ce[q]);
    } else {
      double pseudo = 0.;
      if (P.pseudo_centree && ((qn + qq) * (1.0 / r - 1.0 / rn) < 0.)) pseudo = 0.5 * (qq + qn);
      if (!P.pseudo_centree && (qq * (1.0 / r - 1.0 / rn) < 0.)) pseudo = qq;
      double g = P.env[q].adiabatic_cst;
      double den = 1 + 0.5 * (g - 1.0) * r * (1.0 / r - 1.0 / rn);
      double num = ene[q] - (0.5 * pne[q] + pseudo) * (1.0 / r - 1.0 / rn);
      ee_[q] = num / den;
    }
  }
  if (EULER) {
    // computeVariablesForRemap: U = (V_e, V_e rho_e, V_e rho_e e_e, V q)
    double* U = F.U[0];
    for (int q = 0; q < NE; ++q) {
      bool in = (mask >> q) & 1;
      double Vq = in ? Ve[q] : 0., rq = in ? rhoe[q] : 0.;
      U[q * N + c] = Vq;
      U[(NE + q) * N + c] = in ? Vq * rq : 0.;
      U[(2 * NE + q) * N + c] = in ? Vq * rq * ee_[q] : 0.;
    }
    U[(NV - 1) * N + c] = V * qg;
    F.V[c] = V;
    F.l[c] = l;
    return;
  }
  // Lagrange-only loop: mixed energy average, EOS, pressure average
  double eg = 0.;
  if (pure) {
    for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) eg = ee_[q];
  } else {
    for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) eg += mfe[q] * ee_[q];
  }
  double pg = 0., cg = 0.;
  if (!P.pression_explicite) {
    for (int q = 0; q < NE; ++q) {
      if (!((mask >> q) & 1)) continue;
      double r = pure ? rho : rhoe[q];
      double ev = pure ? eg : ee_[q];
      eos_apply(P.env[q], r, ev, pe[q], ce[q]);
    }
  }
  if (pure) {
    for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) { pg = pe[q]; cg = ce[q]; }
  } else {
    double option = P.calcul_vitson_max ? 1. : 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((mask >> q) & 1)) continue;
      pg += fe[q] * pe[q];
      cg = option * smax(ce[q], cg);
      cg += (1. - option) * fe[q] * ce[q];
    }
  }
  F.rho[c] = rho; F.e[c] = eg; F.p[c] = pg; F.c[c] = cg; F.q[c] = qg; F.V[c] = V; F.l[c] = l;
  if (NE > 1 && !pure) {
    for (int q = 0; q < NE; ++q) {
      if (!((mask >> q) & 1)) continue;
      F.erho[q * N + c] = rhoe[q]; F.ee[q * N + c] = ee_[q]; F.ep[q * N + c] = pe[q];
      F.ec[q * N + c] = ce[q]; F.eq[q * N + c] = qe[q];
    }
  }
}

// ---------------------------------------------------------------------------
// remap sweep, cell part: computeGradPhiFace + computeGradPhiCell +
// computeUpwindFaceQuantitiesForProjection + computeUremap for direction D
// (RemapADIService.cc:119-575, UtilesRemap.cc:108-120, 325-357, classical
// limiters, order <= 2).  Face quantities of the Lagrangian mesh
// (PrepareRemap.cc:18-59) are rebuilt from the node positions: initial face
// normals are the unit axis vectors of the cartesian grid, so every
// dot(., n) reduces to the D component.
// ---------------------------------------------------------------------------
struct SweepArgs {
  const double* Uin;
  double* Uout;
  int first;
  int order;
  int limiter;
};

template <int DIM, int D>
__device__ __forceinline__ void face_node_ijk(int i, int j, int k, int q, int& a, int& b, int& cz) {
  // re-ordered face nodes: smallest uid first, then the smaller neighbour
  a = i; b = j; cz = k;
  if (DIM == 2) {
    if (D == 0) b += q; else a += q;
    return;
  }
  int s1 = (q == 1 || q == 2), s2 = (q == 2 || q == 3);
  if (D == 0) { b += s1; cz += s2; }
  else if (D == 1) { a += s1; cz += s2; }
  else { a += s1; b += s2; }
}

template <int DIM, int NE, int D>
__global__ void __launch_bounds__(256) k_sweep_cells(Mesh M, mhc_case_params P, Fields F, SweepArgs A) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  constexpr int NV = 3 * NE + 1;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  const int id = D == 0 ? i : (D == 1 ? j : k);
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  const long long stride = D == 0 ? 1 : (D == 1 ? (long long)M.ncx : (long long)M.ncx * M.ncy);
  const double dt = F.s->dt;
  const int NBN = DIM == 3 ? 8 : 4;
  const double wc = DIM == 2 ? .25 : .125;
  const double wf = DIM == 2 ? .5 : .25;
  const double* Xd = F.Xn[D];
  double phi[5][NV];
  double xc[5];
  bool ex[5];
  for (int s = 0; s < 5; ++s) {
    int is = id + s - 2;
    ex[s] = is >= 0 && is < nd;
    if (!ex[s]) continue;
    long long cs = c + (s - 2) * stride;
    double u[NV];
    for (int v = 0; v < NV; ++v) u[v] = A.Uin[v * N + cs];
    double den;
    if (A.first) den = F.V[cs];
    else { den = 0.; for (int q = 0; q < NE; ++q) den += u[q]; }
    for (int v = 0; v < NV; ++v) phi[s][v] = u[v] / den;
    int ci = i, cj = j, ck = k;
    if (D == 0) ci += s - 2; else if (D == 1) cj += s - 2; else ck += s - 2;
    double sum = 0.;
    for (int l = 0; l < NBN; ++l) {
      int a, b, d;
      local_node_offset(l, a, b, d);
      sum += Xd[node_id(M, ci + a, cj + b, ck + d)];
    }
    xc[s] = wc * sum;
  }
  // faces: back (between s=1,2) and front (between s=2,3)
  double fcd[2], un[2], L[2], ond[2];
  for (int f = 0; f < 2; ++f) {
    int fi = i, fj = j, fk = k;
    if (D == 0) fi += f; else if (D == 1) fj += f; else fk += f;
    long long fn[4];
    int nfn = DIM == 3 ? 4 : 2;
    double fc = 0., vm = 0.;
    const double* vD = D == 0 ? F.vx : (D == 1 ? F.vy : F.vz);
    for (int q = 0; q < nfn; ++q) {
      int a, b, cz;
      face_node_ijk<DIM, D>(fi, fj, fk, q, a, b, cz);
      fn[q] = node_id(M, a, b, cz);
      fc = fc + wf * Xd[fn[q]];
      vm = vm + vD[fn[q]];
    }
    fcd[f] = fc;
    un[f] = wf * vm;
    if (DIM == 3) {
      R3 x0 = {F.Xn[0][fn[0]], F.Xn[1][fn[0]], F.Xn[2][fn[0]]};
      R3 x1 = {F.Xn[0][fn[1]], F.Xn[1][fn[1]], F.Xn[2][fn[1]]};
      R3 x2 = {F.Xn[0][fn[2]], F.Xn[1][fn[2]], F.Xn[2][fn[2]]};
      R3 x3 = {F.Xn[0][fn[3]], F.Xn[1][fn[3]], F.Xn[2][fn[3]]};
      R3 v1 = x2 - x0, v2 = x3 - x1;
      if (D == 0) L[f] = 0.5 * fabs(produit(v1.y, v2.z, v1.z, v2.y));
      else if (D == 1) L[f] = 0.5 * fabs(produit(v2.x, v1.z, v2.z, v1.x));
      else L[f] = 0.5 * fabs(produit(v1.x, v2.y, v1.y, v2.x));
    } else {
      const double* Xt = F.Xn[1 - D];
      L[f] = fabs(Xt[fn[1]] - Xt[fn[0]]);
    }
    // outer normal of this cell at the face, from the initial grid
    // (MahycoModule.cc:1070-1091)
    R3 sc = {0., 0., 0.};
    for (int l = 0; l < NBN; ++l) {
      int a, b, d;
      local_node_offset(l, a, b, d);
      sc = sc + node_x0(M, i + a, j + b, k + d);
    }
    R3 cc0 = wc * sc;
    R3 fc0 = {0., 0., 0.};
    for (int q = 0; q < nfn; ++q) {
      int a, b, cz;
      face_node_ijk<DIM, D>(fi, fj, fk, q, a, b, cz);
      fc0 = fc0 + wf * node_x0(M, a, b, cz);
    }
    R3 diff = fc0 - cc0;
    ond[f] = comp(diff / norm(diff), D);
  }
  const int order2 = A.order - 1;
  double* Uo = A.Uout;
  double mf_out[NE];
  for (int q = 0; q < NE; ++q) mf_out[q] = 0.;
  double uo[NV];
  for (int v = 0; v < NV; ++v) {
    // face gradients (faces between s and s+1, s = 0..3)
    double gface[4];
    for (int s = 0; s < 4; ++s)
      gface[s] = (ex[s] && ex[s + 1]) ? (phi[s + 1][v] - phi[s][v]) / (xc[s + 1] - xc[s]) : 0.;
    double grad[5] = {0., 0., 0., 0., 0.};
    if (A.order > 1)
      for (int s = 1; s <= 3; ++s)
        if (ex[s]) grad[s] = limited_gradient(A.limiter, gface[s - 1], gface[s]);
    double flux[2] = {0., 0.};
    bool fex[2] = {ex[1], ex[3]};
    for (int f = 0; f < 2; ++f) {
      if (!fex[f]) continue;
      int sb = 1 + f, sf = 2 + f;
      double dx = xc[sf] - xc[sb];
      int su = (un[f] * dx > 0.0) ? sb : sf;
      double pf = phi[su][v] + order2 * (fcd[f] - xc[su]) * grad[su];
      flux[f] = ond[f] * un[f] * L[f] * dt * pf;
    }
    double ff = 0.;
    double dual = 0.;
    // cell local face order: 3D back then front; 2D x: front then back
    int fa = (DIM == 2 && D == 0) ? 1 : 0, fb = 1 - fa;
    if (fex[fa]) { ff += flux[fa]; dual += 0.5 * flux[fa] * ond[fa]; }
    if (fex[fb]) { ff += flux[fb]; dual += 0.5 * flux[fb] * ond[fb]; }
    uo[v] = A.Uin[v * N + c] - ff;
    if (v >= NE && v < 2 * NE) mf_out[v - NE] = dual;
  }
  for (int q = 0; q < NE; ++q) {
    if (uo[NE + q] < 0.) uo[NE + q] = 0.;
    if (uo[2 * NE + q] < 0.) uo[2 * NE + q] = 0.;
  }
  for (int v = 0; v < NV; ++v) Uo[v * N + c] = uo[v];
  for (int q = 0; q < NE; ++q) F.mflux[q * N + c] = mf_out[q];
}

// ---------------------------------------------------------------------------
// remap sweep, node part: RemapADIService::computeDualUremap
// (DualPhaseRemap.cc:38-258, classical limiter)
// ---------------------------------------------------------------------------
struct DualArgs {
  const double* Uin;   // null on the first sweep (U built from m and v)
  double* Uout;
  int order;
  int limiter;
  int done_dirs;       // bit d: direction d already swept this cycle
};

template <int DIM>
__device__ __forceinline__ bool node_inner(const Mesh& M, int i, int j, int k, int d) {
  int id = d == 0 ? i : (d == 1 ? j : k);
  int nn = d == 0 ? M.nnx : (d == 1 ? M.nny : M.nnz);
  return id > 0 && id < nn - 1;
}

template <int DIM, int NE, int D>
__global__ void __launch_bounds__(256) k_sweep_nodes(Mesh M, mhc_case_params P, Fields F, DualArgs A) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= M.nnode) return;
  const long long NN = M.nnode, N = M.ncell;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  const long long stride = D == 0 ? 1 : (D == 1 ? (long long)M.nnx : (long long)M.nnx * M.nny);
  auto loadU = [&](long long m, double* U) {
    if (A.Uin) {
      for (int q = 0; q < 5; ++q) U[q] = A.Uin[q * NN + m];
    } else {
      double mn = F.mn[m], vx = F.vx[m], vy = F.vy[m], vz = F.vz[m];
      U[0] = mn * vx; U[1] = mn * vy; U[2] = mn * vz; U[3] = mn;
      U[4] = 0.5 * mn * (vx * vx + vy * vy + vz * vz);
    }
  };
  double U[5];
  loadU(n, U);
  const bool inner = node_inner<DIM>(M, i, j, k, D);
  if (!inner) {
    for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
    return;
  }
  const int id = D == 0 ? i : (D == 1 ? j : k);
  // Phi of nodes id-2..id+2 and their Lagrangian coordinate along D
  double Ph[5][5], xd[5];
  bool exn[5];
  const int nn = D == 0 ? M.nnx : (D == 1 ? M.nny : M.nnz);
  for (int s = 0; s < 5; ++s) {
    int is = id + s - 2;
    exn[s] = is >= 0 && is < nn;
    if (!exn[s]) continue;
    long long m = n + (s - 2) * stride;
    xd[s] = F.Xn[D][m];
    int mi = i, mj = j, mk = k;
    if (D == 0) mi += s - 2; else if (D == 1) mj += s - 2; else mk += s - 2;
    bool was_inner = false;
    for (int d = 0; d < DIM; ++d)
      if (((A.done_dirs >> d) & 1) && node_inner<DIM>(M, mi, mj, mk, d)) was_inner = true;
    double Um[5];
    loadU(m, Um);
    if (was_inner) {
      Ph[s][0] = Um[0] / Um[3]; Ph[s][1] = Um[1] / Um[3]; Ph[s][2] = Um[2] / Um[3];
      Ph[s][3] = Um[3]; Ph[s][4] = Um[4] / Um[3];
    } else {
      double vx = F.vx[m], vy = F.vy[m], vz = F.vz[m];
      Ph[s][0] = vx; Ph[s][1] = vy; Ph[s][2] = vz; Ph[s][3] = F.mn[m];
      Ph[s][4] = 0.5 * (vx * vx + vy * vy + vz * vz);
    }
  }
  // limited node gradients at id-1, id, id+1 (velocity components only)
  double G[5][5];
  for (int s = 0; s < 5; ++s)
    for (int q = 0; q < 5; ++q) G[s][q] = 0.;
  if (A.order > 1) {
    for (int s = 1; s <= 3; ++s) {
      int is = id + s - 2;
      if (!(is > 0 && is < nn - 1)) continue;
      for (int q = 0; q < 3; ++q) {
        double gf = (Ph[s + 1][q] - Ph[s][q]) / (xd[s + 1] - xd[s]);
        double gb = (Ph[s][q] - Ph[s - 1][q]) / (xd[s] - xd[s - 1]);
        G[s][q] = limited_gradient(A.limiter, gb, gf);
      }
    }
  }
  // node mass fluxes: faces of the node plane in face id order, then envs
  const double w = DIM == 2 ? .5 : .25;
  double bfm = 0., ffm = 0.;
  {
    int nt1 = DIM == 3 ? 2 : 1;
    for (int b2 = 0; b2 < nt1; ++b2) {
      for (int b1 = 0; b1 < 2; ++b1) {
        // transverse cell indices (t1 minor, t2 major)
        int ci = i, cj = j, ck = k;
        int t1 = b1 - 1, t2 = b2 - 1;
        if (D == 0) { cj += t1; ck += (DIM == 3 ? t2 : 0); }
        else if (D == 1) { ci += t1; ck += (DIM == 3 ? t2 : 0); }
        else { ci += t1; cj += t2; }
        if (ci < 0 || cj < 0 || ck < 0) continue;
        if (D != 0 && ci >= M.ncx) continue;
        if (D != 1 && cj >= M.ncy) continue;
        if (DIM == 3 && D != 2 && ck >= M.ncz) continue;
        // behind the plane: index along D = id-1; ahead: id
        int bi = ci, bj = cj, bk = ck;
        if (D == 0) bi = id - 1; else if (D == 1) bj = id - 1; else bk = id - 1;
        int fi = ci, fj = cj, fk = ck;
        if (D == 0) fi = id; else if (D == 1) fj = id; else fk = id;
        int ndc = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
        if (id - 1 >= 0) {
          long long cb = cell_id(M, bi, bj, DIM == 3 ? bk : 0);
          for (int q = 0; q < NE; ++q) bfm += w * F.mflux[q * N + cb];
        }
        if (id < ndc) {
          long long cf = cell_id(M, fi, fj, DIM == 3 ? fk : 0);
          for (int q = 0; q < NE; ++q) ffm += w * F.mflux[q * N + cf];
        }
      }
    }
  }
  const double dt = F.s->dt;
  const int order2 = A.order - 1;
  U[3] += bfm - ffm;
  double FV[3], BV[3], FE, BE;
  {
    double ufront = 0.5 * (Ph[2][D] + Ph[3][D]);
    int signfront = (ufront > 0) ? 1 : -1;
    int src = (ffm < 0.) ? 3 : 2;
    double geo = (signfront * (xd[3] - xd[2]) - dt * ufront);
    for (int q = 0; q < 3; ++q) FV[q] = Ph[src][q] + order2 * (0.5 * G[src][q] * geo);
    FE = Ph[src][4] + order2 * (0.5 * G[src][4] * geo);
  }
  {
    double uback = 0.5 * (Ph[1][D] + Ph[2][D]);
    int signback = (uback > 0) ? 1 : -1;
    int src = (bfm > 0.) ? 1 : 2;
    double geo = (signback * (xd[2] - xd[1]) - dt * uback);
    for (int q = 0; q < 3; ++q) BV[q] = Ph[src][q] + order2 * (0.5 * G[src][q] * geo);
    BE = Ph[src][4] + order2 * (0.5 * G[src][4] * geo);
  }
  for (int q = 0; q < 3; ++q) U[q] += bfm * BV[q] - ffm * FV[q];
  U[4] += bfm * BE - ffm * FE;
  for (int q = 0; q < 3; ++q)
    if (fabs(U[q]) < 1.e-300) U[q] = 0.;
  for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
}

// ---------------------------------------------------------------------------
// remap finalize, cells: RemapADIService::remapVariables (RemapADIFinal.cc:21-319)
// then applyEOS per environment and computePressionMoyenne
// (PrepareRemap.cc:242-249, MahycoModule.cc:1708-1735)
// ---------------------------------------------------------------------------
template <int DIM, int NE>
__global__ void __launch_bounds__(256) k_remap_finalize_cells(Mesh M, mhc_case_params P, Fields F, const double* Ufin) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  constexpr int NV = 3 * NE + 1;
  const double thr = P.remap_threshold;
  double u[NV];
  for (int v = 0; v < NV; ++v) u[v] = Ufin[v * N + c];
  const double Veul = F.Veul[c];
  const uint8_t old = F.mask[c];
  uint8_t nm = old;
  for (int q = 0; q < NE; ++q) {
    bool in = (old >> q) & 1;
    if (((u[q] / Veul) < thr || (u[NE + q] == 0.)) && in) {
      nm &= (uint8_t)~(1 << q);
    } else if ((u[q] / Veul) > thr && !in) {
      double volt = 0.;
      for (int r = 0; r < NE; ++r) volt += u[r];
      double vn = u[q] * Veul / volt;
      if ((vn / Veul) > thr && u[NE + q] != 0.) nm |= (uint8_t)(1 << q);
    }
  }
  const bool oldpure = __popc(old) == 1;
  const bool pure = __popc(nm) == 1;
  // mass fractions survive a cell whose total mass is below threshold^2
  double mfe[NE], mfg;
  mfg = 1.;
  for (int q = 0; q < NE; ++q) mfe[q] = 0.;
  {
    // previous values with the pure-cell storage transfer of the env manager
    for (int q = 0; q < NE; ++q) {
      bool was = (old >> q) & 1;
      if (!was) continue;
      mfe[q] = (NE > 1 && !oldpure) ? F.emf[q * N + c] : 1.;
    }
    if (pure) for (int q = 0; q < NE; ++q) if ((nm >> q) & 1) mfg = ((old >> q) & 1) ? mfe[q] : 1.;
  }
  double vol[NE], dens[NE], ener[NE];
  double volt = 0., masset = 0.;
  for (int q = 0; q < NE; ++q) { vol[q] = u[q]; volt += vol[q]; masset += u[NE + q]; }
  double unsurvolt = 1. / volt;
  for (int q = 0; q < NE; ++q) vol[q] *= Veul * unsurvolt;
  double unsurvol = 1. / Veul;
  double fe[NE], fg = 0.;
  for (int q = 0; q < NE; ++q) fe[q] = 0.;
#define EVF(q) (*(pure ? &fg : &fe[q]))
#define EVMF(q) (*(pure ? &mfg : &mfe[q]))
  double somme_frac = 0.;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    EVF(q) = vol[q] * unsurvol;
    if (EVF(q) < thr) EVF(q) = 0.;
    somme_frac += EVF(q);
  }
  double unsursf = 0.;
  if (somme_frac != 0.) unsursf = 1. / somme_frac;
  for (int q = 0; q < NE; ++q)
    if ((nm >> q) & 1) EVF(q) *= unsursf;
  if (masset > thr * thr) {
    double unsurm = 1. / masset, fm = 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((nm >> q) & 1)) continue;
      EVMF(q) = u[NE + q] * unsurm;
      if (EVF(q) < thr) EVMF(q) = 0.;
      fm += EVMF(q);
    }
    if (fm != 0.) {
      double unsurfm = 1. / fm;
      for (int q = 0; q < NE; ++q)
        if ((nm >> q) & 1) EVMF(q) *= unsurfm;
    }
  }
  double dn = 0.;
  for (int q = 0; q < NE; ++q) {
    dens[q] = 0.;
    if (!((nm >> q) & 1)) continue;
    if (EVF(q) > thr && vol[q] != 0.) dens[q] = u[NE + q] / vol[q];
    dn += EVF(q) * dens[q];
  }
  for (int q = 0; q < NE; ++q) {
    ener[q] = 0.;
    if (!((nm >> q) & 1)) continue;
    if (EVF(q) > thr && u[NE + q] != 0.) ener[q] = u[2 * NE + q] / u[NE + q];
  }
  // aliased stores: g* are the global slots, e*[] the env slots
  double rhog = dn;
  double mg = Veul * dn;
  double eg = 0., qg = 0.;
  double me[NE], rhoe[NE], ee[NE], qe[NE];
  for (int q = 0; q < NE; ++q) { me[q] = rhoe[q] = ee[q] = qe[q] = 0.; }
  double en = 0., ps = 0.;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    if (pure) {
      mg = mfg * mg;
      qg = u[NV - 1] * unsurvol;
      rhog = dens[q];
      eg = ener[q];
      en += mfg * eg;
      ps += fg * qg;
    } else {
      me[q] = mfe[q] * mg;
      qe[q] = u[NV - 1] * unsurvol;
      rhoe[q] = dens[q];
      ee[q] = ener[q];
      en += mfe[q] * ee[q];
      ps += fe[q] * qe[q];
    }
  }
  eg = en;
  qg = ps;
  int st = 0;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    double& r = pure ? rhog : rhoe[q];
    double& ie = pure ? eg : ee[q];
    if (r < 0. || ie < 0.) {
      ie = 0.; r = 0.; EVF(q) = 0.; EVMF(q) = 0.;
    }
    if (r != r || ie != ie) st |= ST_NAN;
  }
  if (st) atomicOr(&F.s->status, st);
  // applyEOS per environment, then computePressionMoyenne
  double pg = 0., cg = 0., pe[NE], ce[NE];
  for (int q = 0; q < NE; ++q) { pe[q] = ce[q] = 0.; }
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    if (pure) eos_apply(P.env[q], rhog, eg, pg, cg);
    else eos_apply(P.env[q], rhoe[q], ee[q], pe[q], ce[q]);
  }
  if (!pure) {
    pg = 0.; cg = 0.;
    double option = P.calcul_vitson_max ? 1. : 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((nm >> q) & 1)) continue;
      pg += fe[q] * pe[q];
      cg = option * smax(ce[q], cg);
      cg += (1. - option) * fe[q] * ce[q];
    }
  }
#undef EVF
#undef EVMF
  F.rho[c] = rhog; F.e[c] = eg; F.p[c] = pg; F.c[c] = cg; F.q[c] = qg; F.m[c] = mg;
  F.V[c] = Veul;
  F.mask[c] = nm;
  if (NE > 1 && !pure) {
    for (int q = 0; q < NE; ++q) {
      F.ef[q * N + c] = fe[q]; F.emf[q * N + c] = mfe[q]; F.em[q * N + c] = me[q];
      F.erho[q * N + c] = rhoe[q]; F.ee[q * N + c] = ee[q]; F.ep[q * N + c] = pe[q];
      F.ec[q * N + c] = ce[q]; F.eq[q * N + c] = qe[q];
    }
  }
}

// remap finalize, nodes: velocity from projected momentum and node mass
// rebuilt from the new cell masses (RemapADIFinal.cc:287-319)
template <int DIM>
__global__ void __launch_bounds__(256) k_remap_finalize_nodes(Mesh M, Fields F, const double* Ud) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= M.nnode) return;
  const long long NN = M.nnode;
  double m = Ud[3 * NN + n];
  if (m != 0.) {
    F.vx[n] = Ud[n] / m;
    F.vy[n] = Ud[NN + n] / m;
    F.vz[n] = Ud[2 * NN + n] / m;
  }
  int i, j, k;
  node_ijk(M, n, i, j, k);
  F.mn[n] = node_mass_gather<DIM>(M, F.m, i, j, k);
}

// ---------------------------------------------------------------------------
// computeDeltaT (MahycoModule.cc:1739-1864): per-cell l / (c + vmax), block
// minimum, then one ordered-bits atomicMin per block.  The minimum of
// non-NaN values does not depend on the reduction order.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(256) k_delta_t(Mesh M, mhc_case_params P, Fields F) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double dx = 1.7976931348623157e308;
  if (c < M.ncell) {
    int i, j, k;
    cell_ijk(M, c, i, j, k);
    double vmax = 0.;
    if (P.is_euler_scheme == MHC_EULER_FULL) {
      for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
        int a, b, d;
        local_node_offset(l, a, b, d);
        long long n = node_id(M, i + a, j + b, k + d);
        double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
        vmax = amax(sqrt(vx * vx + vy * vy + vz * vz), vmax);
      }
    }
    dx = F.l[c] / (F.c[c] + vmax);
    if (!(dx >= 0.)) { atomicOr(&F.s->status, ST_NAN); dx = 1.7976931348623157e308; }
  }
  for (int o = 16; o > 0; o >>= 1) dx = fmin(dx, __shfl_xor_sync(0xffffffffu, dx, o));
  __shared__ double red[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = dx;
  __syncthreads();
  if (wid == 0) {
    dx = (lane < (blockDim.x + 31) / 32) ? red[lane] : 1.7976931348623157e308;
    for (int o = 16; o > 0; o >>= 1) dx = fmin(dx, __shfl_xor_sync(0xffffffffu, dx, o));
    if (lane == 0) atomicMin(&F.s->dt_min_bits, (unsigned long long)__double_as_longlong(dx));
  }
}

// standalone IEquationOfState::applyEOS(env) on the current state of the
// environment cells, followed by computePressionMoyenne for mixed cells
template <int NE>
__global__ void __launch_bounds__(256) k_eos_apply(Mesh M, mhc_case_params P, Fields F, int env) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  const uint8_t mask = F.mask[c];
  if (!((mask >> env) & 1)) return;
  const bool pure = __popc(mask) == 1;
  if (pure) {
    double p, cs;
    eos_apply(P.env[env], F.rho[c], F.e[c], p, cs);
    F.p[c] = p; F.c[c] = cs;
    return;
  }
  double p, cs;
  eos_apply(P.env[env], F.erho[env * N + c], F.ee[env * N + c], p, cs);
  F.ep[env * N + c] = p; F.ec[env * N + c] = cs;
  double option = P.calcul_vitson_max ? 1. : 0.;
  double pg = 0., cg = 0.;
  for (int q = 0; q < NE; ++q) {
    if (!((mask >> q) & 1)) continue;
    double f = F.ef[q * N + c];
    pg += f * F.ep[q * N + c];
    cg = option * smax(F.ec[q * N + c], cg);
    cg += (1. - option) * f * F.ec[q * N + c];
  }
  F.p[c] = pg; F.c[c] = cg;
}

// end of iteration: new deltat, stop test, advance to the next iteration
__global__ void k_delta_t_finalize(mhc_case_params P, Fields F) {
  Scalars* s = F.s;
  double old = s->dt;
  double new_dt;
  if (P.deltat_constant) {
    new_dt = P.deltat_init;
  } else {
    double minimum_aux = __longlong_as_double((long long)s->dt_min_bits);
    new_dt = P.cfl * minimum_aux;
    new_dt = amin(new_dt, 1.05 * old);
    new_dt = amin(new_dt, P.deltat_max);
    if (new_dt < P.deltat_min) s->status |= ST_DT_UNDERFLOW;
  }
  double stop = P.final_time;
  bool not_yet = s->t < stop, finish = s->t > stop, too_much = (s->t + new_dt) > stop;
  if ((not_yet && too_much) || finish) s->status |= ST_STOP;
  s->t_done = s->t;
  s->iteration_done = s->iteration;
  s->dt_next = new_dt;
  s->old_dt = old;
  s->dt = new_dt;
  s->t = s->t + new_dt;
  s->iteration += 1;
  s->dt_min_bits = 0x7fefffffffffffffull;
}

}  // namespace mhc
