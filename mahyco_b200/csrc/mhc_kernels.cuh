// mhc_kernels.cuh -- sm_100a kernels of one MaHyCo hydro cycle.
//
// Data layout (structure of arrays, FP64, device resident):
//   cell globals    rho e p c q m V l Veul          [ncell]
//   env slots       ef emf em erho ee ep ec eq      [NE][ncell]  (mixed cells only)
//   env mask        mask                            [ncell] (bit e = cell holds env e)
//   nodes           vx vy vz mn                     [nnode]
//                   v0 [3][nnode] (sans-lagrange: the prescribed velocities)
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
  long long iteration_limit;  // last iteration this case may run
  int status;        // ST_* flags
  int pad;
  unsigned int eref_first[4];  // Mie-Gruneisen, energie-ref 0: the first cell (reference order) of
                               // each environment with a nonzero initial energy
};

struct Fields {
  double *rho, *e, *p, *c, *q, *m, *V, *l, *Veul;
  double *ef, *emf, *em, *erho, *ee, *ep, *ec, *eq;
  uint8_t* mask;
  double *vx, *vy, *vz, *mn;
  double* X[2][3];         // Lagrangian positions, alternating by iteration
  double *Xp[3], *Xn[3];   // X of the previous / current iteration (resolved per launch)
  double* U[2];
  double* mflux;
  double* Ud[2];
  double* S;               // elasto: stress deviator [6][ncell] (xx yy zz xy yz zx)
  double* cqs;             // corner normals of the last Lagrangian mesh [NBN][3][ncell]
  double *ebc, *pbc;       // cell-variable boundary conditions only: the cells' current internal
                           // energy and pressure once the conditions applied (the values at n stay
                           // in e, p)
  double* phi_pb;          // pente-borne only: projected values (phi) of the next remap's first sweep
                           // [3 nb_env + 1][ncell]; entries of absent environments keep the
                           // values of the last sweep before
  double* v0;              // sans-lagrange: the prescribed node velocities at n [3][nnode];
                           // CSTS: the velocities at n (after the last remap)
  double* fv[3];           // the node terms of the remap's face velocities: vx, vy, vz themselves,
                           // or (CSTS) the means of the velocities at n and n+1
  double* pq;              // CSTS: pressure + pseudo-viscosity of the forces at n+1 [ncell]
  double* spd;             // Full Euler remap: |v| of every node after the remap, for computeDeltaT [nnode]
  double* x0;              // initial node coordinates read from a mesh file [3][nnode] (else the
                           // cartesian grid)
  double* init;            // EXTERNAL initial state given per cell: Materiau, Density, Pressure
                           // [3][ncell] (else environment 0 and its initial state everywhere)
  double *T, *Tn;          // Lagrangian runs: the temperature the EOS services advance and its
                           // previous value [nb_env][ncell] (a pure cell's in its environment's row)
  double* pl;              // elasto: plastic strain, its rate, the deviator's norm [3][ncell]
  double* hf;              // NewHypoModel: deformation gradient F [9][ncell] (row by row), then
                           // the density at the EOS initialisation rho_0 [ncell]
  Scalars* s;
};

// the s-th cell around a node (bits of s: x, y, z offsets - 1) in the order
// of the reference's cell numbering, which its node sums follow: x-fastest,
// or y-fastest for the 2D mesh files numbered column by column
// (mesh_cell_order 1)
__device__ __forceinline__ void around_node(int s, bool colmajor, int& di, int& dj, int& dk) {
  const int b0 = s & 1, b1 = (s >> 1) & 1;
  di = (colmajor ? b1 : b0) - 1;
  dj = (colmajor ? b0 : b1) - 1;
  dk = ((s >> 2) & 1) - 1;
}

// initial position of node (i, j, k): the mesh file's, or the cartesian grid's
__device__ __forceinline__ R3 node_initial(const Mesh& M, const Fields& F, int i, int j, int k) {
  if (F.x0) {
    const long long n = node_id(M, i, j, k), NN = M.nnode;
    return {F.x0[n], F.x0[NN + n], F.x0[2 * NN + n]};
  }
  return node_x0(M, i, j, k);
}

// the previous cycle's Lagrangian positions are X[(iteration-1)&1], this
// cycle's are X[iteration&1]
// (selects rather than a runtime index, so the struct stays in registers)
__device__ __forceinline__ void resolve_positions(Fields& F) {
  const bool odd = ((F.s->iteration - 1) & 1) != 0;
  F.Xp[0] = odd ? F.X[1][0] : F.X[0][0];
  F.Xp[1] = odd ? F.X[1][1] : F.X[0][1];
  F.Xp[2] = odd ? F.X[1][2] : F.X[0][2];
  F.Xn[0] = odd ? F.X[0][0] : F.X[1][0];
  F.Xn[1] = odd ? F.X[0][1] : F.X[1][1];
  F.Xn[2] = odd ? F.X[0][2] : F.X[1][2];
}

// a case takes part in a launch only while it is below its iteration limit
// and has no error flag (a stop or an error retires it on the device)
__device__ __forceinline__ bool case_active(const Fields& F) {
  const Scalars* s = F.s;
  return s->status == 0 && s->iteration <= s->iteration_limit;
}

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

// applyOneCellEOS (PerfectGas 71-88, StiffenedGas 67-83, MieGruneisen
// 101-146): pressure and dp/de of one environment cell
__device__ __forceinline__ void eos_one_cell(const mhc_env_params& o, double rho, double e, double& p, double& dpde) {
  if (o.eos == MHC_EOS_PERFECT_GAS) {
    double g = o.adiabatic_cst;
    p = (g - 1.) * rho * e;
    dpde = (g - 1.) * rho;
  } else if (o.eos == MHC_EOS_STIFFENED_GAS) {
    double g = o.adiabatic_cst, pinf = o.limit_tension;
    p = ((g - 1.) * rho * e) - (g * pinf);
    dpde = (g - 1.) * rho;
  } else {
    double J = o.rho0 / rho;
    double mu = 1. / J - 1.;
    p = mg_pressure(o, rho, e);
    dpde = (o.gamma0 + o.a * mu);
  }
}

// residual of the energy equation and its derivative (fvnr, fvnrderiv:
// MahycoModule.h:378-386)
__device__ __forceinline__ double fvnr(double e, double p, double en, double qnn1, double pn, double rn1, double rn) {
  return e - en + 0.5 * (p + pn + 2. * qnn1) * (1. / rn1 - 1. / rn);
}
__device__ __forceinline__ double fvnrderiv(double dpde, double rn1, double rn) {
  return 1. + 0.5 * dpde * (1. / rn1 - 1. / rn);
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
  } else if (o.eos == MHC_EOS_FICTIF) {
    // FictifEOSService::initEOS (lines 12-34)
    double g = o.adiabatic_cst;
    e = p / ((g - 1.) * rho);
    c = sqrt(g * p / rho);
  } else {
    e = p / o.gamma0;
    c = o.c0;
  }
}

// FictifEOSService::applyEOS (lines 44-78) for one environment cell: the
// pressure p_old kept until tdebut, then p0 + dpdt t, 0 after tfin; the
// sound speed 1 (no influence on the time step); the caller resets the
// internal energy to 0
__device__ __forceinline__ void fictif_apply(const mhc_env_params& o, double t, double p_old, double& p, double& c) {
  p = p_old;
  if (t > o.fictif_tdebut) p = o.fictif_p0 + o.fictif_dpdt * t;
  if (t > o.fictif_tfin) p = 0.;
  c = 1.;
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

// corner normals kept for the next node pass (CQS at n of the next cycle:
// the reference does not recompute them after the remap).  Layout
// [corner][component][cell]; in 2D the z components are always +0 (the 2D
// corner normals have none) and only x, y are kept.
template <int DIM>
__device__ __forceinline__ void store_cqs(const Fields& F, long long N, long long c, const R3* cqs) {
  constexpr int NC = DIM == 3 ? 3 : 2;
#pragma unroll
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    F.cqs[(NC * l) * N + c] = cqs[l].x;
    F.cqs[(NC * l + 1) * N + c] = cqs[l].y;
    if (DIM == 3) F.cqs[(NC * l + 2) * N + c] = cqs[l].z;
  }
}

// read-only path: only for kernels that do not also write the corner normals
template <int DIM>
__device__ __forceinline__ R3 load_cqs(const Fields& F, long long N, long long c, int l) {
  constexpr int NC = DIM == 3 ? 3 : 2;
  return {__ldg(F.cqs + (NC * l) * N + c), __ldg(F.cqs + (NC * l + 1) * N + c),
          DIM == 3 ? __ldg(F.cqs + (NC * l + 2) * N + c) : 0.0};
}
// coherent load, ordered before the same thread's store_cqs
template <int DIM>
__device__ __forceinline__ R3 load_cqs_rw(const Fields& F, long long N, long long c, int l) {
  constexpr int NC = DIM == 3 ? 3 : 2;
  return {F.cqs[(NC * l) * N + c], F.cqs[(NC * l + 1) * N + c], DIM == 3 ? F.cqs[(NC * l + 2) * N + c] : 0.0};
}

// computeCQs (MahycoModule.cc:1869-1932) and the volume of
// computeGeometricValues, face by face: each corner keeps its two partial
// sums (weight 5 and weight 1) and receives the half-face normals of each
// face in the order of the reference sums, so the results are bit-identical
// to computing all 24 half-face normals first; only the corners whose faces
// are not all done stay live.  Stores the corner normals (store_cqs layout)
// and returns the volume.
__device__ __forceinline__ double cell_volume_store3(const R3* nc, const Fields& F, long long N, long long c) {
  const double t = 1. / 12.;
  R3 a0, a1, a2, a3, a4, a5, a6, a7, b0, b1, b2, b3, b4, b5, b6, b7;
  double d[8];
  {  // face 1
    const R3 fc0 = 0.25 * (nc[0] + nc[3] + nc[2] + nc[1]);
    const R3 n1a04 = 0.5 * vecmul(nc[0] - fc0, nc[3] - fc0);
    const R3 n1a03 = 0.5 * vecmul(nc[3] - fc0, nc[2] - fc0);
    const R3 n1a02 = 0.5 * vecmul(nc[2] - fc0, nc[1] - fc0);
    const R3 n1a01 = 0.5 * vecmul(nc[1] - fc0, nc[0] - fc0);
    a0 = n1a01 + n1a04;
    b0 = n1a02 + n1a03;
    a1 = n1a01 + n1a02;
    b1 = n1a04 + n1a03;
    a2 = n1a02 + n1a03;
    b2 = n1a01 + n1a04;
    a3 = n1a03 + n1a04;
    b3 = n1a01 + n1a02;
  }
  {  // face 2
    const R3 fc1 = 0.25 * (nc[0] + nc[4] + nc[7] + nc[3]);
    const R3 n2a05 = 0.5 * vecmul(nc[0] - fc1, nc[4] - fc1);
    const R3 n2a12 = 0.5 * vecmul(nc[4] - fc1, nc[7] - fc1);
    const R3 n2a08 = 0.5 * vecmul(nc[7] - fc1, nc[3] - fc1);
    const R3 n2a04 = 0.5 * vecmul(nc[3] - fc1, nc[0] - fc1);
    a0 = a0 + n2a04;
    a0 = a0 + n2a05;
    b0 = b0 + n2a08;
    b0 = b0 + n2a12;
    a3 = a3 + n2a08;
    a3 = a3 + n2a04;
    b3 = b3 + n2a05;
    b3 = b3 + n2a12;
    a4 = n2a05 + n2a12;
    b4 = n2a08 + n2a04;
    a7 = n2a08 + n2a12;
    b7 = n2a04 + n2a05;
  }
  {  // face 3
    const R3 fc2 = 0.25 * (nc[0] + nc[1] + nc[5] + nc[4]);
    const R3 n3a01 = 0.5 * vecmul(nc[0] - fc2, nc[1] - fc2);
    const R3 n3a06 = 0.5 * vecmul(nc[1] - fc2, nc[5] - fc2);
    const R3 n3a09 = 0.5 * vecmul(nc[5] - fc2, nc[4] - fc2);
    const R3 n3a05 = 0.5 * vecmul(nc[4] - fc2, nc[0] - fc2);
    a0 = a0 + n3a05;
    a0 = a0 + n3a01;
    b0 = b0 + n3a06;
    b0 = b0 + n3a09;
    a1 = a1 + n3a01;
    a1 = a1 + n3a06;
    b1 = b1 + n3a09;
    b1 = b1 + n3a05;
    a4 = a4 + n3a05;
    a4 = a4 + n3a09;
    b4 = b4 + n3a01;
    b4 = b4 + n3a06;
    a5 = n3a06 + n3a09;
    b5 = n3a01 + n3a05;
  }
  {  // corner 0 complete
    const R3 o = (5. * a0 + b0) * t;
    F.cqs[0 * N + c] = o.x; F.cqs[1 * N + c] = o.y; F.cqs[2 * N + c] = o.z;
    d[0] = dot(nc[0], o);
  }
  {  // face 4
    const R3 fc3 = 0.25 * (nc[4] + nc[5] + nc[6] + nc[7]);
    const R3 n4a09 = 0.5 * vecmul(nc[4] - fc3, nc[5] - fc3);
    const R3 n4a10 = 0.5 * vecmul(nc[5] - fc3, nc[6] - fc3);
    const R3 n4a11 = 0.5 * vecmul(nc[6] - fc3, nc[7] - fc3);
    const R3 n4a12 = 0.5 * vecmul(nc[7] - fc3, nc[4] - fc3);
    a4 = a4 + n4a09;
    a4 = a4 + n4a12;
    b4 = b4 + n4a10;
    b4 = b4 + n4a11;
    a5 = a5 + n4a09;
    a5 = a5 + n4a10;
    b5 = b5 + n4a12;
    b5 = b5 + n4a11;
    a6 = n4a11 + n4a10;
    b6 = n4a12 + n4a09;
    a7 = a7 + n4a12;
    a7 = a7 + n4a11;
    b7 = b7 + n4a09;
    b7 = b7 + n4a10;
  }
  {  // corner 4 complete
    const R3 o = (5. * a4 + b4) * t;
    F.cqs[12 * N + c] = o.x; F.cqs[13 * N + c] = o.y; F.cqs[14 * N + c] = o.z;
    d[4] = dot(nc[4], o);
  }
  {  // face 5
    const R3 fc4 = 0.25 * (nc[1] + nc[2] + nc[6] + nc[5]);
    const R3 n5a02 = 0.5 * vecmul(nc[1] - fc4, nc[2] - fc4);
    const R3 n5a07 = 0.5 * vecmul(nc[2] - fc4, nc[6] - fc4);
    const R3 n5a10 = 0.5 * vecmul(nc[6] - fc4, nc[5] - fc4);
    const R3 n5a06 = 0.5 * vecmul(nc[5] - fc4, nc[1] - fc4);
    a1 = a1 + n5a06;
    a1 = a1 + n5a02;
    b1 = b1 + n5a10;
    b1 = b1 + n5a07;
    a2 = a2 + n5a07;
    a2 = a2 + n5a02;
    b2 = b2 + n5a06;
    b2 = b2 + n5a10;
    a5 = a5 + n5a10;
    a5 = a5 + n5a06;
    b5 = b5 + n5a07;
    b5 = b5 + n5a02;
    a6 = a6 + n5a10;
    a6 = a6 + n5a07;
    b6 = b6 + n5a06;
    b6 = b6 + n5a02;
  }
  {  // corner 1 complete
    const R3 o = (5. * a1 + b1) * t;
    F.cqs[3 * N + c] = o.x; F.cqs[4 * N + c] = o.y; F.cqs[5 * N + c] = o.z;
    d[1] = dot(nc[1], o);
  }
  {  // corner 5 complete
    const R3 o = (5. * a5 + b5) * t;
    F.cqs[15 * N + c] = o.x; F.cqs[16 * N + c] = o.y; F.cqs[17 * N + c] = o.z;
    d[5] = dot(nc[5], o);
  }
  {  // face 6
    const R3 fc5 = 0.25 * (nc[2] + nc[3] + nc[7] + nc[6]);
    const R3 n6a03 = 0.5 * vecmul(nc[2] - fc5, nc[3] - fc5);
    const R3 n6a08 = 0.5 * vecmul(nc[3] - fc5, nc[7] - fc5);
    const R3 n6a11 = 0.5 * vecmul(nc[7] - fc5, nc[6] - fc5);
    const R3 n6a07 = 0.5 * vecmul(nc[6] - fc5, nc[2] - fc5);
    a2 = a2 + n6a07;
    a2 = a2 + n6a03;
    b2 = b2 + n6a11;
    b2 = b2 + n6a08;
    a3 = a3 + n6a08;
    a3 = a3 + n6a03;
    b3 = b3 + n6a07;
    b3 = b3 + n6a11;
    a6 = a6 + n6a07;
    a6 = a6 + n6a11;
    b6 = b6 + n6a03;
    b6 = b6 + n6a08;
    a7 = a7 + n6a11;
    a7 = a7 + n6a08;
    b7 = b7 + n6a07;
    b7 = b7 + n6a03;
  }
  {  // corner 2 complete
    const R3 o = (5. * a2 + b2) * t;
    F.cqs[6 * N + c] = o.x; F.cqs[7 * N + c] = o.y; F.cqs[8 * N + c] = o.z;
    d[2] = dot(nc[2], o);
  }
  {  // corner 3 complete
    const R3 o = (5. * a3 + b3) * t;
    F.cqs[9 * N + c] = o.x; F.cqs[10 * N + c] = o.y; F.cqs[11 * N + c] = o.z;
    d[3] = dot(nc[3], o);
  }
  {  // corner 6 complete
    const R3 o = (5. * a6 + b6) * t;
    F.cqs[18 * N + c] = o.x; F.cqs[19 * N + c] = o.y; F.cqs[20 * N + c] = o.z;
    d[6] = dot(nc[6], o);
  }
  {  // corner 7 complete
    const R3 o = (5. * a7 + b7) * t;
    F.cqs[21 * N + c] = o.x; F.cqs[22 * N + c] = o.y; F.cqs[23 * N + c] = o.z;
    d[7] = dot(nc[7], o);
  }
  double volume = 0.;
#pragma unroll
  for (int l = 0; l < 8; ++l) volume += d[l];
  return volume / 3;
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

// POINTTRIPLE's regions (POINTTRIPLEService.cc:26-36, 49-58): 0 for a cell
// centre at x <= 0.01, else 1 at y <= 0.015, else 2
__device__ __forceinline__ int triple_point_region(const R3& cc) {
  if (cc.x <= 0.01) return 0;
  return cc.y <= 0.015 ? 1 : 2;
}

// applyBoundaryCondition's velocity kinds (MahycoModule.cc:756-807) at one
// node, condition by condition in the dataset's order; X is the node's
// position at the start of the cycle (OnFileVelocity: -x / |X|, -y / |X|)
__device__ __forceinline__ void velocity_bcs(const Mesh& M, const mhc_case_params& P, int i, int j, int k, double t,
                                             double dt, const R3& X, double& vx, double& vy, double& vz) {
  const double eps = 1.e-8;
  for (int b = 0; b < P.nb_bc; ++b) {
    const mhc_bc& bc = P.bc[b];
    if ((t - dt * (1 - eps)) < bc.tdebut) continue;
    if ((t - dt * (1 - eps)) > bc.tfin) continue;
    if (!node_on_surface(M, i, j, k, bc.surface)) continue;
    if (bc.kind == MHC_BC_VX) vx = bc.value;
    else if (bc.kind == MHC_BC_VY) vy = bc.value;
    else if (bc.kind == MHC_BC_VZ) vz = bc.value;
    else if (bc.kind == MHC_BC_ON_FILE_VELOCITY) {
      const double r = sqrt(X.x * X.x + X.y * X.y + X.z * X.z);
      vx = -X.x / r;
      vy = -X.y / r;
    }
  }
}

// ---------------------------------------------------------------------------
// init: MahycoModule::hydroStartInit + computeCellMass (MahycoModule.cc:21-237)
// ---------------------------------------------------------------------------
constexpr int CT = 256;  // threads of the one-dimensional cell / node kernels
// projected variables an elasto-plastic case adds with the remap: the
// deviator's xx, yy, xy, yz, zx (times the volume), the plastic strain rate
// and strain (times the mass), after the pseudo-viscosity
constexpr int MHC_ELASTO_XV = 7;

// BUBBLES (CHOCBULLEService::initMat / initVar, the bubble lattice): the
// material of a cell from its centre cc and node coordinates -- 0 the
// medium, 1 a bubble, 0.5 a mixed cell whose bubble volume fraction is
// returned in fbub.  Bubbles are visited x, then y, then z, later ones
// overriding earlier ones; distances are taken in the (x, y) plane.
template <int DIM>
__device__ __forceinline__ double bubble_material(const mhc_case_params& P, const R3& cc, const R3* coord,
                                                  double& fbub) {
  double mat = 0.;
  fbub = 0.;
  const int nz = DIM == 3 ? P.bubbles_n[2] : 1;
  for (int bx = 0; bx < P.bubbles_n[0]; ++bx)
    for (int by = 0; by < P.bubbles_n[1]; ++by)
      for (int bz = 0; bz < nz; ++bz) {
        const double xb = P.bubbles_first[0] + bx * P.bubbles_delta[0];
        const double yb = P.bubbles_first[1] + by * P.bubbles_delta[1];
        const double rb = P.bubbles_radius;
        const double x = cc.x - xb, y = cc.y - yb;
        if (!(sqrt(x * x + y * y) <= rb)) continue;
        mat = 1.;
        fbub = 0.;
        double rmin = 1.e300, rmax = 0.;
        for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
          const double xn = coord[l].x - xb, yn = coord[l].y - yb;
          const double rn = sqrt(xn * xn + yn * yn);
          rmin = smin(rn, rmin);
          rmax = smax(rn, rmax);
        }
        if (rmin < rb && rmax > rb) {
          mat = 0.5;
          fbub = (rb - rmin) / (rmax - rmin);
        }
      }
  return mat;
}

// RIDER (RIDERService.cc): the disc centre of the test (lines 27-30 and
// 76-79) and the range of the cell's node distances to it in the (x, y)
// plane (lines 36-45)
__device__ __forceinline__ bool rider_mono(const mhc_case_params& P) { return P.cas_test <= MHC_TEST_MONO_RIDER_DEFORMATION_REVERSE; }
__device__ __forceinline__ R3 rider_centre(const mhc_case_params& P) {
  const int first_rotation = rider_mono(P) ? MHC_TEST_MONO_RIDER_ROTATION : MHC_TEST_RIDER_ROTATION;
  return P.cas_test < first_rotation ? R3{0.20, 0.20, 0.} : R3{0.50, 0.75, 0.};
}
template <int DIM>
__device__ __forceinline__ void rider_range(const R3& xb, const R3* coord, double& rmin, double& rmax) {
  rmin = 10.;
  rmax = 0.;
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    const double rn = sqrt((coord[l].x - xb.x) * (coord[l].x - xb.x) + (coord[l].y - xb.y) * (coord[l].y - xb.y));
    rmin = smin(rmin, rn);
    rmax = smax(rmax, rn);
  }
}

template <int DIM, int NE>
__device__ __forceinline__ void body_init_cells(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  long long c = bx * (long long)CT + threadIdx.x;
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
    coord[l] = node_initial(M, F, i + a, j + b, k + d);
    s = s + coord[l];
  }
  R3 cc = (DIM == 2 ? .25 : .125) * s;
  // materials (SODService::initMat, SEDOVService::initMat, MahycoAnnexe.cc:102-139)
  double mat = 0.;
  if (P.cas_model == MHC_CASE_SOD) {
    if (P.cas_test == MHC_TEST_BISOD_X || P.cas_test == MHC_TEST_BISOD_Y || P.cas_test == MHC_TEST_BISOD_Z)
      mat = (comp(cc, P.cas_test - MHC_TEST_BISOD_X) < 0.5) ? 0. : 1.;
    else if (P.cas_test == MHC_TEST_BISOD_SPH)
      mat = (sqrt(cc.x * cc.x + cc.y * cc.y + cc.z * cc.z) < 0.5) ? 0. : 1.;
  } else if (P.cas_model == MHC_CASE_TWO_STATE) {
    if (NE > 1) mat = (comp(cc, P.interface_dir) < P.interface_pos) ? 0. : 1.;
  } else if (P.cas_model == MHC_CASE_ONECELL) {
    mat = 0.;  // ONECELLService::initMat
  } else if (P.cas_model == MHC_CASE_TRIPLE_POINT) {
    // POINTTRIPLEService::initMat (lines 42-60); initMatMono for MonoTriplePoint
    if (P.cas_test != MHC_TEST_MONO_TRIPLE_POINT && NE > 1) mat = (double)triple_point_region(cc);
  } else if (P.cas_model == MHC_CASE_EXTERNAL) {
    mat = F.init ? F.init[c] : 0.;  // the dataset's <initialisation> Materiau
  } else if (P.cas_model == MHC_CASE_SEDOV && P.cas_test != MHC_TEST_SEDOV) {
    bool center = false;
    for (int l = 0; l < NBN; ++l) {
      R3 x = coord[l];
      if (sqrt(x.x * x.x + x.y * x.y + x.z * x.z) < 1.e-10) center = true;
    }
    mat = center ? 1. : 0.;
  }
  double fbub = 0.;  // BUBBLES: the bubble's volume fraction of a mixed cell
  if (P.cas_model == MHC_CASE_BUBBLES && NE > 1) mat = bubble_material<DIM>(P, cc, coord, fbub);
  double rmin = 0., rmax = 0.;  // RIDER: node distances to the disc centre
  if (P.cas_model == MHC_CASE_RIDER) {
    rider_range<DIM>(rider_centre(P), coord, rmin, rmax);
    // RIDERService::initMat (lines 18-57); one environment for MonoRider*
    const double rb = P.rider_radius;
    if (!rider_mono(P) && NE > 1) {
      if (rmax < rb) mat = 1;
      else if ((rmax >= rb) && (rmin < rb)) mat = (rb - rmin) / (rmax - rmin);
    }
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
  store_cqs<DIM>(F, N, c, cqs);
  double l = char_length(P, DIM, V, coord);
  // state: globals g*, env slots *e[]
  double rho = 0., p = 0., e = 0., cs = 0.;
  double rhoe[NE], pe[NE], ee[NE], ce[NE];
  for (int q = 0; q < NE; ++q) { rhoe[q] = pe[q] = ee[q] = ce[q] = 0.; }
  double fe[NE], mfe[NE];
  for (int q = 0; q < NE; ++q) { fe[q] = 1.0; mfe[q] = 1.0; }
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
  } else if (P.cas_model == MHC_CASE_TRIPLE_POINT) {
    // POINTTRIPLEService::initVar / initVarMono (lines 14-41, 62-141): the
    // region's environment state (every cell is pure)
    const int st = triple_point_region(cc);
    rho = P.env[st].densite_initiale;
    p = P.env[st].pression_initiale;
  } else if (P.cas_model == MHC_CASE_BUBBLES) {
    // pure cells: their environment's initial state; mixed cells: both
    // environments' initial states, the cell values are their mixture
    const int st = mat == 1. ? 1 : 0;
    rho = P.env[st].densite_initiale;
    p = P.env[st].pression_initiale;
    if (!pure) {
      rho = p = 0.;
      for (int q = 0; q < 2; ++q) { rhoe[q] = P.env[q].densite_initiale; pe[q] = P.env[q].pression_initiale; }
    }
  } else if (P.cas_model == MHC_CASE_RIDER) {
    // RIDERService::initVar / initVarMono (lines 62-173, 178-289): the disc
    // state inside the radius, the surrounding state outside; a boundary
    // cell takes the disc density times its covered fraction (Rider*: the
    // first environment holds the disc's density and fraction)
    const bool lin = P.rider_linear_density != 0;
    const R3 xb = rider_centre(P);
    const double rb = P.rider_radius;
    const double croissance = lin ? 1. / rb : 1.;
    const double d0 = P.env[0].densite_initiale, d1 = P.env[NE > 1 ? 1 : 0].densite_initiale;
    const double p0 = P.env[0].pression_initiale, p1 = P.env[NE > 1 ? 1 : 0].pression_initiale;
    rho = d0;
    p = p0;
    e = P.env[0].energie_initiale;
    const double r = sqrt((cc.x - xb.x) * (cc.x - xb.x) + (cc.y - xb.y) * (cc.y - xb.y));
    const double r_cell = lin ? r : rmax;
    if (r_cell < rb) {
      rho = d1;
      if (lin) rho = d1 * smin(croissance * 2 * (rb - r), 1.);
      p = p1;
    } else if ((rmax >= rb) && (rmin < rb) && !lin) {
      const double frac_b = (rb - rmin) / (rmax - rmin);
      if (NE > 1 && !rider_mono(P) && !pure) {
        constexpr int E1 = NE > 1 ? 1 : 0;
        rhoe[0] = d1; fe[0] = frac_b; mfe[0] = frac_b;
        rhoe[E1] = d0; fe[E1] = 1. - frac_b; mfe[E1] = 1. - frac_b;
      }
      rho = frac_b * d1;
      p = p1;
    }
  } else if (P.cas_model == MHC_CASE_EXTERNAL) {
    // EXTERNALService (no initVar): the dataset's <initialisation> Density
    // and Pressure of the cell
    rho = F.init ? F.init[N + c] : P.env[0].densite_initiale;
    p = F.init ? F.init[2 * N + c] : P.env[0].pression_initiale;
  } else if (P.cas_model == MHC_CASE_ONECELL) {
    // ONECELLService::initVarMono: the first environment's state everywhere
    rho = P.env[0].densite_initiale;
    p = P.env[0].pression_initiale;
    e = P.env[0].energie_initiale;
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
  // EOS init per environment (aliased for pure cells); none at the start
  // of a sans-lagrange run (MahycoModule.cc:143-171)
  for (int q = 0; q < NE && !P.sans_lagrange; ++q) {
    if (!((mask >> q) & 1)) continue;
    if (pure) eos_init(P.env[q], p, rho, e, cs);
    else eos_init(P.env[q], pe[q], rhoe[q], ee[q], ce[q]);
  }
  if (P.cas_model == MHC_CASE_BUBBLES && !pure) {
    // volume fractions of the bubble (environment 1) and the medium, mass
    // fractions f rho / sum of f rho
    fe[0] = 1. - fbub;
    fe[1] = fbub;
    double rm = 0.;
    for (int q = 0; q < 2; ++q) rm += rhoe[q] * fe[q];
    for (int q = 0; q < 2; ++q) mfe[q] = (rhoe[q] * fe[q]) / rm;
  }
  if (!pure && !P.sans_lagrange) {
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
  if (F.phi_pb)  // volume fractions of the first pente-borne remap (MahycoModule.cc hydroStartInit: 1 per environment)
    for (int q = 0; q < NE; ++q) F.phi_pb[q * N + c] = ((mask >> q) & 1) ? fe[q] : 0.;
  if (NE > 1 && !pure) {
    for (int q = 0; q < NE; ++q) {
      F.ef[q * N + c] = fe[q]; F.emf[q * N + c] = mfe[q]; F.em[q * N + c] = me[q];
      F.erho[q * N + c] = rhoe[q]; F.ee[q * N + c] = ee[q]; F.ep[q * N + c] = pe[q];
      F.ec[q * N + c] = ce[q]; F.eq[q * N + c] = 0.;
    }
  } else if (NE > 1) {
    for (int q = 0; q < NE; ++q)
      if ((mask >> q) & 1) F.ef[q * N + c] = 1.0;  // a pure cell's volume fraction (read back only)
  }
}

// ---------------------------------------------------------------------------
// the temperature of initEOS, Lagrangian runs (PerfectGasEOSService.cc:30,
// StiffenedGasEOSService.cc:30: p / (287 rho); MieGruneisenEOSService.cc:
// 17, 29-30: (e - eref) / cv + tref, an energie-ref of 0 taking the first
// nonzero energy of the environment in the reference's cell order).  Two
// passes: the first cell with a nonzero energy of each such environment
// (atomicMin on its reference index), then the temperatures.  env < 0: every
// environment.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ unsigned ref_cell_index(const Mesh& M, const mhc_case_params& P, long long c) {
  if (DIM == 2 && P.mesh_cell_order == 1) {
    int i, j, k;
    cell_ijk(M, c, i, j, k);
    return (unsigned)i * (unsigned)M.ncy + (unsigned)j;
  }
  return (unsigned)c;
}

__device__ __forceinline__ double env_value(const double* g, const double* e, bool pure, int q, long long N,
                                            long long c) {
  return pure ? g[c] : e[q * N + c];
}

template <int DIM, int NE>
__device__ __forceinline__ void body_eref_candidates(const Mesh& M, const mhc_case_params& P, const Fields& F,
                                                     int env, int bx) {
  const long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell || !F.T) return;
  const long long N = M.ncell;
  const uint8_t mask = F.mask[c];
  const bool pure = __popc(mask) == 1;
  for (int q = 0; q < NE; ++q) {
    if ((env >= 0 && q != env) || !((mask >> q) & 1)) continue;
    const mhc_env_params& o = P.env[q];
    if (o.eos != MHC_EOS_MIE_GRUNEISEN || o.energie_ref != 0.) continue;
    if (env_value(F.e, F.ee, pure, q, N, c) != 0.) atomicMin(&F.s->eref_first[q], ref_cell_index<DIM>(M, P, c));
  }
}

template <int DIM, int NE>
__device__ __forceinline__ void body_init_temperature(const Mesh& M, const mhc_case_params& P, const Fields& F,
                                                      int env, int bx) {
  const long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell || !F.T) return;
  const long long N = M.ncell;
  const uint8_t mask = F.mask[c];
  const bool pure = __popc(mask) == 1;
  for (int q = 0; q < NE; ++q) {
    if (env >= 0 && q != env) continue;
    double T = 0.;
    if ((mask >> q) & 1) {
      const mhc_env_params& o = P.env[q];
      const double p = env_value(F.p, F.ep, pure, q, N, c), rho = env_value(F.rho, F.erho, pure, q, N, c);
      const double e = env_value(F.e, F.ee, pure, q, N, c);
      if (o.eos == MHC_EOS_PERFECT_GAS || o.eos == MHC_EOS_STIFFENED_GAS) {
        T = p / (287. * rho);
      } else if (o.eos == MHC_EOS_MIE_GRUNEISEN) {
        double eref = o.energie_ref;
        const unsigned first = F.s->eref_first[q];
        if (eref == 0. && first != 0xffffffffu && ref_cell_index<DIM>(M, P, c) >= first) {
          // the energy of that first cell: the reference index back to the cell
          long long cf = first;
          if (DIM == 2 && P.mesh_cell_order == 1) cf = (long long)(first % M.ncy) * M.ncx + first / M.ncy;
          eref = env_value(F.e, F.ee, __popc(F.mask[cf]) == 1, q, N, cf);
        }
        T = (e - eref) / o.specific_heat + o.temperature_ref;
      }
    }
    F.T[q * N + c] = T;
    F.Tn[q * N + c] = 0.;
  }
}

// computeNodeMass (MahycoModule.cc:247-262): gather of 1/8 (1/4) cell masses in
// ascending cell id; also initial velocity and Lagrangian positions.
template <int DIM>
__device__ __forceinline__ double node_mass_gather(const Mesh& M, const double* cm, int i, int j, int k,
                                                   bool colmajor = false) {
  const double w = DIM == 2 ? .25 : .125;
  double s = 0.;
  for (int q = 0; q < (DIM == 3 ? 8 : 4); ++q) {
    int di, dj, dk;
    around_node(q, DIM == 2 && colmajor, di, dj, dk);
    const int ci = i + di, cj = j + dj, ck = DIM == 3 ? k + dk : 0;
    if (ci < 0 || ci >= M.ncx || cj < 0 || cj >= M.ncy || (DIM == 3 && (ck < 0 || ck >= M.ncz))) continue;
    s += w * cm[cell_id(M, ci, cj, ck)];
  }
  return s;
}

template <int DIM>
__device__ __forceinline__ void body_init_nodes(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  R3 x = node_initial(M, F, i, j, k);
  F.Xp[0][n] = x.x; F.Xp[1][n] = x.y; F.Xp[2][n] = x.z;
  double vx = 0., vy = 0., vz = 0.;
  if (P.cas_model == MHC_CASE_SOD || P.cas_model == MHC_CASE_TWO_STATE || P.cas_model == MHC_CASE_BUBBLES ||
      P.cas_model == MHC_CASE_TRIPLE_POINT) {
    vx = P.env[0].vitesse_initiale[0]; vy = P.env[0].vitesse_initiale[1]; vz = P.env[0].vitesse_initiale[2];
  }
  if (P.cas_model == MHC_CASE_EXTERNAL) {
    // EXTERNALService::initUtilisateur (EXTERNALService.cc:25-40) for every
    // environment that asks for it: its initial velocity, or -x/|x|
    for (int e = 0; e < P.nb_env; ++e) {
      if (!P.env[e].initialisation_utilisateur) continue;
      const double* w = P.env[e].vitesse_initiale;
      if (w[0] == 0. && w[1] == 0. && w[2] == 0.) {
        const double r = sqrt(x.x * x.x + x.y * x.y + x.z * x.z);
        vx = (-x.x) / r; vy = (-x.y) / r; vz = (-x.z) / r;
      } else {
        vx = w[0]; vy = w[1]; vz = w[2];
      }
    }
  }
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  if (F.v0) {
    // RIDER fields are written over these by the host after the launch
    const long long NN = M.nnode;
    F.v0[n] = vx; F.v0[NN + n] = vy; F.v0[2 * NN + n] = vz;
  }
  F.mn[n] = node_mass_gather<DIM>(M, F.m, i, j, k, P.mesh_cell_order == 1);
}

// ---------------------------------------------------------------------------
// Pressure surfaces of applyBoundaryConditionForCellVariables
// (MahycoModule.cc:909-986), Lagrangian runs: for each pressure condition in
// order and each face of its surface holding the node, in face order,
// v -= dt_mid / nb_face_nodes * n * p * S / m_node, with n the unit vector
// from the boundary cell's centre (positions at n) to the face centre of the
// initial grid, S the length of the face edge that starts at the node (2D)
// or the z-projected face area (3D), p the value plus its linear terms in
// the node position and time, zero outside [Tdebut, Tfin).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void face_node_rt(int dim, int d, int q, int& a, int& b, int& c) {
  a = b = c = 0;
  if (dim == 2) {
    if (d == 0) b = q; else a = q;
    return;
  }
  const int s1 = (q == 1 || q == 2), s2 = (q == 2 || q == 3);
  if (d == 0) { b = s1; c = s2; }
  else if (d == 1) { a = s1; c = s2; }
  else { a = s1; b = s2; }
}

// OnFilePressure's value (MahycoModule.cc:987-1008): the first table time
// above t ends the interval, the value is interpolated linearly with the
// weight clamped to [0, 1] (Arcane's math::min / math::max); 0 before the
// first time and from the last time on
__device__ __forceinline__ double onfile_pressure(const mhc_case_params& P, double t) {
  int it = -1;
  for (int i = 0; i < P.pressure_table_n; ++i) {
    if (t < P.pressure_table_t[i]) {
      it = i;
      break;
    }
  }
  if (it <= 0) return 0.;
  double alpha = (t - P.pressure_table_t[it - 1]) / (P.pressure_table_t[it] - P.pressure_table_t[it - 1]);
  alpha = alpha < 1. ? alpha : 1.;
  alpha = alpha < 0. ? 0. : alpha;
  return P.pressure_table_p[it - 1] + alpha * (P.pressure_table_p[it] - P.pressure_table_p[it - 1]);
}

// Compiled into the Lagrangian instances of the node pass only (the only
// runs allowed pressure surfaces): its local arrays and loops stay off the
// register budget of the node pass of the remapped runs.
template <int DIM>
__device__ __forceinline__ R3 pressure_bcs(const Mesh& M, const mhc_case_params& P, const Fields& F, int i, int j,
                                        int k, long long n, double dth, double t, R3 v) {
  double vx = v.x, vy = v.y, vz = v.z;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  const double w = DIM == 2 ? .5 : .25, wc = DIM == 2 ? .25 : .125;
  for (int b = 0; b < P.nb_bc; ++b) {
    const mhc_bc& bc = P.bc[b];
    if (bc.kind != MHC_BC_GEOMETRIC_PRESSURE && bc.kind != MHC_BC_LINEAR_PRESSURE &&
        bc.kind != MHC_BC_SUPER_GAUSSIAN_PRESSURE && bc.kind != MHC_BC_CONTACT_HERZ_PRESSURE &&
        bc.kind != MHC_BC_ON_FILE_PRESSURE)
      continue;
    const bool onfile = bc.kind == MHC_BC_ON_FILE_PRESSURE;
    const int s = bc.surface;
    const int d = (s == MHC_XMIN || s == MHC_XMAX) ? 0 : ((s == MHC_YMIN || s == MHC_YMAX) ? 1 : 2);
    if (d >= DIM) continue;
    const bool maxside = s >= MHC_XMAX;
    const int nid = d == 0 ? i : (d == 1 ? j : k);
    const int nnd = d == 0 ? M.nnx : (d == 1 ? M.nny : M.nnz);
    if (nid != (maxside ? nnd - 1 : 0)) continue;
    // transverse axes a1 < a2 of the surface, node and cell counts along them
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    const int idx[3] = {i, j, k};
    const int nc[3] = {M.ncx, M.ncy, M.ncz};
    for (int o2 = (DIM == 3 ? -1 : 0); o2 <= 0; ++o2) {
      for (int o1 = -1; o1 <= 0; ++o1) {
        const int t1 = idx[a1] + o1, t2 = DIM == 3 ? idx[a2] + o2 : 0;
        if (t1 < 0 || t1 >= nc[a1]) continue;
        if (DIM == 3 && (t2 < 0 || t2 >= nc[a2])) continue;
        int f[3];
        f[d] = nid; f[a1] = t1;
        if (DIM == 3) f[a2] = t2; else f[2] = 0;
        // face nodes in face order, initial face centre, this node's slot
        long long fn[NQ];
        R3 fc = {0., 0., 0.};
        int me = 0;
        for (int q = 0; q < NQ; ++q) {
          int a, bb, c;
          face_node_rt(DIM, d, q, a, bb, c);
          fn[q] = node_id(M, f[0] + a, f[1] + bb, DIM == 3 ? f[2] + c : 0);
          fc = fc + w * node_initial(M, F, f[0] + a, f[1] + bb, DIM == 3 ? f[2] + c : 0);
          if (fn[q] == n) me = q;
        }
        auto X = [&](long long m) { return R3{F.Xp[0][m], F.Xp[1][m], F.Xp[2][m]}; };
        double surface;
        if (DIM == 2 || onfile) {
          const long long n2 = me < NQ - 1 ? fn[me + 1] : fn[0];
          surface = norm(X(n2) - X(n));
        } else {
          const R3 v1 = X(fn[2]) - X(fn[0]), v2 = X(fn[3]) - X(fn[1]);
          surface = 0.5 * produit(v1.x, v2.y, v1.y, v2.x);
        }
        // the boundary cell: first or last along d
        int ci[3] = {f[0], f[1], f[2]};
        if (maxside) ci[d] -= 1;
        R3 sc = {0., 0., 0.};
        for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
          int a, bb, c;
          local_node_offset(l, a, bb, c);
          sc = sc + X(node_id(M, ci[0] + a, ci[1] + bb, DIM == 3 ? ci[2] + c : 0));
        }
        const R3 cc = wc * sc;
        const R3 diff = fc - cc;
        const R3 nrm = diff / norm(diff);
        double value = bc.value;
        if (bc.kind == MHC_BC_LINEAR_PRESSURE) {
          const R3 x = X(n);
          value += bc.dependance[0] * x.x;
          value += bc.dependance[1] * x.y;
          value += bc.dependance[2] * x.z;
          value += bc.dependance[3] * t;
        } else if (bc.kind == MHC_BC_SUPER_GAUSSIAN_PRESSURE) {
          // CUDA's exp and pow, within a few ulps of the reference's libm
          const R3 x = X(n);
          const double ay = x.y * bc.dependance[1];
          value *= exp(-pow(ay, bc.power));
          const double ax = x.x * bc.dependance[0];
          value *= exp(-pow(ax, bc.power));
          if (fabs(x.y) > bc.cutoff[1]) value = 0.;
        } else if (bc.kind == MHC_BC_CONTACT_HERZ_PRESSURE) {
          const double a2 = bc.dependance[0], b2 = bc.dependance[1];
          const double x2 = cc.x * cc.x, y2 = cc.y * cc.y;
          if (x2 / a2 + y2 / b2 < 1.) value *= sqrt(1 - x2 / a2 - y2 / b2);
          else value = 0.;
        }
        if (onfile) {
          value = onfile_pressure(P, t);
        } else {
          if (t < bc.tdebut) value = 0.;
          if (t >= bc.tfin) value = 0.;
        }
        const R3 dv = (dth * w * nrm * value * surface) / F.mn[n];
        vx = vx - dv.x; vy = vy - dv.y; vz = vz - dv.z;
      }
    }
  }
  return R3{vx, vy, vz};
}

// ---------------------------------------------------------------------------
// Lagrange, node pass: updateVelocity + applyBoundaryCondition + updatePosition
// (MahycoModule.cc:438-501, 756-807, 730-741).
//
// One thread per node gathers (p_n + q_n) * CQS_n over its <= 8 cells in
// ascending cell id, then (EL) the elasto-plastic forces -S_n.CQS_n in the
// same order: the reference's cell loops add into the node forces in that
// order, and no atomics are used.  CQS_n are the corner normals the
// previous cell pass stored.  HG: the anti-hourglass correction follows
// (kb_hourglass), so this pass only writes the uncorrected velocity into
// the dual-remap scratch Ud[0] (unused by a Lagrangian run).
// ---------------------------------------------------------------------------
// CSTS (with the remap): the velocities after the remap (at n) are kept
// in v0, then taken back to n-1/2 with the same forces and -old_dt/2
// (updateVelocityBackward, MahycoModule.cc:573-627) before the update
template <int DIM, bool EL, bool HG, bool LAG, bool CSTS = false>
__device__ __forceinline__ void body_lagrange_nodes(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const long long N = M.ncell, NN = M.nnode;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  // the <= 8 cells around the node in ascending id: slot s = (dk, dj, di)
  // bits, the node's local index in the cell is the complement
  constexpr int NS = DIM == 3 ? 8 : 4;
  const bool cm = DIM == 2 && P.mesh_cell_order == 1;
  R3 S = {0., 0., 0.};
  // every load of the node's cells first (a cell outside the mesh reads
  // cell 0 and is skipped), each cell's force (p + q) CQS formed as its
  // loads arrive, then the sums in the reference's order
  R3 fv[NS];
  bool in[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    int di, dj, dk;
    around_node(s, cm, di, dj, dk);
    if (DIM == 2) dk = 0;
    const int ci = i + di, cj = j + dj, ck = k + dk;
    in[s] = !(ci < 0 || cj < 0 || ci >= M.ncx || cj >= M.ncy || (DIM == 3 && (ck < 0 || ck >= M.ncz)));
    const int l = (-dk) * 4 + ((-dj) ? ((-di) ? 2 : 3) : ((-di) ? 1 : 0));
    const long long c = in[s] ? cell_id(M, ci, cj, ck) : 0;
    fv[s] = (__ldg(F.p + c) + __ldg(F.q + c)) * load_cqs<DIM>(F, N, c, l);
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (!in[s]) continue;
    S.x = S.x + fv[s].x; S.y = S.y + fv[s].y; S.z = S.z + fv[s].z;
  }
  if (EL) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      int di, dj, dk;
      around_node(s, cm, di, dj, dk);
      if (DIM == 2) dk = 0;
      const int ci = i + di, cj = j + dj, ck = k + dk;
      if (ci < 0 || cj < 0 || ci >= M.ncx || cj >= M.ncy || (DIM == 3 && (ck < 0 || ck >= M.ncz))) continue;
      const int l = (-dk) * 4 + ((-dj) ? ((-di) ? 2 : 3) : ((-di) ? 1 : 0));
      const long long c = cell_id(M, ci, cj, ck);
      // force_tensor = -S_n; prodTensVec(t, v) = (t.x.v, t.y.v, t.z.v)
      const double sxx = F.S[c], syy = F.S[N + c], szz = F.S[2 * N + c];
      const double sxy = F.S[3 * N + c], syz = F.S[4 * N + c], szx = F.S[5 * N + c];
      const R3 rx = {-sxx, -sxy, -szx}, ry = {-sxy, -syy, -syz}, rz = {-szx, -syz, -szz};
      const R3 cq = load_cqs<DIM>(F, N, c, l);
      S.x = S.x + dot(rx, cq); S.y = S.y + dot(ry, cq); S.z = S.z + dot(rz, cq);
    }
  }
  const double dt = F.s->dt;
  const double dth = 0.5 * (F.s->old_dt + dt);
  const double t = F.s->t;
  double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
  if constexpr (CSTS) {
    F.v0[n] = vx; F.v0[NN + n] = vy; F.v0[2 * NN + n] = vz;
    const double dtb = -0.5 * F.s->old_dt;
    const double fb = dtb / F.mn[n];
    vx = vx + fb * S.x; vy = vy + fb * S.y; vz = vz + fb * S.z;
    vx = vx + dtb * P.gravity[0]; vy = vy + dtb * P.gravity[1]; vz = vz + dtb * P.gravity[2];
  }
  const double f = dth / F.mn[n];
  vx = vx + f * S.x; vy = vy + f * S.y; vz = vz + f * S.z;
  vx = vx + dth * P.gravity[0]; vy = vy + dth * P.gravity[1]; vz = vz + dth * P.gravity[2];
  if (HG) {
    F.Ud[0][n] = vx; F.Ud[0][NN + n] = vy; F.Ud[0][2 * NN + n] = vz;
    return;
  }
  // positions at the start of the cycle: the initial grid after a Full
  // Euler remap (RemapADIService.cc:62-64); otherwise the last ones (a
  // per-axis remap has put its axis back on the grid, kb_euler_axis_reset)
  const R3 x = (!LAG && P.is_euler_scheme == MHC_EULER_FULL) ? node_x0(M, i, j, k)
                                                             : R3{F.Xp[0][n], F.Xp[1][n], F.Xp[2][n]};
  velocity_bcs(M, P, i, j, k, t, dt, x, vx, vy, vz);
  if constexpr (LAG) {
    const R3 v = pressure_bcs<DIM>(M, P, F, i, j, k, n, dth, t, R3{vx, vy, vz});
    vx = v.x; vy = v.y; vz = v.z;
  }
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  F.Xn[0][n] = x.x + dt * vx; F.Xn[1][n] = x.y + dt * vy; F.Xn[2][n] = x.z + dt * vz;
}

// ---------------------------------------------------------------------------
// Anti-hourglass correction of a Lagrangian run (MahycoModule.cc:497-555),
// then applyBoundaryCondition and updatePosition.  Reads the uncorrected
// velocities the node pass left in Ud[0]; each node gathers the corrections
// of its cells in ascending cell id.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void body_hourglass(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const long long NN = M.nnode;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  const double coeff = P.coef_antiderive;
  const double* ux = F.Ud[0];
  const double* uy = ux + NN;
  const double* uz = ux + 2 * NN;
  const double nb = (double)(((i > 0 && i < M.nnx - 1) ? 2 : 1) * ((j > 0 && j < M.nny - 1) ? 2 : 1) *
                             (DIM == 3 ? ((k > 0 && k < M.nnz - 1) ? 2 : 1) : 1));
  R3 h = {0., 0., 0.};
  const bool cm = DIM == 2 && P.mesh_cell_order == 1;
  for (int s = 0; s < (DIM == 3 ? 8 : 4); ++s) {
        int di, dj, dk;
        around_node(s, cm, di, dj, dk);
        if (DIM == 2) dk = 0;
        const int ci = i + di, cj = j + dj, ck = k + dk;
        if (ci < 0 || cj < 0 || ci >= M.ncx || cj >= M.ncy) continue;
        if (DIM == 3 && (ck < 0 || ck >= M.ncz)) continue;
        const int oa = -di, ob = -dj, oc = -dk;  // offset of the node in the cell
        const int l = oc * 4 + (ob ? (oa ? 2 : 3) : (oa ? 1 : 0));
        R3 v[8];
#pragma unroll
        for (int q = 0; q < (DIM == 3 ? 8 : 4); ++q) {
          int a, b, c;
          local_node_offset(q, a, b, c);
          const long long m = node_id(M, ci + a, cj + b, ck + c);
          v[q] = {ux[m], uy[m], uz[m]};
        }
        if (DIM == 2) {
          const R3 psi = coeff * (v[0] + v[2] - v[1] - v[3]);
          if (l == 0 || l == 2) h = h + 1. / nb * psi;
          else h = h - 1. / nb * psi;
        } else {
          const R3 p1 = coeff * (v[0] + v[1] - v[2] - v[3] - v[4] - v[5] + v[6] + v[7]);
          const R3 p2 = coeff * (v[0] - v[1] - v[2] + v[3] - v[4] + v[5] + v[6] - v[7]);
          const R3 p3 = coeff * (v[0] - v[1] + v[2] - v[3] + v[4] - v[5] + v[6] - v[7]);
          const R3 p4 = coeff * (-v[0] + v[1] - v[2] + v[3] + v[4] - v[5] + v[6] - v[7]);
          R3 w;
          switch (l) {
            case 0: w = p1 + p2 + p3 - p4; break;
            case 1: w = p1 - p2 - p3 + p4; break;
            case 2: w = -p1 - p2 + p3 - p4; break;
            case 3: w = -p1 + p2 - p3 + p4; break;
            case 4: w = -p1 - p2 + p3 + p4; break;
            case 5: w = -p1 + p2 - p3 - p4; break;
            case 6: w = p1 + p2 + p3 + p4; break;
            default: w = p1 - p2 - p3 - p4; break;
          }
          h = h + 1. / nb * w;
        }
      }
  double vx = ux[n] - h.x, vy = uy[n] - h.y, vz = uz[n] - h.z;
  const double dt = F.s->dt, t = F.s->t;
  velocity_bcs(M, P, i, j, k, t, dt, R3{F.Xp[0][n], F.Xp[1][n], F.Xp[2][n]}, vx, vy, vz);
  {
    const R3 v = pressure_bcs<DIM>(M, P, F, i, j, k, n, 0.5 * (F.s->old_dt + dt), t, R3{vx, vy, vz});
    vx = v.x; vy = v.y; vz = v.z;
  }
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  F.Xn[0][n] = F.Xp[0][n] + dt * vx; F.Xn[1][n] = F.Xp[1][n] + dt * vy; F.Xn[2][n] = F.Xp[2][n] + dt * vz;
}

// ---------------------------------------------------------------------------
// Lagrange, cell pass: computeGeometricValues + updateDensity +
// computeArtificialViscosity + updateEnergyAndPressure
// (MahycoModule.cc:1097-1316, 386-426, 1430-1502, 1623-1698, 1708-1735).
// EULER: the results are packed directly into the remap conserved variables
// (PrepareRemap.cc:94-193).  Otherwise the EOS is applied here
// (Lagrange-only time loop).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// updateElasticityAndPlasticity (MahycoModule.cc:1327-1353) with
// DefaultModelService (src/elasto/DefaultModelService.cc:27-242), or
// NewHypoModelService (src/elasto/NewHypoModelService.cc:32-308), and the
// constant EPP shear modulus / YEPP yield strength, for one environment:
// velocity gradient from the mean corner normals, deformation rate and
// spin, work with S_n, deviator update with rotation, radial return, work
// with S_n+1.  Returns the two work increments in order.  Where the
// reference relies on undefined or framework behaviour: the deviator
// increment takes trace = 0 (an uninitialised `trace` there,
// DefaultModelService.cc:82,96, whose non-regression curves match 0 and not
// tr(D)), doubleContraction sums row by row, each
// row left to right, pow(x, 2.) is x*x, Real3x3 / Real divides each
// component.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void elasto_cell(const mhc_env_params& o, const Mesh& M, const Fields& F, long long c,
                                            int i, int j, int k, const R3* cqn, const R3* cqs, double V, double Vn,
                                            double mass, double rho, double dt, double& w1, double& w2) {
  constexpr int NBN = DIM == 3 ? 8 : 4;
  const long long N = M.ncell;
  R3 vel[8];
  for (int l = 0; l < NBN; ++l) {
    int a, b, d;
    local_node_offset(l, a, b, d);
    const long long nn = node_id(M, i + a, j + b, k + d);
    vel[l] = {F.vx[nn], F.vy[nn], F.vz[nn]};
  }
  double G[3][3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
  for (int l = 0; l < NBN; ++l) {
    const R3 cq = .5 * (cqn[l] + cqs[l]);
    const double va[3] = {vel[l].x, vel[l].y, vel[l].z}, cb[3] = {cq.x, cq.y, cq.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) G[a][b] = G[a][b] + va[a] * cb[b];
  }
  const double volume = .5 * (Vn + V);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) G[a][b] = G[a][b] / volume;
  double D[3][3];
  D[0][0] = G[0][0]; D[1][1] = G[1][1]; D[2][2] = G[2][2];
  D[0][1] = 0.5 * (G[0][1] + G[1][0]);
  D[0][2] = 0.5 * (G[0][2] + G[2][0]);
  D[1][2] = 0.5 * (G[1][2] + G[2][1]);
  D[1][0] = D[0][1]; D[2][0] = D[0][2]; D[2][1] = D[1][2];
  const double wx = 0.5 * (G[1][2] - G[2][1]), wy = 0.5 * (G[2][0] - G[0][2]), wz = 0.5 * (G[0][1] - G[1][0]);
  double Sv[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) Sv[q] = F.S[q * N + c];
  auto work = [&]() {
    const double r0 = Sv[0] * D[0][0] + Sv[3] * D[0][1] + Sv[5] * D[0][2];
    const double r1 = Sv[3] * D[1][0] + Sv[1] * D[1][1] + Sv[4] * D[1][2];
    const double r2 = Sv[5] * D[2][0] + Sv[4] * D[2][1] + Sv[2] * D[2][2];
    const double dc = r0 + r1 + r2;
    return 0.25 * dt * (V + Vn) * dc / mass;
  };
  w1 = work();
  const double sxx = Sv[0], syy = Sv[1], szz = Sv[2], sxy = Sv[3], syz = Sv[4], szx = Sv[5];
  const double mu = o.shear_modulus, Y = o.yield_strength;
  const double trace = 0.;
  double Pt[3][3];
  if (o.elasto_model == 2) {
    // NewHypoModel: F <- (I + G dt) F, B = F F^T (NewHypoModelService.cc:
    // 48-49, 76-79), J = rho_0 / rho and the deviator's rate
    // mu / J^(5/3) (DB + BD - 2/3 (B:D) I - 5/3 tr(D) dev B) dt (102-128);
    // the thermal term mu' (T - T_n) dev B vanishes for the constant EPP
    // shear modulus (EPPService.cc:26-28)
    double Fo[9], Fn[3][3], B[3][3];
#pragma unroll
    for (int q = 0; q < 9; ++q) Fo[q] = F.hf[q * N + c];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double g0 = (a == 0 ? 1. : 0.) + G[a][0] * dt, g1 = (a == 1 ? 1. : 0.) + G[a][1] * dt,
                     g2 = (a == 2 ? 1. : 0.) + G[a][2] * dt;
        Fn[a][b] = g0 * Fo[0 * 3 + b] + g1 * Fo[1 * 3 + b] + g2 * Fo[2 * 3 + b];
      }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        F.hf[(a * 3 + b) * N + c] = Fn[a][b];
        B[a][b] = Fn[a][0] * Fn[b][0] + Fn[a][1] * Fn[b][1] + Fn[a][2] * Fn[b][2];
      }
    const double J = F.hf[9 * N + c] / rho;
    const double mu_over_J = mu / pow_five_thirds(J);
    const double traceD = D[0][0] + D[1][1] + D[2][2];
    const double traceB = B[0][0] + B[1][1] + B[2][2];
    double dcb = B[0][0] * D[0][0] + B[0][1] * D[0][1] + B[0][2] * D[0][2];
    dcb += B[1][0] * D[1][0] + B[1][1] * D[1][1] + B[1][2] * D[1][2];
    dcb += B[2][0] * D[2][0] + B[2][1] * D[2][1] + B[2][2] * D[2][2];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double id = a == b ? 1. : 0.;
        const double DB = D[a][0] * B[0][b] + D[a][1] * B[1][b] + D[a][2] * B[2][b];
        const double BD = B[a][0] * D[0][b] + B[a][1] * D[1][b] + B[a][2] * D[2][b];
        const double devB = B[a][b] - (1. / 3. * traceB) * id;
        Pt[a][b] = (mu_over_J * (((DB + BD) - (2. / 3. * dcb) * id) - (5. / 3. * traceD) * devB)) * dt;
      }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) Pt[a][b] = 2 * mu * (D[a][b] - (1. / 3.) * trace * (a == b ? 1.0 : 0.0)) * dt;
  }
  if (DIM == 2) {
    if (o.rotation_order == 1) {
      Pt[0][0] += 2 * dt * sxy * wz;
      Pt[1][1] -= 2 * dt * sxy * wz;
      Pt[0][1] -= dt * (sxx - syy) * wz;
      Pt[1][0] = Pt[0][1];
    } else {
      const double syx = sxy;
      const double a = -0.5 * dt * wz;
      const double qxx = (1. - a * a) / (1. + a * a), qyy = qxx;
      const double qxy = -2. * a / (1. + a * a), qyx = -qxy;
      const double blxx = sxx * qxx + sxy * qxy, blxy = sxx * qyx + sxy * qyy;
      const double blyx = syx * qxx + syy * qxy, blyy = syx * qyx + syy * qyy;
      Pt[0][0] = qxx * blxx + qxy * blyx;
      Pt[1][1] = qyx * blxy + qyy * blyy;
      Pt[0][1] = qxx * blxy + qxy * blyy;
      Pt[1][0] = Pt[0][1];
    }
  } else {
    Pt[0][0] -= 2 * dt * (szx * wy - sxy * wz);
    Pt[1][1] -= 2 * dt * (sxy * wz - syz * wx);
    Pt[2][2] -= 2 * dt * (syz * wx - szx * wy);
    Pt[0][1] -= dt * (sxx - syy) * wz - dt * syz * wy - dt * szx * wx;
    Pt[1][2] -= dt * (syy - szz) * wx - dt * szx * wz - dt * sxy * wy;
    Pt[2][0] -= dt * (szz - sxx) * wy - dt * sxy * wx - dt * syz * wz;
  }
  Sv[0] = sxx + Pt[0][0]; Sv[1] = syy + Pt[1][1]; Sv[2] = szz + Pt[2][2];
  Sv[3] = sxy + Pt[0][1]; Sv[4] = syz + Pt[1][2]; Sv[5] = szx + Pt[2][0];
  double j2 = Sv[0] * Sv[0];
  j2 += Sv[1] * Sv[1];
  j2 += Sv[0] * Sv[1];
  j2 += Sv[3] * Sv[3];
  if (DIM == 3) {
    j2 += Sv[4] * Sv[4];
    j2 += Sv[5] * Sv[5];
  }
  if (j2 > (Y * Y) / 3.) {
    const double coeff = Y / sqrt(3. * j2);
#pragma unroll
    for (int q = 0; q < 6; ++q) Sv[q] *= coeff;
    // the plastic strain rate and strain (DefaultModelService.cc:211-214),
    // then the deviator's norm on the yield surface (215)
    const double rate = (1. - coeff) * Y / (3. * mu * coeff * dt);
    F.pl[N + c] = rate;
    F.pl[c] = F.pl[c] + rate;
    j2 = (Y * Y) / 3.;
  }
  F.pl[2 * N + c] = sqrt(j2);  // StrainNorm (224)
  w2 = work();
#pragma unroll
  for (int q = 0; q < 6; ++q) F.S[q * N + c] = Sv[q];
}

// computeGeometricValues of one cell: corner normals (kept for the next
// node pass), volume and characteristic length.  The cell pass reads V and
// l back, so neither kernel holds the corner normals and the
// thermodynamics live at the same time.
template <int DIM>
__device__ __forceinline__ void body_lagrange_geom(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  R3 coord[8];
#pragma unroll
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    int a, b, d;
    local_node_offset(l, a, b, d);
    const long long nn = node_id(M, i + a, j + b, k + d);
    coord[l] = {F.Xn[0][nn], F.Xn[1][nn], F.Xn[2][nn]};
  }
  double V;
  if (DIM == 3) {
    V = cell_volume_store3(coord, F, N, c);
  } else {
    R3 cqs[4];
    V = cell_volume<DIM>(coord, cqs);
    store_cqs<DIM>(F, N, c, cqs);
  }
  if (V < 0.) atomicOr(&F.s->status, ST_NEG_VOLUME);
  F.V[c] = V;
  F.l[c] = char_length(P, DIM, V, coord);
}

// EL: the elasto-plastic model needs the corner normals at n and n+1, so
// this pass computes the geometry itself; otherwise body_lagrange_geom ran
// first and V, l are read back.  CSTS (with the remap) needs them too, for
// the work of the forces in its energy update, and leaves pressure +
// pseudo-viscosity of the forward velocity update in pq.
// the temperature update of applyEOS (PerfectGasEOSService.cc:62-64,
// StiffenedGasEOSService.cc:58-60, MieGruneisenEOSService.cc:67-69) and of
// the PerfectGas / StiffenedGas applyOneCellEOS: the previous value kept
// (keep), the energy gained since the start of the iteration over cv added
// to it; Mie-Gruneisen's applyOneCellEOS (121-122) adds it to the value
// kept before
__device__ __forceinline__ void advance_temperature(const mhc_env_params& o, double e, double e_n, bool keep,
                                                    double& T, double& Tn) {
  if (keep) Tn = T;
  T = (e - e_n) / o.specific_heat + Tn;
}

template <int DIM, int NE, bool EULER, bool EL = false, bool CSTS = false>
__device__ __forceinline__ void body_lagrange_cells(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  constexpr bool GEO = EL || CSTS;
  long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  constexpr int NV = 3 * NE + 1;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  const int NBN = DIM == 3 ? 8 : 4;
  R3 cqs[GEO ? 8 : 1];
  R3 cqn[GEO ? 8 : 1];  // corner normals at n, read before they are replaced
  double V, l;
  if (GEO) {
    R3 coord[8];
    for (int q = 0; q < NBN; ++q) {
      int a, b, d;
      local_node_offset(q, a, b, d);
      long long nn = node_id(M, i + a, j + b, k + d);
      coord[q] = {F.Xn[0][nn], F.Xn[1][nn], F.Xn[2][nn]};
    }
    V = cell_volume<DIM>(coord, cqs);
    for (int q = 0; q < NBN; ++q) cqn[q] = load_cqs_rw<DIM>(F, N, c, q);
    store_cqs<DIM>(F, N, c, cqs);
    if (V < 0.) atomicOr(&F.s->status, ST_NEG_VOLUME);
    l = char_length(P, DIM, V, coord);
  } else {
    V = F.V[c];
    l = F.l[c];
  }
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
  // updateElasticityAndPlasticity: the work is added to the energy the
  // explicit and Newton updates start from (the GP update restarts from e_n)
  double ecur[NE];
  for (int q = 0; q < NE; ++q) ecur[q] = ene[q];
  if (F.ebc && pure) {
    // a boundary condition changed the (pure) cell's current energy
    for (int q = 0; q < NE; ++q) ecur[q] = F.ebc[c];
  }
  if (EL) {
    double w1, w2;
    elasto_cell<DIM>(P.env[0], M, F, c, i, j, k, cqn, cqs, V, F.V[c], me[0], rhoe[0], dt, w1, w2);
    ecur[0] = ecur[0] + w1;
    ecur[0] = ecur[0] + w2;
  }
  // energy deposits (MahycoModule.cc:1364-1417): value x deltat at the
  // Lagrangian cell centre of this iteration, before the energy update
  bool depot = false;
  for (int q = 0; q < NE; ++q) depot = depot || P.env[q].depot_type != MHC_DEPOT_NONE;
  if (depot) {
    R3 s = {0., 0., 0.};
    for (int q = 0; q < NBN; ++q) {
      int a, b, d;
      local_node_offset(q, a, b, d);
      const long long nn = node_id(M, i + a, j + b, DIM == 3 ? k + d : 0);
      s = s + R3{F.Xn[0][nn], F.Xn[1][nn], DIM == 3 ? F.Xn[2][nn] : 0.};
    }
    const R3 cc = (DIM == 2 ? .25 : .125) * s;
    const double t = F.s->t;
    for (int q = 0; q < NE; ++q) {
      const mhc_env_params& o = P.env[q];
      if (o.depot_type == MHC_DEPOT_NONE || !((mask >> q) & 1)) continue;
      double value = o.depot_value;
      if (t < o.depot_tdebut) value = 0.;
      if (t > o.depot_tfin) value = 0.;
      if (o.depot_type == MHC_DEPOT_LINEAIRE) {
        value += o.depot_dependance[0] * cc.x;
        value += o.depot_dependance[1] * cc.y;
        value += o.depot_dependance[2] * cc.z;
        value += o.depot_dependance[3] * t;
      } else if (o.depot_type == MHC_DEPOT_SUPER_GAUSSIAN) {
        // exp(-(y dY)^power) then exp(-(x dX)^power); CUDA's exp and pow,
        // within a few ulps of the reference's libm
        const double ay = cc.y * o.depot_dependance[1];
        value *= exp(-pow(ay, o.depot_power));
        const double ax = cc.x * o.depot_dependance[0];
        value *= exp(-pow(ax, o.depot_power));
      }
      if (fabs(cc.x - o.depot_origin[0]) > o.depot_cutoff[0]) value = 0.;
      if (fabs(cc.y - o.depot_origin[1]) > o.depot_cutoff[1]) value = 0.;
      ecur[q] = ecur[q] + value * dt;
    }
  }
  // CSTS: work of the forces through the corner normals at n+1 and n and
  // the node velocities at n+1/2 and n (MahycoModule.cc:1664-1675), summed
  // in local node order
  double cn1 = 0., cn = 0., cdn = 0., cov = 0.;
  if constexpr (CSTS) {
    const long long NN = M.nnode;
    const double odt = F.s->old_dt;
    for (int q = 0; q < NBN; ++q) {
      int a, b, d;
      local_node_offset(q, a, b, d);
      const long long nn = node_id(M, i + a, j + b, k + d);
      const R3 v = {F.vx[nn], F.vy[nn], F.vz[nn]};
      const R3 vn = {F.v0[nn], F.v0[NN + nn], F.v0[2 * NN + nn]};
      cn1 = cn1 + dot(v, cqs[q]) * dt;
      cn = cn + dot(v, cqn[q]) * dt;
      cdn = cdn + dot(v - vn, cqn[q]) * (dt - odt);
      cov = cov + dot(vn, cqn[q]) * odt;
    }
  }
  // the temperature of a Lagrangian run, advanced by every EOS call below
  // (advance_temperature)
  const bool temp = !EULER && F.T != nullptr;
  double Te[NE], Tne[NE];
  for (int q = 0; q < NE; ++q) {
    Te[q] = temp ? F.T[q * N + c] : 0.;
    Tne[q] = temp ? F.Tn[q * N + c] : 0.;
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
      ee_[q] = ecur[q] - (pne[q] + qq) * (1.0 / r - 1.0 / rn);
      eos_apply(P.env[q], r, ee_[q], pe[q], ce[q]);
      if (temp) advance_temperature(P.env[q], ee_[q], ene[q], true, Te[q], Tne[q]);
    } else if (P.with_newton) {
      // updateEnergyAndPressurebyNewton, non-CSTS branch (MahycoModule.cc:1506-1571):
      // at most 50 Newton steps from the energy at n; the pressure and sound
      // speed of the last step are recomputed from the final energy (EOS of
      // the Lagrange-only loop below, or after the remap) before any use
      double pseudo = 0.;
      if (P.pseudo_centree && ((qn + qq) * (1.0 / r - 1.0 / rn) < 0.)) pseudo = 0.5 * (qq + qn);
      if (!P.pseudo_centree && (qq * (1.0 / r - 1.0 / rn) < 0.)) pseudo = qq;
      const double en = ene[q], pn = pne[q];
      double en1 = ecur[q], pp = pn, dpde = 0.;
      int it = 0;
      while (it < 50 && fabs(fvnr(en1, pp, en, pseudo, pn, r, rn)) >= P.threshold) {
        eos_one_cell(P.env[q], r, en1, pp, dpde);
        if (temp) advance_temperature(P.env[q], en1, en, P.env[q].eos != MHC_EOS_MIE_GRUNEISEN, Te[q], Tne[q]);
        const double enew = en1 - fvnr(en1, pp, en, pseudo, pn, r, rn) / fvnrderiv(dpde, r, rn);
        en1 = enew;
        ++it;
      }
      ee_[q] = en1;
    } else if (CSTS) {
      // updateEnergyAndPressureforGP, CSTS branch (MahycoModule.cc:1676-1694);
      // the pseudo-viscosity at n-1 is 0 with the remap, which resets the
      // values at n after every remap (PrepareRemap.cc:219)
      const double g = P.env[q].adiabatic_cst;
      const double m = me[q], pn = pne[q], qnm1 = 0.;
      const double den = 1 + 0.5 * (g - 1.0) * r * cn1 / m;
      const double num = ecur[q] - (0.5 * (pn + qn) * cn / m) - (0.5 * qq * cn1 / m) + (0.25 * (pn + qn) * cdn / m) -
                         (0.5 * (qn - qnm1) * cov / m);
      ee_[q] = num / den;
    } else {
      double pseudo = 0.;
      if (P.pseudo_centree && ((qn + qq) * (1.0 / r - 1.0 / rn) < 0.)) pseudo = 0.5 * (qq + qn);
      if (!P.pseudo_centree && (qq * (1.0 / r - 1.0 / rn) < 0.)) pseudo = qq;
      double g = P.env[q].adiabatic_cst;
      double den = 1 + 0.5 * (g - 1.0) * r * (1.0 / r - 1.0 / rn);
      // the current pressure: the value at n unless a boundary condition set it
      const double pcur = (F.pbc && pure) ? F.pbc[c] : pne[q];
      double num = ene[q] - (0.5 * pcur + pseudo) * (1.0 / r - 1.0 / rn);
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
    if constexpr (EL) {
      // the deviator times the volume and the plastic strain rate and
      // strain times the mass (PrepareRemap.cc:121-128), one environment
      const double Vq = Ve[0], mq = Ve[0] * rhoe[0];
      U[(NV + 0) * N + c] = Vq * F.S[c];
      U[(NV + 1) * N + c] = Vq * F.S[N + c];
      U[(NV + 2) * N + c] = Vq * F.S[3 * N + c];
      U[(NV + 3) * N + c] = Vq * F.S[4 * N + c];
      U[(NV + 4) * N + c] = Vq * F.S[5 * N + c];
      U[(NV + 5) * N + c] = mq * F.pl[N + c];
      U[(NV + 6) * N + c] = mq * F.pl[c];
    }
    if constexpr (CSTS) {
      // the cell pressure of the forward update: the new one of an explicit
      // update in a pure cell, otherwise the one the cell holds (at n; a
      // mixed cell's average of the last remap)
      double pf = F.p[c];
      if (P.pression_explicite && pure)
        for (int q = 0; q < NE; ++q) if ((mask >> q) & 1) pf = pe[q];
      F.pq[c] = pf + qg;
    }
    if (F.phi_pb) {
      // pente-borne phi of the first sweep (PrepareRemap.cc:138-157): the
      // environment's density and internal energy, the pseudo-viscosity;
      // the volume fractions are those of the last remap
      for (int q = 0; q < NE; ++q) {
        if (!((mask >> q) & 1)) continue;
        F.phi_pb[(NE + q) * N + c] = rhoe[q];
        F.phi_pb[(2 * NE + q) * N + c] = ee_[q];
      }
      F.phi_pb[(NV - 1) * N + c] = qg;
    }
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
      if (temp) advance_temperature(P.env[q], ev, ene[q], true, Te[q], Tne[q]);
    }
  }
  if (temp) {
    for (int q = 0; q < NE; ++q) {
      if (!((mask >> q) & 1)) continue;
      F.T[q * N + c] = Te[q];
      F.Tn[q * N + c] = Tne[q];
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
// sans-lagrange (pure advection), nodes: updateVelocityWithoutLagrange
// (MahycoModule.cc:676-700), applyBoundaryCondition and updatePosition
// (MahycoModule.cc:730-750), where only the nodes shared by exactly four
// cells move.  The velocities at n are the prescribed ones (v0); with the
// RIDER reverse option they are scaled by cos(Pi t parameter), Pi the
// reference's 3.14159265359 (TypesMahyco.h:42).
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void body_advect_nodes(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const long long NN = M.nnode;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  const double dt = F.s->dt;
  const double t = F.s->t;
  const bool rider = P.cas_model == MHC_CASE_RIDER;
  const double option_real = (rider && P.rider_reverse) ? 1. : 0.;
  const double factor = rider ? P.rider_parameter : 0.;
  const double cs = cos(3.14159265359 * t * factor);
  const double ux = F.v0[n], uy = F.v0[NN + n], uz = F.v0[2 * NN + n];
  double vx = ux * (1. - option_real) + option_real * ux * cs;
  double vy = uy * (1. - option_real) + option_real * uy * cs;
  double vz = uz * (1. - option_real) + option_real * uz * cs;
  const R3 x = P.is_euler_scheme == MHC_EULER_FULL ? node_x0(M, i, j, k) : R3{F.Xp[0][n], F.Xp[1][n], F.Xp[2][n]};
  velocity_bcs(M, P, i, j, k, t, dt, x, vx, vy, vz);
  int nc = ((i > 0) + (i < M.ncx)) * ((j > 0) + (j < M.ncy));
  if (DIM == 3) nc *= (k > 0) + (k < M.ncz);
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  if (nc == 4) {
    F.Xn[0][n] = x.x + dt * vx; F.Xn[1][n] = x.y + dt * vy; F.Xn[2][n] = x.z + dt * vz;
  } else {
    F.Xn[0][n] = x.x; F.Xn[1][n] = x.y; F.Xn[2][n] = x.z;
  }
}

// sans-lagrange, cells: after the geometry pass (body_lagrange_geom), only
// computeVariablesForRemap (PrepareRemap.cc:94-193): the density, energy
// and pseudo-viscosity keep their values (updateDensity,
// computeArtificialViscosity and updateEnergyAndPressure return at once),
// the volumes are the new ones (a mixed cell's environment volume its
// fraction of the cell's, computeGeometricValues)
template <int DIM, int NE>
__device__ __forceinline__ void body_advect_cells(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  constexpr int NV = 3 * NE + 1;
  const double V = F.V[c];
  const uint8_t mask = F.mask[c];
  const bool pure = __popc(mask) == 1;
  double* U = F.U[0];
  for (int q = 0; q < NE; ++q) {
    const bool in = (mask >> q) & 1;
    double Vq = 0., rq = 0., eq = 0.;
    if (in) {
      const bool slot = NE > 1 && !pure;
      Vq = slot ? F.ef[q * N + c] * V : V;
      rq = slot ? F.erho[q * N + c] : F.rho[c];
      eq = slot ? F.ee[q * N + c] : F.e[c];
      if (F.phi_pb) {
        F.phi_pb[(NE + q) * N + c] = rq;
        F.phi_pb[(2 * NE + q) * N + c] = eq;
      }
    }
    U[q * N + c] = Vq;
    U[(NE + q) * N + c] = in ? Vq * rq : 0.;
    U[(2 * NE + q) * N + c] = in ? Vq * rq * eq : 0.;
  }
  const double qg = F.q[c];
  U[(NV - 1) * N + c] = V * qg;
  if (F.phi_pb) F.phi_pb[(NV - 1) * N + c] = qg;
}

// ---------------------------------------------------------------------------
// CSTS, before the remap: updateVelocityForward (MahycoModule.cc:637-700),
// the velocities from n+1/2 to n+1 with the forces of the new pressure,
// pseudo-viscosity and corner normals (gathered in ascending cell id), and
// the node terms of the remap's face velocities, the means of the
// velocities at n and n+1 (PrepareRemap.cc:45-52)
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void body_csts_forward(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const long long N = M.ncell, NN = M.nnode;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  constexpr int NS = DIM == 3 ? 8 : 4;
  R3 S = {0., 0., 0.};
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int di = (s & 1) - 1, dj = ((s >> 1) & 1) - 1, dk = DIM == 3 ? ((s >> 2) & 1) - 1 : 0;
    const int ci = i + di, cj = j + dj, ck = k + dk;
    if (ci < 0 || cj < 0 || ci >= M.ncx || cj >= M.ncy || (DIM == 3 && (ck < 0 || ck >= M.ncz))) continue;
    const int l = (-dk) * 4 + ((-dj) ? ((-di) ? 2 : 3) : ((-di) ? 1 : 0));
    const long long c = cell_id(M, ci, cj, ck);
    const R3 fv = F.pq[c] * load_cqs<DIM>(F, N, c, l);
    S.x = S.x + fv.x; S.y = S.y + fv.y; S.z = S.z + fv.z;
  }
  const double dt = 0.5 * F.s->dt;
  const double f = dt / F.mn[n];
  double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
  vx = vx + f * S.x; vy = vy + f * S.y; vz = vz + f * S.z;
  vx = vx + dt * P.gravity[0]; vy = vy + dt * P.gravity[1]; vz = vz + dt * P.gravity[2];
  F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  F.fv[0][n] = 0.5 * (vx + F.v0[n]);
  F.fv[1][n] = 0.5 * (vy + F.v0[NN + n]);
  F.fv[2][n] = 0.5 * (vz + F.v0[2 * NN + n]);
}

// The remap sweeps (one direction, cells and nodes) live in mhc_sweep.cuh.

// ---------------------------------------------------------------------------
// remap finalize, cells: RemapADIService::remapVariables (RemapADIFinal.cc:21-319)
// then applyEOS per environment and computePressionMoyenne
// (PrepareRemap.cc:242-249, MahycoModule.cc:1708-1735)
// ---------------------------------------------------------------------------
// ADV: sans-lagrange (no dual projection): a cell keeps an environment
// whose projected mass is zero, the pressure and sound speed of a mixed
// cell are not averaged (computePressionMoyenne returns at once), and the
// Fictif equation of state applies
template <int DIM, int NE, bool ADV>
__device__ __forceinline__ void body_remap_finalize_cells(const Mesh& M, const mhc_case_params& P, const Fields& F,
                                                          const double* Ufin, const double* Udfin, int bx) {
  long long c = bx * (long long)CT + threadIdx.x;
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
    if ((div_rn(u[q], Veul) < thr || (u[NE + q] == 0. && !ADV)) && in) {
      nm &= (uint8_t)~(1 << q);
    } else if (div_rn(u[q], Veul) > thr && !in) {
      double volt = 0.;
      for (int r = 0; r < NE; ++r) volt += u[r];
      double vn = div_rn(u[q] * Veul, volt);
      if (div_rn(vn, Veul) > thr && u[NE + q] != 0.) nm |= (uint8_t)(1 << q);
    }
  }
  const bool oldpure = __popc(old) == 1;
  const bool pure = __popc(nm) == 1;
  // mass fractions survive a cell whose total mass is below threshold^2.
  // A pure cell's volume and mass fractions (the global slots of the
  // reference) live in the entries of its one environment.
  double mfe[NE];
  for (int q = 0; q < NE; ++q) mfe[q] = 0.;
  {
    // previous values with the pure-cell storage transfer of the env manager
    for (int q = 0; q < NE; ++q) {
      bool was = (old >> q) & 1;
      if (!was) continue;
      mfe[q] = (NE > 1 && !oldpure) ? F.emf[q * N + c] : 1.;
    }
    if (pure)
      for (int q = 0; q < NE; ++q)
        if (((nm >> q) & 1) && !((old >> q) & 1)) mfe[q] = 1.;
  }
  double vol[NE];
  double volt = 0., masset = 0.;
  for (int q = 0; q < NE; ++q) { vol[q] = u[q]; volt += vol[q]; masset += u[NE + q]; }
  double unsurvolt = 1. / volt;
  for (int q = 0; q < NE; ++q) vol[q] *= Veul * unsurvolt;
  double unsurvol = 1. / Veul;
  double fe[NE];
  for (int q = 0; q < NE; ++q) fe[q] = 0.;
  double somme_frac = 0.;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    fe[q] = vol[q] * unsurvol;
    if (fe[q] < thr) fe[q] = 0.;
    somme_frac += fe[q];
  }
  double unsursf = 0.;
  if (somme_frac != 0.) unsursf = 1. / somme_frac;
  for (int q = 0; q < NE; ++q)
    if ((nm >> q) & 1) fe[q] *= unsursf;
  if (masset > thr * thr) {
    double unsurm = 1. / masset, fm = 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((nm >> q) & 1)) continue;
      mfe[q] = u[NE + q] * unsurm;
      if (fe[q] < thr) mfe[q] = 0.;
      fm += mfe[q];
    }
    if (fm != 0.) {
      double unsurfm = 1. / fm;
      for (int q = 0; q < NE; ++q)
        if ((nm >> q) & 1) mfe[q] *= unsurfm;
    }
  }
  // environment densities and energies (0 for an absent environment)
  double rhoe[NE], ee[NE];
  double dn = 0.;
  for (int q = 0; q < NE; ++q) {
    rhoe[q] = 0.;
    if (!((nm >> q) & 1)) continue;
    if (fe[q] > thr && vol[q] != 0.) rhoe[q] = div_rn(u[NE + q], vol[q]);
    dn += fe[q] * rhoe[q];
  }
  for (int q = 0; q < NE; ++q) {
    ee[q] = 0.;
    if (!((nm >> q) & 1)) continue;
    if (fe[q] > thr && u[NE + q] != 0.) ee[q] = div_rn(u[2 * NE + q], u[NE + q]);
  }
  if (NE == 1 && F.S && !ADV && fe[0] > thr && u[NE] != 0.) {
    // an elasto-plastic case: the deviator over the projected volume, its
    // zz from the zero trace, the plastic strain rate and strain over the
    // projected mass (RemapADIFinal.cc:200-214)
    const double xx = Ufin[NV * N + c] / u[0], yy = Ufin[(NV + 1) * N + c] / u[0];
    F.S[c] = xx;
    F.S[N + c] = yy;
    F.S[2 * N + c] = -(xx + yy);
    F.S[3 * N + c] = Ufin[(NV + 2) * N + c] / u[0];
    F.S[4 * N + c] = Ufin[(NV + 3) * N + c] / u[0];
    F.S[5 * N + c] = Ufin[(NV + 4) * N + c] / u[0];
    F.pl[N + c] = Ufin[(NV + 5) * N + c] / u[NE];
    F.pl[c] = Ufin[(NV + 6) * N + c] / u[NE];
  }
  // aliased stores: g* are the global slots, e*[] the env slots (a mixed
  // cell's environment masses mfe * mg and pseudo-viscosities qv are
  // formed at the store)
  double rhog = dn;
  double mg = Veul * dn;
  double eg = 0., qg = 0.;
  const double qv = u[NV - 1] * unsurvol;
  double en = 0., ps = 0.;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    if (pure) {
      mg = mfe[q] * mg;
      qg = qv;
      rhog = rhoe[q];
      eg = ee[q];
      en += mfe[q] * eg;
      ps += fe[q] * qg;
    } else {
      en += mfe[q] * ee[q];
      ps += fe[q] * qv;
    }
  }
  eg = en;
  qg = ps;
  int st = 0;
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    if (pure) {
      if (rhog < 0. || eg < 0.) { eg = 0.; rhog = 0.; fe[q] = 0.; mfe[q] = 0.; }
      if (rhog != rhog || eg != eg) st |= ST_NAN;
    } else {
      if (rhoe[q] < 0. || ee[q] < 0.) { ee[q] = 0.; rhoe[q] = 0.; fe[q] = 0.; mfe[q] = 0.; }
      if (rhoe[q] != rhoe[q] || ee[q] != ee[q]) st |= ST_NAN;
    }
  }
  if (st) atomicOr(&F.s->status, st);
  if (P.conservation_energie_totale) {
    // kinetic energy lost by the dual projection back into the internal
    // energy (RemapADIFinal.cc:320-344): 0.25 per node of the projected
    // minus the reconstructed kinetic energy, in cell node order
    int ci, cj, ck;
    cell_ijk(M, c, ci, cj, ck);
    const long long NN = M.nnode;
    double delta = 0.;
    for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
      int di, dj, dk;
      local_node_offset(l, di, dj, dk);
      const long long n = node_id(M, ci + di, cj + dj, DIM == 3 ? ck + dk : 0);
      const double m = Udfin[3 * NN + n];
      if (m != 0.) {
        const double ec_proj = Udfin[4 * NN + n] / m;
        const double vx = Udfin[n] / m, vy = Udfin[NN + n] / m, vz = Udfin[2 * NN + n] / m;
        const double ec_rec = 0.5 * (vx * vx + vy * vy + vz * vz);
        delta += 0.25 * (ec_proj - ec_rec);
      }
    }
    delta = smax(0., delta);
    for (int q = 0; q < NE; ++q) {
      if (!((nm >> q) & 1)) continue;
      if (pure) eg += mfe[q] * delta;
      else ee[q] += mfe[q] * delta;
    }
    if (!pure) eg += delta;
  }
  // applyEOS per environment, then computePressionMoyenne
  double pg = 0., cg = 0., pe[NE], ce[NE];
  for (int q = 0; q < NE; ++q) { pe[q] = ce[q] = 0.; }
  for (int q = 0; q < NE; ++q) {
    if (!((nm >> q) & 1)) continue;
    if (ADV && P.env[q].eos == MHC_EOS_FICTIF) {
      // the environment's pressure before: its slot value carried through
      // the membership change (a new environment of a mixed cell starts
      // from 0, a pure cell's global slot keeps its value)
      const bool was = (old >> q) & 1;
      double p_old;
      if (pure) p_old = (was && !oldpure && NE > 1) ? F.ep[q * N + c] : F.p[c];
      else p_old = was ? (oldpure ? F.p[c] : F.ep[q * N + c]) : 0.;
      const double t = F.s->t;
      if (pure) { fictif_apply(P.env[q], t, p_old, pg, cg); eg = 0.; }
      else { fictif_apply(P.env[q], t, p_old, pe[q], ce[q]); ee[q] = 0.; }
      continue;
    }
    if (pure) eos_apply(P.env[q], rhog, eg, pg, cg);
    else eos_apply(P.env[q], rhoe[q], ee[q], pe[q], ce[q]);
  }
  if (!pure && ADV) {
    // no pressure average without Lagrange phase (MahycoModule.cc:1711)
    pg = F.p[c];
    cg = F.c[c];
  }
  if (!pure && !ADV) {
    pg = 0.; cg = 0.;
    double option = P.calcul_vitson_max ? 1. : 0.;
    for (int q = 0; q < NE; ++q) {
      if (!((nm >> q) & 1)) continue;
      pg += fe[q] * pe[q];
      cg = option * smax(ce[q], cg);
      cg += (1. - option) * fe[q] * ce[q];
    }
  }
  if (F.phi_pb) {
    // pente-borne phi of the next remap's first sweep: the volume fraction
    // of a present environment (the pure-cell value included); an absent
    // environment keeps the values of this remap's last sweep
    // (RemapADIService.cc:493-530 on the final projected values)
    // (the projected values read again: they are cached, and not keeping
    // them live through the EOS saves registers)
    double sv = 0.;
    for (int q = 0; q < NE; ++q) sv += Ufin[q * N + c];
    for (int q = 0; q < NE; ++q) {
      if ((nm >> q) & 1) {
        F.phi_pb[q * N + c] = fe[q];
      } else {
        const double v = Ufin[q * N + c], m = Ufin[(NE + q) * N + c], ie = Ufin[(2 * NE + q) * N + c];
        F.phi_pb[q * N + c] = div_rn(v, sv);
        F.phi_pb[(NE + q) * N + c] = v != 0. ? div_rn(m, v) : 0.;
        F.phi_pb[(2 * NE + q) * N + c] = m != 0. ? div_rn(ie, m) : 0.;
      }
    }
  }
  F.rho[c] = rhog; F.e[c] = eg; F.p[c] = pg; F.c[c] = cg; F.q[c] = qg; F.m[c] = mg;
  F.V[c] = Veul;
  F.mask[c] = nm;
  if (NE > 1 && !pure) {
    for (int q = 0; q < NE; ++q) {
      const bool in = (nm >> q) & 1;
      F.ef[q * N + c] = fe[q]; F.emf[q * N + c] = mfe[q]; F.em[q * N + c] = in ? mfe[q] * mg : 0.;
      F.erho[q * N + c] = rhoe[q]; F.ee[q * N + c] = ee[q]; F.ep[q * N + c] = pe[q];
      F.ec[q * N + c] = ce[q]; F.eq[q * N + c] = in ? qv : 0.;
    }
  } else if (NE > 1) {
    // a pure cell's volume fraction, the normalised one of the reference
    // (m_fracvol of the cell, which can end an ulp below 1); only read
    // back, in the environment's slot
    for (int q = 0; q < NE; ++q)
      if ((nm >> q) & 1) F.ef[q * N + c] = fe[q];
  }
}

// Cell variables of the boundary conditions (applyBoundaryConditionForCellVariables,
// MahycoModule.cc:838-907), after the node pass and before the position
// update has any effect on the cell pass: the conditions in order, each on
// the cell of every face of its surface.  Global cell values (a pure cell's
// environment value is the same).  Density and Pressure take the value
// inside [Tdebut, Tfin), 0 outside; the energies always add theirs inside
// the x / y cutoffs of the cell centre (the centre of the positions the
// cycle started from), SuperGaussianEnergy times exp(-(y dY)^4).
__device__ __forceinline__ bool cell_on_surface(const Mesh& M, int i, int j, int k, int surf) {
  switch (surf) {
    case MHC_XMIN: return i == 0;
    case MHC_XMAX: return i == M.ncx - 1;
    case MHC_YMIN: return j == 0;
    case MHC_YMAX: return j == M.ncy - 1;
    case MHC_ZMIN: return M.dim == 3 && k == 0;
    default: return M.dim == 3 && k == M.ncz - 1;
  }
}

template <int DIM>
__device__ __forceinline__ void body_cell_bcs(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  const double t = F.s->t;
  bool centre = false;
  R3 cc = {0., 0., 0.};
  double ec = F.e[c], pc = F.p[c];
  for (int b = 0; b < P.nb_bc; ++b) {
    const mhc_bc& bc = P.bc[b];
    if (bc.kind < MHC_BC_DENSITY || bc.kind > MHC_BC_PRESSURE) continue;
    if (!cell_on_surface(M, i, j, k, bc.surface)) continue;
    double value = bc.value;
    if (t < bc.tdebut) value = 0.;
    if (t >= bc.tfin) value = 0.;
    if (bc.kind == MHC_BC_DENSITY) {
      // the density itself is recomputed from this mass by updateDensity
      F.m[c] = value * F.V[c];
    } else if (bc.kind == MHC_BC_PRESSURE) {
      pc = value;
    } else {
      if (!centre) {
        R3 sum = {0., 0., 0.};
        for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
          int a, bb, d;
          local_node_offset(l, a, bb, d);
          const long long nn = node_id(M, i + a, j + bb, DIM == 3 ? k + d : 0);
          sum = sum + R3{F.Xp[0][nn], F.Xp[1][nn], DIM == 3 ? F.Xp[2][nn] : 0.};
        }
        cc = (DIM == 2 ? .25 : .125) * sum;
        centre = true;
      }
      value = bc.value;
      if (bc.kind == MHC_BC_SUPER_GAUSSIAN_ENERGY) {
        // CUDA's exp and pow, within a few ulps of the reference's libm
        const double ay = cc.y * bc.dependance[1];
        value *= exp(-pow(ay, 4.));
      }
      if (fabs(cc.x) > bc.cutoff[0]) value = 0.;
      if (fabs(cc.y) > bc.cutoff[1]) value = 0.;
      ec = ec + value;
    }
  }
  F.ebc[c] = ec;
  F.pbc[c] = pc;
}

// ... and the Density conditions' cell masses added to the node masses: each
// node gathers, condition by condition, the cells of its surface faces in
// face order (the reference adds value * V / nb_nodes to every node of each
// such cell as it walks the faces)
template <int DIM>
__device__ __forceinline__ void body_node_bcs(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  const long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  const double t = F.s->t;
  const double w8 = DIM == 2 ? .25 : .125;
  double mn = F.mn[n];
  bool touched = false;
  for (int b = 0; b < P.nb_bc; ++b) {
    const mhc_bc& bc = P.bc[b];
    if (bc.kind != MHC_BC_DENSITY) continue;
    const int s = bc.surface;
    const int d = (s == MHC_XMIN || s == MHC_XMAX) ? 0 : ((s == MHC_YMIN || s == MHC_YMAX) ? 1 : 2);
    if (d >= DIM) continue;
    const bool maxside = s >= MHC_XMAX;
    const int nid = d == 0 ? i : (d == 1 ? j : k);
    const int nnd = d == 0 ? M.nnx : (d == 1 ? M.nny : M.nnz);
    // the two node layers of the surface's cells (every node of those cells)
    if (maxside ? nid < nnd - 2 : nid > 1) continue;
    double value = bc.value;
    if (t < bc.tdebut) value = 0.;
    if (t >= bc.tfin) value = 0.;
    // the surface's faces around the node, in face id order (the slower
    // transverse axis outermost), and the cell of each
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    const int idx[3] = {i, j, k};
    const int nc[3] = {M.ncx, M.ncy, M.ncz};
    for (int o2 = (DIM == 3 ? -1 : 0); o2 <= 0; ++o2) {
      for (int o1 = -1; o1 <= 0; ++o1) {
        const int t1 = idx[a1] + o1, t2 = DIM == 3 ? idx[a2] + o2 : 0;
        if (t1 < 0 || t1 >= nc[a1]) continue;
        if (DIM == 3 && (t2 < 0 || t2 >= nc[a2])) continue;
        int ci[3];
        ci[d] = maxside ? nc[d] - 1 : 0;
        ci[a1] = t1;
        ci[a2] = DIM == 3 ? t2 : 0;
        const long long cf = cell_id(M, ci[0], ci[1], DIM == 3 ? ci[2] : 0);
        mn = mn + w8 * (value * F.V[cf]);
        touched = true;
      }
    }
  }
  if (touched) F.mn[n] = mn;
}

// per-axis Euler remap (is-euler-scheme X / Y / Z), after the sweeps:
// RemapADIService::computeVolumeEuler (RemapADIService.cc:579-645) gives
// the receiving cell the remapped axis on the initial grid and the other
// coordinates of this iteration's Lagrangian step; its corner normals
// replace the Lagrangian ones for the next node pass
template <int DIM>
__device__ __forceinline__ void body_euler_volume(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  const int ax = P.is_euler_scheme - MHC_EULER_X;
  int i, j, k;
  cell_ijk(M, c, i, j, k);
  R3 coord[8], cqs[8];
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    int a, b, d;
    local_node_offset(l, a, b, d);
    const long long nn = node_id(M, i + a, j + b, DIM == 3 ? k + d : 0);
    const R3 x0 = node_x0(M, i + a, j + b, DIM == 3 ? k + d : 0);
    coord[l] = R3{ax == 0 ? x0.x : F.Xn[0][nn], ax == 1 ? x0.y : F.Xn[1][nn],
                  DIM == 3 ? (ax == 2 ? x0.z : F.Xn[2][nn]) : 0.};
  }
  F.Veul[c] = cell_volume<DIM>(coord, cqs);
  store_cqs<DIM>(F, N, c, cqs);
}

// ... and the remapped axis of the node positions back on the initial grid
// (RemapADIService.cc:65-82); the next Lagrangian step starts from them
__device__ __forceinline__ void body_euler_axis_reset(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const int ax = P.is_euler_scheme - MHC_EULER_X;
  int i, j, k;
  node_ijk(M, n, i, j, k);
  const R3 x0 = node_x0(M, i, j, k);
  F.Xn[ax][n] = ax == 0 ? x0.x : (ax == 1 ? x0.y : x0.z);
}

// remap finalize, nodes: velocity from projected momentum and node mass
// rebuilt from the new cell masses (RemapADIFinal.cc:287-319)
// DUAL: the dual projection ran (not with sans-lagrange, whose velocities
// stay prescribed)
template <int DIM, bool DUAL>
__device__ __forceinline__ void body_remap_finalize_nodes(const Mesh& M, const Fields& F, const double* Ud, int bx) {
  long long n = bx * (long long)CT + threadIdx.x;
  if (n >= M.nnode) return;
  const long long NN = M.nnode;
  double m = DUAL ? Ud[3 * NN + n] : 0.;
  double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
  if (m != 0.) {
    vx = div_rn(Ud[n], m);
    vy = div_rn(Ud[NN + n], m);
    vz = div_rn(Ud[2 * NN + n], m);
    F.vx[n] = vx; F.vy[n] = vy; F.vz[n] = vz;
  }
  // the node speed of computeDeltaT (Vector normL2), once per node
  if (F.spd) F.spd[n] = sqrt(vx * vx + vy * vy + vz * vz);
  int i, j, k;
  node_ijk(M, n, i, j, k);
  F.mn[n] = node_mass_gather<DIM>(M, F.m, i, j, k);
}

// ---------------------------------------------------------------------------
// computeDeltaT (MahycoModule.cc:1739-1864): per-cell l / (c + vmax), block
// minimum, then one ordered-bits atomicMin per block.  The minimum of
// non-NaN values does not depend on the reduction order.
// ---------------------------------------------------------------------------
template <int DIM, bool SPD = false>
__device__ __forceinline__ void body_delta_t(const Mesh& M, const mhc_case_params& P, const Fields& F, int bx) {
  long long c = bx * (long long)CT + threadIdx.x;
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
        if (SPD) {
          vmax = amax(__ldg(F.spd + n), vmax);  // stored by the node finalize pass of this iteration
        } else {
          double vx = F.vx[n], vy = F.vy[n], vz = F.vz[n];
          vmax = amax(sqrt(vx * vx + vy * vy + vz * vz), vmax);
        }
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
    dx = (lane < CT / 32) ? red[lane] : 1.7976931348623157e308;
    for (int o = 16; o > 0; o >>= 1) dx = fmin(dx, __shfl_xor_sync(0xffffffffu, dx, o));
    if (lane == 0) atomicMin(&F.s->dt_min_bits, (unsigned long long)__double_as_longlong(dx));
  }
}

// standalone IEquationOfState::applyEOS(env) on the current state of the
// environment cells, followed by computePressionMoyenne for mixed cells
template <int NE>
__device__ __forceinline__ void body_eos_apply(const Mesh& M, const mhc_case_params& P, const Fields& F, int env, int bx) {
  long long c = bx * (long long)CT + threadIdx.x;
  if (c >= M.ncell) return;
  const long long N = M.ncell;
  const uint8_t mask = F.mask[c];
  if (!((mask >> env) & 1)) return;
  const bool pure = __popc(mask) == 1;
  const mhc_env_params& o = P.env[env];
  const bool fictif = o.eos == MHC_EOS_FICTIF;
  if (pure) {
    double p, cs;
    if (fictif) { fictif_apply(o, F.s->t, F.p[c], p, cs); F.e[c] = 0.; }
    else eos_apply(o, F.rho[c], F.e[c], p, cs);
    F.p[c] = p; F.c[c] = cs;
    return;
  }
  double p, cs;
  if (fictif) { fictif_apply(o, F.s->t, F.ep[env * N + c], p, cs); F.ee[env * N + c] = 0.; }
  else eos_apply(o, F.erho[env * N + c], F.ee[env * N + c], p, cs);
  F.ep[env * N + c] = p; F.ec[env * N + c] = cs;
  if (P.sans_lagrange) return;  // no pressure average (MahycoModule.cc:1711)
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
__device__ __forceinline__ void body_delta_t_finalize(const mhc_case_params& P, const Fields& F) {
  Scalars* s = F.s;
  double old = s->dt;
  double new_dt;
  if (P.sans_lagrange || P.deltat_constant) {
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
