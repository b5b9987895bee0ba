/*
 * mahyco_oracle.cc -- CPU ORACLE for the MaHyCo hydro cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain sequential C++, the
 * reference algorithm of the cycle hot path so that the CUDA library can be
 * checked against it.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it; the product library never links it.
 *
 * Parity pinning: the oracle is checked against the reference's own
 * non-regression time histories (the NONREGRESSION case folders, output/courbes/gnuplot,
 * copied as fixtures under tests/golden/ by tests/golden/make_golden.py).
 *
 * The reference (cea-hpc/MaHyCo) builds only on top of the Arcane framework,
 * which is not vendored, so the reference itself cannot be compiled here.
 * Arcane semantics that the reference relies on are restated as follows:
 *   - cartesian generator: node (i,j,k) at origin + i*(L/n), uid x-fastest;
 *     cells x-fastest; Hexa8 local nodes (0,0,0),(1,0,0),(1,1,0),(0,1,0),
 *     then the same at k+1; Quad4 likewise without k.
 *   - Hexa8 local faces (0,3,2,1),(0,4,7,3),(0,1,5,4),(4,5,6,7),(1,2,6,5),
 *     (2,3,7,6); Quad4 local faces (k,k+1).  Face nodes are re-ordered to
 *     start at the smallest uid and continue towards the smaller neighbour.
 *   - faces and nodes are numbered in creation order (cell by cell), so every
 *     scatter of the reference sums in ascending cell / face local id.
 *   - material variables: a cell holding exactly one environment stores the
 *     environment value in the global slot (EV() below models that aliasing).
 *   - time loop: global_time += deltat before the compute-loop entry points;
 *     old deltat of the first iteration is 0.
 *
 * Quantities the reference projects but never feeds back into the hydro
 * state without an elasto-plastic model (phase fractions, stress deviator,
 * plastic strain, previous energy, temperature) are not carried: the remap
 * keeps volume, mass and energy per environment plus the pseudo-viscosity.
 */
#include "../include/mahyco_case.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace ora {

struct R3 {
  double x, y, z;
};
static inline R3 operator+(R3 a, R3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline R3 operator-(R3 a, R3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline R3 operator*(double s, R3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline R3 operator*(R3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline R3 operator/(R3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline R3& operator+=(R3& a, R3 b) { a = a + b; return a; }
static inline R3& operator-=(R3& a, R3 b) { a = a - b; return a; }
static inline R3 operator-(R3 a) { return {-a.x, -a.y, -a.z}; }
static inline double dot(R3 a, R3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* math::vecMul */
static inline R3 vecmul(R3 u, R3 v) {
  return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
static inline double norm(R3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline double comp(R3 a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
/* Arcane math::min / math::max */
static inline double amin(double a, double b) { return (a < b) ? a : b; }
static inline double amax(double a, double b) { return (a < b) ? b : a; }
/* ---------------------------------------------------------------------------
 * correctly rounded powers (test switch "cr_pow")
 *
 * The reference calls std::pow, and glibc's pow is not correctly rounded
 * (pow(x, 0.5) != sqrt(x) for about 1 input in 1200 with glibc 2.39).  With
 * cr_pow set, the oracle evaluates the same powers correctly rounded, which
 * is what the CUDA library does; the default keeps the literal std::pow.
 * ------------------------------------------------------------------------- */
static inline void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = std::fma(a, b, -p);
}
static inline double cube_cr(double x) {
  double s, sl, t, tl, u, ul;
  two_prod(x, x, s, sl);
  two_prod(s, x, t, tl);
  two_prod(sl, x, u, ul);
  return t + (tl + (u + ul));
}
/* x^(1./3.): cbrt refined to double-double, times exp(-d ln x) with
 * d = 1/3 - double(1/3) = 2^-54/3, rounded once */
static inline double pow_third_cr(double x) {
  if (!(x > 0.0) || std::isinf(x)) return std::pow(x, 1. / 3.);
  double r = std::cbrt(x);
  double s, sl, t, tl;
  two_prod(r, r, s, sl);
  two_prod(s, r, t, tl);
  double res = ((x - t) - tl) - sl * r;
  double c_lo = res / (3.0 * s);
  const double d = (1.0 / 3.0) * 0x1p-54;
  double corr = c_lo - r * (d * std::log(x));
  return r + corr;
}
/* x^(5./3.): x times the double-double square of the refined cbrt, times
 * exp(d ln x) with d = double(5/3) - 5/3 = 2^-52/3, rounded once */
static inline double pow_five_thirds_cr(double x) {
  if (!(x > 0.0) || std::isinf(x)) return std::pow(x, 5. / 3.);
  double r = std::cbrt(x);
  double s, sl, t, tl;
  two_prod(r, r, s, sl);
  two_prod(s, r, t, tl);
  const double c_lo = (((x - t) - tl) - sl * r) / (3.0 * s);
  double q, ql;
  two_prod(x, s, q, ql);
  const double d = (1.0 / 3.0) * 0x1p-52;
  const double corr = (ql + x * (sl + 2.0 * r * c_lo)) + q * (d * std::log(x));
  return q + corr;
}

/* MahycoModule::produit (MahycoModule.cc:1935) */
static inline double produit(double A, double B, double C, double D) { return A * B - C * D; }

struct MatField {
  std::vector<double> g;
  std::vector<double> e[MHC_MAX_ENV];
  void init(long n, int nenv, double v = 0.0) {
    g.assign(n, v);
    for (int k = 0; k < nenv; ++k) e[k].assign(n, v);
  }
  void fill(double v) {
    std::fill(g.begin(), g.end(), v);
    for (auto& a : e) std::fill(a.begin(), a.end(), v);
  }
};

enum { ST_OK = 0, ST_NEG_VOLUME = 1, ST_DT_UNDERFLOW = 2, ST_NAN = 3 };

struct THLine {
  double time;
  double v[MHC_MAX_ENV][4];  /* CellMass, Pressure, Density, InternalEnergy */
  int present[MHC_MAX_ENV];
};

struct Case {
  mhc_case_params P;
  int dim = 3, nenv = 1;
  int ncx = 1, ncy = 1, ncz = 1, nnx = 2, nny = 2, nnz = 1;
  long ncell = 0, nnode = 0;
  int nbn = 8;  /* nodes per cell */
  /* nodes */
  std::vector<R3> coord, coord0, vel, vel_n, force;
  std::vector<double> node_mass;
  /* cells (non material) */
  std::vector<R3> cell_coord;
  std::vector<double> char_len, div_u, euler_volume, materiau;
  std::vector<R3> cqs, cqs_n;         /* ncell * nbn */
  /* elasto-plasticity (single environment): stress deviator at n+1 and n,
   * symmetric, components xx yy zz xy yz zx per cell */
  bool elasto = false;
  std::vector<double> sdev, sdev_n;
  /* elasto outputs: plastic strain, its rate, the deviator's norm */
  std::vector<double> plastic, plastic_rate, strain_norm;
  std::vector<double> tensF;  /* NewHypoModel: the deformation gradient [ncell][3][3] */
  std::vector<R3> hourglass;          /* anti-hourglass velocity correction */
  std::vector<R3> outer_normal;       /* ncell * 2*dim */
  /* faces, per direction */
  long nface[3] = {0, 0, 0};
  std::vector<R3> face_normal[3], face_coord[3];
  std::vector<double> face_len[3];     /* face_length_lagrange component d */
  std::vector<double> face_un[3];      /* face_normal_velocity */
  std::vector<double> deltax[3];
  /* material fields */
  MatField density, density_n, density_0, pressure, pressure_n, pseudo, pseudo_n, pseudo_nm1,
      mass_fraction, cell_mass, internal_energy, internal_energy_n, dpde, fracvol,
      cell_volume, cell_volume_n, tau_density, sound_speed;
  /* the temperature the EOS services advance and its previous value
   * (m_temperature, m_temperature_n), carried in Lagrangian runs */
  MatField temperature, temperature_n;
  bool carries_temperature() const { return !P.with_projection && !P.sans_lagrange; }
  std::vector<uint8_t> envmask, nenvc;
  /* remap */
  int nvars = 4;
  std::vector<double> u_lag, phi_lag, grad_phi, grad_phi_face, phi_face, dual_phi_flux;
  std::vector<double> u_dual, phi_dual, dual_grad;
  std::vector<double> back_flux, front_flux;
  std::vector<double> h_cell;          /* m_h_cell_lagrange of the current direction */
  std::vector<double> delta_ar, delta_av; /* pente-borne fluxes through the back / front faces */
  std::vector<int> est_mixte, est_pure; /* EstMixte / EstPure (Arcane default 0) */
  int sens_projection = 0;
  /* emulation of a protection/reprise restart (test pinning only): after
   * iteration restart_at the reference projects only 3*nb_env+5 variables
   * (MahycoModule.cc:288), which leaves the pseudo-viscosity unprojected */
  long restart_at = 0;
  int nproj() const { return (restart_at > 0 && iteration > restart_at) ? 3 * nenv : nvars; }
  /* time */
  double t = 0.0, dt = 0.0, old_dt = 0.0, m_old_deltat = 0.0;
  long iteration = 0;
  int status = ST_OK;
  bool stop = false;
  std::vector<THLine> th;

  /* EXTERNAL initial state given per cell (the dataset's <initialisation>
   * block); empty: environment 0 and its initial state everywhere */
  std::vector<double> init_mat, init_rho, init_p;
  /* the k-th cell of the reference's numbering (mesh_cell_order) */
  std::vector<long> order;
  long ord(long k) const { return order.empty() ? k : order[k]; }
  long cid(int i, int j, int k) const { return i + (long)ncx * (j + (long)ncy * k); }
  long nid(int i, int j, int k) const { return i + (long)nnx * (j + (long)nny * k); }
  void cijk(long c, int& i, int& j, int& k) const {
    i = (int)(c % ncx); long r = c / ncx; j = (int)(r % ncy); k = (int)(r / ncy);
  }
  void nijk(long n, int& i, int& j, int& k) const {
    i = (int)(n % nnx); long r = n / nnx; j = (int)(r % nny); k = (int)(r / nny);
  }
  bool pure(long c) const { return nenvc[c] == 1; }
  bool has(long c, int e) const { return (envmask[c] >> e) & 1; }
  double& EV(MatField& f, int e, long c) { return pure(c) ? f.g[c] : f.e[e][c]; }

  /* local node l of cell c */
  long cnode(long c, int l) const {
    int i, j, k;
    cijk(c, i, j, k);
    static const int off[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
    return nid(i + off[l][0], j + off[l][1], k + off[l][2]);
  }
  /* face index inside direction d */
  long fid(int d, int i, int j, int k) const {
    if (d == 0) return i + (long)(ncx + 1) * (j + (long)ncy * k);
    if (d == 1) return i + (long)ncx * (j + (long)(ncy + 1) * k);
    return i + (long)ncx * (j + (long)ncy * k);
  }
  void fijk(int d, long f, int& i, int& j, int& k) const {
    int ex = ncx + (d == 0), ey = ncy + (d == 1);
    i = (int)(f % ex); long r = f / ex; j = (int)(r % ey); k = (int)(r / ey);
  }
  /* re-ordered face nodes (smallest uid first, then the smaller neighbour) */
  int face_nodes(int d, int i, int j, int k, long* n) const {
    if (dim == 2) {
      if (d == 0) { n[0] = nid(i, j, 0); n[1] = nid(i, j + 1, 0); }
      else { n[0] = nid(i, j, 0); n[1] = nid(i + 1, j, 0); }
      return 2;
    }
    if (d == 0) { n[0] = nid(i,j,k); n[1] = nid(i,j+1,k); n[2] = nid(i,j+1,k+1); n[3] = nid(i,j,k+1); }
    else if (d == 1) { n[0] = nid(i,j,k); n[1] = nid(i+1,j,k); n[2] = nid(i+1,j,k+1); n[3] = nid(i,j,k+1); }
    else { n[0] = nid(i,j,k); n[1] = nid(i+1,j,k); n[2] = nid(i+1,j+1,k); n[3] = nid(i,j+1,k); }
    return 4;
  }
  /* local face l of cell (i,j,k): direction and face index (Hexa8 / Quad4 order) */
  void cell_face(int i, int j, int k, int l, int& d, long& f) const {
    if (dim == 3) {
      switch (l) {
        case 0: d = 2; f = fid(2, i, j, k); break;
        case 1: d = 0; f = fid(0, i, j, k); break;
        case 2: d = 1; f = fid(1, i, j, k); break;
        case 3: d = 2; f = fid(2, i, j, k + 1); break;
        case 4: d = 0; f = fid(0, i + 1, j, k); break;
        default: d = 1; f = fid(1, i, j + 1, k); break;
      }
    } else {
      switch (l) {
        case 0: d = 1; f = fid(1, i, j, 0); break;
        case 1: d = 0; f = fid(0, i + 1, j, 0); break;
        case 2: d = 1; f = fid(1, i, j + 1, 0); break;
        default: d = 0; f = fid(0, i, j, 0); break;
      }
    }
  }
  int ncd(int d) const { return d == 0 ? ncx : (d == 1 ? ncy : ncz); }
};

/* ---------------------------------------------------------------------------
 * geometry helpers
 * ------------------------------------------------------------------------- */

/* MahycoModule::computeCQs (MahycoModule.cc:1869-1932) */
static void compute_cqs3(const R3* node_coord, const R3* face_coord, R3* out) {
  const R3 c0 = face_coord[0], c1 = face_coord[1], c2 = face_coord[2];
  const R3 c3 = face_coord[3], c4 = face_coord[4], c5 = face_coord[5];
  const R3 n1a04 = 0.5 * vecmul(node_coord[0] - c0, node_coord[3] - c0);
  const R3 n1a03 = 0.5 * vecmul(node_coord[3] - c0, node_coord[2] - c0);
  const R3 n1a02 = 0.5 * vecmul(node_coord[2] - c0, node_coord[1] - c0);
  const R3 n1a01 = 0.5 * vecmul(node_coord[1] - c0, node_coord[0] - c0);
  const R3 n2a05 = 0.5 * vecmul(node_coord[0] - c1, node_coord[4] - c1);
  const R3 n2a12 = 0.5 * vecmul(node_coord[4] - c1, node_coord[7] - c1);
  const R3 n2a08 = 0.5 * vecmul(node_coord[7] - c1, node_coord[3] - c1);
  const R3 n2a04 = 0.5 * vecmul(node_coord[3] - c1, node_coord[0] - c1);
  const R3 n3a01 = 0.5 * vecmul(node_coord[0] - c2, node_coord[1] - c2);
  const R3 n3a06 = 0.5 * vecmul(node_coord[1] - c2, node_coord[5] - c2);
  const R3 n3a09 = 0.5 * vecmul(node_coord[5] - c2, node_coord[4] - c2);
  const R3 n3a05 = 0.5 * vecmul(node_coord[4] - c2, node_coord[0] - c2);
  const R3 n4a09 = 0.5 * vecmul(node_coord[4] - c3, node_coord[5] - c3);
  const R3 n4a10 = 0.5 * vecmul(node_coord[5] - c3, node_coord[6] - c3);
  const R3 n4a11 = 0.5 * vecmul(node_coord[6] - c3, node_coord[7] - c3);
  const R3 n4a12 = 0.5 * vecmul(node_coord[7] - c3, node_coord[4] - c3);
  const R3 n5a02 = 0.5 * vecmul(node_coord[1] - c4, node_coord[2] - c4);
  const R3 n5a07 = 0.5 * vecmul(node_coord[2] - c4, node_coord[6] - c4);
  const R3 n5a10 = 0.5 * vecmul(node_coord[6] - c4, node_coord[5] - c4);
  const R3 n5a06 = 0.5 * vecmul(node_coord[5] - c4, node_coord[1] - c4);
  const R3 n6a03 = 0.5 * vecmul(node_coord[2] - c5, node_coord[3] - c5);
  const R3 n6a08 = 0.5 * vecmul(node_coord[3] - c5, node_coord[7] - c5);
  const R3 n6a11 = 0.5 * vecmul(node_coord[7] - c5, node_coord[6] - c5);
  const R3 n6a07 = 0.5 * vecmul(node_coord[6] - c5, node_coord[2] - c5);
  const double t = 1. / 12.;
  out[0] = (5. * (n1a01 + n1a04 + n2a04 + n2a05 + n3a05 + n3a01) + (n1a02 + n1a03 + n2a08 + n2a12 + n3a06 + n3a09)) * t;
  out[1] = (5. * (n1a01 + n1a02 + n3a01 + n3a06 + n5a06 + n5a02) + (n1a04 + n1a03 + n3a09 + n3a05 + n5a10 + n5a07)) * t;
  out[2] = (5. * (n1a02 + n1a03 + n5a07 + n5a02 + n6a07 + n6a03) + (n1a01 + n1a04 + n5a06 + n5a10 + n6a11 + n6a08)) * t;
  out[3] = (5. * (n1a03 + n1a04 + n2a08 + n2a04 + n6a08 + n6a03) + (n1a01 + n1a02 + n2a05 + n2a12 + n6a07 + n6a11)) * t;
  out[4] = (5. * (n2a05 + n2a12 + n3a05 + n3a09 + n4a09 + n4a12) + (n2a08 + n2a04 + n3a01 + n3a06 + n4a10 + n4a11)) * t;
  out[5] = (5. * (n3a06 + n3a09 + n4a09 + n4a10 + n5a10 + n5a06) + (n3a01 + n3a05 + n4a12 + n4a11 + n5a07 + n5a02)) * t;
  out[6] = (5. * (n4a11 + n4a10 + n5a10 + n5a07 + n6a07 + n6a11) + (n4a12 + n4a09 + n5a06 + n5a02 + n6a03 + n6a08)) * t;
  out[7] = (5. * (n2a08 + n2a12 + n4a12 + n4a11 + n6a11 + n6a08) + (n2a04 + n2a05 + n4a09 + n4a10 + n6a07 + n6a03)) * t;
}

/* face centres of a hexahedron (MahycoModule.cc:1117-1122) */
static void hex_face_centres(const R3* coord, R3* fc) {
  fc[0] = 0.25 * (coord[0] + coord[3] + coord[2] + coord[1]);
  fc[1] = 0.25 * (coord[0] + coord[4] + coord[7] + coord[3]);
  fc[2] = 0.25 * (coord[0] + coord[1] + coord[5] + coord[4]);
  fc[3] = 0.25 * (coord[4] + coord[5] + coord[6] + coord[7]);
  fc[4] = 0.25 * (coord[1] + coord[2] + coord[6] + coord[5]);
  fc[5] = 0.25 * (coord[2] + coord[3] + coord[7] + coord[6]);
}

/* 2D corner normals (MahycoModule.cc:1128-1146) */
static void compute_cqs2(const R3* c4, R3* out) {
  R3 coord[5] = {c4[0], c4[1], c4[2], c4[3], c4[0]};
  R3 npc[5] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int n = 0; n < 4; ++n) {
    npc[n + 1].x = 0.5 * (coord[n + 1].y - coord[n].y);
    npc[n + 1].y = 0.5 * (coord[n].x - coord[n + 1].x);
  }
  npc[0] = npc[4];
  for (int ii = 0; ii < 4; ++ii) out[ii] = npc[ii + 1] + npc[ii];
}

/* ---------------------------------------------------------------------------
 * equation-of-state services
 * ------------------------------------------------------------------------- */

/* pressure of the Mie-Gruneisen law for a given density
 * (MieGruneisenEOSService.cc:55-64 and the two finite-difference copies) */
static bool g_cr_pow = false;
static inline double ipow2(double x) { return g_cr_pow ? x * x : std::pow(x, 2); }
static inline double ipow3(double x) { return g_cr_pow ? cube_cr(x) : std::pow(x, 3); }

static double mg_pressure(const mhc_env_params& o, double density, double e) {
  double J = o.rho0 / density;
  double mu = 1. / J - 1.;
  if (g_cr_pow) {
    if (mu > 0.) {
      double num = o.rho0 * ipow2(o.c0) * mu * (1 + (1. - o.gamma0 / 2.) * mu - o.a * ipow2(mu) / 2.);
      double den = ipow2((1. - (o.s1 - 1.) * mu - o.s2 * ipow2(mu) / (1 + mu) - o.s2 * ipow3(mu) / ipow2(1. + mu)));
      return num / den + (o.gamma0 + o.a * mu) * e;
    }
    return o.rho0 * ipow2(o.c0) * mu + (o.gamma0 + o.a * mu) * e;
  }
  if (mu > 0.) {
    double num = o.rho0 * std::pow(o.c0, 2) * mu * (1 + (1. - o.gamma0 / 2.) * mu - o.a * std::pow(mu, 2) / 2.);
    double den = std::pow((1. - (o.s1 - 1.) * mu - o.s2 * std::pow(mu, 2) / (1 + mu) - o.s2 * std::pow(mu, 3) / std::pow(1. + mu, 2)), 2);
    return num / den + (o.gamma0 + o.a * mu) * e;
  }
  return o.rho0 * std::pow(o.c0, 2) * mu + (o.gamma0 + o.a * mu) * e;
}

/* IEquationOfState::initEOS for one environment */
static void eos_init(Case& C, int env) {
  const mhc_env_params& o = C.P.env[env];
  for (long c = 0; c < C.ncell; ++c) {
    if (!C.has(c, env)) continue;
    double p = C.EV(C.pressure, env, c), rho = C.EV(C.density, env, c);
    if (o.eos == MHC_EOS_PERFECT_GAS) {
      /* PerfectGasEOSService.cc:12-35 */
      double g = o.adiabatic_cst;
      C.EV(C.internal_energy, env, c) = p / ((g - 1.) * rho);
      C.EV(C.sound_speed, env, c) = std::sqrt(g * p / rho);
    } else if (o.eos == MHC_EOS_STIFFENED_GAS) {
      /* StiffenedGasEOSService.cc:14-33 */
      double g = o.adiabatic_cst, pinf = o.limit_tension;
      C.EV(C.internal_energy, env, c) = (p + (g * pinf)) / ((g - 1.) * rho);
      C.EV(C.sound_speed, env, c) = std::sqrt((g / rho) * (p + pinf));
    } else if (o.eos == MHC_EOS_FICTIF) {
      /* FictifEOSService.cc:12-34 (the temperature is not carried) */
      double g = o.adiabatic_cst;
      C.EV(C.internal_energy, env, c) = p / ((g - 1.) * rho);
      C.EV(C.sound_speed, env, c) = std::sqrt(g * p / rho);
    } else {
      /* MieGruneisenEOSService.cc:12-34 */
      C.EV(C.internal_energy, env, c) = C.EV(C.pressure, env, c) / o.gamma0;
      C.EV(C.sound_speed, env, c) = o.c0;
    }
    C.EV(C.density_0, env, c) = C.EV(C.density, env, c);
    /* the temperature of PerfectGas and StiffenedGas (line 30 of both):
     * the air constant 287 */
    if (C.carries_temperature() && (o.eos == MHC_EOS_PERFECT_GAS || o.eos == MHC_EOS_STIFFENED_GAS))
      C.EV(C.temperature, env, c) = p / (287. * rho);
  }
  if (C.carries_temperature() && o.eos == MHC_EOS_MIE_GRUNEISEN) {
    /* MieGruneisenEOSService.cc:17, 29-30: an energie-ref of 0 takes the
     * first nonzero energy of the environment's cells, in cell order */
    double eref = o.energie_ref;
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      if (!C.has(c, env)) continue;
      const double e = C.EV(C.internal_energy, env, c);
      if (eref == 0) eref = e;
      C.EV(C.temperature, env, c) = (e - eref) / o.specific_heat + o.temperature_ref;
    }
  }
}

/* the temperature update of applyEOS (PerfectGas 62-64, StiffenedGas
 * 58-60, MieGruneisen 67-69) and of the PerfectGas / StiffenedGas
 * applyOneCellEOS: the previous value kept, the energy gained since the
 * start of the iteration over cv added to it; Mie-Gruneisen's
 * applyOneCellEOS (121-122) adds it to the kept value instead */
static void advance_temperature(Case& C, const mhc_env_params& o, int env, long c, double e, bool keep) {
  double& T = C.EV(C.temperature, env, c);
  double& Tn = C.EV(C.temperature_n, env, c);
  if (keep) Tn = T;
  T = (e - C.EV(C.internal_energy_n, env, c)) / o.specific_heat + Tn;
}

/* IEquationOfState::applyEOS for one environment (PG 45-67, SG 43-63, MG 44-97).
 * Damage (m_maille_endo) never triggers with the threshold defaults, and the
 * temperature update has no hydro feedback; neither is carried. */
static void eos_apply(Case& C, int env, bool temperature = true) {
  const mhc_env_params& o = C.P.env[env];
  for (long c = 0; c < C.ncell; ++c) {
    if (!C.has(c, env)) continue;
    double e = C.EV(C.internal_energy, env, c);
    double rho = C.EV(C.density, env, c);
    if (o.eos == MHC_EOS_PERFECT_GAS) {
      double g = o.adiabatic_cst;
      double p = (g - 1.) * rho * e;
      C.EV(C.pressure, env, c) = p;
      C.EV(C.sound_speed, env, c) = std::sqrt(g * p / rho);
      C.EV(C.dpde, env, c) = (g - 1.) * rho;
    } else if (o.eos == MHC_EOS_STIFFENED_GAS) {
      double g = o.adiabatic_cst, pinf = o.limit_tension;
      double p = ((g - 1.) * rho * e) - (g * pinf);
      C.EV(C.pressure, env, c) = p;
      C.EV(C.sound_speed, env, c) = std::sqrt((g / rho) * (p + pinf));
      C.EV(C.dpde, env, c) = (g - 1.) * rho;
    } else if (o.eos == MHC_EOS_FICTIF) {
      /* FictifEOSService.cc:44-78: the pressure a function of the time
       * only, the internal energy reset to zero */
      double g = o.adiabatic_cst;
      if (C.t > o.fictif_tdebut) C.EV(C.pressure, env, c) = o.fictif_p0 + o.fictif_dpdt * C.t;
      if (C.t > o.fictif_tfin) C.EV(C.pressure, env, c) = 0.;
      C.EV(C.sound_speed, env, c) = 1.;
      C.EV(C.dpde, env, c) = (g - 1.) * rho;
      C.EV(C.internal_energy, env, c) = 0.;
    } else {
      double J = o.rho0 / rho;
      double mu = 1. / J - 1.;
      C.EV(C.pressure, env, c) = mg_pressure(o, rho, e);
      C.EV(C.dpde, env, c) = (o.gamma0 + o.a * mu);
      double e_now = C.EV(C.internal_energy, env, c);
      double p1 = mg_pressure(o, rho - 1.e-7, e_now);
      double p2 = mg_pressure(o, rho + 1.e-7, e_now);
      if ((p2 - p1) > 0.) C.EV(C.sound_speed, env, c) = std::sqrt((p2 - p1) / 2.e-7);
      else C.EV(C.sound_speed, env, c) = 1.e4;
    }
    if (temperature && C.carries_temperature() && o.eos != MHC_EOS_FICTIF)
      advance_temperature(C, o, env, c, C.EV(C.internal_energy, env, c), true);
  }
}

/* applyOneCellEOS (PerfectGas 71-88, StiffenedGas 67-83, MieGruneisen
 * 101-146): pressure and dp/de of one environment cell; the sound speed and
 * temperature it also writes are not read by the Newton loop */
static void eos_one_cell(const mhc_env_params& o, double rho, double e, double& p, double& dpde) {
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

/* fvnr / fvnrderiv (MahycoModule.h:378-386): residual of the energy
 * equation and its derivative */
static inline double fvnr(double e, double p, double en, double qnn1, double pn, double rn1, double rn) {
  return e - en + 0.5 * (p + pn + 2. * qnn1) * (1. / rn1 - 1. / rn);
}
static inline double fvnrderiv(double dpde, double rn1, double rn) { return 1. + 0.5 * dpde * (1. / rn1 - 1. / rn); }

/* ---------------------------------------------------------------------------
 * init entry points
 * ------------------------------------------------------------------------- */

static void gather_cell_coords(Case& C, long c, R3* out) {
  for (int l = 0; l < C.nbn; ++l) out[l] = C.coord[C.cnode(c, l)];
}

/* MahycoModule::computeGeometricValues (MahycoModule.cc:1097-1253) */
static int compute_geometric_values(Case& C) {
  const double racine = C.dim == 2 ? .5 : 1. / 3.;
  for (long c = 0; c < C.ncell; ++c) {
    R3 coord[8];
    gather_cell_coords(C, c, coord);
    if (C.dim == 3) {
      R3 fc[6];
      hex_face_centres(coord, fc);
      compute_cqs3(coord, fc, &C.cqs[c * 8]);
    } else {
      compute_cqs2(coord, &C.cqs[c * 4]);
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    double volume = 0.;
    for (int n = 0; n < C.nbn; ++n) volume += dot(C.coord[C.cnode(c, n)], C.cqs[c * C.nbn + n]);
    volume /= C.dim;
    C.cell_volume.g[c] = volume;
    if (volume < 0.) { C.status = ST_NEG_VOLUME; return C.status; }
    int lc = C.P.longueur_caracteristique;
    if (lc == MHC_LENGTH_CUBE_ROOT_VOLUME) {
      if (g_cr_pow) C.char_len[c] = C.dim == 2 ? std::sqrt(C.cell_volume.g[c]) : pow_third_cr(C.cell_volume.g[c]);
      else C.char_len[c] = std::pow(C.cell_volume.g[c], racine);
    } else if (lc == MHC_LENGTH_OPPOSITE_FACES) {
      R3 coord[8], fc[6];
      gather_cell_coords(C, c, coord);
      hex_face_centres(coord, fc);
      double d1 = norm(fc[0] - fc[3]), d2 = norm(fc[2] - fc[5]), d3 = norm(fc[1] - fc[4]);
      C.char_len[c] = (d1 * d2 * d3) / (d1 * d2 + d1 * d3 + d2 * d3);
    } else {
      int d = lc - MHC_LENGTH_MONODIM_X;
      double a = comp(C.coord[C.cnode(c, 0)], d), b = comp(C.coord[C.cnode(c, 2)], d);
      C.char_len[c] = std::fabs(b - a);
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c)) continue;
    for (int e = 0; e < C.nenv; ++e)
      if (C.has(c, e)) C.EV(C.cell_volume, e, c) = C.EV(C.fracvol, e, c) * C.cell_volume.g[c];
  }
  return ST_OK;
}

static void cell_centres(Case& C) {
  const double w = C.dim == 2 ? .25 : .125;
  for (long c = 0; c < C.ncell; ++c) {
    R3 s = {0., 0., 0.};
    for (int l = 0; l < C.nbn; ++l) s += C.coord[C.cnode(c, l)];
    C.cell_coord[c] = w * s;
  }
}

/* CHOCBULLEService::initMat / initVar, the bubble lattice
 * (src/casTest/CHOCBULLE/CHOCBULLEService.cc:22-95, 200-290): material of
 * cell c (0 medium, 1 bubble, 0.5 mixed) and the bubble's volume fraction of
 * a mixed cell.  Bubbles in x, y, z order, later ones overriding; distances
 * in the (x, y) plane.  The node distances that decide a mixed cell are
 * taken from the bubble's centre and per cell (the reference measures them
 * from the origin and keeps the extremes across cells, which only agrees
 * for a bubble at the origin). */
/* RIDERService (casTest/RIDER/RIDERService.cc): centre of the disc
 * (Xb, lines 27-30 and 76-79), node-distance range of a cell to it
 * (rmin / rmax, lines 36-45), and the velocity field of the test (lines
 * 141-172 and 255-285).  Pi is TypesMahyco.h:42's 3.14159265359. */
static const double kPi = 3.14159265359;
static bool rider_mono(const mhc_case_params& P) { return P.cas_test >= 23 && P.cas_test <= 30; }
static R3 rider_centre(const mhc_case_params& P) {
  const int first_rotation = rider_mono(P) ? 26 : 34;
  return P.cas_test < first_rotation ? R3{0.20, 0.20, 0.} : R3{0.50, 0.75, 0.};
}
static void rider_range(const Case& C, long c, R3 xb, double& rmin, double& rmax) {
  rmin = 10.;
  rmax = 0.;
  for (int l = 0; l < C.nbn; ++l) {
    const R3 x = C.coord[C.cnode(c, l)];
    const double rn = std::sqrt((x.x - xb.x) * (x.x - xb.x) + (x.y - xb.y) * (x.y - xb.y));
    rmin = std::min(rmin, rn);
    rmax = std::max(rmax, rn);
  }
}
static R3 rider_velocity(const mhc_case_params& P, R3 x) {
  const int kind = (P.cas_test - 23) % 8;  /* Tx Ty T45 Rotation Vortex Deformation VortexR DeformationR */
  const R3 cc = {0.5, 0.5, 0.};
  R3 v = {0.0, 0.0, 0.0};
  if (kind == 0) v.x = 1.;
  if (kind == 1) v.y = 1.;
  if (kind == 2) v = {1.0, 1.0, 0.0};
  if (kind == 3) {
    const R3 dd = x - cc;
    const double theta = std::atan2(dd.y, dd.x);
    const double r = std::sqrt(dd.x * dd.x + dd.y * dd.y);
    const double omega = 4. * kPi;
    v.x = -r * omega * std::sin(omega * 0. + theta);
    v.y = r * omega * std::cos(omega * 0. + theta);
  }
  if (kind == 4 || kind == 6) {
    const R3 dd = x;
    v.x = -2. * std::cos(kPi * dd.y) * std::sin(kPi * dd.y) * std::sin(kPi * dd.x) * std::sin(kPi * dd.x);
    v.y = 2. * std::cos(kPi * dd.x) * std::sin(kPi * dd.x) * std::sin(kPi * dd.y) * std::sin(kPi * dd.y);
  }
  if (kind == 5 || kind == 7) {
    const R3 dd = x + cc;
    v.x = std::sin(4. * kPi * dd.x) * std::sin(4. * kPi * dd.y);
    v.y = std::cos(4. * kPi * dd.x) * std::cos(4. * kPi * dd.y);
  }
  return v;
}

static double bubble_material(const Case& C, long c, double& fbub) {
  const mhc_case_params& P = C.P;
  double mat = 0.;
  fbub = 0.;
  const int nz = C.dim == 3 ? P.bubbles_n[2] : 1;
  for (int bx = 0; bx < P.bubbles_n[0]; ++bx)
    for (int by = 0; by < P.bubbles_n[1]; ++by)
      for (int bz = 0; bz < nz; ++bz) {
        const double xb = P.bubbles_first[0] + bx * P.bubbles_delta[0];
        const double yb = P.bubbles_first[1] + by * P.bubbles_delta[1];
        const double rb = P.bubbles_radius;
        const double x = C.cell_coord[c].x - xb, y = C.cell_coord[c].y - yb;
        if (!(std::sqrt(x * x + y * y) <= rb)) continue;
        mat = 1.;
        fbub = 0.;
        double rmin = 1.e300, rmax = 0.;
        for (int l = 0; l < C.nbn; ++l) {
          const R3& xn = C.coord[C.cnode(c, l)];
          const double dx = xn.x - xb, dy = xn.y - yb;
          const double rn = std::sqrt(dx * dx + dy * dy);
          rmin = (rn < rmin) ? rn : rmin;
          rmax = (rmax < rn) ? rn : rmax;
        }
        if (rmin < rb && rmax > rb) {
          mat = 0.5;
          fbub = (rb - rmin) / (rmax - rmin);
        }
      }
  return mat;
}

/* the regions of POINTTRIPLEService (POINTTRIPLEService.cc:26-36, 49-58) */
static int triple_point_region(const R3& cc) {
  if (cc.x <= 0.01) return 0;
  if (cc.y <= 0.015) return 1;
  return 2;
}

/* SODService::initMat / SEDOVService::initMat and the environment sort of
 * MahycoModule::hydroStartInitEnvAndMat (MahycoAnnexe.cc:86-139) */
static void init_materials(Case& C) {
  const mhc_case_params& P = C.P;
  for (long c = 0; c < C.ncell; ++c) {
    double m = 0.;
    if (P.cas_model == MHC_CASE_SOD) {
      if (P.cas_test == MHC_TEST_BISOD_X || P.cas_test == MHC_TEST_BISOD_Y || P.cas_test == MHC_TEST_BISOD_Z) {
        double r = comp(C.cell_coord[c], P.cas_test - MHC_TEST_BISOD_X);
        m = (r < 0.5) ? 0. : 1.;
      } else if (P.cas_test == MHC_TEST_BISOD_SPH) {
        /* SODService.cc:56-62 */
        const R3& x = C.cell_coord[c];
        m = (std::sqrt(x.x * x.x + x.y * x.y + x.z * x.z) < 0.5) ? 0. : 1.;
      }
    } else if (P.cas_model == MHC_CASE_ONECELL) {
      m = 0.;  /* ONECELLService::initMat */
    } else if (P.cas_model == MHC_CASE_TRIPLE_POINT) {
      /* POINTTRIPLEService::initMat (POINTTRIPLEService.cc:42-60); initMatMono
       * puts every cell in environment 0 */
      if (P.cas_test != MHC_TEST_MONO_TRIPLE_POINT) m = triple_point_region(C.cell_coord[c]);
    } else if (P.cas_model == MHC_CASE_TWO_STATE) {
      if (C.nenv > 1) {
        double r = comp(C.cell_coord[c], P.interface_dir);
        m = (r < P.interface_pos) ? 0. : 1.;
      }
    } else if (P.cas_model == MHC_CASE_SEDOV && P.cas_test != MHC_TEST_SEDOV) {
      bool center = false;
      for (int l = 0; l < C.nbn; ++l) {
        R3 x = C.coord[C.cnode(c, l)];
        if (std::sqrt(x.x * x.x + x.y * x.y + x.z * x.z) < 1.e-10) center = true;
      }
      m = center ? 1. : 0.;
    } else if (P.cas_model == MHC_CASE_BUBBLES && C.nenv > 1) {
      double f;
      m = bubble_material(C, c, f);
    } else if (P.cas_model == MHC_CASE_EXTERNAL) {
      m = C.init_mat.empty() ? 0. : C.init_mat[c];
    } else if (P.cas_model == MHC_CASE_RIDER && !rider_mono(P)) {
      /* RIDERService::initMat (RIDERService.cc:18-57); MonoRider*: initMatMono */
      double rmin, rmax;
      rider_range(C, c, rider_centre(P), rmin, rmax);
      const double rb = P.rider_radius;
      m = 0;
      if (rmax < rb) m = 1;
      else if ((rmax >= rb) && (rmin < rb)) m = (rb - rmin) / (rmax - rmin);
    }
    C.materiau[c] = m;
    uint8_t mask = 0;
    if (m == 0.) mask = 1;
    else if (m > 0. && m < 1.) mask = 3;
    else if (m == 1.) mask = 2;
    else if (m > 1. && m < 2.) mask = 6;
    else if (m == 2.) mask = 4;
    else if (m > 2. && m < 3.) mask = 12;
    else if (m == 3.) mask = 8;
    else mask = 15;
    mask &= (uint8_t)((1 << C.nenv) - 1);
    C.envmask[c] = mask;
    C.nenvc[c] = (uint8_t)__builtin_popcount(mask);
  }
}

/* SODService::initVar(Mono), SEDOVService::initVar(Mono) and the seeded
 * two-state variant (same structure as BiSod with explicit states) */
static void init_variables(Case& C) {
  const mhc_case_params& P = C.P;
  if (P.cas_model == MHC_CASE_SOD) {
    bool mono = P.cas_test == MHC_TEST_SOD_X || P.cas_test == MHC_TEST_SOD_Y || P.cas_test == MHC_TEST_SOD_Z;
    for (long c = 0; c < C.ncell; ++c) {
      if (mono) {
        double r = comp(C.cell_coord[c], P.cas_test - MHC_TEST_SOD_X);
        double p, rho;
        if (r < 0.5) { p = P.env[0].pression_initiale; rho = P.env[0].densite_initiale; }
        else { p = P.env[0].pression_initiale / 10.; rho = P.env[0].densite_initiale / 8.; }
        C.density.g[c] = rho;
        C.pressure.g[c] = p;
      } else {
        int s = (C.materiau[c] == 0) ? 0 : 1;
        C.density.g[c] = P.env[s].densite_initiale;
        C.pressure.g[c] = P.env[s].pression_initiale;
        if (!C.pure(c))
          for (int e = 0; e < C.nenv; ++e)
            if (C.has(c, e)) { C.EV(C.density, e, c) = P.env[s].densite_initiale; C.EV(C.pressure, e, c) = P.env[s].pression_initiale; }
      }
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {P.env[0].vitesse_initiale[0], P.env[0].vitesse_initiale[1], P.env[0].vitesse_initiale[2]};
  } else if (P.cas_model == MHC_CASE_TRIPLE_POINT) {
    /* POINTTRIPLEService::initVar / initVarMono (POINTTRIPLEService.cc:14-41,
     * 62-141): the region's initial state, every node at environment 0's
     * velocity; the cells are pure, so the per-environment branch of initVar
     * never runs */
    for (long c = 0; c < C.ncell; ++c) {
      const int s = triple_point_region(C.cell_coord[c]);
      C.density.g[c] = P.env[s].densite_initiale;
      C.pressure.g[c] = P.env[s].pression_initiale;
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {P.env[0].vitesse_initiale[0], P.env[0].vitesse_initiale[1], P.env[0].vitesse_initiale[2]};
  } else if (P.cas_model == MHC_CASE_TWO_STATE) {
    for (long c = 0; c < C.ncell; ++c) {
      double r = comp(C.cell_coord[c], P.interface_dir);
      int s = (r < P.interface_pos) ? 0 : 1;
      C.density.g[c] = P.env[s].densite_initiale;
      C.pressure.g[c] = P.env[s].pression_initiale;
    }
    // every node starts at the velocity of the first environment (zero in
    // the shock tubes, the impact velocity of a projectile)
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {P.env[0].vitesse_initiale[0], P.env[0].vitesse_initiale[1], P.env[0].vitesse_initiale[2]};
  } else if (P.cas_model == MHC_CASE_BUBBLES) {
    /* pure cells: their environment's initial state; mixed cells: both
     * environments' states, volume fractions (1 - f, f), mass fractions
     * f rho / sum of f rho; the cell values are summed from them at the end
     * of the initialisation */
    for (long c = 0; c < C.ncell; ++c) {
      double f;
      const double m = bubble_material(C, c, f);
      const int s = m == 1. ? 1 : 0;
      C.density.g[c] = P.env[s].densite_initiale;
      C.pressure.g[c] = P.env[s].pression_initiale;
      if (!C.pure(c)) {
        C.density.g[c] = C.pressure.g[c] = 0.;
        C.EV(C.fracvol, 0, c) = 1. - f;
        C.EV(C.fracvol, 1, c) = f;
        double rm = 0.;
        for (int e = 0; e < 2; ++e) {
          C.EV(C.density, e, c) = P.env[e].densite_initiale;
          C.EV(C.pressure, e, c) = P.env[e].pression_initiale;
          rm += C.EV(C.density, e, c) * C.EV(C.fracvol, e, c);
        }
        for (int e = 0; e < 2; ++e)
          C.EV(C.mass_fraction, e, c) = (C.EV(C.density, e, c) * C.EV(C.fracvol, e, c)) / rm;
      }
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {P.env[0].vitesse_initiale[0], P.env[0].vitesse_initiale[1], P.env[0].vitesse_initiale[2]};
  } else if (P.cas_model == MHC_CASE_EXTERNAL) {
    /* the dataset's <initialisation> values, then EXTERNALService::initUtilisateur
     * (EXTERNALService.cc:25-40) for every environment that asks for it
     * (MahycoModule.cc:132-139): its initial velocity, or -x/|x| when that
     * is zero */
    for (long c = 0; c < C.ncell; ++c) {
      C.density.g[c] = C.init_rho.empty() ? P.env[0].densite_initiale : C.init_rho[c];
      C.pressure.g[c] = C.init_p.empty() ? P.env[0].pression_initiale : C.init_p[c];
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {0., 0., 0.};
    for (int e = 0; e < C.nenv; ++e) {
      if (!P.env[e].initialisation_utilisateur) continue;
      const R3 v0 = {P.env[e].vitesse_initiale[0], P.env[e].vitesse_initiale[1], P.env[e].vitesse_initiale[2]};
      const bool zero = v0.x == 0. && v0.y == 0. && v0.z == 0.;
      for (long n = 0; n < C.nnode; ++n) C.vel[n] = zero ? (-C.coord[n]) / norm(C.coord[n]) : v0;
    }
  } else if (P.cas_model == MHC_CASE_RIDER) {
    /* RIDERService::initVar / initVarMono (RIDERService.cc:62-173, 178-289) */
    const bool mono = rider_mono(P), lin = P.rider_linear_density != 0;
    const R3 xb = rider_centre(P);
    const double rb = P.rider_radius;
    const double croissance = lin ? 1. / rb : 1.;
    const double d0 = P.env[0].densite_initiale, d1 = P.env[C.nenv > 1 ? 1 : 0].densite_initiale;
    const double p0 = P.env[0].pression_initiale, p1 = P.env[C.nenv > 1 ? 1 : 0].pression_initiale;
    for (long c = 0; c < C.ncell; ++c) {
      double rmin, rmax;
      rider_range(C, c, xb, rmin, rmax);
      C.density.g[c] = d0;
      C.pressure.g[c] = p0;
      C.internal_energy.g[c] = P.env[0].energie_initiale;
      const R3 cc = C.cell_coord[c];
      const double r = std::sqrt((cc.x - xb.x) * (cc.x - xb.x) + (cc.y - xb.y) * (cc.y - xb.y));
      const double r_cell = lin ? r : rmax;
      if (r_cell < rb) {
        C.density.g[c] = d1;
        if (lin) C.density.g[c] = d1 * std::min(croissance * 2 * (rb - r), 1.);
        C.pressure.g[c] = p1;
      } else if ((rmax >= rb) && (rmin < rb) && !lin) {
        const double frac_b = (rb - rmin) / (rmax - rmin);
        if (!mono) {
          /* the first environment takes the disc's density and fraction */
          for (int e = 0; e < C.nenv; ++e) {
            if (!C.has(c, e)) continue;
            if (e == 0) {
              C.EV(C.density, e, c) = d1;
              C.EV(C.fracvol, e, c) = frac_b;
              C.EV(C.mass_fraction, e, c) = frac_b;
            }
            if (e == 1) {
              C.EV(C.density, e, c) = d0;
              C.EV(C.fracvol, e, c) = 1. - frac_b;
              C.EV(C.mass_fraction, e, c) = 1. - frac_b;
            }
            C.EV(C.pressure, e, c) = 0.;
          }
        }
        C.density.g[c] = frac_b * d1;
        C.pressure.g[c] = p1;
      }
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = rider_velocity(P, C.coord[n]);
    C.vel_n = C.vel;
  } else if (P.cas_model == MHC_CASE_ONECELL) {
    /* ONECELLService::initVarMono: the first environment's state everywhere,
     * nodes at rest */
    for (long c = 0; c < C.ncell; ++c) {
      C.density.g[c] = P.env[0].densite_initiale;
      C.pressure.g[c] = P.env[0].pression_initiale;
      C.internal_energy.g[c] = P.env[0].energie_initiale;
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {0., 0., 0.};
  } else if (P.cas_model == MHC_CASE_SEDOV) {
    double rhoInit = P.env[0].densite_initiale, pInit = P.env[0].pression_initiale;
    bool mono = P.cas_test == MHC_TEST_SEDOV;
    const double e1 = 0.244816e-5;
    for (long c = 0; c < C.ncell; ++c) {
      if (mono) C.internal_energy.g[c] = e1;
      C.density.g[c] = rhoInit;
      C.pressure.g[c] = pInit;
      double vol = C.cell_volume.g[c];
      bool center = false;
      for (int l = 0; l < C.nbn; ++l) {
        R3 x = C.coord[C.cnode(c, l)];
        double rn = C.dim == 3 ? std::sqrt(x.x * x.x + x.y * x.y + x.z * x.z) : std::sqrt(x.x * x.x + x.y * x.y);
        if (rn < 1.e-10) center = true;
      }
      if (center) {
        C.internal_energy.g[c] += P.sedov_energy / vol;
        C.pressure.g[c] = 0.4 * rhoInit * C.internal_energy.g[c];
      }
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] = {0., 0., 0.};
  }
}

/* MahycoModule::InitGeometricValues (MahycoModule.cc:1041-1093) */
static void init_geometric_values(Case& C) {
  C.coord0 = C.coord;
  const double w = C.dim == 2 ? .5 : .25;
  for (int d = 0; d < C.dim; ++d) {
    for (long f = 0; f < C.nface[d]; ++f) {
      int i, j, k;
      C.fijk(d, f, i, j, k);
      long n[4];
      int nb = C.face_nodes(d, i, j, k, n);
      R3 nrm;
      if (C.dim == 3) {
        R3 v1 = C.coord[n[2]] - C.coord[n[0]], v2 = C.coord[n[3]] - C.coord[n[1]];
        nrm.x = produit(v1.y, v2.z, v1.z, v2.y);
        nrm.y = -produit(v2.x, v1.z, v2.z, v1.x);
        nrm.z = produit(v1.x, v2.y, v1.y, v2.x);
      } else {
        nrm.x = (C.coord[n[1]].y - C.coord[n[0]].y);
        nrm.y = (C.coord[n[1]].x - C.coord[n[0]].x);
        nrm.z = 0.;
      }
      C.face_normal[d][f] = nrm / norm(nrm);
      R3 fc = {0., 0., 0.};
      for (int q = 0; q < nb; ++q) fc += w * C.coord[n[q]];
      C.face_coord[d][f] = fc;
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    int i, j, k;
    C.cijk(c, i, j, k);
    for (int l = 0; l < 2 * C.dim; ++l) {
      int d; long f;
      C.cell_face(i, j, k, l, d, f);
      R3 diff = C.face_coord[d][f] - C.cell_coord[c];
      C.outer_normal[c * 2 * C.dim + l] = diff / norm(diff);
    }
  }
}

static void setup(Case& C, const mhc_case_params* p) {
  C.P = *p;
  C.dim = p->dim;
  C.nenv = p->nb_env;
  C.ncx = p->nx; C.ncy = p->ny; C.ncz = (C.dim == 3) ? p->nz : 1;
  C.nnx = C.ncx + 1; C.nny = C.ncy + 1; C.nnz = (C.dim == 3) ? C.ncz + 1 : 1;
  C.ncell = (long)C.ncx * C.ncy * C.ncz;
  C.nnode = (long)C.nnx * C.nny * C.nnz;
  C.nbn = C.dim == 3 ? 8 : 4;
  C.coord.resize(C.nnode);
  double dx = p->lx / p->nx, dy = p->ly / p->ny, dz = (C.dim == 3) ? p->lz / p->nz : 0.;
  for (long n = 0; n < C.nnode; ++n) {
    int i, j, k;
    C.nijk(n, i, j, k);
    C.coord[n] = {p->origin[0] + i * dx, p->origin[1] + j * dy, (C.dim == 3) ? p->origin[2] + k * dz : 0.};
  }
  C.vel.assign(C.nnode, {0, 0, 0});
  C.vel_n = C.vel;
  C.force = C.vel;
  C.node_mass.assign(C.nnode, 0.);
  C.cell_coord.assign(C.ncell, {0, 0, 0});
  C.char_len.assign(C.ncell, 0.);
  C.div_u.assign(C.ncell, 0.);
  C.euler_volume.assign(C.ncell, 0.);
  C.materiau.assign(C.ncell, 0.);
  C.cqs.assign(C.ncell * C.nbn, {0, 0, 0});
  C.cqs_n = C.cqs;
  C.elasto = p->env[0].elasto_model != 0;
  C.sdev.assign(C.elasto ? C.ncell * 6 : 0, 0.);
  C.plastic.assign(C.elasto ? C.ncell : 0, 0.);
  C.plastic_rate.assign(C.elasto ? C.ncell : 0, 0.);
  C.strain_norm.assign(C.elasto ? C.ncell : 0, 0.);
  C.tensF.assign(p->env[0].elasto_model == 2 ? C.ncell * 9 : 0, 0.);
  for (long c = 0; c < (long)C.tensF.size() / 9; ++c) C.tensF[c * 9] = C.tensF[c * 9 + 4] = C.tensF[c * 9 + 8] = 1.;
  C.sdev_n = C.sdev;
  C.hourglass.assign(C.nnode, {0, 0, 0});
  C.outer_normal.assign(C.ncell * 2 * C.dim, {0, 0, 0});
  for (int d = 0; d < C.dim; ++d) {
    long ex = C.ncx + (d == 0), ey = C.ncy + (d == 1), ez = C.ncz + (d == 2);
    if (C.dim == 2) ez = 1;
    C.nface[d] = ex * ey * ez;
    C.face_normal[d].assign(C.nface[d], {0, 0, 0});
    C.face_coord[d].assign(C.nface[d], {0, 0, 0});
    C.face_len[d].assign(C.nface[d], 0.);
    C.face_un[d].assign(C.nface[d], 0.);
    C.deltax[d].assign(C.nface[d], 0.);
  }
  MatField* mf[] = {&C.density, &C.density_n, &C.density_0, &C.pressure, &C.pressure_n, &C.pseudo,
                    &C.pseudo_n, &C.pseudo_nm1, &C.mass_fraction, &C.cell_mass, &C.internal_energy,
                    &C.internal_energy_n, &C.dpde, &C.fracvol, &C.cell_volume, &C.cell_volume_n,
                    &C.tau_density, &C.sound_speed, &C.temperature, &C.temperature_n};
  for (MatField* f : mf) f->init(C.ncell, C.nenv, 0.);
  C.envmask.assign(C.ncell, 1);
  C.nenvc.assign(C.ncell, 1);
  /* elasto-plasticity with the remap: the deviator and plastic strains
   * after the pseudo-viscosity (PrepareRemap.cc:121-128) */
  C.nvars = 3 * C.nenv + 1 + ((C.P.env[0].elasto_model && C.P.with_projection) ? 7 : 0);
  C.u_lag.assign(C.ncell * C.nvars, 0.);
  C.phi_lag = C.u_lag;
  C.grad_phi = C.u_lag;
  C.dual_phi_flux = C.u_lag;
  C.u_dual.assign(C.nnode * 5, 0.);
  C.phi_dual = C.u_dual;
  C.dual_grad = C.u_dual;
  C.back_flux.assign(C.nnode, 0.);
  C.front_flux.assign(C.nnode, 0.);
  C.h_cell.assign(C.ncell, 0.);
  C.delta_ar.assign(C.ncell * C.nvars, 0.);
  C.delta_av.assign(C.ncell * C.nvars, 0.);
  C.est_mixte.assign(C.ncell, 0);
  if (p->mesh_cell_order == 1 && C.dim == 2) {
    C.order.resize(C.ncell);
    long k = 0;
    for (int i = 0; i < C.ncx; ++i)
      for (int j = 0; j < C.ncy; ++j) C.order[k++] = C.cid(i, j, 0);
  }
  C.est_pure.assign(C.ncell, 0);
}

/* MahycoModule::hydroStartInit (MahycoModule.cc:21-210) followed by
 * computeCellMass (221-237) and computeNodeMass (247-262) */
static int hydro_start_init(Case& C) {
  C.dt = C.P.deltat_init;
  C.sens_projection = 0;
  cell_centres(C);                         /* MahycoAnnexe.cc:75-82 */
  init_materials(C);
  if (compute_geometric_values(C) != ST_OK) return C.status;
  C.fracvol.fill(1.0);
  C.mass_fraction.fill(1.0);
  C.pseudo.fill(0.0);
  C.internal_energy_n.fill(0.0);
  init_variables(C);
  /* no equation of state and no mixed-cell averages at the start of a
   * sans-lagrange run (MahycoModule.cc:143-171) */
  if (!C.P.sans_lagrange)
    for (int e = 0; e < C.nenv; ++e) eos_init(C, e);
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c) || C.P.sans_lagrange) continue;
    C.internal_energy.g[c] = 0.;
    for (int e = 0; e < C.nenv; ++e) {
      if (!C.has(c, e)) continue;
      C.internal_energy.g[c] += C.EV(C.internal_energy, e, c) * C.EV(C.mass_fraction, e, c);
      C.sound_speed.g[c] = std::max(C.EV(C.sound_speed, e, c), C.sound_speed.g[c]);
      C.density.g[c] += C.EV(C.density, e, c) * C.EV(C.fracvol, e, c);
      C.pressure.g[c] += C.EV(C.pressure, e, c) * C.EV(C.fracvol, e, c);
    }
  }
  for (long c = 0; c < C.ncell; ++c) C.euler_volume[c] = C.cell_volume.g[c];
  init_geometric_values(C);
  for (long c = 0; c < C.ncell; ++c) {
    double volume = 0.;
    for (int n = 0; n < C.nbn; ++n) volume += dot(C.coord[C.cnode(c, n)], C.cqs[c * C.nbn + n]);
    volume /= C.dim;
    C.cell_volume.g[c] = volume;
  }
  /* computeCellMass */
  for (long c = 0; c < C.ncell; ++c) C.cell_mass.g[c] = C.density.g[c] * C.cell_volume.g[c];
  for (int e = 0; e < C.nenv; ++e)
    for (long c = 0; c < C.ncell; ++c)
      if (C.has(c, e)) C.EV(C.cell_mass, e, c) = C.EV(C.mass_fraction, e, c) * C.cell_mass.g[c];
  /* computeNodeMass */
  std::fill(C.node_mass.begin(), C.node_mass.end(), 0.);
  const double w = C.dim == 2 ? .25 : .125;
  for (long k = 0; k < C.ncell; ++k) {
    const long c = C.ord(k);
    double contrib = w * C.cell_mass.g[c];
    for (int l = 0; l < C.nbn; ++l) C.node_mass[C.cnode(c, l)] += contrib;
  }
  return ST_OK;
}

/* ---------------------------------------------------------------------------
 * compute-loop entry points
 * ------------------------------------------------------------------------- */

/* MahycoModule::saveValuesAtN (MahycoModule.cc:311-382) */
static void save_values_at_n(Case& C) {
  C.old_dt = C.m_old_deltat;
  auto cp = [&](MatField& dst, MatField& src) {
    for (long c = 0; c < C.ncell; ++c) dst.g[c] = src.g[c];
    for (int e = 0; e < C.nenv; ++e)
      for (long c = 0; c < C.ncell; ++c)
        if (C.has(c, e) && !C.pure(c)) dst.e[e][c] = src.e[e][c];
  };
  for (long c = 0; c < C.ncell; ++c) C.pseudo_nm1.g[c] = C.pseudo_n.g[c];
  for (int e = 0; e < C.nenv; ++e)
    for (long c = 0; c < C.ncell; ++c)
      if (C.has(c, e) && !C.pure(c)) C.pseudo_nm1.e[e][c] = C.pseudo_n.e[e][c];
  cp(C.pseudo_n, C.pseudo);
  cp(C.pressure_n, C.pressure);
  cp(C.cell_volume_n, C.cell_volume);
  cp(C.density_n, C.density);
  cp(C.internal_energy_n, C.internal_energy);
  C.cqs_n = C.cqs;
  /* sans-lagrange: the velocities at n stay those of the initialisation */
  if (!C.P.sans_lagrange) C.vel_n = C.vel;
  C.sdev_n = C.sdev;
}

/* MahycoModule::updateVelocityWithoutLagrange (MahycoModule.cc:676-700):
 * the velocities at n, times cos(Pi t parameter) with the reverse option */
static void update_velocity_without_lagrange(Case& C) {
  const double option_real = (double)(C.P.cas_model == MHC_CASE_RIDER && C.P.rider_reverse);
  const double factor = C.P.cas_model == MHC_CASE_RIDER ? C.P.rider_parameter : 0.;
  for (long n = 0; n < C.nnode; ++n) {
    const R3 v = C.vel_n[n];
    const double cs = std::cos(kPi * C.t * factor);
    C.vel[n] = v * (1. - option_real) + option_real * v * cs;
  }
}

/* MahycoModule::updateVelocity (MahycoModule.cc:438-562): pressure forces
 * summed over all cells, then the elasto-plastic forces -S_n.C_n (only
 * with an elasto model: without one they add exact zeros), gravity, and
 * the anti-hourglass correction of a Lagrangian run */
static void update_velocity(Case& C) {
  for (auto& f : C.force) f = {0., 0., 0.};
  for (long k = 0; k < C.ncell; ++k) {
    const long c = C.ord(k);
    double pressure = C.pressure_n.g[c] + C.pseudo_n.g[c];
    for (int l = 0; l < C.nbn; ++l) C.force[C.cnode(c, l)] += pressure * C.cqs_n[c * C.nbn + l];
  }
  if (C.elasto) {
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      const double* S = &C.sdev_n[c * 6];
      /* force_tensor = -S_n; prodTensVec(t, v) = (t.x.v, t.y.v, t.z.v) */
      const R3 tx = {-S[0], -S[3], -S[5]}, ty = {-S[3], -S[1], -S[4]}, tz = {-S[5], -S[4], -S[2]};
      for (int l = 0; l < C.nbn; ++l) {
        const R3 v = C.cqs_n[c * C.nbn + l];
        C.force[C.cnode(c, l)] += R3{dot(tx, v), dot(ty, v), dot(tz, v)};
      }
    }
  }
  R3 g = {C.P.gravity[0], C.P.gravity[1], C.P.gravity[2]};
  if (C.P.schema_csts && C.P.with_projection) {
    /* updateVelocityBackward (MahycoModule.cc:573-627): the velocities after
     * the remap (at n) back to n-1/2 with the same forces, -old_dt/2 */
    const double dtb = -0.5 * C.old_dt;
    for (long n = 0; n < C.nnode; ++n) C.vel[n] += (dtb / C.node_mass[n]) * C.force[n];
    for (long n = 0; n < C.nnode; ++n) C.vel[n] += dtb * g;
  }
  const double dt = 0.5 * (C.old_dt + C.dt);
  for (long n = 0; n < C.nnode; ++n) C.vel[n] += (dt / C.node_mass[n]) * C.force[n];
  for (long n = 0; n < C.nnode; ++n) C.vel[n] += dt * g;
  if (!C.P.with_projection && C.P.coef_antiderive != 0.) {
    /* MahycoModule.cc:497-555 */
    const double coeff = C.P.coef_antiderive;
    for (auto& h : C.hourglass) h = {0., 0., 0.};
    auto nbcell = [&](long n) {
      int i, j, k;
      C.nijk(n, i, j, k);
      int m = ((i > 0 && i < C.nnx - 1) ? 2 : 1) * ((j > 0 && j < C.nny - 1) ? 2 : 1);
      if (C.dim == 3) m *= (k > 0 && k < C.nnz - 1) ? 2 : 1;
      return (double)m;
    };
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      long nd[8];
      R3 v[8];
      for (int l = 0; l < C.nbn; ++l) { nd[l] = C.cnode(c, l); v[l] = C.vel[nd[l]]; }
      if (C.dim == 2) {
        R3 psi = coeff * (v[0] + v[2] - v[1] - v[3]);
        C.hourglass[nd[0]] += 1. / nbcell(nd[0]) * psi;
        C.hourglass[nd[1]] -= 1. / nbcell(nd[1]) * psi;
        C.hourglass[nd[2]] += 1. / nbcell(nd[2]) * psi;
        C.hourglass[nd[3]] -= 1. / nbcell(nd[3]) * psi;
      } else {
        R3 p1 = coeff * (v[0] + v[1] - v[2] - v[3] - v[4] - v[5] + v[6] + v[7]);
        R3 p2 = coeff * (v[0] - v[1] - v[2] + v[3] - v[4] + v[5] + v[6] - v[7]);
        R3 p3 = coeff * (v[0] - v[1] + v[2] - v[3] + v[4] - v[5] + v[6] - v[7]);
        R3 p4 = coeff * (-v[0] + v[1] - v[2] + v[3] + v[4] - v[5] + v[6] - v[7]);
        C.hourglass[nd[0]] += 1. / nbcell(nd[0]) * (p1 + p2 + p3 - p4);
        C.hourglass[nd[1]] += 1. / nbcell(nd[1]) * (p1 - p2 - p3 + p4);
        C.hourglass[nd[2]] += 1. / nbcell(nd[2]) * (-p1 - p2 + p3 - p4);
        C.hourglass[nd[3]] += 1. / nbcell(nd[3]) * (-p1 + p2 - p3 + p4);
        C.hourglass[nd[4]] += 1. / nbcell(nd[4]) * (-p1 - p2 + p3 + p4);
        C.hourglass[nd[5]] += 1. / nbcell(nd[5]) * (-p1 + p2 - p3 - p4);
        C.hourglass[nd[6]] += 1. / nbcell(nd[6]) * (p1 + p2 + p3 + p4);
        C.hourglass[nd[7]] += 1. / nbcell(nd[7]) * (p1 - p2 - p3 - p4);
      }
    }
    for (long n = 0; n < C.nnode; ++n) C.vel[n] -= C.hourglass[n];
  }
}

static bool node_on_surface(const Case& C, long n, int surf) {
  int i, j, k;
  C.nijk(n, i, j, k);
  switch (surf) {
    case MHC_XMIN: return i == 0;
    case MHC_XMAX: return i == C.nnx - 1;
    case MHC_YMIN: return j == 0;
    case MHC_YMAX: return j == C.nny - 1;
    case MHC_ZMIN: return C.dim == 3 && k == 0;
    default: return C.dim == 3 && k == C.nnz - 1;
  }
}

/* MahycoModule::applyBoundaryCondition (MahycoModule.cc:756-807), velocity
 * kinds on the PrepareFaceGroup surfaces.  A node lies on a surface exactly
 * when it belongs to one of the surface's faces. */
static void apply_pressure_bcs(Case& C);
static void apply_boundary_condition(Case& C) {
  const double eps = 1.e-8;
  for (int b = 0; b < C.P.nb_bc; ++b) {
    const mhc_bc& bc = C.P.bc[b];
    bool novalue = false;
    if ((C.t - C.dt * (1 - eps)) < bc.tdebut) novalue = true;
    if ((C.t - C.dt * (1 - eps)) > bc.tfin) novalue = true;
    if (novalue) continue;
    for (long n = 0; n < C.nnode; ++n) {
      if (!node_on_surface(C, n, bc.surface)) continue;
      if (bc.kind == MHC_BC_VX) C.vel[n].x = bc.value;
      else if (bc.kind == MHC_BC_VY) C.vel[n].y = bc.value;
      else if (bc.kind == MHC_BC_VZ) C.vel[n].z = bc.value;
      else if (bc.kind == MHC_BC_ON_FILE_VELOCITY) {
        /* OnFileVelocity (MahycoModule.cc:796-798): Real3::normL2 of the
         * position before updatePosition */
        const R3& X = C.coord[n];
        C.vel[n].x = -X.x / std::sqrt(X.x * X.x + X.y * X.y + X.z * X.z);
        C.vel[n].y = -X.y / std::sqrt(X.x * X.x + X.y * X.y + X.z * X.z);
      }
    }
  }
  apply_pressure_bcs(C);
}

/* applyBoundaryConditionForCellVariables (MahycoModule.cc:811-1037), its
 * conditions in order.  Cell variables (Density, Energy,
 * SuperGaussianEnergy, Pressure) of the cell of every face of the surface;
 * pressure surfaces (MahycoModule.cc:909-986): for every face of the surface in face order and
 * every node of the face, v -= dt_mid / nb_face_nodes * n * p * S / m_node,
 * with n the unit vector from the cell centre to the (initial) face centre,
 * S the length of the face edge from that node (2D) or the z-projected face
 * area (3D), p the BC value (plus its linear terms) inside [Tdebut, Tfin) */
/* OnFilePressure (MahycoModule.cc:987-1008): the table read by
 * lireFichierCDL (MahycoAnnexe.cc:242-269) interpolated at the current time:
 * the interval ends at the first time above it, value 0 when that is the
 * first entry or no entry is above it */
static double onfile_pressure(const Case& C) {
  const mhc_case_params& P = C.P;
  double value = 0.;
  int it = -1;
  for (int i = 0; i < P.pressure_table_n; ++i) {
    if (C.t < P.pressure_table_t[i]) {
      it = i;
      break;
    }
  }
  if (it > 0) {
    double alpha = (C.t - P.pressure_table_t[it - 1]) / (P.pressure_table_t[it] - P.pressure_table_t[it - 1]);
    alpha = alpha < 1. ? alpha : 1.;  /* math::min(alpha, 1.) */
    alpha = alpha < 0. ? 0. : alpha;  /* math::max(alpha, 0.) */
    value = P.pressure_table_p[it - 1] + alpha * (P.pressure_table_p[it] - P.pressure_table_p[it - 1]);
  }
  return value;
}

static void apply_pressure_bcs(Case& C) {
  const double w = C.dim == 2 ? .5 : .25;
  const double w8 = C.dim == 2 ? .25 : .125;
  const double dt = 0.5 * (C.old_dt + C.dt);
  for (int b = 0; b < C.P.nb_bc; ++b) {
    const mhc_bc& bc = C.P.bc[b];
    const bool cellvar = bc.kind >= MHC_BC_DENSITY && bc.kind <= MHC_BC_PRESSURE;
    const bool onfile = bc.kind == MHC_BC_ON_FILE_PRESSURE;
    const bool surface = bc.kind == MHC_BC_GEOMETRIC_PRESSURE || bc.kind == MHC_BC_LINEAR_PRESSURE ||
                         bc.kind == MHC_BC_SUPER_GAUSSIAN_PRESSURE || bc.kind == MHC_BC_CONTACT_HERZ_PRESSURE || onfile;
    if (!surface && !cellvar) continue;
    const int s = bc.surface;
    const int d = (s == MHC_XMIN || s == MHC_XMAX) ? 0 : ((s == MHC_YMIN || s == MHC_YMAX) ? 1 : 2);
    if (d >= C.dim) continue;
    const bool maxside = s >= MHC_XMAX;
    for (long f = 0; f < C.nface[d]; ++f) {
      int i, j, k;
      C.fijk(d, f, i, j, k);
      const int id = d == 0 ? i : (d == 1 ? j : k);
      if (id != (maxside ? C.ncd(d) : 0)) continue;
      /* the one cell of the boundary face */
      const long c = maxside ? (d == 0 ? C.cid(i - 1, j, k) : (d == 1 ? C.cid(i, j - 1, k) : C.cid(i, j, k - 1)))
                             : C.cid(i, j, k);
      if (cellvar) {
        /* MahycoModule.cc:838-907, global cell values (a pure cell's
         * environment value is the same): value 0 outside [Tdebut, Tfin)
         * except for the energies, which re-read it and apply the x / y
         * cutoffs to the cell centre */
        double value = bc.value;
        if (C.t < bc.tdebut) value = 0.;
        if (C.t >= bc.tfin) value = 0.;
        const R3 cc = C.cell_coord[c];
        if (bc.kind == MHC_BC_DENSITY) {
          C.density.g[c] = value;
          C.cell_mass.g[c] = C.density.g[c] * C.cell_volume.g[c];
          const double contrib = w8 * C.cell_mass.g[c];
          for (int l = 0; l < C.nbn; ++l) C.node_mass[C.cnode(c, l)] += contrib;
        } else if (bc.kind == MHC_BC_ENERGY || bc.kind == MHC_BC_SUPER_GAUSSIAN_ENERGY) {
          value = bc.value;
          if (bc.kind == MHC_BC_SUPER_GAUSSIAN_ENERGY) {
            const double ay = cc.y * bc.dependance[1];
            value *= std::exp(-std::pow(ay, 4.));
          }
          if (std::fabs(cc.x) > bc.cutoff[0]) value = 0.;
          if (std::fabs(cc.y) > bc.cutoff[1]) value = 0.;
          C.internal_energy.g[c] += value;
        } else {
          C.pressure.g[c] = value;
        }
        continue;
      }
      long n[4] = {0, 0, 0, 0};
      const int nb = C.face_nodes(d, i, j, k, n);
      for (int q = 0; q < nb; ++q) {
        const long node = n[q];
        double value = bc.value;
        double surface;
        if (C.dim == 2 || onfile) {
          const long node2 = q < nb - 1 ? n[q + 1] : n[0];
          surface = norm(C.coord[node2] - C.coord[node]);
        } else {
          const R3 v1 = C.coord[n[2]] - C.coord[n[0]], v2 = C.coord[n[3]] - C.coord[n[1]];
          surface = 0.5 * produit(v1.x, v2.y, v1.y, v2.x);
        }
        const R3 diff = C.face_coord[d][f] - C.cell_coord[c];
        const R3 nrm = diff / norm(diff);
        if (bc.kind == MHC_BC_LINEAR_PRESSURE) {
          value += bc.dependance[0] * C.coord[node].x;
          value += bc.dependance[1] * C.coord[node].y;
          value += bc.dependance[2] * C.coord[node].z;
          value += bc.dependance[3] * C.t;
        } else if (bc.kind == MHC_BC_SUPER_GAUSSIAN_PRESSURE) {
          /* MahycoModule.cc:952-959 */
          const double ay = C.coord[node].y * bc.dependance[1];
          value *= std::exp(-std::pow(ay, bc.power));
          const double ax = C.coord[node].x * bc.dependance[0];
          value *= std::exp(-std::pow(ax, bc.power));
          if (std::fabs(C.coord[node].y) > bc.cutoff[1]) value = 0.;
        } else if (bc.kind == MHC_BC_CONTACT_HERZ_PRESSURE) {
          /* MahycoModule.cc:960-970, at the boundary cell's centre */
          const double a2 = bc.dependance[0], b2 = bc.dependance[1];
          const double x2 = C.cell_coord[c].x * C.cell_coord[c].x, y2 = C.cell_coord[c].y * C.cell_coord[c].y;
          if (x2 / a2 + y2 / b2 < 1.) value *= std::sqrt(1 - x2 / a2 - y2 / b2);
          else value = 0.;
        }
        if (onfile) {
          value = onfile_pressure(C);
        } else {
          if (C.t < bc.tdebut) value = 0.;
          if (C.t >= bc.tfin) value = 0.;
        }
        C.vel[node] -= (dt * w * nrm * value * surface) / C.node_mass[node];
      }
    }
  }
}

/* MahycoModule::updatePosition (MahycoModule.cc:730-751) */
static void update_position(Case& C) {
  for (long n = 0; n < C.nnode; ++n) {
    if (C.P.sans_lagrange) {
      /* only the nodes shared by exactly four cells move (MahycoModule.cc:737) */
      int i, j, k;
      C.nijk(n, i, j, k);
      int nc = ((i > 0) + (i < C.ncx)) * ((j > 0) + (j < C.ncy));
      if (C.dim == 3) nc *= (k > 0) + (k < C.ncz);
      if (nc != 4) continue;
    }
    C.coord[n] += C.dt * C.vel[n];
  }
  cell_centres(C);
}

/* MahycoModule::updateDensity (MahycoModule.cc:1267-1316) */
static void update_density(Case& C) {
  for (int e = 0; e < C.nenv; ++e) {
    double thr = C.P.env[e].density_damage_thresold;
    for (long c = 0; c < C.ncell; ++c) {
      if (!C.has(c, e)) continue;
      double nd = C.EV(C.cell_mass, e, c) / C.EV(C.cell_volume, e, c);
      C.EV(C.density, e, c) = nd;
      if (C.EV(C.density, e, c) / C.density_0.g[c] < thr) C.EV(C.density, e, c) = thr * C.density_0.g[c];
      C.EV(C.tau_density, e, c) = 0.5 * (1.0 / C.EV(C.density_n, e, c) + 1.0 / C.EV(C.density, e, c));
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    double nd = C.cell_mass.g[c] / C.cell_volume.g[c];
    C.density.g[c] = nd;
    C.tau_density.g[c] = 0.5 * (1.0 / C.density_n.g[c] + 1.0 / C.density.g[c]);
    C.div_u[c] = 1.0 / C.dt * (1.0 / C.density.g[c] - 1.0 / C.density_n.g[c]) / C.tau_density.g[c];
  }
}

/* MahycoModule::computeArtificialViscosity (MahycoModule.cc:386-426) */
static void compute_artificial_viscosity(Case& C) {
  for (int e = 0; e < C.nenv; ++e) {
    double a1 = C.P.env[e].linear_pseudo_coeff, a2 = C.P.env[e].quadratic_pseudo_coeff;
    for (long c = 0; c < C.ncell; ++c) {
      if (!C.has(c, e)) continue;
      C.EV(C.pseudo, e, c) = 0.;
      if (C.div_u[c] < 0.0) {
        C.EV(C.pseudo, e, c) = 1. / C.EV(C.tau_density, e, c) *
            (-a1 * C.char_len[c] * C.sound_speed.g[c] * C.div_u[c] +
             a2 * C.char_len[c] * C.char_len[c] * C.div_u[c] * C.div_u[c]);
      }
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c)) continue;
    C.pseudo.g[c] = 0.;
    for (int e = 0; e < C.nenv; ++e)
      if (C.has(c, e)) C.pseudo.g[c] += C.EV(C.pseudo, e, c) * C.EV(C.fracvol, e, c);
  }
}

/* MahycoModule::updateElasticityAndPlasticity (MahycoModule.cc:1327-1353)
 * with DefaultModelService (src/elasto/DefaultModelService.cc:27-242) and
 * the constant EPP shear modulus / YEPP yield strength, one environment:
 * velocity gradient from the mean corner normals, deformation rate and
 * spin, elasto-plastic work with S_n, deviator update with rotation, radial
 * return, work with S_n+1.  Restated where the reference is undefined or
 * relies on Arcane: the deviator increment takes trace = 0 (the reference
 * reads an uninitialised `trace`, DefaultModelService.cc:82,96; its
 * CAS_Compression_isotherme_ALU_monodimX curves are reproduced with 0 and
 * miss by 7 % with tr(D));
 * doubleContraction sums row by row, each row left to right; pow(x, 2.) is
 * x*x; Real3x3 / Real divides every component. */
static void update_elasticity_and_plasticity(Case& C) {
  if (!C.elasto) return;
  const double dt = C.dt;
  const mhc_env_params& o = C.P.env[0];
  const double mu = o.shear_modulus, Y = o.yield_strength;
  for (long c = 0; c < C.ncell; ++c) {
    double G[3][3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
    for (int l = 0; l < C.nbn; ++l) {
      const R3 vi = C.vel[C.cnode(c, l)];
      const R3 cq = .5 * (C.cqs_n[c * C.nbn + l] + C.cqs[c * C.nbn + l]);
      const double va[3] = {vi.x, vi.y, vi.z}, cb[3] = {cq.x, cq.y, cq.z};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) G[a][b] += va[a] * cb[b];
    }
    const double volume = .5 * (C.cell_volume_n.g[c] + C.cell_volume.g[c]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) G[a][b] = G[a][b] / volume;
    double D[3][3];
    D[0][0] = G[0][0]; D[1][1] = G[1][1]; D[2][2] = G[2][2];
    D[0][1] = 0.5 * (G[0][1] + G[1][0]);
    D[0][2] = 0.5 * (G[0][2] + G[2][0]);
    D[1][2] = 0.5 * (G[1][2] + G[2][1]);
    D[1][0] = D[0][1]; D[2][0] = D[0][2]; D[2][1] = D[1][2];
    const double wx = 0.5 * (G[1][2] - G[2][1]), wy = 0.5 * (G[2][0] - G[0][2]), wz = 0.5 * (G[0][1] - G[1][0]);
    double* S = &C.sdev[c * 6];  /* xx yy zz xy yz zx */
    auto full = [&](double M[3][3]) {
      M[0][0] = S[0]; M[1][1] = S[1]; M[2][2] = S[2];
      M[0][1] = M[1][0] = S[3]; M[1][2] = M[2][1] = S[4]; M[2][0] = M[0][2] = S[5];
    };
    auto work = [&]() {
      double M[3][3];
      full(M);
      double r0 = M[0][0] * D[0][0] + M[0][1] * D[0][1] + M[0][2] * D[0][2];
      double r1 = M[1][0] * D[1][0] + M[1][1] * D[1][1] + M[1][2] * D[1][2];
      double r2 = M[2][0] * D[2][0] + M[2][1] * D[2][1] + M[2][2] * D[2][2];
      double dc = r0 + r1 + r2;
      C.EV(C.internal_energy, 0, c) += 0.25 * dt * (C.cell_volume.g[c] + C.cell_volume_n.g[c]) * dc /
                                       C.EV(C.cell_mass, 0, c);
    };
    work();
    /* ComputeElasticity (78-169) */
    const double sxx = S[0], syy = S[1], szz = S[2], sxy = S[3], syz = S[4], szx = S[5];
    const double trace = 0.;  /* see above */
    double P[3][3], TH[3][3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
    if (o.elasto_model == 2) {
      /* NewHypoModel: the deformation gradient F <- (I + G dt) F and
       * B = F F^T (NewHypoModelService.cc:48-49, 76-79), then the
       * deviator's rate mu / J^(5/3) (DB + BD - 2/3 (B:D) I - 5/3 tr(D)
       * dev B) dt and the thermal term mu' (T - T_n) dev B, mu' = 0 for
       * EPP (102-139); products and contractions in Arcane's order */
      double* Ft = &C.tensF[c * 9];
      double Dg[3][3], Fn[3][3], B[3][3], DB[3][3], BD[3][3], devB[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Dg[a][b] = (a == b ? 1. : 0.) + G[a][b] * dt;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Fn[a][b] = Dg[a][0] * Ft[0 * 3 + b] + Dg[a][1] * Ft[1 * 3 + b] + Dg[a][2] * Ft[2 * 3 + b];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Ft[a * 3 + b] = Fn[a][b];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) B[a][b] = Fn[a][0] * Fn[b][0] + Fn[a][1] * Fn[b][1] + Fn[a][2] * Fn[b][2];
      const double J = C.EV(C.density_0, 0, c) / C.EV(C.density, 0, c);
      const double mu_over_J = mu / (g_cr_pow ? pow_five_thirds_cr(J) : std::pow(J, 5. / 3.));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          DB[a][b] = D[a][0] * B[0][b] + D[a][1] * B[1][b] + D[a][2] * B[2][b];
          BD[a][b] = B[a][0] * D[0][b] + B[a][1] * D[1][b] + B[a][2] * D[2][b];
        }
      const double traceD = D[0][0] + D[1][1] + D[2][2];
      const double traceB = B[0][0] + B[1][1] + B[2][2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) devB[a][b] = B[a][b] - (1. / 3. * traceB) * (a == b ? 1. : 0.);
      double dcb = B[0][0] * D[0][0] + B[0][1] * D[0][1] + B[0][2] * D[0][2];
      dcb += B[1][0] * D[1][0] + B[1][1] * D[1][1] + B[1][2] * D[1][2];
      dcb += B[2][0] * D[2][0] + B[2][1] * D[2][1] + B[2][2] * D[2][2];
      const double dT = C.carries_temperature() ? C.EV(C.temperature, 0, c) - C.EV(C.temperature_n, 0, c) : 0.;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          P[a][b] = (mu_over_J * (((DB[a][b] + BD[a][b]) - (2. / 3. * dcb) * (a == b ? 1. : 0.)) -
                                  (5. / 3. * traceD) * devB[a][b])) * dt;
          TH[a][b] = (0. * dT) * devB[a][b];
        }
    } else {
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) P[a][b] = 2 * mu * (D[a][b] - (1. / 3.) * trace * (a == b ? 1.0 : 0.0)) * dt;
    }
    if (C.dim == 2) {
      if (o.rotation_order == 1) {
        P[0][0] += 2 * dt * sxy * wz;
        P[1][1] -= 2 * dt * sxy * wz;
        P[0][1] -= dt * (sxx - syy) * wz;
        P[1][0] = P[0][1];
      } else {
        const double syx = sxy;
        double a = -0.5 * dt * wz;
        double qxx = (1. - a * a) / (1. + a * a), qyy = qxx;
        double qxy = -2. * a / (1. + a * a), qyx = -qxy;
        double blxx = sxx * qxx + sxy * qxy, blxy = sxx * qyx + sxy * qyy;
        double blyx = syx * qxx + syy * qxy, blyy = syx * qyx + syy * qyy;
        P[0][0] = qxx * blxx + qxy * blyx;
        P[1][1] = qyx * blxy + qyy * blyy;
        P[0][1] = qxx * blxy + qxy * blyy;
        P[1][0] = P[0][1];
      }
    } else {
      P[0][0] -= 2 * dt * (szx * wy - sxy * wz);
      P[1][1] -= 2 * dt * (sxy * wz - syz * wx);
      P[2][2] -= 2 * dt * (syz * wx - szx * wy);
      P[0][1] -= dt * (sxx - syy) * wz - dt * syz * wy - dt * szx * wx;
      P[1][2] -= dt * (syy - szz) * wx - dt * szx * wz - dt * sxy * wy;
      P[2][0] -= dt * (szz - sxx) * wy - dt * sxy * wx - dt * syz * wz;
      P[1][0] = P[0][1]; P[2][1] = P[1][2]; P[0][2] = P[2][0];
    }
    S[0] = (sxx + P[0][0]) + TH[0][0]; S[1] = (syy + P[1][1]) + TH[1][1]; S[2] = (szz + P[2][2]) + TH[2][2];
    S[3] = (sxy + P[0][1]) + TH[0][1]; S[4] = (syz + P[1][2]) + TH[1][2]; S[5] = (szx + P[2][0]) + TH[2][0];
    /* ComputePlasticity (173-226): radial return onto the yield surface;
     * the squares are math::pow(x, 2.) there (glibc's pow, or the correctly
     * rounded square x * x with cr_pow) */
    auto sq = [](double x) { return g_cr_pow ? x * x : std::pow(x, 2.); };
    double j2 = sq(S[0]);
    j2 += sq(S[1]);
    j2 += S[0] * S[1];
    j2 += sq(S[3]);
    if (C.dim == 3) {
      j2 += sq(S[4]);
      j2 += sq(S[5]);
    }
    if (j2 > sq(Y) / 3.) {
      const double coeff = Y / std::sqrt(3. * j2);
      for (int q = 0; q < 6; ++q) S[q] *= coeff;
      /* the plastic strain rate and strain (DefaultModelService.cc:211-214),
       * then the deviator's norm on the yield surface (215, 224) */
      C.plastic_rate[c] = (1. - coeff) * Y / (3. * mu * coeff * dt);
      C.plastic[c] += C.plastic_rate[c];
      j2 = sq(Y) / 3.;
    }
    C.strain_norm[c] = std::sqrt(j2);
    work();
  }
}

/* MahycoModule::computePressionMoyenne (MahycoModule.cc:1708-1735) */
static void compute_pression_moyenne(Case& C) {
  if (C.P.sans_lagrange) return;  /* MahycoModule.cc:1711 */
  double option = C.P.calcul_vitson_max ? 1. : 0.;
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c)) continue;
    C.pressure.g[c] = 0.;
    C.sound_speed.g[c] = 0.;
    for (int e = 0; e < C.nenv; ++e) {
      if (!C.has(c, e)) continue;
      C.pressure.g[c] += C.EV(C.fracvol, e, c) * C.EV(C.pressure, e, c);
      C.sound_speed.g[c] = option * std::max(C.EV(C.sound_speed, e, c), C.sound_speed.g[c]);
      C.sound_speed.g[c] += (1. - option) * C.EV(C.fracvol, e, c) * C.EV(C.sound_speed, e, c);
    }
  }
}

/* MahycoModule::updateEnergyAndPressure (MahycoModule.cc:1430-1480) with
 * updateEnergyAndPressureforGP (1623-1698, non-CSTS branch),
 * updateEnergyAndPressurebyNewton (1506-1571) or
 * updateEnergyAndPressureExplicite (1484-1502) */
/* MahycoModule::DepotEnergy (MahycoModule.cc:1364-1417), constant, linear
 * and super-Gaussian deposits: value x deltat added to the environment's
 * internal energy, zero outside [Tdebut, Tfin] and beyond the x / y cutoffs
 * around the origin (the Lagrangian cell centre of this iteration).  The
 * super-Gaussian profile multiplies by exp(-(y dY)^power), then by
 * exp(-(x dX)^power), with std::exp and std::pow as the reference does. */
static void depot_energy(Case& C) {
  for (int e = 0; e < C.nenv; ++e) {
    const mhc_env_params& o = C.P.env[e];
    if (o.depot_type == MHC_DEPOT_NONE) continue;
    for (long c = 0; c < C.ncell; ++c) {
      if (!C.has(c, e)) continue;
      const R3 cc = C.cell_coord[c];
      double value = o.depot_value;
      if (C.t < o.depot_tdebut) value = 0.;
      if (C.t > o.depot_tfin) value = 0.;
      if (o.depot_type == MHC_DEPOT_LINEAIRE) {
        value += o.depot_dependance[0] * cc.x;
        value += o.depot_dependance[1] * cc.y;
        value += o.depot_dependance[2] * cc.z;
        value += o.depot_dependance[3] * C.t;
      } else if (o.depot_type == MHC_DEPOT_SUPER_GAUSSIAN) {
        const double ay = cc.y * o.depot_dependance[1];
        value *= std::exp(-std::pow(ay, o.depot_power));
        const double ax = cc.x * o.depot_dependance[0];
        value *= std::exp(-std::pow(ax, o.depot_power));
      }
      if (std::fabs(cc.x - o.depot_origin[0]) > o.depot_cutoff[0]) value = 0.;
      if (std::fabs(cc.y - o.depot_origin[1]) > o.depot_cutoff[1]) value = 0.;
      C.EV(C.internal_energy, e, c) += value * C.dt;
    }
  }
}

static void update_energy_and_pressure(Case& C) {
  depot_energy(C);
  if (C.P.pression_explicite) {
    for (int e = 0; e < C.nenv; ++e) {
      for (long c = 0; c < C.ncell; ++c) {
        if (!C.has(c, e)) continue;
        C.EV(C.internal_energy, e, c) -= (C.EV(C.pressure_n, e, c) + C.EV(C.pseudo, e, c)) *
                                          (1.0 / C.EV(C.density, e, c) - 1.0 / C.EV(C.density_n, e, c));
      }
      eos_apply(C, e);
    }
  } else if (C.P.with_newton) {
    /* updateEnergyAndPressurebyNewton, non-CSTS branch (MahycoModule.cc:1506-1571):
     * at most 50 Newton steps on fvnr, starting from the energy at n; the
     * pressure and sound speed left by the last applyOneCellEOS are
     * recomputed from the final energy (final applyEOS of a Lagrange-only
     * loop, or the EOS after the remap) before anything reads them */
    bool pc = C.P.pseudo_centree;
    for (int e = 0; e < C.nenv; ++e) {
      const mhc_env_params& o = C.P.env[e];
      for (long c = 0; c < C.ncell; ++c) {
        if (!C.has(c, e)) continue;
        double q = C.EV(C.pseudo, e, c), qn = C.EV(C.pseudo_n, e, c);
        double rn1 = C.EV(C.density, e, c), rn = C.EV(C.density_n, e, c);
        double pseudo = 0.;
        if (pc && ((qn + q) * (1.0 / rn1 - 1.0 / rn) < 0.)) pseudo = 0.5 * (q + qn);
        if (!pc && (q * (1.0 / rn1 - 1.0 / rn) < 0.)) pseudo = q;
        const double pn = C.EV(C.pressure_n, e, c), en = C.EV(C.internal_energy_n, e, c);
        const double eps = C.P.threshold;
        double en1 = C.EV(C.internal_energy, e, c), p = pn, dpde = 0.;
        int i = 0;
        while (i < 50 && std::fabs(fvnr(en1, p, en, pseudo, pn, rn1, rn)) >= eps) {
          eos_one_cell(o, rn1, en1, p, dpde);
          if (C.carries_temperature()) advance_temperature(C, o, e, c, en1, o.eos != MHC_EOS_MIE_GRUNEISEN);
          double enew = en1 - fvnr(en1, p, en, pseudo, pn, rn1, rn) / fvnrderiv(dpde, rn1, rn);
          en1 = enew;
          i++;
        }
        C.EV(C.internal_energy, e, c) = en1;
      }
    }
  } else if (C.P.schema_csts) {
    /* updateEnergyAndPressureforGP, CSTS branch (MahycoModule.cc:1660-1697):
     * the work of the forces at n and n+1 through the corner normals and
     * node velocities at n and n+1/2 */
    for (int e = 0; e < C.nenv; ++e) {
      double g = C.P.env[e].adiabatic_cst;
      for (long c = 0; c < C.ncell; ++c) {
        if (!C.has(c, e)) continue;
        double cn1 = 0., cn = 0., cdn = 0., cov = 0.;
        for (int l = 0; l < C.nbn; ++l) {
          const long n = C.cnode(c, l);
          const R3 v = C.vel[n], vn = C.vel_n[n];
          cn1 += dot(v, C.cqs[c * C.nbn + l]) * C.dt;
          cn += dot(v, C.cqs_n[c * C.nbn + l]) * C.dt;
          cdn += dot(v - vn, C.cqs_n[c * C.nbn + l]) * (C.dt - C.old_dt);
          cov += dot(vn, C.cqs_n[c * C.nbn + l]) * C.old_dt;
        }
        const double m = C.EV(C.cell_mass, e, c), pn = C.EV(C.pressure_n, e, c);
        const double qn = C.EV(C.pseudo_n, e, c), qn1 = C.EV(C.pseudo, e, c), qnm1 = C.EV(C.pseudo_nm1, e, c);
        double den = 1 + 0.5 * (g - 1.0) * C.EV(C.density, e, c) * cn1 / m;
        double num = C.EV(C.internal_energy, e, c) - (0.5 * (pn + qn) * cn / m) - (0.5 * qn1 * cn1 / m) +
                     (0.25 * (pn + qn) * cdn / m) - (0.5 * (qn - qnm1) * cov / m);
        C.EV(C.internal_energy, e, c) = num / den;
      }
    }
  } else {
    bool pc = C.P.pseudo_centree;
    for (int e = 0; e < C.nenv; ++e) {
      double g = C.P.env[e].adiabatic_cst;
      for (long c = 0; c < C.ncell; ++c) {
        if (!C.has(c, e)) continue;
        double q = C.EV(C.pseudo, e, c), qn = C.EV(C.pseudo_n, e, c);
        double rho = C.EV(C.density, e, c), rhon = C.EV(C.density_n, e, c);
        double pseudo = 0.;
        if (pc && ((qn + q) * (1.0 / rho - 1.0 / rhon) < 0.)) pseudo = 0.5 * (q + qn);
        if (!pc && (q * (1.0 / rho - 1.0 / rhon) < 0.)) pseudo = q;
        double den = 1 + 0.5 * (g - 1.0) * rho * (1.0 / rho - 1.0 / rhon);
        double num = C.EV(C.internal_energy_n, e, c) - (0.5 * C.EV(C.pressure, e, c) + pseudo) * (1.0 / rho - 1.0 / rhon);
        C.EV(C.internal_energy, e, c) = num / den;
      }
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c)) continue;
    C.internal_energy.g[c] = 0.;
    for (int e = 0; e < C.nenv; ++e)
      if (C.has(c, e)) C.internal_energy.g[c] += C.EV(C.mass_fraction, e, c) * C.EV(C.internal_energy, e, c);
  }
  if (!C.P.with_projection) {
    if (!C.P.pression_explicite)
      for (int e = 0; e < C.nenv; ++e) eos_apply(C, e);
    compute_pression_moyenne(C);
  }
}

/* ---------------------------------------------------------------------------
 * remap (PrepareRemap.cc, RemapADIService.cc, UtilesRemap.cc,
 * DualPhaseRemap.cc, RemapADIFinal.cc)
 * ------------------------------------------------------------------------- */

/* RemapADIService::fluxLimiter (UtilesRemap.cc:108-120) */
static double flux_limiter(int id, double r) {
  if (id == MHC_MINMOD) return std::max(0.0, std::min(1.0, r));
  if (id == MHC_SUPERBEE) return std::max(0.0, std::max(std::min(2.0 * r, 1.0), std::min(r, 2.0)));
  if (id == MHC_VANLEER) return (r <= 0.0) ? 0.0 : 2.0 * r / (1.0 + r);
  return 0.0;
}

/* classical branch of computeAndLimitGradPhi (UtilesRemap.cc:329-345) */
static double limited_gradient(int id, double gb, double gf) {
  double g = 0.;
  if (gb != 0.) g += 0.5 * (flux_limiter(id, gf / gb) * gb);
  if (gf != 0.) g += 0.5 * (flux_limiter(id, gb / gf) * gf);
  return g;
}

/* RemapADIService::fluxLimiterG (UtilesRemap.cc:130-190): slope limited
 * with the widths of the three cells (ids 3..7), optionally clipped to the
 * single-slope bound (projection-simple-pente) */
static double generalized_gradient(int id, double gp, double gm, double y0, double yp, double ym,
                                   double h0, double hp, double hm, bool simple_pente) {
  (void)y0;
  if (gp * gm < 0.0) return 0.;
  double g = 0.;
  const double dy = yp - ym;
  if (id == MHC_MINMOD_G) {
    const double a = std::min(std::fabs(gp), std::fabs(gm));
    g = dy > 0. ? a : -a;
  } else if (id == MHC_SUPERBEE_G) {
    const double a = std::max(std::fabs(gp), std::fabs(gm));
    g = dy > 0. ? a : -a;
  } else if (id == MHC_VANLEER_G) {
    const double lp = (h0 / 2. + hp) / (h0 + hp + hm);
    const double lm = (h0 / 2. + hm) / (h0 + hp + hm);
    const double den = lp * gp + lm * gm;
    g = den != 0. ? gp * gm / den : 0.;
  } else if (id == MHC_ULTRABEE_G) {
    g = dy / h0;
  } else if (id == MHC_ARITHMETIC_G) {
    const double lp = (h0 / 2. + hp) / (h0 + hp + hm);
    const double lm = (h0 / 2. + hm) / (h0 + hp + hm);
    g = lm * gp + lp * gm;
  }
  if (simple_pente) {
    const double mp = gp * (h0 + hp) / h0;
    const double mm = gm * (h0 + hm) / h0;
    const double M = std::min(std::fabs(mp), std::fabs(mm));
    const double a = std::min(std::fabs(M), std::fabs(g));
    g = dy > 0. ? a : -a;
  }
  return g;
}

/* third-order face value of the ADI remap (Remap-ordre-3.cc):
 * evaluate_grad (16-27), evaluate_ystar (35-48), evaluate_fm / evaluate_fp
 * (56-78), define_interval / intersection (86-112) and ComputeFluxOrdre3
 * (127-188).  y[0..5] / h[0..5]: values and widths of the cells
 * b-2, b-1, b, f, f+1, f+2 around the face (clamped at the line ends). */
static double o3_grad(double hm, double h0, double hp, double ym, double y0, double yp) {
  return h0 / (hm + h0 + hp) * ((2. * hm + h0) / (h0 + hp) * (yp - y0) + (h0 + 2. * hp) / (hm + h0) * (y0 - ym));
}
static double o3_ystar(double hmm, double hm, double hp, double hpp, double ymm, double ym, double yp, double ypp,
                       double gm, double gp) {
  const double a = (2. * hp * hm) / (hm + hp) * ((hmm + hm) / (2. * hm + hp) - (hpp + hp) / (2. * hp + hm)) * (yp - ym);
  const double b = -hm * (hmm + hm) / (2. * hm + hp) * gp + hp * (hp + hpp) / (hm + 2. * hp) * gm;
  return ym + hm / (hm + hp) * (yp - ym) + 1. / (hmm + hm + hp + hpp) * (a + b);
}
static double order3_face_value(const double* y, const double* h, double vdt) {
  const double g0 = o3_grad(h[0], h[1], h[2], y[0], y[1], y[2]);
  const double g1 = o3_grad(h[1], h[2], h[3], y[1], y[2], y[3]);
  const double g2 = o3_grad(h[2], h[3], h[4], y[2], y[3], y[4]);
  const double g3 = o3_grad(h[3], h[4], h[5], y[3], y[4], y[5]);
  const double sm = o3_ystar(h[0], h[1], h[2], h[3], y[0], y[1], y[2], y[3], g0, g1);
  const double s0 = o3_ystar(h[1], h[2], h[3], h[4], y[1], y[2], y[3], y[4], g1, g2);
  const double sp = o3_ystar(h[2], h[3], h[4], h[5], y[2], y[3], y[4], y[5], g2, g3);
  double v;
  if (vdt > 0.) {
    const double du = s0 - sm, u6 = 6. * (y[2] - 0.5 * (sm + s0));
    v = s0 - 0.5 * vdt / h[2] * (du - (1. - 2. / 3. * vdt / h[2]) * u6);
  } else if (vdt < 0.) {
    const double du = sp - s0, u6 = 6. * (y[3] - 0.5 * (s0 + sp)), x = -vdt;
    v = s0 + 0.5 * x / h[3] * (du - (1. - 2. / 3. * x / h[3]) * u6);
  } else {
    return 0.;
  }
  /* TVD bound: intersection of [y_b, y_f] with the upwind extrapolation */
  const double num = vdt / h[2], nup = vdt / h[3];
  const double ext_b = y[2] + (1. - num) / num * (y[2] - y[1]);
  const double ext_f = y[3] - (1. + nup) / nup * (y[3] - y[4]);
  const double i1a = amin(y[2], y[3]), i1b = amax(y[2], y[3]);
  const double o = vdt >= 0. ? y[2] : y[3], x = vdt >= 0. ? ext_b : ext_f;
  const double i2a = amin(o, x), i2b = amax(o, x);
  double lo, hi;
  if (i1b < i2a || i2b < i1a) {
    lo = hi = 0.;
  } else {
    lo = amax(i1a, i2a);
    hi = amin(i1b, i2b);
  }
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

/* ---------------------------------------------------------------------------
 * pente-borne fluxes (UtilesRemap.cc:84-96, 190-312, 417-832)
 * ------------------------------------------------------------------------- */
/* INTY: integral from -inf to X of the linear piece through (x0, y0),
 * (x1, y1) restricted to [x0, x1] */
static double inty(double X, double x0, double y0, double x1, double y1, double thr) {
  double flux = 0.;
  if (std::fabs(x1 - x0) > thr) {
    const double eta = amin(amax(0., (X - x0) / (x1 - x0)), 1.);
    flux = (y0 + 0.5 * eta * (y1 - y0)) * (x1 - x0) * eta;
  }
  return flux;
}

/* computeY0: monotonicity thresholds y0plus / y0moins of the three-piece
 * reconstruction for the limiter id */
static void pb_y0(int id, double yp, double ym, double h0, double hp, double hm, bool simple_pente,
                  double& y0p, double& y0m) {
  y0p = 0.; y0m = 0.;
  if (id == MHC_MINMOD_G || id == MHC_MINMOD) {
    y0p = yp; y0m = ym;
  } else if (id == MHC_SUPERBEE_G || id == MHC_SUPERBEE) {
    y0p = ((h0 + hm) * yp + h0 * ym) / (2 * h0 + hm);
    y0m = ((h0 + hp) * ym + h0 * yp) / (2 * h0 + hp);
  } else if (id == MHC_VANLEER_G || id == MHC_VANLEER) {
    const double a = amin(yp, ym), b = amax(yp, ym);
    double xp = (h0 * h0 + 3 * h0 * hm + 2 * hm * hm) * yp;
    double xm = (h0 * h0 + 3 * h0 * hp + 2 * hp * hp) * ym;
    xp += (h0 * h0 - h0 * hp - 2 * hp * hp + 2 * h0 * hm) * ym;
    xm += (h0 * h0 - h0 * hm - 2 * hm * hm + 2 * h0 * hp) * yp;
    xp /= (2 * h0 * h0 + 5 * h0 * hm + 2 * hm * hm - h0 * hp - 2 * hp * hp);
    xm /= (2 * h0 * h0 + 5 * h0 * hp + 2 * hp * hp - h0 * hm - 2 * hm * hm);
    y0p = amin(amax(xp, a), b);
    y0m = amin(amax(xm, a), b);
  } else if (id == MHC_ULTRABEE_G) {
    y0p = (yp + ym) / 2.;
    y0m = (yp + ym) / 2.;
  } else if (id == MHC_ARITHMETIC_G) {
    y0p = ((h0 + hm + hp) * yp + h0 * ym) / (2 * h0 + hm + hp);
    y0m = ((h0 + hm + hp) * ym + h0 * yp) / (2 * h0 + hm + hp);
  }
  if (simple_pente) { y0p = yp; y0m = ym; }
}

/* flux of one variable out of a cell through its back (type 0) or front
 * (type 1) face: integral of the three-piece reconstruction (computexgxd,
 * computeygyd) over the swept length, or the cell value times that length
 * at an extremum (formule 16) */
static double pb_flux(int type, double y0, double yp, double ym, double h0, double hp, double hm, double grad,
                      double ppv, int lim, bool simple_pente, double thr) {
  double y0p, y0m;
  pb_y0(lim, yp, ym, h0, hp, hm, simple_pente, y0p, y0m);
  double xplus = 1., xmoins = 1.;
  if (std::fabs(y0p - yp) > thr) xplus = (y0 - yp) / (y0p - yp) - 1. / 2.;
  if (std::fabs(y0m - ym) > thr) xmoins = (y0 - ym) / (y0m - ym) - 1. / 2.;
  const double xd = +h0 * amin(amax(xplus, -1. / 2.), 1. / 2.);
  const double xg = -h0 * amin(amax(xmoins, -1. / 2.), 1. / 2.);
  const double xtd = y0 + h0 / 2 * grad, xtg = y0 - h0 / 2 * grad;
  const double ad = amin(yp, 2. * y0m - ym), bd = amax(yp, 2. * y0m - ym);
  const double ag = amin(ym, 2. * y0p - yp), bg = amax(ym, 2. * y0p - yp);
  const double yd = amin(amax(xtd, ad), bd), yg = amin(amax(xtg, ag), bg);
  double f1, f1m, f2, f2m, f3, f3m;
  if (type == 0) {
    const double X = -h0 / 2. + ppv, X0 = -h0 / 2.;
    f1m = inty(X, -h0 / 2., ym, xg, yg, thr);
    f1 = inty(X0, -h0 / 2., ym, xg, yg, thr);
    f2m = inty(X, xg, yg, xd, yd, thr);
    f2 = inty(X0, xg, yg, xd, yd, thr);
    f3m = inty(X, xd, yd, h0 / 2., yp, thr);
    f3 = inty(X0, xd, yd, h0 / 2., yp, thr);
  } else {
    const double X = h0 / 2. - ppv, X1 = h0 / 2.;
    f1 = inty(X, -h0 / 2., ym, xg, yg, thr);
    f1m = inty(X1, -h0 / 2., ym, xg, yg, thr);
    f2 = inty(X, xg, yg, xd, yd, thr);
    f2m = inty(X1, xg, yg, xd, yd, thr);
    f3 = inty(X, xd, yd, h0 / 2., yp, thr);
    f3m = inty(X1, xd, yd, h0 / 2., yp, thr);
  }
  double F = std::max(((f1m - f1) + (f2m - f2) + (f3m - f3)), 0.);
  if (((yp - y0) * (ym - y0)) >= 0.) F = y0 * ppv;
  return F;
}

/* computeFluxPP / computeFluxPPPure (UtilesRemap.cc:417-832) for cell c
 * with neighbours cf / cb: fluxes of every variable through one face, then
 * the de-barring fix that rebuilds mass and energy fluxes */
static void pb_cell_fluxes(const Case& C, long c, long cf, long cb, double v, int type, bool pure, double* F) {
  const int nv = C.nvars, ne = C.nenv;
  const double thr = C.P.remap_threshold;
  const double ppv = 0.5 * (v + std::fabs(v)) * C.dt;
  const int lim = pure ? C.P.projection_limiteur_pure_id : C.P.projection_limiteur_id;
  const bool sp = C.P.projection_simple_pente != 0;
  const double* P = C.phi_lag.data();
  for (int iv = 0; iv < nv; ++iv) F[iv] = 0.;
  for (int iv = 0; iv < C.nproj(); ++iv)
    F[iv] = pb_flux(type, P[c * nv + iv], P[cf * nv + iv], P[cb * nv + iv], C.h_cell[c], C.h_cell[cf],
                    C.h_cell[cb], C.grad_phi[c * nv + iv], ppv, lim, sp, thr);
  const int fix = C.P.projection_pente_borne_debar_fix;
  if (fix == 1) {
    double sfv = 0.;
    for (int e = 0; e < ne; ++e) sfv += F[e];
    if (std::fabs(sfv) > thr) {
      for (int e = 0; e < ne; ++e) {
        if (!pure) F[ne + e] = (F[ne + e] / sfv) * F[e];
        F[2 * ne + e] = (F[2 * ne + e] / sfv) * F[ne + e];
      }
    } else {
      for (int iv = 0; iv < nv; ++iv) F[iv] = 0.;
    }
  } else if (fix == 2) {
    for (int e = 0; e < ne; ++e) {
      if (!pure) F[ne + e] = P[c * nv + ne + e] * F[e];
      F[2 * ne + e] = P[c * nv + 2 * ne + e] * F[ne + e];
    }
  }
  if (ppv == 0.)
    for (int iv = 0; iv < nv; ++iv) F[iv] = 0.;
}

/* MahycoModule::computeVariablesForRemap (PrepareRemap.cc:94-193) */
static void compute_variables_for_remap(Case& C) {
  const int ne = C.nenv, nv = C.nvars;
  std::fill(C.u_lag.begin(), C.u_lag.end(), 0.);
  for (int e = 0; e < ne; ++e) {
    for (long c = 0; c < C.ncell; ++c) {
      if (!C.has(c, e)) continue;
      double* u = &C.u_lag[c * nv];
      double V = C.EV(C.cell_volume, e, c), rho = C.EV(C.density, e, c);
      u[e] = V;
      u[ne + e] = V * rho;
      u[2 * ne + e] = V * rho * C.EV(C.internal_energy, e, c);
      u[3 * ne] = C.cell_volume.g[c] * C.pseudo.g[c];
      if (nv > 3 * ne + 1) {
        /* the deviator times the volume, the plastic strain rate and strain
         * times the mass (PrepareRemap.cc:121-128) */
        const double* S = &C.sdev[c * 6];  /* xx yy zz xy yz zx */
        double* x = &u[3 * ne + 1];
        x[0] = V * S[0]; x[1] = V * S[1]; x[2] = V * S[3]; x[3] = V * S[4]; x[4] = V * S[5];
        x[5] = V * rho * C.plastic_rate[c];
        x[6] = V * rho * C.plastic[c];
      }
      if (C.P.projection_pente_borne) {
        /* the cell's own environment values; entries of absent
         * environments keep their values of the previous remap */
        double* ph = &C.phi_lag[c * nv];
        ph[e] = C.EV(C.fracvol, e, c);
        ph[ne + e] = rho;
        ph[2 * ne + e] = C.EV(C.internal_energy, e, c);
        ph[3 * ne] = C.pseudo.g[c];
      } else {
        for (int iv = 0; iv < C.nproj(); ++iv) C.phi_lag[c * nv + iv] = u[iv] / C.cell_volume.g[c];
      }
    }
  }
  for (long n = 0; n < C.nnode; ++n) {
    double m = C.node_mass[n];
    R3 v = C.vel[n];
    double* ud = &C.u_dual[n * 5];
    double* pd = &C.phi_dual[n * 5];
    ud[0] = m * v.x; ud[1] = m * v.y; ud[2] = m * v.z; ud[3] = m;
    ud[4] = 0.5 * m * (v.x * v.x + v.y * v.y + v.z * v.z);
    pd[0] = v.x; pd[1] = v.y; pd[2] = v.z; pd[3] = m;
    pd[4] = 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);
  }
}

/* MahycoModule::computeFaceQuantitesForRemap (PrepareRemap.cc:18-59) */
static void compute_face_quantities_for_remap(Case& C) {
  const double w = C.dim == 2 ? .5 : .25;
  for (int d = 0; d < C.dim; ++d) {
    for (long f = 0; f < C.nface[d]; ++f) {
      int i, j, k;
      C.fijk(d, f, i, j, k);
      long n[4];
      int nb = C.face_nodes(d, i, j, k, n);
      if (C.dim == 3) {
        R3 v1 = C.coord[n[2]] - C.coord[n[0]], v2 = C.coord[n[3]] - C.coord[n[1]];
        double L[3];
        L[0] = 0.5 * std::fabs(produit(v1.y, v2.z, v1.z, v2.y));
        L[1] = 0.5 * std::fabs(produit(v2.x, v1.z, v2.z, v1.x));
        L[2] = 0.5 * std::fabs(produit(v1.x, v2.y, v1.y, v2.x));
        C.face_len[d][f] = L[d];
      } else {
        R3 t = C.coord[n[1]] - C.coord[n[0]];
        C.face_len[d][f] = (d == 0) ? std::fabs(t.y) : std::fabs(t.x);
      }
      R3 vm = {0., 0., 0.}, fc = {0., 0., 0.};
      for (int q = 0; q < nb; ++q) {
        fc += w * C.coord[n[q]];
        /* CSTS: the mean of the velocities at n and n+1 */
        if (C.P.schema_csts) vm += 0.5 * (C.vel[n[q]] + C.vel_n[n[q]]);
        else vm += C.vel[n[q]];
      }
      C.face_coord[d][f] = fc;
      C.face_un[d][f] = dot((w * vm), C.face_normal[d][f]);
    }
  }
}

/* previous / next cell of an inner face of direction d */
static void face_cells(const Case& C, int d, long f, long& cb, long& cf) {
  int i, j, k;
  C.fijk(d, f, i, j, k);
  int id = d == 0 ? i : (d == 1 ? j : k);
  cb = cf = -1;
  if (id > 0) cb = (d == 0) ? C.cid(i - 1, j, k) : (d == 1 ? C.cid(i, j - 1, k) : C.cid(i, j, k - 1));
  if (id < C.ncd(d)) cf = C.cid(i, j, k);
}

/* RemapADIService::computeGradPhiFace (RemapADIService.cc:119-149): face
 * gradients and the cell widths along d (distances from the cell centre to
 * the centres of its inner faces of direction d) */
static void compute_grad_phi_face(Case& C, int d) {
  const int nv = C.nvars;
  C.grad_phi_face.assign(C.nface[d] * nv, 0.);
  std::fill(C.h_cell.begin(), C.h_cell.end(), 0.);
  for (long f = 0; f < C.nface[d]; ++f) {
    long cb, cf;
    face_cells(C, d, f, cb, cf);
    if (cb < 0 || cf < 0) continue;
    C.deltax[d][f] = dot((C.cell_coord[cf] - C.cell_coord[cb]), C.face_normal[d][f]);
    for (int iv = 0; iv < C.nproj(); ++iv)
      C.grad_phi_face[f * nv + iv] = (C.phi_lag[cf * nv + iv] - C.phi_lag[cb * nv + iv]) / C.deltax[d][f];
    C.h_cell[cb] += norm(C.face_coord[d][f] - C.cell_coord[cb]);
    C.h_cell[cf] += norm(C.face_coord[d][f] - C.cell_coord[cf]);
  }
}

/* neighbour of cell c at offset s (+-1) along d, or -1 outside the mesh */
static long cell_step(const Case& C, long c, int d, int s) {
  int i, j, k;
  C.cijk(c, i, j, k);
  int& id = d == 0 ? i : (d == 1 ? j : k);
  id += s;
  if (id < 0 || id >= C.ncd(d)) return -1;
  return C.cid(i, j, k);
}

/* back / front face of cell c in direction d */
static void cell_dir_faces(const Case& C, long c, int d, long& fb, long& ff) {
  int i, j, k;
  C.cijk(c, i, j, k);
  fb = C.fid(d, i, j, k);
  ff = (d == 0) ? C.fid(0, i + 1, j, k) : (d == 1 ? C.fid(1, i, j + 1, k) : C.fid(2, i, j, k + 1));
}

/* RemapADIService::computeGradPhiCell (RemapADIService.cc:161-267) with
 * computeAndLimitGradPhi (UtilesRemap.cc:325-357), without pente-borne */
static void compute_grad_phi_cell(Case& C, int d) {
  const int nv = C.nvars;
  const int lim = C.P.projection_limiteur_id;
  std::fill(C.grad_phi.begin(), C.grad_phi.end(), 0.);
  if (C.P.ordre_projection <= 1) return;
  for (long c = 0; c < C.ncell; ++c) {
    long fb, ff;
    cell_dir_faces(C, c, d, fb, ff);
    long cb = cell_step(C, c, d, -1), cf = cell_step(C, c, d, +1);
    if (cb < 0) cb = c;
    if (cf < 0) cf = c;
    /* pure neighbourhood (projection-pente-borne-mixte only) */
    const bool pure = C.P.projection_pente_borne_mixte && C.est_mixte[c] == 0 && C.est_mixte[cf] == 0 &&
                      C.est_mixte[cb] == 0 && C.est_pure[c] == C.est_pure[cf] && C.est_pure[c] == C.est_pure[cb];
    int l = lim;
    if (C.P.projection_limiteur_pure_id == 1 && pure) l = C.P.projection_limiteur_pure_id;
    for (int iv = 0; iv < C.nproj(); ++iv) {
      const double gb = C.grad_phi_face[fb * nv + iv], gf = C.grad_phi_face[ff * nv + iv];
      C.grad_phi[c * nv + iv] = l < MHC_MINMOD_G
          ? limited_gradient(l, gb, gf)
          : generalized_gradient(l, gf, gb, C.phi_lag[c * nv + iv], C.phi_lag[cf * nv + iv], C.phi_lag[cb * nv + iv],
                                 C.h_cell[c], C.h_cell[cf], C.h_cell[cb], C.P.projection_simple_pente != 0);
    }
    if (!C.P.projection_pente_borne) continue;
    /* outgoing normal velocities of the back and front faces
     * (RemapADIService.cc:212-216) */
    int i, j, k;
    C.cijk(c, i, j, k);
    double vb = 0., vf = 0.;
    for (int q = 0; q < 2 * C.dim; ++q) {
      int fd; long f;
      C.cell_face(i, j, k, q, fd, f);
      if (fd != d) continue;
      const double ond = comp(C.outer_normal[c * 2 * C.dim + q], d);
      if (f == fb) vb = ond * C.face_un[d][fb];
      if (f == ff) vf = ond * C.face_un[d][ff];
    }
    pb_cell_fluxes(C, c, cf, cb, vb, 0, pure, &C.delta_ar[c * nv]);
    pb_cell_fluxes(C, c, cf, cb, vf, 1, pure, &C.delta_av[c * nv]);
  }
}

/* RemapADIService::computeUpwindFaceQuantitiesForProjection (279-383),
 * without pente-borne: upwind value plus slope (order 1, 2) or the
 * third-order face value with the mixed-neighbourhood correction */
static void compute_upwind_face_quantities(Case& C, int d) {
  const int nv = C.nvars, ne = C.nenv;
  C.phi_face.assign(C.nface[d] * nv, 0.);
  int order2 = C.P.ordre_projection - 1;
  for (long f = 0; f < C.nface[d]; ++f) {
    long cb, cf;
    face_cells(C, d, f, cb, cf);
    if (cb < 0 || cf < 0) continue;
    if (C.P.ordre_projection <= 2 && C.P.projection_pente_borne) {
      for (int iv = 0; iv < C.nproj(); ++iv)
        C.phi_face[f * nv + iv] = C.delta_av[cb * nv + iv] - C.delta_ar[cf * nv + iv];
      continue;
    }
    if (C.P.ordre_projection <= 2) {
      long cu = (C.face_un[d][f] * C.deltax[d][f] > 0.0) ? cb : cf;
      for (int iv = 0; iv < C.nproj(); ++iv)
        C.phi_face[f * nv + iv] = C.phi_lag[cu * nv + iv] +
            order2 * dot((C.face_coord[d][f] - C.cell_coord[cu]), C.face_normal[d][f]) * C.grad_phi[cu * nv + iv];
      continue;
    }
    /* stencil b-2 .. f+2, repeated at the line ends */
    long s[6];
    s[2] = cb; s[3] = cf;
    s[1] = cell_step(C, cb, d, -1);
    if (s[1] < 0) { s[1] = s[0] = cb; }
    else { s[0] = cell_step(C, s[1], d, -1); if (s[0] < 0) s[0] = s[1]; }
    s[4] = cell_step(C, cf, d, +1);
    if (s[4] < 0) { s[4] = s[5] = cf; }
    else { s[5] = cell_step(C, s[4], d, +1); if (s[5] < 0) s[5] = s[4]; }
    const double vdt = C.face_un[d][f] * C.dt;
    double h[6], y[6];
    for (int q = 0; q < 6; ++q) h[q] = C.h_cell[s[q]];
    for (int iv = 0; iv < C.nproj(); ++iv) {
      for (int q = 0; q < 6; ++q) y[q] = C.phi_lag[s[q] * nv + iv];
      C.phi_face[f * nv + iv] = order3_face_value(y, h, vdt);
    }
    const bool pure_nb = C.est_mixte[cb] == 0 && C.est_mixte[cf] == 0 && C.est_pure[cb] == C.est_pure[cf];
    if (pure_nb) continue;
    /* masses from the volume flux and energies from the mass flux with the
     * upwind cell's density and specific energy */
    double* pf = &C.phi_face[f * nv];
    for (int e = 0; e < ne; ++e) {
      const double* pb = &C.phi_lag[cb * nv];
      const double* pfr = &C.phi_lag[cf * nv];
      if (vdt > 0. && pb[e] != 0. && pb[ne + e] != 0.) {
        pf[ne + e] = (pb[ne + e] / pb[e]) * pf[e];
        pf[2 * ne + e] = (pb[2 * ne + e] / pb[ne + e]) * pf[ne + e];
      } else if (vdt < 0. && pfr[e] != 0. && pfr[ne + e] != 0.) {
        pf[ne + e] = (pfr[ne + e] / pfr[e]) * pf[e];
        pf[2 * ne + e] = (pfr[2 * ne + e] / pfr[ne + e]) * pf[ne + e];
      }
    }
  }
}

/* mixed / pure indicator of a cell from its volume fractions
 * (RemapADIService.cc:558-573, RemapADIFinal.cc:131-145) */
static void set_cell_purity(Case& C, long c, const double* frac, const bool* present) {
  int count = 0, last = -1;
  for (int e = 0; e < C.nenv; ++e)
    if (present[e] && frac[e] > 0.) { ++count; last = e; }
  if (count > 1) { C.est_mixte[c] = 1; C.est_pure[c] = -1; }
  else { C.est_mixte[c] = 0; C.est_pure[c] = last; }
}

/* RemapADIService::computeUremap (RemapADIService.cc:395-575), classical path */
static void compute_uremap(Case& C, int d) {
  const int nv = C.nvars, ne = C.nenv;
  const double dt = C.dt;
  std::fill(C.dual_phi_flux.begin(), C.dual_phi_flux.end(), 0.);
  std::vector<double> flux_face(nv);
  for (long c = 0; c < C.ncell; ++c) {
    int i, j, k;
    C.cijk(c, i, j, k);
    std::fill(flux_face.begin(), flux_face.end(), 0.);
    for (int l = 0; l < 2 * C.dim; ++l) {
      int fd; long f;
      C.cell_face(i, j, k, l, fd, f);
      if (fd != d) continue;
      double un = C.face_un[d][f], L = C.face_len[d][f];
      R3 on = C.outer_normal[c * 2 * C.dim + l];
      double ond = comp(on, d);
      for (int iv = 0; iv < C.nproj(); ++iv) {
        /* pente-borne face values are already integrated fluxes */
        double flux = C.P.projection_pente_borne ? ond * L * C.phi_face[f * nv + iv]
                                                 : ond * un * L * dt * C.phi_face[f * nv + iv];
        flux_face[iv] += flux;
        C.dual_phi_flux[c * nv + iv] += 0.5 * flux * comp(on, d);
      }
    }
    double* u = &C.u_lag[c * nv];
    for (int iv = 0; iv < C.nproj(); ++iv) u[iv] -= flux_face[iv];
    const double thr = C.P.remap_threshold;
    if (C.P.projection_pente_borne && !C.P.sans_lagrange) {
      /* truncation of tiny projected volumes, masses and energies
       * (RemapADIService.cc:440-462, with the dual projection) */
      for (int e = 0; e < ne; ++e) {
        if (u[e] < 1. * thr) { u[e] = 0.; u[ne + e] = 0.; u[2 * ne + e] = 0.; }
        if (u[ne + e] < 1. * thr) { u[e] = 0.; u[ne + e] = 0.; u[2 * ne + e] = 0.; }
        if (u[2 * ne + e] < 1. * thr) { u[e] = 0.; u[ne + e] = 0.; u[2 * ne + e] = 0.; }
      }
    }
    for (int e = 0; e < ne; ++e) {
      if (u[ne + e] < 0.) u[ne + e] = 0.;
      if (u[2 * ne + e] < 0.) u[2 * ne + e] = 0.;
    }
    double sv = 0.;
    for (int e = 0; e < ne; ++e) sv += u[e];
    if (C.P.projection_pente_borne) {
      /* volume fractions, densities and specific energies
       * (RemapADIService.cc:493-530); the pseudo-viscosity keeps its value */
      double* ph = &C.phi_lag[c * nv];
      for (int e = 0; e < ne; ++e) {
        ph[e] = u[e] / sv;
        ph[ne + e] = u[e] != 0. ? u[ne + e] / u[e] : 0.;
      }
      for (int e = 0; e < ne; ++e) ph[2 * ne + e] = u[ne + e] != 0. ? u[2 * ne + e] / u[ne + e] : 0.;
    } else {
      for (int iv = 0; iv < C.nproj(); ++iv) C.phi_lag[c * nv + iv] = u[iv] / sv;
    }
    bool all[MHC_MAX_ENV];
    for (int e = 0; e < ne; ++e) all[e] = true;
    set_cell_purity(C, c, &C.phi_lag[c * nv], all);
  }
}

/* RemapADIService::computeDualUremap (DualPhaseRemap.cc:38-258), classical limiter */
static void compute_dual_uremap(Case& C, int d) {
  const int ne = C.nenv, nv = C.nvars;
  const double dt = C.dt;
  const int nnd = d == 0 ? C.nnx : (d == 1 ? C.nny : C.nnz);
  auto ncoord = [&](long n) { return comp(C.coord[n], d); };
  auto step = [&](long n, int s) -> long {
    int i, j, k;
    C.nijk(n, i, j, k);
    if (d == 0) i += s; else if (d == 1) j += s; else k += s;
    int id = d == 0 ? i : (d == 1 ? j : k);
    if (id < 0 || id >= nnd) return -1;
    return C.nid(i, j, k);
  };
  auto inner = [&](long n) {
    int i, j, k;
    C.nijk(n, i, j, k);
    int id = d == 0 ? i : (d == 1 ? j : k);
    return id > 0 && id < nnd - 1;
  };
  std::fill(C.dual_grad.begin(), C.dual_grad.end(), 0.);
  if (C.P.ordre_projection > 1) {
    for (long n = 0; n < C.nnode; ++n) {
      if (!inner(n)) continue;
      long nb = step(n, -1), nf = step(n, +1);
      /* dual cell widths (UtilesRemap.cc:51-63); a missing second
       * neighbour gives a zero width */
      const long nbb = step(nb, -1), nff = step(nf, +1);
      const double h0 = 0.5 * (ncoord(nf) - ncoord(nb));
      double hm = 0., hp = 0.;
      if (nbb < 0) {
        if (nff >= 0) hp = 0.5 * (ncoord(nff) - ncoord(n));
      } else if (nff < 0) {
        hm = 0.5 * (ncoord(n) - ncoord(nbb));
      } else {
        hm = 0.5 * (ncoord(n) - ncoord(nbb));
        hp = 0.5 * (ncoord(nff) - ncoord(n));
      }
      const int lim = C.P.projection_limiteur_id;
      for (int iv = 0; iv < 3; ++iv) {
        double gf = (C.phi_dual[nf * 5 + iv] - C.phi_dual[n * 5 + iv]) / (ncoord(nf) - ncoord(n));
        double gb = (C.phi_dual[n * 5 + iv] - C.phi_dual[nb * 5 + iv]) / (ncoord(n) - ncoord(nb));
        C.dual_grad[n * 5 + iv] = lim < MHC_MINMOD_G
            ? limited_gradient(lim, gb, gf)
            : generalized_gradient(lim, gf, gb, C.phi_dual[n * 5 + iv], C.phi_dual[nf * 5 + iv],
                                   C.phi_dual[nb * 5 + iv], h0, hp, hm, C.P.projection_simple_pente != 0);
      }
    }
  }
  /* node mass fluxes: faces of direction d in face id order, then envs */
  std::fill(C.back_flux.begin(), C.back_flux.end(), 0.);
  std::fill(C.front_flux.begin(), C.front_flux.end(), 0.);
  const double w = C.dim == 2 ? .5 : .25;
  for (long f = 0; f < C.nface[d]; ++f) {
    long cb, cf;
    face_cells(C, d, f, cb, cf);
    int i, j, k;
    C.fijk(d, f, i, j, k);
    long fn[4];
    int nb = C.face_nodes(d, i, j, k, fn);
    if (cb >= 0)
      for (int q = 0; q < nb; ++q)
        for (int e = 0; e < ne; ++e) C.back_flux[fn[q]] += w * C.dual_phi_flux[cb * nv + ne + e];
    if (cf >= 0)
      for (int q = 0; q < nb; ++q)
        for (int e = 0; e < ne; ++e) C.front_flux[fn[q]] += w * C.dual_phi_flux[cf * nv + ne + e];
  }
  const int order2 = C.P.ordre_projection - 1;
  for (long n = 0; n < C.nnode; ++n) {
    if (!inner(n)) continue;
    long nb = step(n, -1), nf = step(n, +1);
    double* U = &C.u_dual[n * 5];
    const double* P = C.phi_dual.data();
    const double* G = C.dual_grad.data();
    double bfm = C.back_flux[n], ffm = C.front_flux[n];
    U[3] += bfm - ffm;
    double FV[3], BV[3], FE, BE;
    double ufront = 0.5 * (P[n * 5 + d] + P[nf * 5 + d]);
    int signfront = (ufront > 0) ? 1 : -1;
    long src = (ffm < 0.) ? nf : n;
    double geo = (signfront * (ncoord(nf) - ncoord(n)) - dt * ufront);
    for (int iv = 0; iv < 3; ++iv) FV[iv] = P[src * 5 + iv] + order2 * (0.5 * G[src * 5 + iv] * geo);
    FE = P[src * 5 + 4] + order2 * (0.5 * G[src * 5 + 4] * geo);
    double uback = 0.5 * (P[nb * 5 + d] + P[n * 5 + d]);
    int signback = (uback > 0) ? 1 : -1;
    src = (bfm > 0.) ? nb : n;
    geo = (signback * (ncoord(n) - ncoord(nb)) - dt * uback);
    for (int iv = 0; iv < 3; ++iv) BV[iv] = P[src * 5 + iv] + order2 * (0.5 * G[src * 5 + iv] * geo);
    BE = P[src * 5 + 4] + order2 * (0.5 * G[src * 5 + 4] * geo);
    for (int iv = 0; iv < 3; ++iv) U[iv] += bfm * BV[iv] - ffm * FV[iv];
    U[4] += bfm * BE - ffm * FE;
  }
  for (long n = 0; n < C.nnode; ++n) {
    if (!inner(n)) continue;
    double* U = &C.u_dual[n * 5];
    double* P = &C.phi_dual[n * 5];
    for (int iv = 0; iv < 3; ++iv)
      if (std::fabs(U[iv]) < 1.e-300) U[iv] = 0.;
    P[0] = U[0] / U[3];
    P[1] = U[1] / U[3];
    P[2] = U[2] / U[3];
    P[3] = U[3];
    P[4] = U[4] / U[3];
  }
}

/* RemapADIService::remapVariables (RemapADIFinal.cc:21-346) */
static int remap_variables(Case& C) {
  const int ne = C.nenv, nv = C.nvars;
  const double thr = C.P.remap_threshold;
  const bool with_dual = !C.P.sans_lagrange;  /* PrepareRemap.cc:211 */
  /* environment membership update: the add / remove criteria of one
   * environment only read that environment's membership, so the new masks
   * are computed first and the storage transfer is applied once per cell */
  std::vector<uint8_t> newmask(C.envmask);
  for (int e = 0; e < ne; ++e) {
    for (long c = 0; c < C.ncell; ++c) {
      const double* u = &C.u_lag[c * nv];
      bool in = C.has(c, e);
      if (((u[e] / C.euler_volume[c]) < thr || (u[ne + e] == 0. && with_dual)) && in) {
        newmask[c] &= (uint8_t)~(1 << e);
      } else if ((u[e] / C.euler_volume[c]) > thr && !in) {
        double volt = 0.;
        for (int q = 0; q < ne; ++q) volt += u[q];
        double vn = u[e] * C.euler_volume[c] / volt;
        if ((vn / C.euler_volume[c]) > thr && u[ne + e] != 0.) newmask[c] |= (uint8_t)(1 << e);
      }
    }
  }
  {
    MatField* mf[] = {&C.density, &C.density_n, &C.density_0, &C.pressure, &C.pressure_n, &C.pseudo,
                      &C.pseudo_n, &C.pseudo_nm1, &C.mass_fraction, &C.cell_mass, &C.internal_energy,
                      &C.internal_energy_n, &C.dpde, &C.fracvol, &C.cell_volume, &C.cell_volume_n,
                      &C.tau_density, &C.sound_speed};
    for (long c = 0; c < C.ncell; ++c) {
      uint8_t old = C.envmask[c], nm = newmask[c];
      if (old == nm) continue;
      int oldn = __builtin_popcount(old), newn = __builtin_popcount(nm);
      /* values of environments that stay keep their value; a new
       * environment starts from zero */
      for (int e = 0; e < ne; ++e) {
        bool was = (old >> e) & 1, is = (nm >> e) & 1;
        if (!is) continue;
        for (MatField* f : mf) {
          double v = was ? (oldn == 1 ? f->g[c] : f->e[e][c]) : 0.;
          if (newn == 1) { if (was) f->g[c] = v; }
          else f->e[e][c] = v;
        }
      }
      C.envmask[c] = nm;
      C.nenvc[c] = (uint8_t)newn;
    }
  }
  std::vector<double> vol(ne), dens(ne), ener(ne);
  std::fill(C.cell_mass.g.begin(), C.cell_mass.g.end(), 0.);
  for (long c = 0; c < C.ncell; ++c) {
    const double* u = &C.u_lag[c * nv];
    double V = C.euler_volume[c];
    C.cell_volume.g[c] = C.euler_volume[c];
    double volt = 0., masset = 0.;
    for (int e = 0; e < ne; ++e) { vol[e] = u[e]; volt += vol[e]; masset += u[ne + e]; }
    double unsurvolt = 1. / volt;
    for (int e = 0; e < ne; ++e) vol[e] *= V * unsurvolt;
    double somme_frac = 0.;
    double unsurvol = 1. / V;
    for (int e = 0; e < ne; ++e) {
      if (!C.has(c, e)) continue;
      double& f = C.EV(C.fracvol, e, c);
      f = vol[e] * unsurvol;
      if (f < thr) f = 0.;
      somme_frac += f;
    }
    double unsursf = 0.;
    if (somme_frac != 0.) unsursf = 1. / somme_frac;
    for (int e = 0; e < ne; ++e)
      if (C.has(c, e)) C.EV(C.fracvol, e, c) *= unsursf;
    {
      double fr[MHC_MAX_ENV];
      bool pres[MHC_MAX_ENV];
      for (int e = 0; e < ne; ++e) {
        pres[e] = C.has(c, e);
        fr[e] = pres[e] ? C.EV(C.fracvol, e, c) : 0.;
      }
      set_cell_purity(C, c, fr, pres);
    }
    if (masset > thr * thr) {
      double unsurm = 1. / masset, fm = 0.;
      for (int e = 0; e < ne; ++e) {
        if (!C.has(c, e)) continue;
        C.EV(C.mass_fraction, e, c) = u[ne + e] * unsurm;
        if (C.EV(C.fracvol, e, c) < thr) C.EV(C.mass_fraction, e, c) = 0.;
        fm += C.EV(C.mass_fraction, e, c);
      }
      if (fm != 0.) {
        double unsurfm = 1. / fm;
        for (int e = 0; e < ne; ++e)
          if (C.has(c, e)) C.EV(C.mass_fraction, e, c) *= unsurfm;
      }
    }
    double dn = 0.;
    for (int e = 0; e < ne; ++e) {
      if (!C.has(c, e)) continue;
      dens[e] = 0.;
      if (C.EV(C.fracvol, e, c) > thr && vol[e] != 0.) dens[e] = u[ne + e] / vol[e];
      dn += C.EV(C.fracvol, e, c) * dens[e];
    }
    for (int e = 0; e < ne; ++e) {
      if (!C.has(c, e)) continue;
      ener[e] = 0.;
      if (C.EV(C.fracvol, e, c) > thr && u[ne + e] != 0.) ener[e] = u[2 * ne + e] / u[ne + e];
      if (nv > 3 * ne + 1 && C.EV(C.fracvol, e, c) > thr && u[ne + e] != 0.) {
        /* RemapADIFinal.cc:200-214: the deviator over the projected volume,
         * zz from the zero trace, the plastic strains over the mass */
        const double* x = &u[3 * ne + 1];
        double* S = &C.sdev[c * 6];
        S[0] = x[0] / u[e];
        S[1] = x[1] / u[e];
        S[3] = x[2] / u[e];
        S[4] = x[3] / u[e];
        S[5] = x[4] / u[e];
        S[2] = -(S[0] + S[1]);
        C.plastic_rate[c] = x[5] / u[ne + e];
        C.plastic[c] = x[6] / u[ne + e];
      }
    }
    C.density.g[c] = dn;
    C.cell_mass.g[c] = C.euler_volume[c] * dn;
    double en = 0., ps = 0.;
    for (int e = 0; e < ne; ++e) {
      if (!C.has(c, e)) continue;
      C.EV(C.cell_mass, e, c) = C.EV(C.mass_fraction, e, c) * C.cell_mass.g[c];
      C.EV(C.pseudo, e, c) = u[3 * ne] * unsurvol;
      C.EV(C.density, e, c) = dens[e];
      C.EV(C.internal_energy, e, c) = ener[e];
      en += C.EV(C.mass_fraction, e, c) * C.EV(C.internal_energy, e, c);
      ps += C.EV(C.fracvol, e, c) * C.EV(C.pseudo, e, c);
    }
    C.internal_energy.g[c] = en;
    C.pseudo.g[c] = ps;
    for (int e = 0; e < ne; ++e) {
      if (!C.has(c, e)) continue;
      if (C.EV(C.density, e, c) < 0. || C.EV(C.internal_energy, e, c) < 0.) {
        C.EV(C.internal_energy, e, c) = 0.;
        C.EV(C.density, e, c) = 0.;
        C.EV(C.fracvol, e, c) = 0.;
        C.EV(C.mass_fraction, e, c) = 0.;
      }
      double r = C.EV(C.density, e, c), ie = C.EV(C.internal_energy, e, c);
      if (r != r || ie != ie) { C.status = ST_NAN; return C.status; }
    }
  }
  for (long n = 0; n < C.nnode && with_dual; ++n) {
    const double* U = &C.u_dual[n * 5];
    double m = U[3];
    if (m != 0.) C.vel[n] = {U[0] / m, U[1] / m, U[2] / m};
  }
  std::fill(C.node_mass.begin(), C.node_mass.end(), 0.);
  const double w = C.dim == 2 ? .25 : .125;
  for (long c = 0; c < C.ncell; ++c) {
    double contrib = w * C.cell_mass.g[c];
    for (int l = 0; l < C.nbn; ++l) C.node_mass[C.cnode(c, l)] += contrib;
    if (!C.pure(c))
      for (int e = 0; e < ne; ++e)
        if (C.has(c, e)) C.EV(C.cell_volume, e, c) = C.EV(C.fracvol, e, c) * C.cell_volume.g[c];
  }
  if (C.P.conservation_energie_totale) {
    /* kinetic energy lost by the dual projection goes back into the
     * internal energy (RemapADIFinal.cc:320-344): 0.25 per node of the
     * difference between the projected and the reconstructed kinetic
     * energy, in cell node order */
    for (long c = 0; c < C.ncell; ++c) {
      double delta = 0.;
      for (int l = 0; l < C.nbn; ++l) {
        const long n = C.cnode(c, l);
        const double* U = &C.u_dual[n * 5];
        if (U[3] != 0.) {
          const double ec_proj = U[4] / U[3];
          const R3 v = C.vel[n];
          const double ec_rec = 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);
          delta += 0.25 * (ec_proj - ec_rec);
        }
      }
      delta = std::max(0., delta);
      for (int e = 0; e < ne; ++e)
        if (C.has(c, e)) C.EV(C.internal_energy, e, c) += C.EV(C.mass_fraction, e, c) * delta;
      if (!C.pure(c)) C.internal_energy.g[c] += delta;
    }
  }
  return ST_OK;
}

/* RemapADIService::computeVolumeEuler (RemapADIService.cc:579-645): the
 * corner normals and volumes of the receiving grid, once the Euler axis of
 * the node positions is back on the initial grid.  The corner normals
 * replace those of the Lagrangian step (the next node pass uses them). */
static void compute_volume_euler(Case& C) {
  for (long c = 0; c < C.ncell; ++c) {
    R3 coord[8];
    gather_cell_coords(C, c, coord);
    if (C.dim == 3) {
      R3 fc[6];
      hex_face_centres(coord, fc);
      compute_cqs3(coord, fc, &C.cqs[c * 8]);
    } else {
      compute_cqs2(coord, &C.cqs[c * 4]);
    }
  }
  for (long c = 0; c < C.ncell; ++c) {
    double volume = 0.;
    for (int n = 0; n < C.nbn; ++n) volume += dot(C.coord[C.cnode(c, n)], C.cqs[c * C.nbn + n]);
    C.euler_volume[c] = volume / C.dim;
  }
}

/* is-euler-scheme X / Y / Z: the only remapped axis (-1 for Full / NON) */
static int euler_axis(const Case& C) {
  const int s = C.P.is_euler_scheme;
  return (s >= MHC_EULER_X && s <= MHC_EULER_Z) ? s - MHC_EULER_X : -1;
}

/* RemapADIService::appliRemap (RemapADIService.cc:15-90) */
static int appli_remap(Case& C) {
  const int axis = euler_axis(C);
  for (int i = 0; i < C.dim; ++i) {
    int d = (i + C.sens_projection) % C.dim;
    if (C.ncd(d) == 1) continue;
    if (axis >= 0 && d != axis) continue;
    compute_grad_phi_face(C, d);
    compute_grad_phi_cell(C, d);
    compute_upwind_face_quantities(C, d);
    compute_uremap(C, d);
    if (!C.P.sans_lagrange) compute_dual_uremap(C, d);
  }
  C.sens_projection = (C.sens_projection + 1) % C.dim;
  if (C.P.is_euler_scheme == MHC_EULER_FULL) {
    C.coord = C.coord0;
  } else if (axis >= 0) {
    for (long n = 0; n < C.nnode; ++n) {
      R3& x = C.coord[n];
      const R3& x0 = C.coord0[n];
      if (axis == 0) x.x = x0.x;
      else if (axis == 1) x.y = x0.y;
      else x.z = x0.z;
    }
    compute_volume_euler(C);
  }
  return remap_variables(C);
}

/* MahycoModule::remap (PrepareRemap.cc:203-251) */
static int remap(Case& C) {
  if (!C.P.with_projection) return ST_OK;
  if (C.P.schema_csts) {
    /* updateVelocityForward (MahycoModule.cc:637-700): n+1/2 to n+1 with the
     * forces of the new pressure, pseudo-viscosity and corner normals */
    for (auto& f : C.force) f = {0., 0., 0.};
    for (long c = 0; c < C.ncell; ++c) {
      double pressure = C.pressure.g[c] + C.pseudo.g[c];
      for (int l = 0; l < C.nbn; ++l) C.force[C.cnode(c, l)] += pressure * C.cqs[c * C.nbn + l];
    }
    const double dt = 0.5 * C.dt;
    R3 g = {C.P.gravity[0], C.P.gravity[1], C.P.gravity[2]};
    for (long n = 0; n < C.nnode; ++n) C.vel[n] += (dt / C.node_mass[n]) * C.force[n];
    for (long n = 0; n < C.nnode; ++n) C.vel[n] += dt * g;
  }
  compute_variables_for_remap(C);
  compute_face_quantities_for_remap(C);
  if (appli_remap(C) != ST_OK) return C.status;
  /* values at n reset after the remap (PrepareRemap.cc:219-226); the
   * pseudo-viscosity at n-1 of the next iteration is therefore 0 */
  C.pseudo_n.fill(0.0);
  C.cell_volume_n.fill(0.0);
  C.pressure_n.fill(0.0);
  C.density_n.fill(0.0);
  C.tau_density.fill(0.0);
  for (int e = 0; e < C.nenv; ++e) eos_apply(C, e);
  compute_pression_moyenne(C);
  return ST_OK;
}

/* MahycoModule::computeDeltaT (MahycoModule.cc:1739-1864) */
static int compute_delta_t(Case& C) {
  C.old_dt = C.dt;
  C.m_old_deltat = C.old_dt;
  double new_dt;
  if (C.P.sans_lagrange || C.P.deltat_constant) {
    new_dt = C.P.deltat_init;
  } else {
    double minimum_aux = 1.7976931348623157e308;
    for (long c = 0; c < C.ncell; ++c) {
      double vmax = 0.;
      if (C.P.is_euler_scheme == MHC_EULER_FULL)
        for (int l = 0; l < C.nbn; ++l) vmax = amax(norm(C.vel[C.cnode(c, l)]), vmax);
      double dx_sound = C.char_len[c] / (C.sound_speed.g[c] + vmax);
      minimum_aux = amin(minimum_aux, dx_sound);
    }
    new_dt = C.P.cfl * minimum_aux;
    new_dt = amin(new_dt, 1.05 * C.old_dt);
    new_dt = amin(new_dt, C.P.deltat_max);
    if (new_dt < C.P.deltat_min) { C.status = ST_DT_UNDERFLOW; return C.status; }
  }
  C.dt = new_dt;
  double stop = C.P.final_time;
  bool not_yet = C.t < stop, finish = C.t > stop, too_much = (C.t + new_dt) > stop;
  if ((not_yet && too_much) || finish) C.stop = true;
  return ST_OK;
}

/* EnvSummationService::write (EnvSummationService.cc:77-169) */
static void time_history_write(Case& C) {
  int period = C.P.time_history_period > 0 ? C.P.time_history_period : 10;
  if (C.iteration % period != 0) return;
  THLine L;
  L.time = C.t;
  for (int e = 0; e < C.nenv; ++e) {
    long cnt = 0;
    double m = 0., p = 0., rv = 0., vv = 0., em = 0., mm = 0.;
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      if (!C.has(c, e)) continue;
      ++cnt;
      m += C.EV(C.cell_mass, e, c);
      p += C.EV(C.pressure, e, c);
    }
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      if (!C.has(c, e)) continue;
      em += C.EV(C.internal_energy, e, c) * C.EV(C.cell_mass, e, c);
      mm += C.EV(C.cell_mass, e, c);
    }
    for (long k = 0; k < C.ncell; ++k) {
      const long c = C.ord(k);
      if (!C.has(c, e)) continue;
      rv += C.EV(C.density, e, c) * C.EV(C.cell_volume, e, c);
      vv += C.EV(C.cell_volume, e, c);
    }
    L.present[e] = cnt > 0;
    L.v[e][0] = m / cnt;
    L.v[e][1] = p / cnt;
    L.v[e][2] = rv / vv;
    L.v[e][3] = em / mm;
  }
  C.th.push_back(L);
}

/* one iteration of the MahycoLoop / MahycoLagrangeLoop compute loop
 * (Mahyco.config:23-36) */
static int iterate(Case& C) {
  C.iteration += 1;
  C.t = C.t + C.dt;
  save_values_at_n(C);
  if (C.P.sans_lagrange) update_velocity_without_lagrange(C);
  else update_velocity(C);
  apply_boundary_condition(C);
  update_position(C);
  if (compute_geometric_values(C) != ST_OK) return C.status;
  /* updateDensity, computeArtificialViscosity,
   * updateElasticityAndPlasticity and updateEnergyAndPressure return at
   * once without Lagrange phase */
  if (!C.P.sans_lagrange) {
    update_density(C);
    compute_artificial_viscosity(C);
    update_elasticity_and_plasticity(C);
    update_energy_and_pressure(C);
  }
  if (remap(C) != ST_OK) return C.status;
  if (compute_delta_t(C) != ST_OK) return C.status;
  time_history_write(C);
  return ST_OK;
}

}  // namespace ora

/* ===========================================================================
 * C interface used by the tests (ctypes)
 * ========================================================================= */
extern "C" {

void* oracle_create(const mhc_case_params* p) {
  ora::Case* C = new ora::Case();
  ora::setup(*C, p);
  return C;
}

void oracle_destroy(void* h) { delete (ora::Case*)h; }

int oracle_init(void* h) { return ora::hydro_start_init(*(ora::Case*)h); }

/* run up to n iterations; stops early on error or when the final time is reached */
int oracle_iterate(void* h, int n) {
  ora::Case& C = *(ora::Case*)h;
  for (int it = 0; it < n; ++it) {
    if (C.status != ora::ST_OK) return C.status;
    if (C.stop) break;
    if (ora::iterate(C) != ora::ST_OK) return C.status;
  }
  return C.status;
}

/* run until the reference time loop would stop (final time) or max_iter */
int oracle_run(void* h, long max_iter) {
  ora::Case& C = *(ora::Case*)h;
  while (!C.stop && C.iteration < max_iter) {
    if (ora::iterate(C) != ora::ST_OK) return C.status;
  }
  return C.status;
}

/* test-only switches: "restart_at" = iteration after which a
 * protection/reprise restart is emulated; "cr_pow" = correctly rounded
 * powers instead of std::pow (process-wide) */
int oracle_set_option(void* h, const char* name, double value) {
  ora::Case& C = *(ora::Case*)h;
  if (!strcmp(name, "restart_at")) { C.restart_at = (long)value; return 0; }
  if (!strcmp(name, "cr_pow")) { ora::g_cr_pow = value != 0.; return 0; }
  return -1;
}

double oracle_scalar(void* h, const char* name) {
  ora::Case& C = *(ora::Case*)h;
  if (!strcmp(name, "time")) return C.t;
  if (!strcmp(name, "deltat")) return C.dt;
  if (!strcmp(name, "old_deltat")) return C.old_dt;
  if (!strcmp(name, "iteration")) return (double)C.iteration;
  if (!strcmp(name, "stop")) return C.stop ? 1. : 0.;
  if (!strcmp(name, "status")) return C.status;
  if (!strcmp(name, "ncell")) return (double)C.ncell;
  if (!strcmp(name, "nnode")) return (double)C.nnode;
  return NAN;
}

static ora::MatField* mat_field(ora::Case& C, const char* name) {
  struct { const char* n; ora::MatField* f; } tab[] = {
      {"Density", &C.density}, {"Pressure", &C.pressure}, {"InternalEnergy", &C.internal_energy},
      {"SoundSpeed", &C.sound_speed}, {"PseudoViscosity", &C.pseudo}, {"CellMass", &C.cell_mass},
      {"CellVolume", &C.cell_volume}, {"FracVol", &C.fracvol}, {"MassFraction", &C.mass_fraction},
      {"DpDe", &C.dpde}, {"TauxDensity", &C.tau_density}, {"Temperature", &C.temperature}};
  for (auto& t : tab)
    if (!strcmp(name, t.n)) return t.f;
  return nullptr;
}

/* env < 0: global cell value; env >= 0: environment value (0 where the cell
 * is not in the environment).  Node Real3 fields are returned interleaved. */
long oracle_get_field(void* h, const char* name, int env, double* out, long cap) {
  ora::Case& C = *(ora::Case*)h;
  if (ora::MatField* f = mat_field(C, name)) {
    if (cap < C.ncell) return -1;
    for (long c = 0; c < C.ncell; ++c) {
      if (env < 0) out[c] = f->g[c];
      else out[c] = C.has(c, env) ? C.EV(*f, env, c) : 0.;
    }
    return C.ncell;
  }
  if (!strcmp(name, "CaracteristicLength") || !strcmp(name, "EulerVolume") || !strcmp(name, "EnvMask")) {
    if (cap < C.ncell) return -1;
    for (long c = 0; c < C.ncell; ++c)
      out[c] = name[0] == 'C' ? C.char_len[c] : (name[0] == 'E' && name[1] == 'u' ? C.euler_volume[c] : (double)C.envmask[c]);
    return C.ncell;
  }
  static const char* kStrain[] = {"StrainTensorXX", "StrainTensorYY", "StrainTensorZZ", "StrainTensorXY",
                                  "StrainTensorYZ", "StrainTensorXZ"};
  for (int q = 0; q < 6; ++q) {
    if (strcmp(name, kStrain[q])) continue;
    if (cap < C.ncell) return -1;
    for (long c = 0; c < C.ncell; ++c) out[c] = C.elasto ? -C.sdev[c * 6 + q] : 0.;
    return C.ncell;
  }
  if (!strcmp(name, "PlasticDeformation") || !strcmp(name, "PlasticDeformationVelocity") ||
      !strcmp(name, "StrainNorm")) {
    if (cap < C.ncell) return -1;
    const std::vector<double>& v = name[0] == 'S' ? C.strain_norm : (name[18] == 'V' ? C.plastic_rate : C.plastic);
    for (long c = 0; c < C.ncell; ++c) out[c] = v.empty() ? 0. : v[c];
    return C.ncell;
  }
  if (!strcmp(name, "NodeMass")) {
    if (cap < C.nnode) return -1;
    for (long n = 0; n < C.nnode; ++n) out[n] = C.node_mass[n];
    return C.nnode;
  }
  const bool vn = !strcmp(name, "VelocityN");
  if (!strcmp(name, "Velocity") || !strcmp(name, "NodeCoord") || !strcmp(name, "CellCoord") || vn) {
    bool cc = !strcmp(name, "CellCoord");
    long n_ = cc ? C.ncell : C.nnode;
    if (cap < 3 * n_) return -1;
    const std::vector<ora::R3>& v = cc ? C.cell_coord : (vn ? C.vel_n : (name[0] == 'V' ? C.vel : C.coord));
    for (long n = 0; n < n_; ++n) { out[3 * n] = v[n].x; out[3 * n + 1] = v[n].y; out[3 * n + 2] = v[n].z; }
    return 3 * n_;
  }
  return -2;
}

/* the inverse of oracle_get_field for the state a host can upload: env < 0
 * writes the global cell value, env >= 0 the environment value of the cells
 * that hold env (EV: the global slot where env is alone); node Real3 fields
 * interleaved.  Returns the number of values read, < 0 for an unknown or
 * read-only name. */
long oracle_set_field(void* h, const char* name, int env, const double* in, long n) {
  ora::Case& C = *(ora::Case*)h;
  if (ora::MatField* f = mat_field(C, name)) {
    if (n < C.ncell) return -1;
    for (long c = 0; c < C.ncell; ++c) {
      if (env < 0) f->g[c] = in[c];
      else if (C.has(c, env)) C.EV(*f, env, c) = in[c];
    }
    return C.ncell;
  }
  if (!strcmp(name, "NodeMass")) {
    if (n < C.nnode) return -1;
    for (long i = 0; i < C.nnode; ++i) C.node_mass[i] = in[i];
    return C.nnode;
  }
  if (!strcmp(name, "Velocity") || !strcmp(name, "VelocityN")) {
    /* VelocityN: m_velocity_n, the prescribed velocities of a sans-lagrange run */
    if (n < 3 * C.nnode) return -1;
    std::vector<ora::R3>& v = name[8] == 'N' ? C.vel_n : C.vel;
    for (long i = 0; i < C.nnode; ++i) v[i] = ora::R3{in[3 * i], in[3 * i + 1], in[3 * i + 2]};
    return 3 * C.nnode;
  }
  return -2;
}

/* initial state of the EXTERNAL case model and node coordinates read from a
 * mesh file, before oracle_init: NodeCoord (3 per node, interleaved),
 * Materiau, Density, Pressure (one per cell) */
int oracle_set_initial_field(void* h, const char* name, const double* in, long n) {
  ora::Case& C = *(ora::Case*)h;
  if (!strcmp(name, "NodeCoord")) {
    if (n < 3 * C.nnode) return -1;
    for (long i = 0; i < C.nnode; ++i) C.coord[i] = ora::R3{in[3 * i], in[3 * i + 1], in[3 * i + 2]};
    return 3 * C.nnode;
  }
  std::vector<double>* v = !strcmp(name, "Materiau") ? &C.init_mat
                           : !strcmp(name, "Density") ? &C.init_rho
                           : !strcmp(name, "Pressure") ? &C.init_p : nullptr;
  if (!v) return -2;
  if (n < C.ncell) return -1;
  v->assign(in, in + C.ncell);
  return C.ncell;
}

/* IEquationOfState::applyEOS(env) on the current state, then
 * computePressionMoyenne on the mixed cells that hold env (the sequence the
 * library's mhc_eos_apply entry point runs) */
int oracle_eos_apply(void* h, int env) {
  ora::Case& C = *(ora::Case*)h;
  if (env < 0 || env >= C.nenv) return -1;
  /* the library's entry point leaves the temperature (it does not keep the
   * energy at the start of the iteration that the update needs) */
  ora::eos_apply(C, env, false);
  double option = C.P.calcul_vitson_max ? 1. : 0.;
  for (long c = 0; c < C.ncell; ++c) {
    if (C.pure(c) || !C.has(c, env)) continue;
    C.pressure.g[c] = 0.;
    C.sound_speed.g[c] = 0.;
    for (int e = 0; e < C.nenv; ++e) {
      if (!C.has(c, e)) continue;
      C.pressure.g[c] += C.EV(C.fracvol, e, c) * C.EV(C.pressure, e, c);
      C.sound_speed.g[c] = option * std::max(C.EV(C.sound_speed, e, c), C.sound_speed.g[c]);
      C.sound_speed.g[c] += (1. - option) * C.EV(C.fracvol, e, c) * C.EV(C.sound_speed, e, c);
    }
  }
  return 0;
}

/* known-answer hooks for the oracle's own unit tests */
double oracle_flux_limiter(int id, double r) { return ora::flux_limiter(id, r); }
double oracle_limited_gradient(int id, double gb, double gf) { return ora::limited_gradient(id, gb, gf); }
void oracle_eos_point(const mhc_env_params* o, double rho, double e, double* p, double* c, double* dpde) {
  mhc_case_params P;
  memset(&P, 0, sizeof(P));
  P.dim = 2; P.nx = 1; P.ny = 1; P.lx = P.ly = 1.; P.nb_env = 1; P.env[0] = *o;
  ora::Case C;
  ora::setup(C, &P);
  C.density.g[0] = rho;
  C.internal_energy.g[0] = e;
  ora::eos_apply(C, 0, false);
  *p = C.pressure.g[0];
  *c = C.sound_speed.g[0];
  *dpde = C.dpde.g[0];
}

/* the oracle's correctly rounded x^(1./3.), for its own unit test */
double oracle_pow_third_cr(double x) { return ora::pow_third_cr(x); }
double oracle_cube_cr(double x) { return ora::cube_cr(x); }
double oracle_pow_five_thirds_cr(double x) { return ora::pow_five_thirds_cr(x); }

/* number of time-history lines recorded so far */
long oracle_th_count(void* h) { return (long)((ora::Case*)h)->th.size(); }

/* line i: out[0]=time, then per env 4 values (CellMass, Pressure, Density,
 * InternalEnergy) and a presence flag: 1 + 5*nb_env doubles */
int oracle_th_line(void* h, long i, double* out) {
  ora::Case& C = *(ora::Case*)h;
  if (i < 0 || i >= (long)C.th.size()) return -1;
  const ora::THLine& L = C.th[i];
  out[0] = L.time;
  for (int e = 0; e < C.nenv; ++e) {
    for (int q = 0; q < 4; ++q) out[1 + 5 * e + q] = L.v[e][q];
    out[1 + 5 * e + 4] = L.present[e];
  }
  return 0;
}

}  /* extern "C" */
