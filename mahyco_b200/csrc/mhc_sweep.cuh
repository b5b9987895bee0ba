// mhc_sweep.cuh -- one direction of the ADI remap (cells, then nodes)
// without shared memory or barriers.
//
// A warp holds 32 consecutive cells along the sweep direction, one per
// lane; every intermediate of the reference -- phi, face gradient, limited
// cell gradient, upwind face value, face flux -- is computed once per cell
// or face and handed to the neighbour lane by a shuffle.  The 4 warps of a
// block hold neighbouring transverse columns, so for the y and z sweeps the
// block reads whole 32-byte sectors of every row it touches.
//
// Arithmetic and operation order are those of computeGradPhiFace,
// computeGradPhiCell, computeUpwindFaceQuantitiesForProjection and
// computeUremap (RemapADIService.cc:119-575, UtilesRemap.cc:108-120,
// 325-357); face quantities of the Lagrangian mesh (PrepareRemap.cc:18-59)
// are rebuilt from the node positions.  The initial face normals of the
// cartesian grid are unit axis vectors, so dot(., n) is the D component.
#pragma once
#include "mhc_kernels.cuh"

namespace mhc {

struct SweepArgs {
  const double* Uin;
  double* Uout;
  int first;
  int order;
  int limiter;
  int simple_pente;   // projection-simple-pente (generalised limiters)
  int first_remap;    // first remap of the run: every cell counts as pure
};

// face node q (in the order of the reference face, smallest node id first)
// of the face normal to D whose lowest node is (i, j, k)
template <int DIM, int D>
__device__ __forceinline__ void face_node_ijk2(int i, int j, int k, int q, int& a, int& b, int& cz) {
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


constexpr int SW_LANES = 32; // cells along D per warp
#ifndef MHC_SW_ROWS
#define MHC_SW_ROWS 4
#endif
constexpr int SW_ROWS = MHC_SW_ROWS;  // warps (transverse rows) per block
constexpr int SW_THREADS = SW_LANES * SW_ROWS;
constexpr int XOUT = 27;     // cells written per warp (lanes 2 .. 28)
constexpr int XOUT_W = 26;   // wide stencils (3 halo lanes each side): lanes 3 .. 28

// ---------------------------------------------------------------------------
// Initial-grid quantities of the outer normals, one coordinate at a time.
// Node coordinate A of the initial grid depends on the node index along A
// only, so the sums of the reference (cell centre over the local nodes,
// face centre over the face nodes, in their orders) are rebuilt from the
// two coordinate values c0 (offset 0) and c1 (offset 1).
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ double grid_coord(const Mesh& M, int A, int idx) {
  return (DIM == 2 && A == 2) ? 0. : M.o[A] + idx * M.h[A];
}

// component A of the initial cell centre (wc * sum over local nodes)
template <int DIM, int A>
__device__ __forceinline__ double cc0_comp(const Mesh& M, int idx) {
  if (DIM == 2 && A == 2) return 0.;
  const double c0 = grid_coord<DIM>(M, A, idx), c1 = grid_coord<DIM>(M, A, idx + 1);
  double s = 0.;
#pragma unroll
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    int da, db, dc;
    local_node_offset(l, da, db, dc);
    s += (A == 0 ? da : (A == 1 ? db : dc)) ? c1 : c0;
  }
  return (DIM == 2 ? .25 : .125) * s;
}

// component A of the initial centre of a face normal to D (sum over the
// face nodes of wf * coordinate)
template <int DIM, int D, int A>
__device__ __forceinline__ double fc0_comp(const Mesh& M, int idx) {
  if (DIM == 2 && A == 2) return 0.;
  const double wf = DIM == 2 ? .5 : .25;
  const double c0 = grid_coord<DIM>(M, A, idx), c1 = grid_coord<DIM>(M, A, idx + 1);
  double s = 0.;
#pragma unroll
  for (int q = 0; q < (DIM == 3 ? 4 : 2); ++q) {
    int a, b, cz;
    face_node_ijk2<DIM, D>(0, 0, 0, q, a, b, cz);
    const int off = A == 0 ? a : (A == 1 ? b : cz);
    s = s + wf * ((A == D) ? c0 : (off ? c1 : c0));
  }
  return s;
}

// D component of the unit outer normal: diff_D / |diff| with the sum of
// squares in x, y, z order
template <int D>
__device__ __forceinline__ double unit_comp(double dD, double t0, double t1) {
  // t0, t1: transverse differences in increasing axis order
  double ss;
  if (D == 0) ss = dD * dD + t0 * t0 + t1 * t1;
  else if (D == 1) ss = t0 * t0 + dD * dD + t1 * t1;
  else ss = t0 * t0 + t1 * t1 + dD * dD;
  return dD / sqrt(ss);
}

// face-node slot q (face_node_ijk2 order) of local node l of a cell, and
// whether l sits on the front plane along D
template <int DIM, int D>
__device__ __forceinline__ void local_to_plane(int l, int& q, int& front) {
  int da, db, dc;
  local_node_offset(l, da, db, dc);
  int s1, s2;
  if (D == 0) { front = da; s1 = db; s2 = dc; }
  else if (D == 1) { front = db; s1 = da; s2 = dc; }
  else { front = dc; s1 = da; s2 = db; }
  if (DIM == 2) s2 = 0;
  q = s2 ? (s1 ? 2 : 3) : (s1 ? 1 : 0);
}

// Lagrangian plane data: the D coordinates of the face nodes, and the face
// centre, normal velocity and length of the face (PrepareRemap.cc:18-59)
template <int DIM> struct Plane {
  double xd[DIM == 3 ? 4 : 2];
  double fc, un, L;
};

template <int DIM, int D>
__device__ __forceinline__ void load_plane(const Mesh& M, const Fields& F, int i, int j, int k, Plane<DIM>& P) {
  constexpr int NQ = DIM == 3 ? 4 : 2;
  const double wf = DIM == 2 ? .5 : .25;
  const double* vD = F.fv[D];  // the node velocities, or (CSTS) their means at n and n+1
  long long fn[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    int a, b, cz;
    face_node_ijk2<DIM, D>(i, j, k, q, a, b, cz);
    fn[q] = node_id(M, a, b, cz);
  }
  double vm = 0.;
  P.fc = 0.;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    P.xd[q] = __ldg(F.Xn[D] + fn[q]);
    P.fc = P.fc + wf * P.xd[q];
    vm = vm + __ldg(vD + fn[q]);
  }
  P.un = wf * vm;
  if (DIM == 3) {
    R3 x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      x[q].x = D == 0 ? P.xd[q] : __ldg(F.Xn[0] + fn[q]);
      x[q].y = D == 1 ? P.xd[q] : __ldg(F.Xn[1] + fn[q]);
      x[q].z = D == 2 ? P.xd[q] : __ldg(F.Xn[2] + fn[q]);
    }
    const R3 v1 = x[2] - x[0], v2 = x[3] - x[1];
    if (D == 0) P.L = 0.5 * fabs(produit(v1.y, v2.z, v1.z, v2.y));
    else if (D == 1) P.L = 0.5 * fabs(produit(v2.x, v1.z, v2.z, v1.x));
    else P.L = 0.5 * fabs(produit(v1.x, v2.y, v1.y, v2.x));
  } else {
    const double* Xt = F.Xn[1 - D];
    P.L = fabs(__ldg(Xt + fn[1]) - __ldg(Xt + fn[0]));
  }
}

// Lagrangian cell centre along D from its back (B) and front (Fr) planes,
// summed in local node order
template <int DIM, int D>
__device__ __forceinline__ double centre_from_planes(const Plane<DIM>& B, const Plane<DIM>& Fr) {
  double s = 0.;
#pragma unroll
  for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
    int q, front;
    local_to_plane<DIM, D>(l, q, front);
    s += front ? Fr.xd[q] : B.xd[q];
  }
  return (DIM == 2 ? .25 : .125) * s;
}

// ---------------------------------------------------------------------------
// Lane layout of a sweep along D over an nx x ny x nz array of cells or
// nodes.  The array is cut into lines along D; consecutive lines are
// concatenated so that every warp window holds `out` written elements plus
// `hl` halo elements before them (2, or 3 for the wide stencils) and the
// rest after them, whatever the line length.
//  * D = 0: lines are consecutive in memory; window w = vbx * SW_ROWS + row
//    covers flat positions [w*out - hl, w*out - hl + 32).
//  * D = 1, 2: warp `row` of the block owns x column ta = vbx * SW_ROWS +
//    row and walks the lines of that column (slow transverse index tb, then
//    p along D) in windows vby; the 4 warps of a block hold neighbouring x
//    columns at the same positions, so each row of the block is one or two
//    32-byte sectors, and consecutive blocks (vbx fastest) hold the
//    neighbouring columns, so the SMs that run them at the same time read
//    whole DRAM bursts together.
// Returns false when the lane holds nothing; p is the index along D and
// (ta, tb) the transverse indices in increasing axis order.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ bool sweep_lane(int nx, int ny, int nz, int out, int hl, int vbx, int vby, int lane,
                                           int row, int& i, int& j, int& k, int& p, int& ta, int& tb) {
  i = j = k = p = ta = tb = 0;
  // positions in unsigned 32-bit arithmetic (a case has < 2^31 cells)
  if (D == 0) {
    const int g = (vbx * SW_ROWS + row) * out - hl + lane;
    if (g < 0 || g >= nx * ny * nz) return false;
    const unsigned r = (unsigned)g / (unsigned)nx;
    i = (int)((unsigned)g - r * (unsigned)nx);
    k = (int)(r / (unsigned)ny);
    j = (int)(r - (unsigned)k * (unsigned)ny);
    p = i; ta = j; tb = k;
    return true;
  }
  const int nd = D == 1 ? ny : nz, nb = D == 1 ? nz : ny;
  ta = vbx * SW_ROWS + row;
  const int g = vby * out - hl + lane;
  if (ta >= nx || g < 0 || g >= nb * nd) return false;
  tb = (int)((unsigned)g / (unsigned)nd);
  p = g - tb * nd;
  i = ta;
  if (D == 1) { j = p; k = tb; }
  else { j = tb; k = p; }
  return true;
}

// the whole warp holds nothing (warp-uniform test, before any shuffle)
template <int D>
__device__ __forceinline__ bool sweep_warp_empty(int nx, int ny, int nz, int out, int hl, int vbx, int vby, int row) {
  if (D == 0) return (vbx * SW_ROWS + row) * out - hl >= nx * ny * nz;
  const int nd = D == 1 ? ny : nz, nb = D == 1 ? nz : ny;
  return vbx * SW_ROWS + row >= nx || vby * out - hl >= nb * nd;
}

// D coordinates of the face nodes of the node plane whose lowest node is
// (i, j, k)
template <int DIM, int D>
__device__ __forceinline__ void load_plane_xd(const Mesh& M, const Fields& F, int i, int j, int k, Plane<DIM>& P) {
#pragma unroll
  for (int q = 0; q < (DIM == 3 ? 4 : 2); ++q) {
    int a, b, cz;
    face_node_ijk2<DIM, D>(i, j, k, q, a, b, cz);
    P.xd[q] = __ldg(F.Xn[D] + node_id(M, a, b, cz));
  }
}

// all coordinates of the face nodes of the node plane whose lowest node is
// (i, j, k); z = 0 in 2D
template <int DIM, int D>
__device__ __forceinline__ void load_plane_full(const Mesh& M, const Fields& F, int i, int j, int k,
                                                double (&x)[DIM == 3 ? 4 : 2][3]) {
#pragma unroll
  for (int q = 0; q < (DIM == 3 ? 4 : 2); ++q) {
    int a, b, cz;
    face_node_ijk2<DIM, D>(i, j, k, q, a, b, cz);
    const long long n = node_id(M, a, b, cz);
    x[q][0] = __ldg(F.Xn[0] + n);
    x[q][1] = __ldg(F.Xn[1] + n);
    x[q][2] = DIM == 3 ? __ldg(F.Xn[2] + n) : 0.;
  }
}

__device__ __forceinline__ double norm3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

// Width of the lane's cell along D (m_h_cell_lagrange,
// RemapADIService.cc:141-143): distance from the Lagrangian cell centre to
// the centres of its inner faces of direction D, back face first.  Every
// lane of the warp calls it (the front plane comes from lane + 1).
template <int DIM, int D>
__device__ __forceinline__ double lane_cell_width(const Mesh& M, const Fields& F, bool ok, int i, int j, int k,
                                                  int p, int nd) {
  constexpr int NQ = DIM == 3 ? 4 : 2;
  constexpr unsigned FULL = 0xffffffffu;
  double b[NQ][3], f[NQ][3];
  if (ok) load_plane_full<DIM, D>(M, F, i, j, k, b);
  else {
#pragma unroll
    for (int q = 0; q < NQ; ++q) b[q][0] = b[q][1] = b[q][2] = 0.;
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int a = 0; a < 3; ++a) f[q][a] = __shfl_down_sync(FULL, b[q][a], 1);
  // the front plane is loaded at the end of a line, and by the last lane,
  // whose next cell lies outside the warp
  if (ok && (p == nd - 1 || (threadIdx.x % SW_LANES) == SW_LANES - 1))
    load_plane_full<DIM, D>(M, F, D == 0 ? i + 1 : i, D == 1 ? j + 1 : j, D == 2 ? k + 1 : k, f);
  if (!ok) return 0.;
  const double wf = DIM == 2 ? .5 : .25, wc = DIM == 2 ? .25 : .125;
  double cc[3], fb[3], ff[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double s = 0.;
#pragma unroll
    for (int l = 0; l < (DIM == 3 ? 8 : 4); ++l) {
      int q, front;
      local_to_plane<DIM, D>(l, q, front);
      s += front ? f[q][a] : b[q][a];
    }
    cc[a] = wc * s;
    fb[a] = ff[a] = 0.;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      fb[a] = fb[a] + wf * b[q][a];
      ff[a] = ff[a] + wf * f[q][a];
    }
  }
  double h = 0.;
  if (p > 0) h += norm3(fb[0] - cc[0], fb[1] - cc[1], fb[2] - cc[2]);
  if (p < nd - 1) h += norm3(ff[0] - cc[0], ff[1] - cc[1], ff[2] - cc[2]);
  return h;
}

// ---------------------------------------------------------------------------
// Cell sweep along D with warp shuffles.  A warp holds 32 consecutive cells
// along D (lane l: cell x0 - 2 + l), loads the back node plane of each and
// takes the front plane from lane l+1; stencil neighbours come from lanes
// l-1 / l+1.  Lanes 2 .. XOUT+1 write.  Virtual block: x = window index
// along D, y = group of SW_ROWS rows.  Rows are the transverse cells with
// the lowest transverse axis fastest, so the warps of a block read
// neighbouring columns and share L1 sectors.
// ---------------------------------------------------------------------------
// XV: further projected variables after the pseudo-viscosity (the
// deviator and plastic strains of an elasto-plastic case), remapped like it
template <int DIM, int NE, int D, int LIM, int XV = 0>
__device__ __forceinline__ void body_sweep_cells_lanes(const Mesh& M, const Fields& F, const SweepArgs& A,
                                                       int vbx, int vby) {
  constexpr int NV = 3 * NE + 1 + XV;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  constexpr unsigned FULL = 0xffffffffu;
  const long long N = M.ncell;
  const int lane = threadIdx.x % SW_LANES, row = threadIdx.x / SW_LANES;
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  if (sweep_warp_empty<D>(M.ncx, M.ncy, M.ncz, XOUT, 2, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, p, ta, tb;
  const bool ok = sweep_lane<D>(M.ncx, M.ncy, M.ncz, XOUT, 2, vbx, vby, lane, row, i, j, k, p, ta, tb);
  const bool out = ok && lane >= 2 && lane < 2 + XOUT;
  const double dt = F.s->dt;
  const int order2 = LIM == LIM_ORDER1 ? 0 : 1;  // ordre-projection - 1
  const double* __restrict__ Uin = A.Uin;
  // back node plane of the own cell; the front plane is the back plane of
  // the next lane, except at the end of a line
  Plane<DIM> back;
  if (ok) load_plane<DIM, D>(M, F, i, j, k, back);
  else {
#pragma unroll
    for (int q = 0; q < NQ; ++q) back.xd[q] = 0.;
    back.fc = back.un = back.L = 0.;
  }
  Plane<DIM> front;
#pragma unroll
  for (int q = 0; q < NQ; ++q) front.xd[q] = __shfl_down_sync(FULL, back.xd[q], 1);
  if (ok && p == nd - 1)
    load_plane_xd<DIM, D>(M, F, D == 0 ? i + 1 : i, D == 1 ? j + 1 : j, D == 2 ? k + 1 : k, front);
  long long c = 0;
  double u[NV], den = 1., xc = 0., ondB = 0., ondF = 0.;
  if (ok) {
    c = cell_id(M, i, j, k);
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = __ldg(Uin + v * N + c);
    if (A.first) {
      den = __ldg(F.V + c);
    } else {
      den = 0.;
#pragma unroll
      for (int q = 0; q < NE; ++q) den += u[q];
    }
    xc = centre_from_planes<DIM, D>(back, front);
    if (out) {
      // outer normals of the back and front faces (initial grid)
      constexpr int A0 = D == 0 ? 1 : 0, A1 = D == 2 ? 1 : 2;
      const double t0 = fc0_comp<DIM, D, A0>(M, ta) - cc0_comp<DIM, A0>(M, ta);
      const double t1 = fc0_comp<DIM, D, A1>(M, tb) - cc0_comp<DIM, A1>(M, tb);
      const double cc0 = cc0_comp<DIM, D>(M, p);
      ondB = unit_comp<D>(fc0_comp<DIM, D, D>(M, p) - cc0, t0, t1);
      ondF = unit_comp<D>(fc0_comp<DIM, D, D>(M, p + 1) - cc0, t0, t1);
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = 0.;
  }
  // widths of the own and neighbouring cells (generalised limiters only)
  double hw = 0., hw_l = 0., hw_r = 0.;
  if constexpr (LIM == LIM_GEN) {
    hw = lane_cell_width<DIM, D>(M, F, ok, i, j, k, p, nd);
    hw_l = __shfl_up_sync(FULL, hw, 1);
    hw_r = __shfl_down_sync(FULL, hw, 1);
    if (p == 0) hw_l = hw;
    if (p == nd - 1) hw_r = hw;
  }
  const double fc = back.fc, un = back.un, L = back.L;  // back face of the cell
  const bool ok_l = __shfl_up_sync(FULL, ok, 1) && lane > 0 && p > 0;  // same line
  const double xc_l = __shfl_up_sync(FULL, xc, 1);
  const bool face_b = ok && ok_l;                       // face between p-1 and p
  const bool face_f = __shfl_down_sync(FULL, face_b, 1) && lane < 31;
  const double un_r = __shfl_down_sync(FULL, un, 1), L_r = __shfl_down_sync(FULL, L, 1);
  const double dxb = xc - xc_l;
  const bool up_left = un * dxb > 0.0;
  // cell local face order: along x in 2D front then back, otherwise back
  // then front
  constexpr bool FRONT_FIRST = DIM == 2 && D == 0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double phi = ok ? div_rn(u[v], den) : 0.;
    const double phi_l = __shfl_up_sync(FULL, phi, 1);
    const double gf = face_b ? div_rn(phi - phi_l, dxb) : 0.;
    const double gf_r = __shfl_down_sync(FULL, gf, 1);
    double gr;
    if constexpr (LIM == LIM_GEN) {
      // back / front neighbours, the cell itself at the line ends
      const double phi_r = __shfl_down_sync(FULL, phi, 1);
      const double ym = p > 0 ? phi_l : phi, yp = p < nd - 1 ? phi_r : phi;
      gr = ok ? generalized_gradient(A.limiter, gf_r, gf, yp, ym, hw, hw_r, hw_l, A.simple_pente) : 0.;
    } else {
      gr = (LIM != LIM_ORDER1 && ok) ? limited_gradient_t<LIM>(gf, gf_r) : 0.;
    }
    const double gr_l = __shfl_up_sync(FULL, gr, 1);
    double pf = 0.;
    if (face_b) pf = up_left ? phi_l + order2 * (fc - xc_l) * gr_l : phi + order2 * (fc - xc) * gr;
    const double pf_r = __shfl_down_sync(FULL, pf, 1);
    if (out) {
      const double fB = face_b ? ondB * un * L * dt * pf : 0.;
      const double fF = face_f ? ondF * un_r * L_r * dt * pf_r : 0.;
      double sumf = 0., dual = 0.;
      if (FRONT_FIRST) {
        if (face_f) { sumf += fF; dual += 0.5 * fF * ondF; }
        if (face_b) { sumf += fB; dual += 0.5 * fB * ondB; }
      } else {
        if (face_b) { sumf += fB; dual += 0.5 * fB * ondB; }
        if (face_f) { sumf += fF; dual += 0.5 * fF * ondF; }
      }
      double uo = u[v] - sumf;
      if (v >= NE && v < 3 * NE && uo < 0.) uo = 0.;  // masses and energies stay >= 0
      A.Uout[v * N + c] = uo;
      if (v >= NE && v < 2 * NE) F.mflux[(v - NE) * N + c] = dual;
    }
  }
}

// ---------------------------------------------------------------------------
// Pente-borne fluxes (UtilesRemap.cc:84-96 INTY, 190-312 computeY0 /
// computexgxd / computeygyd, 417-832 computeFluxPP / computeFluxPPPure):
// the flux of one variable out of a cell through its back (type 0) or front
// (type 1) face is the integral, over the length swept in deltat, of a
// three-piece reconstruction bounded by the neighbours.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pb_inty(double X, double x0, double y0, double x1, double y1, double thr) {
  double flux = 0.;
  if (fabs(x1 - x0) > thr) {
    const double eta = amin(amax(0., (X - x0) / (x1 - x0)), 1.);
    flux = (y0 + 0.5 * eta * (y1 - y0)) * (x1 - x0) * eta;
  }
  return flux;
}

__device__ __forceinline__ void pb_y0(int id, double yp, double ym, double h0, double hp, double hm, int simple_pente,
                                      double& y0p, double& y0m) {
  y0p = 0.; y0m = 0.;
  if (id == 3 || id == 0) {
    y0p = yp; y0m = ym;
  } else if (id == 4 || id == 1) {
    y0p = ((h0 + hm) * yp + h0 * ym) / (2 * h0 + hm);
    y0m = ((h0 + hp) * ym + h0 * yp) / (2 * h0 + hp);
  } else if (id == 5 || id == 2) {
    const double a = amin(yp, ym), b = amax(yp, ym);
    double xp = (h0 * h0 + 3 * h0 * hm + 2 * hm * hm) * yp;
    double xm = (h0 * h0 + 3 * h0 * hp + 2 * hp * hp) * ym;
    xp += (h0 * h0 - h0 * hp - 2 * hp * hp + 2 * h0 * hm) * ym;
    xm += (h0 * h0 - h0 * hm - 2 * hm * hm + 2 * h0 * hp) * yp;
    xp /= (2 * h0 * h0 + 5 * h0 * hm + 2 * hm * hm - h0 * hp - 2 * hp * hp);
    xm /= (2 * h0 * h0 + 5 * h0 * hp + 2 * hp * hp - h0 * hm - 2 * hm * hm);
    y0p = amin(amax(xp, a), b);
    y0m = amin(amax(xm, a), b);
  } else if (id == 7) {
    y0p = (yp + ym) / 2.;
    y0m = (yp + ym) / 2.;
  } else if (id == 6) {
    y0p = ((h0 + hm + hp) * yp + h0 * ym) / (2 * h0 + hm + hp);
    y0m = ((h0 + hm + hp) * ym + h0 * yp) / (2 * h0 + hm + hp);
  }
  if (simple_pente) { y0p = yp; y0m = ym; }
}

__device__ __forceinline__ double pb_flux(int type, double y0, double yp, double ym, double h0, double hp, double hm,
                                          double grad, double ppv, int lim, int simple_pente, double thr) {
  double y0p, y0m;
  pb_y0(lim, yp, ym, h0, hp, hm, simple_pente, y0p, y0m);
  double xplus = 1., xmoins = 1.;
  if (fabs(y0p - yp) > thr) xplus = (y0 - yp) / (y0p - yp) - 1. / 2.;
  if (fabs(y0m - ym) > thr) xmoins = (y0 - ym) / (y0m - ym) - 1. / 2.;
  const double xd = +h0 * amin(amax(xplus, -1. / 2.), 1. / 2.);
  const double xg = -h0 * amin(amax(xmoins, -1. / 2.), 1. / 2.);
  const double xtd = y0 + h0 / 2 * grad, xtg = y0 - h0 / 2 * grad;
  const double ad = amin(yp, 2. * y0m - ym), bd = amax(yp, 2. * y0m - ym);
  const double ag = amin(ym, 2. * y0p - yp), bg = amax(ym, 2. * y0p - yp);
  const double yd = amin(amax(xtd, ad), bd), yg = amin(amax(xtg, ag), bg);
  double f1, f1m, f2, f2m, f3, f3m;
  if (type == 0) {
    const double X = -h0 / 2. + ppv, X0 = -h0 / 2.;
    f1m = pb_inty(X, -h0 / 2., ym, xg, yg, thr);
    f1 = pb_inty(X0, -h0 / 2., ym, xg, yg, thr);
    f2m = pb_inty(X, xg, yg, xd, yd, thr);
    f2 = pb_inty(X0, xg, yg, xd, yd, thr);
    f3m = pb_inty(X, xd, yd, h0 / 2., yp, thr);
    f3 = pb_inty(X0, xd, yd, h0 / 2., yp, thr);
  } else {
    const double X = h0 / 2. - ppv, X1 = h0 / 2.;
    f1 = pb_inty(X, -h0 / 2., ym, xg, yg, thr);
    f1m = pb_inty(X1, -h0 / 2., ym, xg, yg, thr);
    f2 = pb_inty(X, xg, yg, xd, yd, thr);
    f2m = pb_inty(X1, xg, yg, xd, yd, thr);
    f3 = pb_inty(X, xd, yd, h0 / 2., yp, thr);
    f3m = pb_inty(X1, xd, yd, h0 / 2., yp, thr);
  }
  double F = smax(((f1m - f1) + (f2m - f2) + (f3m - f3)), 0.);
  if (((yp - y0) * (ym - y0)) >= 0.) F = y0 * ppv;  // extremum: formule 16
  return F;
}

// ---------------------------------------------------------------------------
// Cell sweep along D with the pente-borne fluxes (computeGradPhiCell,
// computeUpwindFaceQuantitiesForProjection, computeUremap with
// projection-pente-borne, RemapADIService.cc:196-266, 314-318, 419-530).
// The lane layout of the classical sweep (2 halo lanes).  Every lane computes
// the fluxes out of its cell through both faces; the value of the face
// between lanes l-1 and l is front(l-1) - back(l).  The projected values
// (phi) are the volume fraction, density and specific internal energy per
// environment and the pseudo-viscosity, read from phi_pb on the first sweep
// of a remap and rebuilt from the projected quantities on the others.
// ---------------------------------------------------------------------------
template <int DIM, int NE, int D>
__device__ __forceinline__ void body_sweep_cells_pb(const Mesh& M, const Fields& F, const mhc_case_params& P,
                                                    const SweepArgs& A, int vbx, int vby) {
  constexpr int NV = 3 * NE + 1;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  constexpr unsigned FULL = 0xffffffffu;
  const long long N = M.ncell;
  const int lane = threadIdx.x % SW_LANES, row = threadIdx.x / SW_LANES;
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  if (sweep_warp_empty<D>(M.ncx, M.ncy, M.ncz, XOUT, 2, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, p, ta, tb;
  const bool ok = sweep_lane<D>(M.ncx, M.ncy, M.ncz, XOUT, 2, vbx, vby, lane, row, i, j, k, p, ta, tb);
  const bool out = ok && lane >= 2 && lane < 2 + XOUT;
  const double dt = F.s->dt;
  const double thr = P.remap_threshold;
  const int fix = P.projection_pente_borne_debar_fix;
  const double* __restrict__ Uin = A.Uin;
  Plane<DIM> back;
  if (ok) load_plane<DIM, D>(M, F, i, j, k, back);
  else {
#pragma unroll
    for (int q = 0; q < NQ; ++q) back.xd[q] = 0.;
    back.fc = back.un = back.L = 0.;
  }
  Plane<DIM> front;
#pragma unroll
  for (int q = 0; q < NQ; ++q) front.xd[q] = __shfl_down_sync(FULL, back.xd[q], 1);
  if (ok && p == nd - 1)
    load_plane_xd<DIM, D>(M, F, D == 0 ? i + 1 : i, D == 1 ? j + 1 : j, D == 2 ? k + 1 : k, front);
  long long c = 0;
  double u[NV], ph[NV], xc = 0., ondB = 0., ondF = 0.;
  uint8_t mask = 0;
  if (ok) {
    c = cell_id(M, i, j, k);
    mask = F.mask[c];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = __ldg(Uin + v * N + c);
    if (A.first) {
#pragma unroll
      for (int v = 0; v < NV; ++v) ph[v] = __ldg(F.phi_pb + v * N + c);
    } else {
      double sv = 0.;
#pragma unroll
      for (int q = 0; q < NE; ++q) sv += u[q];
#pragma unroll
      for (int q = 0; q < NE; ++q) {
        ph[q] = div_rn(u[q], sv);
        ph[NE + q] = u[q] != 0. ? div_rn(u[NE + q], u[q]) : 0.;
        ph[2 * NE + q] = u[NE + q] != 0. ? div_rn(u[2 * NE + q], u[NE + q]) : 0.;
      }
      ph[NV - 1] = __ldg(F.phi_pb + (NV - 1) * N + c);  // the pseudo-viscosity is not rebuilt
    }
    xc = centre_from_planes<DIM, D>(back, front);
    constexpr int A0 = D == 0 ? 1 : 0, A1 = D == 2 ? 1 : 2;
    const double t0 = fc0_comp<DIM, D, A0>(M, ta) - cc0_comp<DIM, A0>(M, ta);
    const double t1 = fc0_comp<DIM, D, A1>(M, tb) - cc0_comp<DIM, A1>(M, tb);
    const double cc0 = cc0_comp<DIM, D>(M, p);
    ondB = unit_comp<D>(fc0_comp<DIM, D, D>(M, p) - cc0, t0, t1);
    ondF = unit_comp<D>(fc0_comp<DIM, D, D>(M, p + 1) - cc0, t0, t1);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = ph[v] = 0.;
  }
  // cell widths, the cell itself beyond the line ends
  const double hw = lane_cell_width<DIM, D>(M, F, ok, i, j, k, p, nd);
  double hw_l = __shfl_up_sync(FULL, hw, 1), hw_r = __shfl_down_sync(FULL, hw, 1);
  if (p == 0) hw_l = hw;
  if (p == nd - 1) hw_r = hw;
  // pure neighbourhood (projection-pente-borne-mixte): purity codes -2 mixed,
  // else the last environment with a positive volume fraction (-1: none)
  int code = 0;
  if (ok && !A.first_remap) {
    int cnt = 0;
    code = -1;
#pragma unroll
    for (int q = 0; q < NE; ++q)
      if ((!A.first || ((mask >> q) & 1)) && ph[q] > 0.) { ++cnt; code = q; }
    if (cnt > 1) code = -2;
  }
  int code_l = __shfl_up_sync(FULL, code, 1), code_r = __shfl_down_sync(FULL, code, 1);
  if (p == 0) code_l = code;
  if (p == nd - 1) code_r = code;
  const bool pure = P.projection_pente_borne_mixte && code != -2 && code_l != -2 && code_r != -2 &&
                    code == code_l && code == code_r;
  const int lim_g = (P.projection_limiteur_pure_id == 1 && pure) ? P.projection_limiteur_pure_id : A.limiter;
  const int lim_y = pure ? P.projection_limiteur_pure_id : A.limiter;
  const double un = back.un, L = back.L;  // back face of the cell
  const bool ok_l = __shfl_up_sync(FULL, ok, 1) && lane > 0 && p > 0;  // same line
  const double xc_l = __shfl_up_sync(FULL, xc, 1);
  const bool face_b = ok && ok_l;
  const bool face_f = __shfl_down_sync(FULL, face_b, 1) && lane < 31;
  const double un_r = __shfl_down_sync(FULL, un, 1), L_r = __shfl_down_sync(FULL, L, 1);
  const double dxb = xc - xc_l;
  // outgoing normal velocities and swept lengths of the back / front faces
  const double vb = ondB * un, vf = ondF * un_r;
  const double ppv_b = 0.5 * (vb + fabs(vb)) * dt, ppv_f = 0.5 * (vf + fabs(vf)) * dt;
  // raw flux of variable v through both faces
  auto raw = [&](int v, double& Fb, double& Ff) {
    const double y0 = ph[v];
    const double y_l = __shfl_up_sync(FULL, y0, 1), y_r = __shfl_down_sync(FULL, y0, 1);
    const double gf = face_b ? div_rn(y0 - y_l, dxb) : 0.;
    const double gf_r = __shfl_down_sync(FULL, gf, 1);
    const double ym = p > 0 ? y_l : y0, yp = p < nd - 1 ? y_r : y0;
    double gr = 0.;
    if (ok)
      gr = lim_g < 3 ? limited_gradient(lim_g, gf, gf_r)
                     : generalized_gradient(lim_g, gf_r, gf, yp, ym, hw, hw_r, hw_l, A.simple_pente);
    Fb = ok ? pb_flux(0, y0, yp, ym, hw, hw_r, hw_l, gr, ppv_b, lim_y, A.simple_pente, thr) : 0.;
    Ff = ok ? pb_flux(1, y0, yp, ym, hw, hw_r, hw_l, gr, ppv_f, lim_y, A.simple_pente, thr) : 0.;
  };
  // volume fluxes first: the de-barring fix 1 divides by their sum
  double vol_b[NE], vol_f[NE], mass_b[NE], mass_f[NE];
  double sfb = 0., sff = 0.;
#pragma unroll
  for (int q = 0; q < NE; ++q) {
    raw(q, vol_b[q], vol_f[q]);
    sfb += vol_b[q];
    sff += vol_f[q];
  }
  const bool zb = (fix == 1 && !(fabs(sfb) > thr)) || ppv_b == 0.;
  const bool zf = (fix == 1 && !(fabs(sff) > thr)) || ppv_f == 0.;
  constexpr bool FRONT_FIRST = DIM == 2 && D == 0;
  double uo[NV], dual[NE];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double Fb, Ff;
    if (v < NE) { Fb = vol_b[v]; Ff = vol_f[v]; }
    else raw(v, Fb, Ff);
    if (v >= NE && v < 2 * NE) {
      const int q = v - NE;
      if (fix == 1 && !pure) { Fb = (Fb / sfb) * vol_b[q]; Ff = (Ff / sff) * vol_f[q]; }
      if (fix == 2 && !pure) { Fb = ph[v] * vol_b[q]; Ff = ph[v] * vol_f[q]; }
      mass_b[q] = Fb; mass_f[q] = Ff;
    } else if (v >= 2 * NE && v < 3 * NE) {
      const int q = v - 2 * NE;
      if (fix == 1) { Fb = (Fb / sfb) * mass_b[q]; Ff = (Ff / sff) * mass_f[q]; }
      if (fix == 2) { Fb = ph[v] * mass_b[q]; Ff = ph[v] * mass_f[q]; }
    }
    if (zb) Fb = 0.;
    if (zf) Ff = 0.;
    const double Ff_l = __shfl_up_sync(FULL, Ff, 1);
    const double pf = face_b ? Ff_l - Fb : 0.;  // face value: front flux of l-1 minus back flux of l
    const double pf_r = __shfl_down_sync(FULL, pf, 1);
    const double fB = face_b ? ondB * L * pf : 0.;
    const double fF = face_f ? ondF * L_r * pf_r : 0.;
    double sumf = 0., du = 0.;
    if (FRONT_FIRST) {
      if (face_f) { sumf += fF; du += 0.5 * fF * ondF; }
      if (face_b) { sumf += fB; du += 0.5 * fB * ondB; }
    } else {
      if (face_b) { sumf += fB; du += 0.5 * fB * ondB; }
      if (face_f) { sumf += fF; du += 0.5 * fF * ondF; }
    }
    uo[v] = u[v] - sumf;
    if (v >= NE && v < 2 * NE) dual[v - NE] = du;
  }
  if (!out) return;
  // truncation of tiny volumes, masses and energies (with the dual
  // projection only, not in a sans-lagrange advection), then the clip of
  // negative masses and energies
  const bool trunc = !P.sans_lagrange;
#pragma unroll
  for (int q = 0; q < NE; ++q) {
    if (trunc && uo[q] < 1. * thr) { uo[q] = 0.; uo[NE + q] = 0.; uo[2 * NE + q] = 0.; }
    if (trunc && uo[NE + q] < 1. * thr) { uo[q] = 0.; uo[NE + q] = 0.; uo[2 * NE + q] = 0.; }
    if (trunc && uo[2 * NE + q] < 1. * thr) { uo[q] = 0.; uo[NE + q] = 0.; uo[2 * NE + q] = 0.; }
    if (uo[NE + q] < 0.) uo[NE + q] = 0.;
    if (uo[2 * NE + q] < 0.) uo[2 * NE + q] = 0.;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) A.Uout[v * N + c] = uo[v];
#pragma unroll
  for (int q = 0; q < NE; ++q) F.mflux[q * N + c] = dual[q];
}

// ---------------------------------------------------------------------------
// Third-order face value (Remap-ordre-3.cc:16-188: evaluate_grad,
// evaluate_ystar, evaluate_fm / evaluate_fp, the TVD interval bound of
// ComputeFluxOrdre3).  y[0..5], h[0..5]: values and widths of the cells
// b-2 .. f+2 around the face, repeated at the line ends; vdt = face normal
// velocity x deltat.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double o3_grad(double hm, double h0, double hp, double ym, double y0, double yp) {
  return h0 / (hm + h0 + hp) * ((2. * hm + h0) / (h0 + hp) * (yp - y0) + (h0 + 2. * hp) / (hm + h0) * (y0 - ym));
}
__device__ __forceinline__ double o3_ystar(double hmm, double hm, double hp, double hpp, double ymm, double ym,
                                           double yp, double ypp, double gm, double gp) {
  const double a =
      (2. * hp * hm) / (hm + hp) * ((hmm + hm) / (2. * hm + hp) - (hpp + hp) / (2. * hp + hm)) * (yp - ym);
  const double b = -hm * (hmm + hm) / (2. * hm + hp) * gp + hp * (hp + hpp) / (hm + 2. * hp) * gm;
  return ym + hm / (hm + hp) * (yp - ym) + 1. / (hmm + hm + hp + hpp) * (a + b);
}
__device__ __forceinline__ double order3_face_value(const double (&y)[6], const double (&h)[6], double vdt) {
  if (!(vdt > 0.) && !(vdt < 0.)) return 0.;
  const double g0 = o3_grad(h[0], h[1], h[2], y[0], y[1], y[2]);
  const double g1 = o3_grad(h[1], h[2], h[3], y[1], y[2], y[3]);
  const double g2 = o3_grad(h[2], h[3], h[4], y[2], y[3], y[4]);
  const double g3 = o3_grad(h[3], h[4], h[5], y[3], y[4], y[5]);
  const double s0 = o3_ystar(h[1], h[2], h[3], h[4], y[1], y[2], y[3], y[4], g1, g2);
  double v;
  if (vdt > 0.) {
    const double sm = o3_ystar(h[0], h[1], h[2], h[3], y[0], y[1], y[2], y[3], g0, g1);
    const double du = s0 - sm, u6 = 6. * (y[2] - 0.5 * (sm + s0));
    v = s0 - 0.5 * vdt / h[2] * (du - (1. - 2. / 3. * vdt / h[2]) * u6);
  } else {
    const double sp = o3_ystar(h[2], h[3], h[4], h[5], y[2], y[3], y[4], y[5], g2, g3);
    const double du = sp - s0, u6 = 6. * (y[3] - 0.5 * (s0 + sp)), x = -vdt;
    v = s0 + 0.5 * x / h[3] * (du - (1. - 2. / 3. * x / h[3]) * u6);
  }
  // TVD bound: [y_b, y_f] intersected with the upwind extrapolation
  double o, x;
  if (vdt > 0.) {
    const double num = vdt / h[2];
    o = y[2];
    x = y[2] + (1. - num) / num * (y[2] - y[1]);
  } else {
    const double nup = vdt / h[3];
    o = y[3];
    x = y[3] - (1. + nup) / nup * (y[3] - y[4]);
  }
  const double i1a = amin(y[2], y[3]), i1b = amax(y[2], y[3]);
  const double i2a = amin(o, x), i2b = amax(o, x);
  double lo = 0., hi = 0.;
  if (!(i1b < i2a || i2b < i1a)) {
    lo = amax(i1a, i2a);
    hi = amin(i1b, i2b);
  }
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}

// ---------------------------------------------------------------------------
// Cell sweep along D with the third-order face values
// (computeUpwindFaceQuantitiesForProjection, RemapADIService.cc:319-380):
// the same lane layout with 3 halo lanes on each side (lane l: cell
// x0 - 3 + l, lanes 3 .. 28 write).  Faces between two cells that are not
// both pure in the same material (EstMixte / EstPure, which equal the
// volume-fraction signs of the cell values read here; every cell is pure in
// material 0 before the first remap of the run) take their mass and energy
// values from the volume value with the upwind cell's density and specific
// energy.
// ---------------------------------------------------------------------------
template <int DIM, int NE, int D>
__device__ __forceinline__ void body_sweep_cells_o3(const Mesh& M, const Fields& F, const SweepArgs& A, int vbx,
                                                    int vby) {
  constexpr int NV = 3 * NE + 1;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  constexpr int HL = 3;
  constexpr unsigned FULL = 0xffffffffu;
  const long long N = M.ncell;
  const int lane = threadIdx.x % SW_LANES, row = threadIdx.x / SW_LANES;
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  if (sweep_warp_empty<D>(M.ncx, M.ncy, M.ncz, XOUT_W, HL, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, p, ta, tb;
  const bool ok = sweep_lane<D>(M.ncx, M.ncy, M.ncz, XOUT_W, HL, vbx, vby, lane, row, i, j, k, p, ta, tb);
  const bool out = ok && lane >= HL && lane < HL + XOUT_W;
  const double dt = F.s->dt;
  const double* __restrict__ Uin = A.Uin;
  Plane<DIM> back;
  if (ok) load_plane<DIM, D>(M, F, i, j, k, back);
  else {
#pragma unroll
    for (int q = 0; q < NQ; ++q) back.xd[q] = 0.;
    back.fc = back.un = back.L = 0.;
  }
  long long c = 0;
  double u[NV], den = 1., ondB = 0., ondF = 0.;
  if (ok) {
    c = cell_id(M, i, j, k);
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = __ldg(Uin + v * N + c);
    if (A.first) {
      den = __ldg(F.V + c);
    } else {
      den = 0.;
#pragma unroll
      for (int q = 0; q < NE; ++q) den += u[q];
    }
    if (out) {
      constexpr int A0 = D == 0 ? 1 : 0, A1 = D == 2 ? 1 : 2;
      const double t0 = fc0_comp<DIM, D, A0>(M, ta) - cc0_comp<DIM, A0>(M, ta);
      const double t1 = fc0_comp<DIM, D, A1>(M, tb) - cc0_comp<DIM, A1>(M, tb);
      const double cc0 = cc0_comp<DIM, D>(M, p);
      ondB = unit_comp<D>(fc0_comp<DIM, D, D>(M, p) - cc0, t0, t1);
      ondF = unit_comp<D>(fc0_comp<DIM, D, D>(M, p + 1) - cc0, t0, t1);
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = 0.;
  }
  // widths of the stencil b-2 .. f+2 of the back face (f = this cell)
  const double hw = lane_cell_width<DIM, D>(M, F, ok, i, j, k, p, nd);
  const bool m2 = p >= 2, m3 = p >= 3, p1 = p + 1 < nd, p2 = p + 2 < nd;
  double h[6];
  {
    const double a1 = __shfl_up_sync(FULL, hw, 1), a2 = __shfl_up_sync(FULL, hw, 2),
                 a3 = __shfl_up_sync(FULL, hw, 3), b1 = __shfl_down_sync(FULL, hw, 1),
                 b2 = __shfl_down_sync(FULL, hw, 2);
    h[2] = a1; h[1] = m2 ? a2 : h[2]; h[0] = m3 ? a3 : h[1];
    h[3] = hw; h[4] = p1 ? b1 : h[3]; h[5] = p2 ? b2 : h[4];
  }
  // purity code: -2 mixed, else the last material with a positive volume
  // fraction (-1: none)
  int code = 0;
  if (ok && !A.first_remap) {
    int cnt = 0;
    code = -1;
#pragma unroll
    for (int q = 0; q < NE; ++q)
      if (div_rn(u[q], den) > 0.) { ++cnt; code = q; }
    if (cnt > 1) code = -2;
  }
  const int code_l = __shfl_up_sync(FULL, code, 1);
  const bool pure_nb = code_l == code && code != -2;
  const double un = back.un, L = back.L;  // back face of the cell
  const bool ok_l = __shfl_up_sync(FULL, ok, 1) && lane > 0 && p > 0;  // same line
  const bool face_b = ok && ok_l;
  const bool face_f = __shfl_down_sync(FULL, face_b, 1) && lane < 31;
  const double un_r = __shfl_down_sync(FULL, un, 1), L_r = __shfl_down_sync(FULL, L, 1);
  const double vdt = un * dt;
  constexpr bool FRONT_FIRST = DIM == 2 && D == 0;
  double pf_v[NE], yb_v[NE], yf_v[NE], pf_m[NE], yb_m[NE], yf_m[NE];
  bool corr[NE];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double phi = ok ? div_rn(u[v], den) : 0.;
    double y[6];
    {
      const double a1 = __shfl_up_sync(FULL, phi, 1), a2 = __shfl_up_sync(FULL, phi, 2),
                   a3 = __shfl_up_sync(FULL, phi, 3), b1 = __shfl_down_sync(FULL, phi, 1),
                   b2 = __shfl_down_sync(FULL, phi, 2);
      y[2] = a1; y[1] = m2 ? a2 : y[2]; y[0] = m3 ? a3 : y[1];
      y[3] = phi; y[4] = p1 ? b1 : y[3]; y[5] = p2 ? b2 : y[4];
    }
    double pf = face_b ? order3_face_value(y, h, vdt) : 0.;
    if (v < NE) {
      pf_v[v] = pf; yb_v[v] = y[2]; yf_v[v] = y[3];
    } else if (v < 2 * NE) {
      const int e = v - NE;
      const bool cb = vdt > 0. && yb_v[e] != 0. && y[2] != 0.;
      const bool cf = vdt < 0. && yf_v[e] != 0. && y[3] != 0.;
      corr[e] = !pure_nb && (cb || cf);
      if (corr[e]) pf = (cb ? (y[2] / yb_v[e]) : (y[3] / yf_v[e])) * pf_v[e];
      pf_m[e] = pf; yb_m[e] = y[2]; yf_m[e] = y[3];
    } else if (v < 3 * NE) {
      const int e = v - 2 * NE;
      if (corr[e]) pf = (vdt > 0. ? (y[2] / yb_m[e]) : (y[3] / yf_m[e])) * pf_m[e];
    }
    const double pf_r = __shfl_down_sync(FULL, pf, 1);
    if (out) {
      const double fB = face_b ? ondB * un * L * dt * pf : 0.;
      const double fF = face_f ? ondF * un_r * L_r * dt * pf_r : 0.;
      double sumf = 0., dual = 0.;
      if (FRONT_FIRST) {
        if (face_f) { sumf += fF; dual += 0.5 * fF * ondF; }
        if (face_b) { sumf += fB; dual += 0.5 * fB * ondB; }
      } else {
        if (face_b) { sumf += fB; dual += 0.5 * fB * ondB; }
        if (face_f) { sumf += fF; dual += 0.5 * fF * ondF; }
      }
      double uo = u[v] - sumf;
      if (v >= NE && v < 3 * NE && uo < 0.) uo = 0.;  // masses and energies stay >= 0
      A.Uout[v * N + c] = uo;
      if (v >= NE && v < 2 * NE) F.mflux[(v - NE) * N + c] = dual;
    }
  }
}

// ---------------------------------------------------------------------------
// Cell sweep along D = 1, 2, classical limiters and first order, with one
// thread per line: the threads of a warp hold consecutive x columns, so
// every load and store is coalesced, and each thread walks a chunk of its
// line in order with the stencil carried in registers.  Iteration q loads
// cell q and the node plane in front of it; it completes the face gradient
// of face q, the limited gradient of cell q-1, the value of face q-1 and the
// update of cell q-2.  A chunk writes cells [o0, o1) and starts two cells
// before o0.  Same arithmetic, in the same order, as
// body_sweep_cells_lanes.
// ---------------------------------------------------------------------------
constexpr int SWC_CHUNK = 16;   // cells written per thread at most

// chunks of a line of nd cells, and the cells [o0, o1) of chunk ch
__host__ __device__ inline int col_chunks(int nd) { return (nd + SWC_CHUNK - 1) / SWC_CHUNK; }
__host__ __device__ inline void col_chunk_range(int nd, int ch, int& o0, int& o1) {
  const int n = col_chunks(nd);
  const int len = (nd + n - 1) / n;
  o0 = ch * len;
  o1 = o0 + len < nd ? o0 + len : nd;
}

template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_cells_cols(const Mesh& M, const Fields& F, const SweepArgs& A, int vbx,
                                                      int vby) {
  static_assert(D >= 1, "x sweeps use the lane layout");
  constexpr int NV = 3 * NE + 1;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  const long long N = M.ncell;
  const int nd = D == 1 ? M.ncy : M.ncz;
  const int nb = D == 1 ? M.ncz : M.ncy;           // slow transverse extent
  const long long col = (long long)vbx * SW_THREADS + threadIdx.x;
  if (col >= (long long)M.ncx * nb) return;
  const int tb = (int)((unsigned)col / (unsigned)M.ncx), i = (int)col - tb * M.ncx;
  int o0, o1;
  col_chunk_range(nd, vby, o0, o1);
  if (o0 >= o1) return;
  const double dt = F.s->dt;
  const int order2 = LIM == LIM_ORDER1 ? 0 : 1;  // ordre-projection - 1
  const double* __restrict__ Uin = A.Uin;
  // transverse parts of the initial outer normals (grid formula)
  constexpr int A0 = 0, A1 = D == 2 ? 1 : 2;
  const double t0 = fc0_comp<DIM, D, A0>(M, i) - cc0_comp<DIM, A0>(M, i);
  const double t1 = fc0_comp<DIM, D, A1>(M, tb) - cc0_comp<DIM, A1>(M, tb);
  auto cell_at = [&](int p) -> long long { return D == 1 ? cell_id(M, i, p, tb) : cell_id(M, i, tb, p); };
  auto plane_at = [&](int p, Plane<DIM>& P) {
    if (D == 1) load_plane<DIM, D>(M, F, i, p, tb, P);
    else load_plane<DIM, D>(M, F, i, tb, p, P);
  };
  // carried state: 1 = previous cell / face, 2 = the one before; lc = the
  // upwind value of face q-1 taken from its back cell q-2 (made one
  // iteration early, when that cell's limited gradient is known, so that
  // neither the gradient nor phi of cell q-2 has to be carried)
  double phi1[NV], gf1[NV], lc[NV], pf2[NV];
  double xc1 = 0., xc2 = 0., fc1 = 0., un1 = 0., un2 = 0., L1 = 0., L2 = 0.;
  const int qs = o0 - 2 > 0 ? o0 - 2 : 0;
  Plane<DIM> cur;       // back plane of cell q
  plane_at(qs, cur);
#pragma unroll
  for (int v = 0; v < NV; ++v) phi1[v] = gf1[v] = lc[v] = pf2[v] = 0.;
  for (int q = qs; q <= o1 + 1; ++q) {
    const bool cell = q < nd;                 // a cell is loaded at q
    double phi[NV], xc = 0.;
    Plane<DIM> nxt;
    if (cell) {
      plane_at(q + 1, nxt);
      xc = centre_from_planes<DIM, D>(cur, nxt);
      const long long c = cell_at(q);
      double u[NV], den;
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = __ldg(Uin + v * N + c);
      if (A.first) {
        den = __ldg(F.V + c);
      } else {
        den = 0.;
#pragma unroll
        for (int e = 0; e < NE; ++e) den += u[e];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) phi[v] = div_rn(u[v], den);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) phi[v] = 0.;
    }
    const bool face_q = cell && q > 0;        // face q (between q-1 and q) is inner
    const double dx = xc - xc1;
    const bool face_q1 = q - 1 > 0 && q - 1 < nd;  // face q-1 is inner
    // face q-1 upwind test (its normal velocity and the centres of q-2, q-1)
    const bool up_left = un1 * (xc1 - xc2) > 0.0;
    double pf1[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double gf = face_q ? div_rn(phi[v] - phi1[v], dx) : 0.;
      // limited gradient of cell q-1 from its back (gf1) and front (gf) faces
      const double gr1 = (LIM != LIM_ORDER1 && q - 1 >= 0 && q - 1 < nd) ? limited_gradient_t<LIM>(gf1[v], gf) : 0.;
      pf1[v] = 0.;
      if (face_q1) pf1[v] = up_left ? lc[v] : phi1[v] + order2 * (fc1 - xc1) * gr1;
      // face q seen from its back cell q-1 (fc of face q = cur.fc)
      lc[v] = phi1[v] + order2 * (cur.fc - xc1) * gr1;
      gf1[v] = gf;
    }
    // update of cell o = q - 2 from faces o (pf2) and o + 1 (pf1)
    const int o = q - 2;
    if (o >= o0 && o < o1) {
      const long long c = cell_at(o);
      const double cc0 = cc0_comp<DIM, D>(M, o);
      const double ondB = unit_comp<D>(fc0_comp<DIM, D, D>(M, o) - cc0, t0, t1);
      const double ondF = unit_comp<D>(fc0_comp<DIM, D, D>(M, o + 1) - cc0, t0, t1);
      const bool fb = o > 0, ff = o + 1 < nd;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double fB = fb ? ondB * un2 * L2 * dt * pf2[v] : 0.;
        const double fF = ff ? ondF * un1 * L1 * dt * pf1[v] : 0.;
        double sumf = 0., dual = 0.;
        if (fb) { sumf += fB; dual += 0.5 * fB * ondB; }
        if (ff) { sumf += fF; dual += 0.5 * fF * ondF; }
        double uo = __ldg(Uin + v * N + c) - sumf;
        if (v >= NE && v < 3 * NE && uo < 0.) uo = 0.;  // masses and energies stay >= 0
        A.Uout[v * N + c] = uo;
        if (v >= NE && v < 2 * NE) F.mflux[(v - NE) * N + c] = dual;
      }
    }
    // shift
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      phi1[v] = phi[v];
      pf2[v] = pf1[v];
    }
    xc2 = xc1; xc1 = xc;
    un2 = un1; L2 = L1;
    un1 = cur.un; L1 = cur.L; fc1 = cur.fc;
    if (cell) cur = nxt;
  }
}

// ---------------------------------------------------------------------------
// Cell sweep along D = 1, 2 through a shared-memory tile, classical limiters
// and first order.  A block holds SWT_COLS neighbouring x columns and one
// window of 32 positions along D (the concatenated lines of the lane layout:
// 2 halo cells, XOUT written, the rest after them).
//  1. Load: thread t takes column t % SWT_COLS and position t / SWT_COLS, so
//     the SWT_COLS threads of one position read consecutive x cells (every
//     global load and store is a contiguous 64-byte run); each thread
//     stages its cell's projected quantities, divisor, Lagrangian centre
//     along D and back-face centre, normal velocity and length.
//  2. Sweep: warp w takes column w, lane = position along D, and runs the
//     arithmetic of body_sweep_cells_lanes, in the same order, from the
//     staged values (neighbours by shuffles); results go back to the tile.
//  3. Store: the load layout again, written cells only.
// The staged front-plane coordinates of a cell are loaded, not shuffled, so
// the cell centre is the same sum of the same node coordinates.
// ---------------------------------------------------------------------------
constexpr int SWT_COLS = 8;                     // x columns (warps) per block
constexpr int SWT_THREADS = SWT_COLS * SW_LANES;
constexpr int SWT_PITCH = SWT_COLS + 1;         // padded row: two wavefronts per warp access
constexpr int SWT_FIELD = SW_LANES * SWT_PITCH;  // doubles per staged quantity

// staged quantities: NV projected values, divisor, centre, face centre,
// normal velocity, face length (outputs reuse the first NV + NE slots)
__host__ __device__ constexpr int swt_slots(int ne) { return 3 * ne + 1 + 5; }
__host__ __device__ constexpr int swt_smem_bytes(int ne) { return swt_slots(ne) * SWT_FIELD * 8; }

template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_cells_tile(const Mesh& M, const Fields& F, const SweepArgs& A, int vbx,
                                                      int vby, double* __restrict__ sm) {
  static_assert(D >= 1, "x sweeps use the lane layout");
  constexpr int NV = 3 * NE + 1;
  constexpr int S_DEN = NV, S_XC = NV + 1, S_FC = NV + 2, S_UN = NV + 3, S_L = NV + 4;
  constexpr unsigned FULL = 0xffffffffu;
  const long long N = M.ncell;
  const int nd = D == 1 ? M.ncy : M.ncz, nb = D == 1 ? M.ncz : M.ncy;
  const int x0 = vbx * SWT_COLS;
  const int g0 = vby * XOUT - 2;  // first position of the window (2 halo cells)
  const double* __restrict__ Uin = A.Uin;
  // -- 1. load (row layout)
  {
    const int col = threadIdx.x % SWT_COLS, pos = threadIdx.x / SWT_COLS;
    const int i = x0 + col, g = g0 + pos;
    if (i < M.ncx && g >= 0 && g < nb * nd) {
      const int tb = (int)((unsigned)g / (unsigned)nd), p = g - tb * nd;
      const int j = D == 1 ? p : tb, k = D == 1 ? tb : p;
      Plane<DIM> back, front;
      load_plane<DIM, D>(M, F, i, j, k, back);
      load_plane_xd<DIM, D>(M, F, i, D == 1 ? j + 1 : j, D == 2 ? k + 1 : k, front);
      const long long c = cell_id(M, i, j, k);
      double* s = sm + pos * SWT_PITCH + col;
      double den = 0.;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double u = __ldg(Uin + v * N + c);
        s[v * SWT_FIELD] = u;
        if (v < NE) den += u;
      }
      if (A.first) den = __ldg(F.V + c);
      s[S_DEN * SWT_FIELD] = den;
      s[S_XC * SWT_FIELD] = centre_from_planes<DIM, D>(back, front);
      s[S_FC * SWT_FIELD] = back.fc;
      s[S_UN * SWT_FIELD] = back.un;
      s[S_L * SWT_FIELD] = back.L;
    }
  }
  __syncthreads();
  // -- 2. sweep (warp w: column x0 + w, lane: position along D)
  const int lane = threadIdx.x % SW_LANES, w = threadIdx.x / SW_LANES;
  const int ta = x0 + w;
  if (ta < M.ncx && g0 < nb * nd) {  // warp-uniform
    const int g = g0 + lane;
    const bool ok = g >= 0 && g < nb * nd;
    int tb = 0, p = 0;
    if (ok) {
      tb = (int)((unsigned)g / (unsigned)nd);
      p = g - tb * nd;
    }
    const bool out = ok && lane >= 2 && lane < 2 + XOUT;
    const double dt = F.s->dt;
    const int order2 = LIM == LIM_ORDER1 ? 0 : 1;  // ordre-projection - 1
    double* s = sm + lane * SWT_PITCH + w;
    double u[NV], den = 1., xc = 0., fc = 0., un = 0., L = 0., ondB = 0., ondF = 0.;
    if (ok) {
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = s[v * SWT_FIELD];
      den = s[S_DEN * SWT_FIELD];
      xc = s[S_XC * SWT_FIELD];
      fc = s[S_FC * SWT_FIELD];
      un = s[S_UN * SWT_FIELD];
      L = s[S_L * SWT_FIELD];
      if (out) {
        // outer normals of the back and front faces (initial grid)
        constexpr int A0 = 0, A1 = D == 2 ? 1 : 2;
        const double t0 = fc0_comp<DIM, D, A0>(M, ta) - cc0_comp<DIM, A0>(M, ta);
        const double t1 = fc0_comp<DIM, D, A1>(M, tb) - cc0_comp<DIM, A1>(M, tb);
        const double cc0 = cc0_comp<DIM, D>(M, p);
        ondB = unit_comp<D>(fc0_comp<DIM, D, D>(M, p) - cc0, t0, t1);
        ondF = unit_comp<D>(fc0_comp<DIM, D, D>(M, p + 1) - cc0, t0, t1);
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = 0.;
    }
    const bool ok_l = __shfl_up_sync(FULL, ok, 1) && lane > 0 && p > 0;  // same line
    const double xc_l = __shfl_up_sync(FULL, xc, 1);
    const bool face_b = ok && ok_l;                       // face between p-1 and p
    const bool face_f = __shfl_down_sync(FULL, face_b, 1) && lane < 31;
    const double un_r = __shfl_down_sync(FULL, un, 1), L_r = __shfl_down_sync(FULL, L, 1);
    const double dxb = xc - xc_l;
    const bool up_left = un * dxb > 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double phi = ok ? div_rn(u[v], den) : 0.;
      const double phi_l = __shfl_up_sync(FULL, phi, 1);
      const double gf = face_b ? div_rn(phi - phi_l, dxb) : 0.;
      const double gf_r = __shfl_down_sync(FULL, gf, 1);
      const double gr = (LIM != LIM_ORDER1 && ok) ? limited_gradient_t<LIM>(gf, gf_r) : 0.;
      const double gr_l = __shfl_up_sync(FULL, gr, 1);
      double pf = 0.;
      if (face_b) pf = up_left ? phi_l + order2 * (fc - xc_l) * gr_l : phi + order2 * (fc - xc) * gr;
      const double pf_r = __shfl_down_sync(FULL, pf, 1);
      if (out) {
        // cell local face order along y and z: back then front
        const double fB = face_b ? ondB * un * L * dt * pf : 0.;
        const double fF = face_f ? ondF * un_r * L_r * dt * pf_r : 0.;
        double sumf = 0., dual = 0.;
        if (face_b) { sumf += fB; dual += 0.5 * fB * ondB; }
        if (face_f) { sumf += fF; dual += 0.5 * fF * ondF; }
        double uo = u[v] - sumf;
        if (v >= NE && v < 3 * NE && uo < 0.) uo = 0.;  // masses and energies stay >= 0
        s[v * SWT_FIELD] = uo;                          // the lane's own slots: read above
        if (v >= NE && v < 2 * NE) s[(S_XC + v - NE) * SWT_FIELD] = dual;
      }
    }
  }
  __syncthreads();
  // -- 3. store (row layout), written positions only
  {
    const int col = threadIdx.x % SWT_COLS, pos = threadIdx.x / SWT_COLS;
    const int i = x0 + col, g = g0 + pos;
    if (pos >= 2 && pos < 2 + XOUT && i < M.ncx && g < nb * nd) {
      const int tb = (int)((unsigned)g / (unsigned)nd), p = g - tb * nd;
      const long long c = cell_id(M, i, D == 1 ? p : tb, D == 1 ? tb : p);
      const double* s = sm + pos * SWT_PITCH + col;
#pragma unroll
      for (int v = 0; v < NV; ++v) A.Uout[v * N + c] = s[v * SWT_FIELD];
#pragma unroll
      for (int e = 0; e < NE; ++e) F.mflux[e * N + c] = s[(S_XC + e) * SWT_FIELD];
    }
  }
  __syncthreads();  // the tile is reused by the block's next work item
}

// ---------------------------------------------------------------------------
// Node part: RemapADIService::computeDualUremap (DualPhaseRemap.cc:38-258,
// classical limiter) with the same lane layout.  Lane l holds node
// x0 - 2 + l along D; lanes 2 .. NOUT+1 write.  The mass flux through the
// back half-plane of a node is the flux through the front half-plane of the
// node behind it, summed over the same cells in the same order, so each
// lane sums its front cells once and hands the sum to lane l+1.
// ---------------------------------------------------------------------------
constexpr int NOUT = 28;    // nodes written per warp (lanes 2 .. 29)
constexpr int NOUT_W = 26;  // generalised limiters (widths need 2 more nodes): lanes 3 .. 28

struct DualArgs {
  const double* Uin;   // null on the first sweep (U built from m and v)
  double* Uout;
  int order;
  int limiter;
  int simple_pente;    // projection-simple-pente (generalised limiters)
  int done_dirs;       // bit d: direction d already swept this cycle
};

__device__ __forceinline__ bool node_inner_dir(const Mesh& M, int i, int j, int k, int d) {
  int id = d == 0 ? i : (d == 1 ? j : k);
  int nn = d == 0 ? M.nnx : (d == 1 ? M.nny : M.nnz);
  return id > 0 && id < nn - 1;
}

template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_nodes_lanes(const Mesh& M, const Fields& F, const DualArgs& A,
                                                       int vbx, int vby) {
  constexpr unsigned FULL = 0xffffffffu;
  const long long NN = M.nnode, N = M.ncell;
  const int lane = threadIdx.x % SW_LANES, row = threadIdx.x / SW_LANES;
  const int nn = D == 0 ? M.nnx : (D == 1 ? M.nny : M.nnz);
  constexpr int HL = LIM == LIM_GEN ? 3 : 2;
  constexpr int NO = LIM == LIM_GEN ? NOUT_W : NOUT;
  if (sweep_warp_empty<D>(M.nnx, M.nny, M.nnz, NO, HL, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, id, ta, tb;
  const bool ok = sweep_lane<D>(M.nnx, M.nny, M.nnz, NO, HL, vbx, vby, lane, row, i, j, k, id, ta, tb);
  const bool inner = ok && id > 0 && id < nn - 1;
  const bool out = ok && lane >= HL && lane < HL + NO;
  long long n = 0;
  double U[5] = {0., 0., 0., 0., 0.};
  double ph[4] = {0., 0., 0., 0.};
  double x = 0., ffm = 0.;
  if (ok) {
    n = node_id(M, i, j, k);
    x = __ldg(F.Xn[D] + n);
    bool was_inner = false;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      if (((A.done_dirs >> d) & 1) && node_inner_dir(M, i, j, k, d)) was_inner = true;
    if (A.Uin) {
      if (was_inner || out) {
#pragma unroll
        for (int q = 0; q < 5; ++q) U[q] = __ldg(A.Uin + q * NN + n);
      }
    } else {
      const double mn = __ldg(F.mn + n), vx = __ldg(F.vx + n), vy = __ldg(F.vy + n), vz = __ldg(F.vz + n);
      U[0] = mn * vx; U[1] = mn * vy; U[2] = mn * vz; U[3] = mn;
      U[4] = 0.5 * mn * (vx * vx + vy * vy + vz * vz);
    }
    if (was_inner) {
      ph[0] = div_rn(U[0], U[3]); ph[1] = div_rn(U[1], U[3]); ph[2] = div_rn(U[2], U[3]);
      ph[3] = div_rn(U[4], U[3]);
    } else {
      const double vx = __ldg(F.vx + n), vy = __ldg(F.vy + n), vz = __ldg(F.vz + n);
      ph[0] = vx; ph[1] = vy; ph[2] = vz;
      ph[3] = 0.5 * (vx * vx + vy * vy + vz * vz);
    }
    // mass flux through the front half-plane: faces of the node plane in
    // face id order, then environments
    const int ndc = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
    if (id < ndc) {
      const double w = DIM == 2 ? .5 : .25;
#pragma unroll
      for (int b2 = 0; b2 < (DIM == 3 ? 2 : 1); ++b2) {
#pragma unroll
        for (int b1 = 0; b1 < 2; ++b1) {
          int ci = i, cj = j, ck = k;
          const int t1 = b1 - 1, t2 = b2 - 1;
          if (D == 0) { cj += t1; ck += (DIM == 3 ? t2 : 0); }
          else if (D == 1) { ci += t1; ck += (DIM == 3 ? t2 : 0); }
          else { ci += t1; cj += t2; }
          if (ci < 0 || cj < 0 || ck < 0) continue;
          if (D != 0 && ci >= M.ncx) continue;
          if (D != 1 && cj >= M.ncy) continue;
          if (DIM == 3 && D != 2 && ck >= M.ncz) continue;
          const long long cf = cell_id(M, ci, cj, DIM == 3 ? ck : 0);
#pragma unroll
          for (int q = 0; q < NE; ++q) ffm += w * __ldg(F.mflux + q * N + cf);
        }
      }
    }
  }
  // neighbours
  const double x_l = __shfl_up_sync(FULL, x, 1), x_r = __shfl_down_sync(FULL, x, 1);
  double ph_l[4], ph_r[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    ph_l[q] = __shfl_up_sync(FULL, ph[q], 1);
    ph_r[q] = __shfl_down_sync(FULL, ph[q], 1);
  }
  const double bfm = __shfl_up_sync(FULL, ffm, 1);
  // dual cell widths for the generalised limiters (UtilesRemap.cc:51-63);
  // a missing second neighbour gives a zero width
  double h0 = 0., hm = 0., hp = 0.;
  if constexpr (LIM == LIM_GEN) {
    const double x_ll = __shfl_up_sync(FULL, x, 2), x_rr = __shfl_down_sync(FULL, x, 2);
    const bool bb = id >= 2, ff = id + 2 < nn;
    h0 = 0.5 * (x_r - x_l);
    if (!bb) {
      if (ff) hp = 0.5 * (x_rr - x);
    } else if (!ff) {
      hm = 0.5 * (x - x_ll);
    } else {
      hm = 0.5 * (x - x_ll);
      hp = 0.5 * (x_rr - x);
    }
  }
  // limited gradients of the velocity components (inner nodes only).  The
  // backward difference of a node is the forward difference of the node
  // before it (same operands), taken from the previous lane: an inner node
  // (id > 0) sits one lane after its back neighbour on the same line
  double g[3], g_l[3], g_r[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    g[q] = 0.;
    const double gfw = LIM != LIM_ORDER1 ? div_rn(ph_r[q] - ph[q], x_r - x) : 0.;
    const double gbw = __shfl_up_sync(FULL, gfw, 1);
    if (LIM != LIM_ORDER1 && inner) {
      if constexpr (LIM == LIM_GEN)
        g[q] = generalized_gradient(A.limiter, gfw, gbw, ph_r[q], ph_l[q], h0, hp, hm, A.simple_pente);
      else
        g[q] = limited_gradient_t<LIM>(gbw, gfw);
    }
    g_l[q] = __shfl_up_sync(FULL, g[q], 1);
    g_r[q] = __shfl_down_sync(FULL, g[q], 1);
  }
  if (!out) return;
  if (!inner) {
#pragma unroll
    for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
    return;
  }
  const double dt = F.s->dt;
  const int order2 = LIM == LIM_ORDER1 ? 0 : A.order - 1;  // ordre-projection - 1
  U[3] += bfm - ffm;
  double FV[3], BV[3], FE, BE;
  {
    const double ufront = 0.5 * (ph[D] + ph_r[D]);
    const int signfront = (ufront > 0) ? 1 : -1;
    const bool fr = ffm < 0.;
    const double geo = (signfront * (x_r - x) - dt * ufront);
#pragma unroll
    for (int q = 0; q < 3; ++q) FV[q] = (fr ? ph_r[q] : ph[q]) + order2 * (0.5 * (fr ? g_r[q] : g[q]) * geo);
    FE = (fr ? ph_r[3] : ph[3]) + order2 * (0.5 * 0. * geo);
  }
  {
    const double uback = 0.5 * (ph_l[D] + ph[D]);
    const int signback = (uback > 0) ? 1 : -1;
    const bool bk = bfm > 0.;
    const double geo = (signback * (x - x_l) - dt * uback);
#pragma unroll
    for (int q = 0; q < 3; ++q) BV[q] = (bk ? ph_l[q] : ph[q]) + order2 * (0.5 * (bk ? g_l[q] : g[q]) * geo);
    BE = (bk ? ph_l[3] : ph[3]) + order2 * (0.5 * 0. * geo);
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) U[q] += bfm * BV[q] - ffm * FV[q];
  U[4] += bfm * BE - ffm * FE;
#pragma unroll
  for (int q = 0; q < 3; ++q)
    if (fabs(U[q]) < 1.e-300) U[q] = 0.;
#pragma unroll
  for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
}

// ---------------------------------------------------------------------------
// Node sweep along D = 1, 2, classical limiters and first order, one thread
// per line chunk (the layout of body_sweep_cells_cols).  Iteration q loads
// node q; it completes the limited gradient of node q-1 and the update of
// node q-2.  A chunk writes nodes [o0, o1) and starts two nodes before o0.
// Same arithmetic, in the same order, as body_sweep_nodes_lanes.
// ---------------------------------------------------------------------------
// projected and phi values, position along D and front mass flux of node
// (i, j, k) with index id along D
// projected dual variables of node n before this sweep: the previous
// sweep's output, or momentum, mass and kinetic energy from the node state
__device__ __forceinline__ void node_u(const Fields& F, const DualArgs& A, long long NN, long long n, double (&U)[5]) {
  if (A.Uin) {
#pragma unroll
    for (int q = 0; q < 5; ++q) U[q] = __ldg(A.Uin + q * NN + n);
  } else {
    const double mn = __ldg(F.mn + n), vx = __ldg(F.vx + n), vy = __ldg(F.vy + n), vz = __ldg(F.vz + n);
    U[0] = mn * vx; U[1] = mn * vy; U[2] = mn * vz; U[3] = mn;
    U[4] = 0.5 * mn * (vx * vx + vy * vy + vz * vz);
  }
}

template <int DIM, int NE, int D>
__device__ __forceinline__ void node_state(const Mesh& M, const Fields& F, const DualArgs& A, int i, int j, int k,
                                           int id, double (&ph)[4], double& x, double& ffm) {
  const long long NN = M.nnode, N = M.ncell;
  const long long n = node_id(M, i, j, k);
  x = __ldg(F.Xn[D] + n);
  bool was_inner = false;
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    if (((A.done_dirs >> d) & 1) && node_inner_dir(M, i, j, k, d)) was_inner = true;
  double U[5];
  node_u(F, A, NN, n, U);
  if (was_inner) {
    ph[0] = div_rn(U[0], U[3]); ph[1] = div_rn(U[1], U[3]); ph[2] = div_rn(U[2], U[3]);
    ph[3] = div_rn(U[4], U[3]);
  } else {
    const double vx = __ldg(F.vx + n), vy = __ldg(F.vy + n), vz = __ldg(F.vz + n);
    ph[0] = vx; ph[1] = vy; ph[2] = vz;
    ph[3] = 0.5 * (vx * vx + vy * vy + vz * vz);
  }
  ffm = 0.;
  const int ndc = D == 1 ? M.ncy : M.ncz;
  if (id < ndc) {
    const double w = DIM == 2 ? .5 : .25;
#pragma unroll
    for (int b2 = 0; b2 < (DIM == 3 ? 2 : 1); ++b2) {
#pragma unroll
      for (int b1 = 0; b1 < 2; ++b1) {
        int ci = i, cj = j, ck = k;
        const int t1 = b1 - 1, t2 = b2 - 1;
        if (D == 1) { ci += t1; ck += (DIM == 3 ? t2 : 0); }
        else { ci += t1; cj += t2; }
        if (ci < 0 || cj < 0 || ck < 0) continue;
        if (ci >= M.ncx) continue;
        if (D != 1 && cj >= M.ncy) continue;
        if (DIM == 3 && D != 2 && ck >= M.ncz) continue;
        const long long cf = cell_id(M, ci, cj, DIM == 3 ? ck : 0);
#pragma unroll
        for (int q = 0; q < NE; ++q) ffm += w * __ldg(F.mflux + q * N + cf);
      }
    }
  }
}

template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_nodes_cols(const Mesh& M, const Fields& F, const DualArgs& A, int vbx,
                                                      int vby) {
  static_assert(D >= 1, "x sweeps use the lane layout");
  const long long NN = M.nnode;
  const int nn = D == 1 ? M.nny : M.nnz;
  const int nb = D == 1 ? M.nnz : M.nny;
  const long long col = (long long)vbx * SW_THREADS + threadIdx.x;
  if (col >= (long long)M.nnx * nb) return;
  const int tb = (int)((unsigned)col / (unsigned)M.nnx), i = (int)col - tb * M.nnx;
  int o0, o1;
  col_chunk_range(nn, vby, o0, o1);
  if (o0 >= o1) return;
  const double dt = F.s->dt;
  const int order2 = LIM == LIM_ORDER1 ? 0 : A.order - 1;  // ordre-projection - 1
  // carried state: 1 = node q-1, 2 = node q-2, 3 = node q-3
  // fd1: forward difference of node q-2 (= backward difference of q-1);
  // the projected variables of the node being updated are read again
  // (cached) rather than carried, to keep registers for resident warps
  double ph1[4], ph2[4], ph3[4], g1[3], g2[3], g3[3], fd1[3];
  double x1 = 0., x2 = 0., x3 = 0., ffm1 = 0., ffm2 = 0., ffm3 = 0.;
#pragma unroll
  for (int q = 0; q < 4; ++q) ph1[q] = ph2[q] = ph3[q] = 0.;
#pragma unroll
  for (int q = 0; q < 3; ++q) g1[q] = g2[q] = g3[q] = fd1[q] = 0.;
  const int qs = o0 - 2 > 0 ? o0 - 2 : 0;
  for (int q = qs; q <= o1 + 1; ++q) {
    double ph[4] = {0., 0., 0., 0.}, x = 0., ffm = 0.;
    if (q < nn) {
      if (D == 1) node_state<DIM, NE, D>(M, F, A, i, q, tb, q, ph, x, ffm);
      else node_state<DIM, NE, D>(M, F, A, i, tb, q, q, ph, x, ffm);
    }
    // limited gradients of node q-1 (inner nodes only); its backward
    // difference is the forward difference of node q-2, carried from the
    // previous iteration (valid from the second iteration on, the first
    // node whose gradient an update needs)
    const int m = q - 1;
    double gm[3], fd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      gm[c] = 0.;
      fd[c] = LIM != LIM_ORDER1 ? div_rn(ph[c] - ph1[c], x - x1) : 0.;
      if (LIM != LIM_ORDER1 && m > 0 && m < nn - 1) gm[c] = limited_gradient_t<LIM>(fd1[c], fd[c]);
    }
    // update of node o = q - 2: neighbours o-1 (3), o (2), o+1 (1)
    const int o = q - 2;
    if (o >= o0 && o < o1) {
      const long long n = D == 1 ? node_id(M, i, o, tb) : node_id(M, i, tb, o);
      double V[5];
      node_u(F, A, NN, n, V);
      if (o > 0 && o < nn - 1) {
        const double bfm = ffm3, ffm_o = ffm2;
        V[3] += bfm - ffm_o;
        double FV[3], BV[3], FE, BE;
        {
          const double ufront = 0.5 * (ph2[D] + ph1[D]);
          const int signfront = (ufront > 0) ? 1 : -1;
          const bool fr = ffm_o < 0.;
          const double geo = (signfront * (x1 - x2) - dt * ufront);
#pragma unroll
          for (int c = 0; c < 3; ++c) FV[c] = (fr ? ph1[c] : ph2[c]) + order2 * (0.5 * (fr ? gm[c] : g1[c]) * geo);
          FE = (fr ? ph1[3] : ph2[3]) + order2 * (0.5 * 0. * geo);
        }
        {
          const double uback = 0.5 * (ph3[D] + ph2[D]);
          const int signback = (uback > 0) ? 1 : -1;
          const bool bk = bfm > 0.;
          const double geo = (signback * (x2 - x3) - dt * uback);
#pragma unroll
          for (int c = 0; c < 3; ++c) BV[c] = (bk ? ph3[c] : ph2[c]) + order2 * (0.5 * (bk ? g2[c] : g1[c]) * geo);
          BE = (bk ? ph3[3] : ph2[3]) + order2 * (0.5 * 0. * geo);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) V[c] += bfm * BV[c] - ffm_o * FV[c];
        V[4] += bfm * BE - ffm_o * FE;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (fabs(V[c]) < 1.e-300) V[c] = 0.;
      }
#pragma unroll
      for (int c = 0; c < 5; ++c) A.Uout[c * NN + n] = V[c];
    }
    // shift
#pragma unroll
    for (int c = 0; c < 4; ++c) { ph3[c] = ph2[c]; ph2[c] = ph1[c]; ph1[c] = ph[c]; }
#pragma unroll
    for (int c = 0; c < 3; ++c) { g3[c] = g2[c]; g2[c] = g1[c]; g1[c] = gm[c]; fd1[c] = fd[c]; }
    x3 = x2; x2 = x1; x1 = x;
    ffm3 = ffm2; ffm2 = ffm1; ffm1 = ffm;
  }
}

// ---------------------------------------------------------------------------
// Node sweep along D = 1, 2 through a shared-memory tile, classical limiters
// and first order (the layout of body_sweep_cells_tile): the load layout
// stages, per node, its position along D, its projected dual variables, the
// values phi of the limited reconstruction and the mass flux through its
// front half-plane; warp w then runs the arithmetic of
// body_sweep_nodes_lanes on column w, in the same order, and the store
// layout writes the updated variables of the written nodes (NOUT per
// window).
// ---------------------------------------------------------------------------
constexpr int SWTN_SLOTS = 11;  // x, U[5], phi[4], front mass flux
constexpr int SWTN_SMEM_BYTES = SWTN_SLOTS * SWT_FIELD * 8;

template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_nodes_tile(const Mesh& M, const Fields& F, const DualArgs& A, int vbx,
                                                      int vby, double* __restrict__ sm) {
  static_assert(D >= 1, "x sweeps use the lane layout");
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int S_X = 0, S_U = 1, S_PH = 6, S_FFM = 10;
  const long long NN = M.nnode;
  const int nn = D == 1 ? M.nny : M.nnz, nb = D == 1 ? M.nnz : M.nny;
  const int x0 = vbx * SWT_COLS;
  const int g0 = vby * NOUT - 2;  // first position of the window (2 halo nodes)
  // -- 1. load (row layout)
  {
    const int col = threadIdx.x % SWT_COLS, pos = threadIdx.x / SWT_COLS;
    const int i = x0 + col, g = g0 + pos;
    if (i < M.nnx && g >= 0 && g < nb * nn) {
      const int tb = (int)((unsigned)g / (unsigned)nn), id = g - tb * nn;
      const int j = D == 1 ? id : tb, k = D == 1 ? tb : id;
      double ph[4], x, ffm, U[5];
      node_state<DIM, NE, D>(M, F, A, i, j, k, id, ph, x, ffm);
      node_u(F, A, NN, node_id(M, i, j, k), U);
      double* s = sm + pos * SWT_PITCH + col;
      s[S_X * SWT_FIELD] = x;
#pragma unroll
      for (int q = 0; q < 5; ++q) s[(S_U + q) * SWT_FIELD] = U[q];
#pragma unroll
      for (int q = 0; q < 4; ++q) s[(S_PH + q) * SWT_FIELD] = ph[q];
      s[S_FFM * SWT_FIELD] = ffm;
    }
  }
  __syncthreads();
  // -- 2. sweep (warp w: column x0 + w, lane: position along D)
  const int lane = threadIdx.x % SW_LANES, w = threadIdx.x / SW_LANES;
  if (x0 + w < M.nnx && g0 < nb * nn) {  // warp-uniform
    const int g = g0 + lane;
    const bool ok = g >= 0 && g < nb * nn;
    const int id = ok ? g - (int)((unsigned)g / (unsigned)nn) * nn : 0;
    const bool inner = ok && id > 0 && id < nn - 1;
    const bool out = ok && lane >= 2 && lane < 2 + NOUT;
    double* s = sm + lane * SWT_PITCH + w;
    double U[5] = {0., 0., 0., 0., 0.}, ph[4] = {0., 0., 0., 0.}, x = 0., ffm = 0.;
    if (ok) {
      x = s[S_X * SWT_FIELD];
#pragma unroll
      for (int q = 0; q < 5; ++q) U[q] = s[(S_U + q) * SWT_FIELD];
#pragma unroll
      for (int q = 0; q < 4; ++q) ph[q] = s[(S_PH + q) * SWT_FIELD];
      ffm = s[S_FFM * SWT_FIELD];
    }
    const double x_l = __shfl_up_sync(FULL, x, 1), x_r = __shfl_down_sync(FULL, x, 1);
    double ph_l[4], ph_r[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ph_l[q] = __shfl_up_sync(FULL, ph[q], 1);
      ph_r[q] = __shfl_down_sync(FULL, ph[q], 1);
    }
    const double bfm = __shfl_up_sync(FULL, ffm, 1);
    double gr[3], g_l[3], g_r[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      gr[q] = 0.;
      const double gfw = LIM != LIM_ORDER1 ? div_rn(ph_r[q] - ph[q], x_r - x) : 0.;
      const double gbw = __shfl_up_sync(FULL, gfw, 1);
      if (LIM != LIM_ORDER1 && inner) gr[q] = limited_gradient_t<LIM>(gbw, gfw);
      g_l[q] = __shfl_up_sync(FULL, gr[q], 1);
      g_r[q] = __shfl_down_sync(FULL, gr[q], 1);
    }
    if (out && inner) {
      const double dt = F.s->dt;
      const int order2 = LIM == LIM_ORDER1 ? 0 : A.order - 1;  // ordre-projection - 1
      U[3] += bfm - ffm;
      double FV[3], BV[3], FE, BE;
      {
        const double ufront = 0.5 * (ph[D] + ph_r[D]);
        const int signfront = (ufront > 0) ? 1 : -1;
        const bool fr = ffm < 0.;
        const double geo = (signfront * (x_r - x) - dt * ufront);
#pragma unroll
        for (int q = 0; q < 3; ++q) FV[q] = (fr ? ph_r[q] : ph[q]) + order2 * (0.5 * (fr ? g_r[q] : gr[q]) * geo);
        FE = (fr ? ph_r[3] : ph[3]) + order2 * (0.5 * 0. * geo);
      }
      {
        const double uback = 0.5 * (ph_l[D] + ph[D]);
        const int signback = (uback > 0) ? 1 : -1;
        const bool bk = bfm > 0.;
        const double geo = (signback * (x - x_l) - dt * uback);
#pragma unroll
        for (int q = 0; q < 3; ++q) BV[q] = (bk ? ph_l[q] : ph[q]) + order2 * (0.5 * (bk ? g_l[q] : gr[q]) * geo);
        BE = (bk ? ph_l[3] : ph[3]) + order2 * (0.5 * 0. * geo);
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) U[q] += bfm * BV[q] - ffm * FV[q];
      U[4] += bfm * BE - ffm * FE;
#pragma unroll
      for (int q = 0; q < 3; ++q)
        if (fabs(U[q]) < 1.e-300) U[q] = 0.;
#pragma unroll
      for (int q = 0; q < 5; ++q) s[(S_U + q) * SWT_FIELD] = U[q];  // the lane's own slots
    }
    // outer nodes (not inner) keep their staged U
  }
  __syncthreads();
  // -- 3. store (row layout), written positions only
  {
    const int col = threadIdx.x % SWT_COLS, pos = threadIdx.x / SWT_COLS;
    const int i = x0 + col, g = g0 + pos;
    if (pos >= 2 && pos < 2 + NOUT && i < M.nnx && g < nb * nn) {
      const int tb = (int)((unsigned)g / (unsigned)nn), id = g - tb * nn;
      const long long n = node_id(M, i, D == 1 ? id : tb, D == 1 ? tb : id);
      const double* s = sm + pos * SWT_PITCH + col;
#pragma unroll
      for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = s[(S_U + q) * SWT_FIELD];
    }
  }
  __syncthreads();  // the tile is reused by the block's next work item
}

}  // namespace mhc
