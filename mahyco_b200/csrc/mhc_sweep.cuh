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
  const double* vD = D == 0 ? F.vx : (D == 1 ? F.vy : F.vz);
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
// two halo elements on each side, whatever the line length.
//  * D = 0: lines are consecutive in memory; window w = vbx * SW_ROWS + row
//    covers flat positions [w*out - 2, w*out + 30).
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
__device__ __forceinline__ bool sweep_lane(int nx, int ny, int nz, int out, int vbx, int vby, int lane, int row,
                                           int& i, int& j, int& k, int& p, int& ta, int& tb) {
  i = j = k = p = ta = tb = 0;
  if (D == 0) {
    const long long g = ((long long)vbx * SW_ROWS + row) * out - 2 + lane;
    if (g < 0 || g >= (long long)nx * ny * nz) return false;
    i = (int)(g % nx);
    const long long r = g / nx;
    j = (int)(r % ny);
    k = (int)(r / ny);
    p = i; ta = j; tb = k;
    return true;
  }
  const int nd = D == 1 ? ny : nz, nb = D == 1 ? nz : ny;
  ta = vbx * SW_ROWS + row;
  const long long g = (long long)vby * out - 2 + lane;
  if (ta >= nx || g < 0 || g >= (long long)nb * nd) return false;
  tb = (int)(g / nd);
  p = (int)(g % nd);
  i = ta;
  if (D == 1) { j = p; k = tb; }
  else { j = tb; k = p; }
  return true;
}

// the whole warp holds nothing (warp-uniform test, before any shuffle)
template <int D>
__device__ __forceinline__ bool sweep_warp_empty(int nx, int ny, int nz, int out, int vbx, int vby, int row) {
  if (D == 0) return ((long long)vbx * SW_ROWS + row) * out - 2 >= (long long)nx * ny * nz;
  const int nd = D == 1 ? ny : nz, nb = D == 1 ? nz : ny;
  return vbx * SW_ROWS + row >= nx || (long long)vby * out - 2 >= (long long)nb * nd;
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

// ---------------------------------------------------------------------------
// Cell sweep along D with warp shuffles.  A warp holds 32 consecutive cells
// along D (lane l: cell x0 - 2 + l), loads the back node plane of each and
// takes the front plane from lane l+1; stencil neighbours come from lanes
// l-1 / l+1.  Lanes 2 .. XOUT+1 write.  Virtual block: x = window index
// along D, y = group of SW_ROWS rows.  Rows are the transverse cells with
// the lowest transverse axis fastest, so the warps of a block read
// neighbouring columns and share L1 sectors.
// ---------------------------------------------------------------------------
template <int DIM, int NE, int D, int LIM>
__device__ __forceinline__ void body_sweep_cells_lanes(const Mesh& M, const Fields& F, const SweepArgs& A,
                                                       int vbx, int vby) {
  constexpr int NV = 3 * NE + 1;
  constexpr int NQ = DIM == 3 ? 4 : 2;
  constexpr unsigned FULL = 0xffffffffu;
  const long long N = M.ncell;
  const int lane = threadIdx.x % SW_LANES, row = threadIdx.x / SW_LANES;
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  if (sweep_warp_empty<D>(M.ncx, M.ncy, M.ncz, XOUT, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, p, ta, tb;
  const bool ok = sweep_lane<D>(M.ncx, M.ncy, M.ncz, XOUT, vbx, vby, lane, row, i, j, k, p, ta, tb);
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
    const double gr = (LIM != LIM_ORDER1 && ok) ? limited_gradient_t<LIM>(gf, gf_r) : 0.;
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
// Node part: RemapADIService::computeDualUremap (DualPhaseRemap.cc:38-258,
// classical limiter) with the same lane layout.  Lane l holds node
// x0 - 2 + l along D; lanes 2 .. NOUT+1 write.  The mass flux through the
// back half-plane of a node is the flux through the front half-plane of the
// node behind it, summed over the same cells in the same order, so each
// lane sums its front cells once and hands the sum to lane l+1.
// ---------------------------------------------------------------------------
constexpr int NOUT = 28;  // nodes written per warp (lanes 2 .. 29)

struct DualArgs {
  const double* Uin;   // null on the first sweep (U built from m and v)
  double* Uout;
  int order;
  int limiter;
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
  if (sweep_warp_empty<D>(M.nnx, M.nny, M.nnz, NOUT, vbx, vby, row)) return;  // whole warp leaves together
  int i, j, k, id, ta, tb;
  const bool ok = sweep_lane<D>(M.nnx, M.nny, M.nnz, NOUT, vbx, vby, lane, row, i, j, k, id, ta, tb);
  const bool inner = ok && id > 0 && id < nn - 1;
  const bool out = ok && lane >= 2 && lane < 2 + NOUT;
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
  // limited gradients of the velocity components (inner nodes only)
  double g[3], g_l[3], g_r[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    g[q] = 0.;
    if (LIM != LIM_ORDER1 && inner) {
      const double gfw = div_rn(ph_r[q] - ph[q], x_r - x);
      const double gbw = div_rn(ph[q] - ph_l[q], x - x_l);
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
  const int order2 = LIM == LIM_ORDER1 ? 0 : 1;  // ordre-projection - 1
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

}  // namespace mhc
