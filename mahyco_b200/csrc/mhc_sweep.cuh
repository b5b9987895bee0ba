// mhc_sweep.cuh -- one direction of the ADI remap, tiled along the sweep.
//
// Blocks own a tile of TD cells (nodes) along the sweep direction D times TW
// lanes along x (TW = 1 for the x sweep, whose tile then runs along x).  Each
// tile reads its cells once plus two halo cells on each side into shared
// memory, and every intermediate of the reference -- phi, face gradient,
// limited cell gradient, upwind face value -- is computed once per cell or
// face and shared by the neighbours, with the operation order of the
// reference function it replaces.  Variables are processed one at a time so
// the shared footprint does not grow with the number of environments.
#pragma once
#include "mhc_kernels.cuh"

namespace mhc {

template <int D> struct SweepTile {
  static constexpr int TW = D == 0 ? 1 : 32;
  static constexpr int TD = D == 0 ? 128 : 16;
  static constexpr int THREADS = TW * TD;
  static constexpr int NS = TD + 4;  // slots -2 .. TD+1
};

// cell (or node) coordinates of tile slot s (along D) and lane tw
template <int D>
__device__ __forceinline__ void tile_coord(int s, int tw, int& i, int& j, int& k) {
  constexpr int TW = SweepTile<D>::TW, TD = SweepTile<D>::TD;
  if (D == 0) { i = blockIdx.x * TD + s; j = blockIdx.y; k = blockIdx.z; }
  else if (D == 1) { i = blockIdx.x * TW + tw; j = blockIdx.y * TD + s; k = blockIdx.z; }
  else { i = blockIdx.x * TW + tw; j = blockIdx.z; k = blockIdx.y * TD + s; }
}

template <int D>
__device__ __forceinline__ int along(int i, int j, int k) { return D == 0 ? i : (D == 1 ? j : k); }

struct SweepArgs {
  const double* Uin;
  double* Uout;
  int first;
  int order;
  int limiter;
};

// ---------------------------------------------------------------------------
// cell part: computeGradPhiFace + computeGradPhiCell +
// computeUpwindFaceQuantitiesForProjection + computeUremap
// (RemapADIService.cc:119-575, UtilesRemap.cc:108-120, 325-357; classical
// limiters, order <= 2).  Face quantities of the Lagrangian mesh
// (PrepareRemap.cc:18-59) are rebuilt from the node positions; the initial
// face normals are the unit axis vectors of the cartesian grid, so every
// dot(., n) of the reference reduces to the D component.
// ---------------------------------------------------------------------------
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

template <int DIM, int NE, int D>
__global__ void __launch_bounds__(SweepTile<D>::THREADS)
k_sweep_cells(Mesh M, mhc_case_params P, Fields F, SweepArgs A) {
  using T = SweepTile<D>;
  constexpr int TW = T::TW, TD = T::TD, NS = T::NS;
  constexpr int NV = 3 * NE + 1;
  __shared__ double s_den[NS * TW];     // phi denominator per slot
  __shared__ double s_xc[NS * TW];      // Lagrangian cell centre along D
  __shared__ double s_phi[NS * TW];     // phi of the current variable
  __shared__ double s_gf[(NS - 1) * TW];  // face gradient, then upwind face value
  __shared__ double s_gr[(NS - 2) * TW];  // limited cell gradient (slots -1 .. TD)
  __shared__ double s_un[(TD + 1) * TW], s_L[(TD + 1) * TW], s_fc[(TD + 1) * TW];
  __shared__ unsigned char s_ok[NS * TW];
  const long long N = M.ncell;
  const int nd = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  const double dt = F.s->dt;
  const int NBN = DIM == 3 ? 8 : 4;
  const double wc = DIM == 2 ? .25 : .125;
  const double wf = DIM == 2 ? .5 : .25;
  const double* Xd = F.Xn[D];
  const double* vD = D == 0 ? F.vx : (D == 1 ? F.vy : F.vz);
  const int tid = threadIdx.x;

  // stage 0: slots (cells) -- validity, phi denominator, centre along D;
  // faces 0..TD (back face of slots 0..TD) -- Lagrangian geometry
  for (int it = tid; it < NS * TW; it += T::THREADS) {
    const int tw = it % TW, s = it / TW - 2;
    int i, j, k;
    tile_coord<D>(s, tw, i, j, k);
    const int a = along<D>(i, j, k);
    bool ok = a >= 0 && a < nd && i < M.ncx && j < M.ncy && (DIM == 2 || k < M.ncz);
    s_ok[it] = ok;
    if (!ok) continue;
    const long long c = cell_id(M, i, j, k);
    double den;
    if (A.first) den = F.V[c];
    else { den = 0.; for (int q = 0; q < NE; ++q) den += A.Uin[q * N + c]; }
    s_den[it] = den;
    double sum = 0.;
    for (int l = 0; l < NBN; ++l) {
      int da, db, dc;
      local_node_offset(l, da, db, dc);
      sum += Xd[node_id(M, i + da, j + db, k + dc)];
    }
    s_xc[it] = wc * sum;
    if (s >= 0 && s <= TD) {
      // back face of this cell
      long long fn[4];
      const int nfn = DIM == 3 ? 4 : 2;
      double fc = 0., vm = 0.;
      for (int q = 0; q < nfn; ++q) {
        int fa, fb, fz;
        face_node_ijk2<DIM, D>(i, j, k, q, fa, fb, fz);
        fn[q] = node_id(M, fa, fb, fz);
        fc = fc + wf * Xd[fn[q]];
        vm = vm + vD[fn[q]];
      }
      double L;
      if (DIM == 3) {
        R3 x0 = {F.Xn[0][fn[0]], F.Xn[1][fn[0]], F.Xn[2][fn[0]]};
        R3 x1 = {F.Xn[0][fn[1]], F.Xn[1][fn[1]], F.Xn[2][fn[1]]};
        R3 x2 = {F.Xn[0][fn[2]], F.Xn[1][fn[2]], F.Xn[2][fn[2]]};
        R3 x3 = {F.Xn[0][fn[3]], F.Xn[1][fn[3]], F.Xn[2][fn[3]]};
        R3 v1 = x2 - x0, v2 = x3 - x1;
        if (D == 0) L = 0.5 * fabs(produit(v1.y, v2.z, v1.z, v2.y));
        else if (D == 1) L = 0.5 * fabs(produit(v2.x, v1.z, v2.z, v1.x));
        else L = 0.5 * fabs(produit(v1.x, v2.y, v1.y, v2.x));
      } else {
        const double* Xt = F.Xn[1 - D];
        L = fabs(Xt[fn[1]] - Xt[fn[0]]);
      }
      const int f = s * TW + tw;
      s_fc[f] = fc;
      s_un[f] = wf * vm;
      s_L[f] = L;
    }
  }
  // own cell: outer normals (initial grid, MahycoModule.cc:1070-1091)
  const int tw0 = tid % TW, s0 = tid / TW;
  int i0, j0, k0;
  tile_coord<D>(s0, tw0, i0, j0, k0);
  const int me = (s0 + 2) * TW + tw0;
  __syncthreads();
  const bool mine = s_ok[me];
  double ond[2] = {0., 0.};
  long long c0 = 0;
  if (mine) {
    c0 = cell_id(M, i0, j0, k0);
    R3 sc = {0., 0., 0.};
    for (int l = 0; l < NBN; ++l) {
      int da, db, dc;
      local_node_offset(l, da, db, dc);
      sc = sc + node_x0(M, i0 + da, j0 + db, k0 + dc);
    }
    const R3 cc0 = wc * sc;
    for (int f = 0; f < 2; ++f) {
      int fi = i0, fj = j0, fk = k0;
      if (D == 0) fi += f; else if (D == 1) fj += f; else fk += f;
      R3 fc0 = {0., 0., 0.};
      for (int q = 0; q < (DIM == 3 ? 4 : 2); ++q) {
        int a, b, cz;
        face_node_ijk2<DIM, D>(fi, fj, fk, q, a, b, cz);
        fc0 = fc0 + wf * node_x0(M, a, b, cz);
      }
      R3 diff = fc0 - cc0;
      ond[f] = comp(diff / norm(diff), D);
    }
  }
  const int order2 = A.order - 1;
  double uo[NV], dualm[NE];
  for (int q = 0; q < NE; ++q) dualm[q] = 0.;
  // cell local face order: 3D back then front; 2D x sweep: front then back
  constexpr int FA = (DIM == 2 && D == 0) ? 1 : 0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    // a: phi of every slot
    for (int it = tid; it < NS * TW; it += T::THREADS) {
      if (!s_ok[it]) continue;
      const int tw = it % TW, s = it / TW - 2;
      int i, j, k;
      tile_coord<D>(s, tw, i, j, k);
      s_phi[it] = A.Uin[v * N + cell_id(M, i, j, k)] / s_den[it];
    }
    __syncthreads();
    // b: face gradients, faces between slots s-1 and s for s = -1 .. TD+1
    for (int it = tid; it < (NS - 1) * TW; it += T::THREADS) {
      const int hi = it + TW, lo = it;  // slot indices (offset by 2) of the two cells
      s_gf[it] = (s_ok[lo] && s_ok[hi]) ? (s_phi[hi] - s_phi[lo]) / (s_xc[hi] - s_xc[lo]) : 0.;
    }
    __syncthreads();
    // c: limited gradients of slots -1 .. TD
    for (int it = tid; it < (NS - 2) * TW; it += T::THREADS) {
      const int slot = it + TW;  // offset-2 index of slot s = it/TW - 1
      double g = 0.;
      if (A.order > 1 && s_ok[slot]) g = limited_gradient(A.limiter, s_gf[it], s_gf[it + TW]);
      s_gr[it] = g;
    }
    __syncthreads();
    // d: upwind face values of faces 0 .. TD (between slots f-1 and f)
    for (int it = tid; it < (TD + 1) * TW; it += T::THREADS) {
      const int lo = it + TW, hi = it + 2 * TW;  // offset-2 slot indices of f-1, f
      double pf = 0.;
      if (s_ok[lo] && s_ok[hi]) {
        const double dx = s_xc[hi] - s_xc[lo];
        const bool back = s_un[it] * dx > 0.0;
        const int su = back ? lo : hi;
        pf = s_phi[su] + order2 * (s_fc[it] - s_xc[su]) * s_gr[su - TW];
      }
      s_gf[it] = pf;  // reuse: upwind value of face it
    }
    __syncthreads();
    // e: conservative update of the own cell
    if (mine) {
      const int fb = s0 * TW + tw0, ff = fb + TW;  // back and front faces
      const bool exb = s_ok[me - TW], exf = s_ok[me + TW];
      double flux[2];
      flux[0] = exb ? ond[0] * s_un[fb] * s_L[fb] * dt * s_gf[fb] : 0.;
      flux[1] = exf ? ond[1] * s_un[ff] * s_L[ff] * dt * s_gf[ff] : 0.;
      const bool ex[2] = {exb, exf};
      double sumf = 0., dual = 0.;
      if (ex[FA]) { sumf += flux[FA]; dual += 0.5 * flux[FA] * ond[FA]; }
      if (ex[1 - FA]) { sumf += flux[1 - FA]; dual += 0.5 * flux[1 - FA] * ond[1 - FA]; }
      uo[v] = A.Uin[v * N + c0] - sumf;
      if (v >= NE && v < 2 * NE) dualm[v - NE] = dual;
    }
    __syncthreads();
  }
  if (!mine) return;
  for (int q = 0; q < NE; ++q) {
    if (uo[NE + q] < 0.) uo[NE + q] = 0.;
    if (uo[2 * NE + q] < 0.) uo[2 * NE + q] = 0.;
  }
  for (int v = 0; v < NV; ++v) A.Uout[v * N + c0] = uo[v];
  for (int q = 0; q < NE; ++q) F.mflux[q * N + c0] = dualm[q];
}

// ---------------------------------------------------------------------------
// node part: RemapADIService::computeDualUremap (DualPhaseRemap.cc:38-258,
// classical limiter), tiled along D over the nodes.
// ---------------------------------------------------------------------------
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

template <int DIM, int NE, int D>
__global__ void __launch_bounds__(SweepTile<D>::THREADS)
k_sweep_nodes(Mesh M, mhc_case_params P, Fields F, DualArgs A) {
  using T = SweepTile<D>;
  constexpr int TW = T::TW, TD = T::TD, NS = T::NS;
  __shared__ double s_ph[4][NS * TW];  // phi components 0,1,2 and 4
  __shared__ double s_x[NS * TW];
  __shared__ double s_g[3][(NS - 2) * TW];
  __shared__ unsigned char s_ok[NS * TW], s_in[NS * TW];
  const long long NN = M.nnode, N = M.ncell;
  const int nn = D == 0 ? M.nnx : (D == 1 ? M.nny : M.nnz);
  const int tid = threadIdx.x;
  auto loadU = [&](long long m, double* U) {
    if (A.Uin) {
      for (int q = 0; q < 5; ++q) U[q] = A.Uin[q * NN + m];
    } else {
      double mn = F.mn[m], vx = F.vx[m], vy = F.vy[m], vz = F.vz[m];
      U[0] = mn * vx; U[1] = mn * vy; U[2] = mn * vz; U[3] = mn;
      U[4] = 0.5 * mn * (vx * vx + vy * vy + vz * vz);
    }
  };
  // stage a: phi_dual and Lagrangian coordinate of every slot
  for (int it = tid; it < NS * TW; it += T::THREADS) {
    const int tw = it % TW, s = it / TW - 2;
    int i, j, k;
    tile_coord<D>(s, tw, i, j, k);
    const int a = along<D>(i, j, k);
    bool ok = a >= 0 && a < nn && i < M.nnx && j < M.nny && (DIM == 2 || k < M.nnz);
    s_ok[it] = ok;
    if (!ok) continue;
    s_in[it] = node_inner_dir(M, i, j, k, D);
    const long long m = node_id(M, i, j, k);
    s_x[it] = F.Xn[D][m];
    bool was_inner = false;
    for (int d = 0; d < DIM; ++d)
      if (((A.done_dirs >> d) & 1) && node_inner_dir(M, i, j, k, d)) was_inner = true;
    if (was_inner) {
      double U[5];
      loadU(m, U);
      s_ph[0][it] = U[0] / U[3]; s_ph[1][it] = U[1] / U[3]; s_ph[2][it] = U[2] / U[3];
      s_ph[3][it] = U[4] / U[3];
    } else {
      double vx = F.vx[m], vy = F.vy[m], vz = F.vz[m];
      s_ph[0][it] = vx; s_ph[1][it] = vy; s_ph[2][it] = vz;
      s_ph[3][it] = 0.5 * (vx * vx + vy * vy + vz * vz);
    }
  }
  __syncthreads();
  // stage b: limited gradients of inner nodes, slots -1 .. TD
  for (int it = tid; it < (NS - 2) * TW; it += T::THREADS) {
    const int sl = it + TW;  // offset-2 slot index
    for (int q = 0; q < 3; ++q) {
      double g = 0.;
      if (A.order > 1 && s_ok[sl] && s_in[sl]) {
        double gf = (s_ph[q][sl + TW] - s_ph[q][sl]) / (s_x[sl + TW] - s_x[sl]);
        double gb = (s_ph[q][sl] - s_ph[q][sl - TW]) / (s_x[sl] - s_x[sl - TW]);
        g = limited_gradient(A.limiter, gb, gf);
      }
      s_g[q][it] = g;
    }
  }
  __syncthreads();
  const int tw0 = tid % TW, s0 = tid / TW;
  const int me = (s0 + 2) * TW + tw0;
  if (!s_ok[me]) return;
  int i, j, k;
  tile_coord<D>(s0, tw0, i, j, k);
  const long long n = node_id(M, i, j, k);
  double U[5];
  loadU(n, U);
  if (!s_in[me]) {
    for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
    return;
  }
  const int id = along<D>(i, j, k);
  // node mass fluxes: faces of the node plane in face id order, then envs
  const double w = DIM == 2 ? .5 : .25;
  double bfm = 0., ffm = 0.;
  const int ndc = D == 0 ? M.ncx : (D == 1 ? M.ncy : M.ncz);
  for (int b2 = 0; b2 < (DIM == 3 ? 2 : 1); ++b2) {
    for (int b1 = 0; b1 < 2; ++b1) {
      int ci = i, cj = j, ck = k;
      int t1 = b1 - 1, t2 = b2 - 1;
      if (D == 0) { cj += t1; ck += (DIM == 3 ? t2 : 0); }
      else if (D == 1) { ci += t1; ck += (DIM == 3 ? t2 : 0); }
      else { ci += t1; cj += t2; }
      if (ci < 0 || cj < 0 || ck < 0) continue;
      if (D != 0 && ci >= M.ncx) continue;
      if (D != 1 && cj >= M.ncy) continue;
      if (DIM == 3 && D != 2 && ck >= M.ncz) continue;
      int bi = ci, bj = cj, bk = ck, fi = ci, fj = cj, fk = ck;
      if (D == 0) { bi = id - 1; fi = id; } else if (D == 1) { bj = id - 1; fj = id; } else { bk = id - 1; fk = id; }
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
  const double dt = F.s->dt;
  const int order2 = A.order - 1;
  const int sb = me - TW, sf = me + TW;
  const int gme = me - TW;  // index into s_g (slot offset 1)
  U[3] += bfm - ffm;
  double FV[3], BV[3], FE, BE;
  {
    double ufront = 0.5 * (s_ph[D][me] + s_ph[D][sf]);
    int signfront = (ufront > 0) ? 1 : -1;
    bool fr = ffm < 0.;
    int src = fr ? sf : me, gsrc = fr ? gme + TW : gme;
    double geo = (signfront * (s_x[sf] - s_x[me]) - dt * ufront);
    for (int q = 0; q < 3; ++q) FV[q] = s_ph[q][src] + order2 * (0.5 * s_g[q][gsrc] * geo);
    FE = s_ph[3][src] + order2 * (0.5 * 0. * geo);
  }
  {
    double uback = 0.5 * (s_ph[D][sb] + s_ph[D][me]);
    int signback = (uback > 0) ? 1 : -1;
    bool bk_ = bfm > 0.;
    int src = bk_ ? sb : me, gsrc = bk_ ? gme - TW : gme;
    double geo = (signback * (s_x[me] - s_x[sb]) - dt * uback);
    for (int q = 0; q < 3; ++q) BV[q] = s_ph[q][src] + order2 * (0.5 * s_g[q][gsrc] * geo);
    BE = s_ph[3][src] + order2 * (0.5 * 0. * geo);
  }
  for (int q = 0; q < 3; ++q) U[q] += bfm * BV[q] - ffm * FV[q];
  U[4] += bfm * BE - ffm * FE;
  for (int q = 0; q < 3; ++q)
    if (fabs(U[q]) < 1.e-300) U[q] = 0.;
  for (int q = 0; q < 5; ++q) A.Uout[q * NN + n] = U[q];
}

}  // namespace mhc
