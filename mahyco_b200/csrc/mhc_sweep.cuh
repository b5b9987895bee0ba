// mhc_sweep.cuh -- node part of one direction of the ADI remap, tiled along
// the sweep.
//
// Blocks own a tile of TD nodes along the sweep direction D times TW lanes
// along x (TW = 1 for the x sweep, whose tile then runs along x).  Each tile
// reads its nodes once plus two halo nodes on each side into shared memory,
// and every intermediate of the reference -- phi, limited gradient -- is
// computed once per node and shared by the neighbours, with the operation
// order of the reference function it replaces.
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
struct VB { int x, y, z; };  // virtual block index of a tile

template <int D>
__device__ __forceinline__ void tile_coord(const VB& b, int s, int tw, int& i, int& j, int& k) {
  constexpr int TW = SweepTile<D>::TW, TD = SweepTile<D>::TD;
  if (D == 0) { i = b.x * TD + s; j = b.y; k = b.z; }
  else if (D == 1) { i = b.x * TW + tw; j = b.y * TD + s; k = b.z; }
  else { i = b.x * TW + tw; j = b.z; k = b.y * TD + s; }
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
__device__ __forceinline__ void body_sweep_nodes(const Mesh& M, const mhc_case_params& P, const Fields& F,
                                                 const DualArgs& A, VB vb) {
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
    tile_coord<D>(vb, s, tw, i, j, k);
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
  tile_coord<D>(vb, s0, tw0, i, j, k);
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
