// mhc_launch.cuh -- persistent kernels that run one phase of the cycle over
// a work list of (case, virtual block) items.
//
// A single case is a work list over its own blocks; a batch of uneven cases
// is one list per phase covering every block of every case, so one launch
// per phase advances all of them.  Blocks stride over the list; the case
// descriptor of each item gives its mesh, fields and parameters.  Items of a
// case that is stopped, failed or past its iteration limit are skipped (the
// test is uniform per block).
#pragma once
#include "mhc_kernels.cuh"
#include "mhc_sweep.cuh"

namespace mhc {

struct CaseDesc {
  Mesh M;
  Fields F;
  const mhc_case_params* P;  // device copy of the case parameters
};

struct WorkItem {
  int c;        // case index in the descriptor table
  int x, y, z;  // virtual block index inside the case
};

// work decomposition of the phases: virtual blocks of one case
enum PhaseKind {
  PH_CELLS = 0,      // one block per CT cells
  PH_NODES = 1,      // one block per CT nodes
  PH_UNUSED = 2,
  PH_SWC0 = 3,       // cell sweep along D = PH - PH_SWC0
  PH_SWN0 = 6,       // node sweep along D = PH - PH_SWN0
  PH_SWCW0 = 9,      // cell sweep with the wide (third-order) stencil
  PH_SWNW0 = 12,     // node sweep with the wide (generalised limiter) stencil
  PH_SWCC0 = 15,     // cell sweep along D = 1, 2, one thread per line chunk
  PH_SWNC0 = 18,     // node sweep along D = 1, 2, one thread per line chunk
  PH_SWCT0 = 21,     // cell sweep along D = 1, 2 through a shared-memory tile
  PH_SWNT0 = 24      // node sweep along D = 1, 2 through a shared-memory tile
};

// phase of the cell sweep along D for a cell-sweep instance
__host__ __device__ constexpr int cell_sweep_phase(int lim, int D) {
  return (D > 0 && lim >= LIM_COLS) ? PH_SWCC0 + D : (lim == LIM_O3 ? PH_SWCW0 : PH_SWC0) + D;
}
__host__ __device__ constexpr int node_sweep_phase(int lim, int D) {
  return (D > 0 && lim >= LIM_COLS) ? PH_SWNC0 + D : (lim == LIM_GEN ? PH_SWNW0 : PH_SWN0) + D;
}

// ceil(a / b) for 0 <= a < 2^31 (every count of a case: it has fewer than
// 2^31 nodes), in unsigned 32-bit arithmetic
__host__ __device__ inline int cdiv_i(long long a, int b) {
  return (int)(((unsigned)a + (unsigned)b - 1u) / (unsigned)b);
}

// virtual-block grid (gx, gy, gz) of one case in a phase; blocks are
// numbered with x fastest
__host__ __device__ inline void phase_grid(int ph, const Mesh& M, int& gx, int& gy, int& gz) {
  gy = gz = 1;
  if (ph == PH_CELLS) { gx = cdiv_i(M.ncell, CT); return; }
  if (ph == PH_NODES) { gx = cdiv_i(M.nnode, CT); return; }
  if (ph >= PH_SWNT0) {  // body_sweep_nodes_tile
    const int D = ph - PH_SWNT0;
    const int nb = D == 1 ? M.nnz : M.nny, nd = D == 1 ? M.nny : M.nnz;
    gx = cdiv_i(M.nnx, SWT_COLS);
    gy = cdiv_i((long long)nb * nd, NOUT);
    return;
  }
  if (ph >= PH_SWCT0) {  // body_sweep_cells_tile
    const int D = ph - PH_SWCT0;
    const int nb = D == 1 ? M.ncz : M.ncy, nd = D == 1 ? M.ncy : M.ncz;
    gx = cdiv_i(M.ncx, SWT_COLS);
    gy = cdiv_i((long long)nb * nd, XOUT);
    return;
  }
  if (ph >= PH_SWNC0) {  // body_sweep_nodes_cols
    const int D = ph - PH_SWNC0;
    const int nb = D == 1 ? M.nnz : M.nny, nd = D == 1 ? M.nny : M.nnz;
    gx = cdiv_i((long long)M.nnx * nb, SW_THREADS);
    gy = col_chunks(nd);
    return;
  }
  if (ph >= PH_SWCC0) {  // body_sweep_cells_cols
    const int D = ph - PH_SWCC0;
    const int nb = D == 1 ? M.ncz : M.ncy, nd = D == 1 ? M.ncy : M.ncz;
    gx = cdiv_i((long long)M.ncx * nb, SW_THREADS);
    gy = col_chunks(nd);
    return;
  }
  // lane layout of mhc_sweep.cuh (sweep_lane)
  const bool wide = ph >= PH_SWCW0;
  const int base = wide ? (ph >= PH_SWNW0 ? PH_SWNW0 : PH_SWCW0) : (ph >= PH_SWN0 ? PH_SWN0 : PH_SWC0);
  const bool nodes = base == PH_SWN0 || base == PH_SWNW0;
  const int D = ph - base;
  const int nx = nodes ? M.nnx : M.ncx, ny = nodes ? M.nny : M.ncy, nz = nodes ? M.nnz : M.ncz;
  const int out = wide ? (nodes ? NOUT_W : XOUT_W) : (nodes ? NOUT : XOUT);
  if (D == 0) {
    gx = cdiv_i(cdiv_i((long long)nx * ny * nz, out), SW_ROWS);
  } else {
    gx = cdiv_i(nx, SW_ROWS);
    gy = cdiv_i((long long)ny * nz, out);
  }
}

// the cases of one group and the first virtual block of each (ascending
// prefix sums); a launch covers `total` virtual blocks
struct PhaseList {
  const int* cases;
  const int* start;
  int n;
  int total;
};

// case and virtual block of global block w: binary search of the prefix sums
template <int PH>
__device__ __forceinline__ WorkItem item_at(const CaseDesc* __restrict__ C, const PhaseList& L, int w) {
  int lo = 0, hi = L.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(L.start + mid) <= w) lo = mid;
    else hi = mid - 1;
  }
  const int c = __ldg(L.cases + lo);
  const unsigned b = (unsigned)(w - __ldg(L.start + lo));
  int gx, gy, gz;
  phase_grid(PH, C[c].M, gx, gy, gz);
  if (gy == 1) return WorkItem{c, (int)b, 0, 0};  // every phase but the sweeps
  const unsigned r = b / (unsigned)gx, z = r / (unsigned)gy;
  return WorkItem{c, (int)(b - r * (unsigned)gx), (int)(r - z * (unsigned)gy), (int)z};
}

#define MHC_FOR_ITEMS(L) for (int w_ = blockIdx.x; w_ < (L).total; w_ += gridDim.x)

// directions swept before the k-th sweep of the iteration
// (RemapADIService.cc:23-33)
template <int DIM>
__device__ __forceinline__ int sweep_done_dirs(const Mesh& M, const mhc_case_params& P, long long iteration, int k) {
  int done = 0;
  const int sens = (int)((iteration - 1) % DIM);
  int cnt = 0;
  for (int i = 0; i < M.dim; ++i) {
    const int d = (i + sens) % M.dim;
    const int ncd = d == 0 ? M.ncx : (d == 1 ? M.ncy : M.ncz);
    if (ncd == 1) continue;
    if (P.is_euler_scheme >= MHC_EULER_X && P.is_euler_scheme <= MHC_EULER_Z && d != P.is_euler_scheme - MHC_EULER_X)
      continue;
    if (cnt < k) done |= 1 << d;
    ++cnt;
  }
  return done;
}

template <int DIM, int NE>
__global__ void __launch_bounds__(CT) kb_init_cells(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_init_cells<DIM, NE>(M, *C[wi.c].P, F, wi.x);
  }
}

// the temperature of initEOS (Lagrangian runs; env < 0: every environment)
template <int DIM, int NE>
__global__ void __launch_bounds__(CT) kb_eref_candidates(const CaseDesc* __restrict__ C, PhaseList L, int env) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    const Fields F = C[wi.c].F;
    const Mesh M = C[wi.c].M;
    body_eref_candidates<DIM, NE>(M, *C[wi.c].P, F, env, wi.x);
  }
}

template <int DIM, int NE>
__global__ void __launch_bounds__(CT) kb_init_temperature(const CaseDesc* __restrict__ C, PhaseList L, int env) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    const Fields F = C[wi.c].F;
    const Mesh M = C[wi.c].M;
    body_init_temperature<DIM, NE>(M, *C[wi.c].P, F, env, wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_init_nodes(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_init_nodes<DIM>(M, *C[wi.c].P, F, wi.x);
  }
}

// resident blocks per SM asked of the compiler for the Lagrange cell pass:
// 3 (80 registers) spills a little but hides more of its loads than 2
// (124 registers, no spills)
#ifndef MHC_LAG_MIN_BLOCKS
#define MHC_LAG_MIN_BLOCKS 3
#endif

// resident blocks per SM asked of the compiler for the node pass (a latency
// bound gather: more warps in flight hide more of it)
#ifndef MHC_NODES_MIN_BLOCKS
#define MHC_NODES_MIN_BLOCKS 4
#endif

// LAG: a Lagrangian run (no remap): last positions, pressure surfaces
template <int DIM, bool EL, bool HG, bool LAG, bool CSTS = false>
__global__ void __launch_bounds__(CT, MHC_NODES_MIN_BLOCKS) kb_lagrange_nodes(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_lagrange_nodes<DIM, EL, HG, LAG, CSTS>(M, *C[wi.c].P, F, wi.x);
  }
}

// resident blocks per SM asked of the compiler for the geometry pass
#ifndef MHC_GEOM_MIN_BLOCKS
#define MHC_GEOM_MIN_BLOCKS 1
#endif

template <int DIM>
__global__ void __launch_bounds__(CT, MHC_GEOM_MIN_BLOCKS) kb_lagrange_geom(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_lagrange_geom<DIM>(M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM, int NE, bool EULER, bool EL, bool CSTS = false>
__global__ void __launch_bounds__(CT, MHC_LAG_MIN_BLOCKS) kb_lagrange_cells(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_lagrange_cells<DIM, NE, EULER, EL, CSTS>(M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_hourglass(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_hourglass<DIM>(M, *C[wi.c].P, F, wi.x);
  }
}

// k-th performed sweep of the cycle in direction D: U[k&1] -> U[(k+1)&1]
// resident blocks per SM asked of the compiler for the sweeps (caps their
// registers at 65536 / (SW_THREADS * value)); measured best on B200: 6 for
// the cell sweeps (80 registers), 8 for the node sweeps (64 registers)
#ifndef MHC_SW_MIN_BLOCKS_CELLS
#define MHC_SW_MIN_BLOCKS_CELLS 6
#endif
#ifndef MHC_SW_MIN_BLOCKS_NODES
#define MHC_SW_MIN_BLOCKS_NODES 8
#endif

// the generalised-limiter and third-order instances hold more state per
// lane and are asked for fewer resident blocks
#ifndef MHC_SW_MIN_BLOCKS_COLS
#define MHC_SW_MIN_BLOCKS_COLS 3
#endif
template <int DIM, int NE, int D, int LIM, int XV = 0>
__global__ void __launch_bounds__(SW_THREADS, LIM >= LIM_COLS ? MHC_SW_MIN_BLOCKS_COLS
                                              : (LIM >= LIM_GEN ? 2 : MHC_SW_MIN_BLOCKS_CELLS))
kb_sweep_cells(const CaseDesc* __restrict__ C, PhaseList L, int k) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<cell_sweep_phase(LIM, D)>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const mhc_case_params& P = *C[wi.c].P;
    SweepArgs A;
    A.Uin = (k & 1) ? F.U[1] : F.U[0];
    A.Uout = (k & 1) ? F.U[0] : F.U[1];
    A.first = k == 0;
    A.order = P.ordre_projection;
    A.limiter = P.projection_limiteur_id;
    A.simple_pente = P.projection_simple_pente;
    // EstMixte / EstPure are zero before the first remap of the run
    A.first_remap = k == 0 && F.s->iteration == 1;
    const Mesh M = C[wi.c].M;
    if constexpr (LIM >= LIM_COLS && D > 0) body_sweep_cells_cols<DIM, NE, D, LIM - LIM_COLS>(M, F, A, wi.x, wi.y);
    else if constexpr (LIM >= LIM_COLS) body_sweep_cells_lanes<DIM, NE, D, LIM - LIM_COLS>(M, F, A, wi.x, wi.y);
    else if constexpr (LIM == LIM_O3) body_sweep_cells_o3<DIM, NE, D>(M, F, A, wi.x, wi.y);
    else if constexpr (LIM == LIM_PB) body_sweep_cells_pb<DIM, NE, D>(M, F, P, A, wi.x, wi.y);
    else body_sweep_cells_lanes<DIM, NE, D, LIM, XV>(M, F, A, wi.x, wi.y);
  }
}

// cell sweep along D = 1, 2 through a shared-memory tile (classical
// limiters, first order): SWT_THREADS threads, swt_smem_bytes(NE) of
// dynamic shared memory
#ifndef MHC_SWT_MIN_BLOCKS
#define MHC_SWT_MIN_BLOCKS 3
#endif
template <int DIM, int NE, int D, int LIM>
__global__ void __launch_bounds__(SWT_THREADS, MHC_SWT_MIN_BLOCKS)
kb_sweep_cells_tile(const CaseDesc* __restrict__ C, PhaseList L, int k) {
  extern __shared__ double swt_tile[];
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_SWCT0 + D>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;  // uniform over the block (one case per item)
    resolve_positions(F);
    const mhc_case_params& P = *C[wi.c].P;
    SweepArgs A;
    A.Uin = (k & 1) ? F.U[1] : F.U[0];
    A.Uout = (k & 1) ? F.U[0] : F.U[1];
    A.first = k == 0;
    A.order = P.ordre_projection;
    A.limiter = P.projection_limiteur_id;
    A.simple_pente = P.projection_simple_pente;
    A.first_remap = k == 0 && F.s->iteration == 1;
    const Mesh M = C[wi.c].M;
    body_sweep_cells_tile<DIM, NE, D, LIM>(M, F, A, wi.x, wi.y, swt_tile);
  }
}

// node sweep along D = 1, 2 through a shared-memory tile
#ifndef MHC_SWTN_MIN_BLOCKS
#define MHC_SWTN_MIN_BLOCKS 3
#endif
template <int DIM, int NE, int D, int LIM>
__global__ void __launch_bounds__(SWT_THREADS, MHC_SWTN_MIN_BLOCKS)
kb_sweep_nodes_tile(const CaseDesc* __restrict__ C, PhaseList L, int k) {
  extern __shared__ double swtn_tile[];
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_SWNT0 + D>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;  // uniform over the block (one case per item)
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    const mhc_case_params& P = *C[wi.c].P;
    DualArgs A;
    A.Uin = k == 0 ? nullptr : (((k - 1) & 1) ? F.Ud[1] : F.Ud[0]);
    A.Uout = (k & 1) ? F.Ud[1] : F.Ud[0];
    A.order = P.ordre_projection;
    A.limiter = P.projection_limiteur_id;
    A.simple_pente = P.projection_simple_pente;
    A.done_dirs = sweep_done_dirs<DIM>(M, P, F.s->iteration, k);
    body_sweep_nodes_tile<DIM, NE, D, LIM>(M, F, A, wi.x, wi.y, swtn_tile);
  }
}

#ifndef MHC_SW_MIN_BLOCKS_NODECOLS
#define MHC_SW_MIN_BLOCKS_NODECOLS 4
#endif
template <int DIM, int NE, int D, int LIM>
__global__ void __launch_bounds__(SW_THREADS, LIM >= LIM_COLS ? MHC_SW_MIN_BLOCKS_NODECOLS
                                              : (LIM == LIM_GEN ? 4 : MHC_SW_MIN_BLOCKS_NODES))
kb_sweep_nodes(const CaseDesc* __restrict__ C, PhaseList L, int k) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<node_sweep_phase(LIM, D)>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    const mhc_case_params& P = *C[wi.c].P;
    const int done = sweep_done_dirs<DIM>(M, P, F.s->iteration, k);
    DualArgs A;
    A.Uin = k == 0 ? nullptr : (((k - 1) & 1) ? F.Ud[1] : F.Ud[0]);
    A.Uout = (k & 1) ? F.Ud[1] : F.Ud[0];
    A.order = P.ordre_projection;
    A.limiter = P.projection_limiteur_id;
    A.simple_pente = P.projection_simple_pente;
    A.done_dirs = done;
    if constexpr (LIM >= LIM_COLS && D > 0) body_sweep_nodes_cols<DIM, NE, D, LIM - LIM_COLS>(M, F, A, wi.x, wi.y);
    else if constexpr (LIM >= LIM_COLS) body_sweep_nodes_lanes<DIM, NE, D, LIM - LIM_COLS>(M, F, A, wi.x, wi.y);
    else body_sweep_nodes_lanes<DIM, NE, D, LIM>(M, F, A, wi.x, wi.y);
  }
}

// remap finalize after K performed sweeps: cells read U[K&1], nodes Ud[(K-1)&1]
#ifndef MHC_FIN_MIN_BLOCKS
#define MHC_FIN_MIN_BLOCKS 3
#endif

template <int DIM, int NE, bool ADV = false>
__global__ void __launch_bounds__(CT, MHC_FIN_MIN_BLOCKS) kb_remap_finalize_cells(const CaseDesc* __restrict__ C, PhaseList L, int K) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_remap_finalize_cells<DIM, NE, ADV>(M, *C[wi.c].P, F, (K & 1) ? F.U[1] : F.U[0],
                                            ((K - 1) & 1) ? F.Ud[1] : F.Ud[0], wi.x);
  }
}

template <int DIM, bool DUAL = true>
__global__ void __launch_bounds__(CT) kb_remap_finalize_nodes(const CaseDesc* __restrict__ C, PhaseList L, int K) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_remap_finalize_nodes<DIM, DUAL>(M, F, ((K - 1) & 1) ? F.Ud[1] : F.Ud[0], wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_csts_forward(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_csts_forward<DIM>(M, *C[wi.c].P, F, wi.x);
  }
}

// sans-lagrange (pure advection): prescribed node velocities and positions,
// then the remap quantities of the cells (after kb_lagrange_geom)
template <int DIM>
__global__ void __launch_bounds__(CT) kb_advect_nodes(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_advect_nodes<DIM>(M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM, int NE>
__global__ void __launch_bounds__(CT) kb_advect_cells(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_advect_cells<DIM, NE>(M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_cell_bcs(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    body_cell_bcs<DIM>(C[wi.c].M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_node_bcs(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    body_node_bcs<DIM>(C[wi.c].M, *C[wi.c].P, F, wi.x);
  }
}

template <int DIM>
__global__ void __launch_bounds__(CT) kb_euler_volume(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    body_euler_volume<DIM>(C[wi.c].M, *C[wi.c].P, F, wi.x);
  }
}

static __global__ void __launch_bounds__(CT) kb_euler_axis_reset(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_NODES>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    body_euler_axis_reset(C[wi.c].M, *C[wi.c].P, F, wi.x);
  }
}

// SPD: the node speeds stored by the node finalize pass (remap cases)
template <int DIM, bool SPD = false>
__global__ void __launch_bounds__(CT) kb_delta_t(const CaseDesc* __restrict__ C, PhaseList L) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    if (!case_active(F)) continue;
    resolve_positions(F);
    const Mesh M = C[wi.c].M;
    body_delta_t<DIM, SPD>(M, *C[wi.c].P, F, wi.x);
    __syncthreads();
  }
}

// one thread per case
static __global__ void kb_delta_t_finalize(const CaseDesc* __restrict__ C, const int* __restrict__ cases, int n) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const CaseDesc& cd = C[cases[t]];
    if (!case_active(cd.F)) continue;
    body_delta_t_finalize(*cd.P, cd.F);
  }
}

// copy of every case's scalars into one array (one read-back per poll)
static __global__ void kb_gather_scalars(const CaseDesc* __restrict__ C, int n, Scalars* __restrict__ out) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) out[t] = *C[t].F.s;
}

template <int NE>
__global__ void __launch_bounds__(CT) kb_eos_apply(const CaseDesc* __restrict__ C, PhaseList L, int env) {
  MHC_FOR_ITEMS(L) {
    const WorkItem wi = item_at<PH_CELLS>(C, L, w_);
    Fields F = C[wi.c].F;
    const Mesh M = C[wi.c].M;
    body_eos_apply<NE>(M, *C[wi.c].P, F, env, wi.x);
  }
}

}  // namespace mhc
