// mhc_sweeps.cu -- launches of the remap sweeps, one kernel per (dimension,
// number of environments, direction, sweep instance).  They are the bulk of
// the template instances, so this file is compiled once per number of
// environments (MHC_SWEEP_PART = NE - 1) and the parts build in parallel;
// part 0 also holds the dispatcher.
#include "mhc_engine.cuh"

#ifndef MHC_SWEEP_PART
#error "compile with -DMHC_SWEEP_PART=0..3 (number of environments - 1)"
#endif

namespace {

// elasto-plastic cases with the remap: one environment, the warp-per-line
// sweep with the seven elasto variables
template <int DIM, int LIM>
void cell_sweep_elasto(Engine* e, Group& g, int D, int k) {
  StageTimer tm(e, MHC_STAGE_SWEEP_CELLS);
  if (D == 0) plaunch(e, kb_sweep_cells<DIM, 1, 0, LIM, MHC_ELASTO_XV>, SW_THREADS, 0, g.sw_cells[0], k);
  else if (D == 1) plaunch(e, kb_sweep_cells<DIM, 1, 1, LIM, MHC_ELASTO_XV>, SW_THREADS, 0, g.sw_cells[1], k);
  else if constexpr (DIM == 3) plaunch(e, kb_sweep_cells<DIM, 1, 2, LIM, MHC_ELASTO_XV>, SW_THREADS, 0, g.sw_cells[2], k);
}

template <int DIM, int NE, int LIM>
void cell_sweep(Engine* e, Group& g, int D, int k) {
  StageTimer tm(e, MHC_STAGE_SWEEP_CELLS);
  if (D == 0) plaunch(e, kb_sweep_cells<DIM, NE, 0, LIM>, SW_THREADS, 0, g.sw_cells[0], k);
  else if (D == 1) plaunch(e, kb_sweep_cells<DIM, NE, 1, LIM>, SW_THREADS, 0, g.sw_cells[1], k);
  else if constexpr (DIM == 3) plaunch(e, kb_sweep_cells<DIM, NE, 2, LIM>, SW_THREADS, 0, g.sw_cells[2], k);
}

// y / z cell sweeps through the shared-memory tile
template <int DIM, int NE, int LIM>
void cell_sweep_tile(Engine* e, Group& g, int D, int k) {
  StageTimer tm(e, MHC_STAGE_SWEEP_CELLS);
  if (D == 1) plaunch(e, kb_sweep_cells_tile<DIM, NE, 1, LIM>, SWT_THREADS, swt_smem_bytes(NE), g.sw_cells[1], k);
  else if constexpr (DIM == 3) plaunch(e, kb_sweep_cells_tile<DIM, NE, 2, LIM>, SWT_THREADS, swt_smem_bytes(NE), g.sw_cells[2], k);
}

// y / z node sweeps through the shared-memory tile
template <int DIM, int NE, int LIM>
void node_sweep_tile(Engine* e, Group& g, int D, int k) {
  StageTimer tm(e, MHC_STAGE_SWEEP_NODES);
  if (D == 1) plaunch(e, kb_sweep_nodes_tile<DIM, NE, 1, LIM>, SWT_THREADS, SWTN_SMEM_BYTES, g.sw_nodes[1], k);
  else if constexpr (DIM == 3) plaunch(e, kb_sweep_nodes_tile<DIM, NE, 2, LIM>, SWT_THREADS, SWTN_SMEM_BYTES, g.sw_nodes[2], k);
}

template <int DIM, int NE, int LIM>
void node_sweep(Engine* e, Group& g, int D, int k) {
  StageTimer tm(e, MHC_STAGE_SWEEP_NODES);
  if (D == 0) plaunch(e, kb_sweep_nodes<DIM, NE, 0, LIM>, SW_THREADS, 0, g.sw_nodes[0], k);
  else if (D == 1) plaunch(e, kb_sweep_nodes<DIM, NE, 1, LIM>, SW_THREADS, 0, g.sw_nodes[1], k);
  else if constexpr (DIM == 3) plaunch(e, kb_sweep_nodes<DIM, NE, 2, LIM>, SW_THREADS, 0, g.sw_nodes[2], k);
}

}  // namespace

// one direction of the remap for a group: cell sweep, then node sweep
template <int DIM, int NE>
void sweep_step_dn(Engine* e, Group& g, int D, int k) {
  const int cl = ((g.COLS >> D) & 1) ? LIM_COLS + g.CLIM : g.CLIM;
  if (NE == 1 && g.EL && g.EULER) {
    if constexpr (NE == 1) {
      switch (g.CLIM) {
        case 0: cell_sweep_elasto<DIM, 0>(e, g, D, k); break;
        case 1: cell_sweep_elasto<DIM, 1>(e, g, D, k); break;
        case 2: cell_sweep_elasto<DIM, 2>(e, g, D, k); break;
        default: cell_sweep_elasto<DIM, LIM_ORDER1>(e, g, D, k); break;
      }
    }
  } else if (D > 0 && !((g.COLS >> D) & 1) && ((g.TILE >> D) & 1)) {
    switch (g.CLIM) {
      case 0: cell_sweep_tile<DIM, NE, 0>(e, g, D, k); break;
      case 1: cell_sweep_tile<DIM, NE, 1>(e, g, D, k); break;
      case 2: cell_sweep_tile<DIM, NE, 2>(e, g, D, k); break;
      default: cell_sweep_tile<DIM, NE, LIM_ORDER1>(e, g, D, k); break;
    }
  } else switch (cl) {
    case LIM_COLS + 0: cell_sweep<DIM, NE, LIM_COLS + 0>(e, g, D, k); break;
    case LIM_COLS + 1: cell_sweep<DIM, NE, LIM_COLS + 1>(e, g, D, k); break;
    case LIM_COLS + 2: cell_sweep<DIM, NE, LIM_COLS + 2>(e, g, D, k); break;
    case LIM_COLS + LIM_ORDER1: cell_sweep<DIM, NE, LIM_COLS + LIM_ORDER1>(e, g, D, k); break;
    case 0: cell_sweep<DIM, NE, 0>(e, g, D, k); break;
    case 1: cell_sweep<DIM, NE, 1>(e, g, D, k); break;
    case 2: cell_sweep<DIM, NE, 2>(e, g, D, k); break;
    case LIM_GEN: cell_sweep<DIM, NE, LIM_GEN>(e, g, D, k); break;
    case LIM_O3: cell_sweep<DIM, NE, LIM_O3>(e, g, D, k); break;
    case LIM_PB: cell_sweep<DIM, NE, LIM_PB>(e, g, D, k); break;
    default: cell_sweep<DIM, NE, LIM_ORDER1>(e, g, D, k); break;
  }
  if (g.ADV) return;  // sans-lagrange: no dual projection (PrepareRemap.cc:211)
  const int nl = ((g.NCOLS >> D) & 1) ? LIM_COLS + g.LIM : g.LIM;
  if (D > 0 && !((g.NCOLS >> D) & 1) && ((g.NTILE >> D) & 1)) {
    switch (g.LIM) {
      case 0: node_sweep_tile<DIM, NE, 0>(e, g, D, k); break;
      case 1: node_sweep_tile<DIM, NE, 1>(e, g, D, k); break;
      case 2: node_sweep_tile<DIM, NE, 2>(e, g, D, k); break;
      default: node_sweep_tile<DIM, NE, LIM_ORDER1>(e, g, D, k); break;
    }
  } else switch (nl) {
    case LIM_COLS + 0: node_sweep<DIM, NE, LIM_COLS + 0>(e, g, D, k); break;
    case LIM_COLS + 1: node_sweep<DIM, NE, LIM_COLS + 1>(e, g, D, k); break;
    case LIM_COLS + 2: node_sweep<DIM, NE, LIM_COLS + 2>(e, g, D, k); break;
    case LIM_COLS + LIM_ORDER1: node_sweep<DIM, NE, LIM_COLS + LIM_ORDER1>(e, g, D, k); break;
    case 0: node_sweep<DIM, NE, 0>(e, g, D, k); break;
    case 1: node_sweep<DIM, NE, 1>(e, g, D, k); break;
    case 2: node_sweep<DIM, NE, 2>(e, g, D, k); break;
    case LIM_GEN: node_sweep<DIM, NE, LIM_GEN>(e, g, D, k); break;
    default: node_sweep<DIM, NE, LIM_ORDER1>(e, g, D, k); break;
  }
}

template void sweep_step_dn<2, MHC_SWEEP_PART + 1>(Engine*, Group&, int, int);
template void sweep_step_dn<3, MHC_SWEEP_PART + 1>(Engine*, Group&, int, int);

#if MHC_SWEEP_PART == 0
extern template void sweep_step_dn<2, 2>(Engine*, Group&, int, int);
extern template void sweep_step_dn<3, 2>(Engine*, Group&, int, int);
extern template void sweep_step_dn<2, 3>(Engine*, Group&, int, int);
extern template void sweep_step_dn<3, 3>(Engine*, Group&, int, int);
extern template void sweep_step_dn<2, 4>(Engine*, Group&, int, int);
extern template void sweep_step_dn<3, 4>(Engine*, Group&, int, int);

void sweep_step_any(Engine* e, Group& g, int D, int k) {
  DISPATCH_GROUP(g, (sweep_step_dn<DIM_, NE_>(e, g, D, k)));
}
#endif
