// mhc_sweeps.cu -- launches of the remap sweeps, one kernel per (dimension,
// number of environments, direction, limiter); kept in their own
// translation unit because they are the bulk of the template instances.
#include "mhc_engine.cuh"

namespace {

template <int DIM, int NE, int LIM>
void sweep_step(Engine* e, Group& g, int D, int k) {
  {
    StageTimer tm(e, MHC_STAGE_SWEEP_CELLS);
    if (D == 0) plaunch(e, kb_sweep_cells<DIM, NE, 0, LIM>, SW_THREADS, 0, g.sw_cells[0], k);
    else if (D == 1) plaunch(e, kb_sweep_cells<DIM, NE, 1, LIM>, SW_THREADS, 0, g.sw_cells[1], k);
    else if constexpr (DIM == 3) plaunch(e, kb_sweep_cells<DIM, NE, 2, LIM>, SW_THREADS, 0, g.sw_cells[2], k);
  }
  {
    StageTimer tm(e, MHC_STAGE_SWEEP_NODES);
    if (D == 0) plaunch(e, kb_sweep_nodes<DIM, NE, 0, LIM>, SW_THREADS, 0, g.sw_nodes[0], k);
    else if (D == 1) plaunch(e, kb_sweep_nodes<DIM, NE, 1, LIM>, SW_THREADS, 0, g.sw_nodes[1], k);
    else if constexpr (DIM == 3) plaunch(e, kb_sweep_nodes<DIM, NE, 2, LIM>, SW_THREADS, 0, g.sw_nodes[2], k);
  }
}

template <int DIM, int NE>
void sweep_step_lim(Engine* e, Group& g, int D, int k) {
  switch (g.LIM) {
    case 0: sweep_step<DIM, NE, 0>(e, g, D, k); break;
    case 1: sweep_step<DIM, NE, 1>(e, g, D, k); break;
    case 2: sweep_step<DIM, NE, 2>(e, g, D, k); break;
    default: sweep_step<DIM, NE, LIM_ORDER1>(e, g, D, k); break;
  }
}

}  // namespace

void sweep_step_any(Engine* e, Group& g, int D, int k) {
  DISPATCH_GROUP(g, (sweep_step_lim<DIM_, NE_>(e, g, D, k)));
}
