// mhc_engine.cuh -- host-side engine shared by the C ABI translation units:
// cases, groups of cases that share kernel templates, per-phase work lists,
// and the persistent launch helper.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "../../include/mahyco_b200.h"
#include "mhc_launch.cuh"

namespace mhc {

// records the calling thread's error message (mhc_last_error) and returns code
int set_err(int code, const std::string& msg);

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return ::mhc::set_err(MHC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

enum Stage { S_IDLE = 0, S_SAVED, S_VELOCITY, S_BC, S_POSITION, S_GEOM, S_DENSITY, S_VISCO, S_ELASTO, S_ENERGY, S_REMAP,
             S_SWEPT /* remap sweeps done, remapVariables pending */ };

inline int cdiv(long long a, int b) { return (int)((a + b - 1) / b); }

}  // namespace mhc

struct Engine;

using namespace mhc;

struct mhc_case {
  mhc_case_params P;
  Mesh M;
  int DIM = 3, NE = 1, NV = 4;
  Fields F;
  Scalars* d_scal = nullptr;
  mhc_case_params* d_params = nullptr;
  cudaStream_t stream = nullptr;   // allocation stream (and launches when standalone)
  bool own_stream = false;
  std::vector<void*> allocs;
  std::vector<size_t> alloc_bytes;  // size of each allocation (checkpoints)
  // asynchronous status read-back: two pinned slots and their events
  Scalars* h_scal = nullptr;
  cudaEvent_t scal_ev[2] = {nullptr, nullptr};
  int scal_next = 0;
  long long it_host = 1;           // iteration the next launched cycle runs
  int stage = S_IDLE;
  bool initialised = false;
  Engine* solo = nullptr;          // private engine of a standalone case
  int slot = -1;                   // index inside its engine
};

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
struct DevList {
  size_t off_cases = 0;  // offsets inside the engine's int arena
  size_t off_start = 0;
  int n = 0;             // member cases
  int total = 0;         // virtual blocks of all members
};

struct Group {
  int DIM, NE, EULER, skip;
  int EL = 0, HG = 0;          // elasto-plastic model; anti-hourglass correction
  int CBC = 0;                 // cell-variable boundary conditions (Density, Energy, Pressure)
  int LIM = 0;                 // node-sweep instance: limiter 0-2, LIM_ORDER1 or LIM_GEN
  int CLIM = 0;                // cell-sweep instance: the same, LIM_O3 (third order) or LIM_PB (pente-borne)
  int COLS = 0;                // bit D: the classical cell sweep along D uses one thread per line chunk
  int TILE = 0;                // bit D: ... or a shared-memory tile (when not COLS)
  int NTILE = 0;               // bit D: the node sweep along D uses a shared-memory tile (when not NCOLS)
  int NCOLS = 0;               // bit D: the same for the node sweep
  int ADV = 0;                 // sans-lagrange: prescribed velocities, no Lagrange phase, no dual projection
  int CSTS = 0;                // schema-csts with the remap: half-step velocity updates around the step
  long long it0;               // iteration of the members when the lists were built
  std::vector<int> members;
  DevList init_cells, init_nodes, lag_nodes, lag_cells, fin_cells, fin_nodes, dt;
  DevList sw_cells[3], sw_nodes[3];
  DevList cases;               // offset into the case-index arena
};

struct Engine {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<mhc_case*> cases;
  CaseDesc* d_desc = nullptr;
  int desc_cap = 0;
  int* d_ints = nullptr;   // case indices and block prefix sums of every list
  size_t ints_cap = 0;
  std::vector<Group> groups;
  bool dirty = true;
  long long cycles_since_build = 0;
  int nsm = 0;
  // timing
  bool timing = false;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double stage_ms[MHC_NUM_STAGES] = {0};
  long long stage_launches[MHC_NUM_STAGES] = {0};
  // graph of one rotation period
  cudaGraphExec_t graph = nullptr;
  // grid of the work-list launches: 0 = one block per work item (the block
  // scheduler balances), k > 0 = k x the blocks the device holds at once
  // (persistent blocks striding over the list)
  int grid_scale = 0;
  // per-phase override of grid_scale (-1 = use grid_scale), set by a tuner
  int stage_scale[MHC_NUM_STAGES] = {-1, -1, -1, -1, -1, -1, -1};
  int cur_stage = -1;  // phase being launched (StageTimer scope)
  // layout of the y / z sweeps of classical-limiter cases, set by a caller
  // or the tuner (mhc_*_set_sweep_layout): 0 = by mesh size (the line-chunk
  // thresholds), 1 = warp per line, 2 = shared-memory tile, 3 = line chunks
  int cell_layout = 0, node_layout = 0;
  // kernels this engine put on the GPU (graph replays count their nodes)
  long long launches = 0;
  long long graph_launches = 0;  // kernel nodes of the captured graph
  // page-locked staging of the launch lists (case descriptors, then the
  // int arena) and the event after their last upload, so that a rebuild
  // does not wait for the work in flight
  char* h_stage = nullptr;
  size_t stage_cap = 0;
  cudaEvent_t stage_ev = nullptr;
  // status gather of every case (one kernel + one copy)
  Scalars* d_gather = nullptr;
  Scalars* h_gather = nullptr;   // pinned
  int gather_cap = 0;
};


struct StageTimer {
  Engine* e;
  int stage;
  StageTimer(Engine* e_, int s) : e(e_), stage(s) {
    e->cur_stage = s;
    if (e->timing) cudaEventRecord(e->ev[0], e->stream);
  }
  ~StageTimer() {
    e->cur_stage = -1;
    if (!e->timing) return;
    cudaEventRecord(e->ev[1], e->stream);
    cudaEventSynchronize(e->ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    e->stage_ms[stage] += ms;
    e->stage_launches[stage] += 1;
  }
};

// sweep instances of a case (the template argument LIM of kb_sweep_nodes /
// kb_sweep_cells)
inline int node_sweep_mode(const mhc_case_params& P) {
  if (P.ordre_projection == 1) return LIM_ORDER1;
  return P.projection_limiteur_id >= MHC_MINMOD_G ? LIM_GEN : P.projection_limiteur_id;
}
inline int cell_sweep_mode(const mhc_case_params& P) {
  if (P.projection_pente_borne) return LIM_PB;
  return P.ordre_projection == 3 ? LIM_O3 : node_sweep_mode(P);
}

// Directions whose classical cell sweep runs one thread per line chunk
// (body_sweep_cells_cols): coalesced but with one line chunk per thread, it
// pays when the sweep has enough line chunks to fill the device many times
// over (large meshes); smaller meshes keep the warp-per-line layout.  The
// node sweep, with fewer registers per line, pays from a quarter of that.
// The thresholds (line chunks of the sweep) can be changed with the
// environment variables MHC_SWEEP_COLS_MIN_THREADS (cells) and
// MHC_SWEEP_NODE_COLS_MIN_THREADS (nodes; default: the cell threshold / 4),
// read when the launch lists are built (0: every y / z sweep in this layout).
inline long long cols_min_threads() {
  const char* s = getenv("MHC_SWEEP_COLS_MIN_THREADS");
  if (s && *s) return atoll(s);
  return 1LL << 18;
}
inline long long node_cols_min_threads() {
  const char* s = getenv("MHC_SWEEP_NODE_COLS_MIN_THREADS");
  if (s && *s) return atoll(s);
  return cols_min_threads() / 4;
}
inline int cols_mask(const mhc_case* h) {
  if (cell_sweep_mode(h->P) > LIM_ORDER1) return 0;
  const long long lim = cols_min_threads();
  int m = 0;
  for (int D = 1; D < h->DIM; ++D) {
    const int nd = D == 1 ? h->M.ncy : h->M.ncz, nb = D == 1 ? h->M.ncz : h->M.ncy;
    if ((long long)h->M.ncx * nb * col_chunks(nd) >= lim) m |= 1 << D;
  }
  return m;
}
inline int node_cols_mask(const mhc_case* h) {
  if (node_sweep_mode(h->P) > LIM_ORDER1) return 0;
  const long long lim = node_cols_min_threads();
  int m = 0;
  for (int D = 1; D < h->DIM; ++D) {
    const int nd = D == 1 ? h->M.nny : h->M.nnz, nb = D == 1 ? h->M.nnz : h->M.nny;
    if ((long long)h->M.nnx * nb * col_chunks(nd) >= lim) m |= 1 << D;
  }
  return m;
}

// Directions whose classical cell sweep goes through a shared-memory tile
// (body_sweep_cells_tile: coalesced loads and stores, the warp-per-line
// arithmetic): every y / z sweep that does not take the line-chunk layout.
// MHC_SWEEP_TILE=0 in the environment keeps the warp-per-line layout.
inline int tile_mask(const mhc_case* h) {
  if (cell_sweep_mode(h->P) > LIM_ORDER1) return 0;
  const char* s = getenv("MHC_SWEEP_TILE");
  if (s && *s == '0') return 0;
  int m = 0;
  for (int D = 1; D < h->DIM; ++D) m |= 1 << D;
  return m & ~cols_mask(h);
}

// the same for the node sweeps (MHC_SWEEP_TILE=0 also keeps their
// warp-per-line layout)
inline int node_tile_mask(const mhc_case* h) {
  if (node_sweep_mode(h->P) > LIM_ORDER1) return 0;
  const char* s = getenv("MHC_SWEEP_TILE");
  if (s && *s == '0') return 0;
  int m = 0;
  for (int D = 1; D < h->DIM; ++D) m |= 1 << D;
  return m & ~node_cols_mask(h);
}

inline int group_node_phase(int LIM, int NCOLS, int NTILE, int D) {
  if ((NCOLS >> D) & 1) return node_sweep_phase(LIM_COLS + LIM, D);
  if ((NTILE >> D) & 1) return PH_SWNT0 + D;
  return node_sweep_phase(LIM, D);
}

// the (line-chunk, tile) direction masks of a case's cell or node sweeps
// under an engine's layout choice
inline void sweep_masks(const mhc_case* h, int layout, bool nodes, int& cols, int& tile) {
  if (!nodes && h->P.env[0].elasto_model && h->P.with_projection) {
    // the seven elasto variables ride through the warp-per-line cell sweeps only
    cols = tile = 0;
    return;
  }
  cols = nodes ? node_cols_mask(h) : cols_mask(h);
  tile = nodes ? node_tile_mask(h) : tile_mask(h);
  const int mode = nodes ? node_sweep_mode(h->P) : cell_sweep_mode(h->P);
  if (layout == 0 || mode > LIM_ORDER1) return;
  int all = 0;
  for (int D = 1; D < h->DIM; ++D) all |= 1 << D;
  cols = layout == 3 ? all : 0;
  tile = layout == 2 ? all : 0;
}

// phase of the cell sweep of a group along D
inline int group_cell_phase(int CLIM, int COLS, int TILE, int D) {
  if ((COLS >> D) & 1) return cell_sweep_phase(LIM_COLS + CLIM, D);
  if ((TILE >> D) & 1) return PH_SWCT0 + D;
  return cell_sweep_phase(CLIM, D);
}

// directions the remap does not sweep: one cell thick, or not the axis of a
// per-axis Euler scheme (RemapADIService.cc:26-32)
inline int skip_mask(const mhc_case* h) {
  int m = 0;
  if (h->M.ncx == 1) m |= 1;
  if (h->M.ncy == 1) m |= 2;
  if (h->DIM == 3 && h->M.ncz == 1) m |= 4;
  const int s = h->P.is_euler_scheme;
  if (s >= MHC_EULER_X && s <= MHC_EULER_Z) m |= 7 & ~(1 << (s - MHC_EULER_X));
  return m;
}

// persistent grid for a kernel: resident blocks on the device (cached)
template <class K>
inline int resident_blocks(Engine* e, K kernel, int threads, size_t smem) {
  static std::map<const void*, int> cache;
  auto it = cache.find((const void*)kernel);
  if (it != cache.end()) return it->second * e->nsm;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  cache[(const void*)kernel] = per_sm;
  return per_sm * e->nsm;
}

template <class K, class... Args>
inline void plaunch(Engine* e, K kernel, int threads, size_t smem, const DevList& L, Args... args) {
  if (L.total <= 0) return;
  const int sc = (e->cur_stage >= 0 && e->stage_scale[e->cur_stage] >= 0) ? e->stage_scale[e->cur_stage] : e->grid_scale;
  int grid = sc == 0 ? L.total : std::min(L.total, resident_blocks(e, kernel, threads, smem) * sc);
  const PhaseList pl{e->d_ints + L.off_cases, e->d_ints + L.off_start, L.n, L.total};
  kernel<<<grid, threads, smem, e->stream>>>(e->d_desc, pl, args...);
  ++e->launches;
}


#define DISPATCH_GROUP(g, CALL)                                   \
  do {                                                            \
    if ((g).DIM == 2) {                                           \
      constexpr int DIM_ = 2;                                     \
      switch ((g).NE) {                                           \
        case 1: { constexpr int NE_ = 1; CALL; } break;           \
        case 2: { constexpr int NE_ = 2; CALL; } break;           \
        case 3: { constexpr int NE_ = 3; CALL; } break;           \
        default: { constexpr int NE_ = 4; CALL; } break;          \
      }                                                           \
    } else {                                                      \
      constexpr int DIM_ = 3;                                     \
      switch ((g).NE) {                                           \
        case 1: { constexpr int NE_ = 1; CALL; } break;           \
        case 2: { constexpr int NE_ = 2; CALL; } break;           \
        case 3: { constexpr int NE_ = 3; CALL; } break;           \
        default: { constexpr int NE_ = 4; CALL; } break;          \
      }                                                           \
    }                                                             \
  } while (0)


// one performed sweep (cells, then nodes) of direction D as the k-th of the
// cycle, for the members of a group (mhc_sweeps.cu)
void sweep_step_any(Engine* e, Group& g, int D, int k);

// engine operations defined in mhc_capi.cu and shared with the other C ABI
// translation units (mhc_services.cu)
namespace mhc {
int engine_rebuild_shared(Engine* e);
int solo_engine_shared(mhc_case* h);
void launch_remap_sweeps_shared(Engine* e);
void launch_remap_variables_shared(Engine* e);
int fetch_shared(cudaStream_t s, const void* dev, void* host, size_t bytes);
}  // namespace mhc
