// fsl_group.cuh -- host-side state shared by the single-instance, batched
// and serving entry points.
//
//   Slot  : the device buffers of one instance (one allocation, carved up),
//           sized for a particle capacity that may exceed its current count.
//   Group : instances of one size class (grid extents, neighbour-grid
//           extents, kernel width) that every launch of a stage serves
//           together; they share one FFT plan and one device table of Rep.
//   Exec  : the groups stepped together, each on its own stream, with the
//           whole step captured in one CUDA graph.
#pragma once

#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/fluamsl.h"
#include "fsl_internal.cuh"

namespace fsl {

// printf-style message for fsl_last_error(); returns code
int errorf(int code, const char* fmt, ...);
const char* last_error();
// FSL_E_NOMEM for allocation failures, FSL_E_CUDA otherwise
int cuda_fail(cudaError_t e, const char* what);

#define FSL_TRY(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return ::fsl::cuda_fail(e_, #call); \
  } while (0)

// Validates c (np particles) and derives the kernel parameters: spacings
// (src/createCellsStokesLimitGPU.cu:58-91), neighbour grid
// (src/createBoundariesRK2GPU.cu:134-141), noise prefactors.
int make_params(const fsl_config& c, int64_t np, Params& P);

// Size-class key: instances that can share every launch of a step.
struct ClassKey {
  int mx, my, mz, mnx, mny, mnz, kernel, scheme, prec, observe;
  bool operator<(const ClassKey& o) const;
  bool operator==(const ClassKey& o) const;
};
ClassKey class_of(const Params& P);

// Device bytes one slot of this class takes with room for np_cap particles.
size_t slot_bytes(const Params& P, int np_cap);

struct Slot {
  Rep r{};                 // parameters and device pointers (host copy)
  int np_cap = 0;          // particle capacity of the buffers
  void* arena = nullptr;   // every fixed-size buffer
  void* bonds = nullptr;   // bond tables (fsl_load_bonds)
  size_t bytes = 0;
};

// Allocates the slot's buffers for class P with room for np_cap particles
// and zeroes them on st (the spread field must start cleared).  The slot
// stays inactive until slot_reset.
int slot_alloc(Slot& s, const Params& P, int np_cap, cudaStream_t st);
void slot_free(Slot& s);
// Puts a new instance (parameters P, positions q on the host) into an
// allocated slot of its class: positions, LJ table, cleared forces, error
// word, step counter and bonds.  Enqueued on st.
int slot_reset(Slot& s, const Params& P, const double* q, const fsl_config& c, cudaStream_t st);
// slot_force_lists: the pair list is rebuilt at the next force evaluation
// (a new instance).  slot_mark_moved: positions changed from the host, the
// list is rebuilt if a particle left its skin.  slot_request_lists: the next
// launch_pair_lists builds the cell list whatever the path (the component
// entry points).
int slot_force_lists(Slot& s, cudaStream_t st);
// error word cleared, cell-list counters and barrier reset, lists rebuilt at
// the next force evaluation
int slot_clear_errors(Slot& s, cudaStream_t st);
int slot_mark_moved(Slot& s, cudaStream_t st);
int slot_request_lists(Slot& s, cudaStream_t st);
// q0 := q, observables accumulators cleared (enqueued on st).
int slot_reset_observables(Slot& s, cudaStream_t st);
// The accumulators of the slot (synchronises st).
int slot_read_observables(const Slot& s, cudaStream_t st, fsl_observables* out);
// Bond tables in the reference's CSR (src/initializeBondedForces.cpp:31-150).
// directed: entry b acts on particle bi[b] only (the old bond-file format)
int slot_bonds(Slot& s, int64_t nbonds, const int32_t* bi, const int32_t* bj, const double* k,
               const double* r0, int64_t nfixed, const int32_t* fi, const double* fk,
               const double* fr0, const double* fxyz, cudaStream_t st, bool directed = false);

struct Group {
  ClassKey key{};
  Params P0{};                  // parameters the plan was made for
  FftPlan* fft = nullptr;
  std::vector<Slot*> slots;     // not owned
  Rep* d_reps = nullptr;        // device table, capacity d_cap
  int* d_boff = nullptr;        // device block offsets, [NKIND][d_cap + 1]
  int d_cap = 0;
  std::vector<Rep> h_reps;      // host copy of the device table
  std::vector<int> h_boff;
  Batch B{};
  bool dirty = true;            // host table changed since the last upload
  bool allow_one = true;        // a lone instance may travel by value (its
                                // changes then need a new graph capture)
  cudaStream_t stream = nullptr;
  // the noise of a step runs beside the cell list and forces on this stream
  // (fork and join events); profiled steps keep everything on `stream`
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;  // noise parts 0, 1
  // the spread field is cleared on `side` after each W build (ev_w) and
  // waited for before the next spread or the end of the step (ev_c)
  cudaEvent_t ev_w[2] = {}, ev_c[2] = {};
  Prof prof;
  std::map<std::string, std::pair<int64_t, double>> stage_acc;
  int launches = 0;             // kernels of this group in one step
  // the list build of a batch of small instances, timed at the class's first
  // uncaptured step (us per build: separate kernels, block per instance)
  bool lists_tuned = false;
  float lists_us[2] = {};
  // an input/output step of a single instance (fsl_step_io): the positions
  // come from pinned host memory io_in at the start of the step and go to
  // io_out at its end, both inside the step's graph (null: a plain step)
  const double* io_in = nullptr;
  double* io_out = nullptr;
  size_t io_bytes = 0;
  // an input/output step of a batch: the step's main branch waits for this
  // event (the inputs copied in and scattered on the Exec's io stream)
  // after forking its noise
  cudaEvent_t io_wait = nullptr;
  const char* fail_stage = nullptr;  // first stage whose launch failed
};

int group_init(Group& g, const Params& P0);
void group_destroy(Group& g);  // plan, table, events; not the slots
// Rebuilds the Rep table from the slots (and their active flags) and
// uploads it on the group's stream when it changed.
int group_upload(Group& g);
void group_enqueue_step(Group& g);  // one midpoint step of every active slot
int group_prof_collect(Group& g);
// The class's tuner picks and timings (fsl_batch_get_class_tuning)
void group_tuning(const Group& g, fsl_class_tuning* out);

struct Exec {
  int device = 0;
  cudaStream_t stream = nullptr;      // the caller-visible stream
  std::vector<Group*> groups;         // not owned
  std::vector<cudaStream_t> side;     // one per group beyond the first
  std::vector<cudaEvent_t> ev;        // fork + one join per group
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<long long> shape;       // what the graph was captured for
  uint64_t steps = 0;
  int launches_per_step = 0;
  int64_t captures = 0;               // graphs captured so far
  // an input/output step of a batch (fsl_batch_step_io): io_in enqueues the
  // copy in and scatter on io_stream, forked at the start of the step so
  // that the groups' noise runs beside it; io_out enqueues the gather and
  // copy out on the main stream after the join.  io_key (the host buffers)
  // is part of the captured graph's shape.  Unset: a plain step.
  std::function<void(cudaStream_t)> io_in, io_out;
  const void* io_key[2] = {};
  cudaStream_t io_stream = nullptr;
  cudaEvent_t io_fork = nullptr, io_ev = nullptr;
};

// Whether p is page-locked host memory (a copy from or to it can be a node
// of a CUDA graph).
bool pinned_host(const void* p);

int exec_init(Exec& e, int device);
void exec_destroy(Exec& e);
void exec_drop_graph(Exec& e);
// nsteps midpoint steps of every group; the first step of an Exec runs
// eagerly, later ones replay the captured graph.
int exec_step(Exec& e, int64_t nsteps);

// src/initForcesNonBonded.cu:21-53 (float accumulation, float sqrt,
// sigma = 2 dx, epsilon = kT, first and last entries zero).
void build_ljtable(const Params& P, double temperature, double cutoff, std::vector<float>& t);

}  // namespace fsl
