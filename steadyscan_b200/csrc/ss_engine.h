// C++ view of the batched engine (used by the C ABI and the serving runtime).
#pragma once

#include <stddef.h>

#include <string>

#include "steadyscan_b200.h"

namespace ss {

struct GroupCtl;

int fail(int code, const std::string& msg);
const char* last_error();

class Batch {
 public:
  struct Impl;
  Batch();
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Validates the groups, lays out and fills device memory (one arena; or the caller's
  // `external` buffer of `external_bytes` when given). Outputs are remembered for collect().
  // sessions[i], when given and not null, is a prepared batch whose first group's template and
  // geometry buffers group i uses instead of its own (they must outlive this batch). With
  // measure_only the call stops after computing arena_bytes(): no device work. borrow_stream (a
  // cudaStream_t) runs the batch on the caller's stream without blocking on it.
  int prepare(int n, const ss_inputs* in, ss_outputs* out, void* external, size_t external_bytes,
              const Batch* const* sessions = nullptr, bool measure_only = false, void* borrow_stream = nullptr);
  // Before prepare(): upload the frames of host-resident groups on a second stream while earlier
  // groups already run (each group joins the run when its frames have arrived). For batches run
  // once, such as ss_align_groups; results are those of an unstreamed run.
  void set_stream_frames(bool on);
  // Runs every group from its initial knots to its stop criterion.
  int run();
  // The same run one cycle at a time without blocking: start() resets every group to its initial
  // knots, step() launches one cycle on the batch stream, poll() returns 0 while that cycle runs,
  // 1 when it has finished and another is needed, 2 when every group has stopped.
  int start();
  int step();
  int poll();
  // Resets every group to its initial state (the start of a server slot; waits on an own stream).
  int reset();
  // Copies the results into the ss_outputs given to prepare().
  int collect();

  void set_timing(bool on);
  void set_graph(bool on);
  void stats(ss_batch_stats* st) const;
  size_t arena_bytes() const;
  int cycles() const;
  int rounds() const;
  int n_groups() const;
  const GroupCtl* host_ctl() const;
  void* stream() const;

 private:
  friend class Server;
  friend int estimate_displacements(const ss_recording* rec, ss_recording_outputs* out);
  Impl* d;
};

// The recording-level estimate of ss_estimate_displacements: every set of the recording as one
// group of one batch, then the caller's post-estimate rules on the device.
int estimate_displacements(const ss_recording* rec, ss_recording_outputs* out);
// Set split of ss_recording_sets (0-based first frame and frame count per set, overlap included).
// ss_prepare_frames: prefilter, crop and block-reorder raw frames on the device (ss_frontend.cuh).
int prepare_frames(const ss_prep_frames* p);

// ss_reconstruct_frames: invert_bilinear_sampling of one set's frames (ss_reconstruct.cuh).
int reconstruct_frames(const ss_reconstruct* r);

int recording_sets(int n_frames, int frames_per_set, int min_frames_per_set, int* first, int* count, int max_sets,
                   int* n_sets);

// Continuous batching: a table of `capacity` group slots on one stream. admit() prepares a group
// (in the caller's arena, with a session's resident buffers) into a free slot; step() applies the
// admissions and retirements since the last cycle and launches one cycle of every active group;
// poll() returns 0 while the cycle runs, else 1 after collecting the outputs of the groups that
// stopped (their slots listed in `done`, their arenas free again).
class Server {
 public:
  struct Impl;
  Server();
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  int create(int capacity, int device);
  int admit(const ss_inputs* in, ss_outputs* out, const Batch* session, void* arena, size_t arena_bytes,
            int* slot);
  int step();
  int poll(int* done, int max_done, int* n_done);
  int active() const;

 private:
  Impl* d;
};

}  // namespace ss
