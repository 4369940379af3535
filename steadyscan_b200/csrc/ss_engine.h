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
  int prepare(int n, const ss_inputs* in, ss_outputs* out, void* external, size_t external_bytes);
  // Runs every group from its initial knots to its stop criterion.
  int run();
  // Copies the results into the ss_outputs given to prepare().
  int collect();

  void set_timing(bool on);
  void stats(ss_batch_stats* st) const;
  size_t arena_bytes() const;
  int cycles() const;
  int rounds() const;
  int n_groups() const;
  const GroupCtl* host_ctl() const;
  void* stream() const;

 private:
  Impl* d;
};

}  // namespace ss
