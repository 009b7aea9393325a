// Serving loop: continuous batching of wide-Fibonacci proofs on one device.
//
// Requests are admitted in arrival order as a slot (a prover with its own stream
// and host thread) is free and the in-flight device workspace stays within the
// memory budget; each admitted proof then runs concurrently with the others, so
// their kernels overlap on the GPU. Per-request limits follow the reference's
// resource profiles (src/prover/native/resource_admission.zig:5-19,
// 16 accounted bytes per committed cell).
#pragma once
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "prover.hpp"

namespace sb {

struct ResourceLimits {
  uint64_t max_committed_cells, max_accounted_bytes;
};
// Profiles 0 standard, 1 large, 2 extreme (resource_admission.zig:14-19).
bool profile_limits(uint32_t profile, ResourceLimits* out);
constexpr uint64_t ACCOUNTED_BYTES_PER_CELL = 16;
constexpr uint32_t ADMISSION_MAX_LOG_ROWS = 22;

struct RequestStats {
  uint64_t accounted_bytes = 0, workspace_bytes = 0;
  double queued_ms = 0, run_ms = 0;
  uint32_t slot = 0;
  StageTimes stages;  // device time per stage
};

// Server flags.
constexpr uint32_t SERVER_PERSISTENT_WORKSPACES = 1;  // slots keep their workspace between proofs
constexpr uint32_t SERVER_VERIFY = 2;                 // verify every proof on the slot's host thread

struct ServerSnapshot {
  uint64_t submitted = 0, completed = 0, failed = 0, rejected = 0;
  uint64_t peak_in_flight = 0, peak_workspace_bytes = 0, budget_bytes = 0;
};

class Server {
 public:
  Server(Context* ctx, uint32_t slots, uint64_t budget, uint32_t profile, uint32_t flags);
  ~Server();
  int32_t start();
  int32_t submit(const ProveRequest& r, uint64_t* ticket, std::string* err);
  int32_t submit_xor(const XorRequest& r, uint64_t* ticket, std::string* err);
  // Sizes every slot for the largest shapes it will serve before traffic arrives (the reference's
  // warmup / initializeRuntime hooks): persistent workspaces grow to the largest wide-Fibonacci
  // shape, and the stream-ordered pool is pre-grown for transient workspaces and XOR proofs. Call
  // it while the server is idle.
  int32_t warmup(uint32_t max_log_n_rows, uint32_t max_sequence_len, uint32_t log_blowup, uint32_t max_xor_log_n,
                 std::string* err);
  // Time limit of every request submitted from now on, from its submission (0: none). A request
  // still queued at its deadline ends with E_TIMEOUT without running; a running proof checks the
  // deadline between stages and proof-of-work rounds and ends with E_TIMEOUT.
  void set_request_timeout(uint32_t ms);
  // Blocks until the request is done. E_BUFFER_TOO_SMALL keeps the result for another call.
  int32_t wait(uint64_t ticket, uint8_t* out, size_t cap, size_t* len, RequestStats* stats, std::string* err);
  ServerSnapshot snapshot();

 private:
  struct Entry {
    bool is_xor = false;
    ProveRequest req;
    XorRequest xreq;
    uint64_t ticket = 0;
    size_t workspace = 0;
    RequestStats stats;
    std::chrono::steady_clock::time_point t_submit, t_start;
    Deadline deadline;
    bool done = false;
    int32_t status = 0;
    std::string proof, error;
  };
  void worker(uint32_t slot);
  int32_t enqueue(Entry* e, uint64_t cells, size_t workspace, uint64_t* ticket, std::string* err);
  // Workspace bytes the request would add to in_use_ on `slot` (caller holds mu_).
  uint64_t extra_on(uint32_t slot, const Entry* e) const;
  // The idle slot on which the request adds the least (lowest index on ties), or -1.
  int64_t best_idle_slot(const Entry* e) const;
  // Marks a request done with `status` and wakes its waiter (caller holds mu_).
  void finish(Entry* e, int32_t status, std::string&& proof, std::string&& error);

  Context* ctx_;
  uint32_t n_slots_;
  uint64_t budget_;
  uint32_t flags_;
  ResourceLimits limits_;
  std::vector<uint64_t> held_;  // persistent mode: workspace bytes each slot holds
  std::vector<uint8_t> idle_;   // slots waiting for a request
  uint32_t timeout_ms_ = 0;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Entry*> queue_;
  std::unordered_map<uint64_t, Entry*> table_;
  uint64_t next_ticket_ = 1, in_use_ = 0, in_flight_ = 0;
  bool stopping_ = false;
  ServerSnapshot snap_;
  std::vector<WideFibProver*> provers_;
  std::vector<LogupXorProver*> xor_provers_;  // created on a slot's first XOR request
  std::vector<std::thread> threads_;
};

}  // namespace sb
