// Host orchestration of one wide-Fibonacci proof on one device stream.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace sb {

struct PcsConfig {
  uint32_t pow_bits = 10;
  uint32_t log_blowup_factor = 1;
  uint32_t log_last_layer_degree_bound = 0;
  uint32_t n_queries = 3;
};

constexpr int TRACE_FIRST_COLUMNS = 2;

// Largest accepted proof-of-work difficulty. The grind tests 2^pow_bits nonces on average
// (about 40 s on one B200 at 40 bits) and holds its stream meanwhile; the reference accepts any
// u32, so the cap is this backend's own.
constexpr uint32_t MAX_POW_BITS = 40;

using Clock = std::chrono::steady_clock;
// Optional time limit of one proof, checked between stages and between proof-of-work rounds; a
// proof past it ends with E_TIMEOUT and leaves no work in flight.
struct Deadline {
  Clock::time_point at = Clock::time_point::max();
  bool set() const { return at != Clock::time_point::max(); }
  bool passed() const { return set() && Clock::now() >= at; }
};

struct ProveRequest {
  uint32_t log_n_rows = 0, sequence_len = 0;
  PcsConfig config;
  const uint32_t* trace_host = nullptr;    // column-major, bit-reversed circle order
  const uint32_t* trace_device = nullptr;  // same layout, device memory
  // Without a trace pointer: 0 (1,row), 1 seeded. TRACE_FIRST_COLUMNS: the pointer holds only
  // col0 and col1 and the device derives the rest of the trace.
  int trace_kind = 0;
  uint64_t trace_seed = 0;
  bool has_channel_seed = false;
  uint64_t channel_seed = 0;
};

// Stage timings of one proof (milliseconds of device time between events), the host time spent
// after the last device stage (proof encoding and the OODS self-check), and the host time between
// a stream synchronization of the transcript and the next device work (the device may idle then
// when the proof runs alone: total - host_gaps bounds its device work).
struct StageTimes {
  float upload = 0, trace = 0, main_commit = 0, composition = 0, composition_commit = 0, oods = 0,
        quotients = 0, fri = 0, pow = 0, decommit = 0, total = 0, host_encode = 0, host_gaps = 0;
};

// Status codes shared with the C ABI.
enum : int32_t {
  OK = 0,
  E_INVALID = -1,
  E_OOM = -2,
  E_CUDA = -3,
  E_TIMEOUT = -4,
  E_CONSTRAINTS = -5,
  E_BUFFER_TOO_SMALL = -6,
  E_FALLBACK = -7,
  E_NO_DEVICE = -8,
  E_DIVISION_BY_ZERO = -9,
  E_REJECTED = -10,
};

struct Context;

// Per-proof device workspace, reused across proofs of the same shape.
class WideFibProver {
 public:
  WideFibProver(Context* ctx, cudaStream_t stream);
  ~WideFibProver();
  int32_t prove(const ProveRequest& req, std::string& proof_json, StageTimes* times);
  const std::string& error() const { return err_; }
  // Device workspace one proof of this shape uses (bytes).
  static size_t workspace_bytes(uint32_t log_n, uint32_t W, uint32_t B);
  // Transient mode: the workspace is taken from the device's stream-ordered pool at the start of
  // each proof and returned at its end, so the device memory a prover holds between proofs is
  // only its pinned staging. Used by the serving loop, which admits by in-flight workspace bytes.
  void set_transient(bool on);
  // Grows the persistent workspace to a shape ahead of use (no-op in transient mode); returns the
  // bytes the prover holds afterwards in *held.
  int32_t reserve(uint32_t log_n, uint32_t W, uint32_t B, size_t* held);
  // Frees the persistent workspace (the serving loop gives back an idle slot's memory).
  void drop_workspace();
  // Device workspace held between proofs (0 in transient mode).
  size_t held_bytes() const { return transient_ ? 0 : arena_size_; }
  // Time limit of the next proofs (a default Deadline: none).
  void set_deadline(Deadline d) { deadline_ = d; }

 private:
  int32_t ensure_workspace(uint32_t log_n, uint32_t W, uint32_t B);
  void release();
  int32_t fail(int32_t code, const std::string& msg) { err_ = msg; return code; }

  Context* ctx_;
  cudaStream_t stream_;
  // High-priority stream for the latency-bound chain after the composition commit (OODS,
  // quotients, FRI layers with their root readbacks, decommitment): when several proofs
  // share the device, its kernels are scheduled ahead of other proofs' bulk work.
  cudaStream_t fast_ = nullptr;
  // The proof-of-work grind's stream, at the least priority (StreamPriorities).
  cudaStream_t pow_ = nullptr;
  std::string err_;
  // workspace
  uint8_t* arena_ = nullptr;
  size_t arena_size_ = 0;
  uint32_t ws_log_n_ = 0, ws_W_ = 0, ws_B_ = 0;
  bool transient_ = false;
  uint8_t* pinned_ = nullptr;
  size_t pinned_size_ = 0;
  cudaEvent_t ev_[12];
  Deadline deadline_;
};

// LogUp XOR-lookup AIR request (xor_prover.cu): 2^log_n lookups of seeded w-bit pairs
// (w = log_table / 2) into the 2^log_table-row XOR table.
struct XorRequest {
  uint32_t log_n = 0, log_table = 16;
  uint64_t seed = 0;
  PcsConfig config;
  bool has_channel_seed = false;
  uint64_t channel_seed = 0;
};

// Prover of the LogUp XOR-lookup AIR; its workspace comes from the stream-ordered pool per proof.
// Stream priorities of a proof's work when several proofs share the device: the latency-bound
// chain after the composition commit at the greatest priority, the bulk stages (trace, FFTs,
// commitments, composition) one level above the least, and the proof-of-work grind at the least,
// so that the grind, whose launches fill every multiprocessor they are given, takes what the other
// proofs' stages leave rather than holding them behind its waves.
struct StreamPriorities {
  int least = 0, greatest = 0, bulk = 0;
};
StreamPriorities stream_priorities();

class LogupXorProver {
 public:
  explicit LogupXorProver(Context* ctx);
  ~LogupXorProver();
  int32_t prove(const XorRequest& req, std::string& proof_json);
  // Allocates the pinned staging buffer now rather than at the first proof (E_OOM on failure).
  int32_t reserve_staging();
  const std::string& error() const { return err_; }
  // Device workspace of one proof of this shape (bytes); 0 for an impossible shape.
  static size_t workspace_bytes(uint32_t log_n, uint32_t log_table, uint32_t log_blowup, uint32_t log_last_layer);
  void set_deadline(Deadline d) { deadline_ = d; }

 private:
  static constexpr size_t PINNED_BYTES = (8 << 20) + (1 << 20);
  int32_t fail(int32_t code, const std::string& msg) { err_ = msg; return code; }
  Context* ctx_;
  cudaStream_t stream_ = nullptr, fast_ = nullptr, pow_ = nullptr;
  uint8_t* pinned_ = nullptr;
  std::string err_;
  Deadline deadline_;
};

struct Context {
  int device = 0;
  int sm_count = 0;
  DeviceTables tables;
  std::mutex mu;
  std::vector<WideFibProver*> pool;  // idle provers
  std::vector<LogupXorProver*> xor_pool;
  cudaStream_t stream = nullptr;
  uint32_t* small = nullptr;  // 256 bytes of device scratch for single-value results (PoW nonce)
  std::mutex h2d_mu;          // serialises host-to-device trace uploads of concurrent proofs
  std::mutex small_mu;
  ~Context();
  int32_t init(int device, uint32_t tower_log);
  WideFibProver* acquire();
  void release(WideFibProver* p);
  LogupXorProver* acquire_xor();
  void release_xor(LogupXorProver* p);
};

const char* status_string(int32_t code);

}  // namespace sb
