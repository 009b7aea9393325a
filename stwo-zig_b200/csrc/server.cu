// Serving loop (continuous batching) over WideFibProver slots; see server.hpp.
#include "server.hpp"

#include "verifier.hpp"

#include <algorithm>
#include <cstring>

namespace sb {

bool profile_limits(uint32_t profile, ResourceLimits* out) {
  // STANDARD/LARGE/EXTREME_MAX_COMMITTED_CELLS and _ACCOUNTED_BYTES, resource_admission.zig:14-19.
  switch (profile) {
    case 0: *out = {33554432ull, 536870912ull}; return true;
    case 1: *out = {134217728ull, 2147483648ull}; return true;
    case 2: *out = {419430400ull, 6710886400ull}; return true;
    default: return false;
  }
}

Server::Server(Context* ctx, uint32_t slots, uint64_t budget, uint32_t profile, uint32_t flags)
    : ctx_(ctx), n_slots_(slots), budget_(budget), flags_(flags), held_(slots, 0), idle_(slots, 0) {
  if (!profile_limits(profile, &limits_)) limits_ = {0, 0};
  snap_.budget_bytes = budget;
}

int32_t Server::start() {
  if (limits_.max_committed_cells == 0) return E_INVALID;
  cudaSetDevice(ctx_->device);
  for (uint32_t i = 0; i < n_slots_; ++i) {
    cudaStream_t s;
    if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, stream_priorities().bulk) != cudaSuccess) return E_CUDA;
    WideFibProver* p = new WideFibProver(ctx_, s);
    p->set_transient(!(flags_ & SERVER_PERSISTENT_WORKSPACES));
    provers_.push_back(p);
  }
  for (uint32_t i = 0; i < n_slots_; ++i) xor_provers_.push_back(new LogupXorProver(ctx_));
  for (uint32_t i = 0; i < n_slots_; ++i) threads_.emplace_back(&Server::worker, this, i);
  return OK;
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> g(mu_);
    stopping_ = true;
  }
  cv_work_.notify_all();
  for (auto& t : threads_) t.join();
  for (auto* p : provers_) delete p;
  for (auto* p : xor_provers_) delete p;
  for (auto& kv : table_) delete kv.second;
}

int32_t Server::enqueue(Entry* e, uint64_t cells, size_t ws, uint64_t* ticket, std::string* err) {
  const uint64_t accounted = cells * ACCOUNTED_BYTES_PER_CELL;
  std::lock_guard<std::mutex> g(mu_);
  if (cells > limits_.max_committed_cells || accounted > limits_.max_accounted_bytes) {
    ++snap_.rejected;
    delete e;
    *err = "committed cell budget of the resource profile exceeded";
    return E_REJECTED;
  }
  if (ws == 0 || ws > budget_) {
    ++snap_.rejected;
    delete e;
    *err = "proof workspace exceeds the server's device memory budget";
    return E_REJECTED;
  }
  e->ticket = next_ticket_++;
  e->workspace = ws;
  e->stats.accounted_bytes = accounted;
  e->stats.workspace_bytes = ws;
  e->t_submit = std::chrono::steady_clock::now();
  if (timeout_ms_) e->deadline.at = e->t_submit + std::chrono::milliseconds(timeout_ms_);
  table_[e->ticket] = e;
  queue_.push_back(e);
  ++snap_.submitted;
  *ticket = e->ticket;
  // Every idle slot looks at the new head: the one it fits on takes it.
  cv_work_.notify_all();
  return OK;
}

void Server::set_request_timeout(uint32_t ms) {
  std::lock_guard<std::mutex> g(mu_);
  timeout_ms_ = ms;
}

uint64_t Server::extra_on(uint32_t slot, const Entry* e) const {
  // Transient workspaces count while their proof runs; a persistent one counts for as long as its
  // slot holds it (a slot grows to the largest proof it has run). XOR-lookup proofs always take
  // their workspace from the pool for the proof's duration.
  if (!(flags_ & SERVER_PERSISTENT_WORKSPACES) || e->is_xor) return e->workspace;
  return e->workspace > held_[slot] ? e->workspace - held_[slot] : 0;
}

int64_t Server::best_idle_slot(const Entry* e) const {
  int64_t best = -1;
  uint64_t best_extra = 0;
  for (uint32_t i = 0; i < n_slots_; ++i) {
    if (!idle_[i]) continue;
    uint64_t x = extra_on(i, e);
    if (best < 0 || x < best_extra) { best = i; best_extra = x; }
  }
  return best;
}

void Server::finish(Entry* e, int32_t status, std::string&& proof, std::string&& error) {
  e->status = status;
  if (status == OK) {
    e->proof = std::move(proof);
    ++snap_.completed;
  } else {
    e->error = std::move(error);
    ++snap_.failed;
  }
  e->done = true;
  cv_done_.notify_all();
}

int32_t Server::submit(const ProveRequest& r, uint64_t* ticket, std::string* err) {
  // admit(profile, log_rows, columns), resource_admission.zig: rows in [1, 22], cells and
  // accounted bytes within the profile.
  if (r.log_n_rows < 1 || r.log_n_rows > ADMISSION_MAX_LOG_ROWS || r.sequence_len < 2 || r.sequence_len > 1000 ||
      r.config.log_blowup_factor < 1 || r.config.log_blowup_factor > 4) {
    *err = "invalid proof shape";
    return E_INVALID;
  }
  Entry* e = new Entry();
  e->req = r;
  return enqueue(e, (uint64_t)r.sequence_len << r.log_n_rows,
                 WideFibProver::workspace_bytes(r.log_n_rows, r.sequence_len, r.config.log_blowup_factor), ticket,
                 err);
}

int32_t Server::submit_xor(const XorRequest& r, uint64_t* ticket, std::string* err) {
  if (r.log_n < 1 || r.log_n > ADMISSION_MAX_LOG_ROWS || (r.log_table != 8 && r.log_table != 16) ||
      r.config.log_blowup_factor < 1 || r.config.log_blowup_factor > 4) {
    *err = "invalid proof shape";
    return E_INVALID;
  }
  Entry* e = new Entry();
  e->is_xor = true;
  e->xreq = r;
  // Committed columns: 4 preprocessed, 4 main, 8 interaction, of 2^max(log_n, log_table) rows.
  const uint32_t L = std::max(r.log_n, r.log_table);
  return enqueue(e, 16ull << L,
                 LogupXorProver::workspace_bytes(r.log_n, r.log_table, r.config.log_blowup_factor,
                                                 r.config.log_last_layer_degree_bound),
                 ticket, err);
}

void Server::worker(uint32_t slot) {
  cudaSetDevice(ctx_->device);
  WideFibProver* prover = provers_[slot];
  const bool persistent = flags_ & SERVER_PERSISTENT_WORKSPACES;
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    // Admission, first in first admitted: the head runs on a free slot once its workspace fits the
    // budget. Every idle slot re-evaluates on each change (submit, admission, completion, release):
    // - the head fits here: take it;
    // - it fits on another idle slot (one that holds more workspace): leave it to that slot;
    // - it fits nowhere: an idle slot whose held workspace is not what the head would reuse gives it
    //   back, so the head fits once the proofs in flight finish (a workspace never exceeds the
    //   budget, which submit checks).
    idle_[slot] = 1;
    Entry* e = nullptr;
    for (;;) {
      if (queue_.empty()) {
        if (stopping_) {
          idle_[slot] = 0;
          return;
        }
        cv_work_.wait(lk);
        continue;
      }
      Entry* h = queue_.front();
      if (h->deadline.passed()) {
        queue_.pop_front();
        h->t_start = std::chrono::steady_clock::now();
        h->stats.queued_ms = std::chrono::duration<double, std::milli>(h->t_start - h->t_submit).count();
        finish(h, E_TIMEOUT, std::string(), std::string("request deadline passed before admission"));
        cv_work_.notify_all();
        continue;
      }
      if (in_use_ + extra_on(slot, h) <= budget_) {
        e = h;
        break;
      }
      const int64_t best = best_idle_slot(h);
      const bool fits_elsewhere = best >= 0 && best != (int64_t)slot && in_use_ + extra_on((uint32_t)best, h) <= budget_;
      if (!fits_elsewhere && persistent && held_[slot] > 0 && (best != (int64_t)slot || h->is_xor)) {
        // Give back this idle slot's workspace (cudaFree waits for the device; no proof of this slot
        // is in flight, and the others do not need the lock until they finish).
        prover->drop_workspace();
        in_use_ -= held_[slot];
        held_[slot] = 0;
        cv_work_.notify_all();
        continue;
      }
      cv_work_.wait(lk);
    }
    queue_.pop_front();
    idle_[slot] = 0;
    const uint64_t added = extra_on(slot, e);
    in_use_ += added;
    if (persistent && !e->is_xor) held_[slot] += added;
    ++in_flight_;
    snap_.peak_in_flight = std::max(snap_.peak_in_flight, in_flight_);
    snap_.peak_workspace_bytes = std::max<uint64_t>(snap_.peak_workspace_bytes, in_use_);
    e->t_start = std::chrono::steady_clock::now();
    e->stats.slot = slot;
    lk.unlock();
    // Another head may fit beside this one.
    cv_work_.notify_all();
    std::string proof, xerr;
    int32_t rc;
    if (e->is_xor) {
      xor_provers_[slot]->set_deadline(e->deadline);
      rc = xor_provers_[slot]->prove(e->xreq, proof);
      if (rc != OK) xerr = xor_provers_[slot]->error();
    } else {
      prover->set_deadline(e->deadline);
      rc = prover->prove(e->req, proof, &e->stats.stages);
      if (rc != OK) xerr = prover->error();
    }
    if (rc == OK && (flags_ & SERVER_VERIFY)) {
      // The device keeps serving the other slots meanwhile.
      std::string verr;
      int32_t vrc = e->is_xor ? verify_logup_xor_json(proof, e->xreq.log_n, e->xreq.log_table,
                                                      e->xreq.has_channel_seed, e->xreq.channel_seed, verr)
                              : verify_wide_fib_json(proof, e->req.log_n_rows, e->req.sequence_len,
                                                     e->req.has_channel_seed, e->req.channel_seed, verr);
      if (vrc != OK) {
        rc = vrc;
        xerr = "served proof failed verification: " + verr;
      }
    }
    auto t_end = std::chrono::steady_clock::now();
    lk.lock();
    if (!persistent || e->is_xor) {
      in_use_ -= e->workspace;
    } else {
      // The slot's accounting follows what its prover holds (a failed growth holds nothing).
      const uint64_t actual = prover->held_bytes();
      in_use_ = in_use_ - held_[slot] + actual;
      held_[slot] = actual;
    }
    --in_flight_;
    e->stats.queued_ms = std::chrono::duration<double, std::milli>(e->t_start - e->t_submit).count();
    e->stats.run_ms = std::chrono::duration<double, std::milli>(t_end - e->t_start).count();
    finish(e, rc, std::move(proof), std::move(xerr));
    cv_work_.notify_all();
  }
}

int32_t Server::wait(uint64_t ticket, uint8_t* out, size_t cap, size_t* len, RequestStats* stats, std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = table_.find(ticket);
  if (it == table_.end()) {
    *err = "unknown ticket";
    return E_INVALID;
  }
  Entry* e = it->second;
  cv_done_.wait(lk, [&] { return e->done; });
  if (stats) *stats = e->stats;
  if (e->status != OK) {
    *err = e->error;
    int32_t rc = e->status;
    table_.erase(it);
    delete e;
    return rc;
  }
  if (len) *len = e->proof.size();
  if (!out || cap < e->proof.size()) {
    *err = "proof buffer too small";
    return E_BUFFER_TOO_SMALL;
  }
  std::memcpy(out, e->proof.data(), e->proof.size());
  table_.erase(it);
  delete e;
  return OK;
}

int32_t Server::warmup(uint32_t max_log_n_rows, uint32_t max_sequence_len, uint32_t log_blowup,
                       uint32_t max_xor_log_n, std::string* err) {
  std::lock_guard<std::mutex> g(mu_);
  if (in_flight_ != 0 || !queue_.empty()) {
    *err = "warmup needs an idle server";
    return E_INVALID;
  }
  cudaSetDevice(ctx_->device);
  const bool persistent = flags_ & SERVER_PERSISTENT_WORKSPACES;
  size_t wf = max_log_n_rows ? WideFibProver::workspace_bytes(max_log_n_rows, max_sequence_len, log_blowup) : 0;
  size_t xr = max_xor_log_n ? LogupXorProver::workspace_bytes(max_xor_log_n, 16, log_blowup, 0) : 0;
  if (persistent && wf) {
    for (uint32_t slot = 0; slot < n_slots_; ++slot) {
      if (held_[slot] >= wf) continue;
      if (in_use_ - held_[slot] + wf > budget_) break;  // slots beyond the budget stay small
      size_t held = 0;
      int32_t rc = provers_[slot]->reserve(max_log_n_rows, max_sequence_len, log_blowup, &held);
      if (rc != OK) {
        *err = provers_[slot]->error();
        return rc;
      }
      in_use_ = in_use_ - held_[slot] + held;
      held_[slot] = held;
    }
  }
  // The XOR-lookup provers' pinned staging (a page-locked host allocation at a slot's first such
  // proof otherwise, inside the serving run).
  if (xr) {
    for (auto* x : xor_provers_) {
      int32_t rc = x->reserve_staging();
      if (rc != OK) {
        *err = x->error();
        return rc;
      }
    }
  }
  // Pre-grow the stream-ordered pool (kept: release threshold = unlimited) by what the transient
  // workspaces of a full set of slots can take at once.
  size_t per_slot = std::max(xr, persistent ? (size_t)0 : wf);
  uint64_t pool = std::min<uint64_t>((uint64_t)per_slot * n_slots_, persistent ? budget_ - std::min(budget_, in_use_)
                                                                               : budget_);
  if (pool) {
    void* p = nullptr;
    cudaStream_t s = ctx_->stream;
    if (cudaMallocAsync(&p, pool, s) != cudaSuccess) {
      cudaGetLastError();
      *err = "pool pre-growth failed";
      return E_OOM;
    }
    cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  }
  snap_.peak_workspace_bytes = std::max<uint64_t>(snap_.peak_workspace_bytes, in_use_);
  return OK;
}

ServerSnapshot Server::snapshot() {
  std::lock_guard<std::mutex> g(mu_);
  return snap_;
}

}  // namespace sb
