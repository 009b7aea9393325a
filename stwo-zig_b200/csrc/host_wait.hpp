// Host waits of the provers for their streams and events.
//
// The runtime's synchronize calls spin on a host core for the whole wait when the context runs
// under the default scheduling policy (spin while the process holds fewer CUDA contexts than the
// host has logical processors), and the context is usually created by the embedder, so the
// library cannot choose the policy. With more proofs in flight than host cores, the spinning
// waiters took the cores from the proof threads that had host work to do (transcript, decommitment
// plan, JSON). These waits poll and give the processor up between polls instead: with a core to
// spare the yield returns at once and the wait ends as soon as the work does.
#pragma once
#include <cuda_runtime.h>

#include <thread>

namespace sb {

inline cudaError_t stream_wait(cudaStream_t s) {
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e != cudaErrorNotReady) return e;
    std::this_thread::yield();
  }
}

inline cudaError_t event_wait(cudaEvent_t ev) {
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e != cudaErrorNotReady) return e;
    std::this_thread::yield();
  }
}

}  // namespace sb
