//! B200 (sm_100a) CUDA backend of the circle-STARK prover: libstwo_b200 behind the reference's
//! backend contract. Drops in beside src/backends/metal/mod.zig:
//!   const backend = @import("backends/cuda_b200/mod.zig").CudaB200CommitBackend;
//! and the example's engine selection (ProverEngineForBackend, src/examples/wide_fibonacci.zig:35-37).

pub const ffi = @import("ffi.zig");
pub const device = @import("device.zig");
pub const commit_backend = @import("commit_backend.zig");
pub const CudaB200CommitBackend = commit_backend.CudaB200CommitBackend;

test {
    _ = ffi;
    _ = device;
}
