//! Extern declarations of libstwo_b200 (include/stwo_b200.h), the B200 (sm_100a) backend library.
//!
//! One `extern fn` per entry point and one `extern struct` per C struct, in the header's order
//! and with its field names, the way src/backends/cuda/ffi.zig binds the stwo-cuda prototypes.
//! Every function returns an i32 status (0 = ok, negative = error; `statusError` maps it).
//! The doc comment above each struct names its C typedef; a CPU test of the library
//! (tests/test_zig_glue.py) checks every declaration here against the header: names, field order,
//! widths, pointer shapes, arity and the C layout (sizes and offsets).
//! Linked by build_support/backends/cuda_b200.zig.

// ---------------------------------------------------------------
// Status codes
// ---------------------------------------------------------------

pub const OK: i32 = 0;
pub const E_INVALID: i32 = -1;
pub const E_OOM: i32 = -2;
pub const E_CUDA: i32 = -3;
pub const E_TIMEOUT: i32 = -4;
pub const E_CONSTRAINTS: i32 = -5;
pub const E_BUFFER_TOO_SMALL: i32 = -6;
pub const E_FALLBACK: i32 = -7;
pub const E_NO_DEVICE: i32 = -8;
pub const E_DIVISION_BY_ZERO: i32 = -9;
pub const E_REJECTED: i32 = -10;

pub const TRACE_REFERENCE: u32 = 0;
pub const TRACE_SEEDED: u32 = 1;
pub const TRACE_FIRST_COLUMNS: u32 = 2;
pub const SERVER_PERSISTENT_WORKSPACES: u32 = 1;
pub const SERVER_VERIFY: u32 = 2;
pub const NOALLOC_EVAL_SCRATCH: u32 = 65536;
pub const EVAL_AT_POINT_MAX_COLS: u32 = 65535;
pub const MAX_POW_BITS: u32 = 40;
pub const LOGUP_MAX_WORDS = 8;
pub const LOGUP_MAX_USES = 32;

pub const Error = error{
    ShapeMismatch,
    OutOfMemory,
    BackendFailure,
    DeviceTimeout,
    ConstraintsNotSatisfied,
    BufferTooSmall,
    BackendFallback,
    NoDevice,
    DivisionByZero,
    CommittedCellBudgetExceeded,
};

/// Status code -> Zig error, in the reference's error vocabulary where one exists
/// (error.ShapeMismatch, error.ConstraintsNotSatisfied, error.DivisionByZero,
/// error.CommittedCellBudgetExceeded of src/prover/native/resource_admission.zig).
pub fn statusError(rc: i32) Error!void {
    return switch (rc) {
        OK => {},
        E_INVALID => error.ShapeMismatch,
        E_OOM => error.OutOfMemory,
        E_TIMEOUT => error.DeviceTimeout,
        E_CONSTRAINTS => error.ConstraintsNotSatisfied,
        E_BUFFER_TOO_SMALL => error.BufferTooSmall,
        E_FALLBACK => error.BackendFallback,
        E_NO_DEVICE => error.NoDevice,
        E_DIVISION_BY_ZERO => error.DivisionByZero,
        E_REJECTED => error.CommittedCellBudgetExceeded,
        else => error.BackendFailure,
    };
}

// ---------------------------------------------------------------
// Types
// ---------------------------------------------------------------

pub const Context = opaque {};
pub const Server = opaque {};

/// stwo_b200_qm31: (c0.a, c0.b, c1.a, c1.b), the layout of CudaQM31 in src/backends/cuda/ffi.zig.
pub const Qm31 = extern struct {
    a: u32,
    b: u32,
    c: u32,
    d: u32,
};

/// stwo_b200_pcs_config
pub const PcsConfig = extern struct {
    pow_bits: u32,
    log_blowup_factor: u32,
    log_last_layer_degree_bound: u32,
    n_queries: u32,
};

/// stwo_b200_wide_fib_request
pub const WideFibRequest = extern struct {
    log_n_rows: u32,
    sequence_len: u32,
    config: PcsConfig,
    trace_host: ?[*]const u32,
    trace_device: ?[*]const u32,
    trace_kind: u32,
    has_channel_seed: u32,
    trace_seed: u64,
    channel_seed: u64,
};

/// stwo_b200_stage_times
pub const StageTimes = extern struct {
    upload: f32,
    trace: f32,
    main_commit: f32,
    composition: f32,
    composition_commit: f32,
    oods: f32,
    quotients: f32,
    fri: f32,
    pow: f32,
    decommit: f32,
    total: f32,
    host_encode: f32,
    host_gaps: f32,
};

/// stwo_b200_telemetry
pub const Telemetry = extern struct {
    kernel_launches: u64,
};

/// stwo_b200_xor_request
pub const XorRequest = extern struct {
    log_n: u32,
    log_table: u32,
    config: PcsConfig,
    seed: u64,
    has_channel_seed: u32,
    reserved: u32,
    channel_seed: u64,
};

/// stwo_b200_server_config
pub const ServerConfig = extern struct {
    slots: u32,
    profile: u32,
    memory_budget: u64,
    flags: u32,
};

/// stwo_b200_request_stats
pub const RequestStats = extern struct {
    accounted_bytes: u64,
    workspace_bytes: u64,
    queued_ms: f64,
    run_ms: f64,
    slot: u32,
    stages: StageTimes,
};

/// stwo_b200_server_snapshot
pub const ServerSnapshot = extern struct {
    submitted: u64,
    completed: u64,
    failed: u64,
    rejected: u64,
    peak_in_flight: u64,
    peak_workspace_bytes: u64,
    budget_bytes: u64,
};

/// stwo_b200_logup_use
pub const LogupUse = extern struct {
    n_words: u32,
    negate: u32,
    words: [LOGUP_MAX_WORDS]?[*]const u32,
    constants: [LOGUP_MAX_WORDS]u32,
    multiplicity: ?[*]const u32,
};

// ---------------------------------------------------------------
// Runtime
// ---------------------------------------------------------------

pub extern fn stwo_b200_context_create(device: i32, out: *?*Context) i32;
pub extern fn stwo_b200_context_destroy(ctx: ?*Context) i32;
pub extern fn stwo_b200_last_error() [*:0]const u8;
pub extern fn stwo_b200_status_string(status: i32) [*:0]const u8;
pub extern fn stwo_b200_version() [*:0]const u8;
pub extern fn stwo_b200_telemetry_snapshot(out: *Telemetry) i32;

// ---------------------------------------------------------------
// Engine level
// ---------------------------------------------------------------

pub extern fn stwo_b200_prove_wide_fibonacci(ctx: *Context, req: *const WideFibRequest, proof_out: ?[*]u8,
    proof_cap: usize, proof_len: ?*usize, times: ?*StageTimes) i32;
pub extern fn stwo_b200_prove_wide_fibonacci_batch(ctx: *Context, reqs: [*]const WideFibRequest, n: usize,
    proof_outs: [*]const [*]u8, proof_caps: [*]const usize, proof_lens: [*]usize, statuses: [*]i32,
    max_in_flight: u32, times: ?[*]StageTimes) i32;
pub extern fn stwo_b200_prove_logup_xor(ctx: *Context, req: *const XorRequest, proof_out: ?[*]u8,
    proof_cap: usize, proof_len: ?*usize) i32;

// ---------------------------------------------------------------
// Verifier (host)
// ---------------------------------------------------------------

pub extern fn stwo_b200_verify_wide_fibonacci(proof: [*]const u8, proof_len: usize, log_n_rows: u32,
    sequence_len: u32, has_channel_seed: u32, channel_seed: u64) i32;
pub extern fn stwo_b200_verify_logup_xor(proof: [*]const u8, proof_len: usize, log_n: u32, log_table: u32,
    has_channel_seed: u32, channel_seed: u64) i32;

// ---------------------------------------------------------------
// Serving loop
// ---------------------------------------------------------------

pub extern fn stwo_b200_server_create(ctx: *Context, cfg: *const ServerConfig, out: *?*Server) i32;
pub extern fn stwo_b200_server_submit(server: *Server, req: *const WideFibRequest, ticket: *u64) i32;
pub extern fn stwo_b200_server_submit_xor(server: *Server, req: *const XorRequest, ticket: *u64) i32;
pub extern fn stwo_b200_server_wait(server: *Server, ticket: u64, proof_out: ?[*]u8, proof_cap: usize,
    proof_len: ?*usize, stats: ?*RequestStats) i32;
pub extern fn stwo_b200_server_warmup(server: *Server, max_log_n_rows: u32, max_sequence_len: u32,
    log_blowup: u32, max_xor_log_n: u32) i32;
pub extern fn stwo_b200_server_snapshot_get(server: *Server, out: *ServerSnapshot) i32;
pub extern fn stwo_b200_server_set_request_timeout(server: *Server, timeout_ms: u32) i32;
pub extern fn stwo_b200_server_destroy(server: ?*Server) i32;

// ---------------------------------------------------------------
// PolyOps (device pointers; `stream` is a cudaStream_t or null for the legacy stream)
// ---------------------------------------------------------------

pub extern fn stwo_b200_interpolate_columns(ctx: *Context, log_size: u32, n_cols: u32, cols: [*]u32,
    stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_evaluate_columns(ctx: *Context, log_size: u32, n_cols: u32, cols: [*]u32,
    stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_interpolate_and_extend(ctx: *Context, log_size: u32, log_blowup: u32, n_cols: u32,
    evals: [*]const u32, evals_stride: u64, coeffs: [*]u32, coeffs_stride: u64, lde: [*]u32, lde_stride: u64,
    stream: ?*anyopaque) i32;
pub extern fn stwo_b200_extend_columns(ctx: *Context, log_size: u32, log_blowup: u32, n_cols: u32,
    coeffs: [*]const u32, coeffs_stride: u64, lde: [*]u32, lde_stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_eval_at_point(ctx: *Context, log_size: u32, n_cols: u32, coeffs: [*]const u32,
    stride: u64, px: Qm31, py: Qm31, out_dev: [*]Qm31, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_eval_at_point_noalloc(ctx: *Context, log_size: u32, n_cols: u32, coeffs: [*]const u32,
    stride: u64, px: Qm31, py: Qm31, out_dev: [*]Qm31, stream: ?*anyopaque) i32;

// ---------------------------------------------------------------
// MerkleOps
// ---------------------------------------------------------------

pub extern fn stwo_b200_merkle_commit(ctx: *Context, log_size: u32, n_cols: u32, cols: ?[*]const u32,
    stride: u64, layers_dev: [*]u8, root_host: ?*[32]u8, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_merkle_commit_lifted(ctx: *Context, n_cols: u32, cols: [*]const [*]const u32,
    log_sizes: [*]const u32, layers_dev: [*]u8, root_host: ?*[32]u8, stream: ?*anyopaque) i32;

// ---------------------------------------------------------------
// FriOps
// ---------------------------------------------------------------

pub extern fn stwo_b200_fold_circle_into_line(ctx: *Context, src_log: u32, src: [*]const u32, src_stride: u64,
    alpha: Qm31, dst: [*]u32, dst_stride: u64, accumulate: i32, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_fold_line(ctx: *Context, src_log: u32, src: [*]const u32, src_stride: u64,
    alpha: Qm31, dst: [*]u32, dst_stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_fold_and_commit(ctx: *Context, circle: i32, src_log: u32, src: [*]const u32,
    src_stride: u64, alpha: Qm31, dst: [*]u32, dst_stride: u64, layers_dev: ?[*]u8, root_host: ?*[32]u8,
    stream: ?*anyopaque) i32;
pub extern fn stwo_b200_commit_columns(ctx: *Context, log_size: u32, log_blowup: u32, n_cols: u32,
    evals: [*]const u32, evals_stride: u64, coeffs: [*]u32, coeffs_stride: u64, lde: [*]u32, lde_stride: u64,
    layers_dev: [*]u8, root_host: ?*[32]u8, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_interpolate_secure_composition(ctx: *Context, comp_log: u32, comp: [*]u32,
    comp_stride: u64, log_blowup: u32, lde: [*]u32, lde_stride: u64, stream: ?*anyopaque) i32;

// ---------------------------------------------------------------
// QuotientOps and AccumulationOps
// ---------------------------------------------------------------

pub extern fn stwo_b200_accumulate_quotients(ctx: *Context, log_size: u32, n_cols: u32,
    col_ptrs_dev: [*]const [*]const u32, c_dev: [*]const Qm31, px: Qm31, py: Qm31, sum_a: Qm31, sum_b: Qm31,
    out: [*]u32, out_stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_accumulate(ctx: *Context, dst_log: u32, dst: [*]u32, dst_stride: u64, src_log: u32,
    src: [*]const u32, src_stride: u64, coeff: Qm31, stream: ?*anyopaque) i32;

// ---------------------------------------------------------------
// Wide-Fibonacci AIR
// ---------------------------------------------------------------

pub extern fn stwo_b200_wide_fib_trace(ctx: *Context, log_n_rows: u32, sequence_len: u32, trace_kind: u32,
    seed: u64, out: [*]u32, stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_quadratic_recurrence_trace(ctx: *Context, log_n_rows: u32, n_cols: u32,
    recipe: *const [7]u32, out: [*]u32, stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_wide_fib_composition(ctx: *Context, log_n_rows: u32, sequence_len: u32,
    eval: [*]const u32, stride: u64, coeffs_dev: [*]const Qm31, den_inv0: u32, den_inv1: u32, out: [*]u32,
    out_stride: u64, stream: ?*anyopaque) i32;

// ---------------------------------------------------------------
// FieldOps, LogUp, XOR lookup trace, proof of work
// ---------------------------------------------------------------

pub extern fn stwo_b200_batch_inverse(ctx: *Context, degree: u32, n: u64, src: [*]const u32, src_stride: u64,
    dst: [*]u32, dst_stride: u64, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_logup_interaction(ctx: *Context, log_rows: u32, n_uses: u32, uses: [*]const LogupUse,
    alphas: [*]const Qm31, z: Qm31, batch: u32, order: u32, out: [*]u32, out_stride: u64, claimed_host: *Qm31,
    stream: ?*anyopaque) i32;
pub extern fn stwo_b200_xor_lookup_trace(ctx: *Context, log_n: u32, seed: u64, main_cols: [*]u32,
    table: [*]u32, multiplicity: [*]u32, stream: ?*anyopaque) i32;
pub extern fn stwo_b200_pow_grind(ctx: *Context, prefix_digest: *const [32]u8, n_bits: u32, nonce_out: *u64) i32;

// ---------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------

/// stwo_b200_tune_entry
pub const TuneEntry = extern struct {
    op: u32,
    log_size: u32,
    n_cols: u32,
    variant: i32,
    ms: [4]f32,
};

pub extern fn stwo_b200_autotune_mode(mode: i32) i32;
pub extern fn stwo_b200_autotune_wide_fibonacci(ctx: *Context, log_n_rows: u32, sequence_len: u32,
    log_blowup: u32) i32;
pub extern fn stwo_b200_autotune_table(out: ?[*]TuneEntry, cap: usize, n: *usize) i32;

// ---------------------------------------------------------------
// Testing
// ---------------------------------------------------------------

pub extern fn stwo_b200_arm_allocation_failure_for_testing(nth: u32) i32;
pub extern fn stwo_b200_arm_quotient_stage_timeout_for_testing() i32;
