//! CudaB200CommitBackend: the reference's backend contract (src/backend/mod.zig) and the optional
//! hooks it probes with @hasDecl, routed through libstwo_b200 (ffi.zig). It mirrors the hook names
//! and signatures of MetalCommitBackend (src/backends/metal/commit_backend.zig:35-823) so that the
//! generic prover (src/prover/pcs/*.zig, src/prover/fri.zig, src/examples/wide_fibonacci/trace.zig)
//! drives it unchanged.
//!
//! The reference's hooks hand the backend host slices. Each hook here stages its columns into
//! device memory (device.zig), calls one library entry point and copies the result back; that is
//! the drop-in path. Below a size threshold, for domains other than the canonic ones the library
//! transforms, and for hashers other than the "leaf"/"node"-prefixed Blake2s Merkle hasher, a hook
//! takes the CPU path, as MetalCommitBackend does (commit_backend.zig:199-221,341-386). Ops the
//! device does not take delegate to `cpu` (commit_backend.zig:438-442,817-823).
//!
//! The fastest route is the engine-level call `proveWideFibonacci` below: every column stays on the
//! device for the whole proof and only roots, sampled values, the last FRI layer, the nonce and the
//! decommitment cross the bus; its output is the reference's JSON wire encoding
//! (src/interop/proof_wire.zig), which `decodeProofBytes` turns into a StarkProof.

const std = @import("std");
const ffi = @import("ffi.zig");
const device = @import("device.zig");
const cpu = @import("../cpu_scalar/mod.zig").CpuBackend;
const merkle = @import("stwo_prover_impl").vcs_lifted.prover;
const blake2_merkle = @import("stwo_core").vcs_lifted.blake2_merkle;
const canonic = @import("stwo_core").poly.circle.canonic;
const poly = @import("stwo_prover_impl").poly.circle.poly;

const M31 = @import("stwo_core").fields.m31.M31;
const QM31 = @import("stwo_core").fields.qm31.QM31;
const CircleDomain = @import("stwo_core").poly.circle.domain.CircleDomain;
const TwiddleTree = @import("stwo_prover_impl").poly.twiddles.TwiddleTree([]const M31);
const SecureColumnByCoords = @import("stwo_prover_impl").secure_column.SecureColumnByCoords;

/// Columns below this many cells stay on the host: staging them costs more than the CPU work.
pub const device_min_cells: usize = 1 << 16;

// ---------------------------------------------------------------
// Runtime: one library context per process, on one device.
// ---------------------------------------------------------------

pub const RuntimeInitializationPolicy = struct {
    device: i32 = 0,
};

pub const RuntimeLifecycleSnapshot = struct {
    initialized: bool,
    device: i32,
};

pub const TelemetrySnapshot = struct {
    kernel_launches: u64,
};

var runtime_mutex: std.Thread.Mutex = .{};
var runtime_ctx: ?*ffi.Context = null;
var runtime_device: i32 = 0;

fn context() !*ffi.Context {
    runtime_mutex.lock();
    defer runtime_mutex.unlock();
    if (runtime_ctx) |ctx| return ctx;
    var out: ?*ffi.Context = null;
    try ffi.statusError(ffi.stwo_b200_context_create(runtime_device, &out));
    runtime_ctx = out;
    return out.?;
}

fn isCanonicDomain(domain: CircleDomain) bool {
    const want = canonic.CanonicCoset.new(domain.logSize()).circleDomain();
    return domain.half_coset.initial_index.eql(want.half_coset.initial_index) and
        domain.half_coset.step_size.eql(want.half_coset.step_size);
}

fn words(column: []const M31) []const u32 {
    return @as([*]const u32, @ptrCast(column.ptr))[0..column.len];
}

fn wordsMut(column: []M31) []u32 {
    return @as([*]u32, @ptrCast(column.ptr))[0..column.len];
}

fn qm31(v: QM31) ffi.Qm31 {
    const c = v.toM31Array();
    return .{ .a = c[0].v, .b = c[1].v, .c = c[2].v, .d = c[3].v };
}

pub const CudaB200CommitBackend = struct {
    pub const TelemetryError = error{RuntimeNotInitialized};
    pub const preferContiguousQuadraticRecurrenceTrace = true;

    pub fn warmup() !void {
        _ = try context();
    }

    pub fn initializeRuntime(allocator: std.mem.Allocator, policy: RuntimeInitializationPolicy) !void {
        _ = allocator;
        runtime_mutex.lock();
        const busy = runtime_ctx != null and runtime_device != policy.device;
        if (!busy) runtime_device = policy.device;
        runtime_mutex.unlock();
        if (busy) return error.RuntimeAlreadyInitialized;
        _ = try context();
    }

    pub fn runtimeLifecycleSnapshot() RuntimeLifecycleSnapshot {
        runtime_mutex.lock();
        defer runtime_mutex.unlock();
        return .{ .initialized = runtime_ctx != null, .device = runtime_device };
    }

    pub fn shutdown() !void {
        runtime_mutex.lock();
        defer runtime_mutex.unlock();
        if (runtime_ctx) |ctx| try ffi.statusError(ffi.stwo_b200_context_destroy(ctx));
        runtime_ctx = null;
    }

    pub fn telemetrySnapshot() TelemetryError!TelemetrySnapshot {
        if (!runtimeLifecycleSnapshot().initialized) return error.RuntimeNotInitialized;
        var t: ffi.Telemetry = undefined;
        ffi.statusError(ffi.stwo_b200_telemetry_snapshot(&t)) catch return error.RuntimeNotInitialized;
        return .{ .kernel_launches = t.kernel_launches };
    }

    // -----------------------------------------------------------
    // Ops the device does not take (src/backend/mod.zig contract)
    // -----------------------------------------------------------

    pub const ColumnType = cpu.ColumnType;
    pub const batchInverse = cpu.batchInverse;
    pub const interpolate = cpu.interpolate;
    pub const evaluateOnDomain = cpu.evaluateOnDomain;
    pub const evalAtPoint = cpu.evalAtPoint;
    pub const foldLine = cpu.foldLine;
    pub const foldLineN = cpu.foldLineN;
    pub const accumulateQuotients = cpu.accumulateQuotients;
    pub const accumulate = cpu.accumulate;
    pub const genEqEvals = cpu.genEqEvals;
    pub const nextLayer = cpu.nextLayer;
    pub const sumAsPolyInFirstVariable = cpu.sumAsPolyInFirstVariable;
    pub const computeCompositionEvaluation = cpu.computeCompositionEvaluation;

    // -----------------------------------------------------------
    // MerkleOps (src/backend/merkle_ops.zig:20-56)
    // -----------------------------------------------------------

    /// The CPU backend's tree type: the device computes every layer, the host keeps them for
    /// decommitment (root-first, as MerkleProverLifted stores them).
    pub fn MerkleTree(comptime H: type) type {
        return merkle.MerkleProverLifted(H);
    }

    pub fn commitMerkle(comptime H: type, allocator: std.mem.Allocator, columns: []const []const M31) !MerkleTree(H) {
        if (H != blake2_merkle.Blake2sMerkleHasher) return cpu.commitMerkle(H, allocator, columns);
        var cells: usize = 0;
        var max_len: usize = 0;
        var same = true;
        for (columns) |column| {
            cells = try std.math.add(usize, cells, column.len);
            max_len = @max(max_len, column.len);
            if (column.len != columns[0].len) same = false;
        }
        if (cells < device_min_cells or !std.math.isPowerOfTwo(max_len)) return cpu.commitMerkle(H, allocator, columns);
        const ctx = try context();
        const log_size: u32 = @intCast(std.math.log2_int(usize, max_len));
        const n_hashes = 2 * max_len - 1;
        var layers = try device.Buffer(u8).alloc(n_hashes * 32);
        defer layers.deinit();
        if (same) {
            var cols = try device.uploadColumns(u32, columns);
            defer cols.deinit();
            try ffi.statusError(ffi.stwo_b200_merkle_commit(ctx, log_size, @intCast(columns.len), cols.ptr, max_len,
                layers.ptr, null, null));
        } else {
            // Columns of mixed sizes: one device buffer each, hashed at their lifted index.
            const bufs = try allocator.alloc(device.Buffer(u32), columns.len);
            defer allocator.free(bufs);
            const ptrs = try allocator.alloc([*]const u32, columns.len);
            defer allocator.free(ptrs);
            const logs = try allocator.alloc(u32, columns.len);
            defer allocator.free(logs);
            var made: usize = 0;
            defer for (bufs[0..made]) |*b| b.deinit();
            for (columns, 0..) |column, i| {
                if (!std.math.isPowerOfTwo(column.len)) return error.InvalidColumnSize;
                bufs[i] = try device.Buffer(u32).alloc(column.len);
                made += 1;
                try bufs[i].upload(0, words(column));
                ptrs[i] = bufs[i].ptr;
                logs[i] = @intCast(std.math.log2_int(usize, column.len));
            }
            try ffi.statusError(ffi.stwo_b200_merkle_commit_lifted(ctx, @intCast(columns.len), ptrs.ptr, logs.ptr,
                layers.ptr, null, null));
        }
        return treeFromDevice(H, allocator, layers, log_size);
    }

    /// Layers come back leaves first (2^L leaves, then each parent layer); MerkleProverLifted keeps
    /// them root first.
    fn treeFromDevice(comptime H: type, allocator: std.mem.Allocator, layers: device.Buffer(u8), log_size: u32) !MerkleTree(H) {
        comptime std.debug.assert(@sizeOf(H.Hash) == 32);
        const out = try allocator.alloc([]H.Hash, log_size + 1);
        var filled: usize = 0;
        errdefer {
            for (out[0..filled]) |layer| allocator.free(layer);
            allocator.free(out);
        }
        var at: usize = 0;
        var width: usize = @as(usize, 1) << @intCast(log_size);
        var level: usize = log_size + 1;
        while (level > 0) : (level -= 1) {
            const layer = try allocator.alloc(H.Hash, width);
            out[level - 1] = layer;
            filled += 1;
            try layers.download(at * 32, std.mem.sliceAsBytes(layer));
            at += width;
            width /= 2;
        }
        return .{ .layers = out, .layer_allocator = allocator };
    }

    pub fn commitMerkleWithBacking(
        comptime H: type,
        allocator: std.mem.Allocator,
        columns: []const []const M31,
        backing_buffers: []const []M31,
    ) !MerkleTree(H) {
        _ = backing_buffers;
        return commitMerkle(H, allocator, columns);
    }

    /// Quotients computed by the prover's provider, their four coordinate columns committed on the
    /// device (the engine-level call keeps both on the device).
    pub fn commitLazyMerkle(comptime H: type, allocator: std.mem.Allocator, provider: anytype, out: anytype) !MerkleTree(H) {
        try provider.computeAll(allocator, out);
        const columns = [_][]const M31{ out.columns[0], out.columns[1], out.columns[2], out.columns[3] };
        return commitMerkle(H, allocator, columns[0..]);
    }

    // -----------------------------------------------------------
    // PolyOps hooks (src/prover/pcs/columns/circle_transforms.zig:212,248;
    // src/prover/pcs/columns/preparation.zig:249)
    // -----------------------------------------------------------

    fn transformInPlace(values: []const []M31, domain: CircleDomain, inverse: bool) !void {
        const ctx = try context();
        const n = domain.size();
        const cols: []const []const M31 = @ptrCast(values);
        var buf = try device.uploadColumns(u32, cols);
        defer buf.deinit();
        const rc = if (inverse)
            ffi.stwo_b200_interpolate_columns(ctx, domain.logSize(), @intCast(values.len), buf.ptr, n, null)
        else
            ffi.stwo_b200_evaluate_columns(ctx, domain.logSize(), @intCast(values.len), buf.ptr, n, null);
        try ffi.statusError(rc);
        for (values, 0..) |column, c| try buf.download(c * n, wordsMut(column));
    }

    fn onDevice(values: []const []M31, domain: CircleDomain) bool {
        if (domain.logSize() < 3 or !isCanonicDomain(domain) or values.len == 0) return false;
        for (values) |column| if (column.len != domain.size()) return false;
        return values.len * domain.size() >= device_min_cells;
    }

    pub fn interpolateCircleBuffers(allocator: std.mem.Allocator, values: []const []M31, domain: CircleDomain,
        twiddle_tree: TwiddleTree) !void {
        _ = allocator;
        if (!onDevice(values, domain)) return poly.interpolateBuffersWithTwiddles(values, domain, twiddle_tree);
        return transformInPlace(values, domain, true);
    }

    pub fn evaluateCircleBuffers(allocator: std.mem.Allocator, values: []const []M31, domain: CircleDomain,
        twiddle_tree: TwiddleTree) !void {
        _ = allocator;
        if (!onDevice(values, domain)) return poly.evaluateBuffersWithTwiddles(values, domain, twiddle_tree);
        return transformInPlace(values, domain, false);
    }

    pub fn interpolateAndEvaluateCircleBuffers(
        allocator: std.mem.Allocator,
        source_values: []const []const M31,
        base_values: []const []M31,
        extended_values: []const []M31,
        transform_buffer: []M31,
        extended_start: usize,
        extended_stride: usize,
        base_domain: CircleDomain,
        base_twiddles: TwiddleTree,
        extended_domain: CircleDomain,
        extended_twiddles: TwiddleTree,
    ) !void {
        const log_n = base_domain.logSize();
        const log_e = extended_domain.logSize();
        const device_ok = log_n >= 3 and log_e > log_n and log_e - log_n <= 4 and isCanonicDomain(base_domain) and
            isCanonicDomain(extended_domain) and source_values.len * base_domain.size() >= device_min_cells;
        if (!device_ok) {
            return cpu.interpolateAndEvaluateCircleBuffers(allocator, source_values, base_values, extended_values,
                transform_buffer, extended_start, extended_stride, base_domain, base_twiddles, extended_domain,
                extended_twiddles);
        }
        const ctx = try context();
        const n = base_domain.size();
        const e = extended_domain.size();
        var src = try device.uploadColumns(u32, source_values);
        defer src.deinit();
        var coeffs = try device.Buffer(u32).alloc(n * source_values.len);
        defer coeffs.deinit();
        var lde = try device.Buffer(u32).alloc(e * source_values.len);
        defer lde.deinit();
        try ffi.statusError(ffi.stwo_b200_interpolate_and_extend(ctx, log_n, log_e - log_n, @intCast(source_values.len),
            src.ptr, n, coeffs.ptr, n, lde.ptr, e, null));
        for (base_values, 0..) |column, c| try coeffs.download(c * n, wordsMut(column));
        for (extended_values, 0..) |column, c| try lde.download(c * e, wordsMut(column));
    }

    /// The composition's four coordinate columns interpolated in place
    /// (src/prover/poly/circle/secure_poly.zig:173).
    pub fn interpolateSecureComposition(allocator: std.mem.Allocator, values: *SecureColumnByCoords,
        domain: CircleDomain, twiddle_tree: TwiddleTree) !bool {
        const cols = values.columns[0..];
        if (!onDevice(cols, domain)) return cpu.interpolateSecureComposition(allocator, values, domain, twiddle_tree);
        try transformInPlace(cols, domain, true);
        return true;
    }

    // -----------------------------------------------------------
    // FriOps hooks (src/backend/fri_ops.zig:29-37; src/prover/fri.zig:341-350)
    // -----------------------------------------------------------

    /// dst = dst * alpha^2 + fold(src): the accumulating fold of the CPU backend.
    pub fn foldCircleIntoLine(
        allocator: std.mem.Allocator,
        dst: []QM31,
        src_columns: [4][]const M31,
        src_domain: CircleDomain,
        alpha: QM31,
        workspace: anytype,
    ) !void {
        const n = src_domain.size();
        if (n < device_min_cells or !isCanonicDomain(src_domain) or dst.len * 2 != n)
            return cpu.foldCircleIntoLine(allocator, dst, src_columns, src_domain, alpha, workspace);
        const ctx = try context();
        const half = n / 2;
        var src = try device.uploadColumns(u32, src_columns[0..]);
        defer src.deinit();
        var acc = try device.Buffer(u32).alloc(4 * half);
        defer acc.deinit();
        const coords = try allocator.alloc(u32, 4 * half);
        defer allocator.free(coords);
        for (dst, 0..) |v, i| {
            const c = v.toM31Array();
            for (0..4) |k| coords[k * half + i] = c[k].v;
        }
        try acc.upload(0, coords);
        try ffi.statusError(ffi.stwo_b200_fold_circle_into_line(ctx, src_domain.logSize(), src.ptr, n, qm31(alpha),
            acc.ptr, half, 1, null));
        try acc.download(0, coords);
        for (dst, 0..) |*v, i| v.* = QM31.fromU32Unchecked(coords[i], coords[half + i], coords[2 * half + i], coords[3 * half + i]);
    }

    // -----------------------------------------------------------
    // Trace hooks (src/examples/wide_fibonacci/trace.zig:63-74)
    // -----------------------------------------------------------

    pub fn admitsQuadraticRecurrenceTrace(row_count: usize, column_count: usize) bool {
        const cells = std.math.mul(usize, row_count, column_count) catch return false;
        return column_count >= 2 and column_count <= 1000 and std.math.isPowerOfTwo(row_count) and
            row_count <= (1 << 22) and cells >= device_min_cells;
    }

    pub fn fillQuadraticRecurrenceTrace(columns: [][]M31, log_n_rows: u32, recipe: [7]u32) !void {
        const ctx = try context();
        const n = @as(usize, 1) << @intCast(log_n_rows);
        var buf = try device.Buffer(u32).alloc(n * columns.len);
        defer buf.deinit();
        try ffi.statusError(ffi.stwo_b200_quadratic_recurrence_trace(ctx, log_n_rows, @intCast(columns.len), &recipe,
            buf.ptr, n, null));
        for (columns, 0..) |column, c| try buf.download(c * n, wordsMut(column));
    }

    // -----------------------------------------------------------
    // Engine level: a whole wide-Fibonacci proof on the device
    // (ProverEngine.prove, src/prover/engine.zig:163-181)
    // -----------------------------------------------------------

    /// Proves `statement` under `config` from a trace prepared in bit-reversed circle order
    /// (`trace` holds sequence_len columns of 2^log_n_rows words, or null for the reference's
    /// (1, row) seeds) and returns the proof's JSON wire bytes, owned by `allocator`.
    pub fn proveWideFibonacci(
        allocator: std.mem.Allocator,
        log_n_rows: u32,
        sequence_len: u32,
        config: ffi.PcsConfig,
        trace: ?[]const u32,
        channel_seed: ?u64,
    ) ![]u8 {
        const ctx = try context();
        const req = ffi.WideFibRequest{
            .log_n_rows = log_n_rows,
            .sequence_len = sequence_len,
            .config = config,
            .trace_host = if (trace) |t| t.ptr else null,
            .trace_device = null,
            .trace_kind = ffi.TRACE_REFERENCE,
            .has_channel_seed = @intFromBool(channel_seed != null),
            .trace_seed = 0,
            .channel_seed = channel_seed orelse 0,
        };
        // A secure 2^20 x 100 proof is about 1.1 MB of JSON; a larger one reports its length and is
        // proven again into a buffer of that size (proofs are deterministic).
        var out = try allocator.alloc(u8, 4 << 20);
        errdefer allocator.free(out);
        var len: usize = 0;
        const rc = ffi.stwo_b200_prove_wide_fibonacci(ctx, &req, out.ptr, out.len, &len, null);
        if (rc == ffi.E_BUFFER_TOO_SMALL) {
            out = try allocator.realloc(out, len);
            try ffi.statusError(ffi.stwo_b200_prove_wide_fibonacci(ctx, &req, out.ptr, out.len, &len, null));
        } else {
            try ffi.statusError(rc);
        }
        return allocator.realloc(out, len);
    }
};
