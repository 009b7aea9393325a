//! Device buffers for the hooks that receive host slices: the reference's backend hooks hand the
//! backend host memory (the Metal backend's memory is shared with its GPU), so each hook here
//! stages its columns into device memory, calls libstwo_b200 and copies the results back. The
//! CUDA runtime is linked by build_support/backends/cuda_b200.zig.

const std = @import("std");
const ffi = @import("ffi.zig");

const cudaMemcpyHostToDevice: c_int = 1;
const cudaMemcpyDeviceToHost: c_int = 2;

extern fn cudaMalloc(ptr: *?*anyopaque, size: usize) c_int;
extern fn cudaFree(ptr: ?*anyopaque) c_int;
extern fn cudaMemcpy(dst: ?*anyopaque, src: ?*const anyopaque, count: usize, kind: c_int) c_int;
extern fn cudaDeviceSynchronize() c_int;

pub const Error = error{ OutOfMemory, BackendFailure };

/// One device allocation of `len` elements of T; freed by `deinit`.
pub fn Buffer(comptime T: type) type {
    return struct {
        ptr: [*]T,
        len: usize,

        const Self = @This();

        pub fn alloc(len: usize) Error!Self {
            var raw: ?*anyopaque = null;
            if (cudaMalloc(&raw, @max(len, 1) * @sizeOf(T)) != 0 or raw == null) return error.OutOfMemory;
            return .{ .ptr = @ptrCast(@alignCast(raw.?)), .len = len };
        }

        pub fn deinit(self: *Self) void {
            _ = cudaFree(self.ptr);
            self.* = undefined;
        }

        /// Copies `src` to elements [at, at + src.len).
        pub fn upload(self: Self, at: usize, src: []const T) Error!void {
            std.debug.assert(at + src.len <= self.len);
            if (src.len == 0) return;
            if (cudaMemcpy(self.ptr + at, src.ptr, src.len * @sizeOf(T), cudaMemcpyHostToDevice) != 0)
                return error.BackendFailure;
        }

        /// Copies elements [at, at + dst.len) to `dst` (waits for the device).
        pub fn download(self: Self, at: usize, dst: []T) Error!void {
            std.debug.assert(at + dst.len <= self.len);
            if (dst.len == 0) return;
            if (cudaMemcpy(dst.ptr, self.ptr + at, dst.len * @sizeOf(T), cudaMemcpyDeviceToHost) != 0)
                return error.BackendFailure;
        }
    };
}

/// Columns of one length packed column-major into one device buffer (stride = column length).
pub fn uploadColumns(comptime T: type, columns: anytype) Error!Buffer(T) {
    const n = if (columns.len == 0) 0 else columns[0].len;
    var buf = try Buffer(T).alloc(n * columns.len);
    errdefer buf.deinit();
    for (columns, 0..) |column, c| {
        std.debug.assert(column.len == n);
        try buf.upload(c * n, @as([*]const T, @ptrCast(column.ptr))[0..n]);
    }
    return buf;
}

pub fn synchronize() Error!void {
    if (cudaDeviceSynchronize() != 0) return error.BackendFailure;
}

test "buffer types are plain words" {
    try std.testing.expectEqual(@as(usize, 4), @sizeOf(u32));
    try std.testing.expectEqual(@as(usize, 16), @sizeOf(ffi.Qm31));
}
