//! Link contract of the B200 backend: libstwo_b200 (built by `make -C stwo-zig_b200`, sm_100a)
//! in place of the external libstwo_cuda that build_support/backends/cuda.zig links by name.
//! Explicit directories only, as the reference's CUDA toolchain contract requires.

const std = @import("std");

pub const Toolchain = struct {
    /// Directory holding libstwo_b200.so (stwo-zig_b200/lib of this repository).
    library_dir: ?[]const u8 = null,
    /// Directory holding libcudart (the CUDA 12 runtime).
    runtime_dir: ?[]const u8 = null,
    /// Directory holding stwo_b200.h (include/ of this repository), for @cImport users.
    include_dir: ?[]const u8 = null,

    pub fn validate(self: Toolchain) !void {
        if (empty(self.library_dir)) return error.MissingCudaB200LibraryDirectory;
        if (empty(self.runtime_dir)) return error.MissingCudaRuntimeDirectory;
    }
};

pub fn linkRuntime(artifact: *std.Build.Step.Compile, toolchain: Toolchain) void {
    toolchain.validate() catch |err| std.debug.panic("invalid B200 CUDA toolchain: {s}", .{@errorName(err)});
    artifact.addLibraryPath(.{ .cwd_relative = toolchain.library_dir.? });
    artifact.addLibraryPath(.{ .cwd_relative = toolchain.runtime_dir.? });
    artifact.addRPath(.{ .cwd_relative = toolchain.library_dir.? });
    if (toolchain.include_dir) |dir| artifact.addIncludePath(.{ .cwd_relative = dir });
    artifact.linkSystemLibrary("stwo_b200");
    artifact.linkSystemLibrary("cudart");
    artifact.linkSystemLibrary("stdc++");
    artifact.linkLibC();
}

fn empty(value: ?[]const u8) bool {
    return value == null or value.?.len == 0;
}

test "B200 toolchain has no implicit local paths" {
    try std.testing.expectError(error.MissingCudaB200LibraryDirectory, (Toolchain{}).validate());
    try std.testing.expectError(
        error.MissingCudaRuntimeDirectory,
        (Toolchain{ .library_dir = "/explicit/stwo_b200/lib" }).validate(),
    );
    try (Toolchain{ .library_dir = "/explicit/stwo_b200/lib", .runtime_dir = "/explicit/cuda/lib64" }).validate();
}
