//! Native + B200 CUDA product descriptor: replaces the unavailable experimental descriptor of
//! build_support/products/native_cuda.zig:5-19 with the parity-gated libstwo_b200 backend.

const policy = @import("../graph/product.zig");

pub const descriptor = policy.Descriptor{
    .product = .{
        .name = "stwo-native-cuda-b200",
        .frontend = .native,
        .backend = .cuda,
        .role = .cli,
        .protocol_features = "native-examples-v1+cuda-b200-sm100a",
    },
    .state = .experimental,
    .target_support = .any,
    .unavailable_reason = null,
    .build_step = "stwo-native-cuda-b200",
    .test_step = null,
    .executable = null,
};
