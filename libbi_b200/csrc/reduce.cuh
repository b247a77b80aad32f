// Block-then-grid log-sum-exp + ESS reduction: the device functions live in
// the public header include/bpf_device.cuh, which kernels compiled outside
// the library (a model's own fused transition) use as well.
#pragma once
#include "internal.cuh"
#include "../../include/bpf_device.cuh"
