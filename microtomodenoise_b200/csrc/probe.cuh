#pragma once
namespace inlm {
// FP32 FMA throughput (TFLOP/s, 2 flops per FFMA) of the device, best of 5.
int probe_fp32_fma(int device, double* tflops);
}
