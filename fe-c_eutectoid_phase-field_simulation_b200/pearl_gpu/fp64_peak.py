"""FP64 throughput of this GPU: independent FMA chains in every thread of a
full grid, timed with CUDA events.  Reports TFLOP/s (an FMA counts 2).

    python -m pearl_gpu.fp64_peak

Compiles a small kernel with nvcc at run time (the GPU machines carry the same
toolkit).  Used as the FP64 roofline of the compute-bound phases (PROPOSE,
FINAL), since the measured peaks file lists only memory and bf16 figures."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

SRC = r"""
#include <cuda_runtime.h>
__global__ void fma_chains(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
extern "C" double fp64_tflops(int device) {
    cudaSetDevice(device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return -1;
    fma_chains<<<blocks, threads>>>(out, 16, 0.999999, 1e-7);  // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    fma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return -1;
    return 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
}
"""


def measure(device: int = 0) -> float:
    nvcc = os.environ.get("NVCC", "nvcc")
    with tempfile.TemporaryDirectory() as tmp:
        src = Path(tmp) / "fp64_peak.cu"
        lib = Path(tmp) / "fp64_peak.so"
        src.write_text(SRC)
        subprocess.run([nvcc, "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
                        str(src), "-o", str(lib)], check=True)
        L = C.CDLL(str(lib))
        L.fp64_tflops.restype = C.c_double
        L.fp64_tflops.argtypes = [C.c_int]
        return max(L.fp64_tflops(device) for _ in range(3))


if __name__ == "__main__":
    print(f"fp64_tflops: {measure():.2f}")
