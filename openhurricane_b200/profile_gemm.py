"""The surrogate's BF16 tensor-core GEMM on its own, for timing and ncu.

    python -m openhurricane_b200.profile_gemm M N K

C[M][N] = A[M][K] B[N][K]^T (bf16 in, fp32 out, tcgen05 + TMA); three
untimed launches, then ten timed with CUDA events; prints one JSON line
with the median time and TFLOP/s (2 M N K per launch).
"""
import json
import sys

import torch

from .surrogate import gemm_bf16


def main(argv):
    M, N, K = (int(x) for x in (argv + ["8192", "256", "256"][len(argv):])[:3])
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    for _ in range(3):
        gemm_bf16(A, B)
    st = torch.cuda.current_stream()
    times = []
    for _ in range(10):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        gemm_bf16(A, B)
        b.record(st)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms = sorted(times)[len(times) // 2]
    print(json.dumps({"M": M, "N": N, "K": K, "ms": ms, "TFLOPs": 2.0 * M * N * K / (ms * 1e-3) / 1e12}))


if __name__ == "__main__":
    main(sys.argv[1:])
