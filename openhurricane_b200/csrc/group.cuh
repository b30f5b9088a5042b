// Cooperative "cell group": G lanes (half a warp for G = 16, one warp for
// G = 32, two warps for G = 64) that integrate one cell together, lane i
// owning row i of the Newton matrix and element i of every state vector.
// Two 16-lane groups share a warp and run independently: their shuffles and
// warp barriers use the group's half-warp mask.
//
// All reductions return bit-identical results in every lane of the group
// (xor-butterfly within a warp; the two warp partials are combined in a
// fixed order), so control flow driven by reduced values stays uniform
// across the group and every barrier is reached by all of its lanes.
#pragma once

#include <cuda_runtime.h>

namespace hc {

template <int G>
struct Group {
    static_assert(G == 16 || G == 32 || G == 64, "cell group is half a warp, one or two warps");
    static constexpr int GW = G < 32 ? G : 32;   // lanes of the group within one warp
    int lane;    // 0 .. G-1
    int wlane;   // lane within the group's part of its warp (0 .. GW-1)
    int warp;    // warp within the group
    int barid;   // named barrier (G == 64)
    int base;    // first lane of the group within its warp (G == 16: 0 or 16)
    unsigned mask;   // the group's lanes within its warp
    double *red; // [4] cross-warp scratch
    int *redi;   // [4]

    __device__ __forceinline__ void sync() const {
        if (G <= 32) {
            __syncwarp(mask);
        } else {
            asm volatile("bar.sync %0, %1;" ::"r"(barid), "r"(64) : "memory");
        }
    }

    __device__ __forceinline__ double sum(double v) const {
#pragma unroll
        for (int o = GW / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        if (G == 64) {
            if (wlane == 0) red[warp] = v;
            sync();
            v = red[0] + red[1];
            sync();
        }
        return v;
    }

    __device__ __forceinline__ double max(double v) const {
#pragma unroll
        for (int o = GW / 2; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(mask, v, o);
            v = (v < w) ? w : v;
        }
        if (G == 64) {
            if (wlane == 0) red[warp] = v;
            sync();
            v = (red[0] < red[1]) ? red[1] : red[0];
            sync();
        }
        return v;
    }

    __device__ __forceinline__ int min_int(int v) const {
#pragma unroll
        for (int o = GW / 2; o > 0; o >>= 1) v = ::min(v, __shfl_xor_sync(mask, v, o));
        if (G == 64) {
            if (wlane == 0) redi[warp] = v;
            sync();
            v = ::min(redi[0], redi[1]);
            sync();
        }
        return v;
    }

    // index of the largest v (ties -> smallest index); v < 0 marks "not a candidate"
    __device__ __forceinline__ int argmax(double v) const {
        int idx = lane;
#pragma unroll
        for (int o = GW / 2; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(mask, v, o);
            const int j = __shfl_xor_sync(mask, idx, o);
            if (w > v || (w == v && j < idx)) {
                v = w;
                idx = j;
            }
        }
        if (G == 64) {
            if (wlane == 0) {
                red[warp] = v;
                redi[warp] = idx;
            }
            sync();
            const double v0 = red[0], v1 = red[1];
            const int i0 = redi[0], i1 = redi[1];
            idx = (v1 > v0) ? i1 : i0;
            sync();
        }
        return idx;
    }

    __device__ __forceinline__ bool any(bool b) const { return min_int(b ? 0 : 1) == 0; }
};

}  // namespace hc
