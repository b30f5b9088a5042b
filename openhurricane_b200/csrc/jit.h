// Run-time generated, mechanism-specialised kernels (jit.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rtc_base.cuh"

namespace hc {

// host copy of the mechanism tables in the device order (reactions regrouped
// by rate class, as uploaded to DevMech)
struct HostMech {
    int nsp = 0, nrc = 0;
    std::vector<double> W, Trange, nasa;
    std::vector<int32_t> rate_type, reversible, nf, nb, fidx, bidx;
    std::vector<double> arr, arr0, troe, eff, fnu, bnu, ford, bord, sum_stoi;
    std::vector<double> sri, arr_rev;
    std::vector<int32_t> activated;        // [nrc] chemically activated bimolecular
    std::vector<double> lt;                // [nrc*2] Landau-Teller B, C
    std::vector<double> xcoef;             // [nrc*9] Janev / power-series coefficients
    std::vector<int32_t> plog_ptr;         // [nrc+1], in device reaction order
    std::vector<double> plog_p, plog_arr;
    // device reaction r is reaction perm[r] of the mechanism as given
    std::vector<int32_t> perm;
    // the mechanism uses rate forms only the cell-group kernels evaluate
    // (SRI fall-off, explicit reverse parameters, PLOG tables, chemically
    // activated and Landau-Teller rates)
    bool ext = false;
};

struct JitKernel {
    void *module = nullptr;   // CUmodule
    void *func = nullptr;     // CUfunction
    int N = 0, block = 0;
    size_t smem = 0;
    int per_sm = 0;
};

std::string jit_t1_source(const HostMech &h, int block);
// the compact thread-per-cell kernel (kernel 5, jit_t3.cu, t4_cell.cuh) and
// its shared memory per thread in doubles
std::string jit_t3_source(const HostMech &h, int block);
int t3_slots(int nsp);
// NVRTC compile of generated source to an sm_100a cubin (host only)
int jit_compile(const std::string &src, std::vector<char> &cubin, std::string &err);
// compile (NVRTC, sm_100a) and load the thread-per-cell kernel for h;
// modules are cached per source text for the life of the process
int jit_build_t1(const HostMech &h, int block, JitKernel *out, std::string &err);
// the same for the compact kernel (kernel 5)
int jit_build_t3(const HostMech &h, int block, JitKernel *out, std::string &err);
int jit_launch_t1(const JitKernel &k, int num_sms, const IntegratorParams &P, const CellIO &io,
                  double *ylast, cudaStream_t st, std::string &err);

}  // namespace hc
