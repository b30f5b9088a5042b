// C ABI of libhurchem_b200.so (declared in include/hurchem_b200.h).
//
// Host side of the drop-in boundary: uploads a flattened mechanism, picks
// the compiled kernel variant for its size, and launches the integrators,
// the right-hand-side/Jacobian evaluator, the source-term and the property
// kernels. No entry point aborts; errors are returned as status codes with a
// message in hc_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/hurchem_b200.h"
#include "integrator_t2.cuh"
#include "jit.h"
#include "surrogate.cuh"
#include "variants.h"
#include "wcell.cuh"

using namespace hc;


namespace {

thread_local std::string g_err;

}  // namespace

namespace hc {
// the message hc_last_error() returns, shared by every translation unit
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace hc

namespace {

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define HC_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(HC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int upload(std::vector<void *> &owned, const T *src, size_t n, const T **dst) {
    if (n == 0) {
        *dst = nullptr;
        return HC_OK;
    }
    void *d = nullptr;
    HC_CUDA(cudaMalloc(&d, n * sizeof(T)));
    owned.push_back(d);
    HC_CUDA(cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice));
    *dst = static_cast<const T *>(d);
    return HC_OK;
}

enum Variant { kV10 = 0, kV16, kV32, kV54, kV64 };

}  // namespace

struct hc_mech_s {
    DevMech dm{};
    int variant = -1;
    std::vector<void *> owned;
    // reusable device workspace for the host-buffer entry points
    std::mutex mu;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    unsigned long long *queue = nullptr;   // [1 + 6] queue head, counters
    int num_sms = 0;
    // thread-per-cell integrator: per-cell buffer for the two previous step
    // states (ImplicitEuler's yklast_), grown on demand
    double *ylast = nullptr;
    size_t ylast_cells = 0;
    // kernel choice (hc_set_tuning): 0 automatic, 1 thread per cell, 2 cell
    // group, 3 mechanism-specialised thread per cell (generated, NVRTC)
    int kernel = 0;
    int block = 64;
    // host tables in device order, for the generated kernels
    HostMech host;
    // the mechanism in the compact thread-per-cell kernel's parameter form
    T2Mech t2{};
    bool t2_ok = false;
    JitKernel jit;
    bool jit_tried = false;
    std::string jit_err;
    // the compact thread-per-cell kernel (kernel 5, generated)
    JitKernel jit5;
    bool jit5_tried = false;
    std::string jit5_err;
    // the warp-per-cell kernel's tables (kernel 6)
    WMech w{};
    bool w_ok = false;
};

namespace {

int variant_for(int N) {
    if (N == 10) return kV10;
    if (N <= 16) return kV16;
    if (N <= 32) return kV32;
    if (N == 54) return kV54;
    if (N <= 64) return kV64;
    return -1;
}

#define HC_DISPATCH(m, FN, ...)                                        \
    switch ((m)->variant) {                                            \
    case kV10: return variant_##FN##_10(__VA_ARGS__);                  \
    case kV16: return variant_##FN##_16(__VA_ARGS__);                  \
    case kV32: return variant_##FN##_32(__VA_ARGS__);                  \
    case kV54: return variant_##FN##_54(__VA_ARGS__);                  \
    case kV64: return variant_##FN##_64(__VA_ARGS__);                  \
    default: return fail(HC_E_UNSUPPORTED, "no kernel variant");       \
    }

IntegratorParams make_params(const hc_opts *o) {
    IntegratorParams P;
    P.maxstep = o->maxstep;
    P.auto_update_jacobian = o->auto_update_jacobian;
    P.step_to_update_jac = o->step_to_update_jac;
    P.atol = o->atol;
    P.rtol = o->rtol;
    P.safescale = o->safescale;
    P.minscale = o->minscale;
    P.maxscale = o->maxscale;
    P.alphainc = o->alphainc;
    P.atol_inc = o->atol_increment;
    P.rtol_inc = o->rtol_increment;
    P.T_threshold = o->T_threshold;
    P.T_alpha = o->T_alpha;
    P.T_beta = o->T_beta;
    P.dt_max = o->dt_max;
    // evaluated with the host libm, as the reference does at run time (ImplicitEuler.cpp:287)
    P.err_accept_limit = std::pow(o->maxscale / o->safescale, -1.0 / o->alphainc);
    P.max_newton_total = o->max_newton_total;
    P.reactor = o->reactor;
    return P;
}

int check_opts(const hc_opts *o) {
    if (!o) return fail(HC_E_INVALID, "opts is null");
    if (o->reactor != 0 && o->reactor != 1)
        return fail(HC_E_INVALID, "reactor must be 0 (constant pressure) or 1 (constant volume)");
    if (o->maxstep <= 0 || o->step_to_update_jac <= 0)
        return fail(HC_E_INVALID, "maxstep and step_to_update_jac must be positive");
    if (!(o->alphainc > 0) || !(o->safescale > 0))
        return fail(HC_E_INVALID, "alphainc and safescale must be positive");
    return HC_OK;
}

}  // namespace

// Host copy of the tables in device order. Reactions are regrouped by rate
// law (plain Arrhenius, third-body, fall-off), stable within a group, so that
// the lanes of a cell group evaluating one chunk of reactions mostly follow
// the same code path. Source terms are sums over reactions; only their
// summation order changes.
static void make_host(const hc_mech_desc *d, HostMech &h) {
    const int nsp = d->nsp, nrc = d->nrc;
    std::vector<int> perm(nrc);
    for (int r = 0; r < nrc; ++r) perm[r] = r;
    auto cls = [&](int r) { return d->rate_type[r] >= HC_RATE_LINDEMANN ? 2 : d->rate_type[r]; };
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return cls(a) < cls(b); });
    auto permute = [&](const auto *src, int width) {
        using V = std::remove_const_t<std::remove_pointer_t<decltype(src)>>;
        std::vector<V> outv((size_t)nrc * width);
        for (int r = 0; r < nrc; ++r)
            for (int k = 0; k < width; ++k)
                outv[(size_t)r * width + k] = src[(size_t)perm[r] * width + k];
        return outv;
    };
    h.nsp = nsp;
    h.nrc = nrc;
    h.perm.assign(perm.begin(), perm.end());
    h.W.assign(d->W, d->W + nsp);
    h.Trange.assign(d->Trange, d->Trange + 3 * (size_t)nsp);
    h.nasa.assign(d->nasa, d->nasa + 14 * (size_t)nsp);
    h.rate_type = permute(d->rate_type, 1);
    h.reversible = permute(d->reversible, 1);
    h.arr = permute(d->arr, 3);
    h.arr0 = permute(d->arr0, 3);
    h.troe = permute(d->troe, 4);
    h.eff = permute(d->eff, nsp);
    h.nf = permute(d->nf, 1);
    h.nb = permute(d->nb, 1);
    h.fidx = permute(d->fidx, HC_MAX_SIDE);
    h.bidx = permute(d->bidx, HC_MAX_SIDE);
    h.fnu = permute(d->fnu, HC_MAX_SIDE);
    h.bnu = permute(d->bnu, HC_MAX_SIDE);
    h.ford = permute(d->ford, HC_MAX_SIDE);
    h.bord = permute(d->bord, HC_MAX_SIDE);
    const std::vector<double> zeros5((size_t)nrc * 5, 0.0), zeros3((size_t)nrc * 3, 0.0);
    h.sri = permute(d->sri ? d->sri : zeros5.data(), 5);
    h.arr_rev = permute(d->arr_rev ? d->arr_rev : zeros3.data(), 3);
    const std::vector<int32_t> zeros1i((size_t)nrc, 0);
    const std::vector<double> zeros2((size_t)nrc * 2, 0.0);
    h.activated = permute(d->activated ? d->activated : zeros1i.data(), 1);
    h.lt = permute(d->lt ? d->lt : zeros2.data(), 2);
    const std::vector<double> zeros9((size_t)nrc * 9, 0.0);
    h.xcoef = permute(d->xcoef ? d->xcoef : zeros9.data(), 9);
    h.ext = false;
    for (int r = 0; r < nrc; ++r)
        if (d->rate_type[r] >= HC_RATE_SRI || d->reversible[r] == HC_REVERSIBLE_REV ||
            (d->activated && d->activated[r]))
            h.ext = true;
    // PLOG tables follow their reactions into device order
    h.plog_ptr.assign((size_t)nrc + 1, 0);
    h.plog_p.clear();
    h.plog_arr.clear();
    for (int r = 0; r < nrc; ++r) {
        const int src = perm[r];
        if (d->plog_ptr && d->rate_type[src] == HC_RATE_PLOG) {
            for (int k = d->plog_ptr[src]; k < d->plog_ptr[src + 1]; ++k) {
                h.plog_p.push_back(d->plog_p[k]);
                for (int j = 0; j < 3; ++j) h.plog_arr.push_back(d->plog_arr[3 * (size_t)k + j]);
            }
        }
        h.plog_ptr[r + 1] = (int32_t)h.plog_p.size();
    }
    h.sum_stoi.assign(nrc, 0.0);
    for (int r = 0; r < nrc; ++r) {
        double s = 0.0;
        for (int k = 0; k < h.nf[r]; ++k) s -= h.fnu[HC_MAX_SIDE * r + k];
        for (int k = 0; k < h.nb[r]; ++k) s += h.bnu[HC_MAX_SIDE * r + k];
        h.sum_stoi[r] = s;
    }
}

// the mechanism in T2Mech form, if it fits the compact kernel's tables
static bool pack_t2(const HostMech &h, const hc_mech_desc *d, T2Mech &t) {
    if (h.nsp > kT2MaxSp || h.nrc > kT2MaxRxn || h.ext) return false;
    std::memset(&t, 0, sizeof(t));
    t.nsp = h.nsp;
    t.nrc = h.nrc;
    for (int i = 0; i < h.nsp; ++i) {
        t.W[i] = h.W[i];
        for (int k = 0; k < 3; ++k) t.thermo[i][k] = h.Trange[3 * i + k];
        for (int k = 0; k < 14; ++k) t.thermo[i][3 + k] = h.nasa[14 * i + k];
    }
    int ne = 0;
    for (int r = 0; r < h.nrc; ++r) {
        T2Rxn &R = t.rxn[r];
        R.A = h.arr[3 * r];
        R.b = h.arr[3 * r + 1];
        R.Ta = h.arr[3 * r + 2];
        R.A0 = h.arr0[3 * r];
        R.b0 = h.arr0[3 * r + 1];
        R.Ta0 = h.arr0[3 * r + 2];
        for (int k = 0; k < 4; ++k) R.troe[k] = h.troe[4 * r + k];
        for (int k = 0; k < HC_MAX_SIDE; ++k) {
            R.fnu[k] = h.fnu[HC_MAX_SIDE * r + k];
            R.bnu[k] = h.bnu[HC_MAX_SIDE * r + k];
            R.ford[k] = h.ford[HC_MAX_SIDE * r + k];
            R.bord[k] = h.bord[HC_MAX_SIDE * r + k];
            R.fidx[k] = (int8_t)h.fidx[HC_MAX_SIDE * r + k];
            R.bidx[k] = (int8_t)h.bidx[HC_MAX_SIDE * r + k];
        }
        R.sum_stoi = h.sum_stoi[r];
        R.type = (int8_t)h.rate_type[r];
        R.rev = (int8_t)(h.reversible[r] != 0);
        R.nf = (int8_t)h.nf[r];
        R.nb = (int8_t)h.nb[r];
        R.eff_begin = (int16_t)ne;
        if (h.rate_type[r] != HC_RATE_ARRHENIUS) {
            for (int i = 0; i < h.nsp; ++i) {
                const double e = h.eff[(size_t)r * h.nsp + i];
                if (e == 0.0) continue;
                if (ne >= kT2MaxEff) return false;
                t.eff_val[ne] = e;
                t.eff_idx[ne] = (int8_t)i;
                ++ne;
            }
        }
        R.eff_end = (int16_t)ne;
    }
    (void)d;
    return true;
}

// The mechanism in the warp- and segment-per-cell kernels' tables
// (wcell.cuh, scell.cuh): species NASA-7 pre-multiplied by W and the
// polynomial factors; reactions in table slots grouped by rate form (plain
// Arrhenius, third body, fall-off; mechanism order within each group), so
// that the lanes evaluating one round of slots mostly take the same branch;
// each species' participation list in the mechanism's own order (the order
// the reference sums f and J in), naming slots; the third-body / fall-off
// reactions in mechanism order.
struct WHost {
    std::vector<double> th, rd, eff, raw, lnu, xj;
    std::vector<int32_t> ri, lptr, lent, tbl;
    int nsp = 0, nrc = 0, nrc32 = 0, njob = 0, njob32 = 0;
    double glim = 0.0;
};

static bool pack_w(const HostMech &h, WHost &w) {
    if (h.nsp + 1 > 16 || h.ext) return false;
    const int nsp = h.nsp, nrc = h.nrc, S = HC_MAX_SIDE;
    w.nsp = nsp;
    w.nrc = nrc;
    w.nrc32 = std::max(32, ((nrc + 31) / 32) * 32);
    const int n32 = w.nrc32;
    w.th.assign((size_t)kWTHn * 32, 0.0);
    auto T = [&](int f, int i) -> double & { return w.th[(size_t)f * 32 + i]; };
    for (int i = 0; i < nsp; ++i) {
        const double W = h.W[i];
        T(kWtl, i) = h.Trange[3 * i];
        T(kWtc, i) = h.Trange[3 * i + 1];
        T(kWth, i) = h.Trange[3 * i + 2];
        T(kWW, i) = W;
        for (int rg = 0; rg < 2; ++rg) {
            const double *a = &h.nasa[14 * i + 7 * rg];
            const int b = kWrange + rg * kWRangeN;
            for (int k = 0; k < 5; ++k) T(b + k, i) = W * a[k] / (k + 1);
            T(b + 5, i) = W * a[5];
            T(b + 6, i) = W * a[0];
            for (int k = 1; k < 5; ++k) T(b + 6 + k, i) = W * a[k] / k;
            T(b + 11, i) = W * a[6];
            for (int k = 0; k < 5; ++k) T(b + 12 + k, i) = W * a[k];
            for (int k = 1; k < 5; ++k) T(b + 16 + k, i) = k * W * a[k];
        }
    }
    std::vector<int> dev(nrc);   // mechanism order -> device order
    for (int r = 0; r < nrc; ++r) dev[((int)h.perm.size() == nrc) ? h.perm[r] : r] = r;
    std::vector<int> slot(nrc);  // mechanism order -> table slot
    {
        auto cls = [&](int o) {
            const int t = h.rate_type[dev[o]];
            return (t == HC_RATE_ARRHENIUS) ? 0 : (t == HC_RATE_THIRD_BODY) ? 1 : 2;
        };
        int q = 0;
        for (int c = 0; c < 3; ++c)
            for (int o = 0; o < nrc; ++o)
                if (cls(o) == c) slot[o] = q++;
    }
    w.rd.assign((size_t)kWRDn * n32, 0.0);
    w.ri.assign((size_t)kWRIn * n32, 0);
    w.eff.assign((size_t)std::max(nrc, 1) * nsp, 0.0);
    double worst = 1.0;
    for (int o = 0; o < nrc; ++o) {
        const int r = dev[o], q = slot[o];
        const int type = h.rate_type[r], nf = h.nf[r], nb = h.nb[r];
        if (nf + nb > 8) return false;
        // round-major: [round][field][32]
        auto RI = [&](int f) -> int32_t & { return w.ri[((size_t)(q >> 5) * kWRIn + f) * 32 + (q & 31)]; };
        auto RD = [&](int f) -> double & { return w.rd[((size_t)(q >> 5) * kWRDn + f) * 32 + (q & 31)]; };
        RI(kWtype) = type;
        RI(kWrev) = h.reversible[r] ? 1 : 0;
        RI(kWnf) = nf;
        RI(kWnb) = nb;
        RD(kWA) = h.arr[3 * r];
        RD(kWb) = h.arr[3 * r + 1];
        RD(kWTa) = h.arr[3 * r + 2];
        RD(kWA0) = h.arr0[3 * r];
        RD(kWb0) = h.arr0[3 * r + 1];
        RD(kWTa0) = h.arr0[3 * r + 2];
        if (type == HC_RATE_TROE3 || type == HC_RATE_TROE4) {
            RD(kWalpha) = h.troe[4 * r];
            RD(kWTsss) = h.troe[4 * r + 1];
            RD(kWTs) = h.troe[4 * r + 2];
            RD(kWiTsss) = 1.0 / h.troe[4 * r + 1];
            RD(kWiTs) = 1.0 / h.troe[4 * r + 2];
            RD(kWTss) = h.troe[4 * r + 3];
        }
        RD(kWs) = h.sum_stoi[r];
        double sn = 0.0;
        for (int k = 0; k < nf; ++k) {
            RI(kWidx + k) = h.fidx[S * r + k];
            RD(kWnu + k) = -h.fnu[S * r + k];
            RD(kWord + k) = h.ford[S * r + k];
            sn += std::fabs(h.fnu[S * r + k]);
        }
        for (int k = 0; k < nb; ++k) {
            RI(kWidx + nf + k) = h.bidx[S * r + k];
            RD(kWnu + nf + k) = h.bnu[S * r + k];
            RD(kWord + nf + k) = h.bord[S * r + k];
            sn += std::fabs(h.bnu[S * r + k]);
        }
        for (int k = nf + nb; k < 8; ++k) RD(kWord + k) = 1.0;
        if (h.reversible[r]) worst = std::max(worst, sn);
        if (type != HC_RATE_ARRHENIUS) {
            for (int i = 0; i < nsp; ++i) w.eff[(size_t)q * nsp + i] = h.eff[(size_t)r * nsp + i];
            w.tbl.push_back(q);
        }
    }
    // participation lists: per entry the reaction, the species' position
    // among its participants, their number, a third-body flag, the
    // participants' columns (8 bits each) and the species' signed coefficient
    // exponential jobs: each reaction's Arrhenius factor, then the fall-off
    // reactions' low-pressure factor and Troe centering terms
    {
        std::vector<std::array<double, 3>> jobs(nrc);
        for (int o = 0; o < nrc; ++o) {
            const int r = dev[o];
            jobs[slot[o]] = {h.arr[3 * r + 1], -h.arr[3 * r + 2], 0.0};
        }
        for (int o = 0; o < nrc; ++o) {
            const int r = dev[o], type = h.rate_type[r], q = slot[o];
            if (type < HC_RATE_LINDEMANN) continue;
            w.ri[((size_t)(q >> 5) * kWRIn + kWxj) * 32 + (q & 31)] = (int32_t)jobs.size();
            jobs.push_back({h.arr0[3 * r + 1], -h.arr0[3 * r + 2], 0.0});
            if (type == HC_RATE_TROE3 || type == HC_RATE_TROE4) {
                jobs.push_back({0.0, 0.0, -1.0 / h.troe[4 * r + 1]});
                jobs.push_back({0.0, 0.0, -1.0 / h.troe[4 * r + 2]});
                if (type == HC_RATE_TROE4) jobs.push_back({0.0, -h.troe[4 * r + 3], 0.0});
            }
        }
        w.njob = (int)jobs.size();
        w.njob32 = std::max(32, ((w.njob + 31) / 32) * 32);
        w.xj.assign((size_t)3 * w.njob32, 0.0);
        for (int j = 0; j < w.njob; ++j)
            for (int f = 0; f < 3; ++f) w.xj[((size_t)(j >> 5) * 3 + f) * 32 + (j & 31)] = jobs[j][f];
    }
    w.lptr.assign(nsp + 1, 0);
    w.lent.clear();
    w.lnu.clear();
    for (int i = 0; i < nsp; ++i) {
        w.lptr[i] = (int32_t)w.lnu.size();
        for (int o = 0; o < nrc; ++o) {
            const int q = slot[o];
            auto RI = [&](int f) { return w.ri[((size_t)(q >> 5) * kWRIn + f) * 32 + (q & 31)]; };
            auto RD = [&](int f) { return w.rd[((size_t)(q >> 5) * kWRDn + f) * 32 + (q & 31)]; };
            const int np = RI(kWnf) + RI(kWnb);
            uint32_t c[2] = {0u, 0u};
            for (int k = 0; k < np; ++k) c[k >> 2] |= (uint32_t)RI(kWidx + k) << (8 * (k & 3));
            for (int k = 0; k < np; ++k) {
                if (RI(kWidx + k) != i) continue;
                w.lent.push_back(q | (k << 16) | (np << 20) | ((RI(kWtype) != HC_RATE_ARRHENIUS) ? (1 << 24) : 0));
                w.lent.push_back((int32_t)c[0]);
                w.lent.push_back((int32_t)c[1]);
                w.lnu.push_back(RD(kWnu + k));
            }
        }
    }
    w.lptr[nsp] = (int32_t)w.lnu.size();
    if (w.lnu.empty()) {
        w.lent.assign(3, 0);
        w.lnu.push_back(0.0);
    }
    if (nrc >= (1 << 16)) return false;
    if (w.tbl.empty()) w.tbl.push_back(0);
    w.raw.assign(h.nasa.begin(), h.nasa.end());
    w.glim = std::min(300.0, 580.0 / worst);
    return true;
}

static int check_desc(const hc_mech_desc *d) {
    const int nsp = d->nsp, nrc = d->nrc;
    if (nsp < 1 || nrc < 0) return fail(HC_E_INVALID, "bad mechanism size");
    if (!d->W || !d->Trange || !d->nasa || (nrc > 0 && (!d->rate_type || !d->reversible ||
        !d->arr || !d->arr0 || !d->troe || !d->eff || !d->nf || !d->nb || !d->fidx ||
        !d->bidx || !d->fnu || !d->bnu || !d->ford || !d->bord)))
        return fail(HC_E_INVALID, "null table in mechanism");
    for (int r = 0; r < nrc; ++r) {
        if (d->nf[r] < 0 || d->nf[r] > HC_MAX_SIDE || d->nb[r] < 0 || d->nb[r] > HC_MAX_SIDE)
            return fail(HC_E_INVALID, "reaction side larger than HC_MAX_SIDE");
        if (d->rate_type[r] < 0 || d->rate_type[r] > HC_RATE_COLLISION)
            return fail(HC_E_INVALID, "unknown rate type");
        if (d->rate_type[r] >= HC_RATE_JANEV) {
            if (!d->xcoef)
                return fail(HC_E_INVALID, "Janev / power-series / collision reaction without coefficients");
            if (d->reversible[r] == HC_REVERSIBLE_REV)
                return fail(HC_E_INVALID,
                            "explicit reverse parameters on a Janev / power-series / collision reaction");
        }
        if (d->activated && d->activated[r] &&
            (d->rate_type[r] < HC_RATE_LINDEMANN || d->rate_type[r] > HC_RATE_SRI))
            return fail(HC_E_INVALID, "chemically activated reaction without a fall-off form");
        if (d->rate_type[r] == HC_RATE_LANDAU_TELLER) {
            if (!d->lt) return fail(HC_E_INVALID, "Landau-Teller reaction without its B, C");
            if (d->reversible[r] == HC_REVERSIBLE_REV && !d->xcoef)
                return fail(HC_E_INVALID,
                            "Landau-Teller reaction with REV parameters but no reverse B, C");
        }
        if (d->reversible[r] < HC_IRREVERSIBLE || d->reversible[r] > HC_REVERSIBLE_REV)
            return fail(HC_E_INVALID, "unknown reversibility code");
        if (d->rate_type[r] == HC_RATE_SRI && !d->sri)
            return fail(HC_E_INVALID, "SRI reaction without SRI parameters");
        if (d->rate_type[r] == HC_RATE_PLOG) {
            if (!d->plog_ptr || !d->plog_p || !d->plog_arr)
                return fail(HC_E_INVALID, "PLOG reaction without PLOG tables");
            const int b = d->plog_ptr[r], e = d->plog_ptr[r + 1];
            if (b < 0 || e <= b) return fail(HC_E_INVALID, "PLOG reaction with an empty table");
            for (int k = b; k < e; ++k) {
                if (!(d->plog_p[k] > 0)) return fail(HC_E_INVALID, "PLOG pressure not positive");
                if (k > b && d->plog_p[k] < d->plog_p[k - 1])
                    return fail(HC_E_INVALID, "PLOG pressures not sorted");
            }
            // logInterpolationRR::DkDT reads past its list for a repeated
            // highest pressure (logInterpolationRR.cpp:170-179)
            if (e - b > 1 && d->plog_p[e - 1] == d->plog_p[e - 2])
                return fail(HC_E_INVALID, "PLOG table with its highest pressure twice");
            if (d->reversible[r] == HC_REVERSIBLE_REV)
                return fail(HC_E_INVALID, "explicit reverse parameters on a PLOG reaction");
        }
        if (d->reversible[r] == HC_REVERSIBLE_REV) {
            if (!d->arr_rev) return fail(HC_E_INVALID, "REV reaction without reverse parameters");
            // reversibleReactionWithRevPars takes Arrhenius, third-body and, with
            // the reverse B, C of RLT, Landau-Teller rates (chemkinFileRead.cpp:1387-1444,
            // 1502-1516)
            if (d->rate_type[r] != HC_RATE_ARRHENIUS && d->rate_type[r] != HC_RATE_THIRD_BODY &&
                d->rate_type[r] != HC_RATE_LANDAU_TELLER)
                return fail(HC_E_INVALID,
                            "explicit reverse parameters on a fall-off or PLOG reaction");
        }
        for (int k = 0; k < d->nf[r]; ++k)
            if (d->fidx[HC_MAX_SIDE * r + k] < 0 || d->fidx[HC_MAX_SIDE * r + k] >= nsp)
                return fail(HC_E_INVALID, "species index out of range");
        for (int k = 0; k < d->nb[r]; ++k)
            if (d->bidx[HC_MAX_SIDE * r + k] < 0 || d->bidx[HC_MAX_SIDE * r + k] >= nsp)
                return fail(HC_E_INVALID, "species index out of range");
    }
    return HC_OK;
}

extern "C" {

int hc_abi_version(void) { return HC_ABI_VERSION; }

const char *hc_last_error(void) { return g_err.c_str(); }

void hc_default_opts(hc_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->maxstep = 10000;
    o->auto_update_jacobian = 0;
    o->step_to_update_jac = 10;
    o->reactor = 0;
    o->atol = 1e-15;
    o->rtol = 1e-4;
    o->safescale = 0.8;
    o->minscale = 0.25;
    o->maxscale = 2.0;
    o->alphainc = 0.25;
    o->atol_increment = 1e-7;
    o->rtol_increment = 1e-3;
    o->T_threshold = 200.0;
    o->T_alpha = 0.2;
    o->T_beta = 0.25;
    o->dt_max = 1e15;
    o->max_newton_total = 20000000;
}

int hc_mech_create(const hc_mech_desc *d, hc_mech_t *out) {
    if (!d || !out) return fail(HC_E_INVALID, "null argument");
    *out = nullptr;
    const int nsp = d->nsp, nrc = d->nrc;
    {
        const int vrc = check_desc(d);
        if (vrc != HC_OK) return vrc;
    }
    const int variant = variant_for(nsp + 1);
    if (variant < 0)
        return fail(HC_E_UNSUPPORTED, "mechanisms with more than 63 species are not built");
    HostMech hm;
    make_host(d, hm);
    const auto &p_type = hm.rate_type, &p_rev = hm.reversible;
    const auto &p_arr = hm.arr, &p_arr0 = hm.arr0, &p_troe = hm.troe, &p_eff = hm.eff;
    const auto &p_nf = hm.nf, &p_nb = hm.nb, &p_fidx = hm.fidx, &p_bidx = hm.bidx;
    const auto &p_fnu = hm.fnu, &p_bnu = hm.bnu, &p_ford = hm.ford, &p_bord = hm.bord;
    // participation lists per species, in (regrouped) reaction order:
    // coef = -nu' (reactant) / +nu'' (product)
    std::vector<std::vector<std::pair<int, double>>> part(nsp);
    const std::vector<double> &sum_stoi = hm.sum_stoi;
    for (int r = 0; r < nrc; ++r) {
        for (int k = 0; k < p_nf[r]; ++k)
            part[p_fidx[HC_MAX_SIDE * r + k]].push_back({r, -p_fnu[HC_MAX_SIDE * r + k]});
        for (int k = 0; k < p_nb[r]; ++k)
            part[p_bidx[HC_MAX_SIDE * r + k]].push_back({r, p_bnu[HC_MAX_SIDE * r + k]});
    }
    std::vector<int32_t> sp_ptr(nsp + 1, 0), sp_rxn;
    std::vector<double> sp_coef;
    for (int i = 0; i < nsp; ++i) {
        sp_ptr[i] = (int32_t)sp_rxn.size();
        for (auto &pr : part[i]) {
            sp_rxn.push_back(pr.first);
            sp_coef.push_back(pr.second);
        }
    }
    sp_ptr[nsp] = (int32_t)sp_rxn.size();

    hc_mech_s *m = new hc_mech_s();
    m->variant = variant;
    m->host = hm;
    m->t2_ok = pack_t2(hm, d, m->t2);
    DevMech &dm = m->dm;
    dm.nsp = nsp;
    dm.nrc = nrc;
    dm.ext = hm.ext ? 1 : 0;
    int rc = HC_OK;
    auto up = [&](auto *src, size_t n, auto **dst) {
        if (rc == HC_OK) rc = upload(m->owned, src, n, dst);
    };
    up(d->W, nsp, &dm.W);
    up(d->Trange, 3 * (size_t)nsp, &dm.Trange);
    up(d->nasa, 14 * (size_t)nsp, &dm.nasa);
    up(p_type.data(), nrc, &dm.rate_type);
    up(p_rev.data(), nrc, &dm.reversible);
    up(p_arr.data(), 3 * (size_t)nrc, &dm.arr);
    up(p_arr0.data(), 3 * (size_t)nrc, &dm.arr0);
    up(p_troe.data(), 4 * (size_t)nrc, &dm.troe);
    up(hm.sri.data(), 5 * (size_t)nrc, &dm.sri);
    up(hm.arr_rev.data(), 3 * (size_t)nrc, &dm.arr_rev);
    up(hm.activated.data(), (size_t)nrc, &dm.activated);
    up(hm.lt.data(), 2 * (size_t)nrc, &dm.lt);
    up(hm.xcoef.data(), 9 * (size_t)nrc, &dm.xcoef);
    up(hm.plog_ptr.data(), (size_t)nrc + 1, &dm.plog_ptr);
    {
        // the warp-per-cell kernel's tables (nsp + 1 <= 32, the common rate forms)
        WHost wh;
        if (pack_w(hm, wh)) {
            WMech &w = m->w;
            w.nsp = wh.nsp;
            w.nrc = wh.nrc;
            w.nrc32 = wh.nrc32;
            w.ntb = (int)wh.tbl.size();
            if (wh.tbl.size() == 1) {
                const int o = wh.tbl[0];
                if (wh.nrc == 0 || wh.ri[((size_t)(o >> 5) * kWRIn + kWtype) * 32 + (o & 31)] == HC_RATE_ARRHENIUS)
                    w.ntb = 0;   // placeholder entry only
            }
            w.nent = (int)wh.lnu.size();
            w.njob = wh.njob;
            w.njob32 = wh.njob32;
            w.glim = wh.glim;
            up(wh.th.data(), wh.th.size(), &w.th);
            up(wh.rd.data(), wh.rd.size(), &w.rd);
            up(wh.ri.data(), wh.ri.size(), &w.ri);
            up(wh.eff.data(), wh.eff.size(), &w.eff);
            up(wh.lptr.data(), wh.lptr.size(), &w.lptr);
            up(wh.lent.data(), wh.lent.size(), &w.lent);
            up(wh.lnu.data(), wh.lnu.size(), &w.lnu);
            up(wh.xj.data(), wh.xj.size(), &w.xj);
            up(wh.tbl.data(), wh.tbl.size(), &w.tbl);
            up(wh.raw.data(), wh.raw.size(), &w.raw);
            m->w_ok = (rc == HC_OK);
        }
    }
    up(hm.plog_p.data(), hm.plog_p.size(), &dm.plog_p);
    up(hm.plog_arr.data(), hm.plog_arr.size(), &dm.plog_arr);
    up(p_eff.data(), (size_t)nrc * nsp, &dm.eff);
    up(p_nf.data(), nrc, &dm.nf);
    up(p_nb.data(), nrc, &dm.nb);
    up(p_fidx.data(), HC_MAX_SIDE * (size_t)nrc, &dm.fidx);
    up(p_bidx.data(), HC_MAX_SIDE * (size_t)nrc, &dm.bidx);
    up(p_ford.data(), HC_MAX_SIDE * (size_t)nrc, &dm.ford);
    up(p_bord.data(), HC_MAX_SIDE * (size_t)nrc, &dm.bord);
    up(p_fnu.data(), HC_MAX_SIDE * (size_t)nrc, &dm.fnu);
    up(p_bnu.data(), HC_MAX_SIDE * (size_t)nrc, &dm.bnu);
    up(sum_stoi.data(), nrc, &dm.sum_stoi);
    up(sp_ptr.data(), nsp + 1, &dm.sp_ptr);
    up(sp_rxn.data(), sp_rxn.size(), &dm.sp_rxn);
    up(sp_coef.data(), sp_coef.size(), &dm.sp_coef);
    if (d->geom) up(d->geom, nsp, &dm.geom);
    if (d->eps_k) up(d->eps_k, nsp, &dm.eps_k);
    if (d->sigma) up(d->sigma, nsp, &dm.sigma);
    if (d->eps_k && d->sigma) {
        // pair constants of kineticTheory::Di (kineticTheory.cpp:126-141) and of
        // the Wilke factors (transportList.cpp:31-56), with the host libm
        const size_t nn = (size_t)nsp * nsp;
        std::vector<double> pD(nn), pP(nn), pR(nn), pPhi(nn), pW(nn);
        const double c8 = 1.0 / std::sqrt(8.0);
        for (int i = 0; i < nsp; ++i) {
            const double invW = 1.0 / d->W[i];
            for (int j = 0; j < nsp; ++j) {
                const size_t k = (size_t)i * nsp + j;
                const double sij = 0.5 * (d->sigma[i] + d->sigma[j]);
                pD[k] = 1.858e-7 * std::sqrt(invW + 1.0 / d->W[j]) / (sij * sij) * 1.01325e5;
                pR[k] = 1.0 / std::sqrt(d->eps_k[i] * d->eps_k[j]);
                pP[k] = std::exp(-0.145 * std::log(pR[k]));
                pPhi[k] = c8 / std::sqrt(1.0 + d->W[i] / d->W[j]);
                pW[k] = std::sqrt(d->W[i] / d->W[j]);
            }
        }
        up(pD.data(), nn, &dm.pair_D);
        up(pP.data(), nn, &dm.pair_Dpow);
        up(pR.data(), nn, &dm.pair_r);
        up(pPhi.data(), nn, &dm.pair_phi);
        up(pW.data(), nn, &dm.pair_w);
    }
    if (rc == HC_OK) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, 8 * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            rc = fail(HC_E_CUDA, cudaGetErrorString(e));
        } else {
            m->owned.push_back(q);
            m->queue = static_cast<unsigned long long *>(q);
        }
    }
    if (rc == HC_OK) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    if (rc != HC_OK) {
        for (void *p : m->owned) cudaFree(p);
        delete m;
        return rc;
    }
    *out = m;
    return HC_OK;
}

int hc_set_tuning(hc_mech_t m, int kernel, int block) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (kernel < 0 || kernel > 7) return fail(HC_E_INVALID, "kernel must be 0 .. 7");
    if (block != 32 && block != 64 && block != 128)
        return fail(HC_E_INVALID, "block must be 32, 64 or 128");
    if (block != m->block) {
        m->jit_tried = false;   // the generated kernels are built per block size
        m->jit = JitKernel();
        m->jit5_tried = false;
        m->jit5 = JitKernel();
    }
    m->kernel = kernel;
    m->block = block;
    return HC_OK;
}

int hc_jit_compile_kernel(const hc_mech_desc *d, int kernel, int block, int64_t *cubin_bytes) {
    if (!d || !cubin_bytes) return fail(HC_E_INVALID, "null argument");
    int64_t len = 0;
    int rc = hc_jit_source_kernel(d, kernel, block, nullptr, 0, &len);
    if (rc != HC_OK) return rc;
    HostMech h;
    make_host(d, h);
    std::vector<char> cubin;
    std::string err;
    rc = jit_compile(kernel == 5 ? jit_t3_source(h, block) : jit_t1_source(h, block), cubin, err);
    if (rc != HC_OK) return fail(rc, err);
    *cubin_bytes = (int64_t)cubin.size();
    return HC_OK;
}

int hc_jit_source_kernel(const hc_mech_desc *d, int kernel, int block, char *buf, int64_t cap,
                         int64_t *len) {
    if (!d || !len) return fail(HC_E_INVALID, "null argument");
    if (kernel != 3 && kernel != 5) return fail(HC_E_INVALID, "generated kernels are 3 and 5");
    const int vrc = check_desc(d);
    if (vrc != HC_OK) return vrc;
    if (d->nsp + 1 > 16) return fail(HC_E_UNSUPPORTED, "no generated kernel for nsp + 1 > 16");
    if (block != 32 && block != 64 && block != 128)
        return fail(HC_E_INVALID, "block must be 32, 64 or 128");
    HostMech h;
    make_host(d, h);
    if (h.ext)
        return fail(HC_E_UNSUPPORTED,
                    "no generated kernel for SRI, explicit reverse (REV), PLOG, HIGH, LT, JAN, FIT1 or "
                    "collision rate laws");
    const std::string src = (kernel == 5) ? jit_t3_source(h, block) : jit_t1_source(h, block);
    *len = (int64_t)src.size();
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, src.size());
        std::memcpy(buf, src.data(), n);
        buf[n] = 0;
    }
    return HC_OK;
}

int hc_jit_compile(const hc_mech_desc *d, int block, int64_t *cubin_bytes) {
    return hc_jit_compile_kernel(d, 3, block, cubin_bytes);
}

int hc_jit_source(const hc_mech_desc *d, int block, char *buf, int64_t cap, int64_t *len) {
    return hc_jit_source_kernel(d, 3, block, buf, cap, len);
}

int hc_mech_destroy(hc_mech_t m) {
    if (!m) return HC_OK;
    for (void *p : m->owned) cudaFree(p);
    if (m->ws) cudaFree(m->ws);
    if (m->ylast) cudaFree(m->ylast);
    delete m;
    return HC_OK;
}

int hc_mech_nsp(hc_mech_t m) { return m ? m->dm.nsp : -1; }
int hc_mech_nrc(hc_mech_t m) { return m ? m->dm.nrc : -1; }

}  // extern "C"

static int integrate_impl(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *T,
                          const double *p, double *rho, double *Y, const double *dt,
                          double dt_factor, double *subdt, double *Ri, int32_t *status,
                          const int32_t *order, int64_t *cost, cudaStream_t st,
                          int64_t nqueue = -1) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    int rc = check_opts(opts);
    if (rc != HC_OK) return rc;
    if (ncells < 0) return fail(HC_E_INVALID, "negative cell count");
    HC_CUDA(cudaMemsetAsync(m->queue, 0, 7 * sizeof(unsigned long long), st));
    if (ncells == 0) return HC_OK;
    if (!T || !p || !rho || !Y || !dt || !subdt) return fail(HC_E_INVALID, "null field");
    if (!(dt_factor > 0)) return fail(HC_E_INVALID, "dt_factor must be positive");
    const IntegratorParams P = make_params(opts);
    CellIO io;
    io.ncells = ncells;
    io.nqueue = (nqueue < 0) ? ncells : nqueue;
    if (io.nqueue > ncells || (nqueue >= 0 && !order))
        return fail(HC_E_INVALID, "subset needs a cell list no longer than the fields");
    if (io.nqueue == 0) return HC_OK;
    io.T = T;
    io.p = p;
    io.rho = rho;
    io.Y = Y;
    io.dt = dt;
    io.dt_factor = dt_factor;
    io.subdt = subdt;
    io.Ri = Ri;
    io.status = status;
    io.order = order;
    io.cost = cost;
    io.queue_head = m->queue;
    io.counters = m->queue + 1;
    const int N = m->dm.nsp + 1;
    const bool t1_ok = N <= 16 && !opts->auto_update_jacobian && !m->host.ext && opts->reactor == 0;
    if (m->kernel == 1 && !t1_ok)
        return fail(HC_E_UNSUPPORTED,
                    "thread-per-cell kernel needs nsp <= 15, autoUpdateJacobian off, the "
                    "constant-pressure reactor and no SRI or explicit reverse (REV), PLOG, HIGH, "
                    "LT, JAN, FIT1 or collision rate laws");
    if (m->kernel == 4 && !(t1_ok && m->t2_ok))
        return fail(HC_E_UNSUPPORTED,
                    "compact thread-per-cell kernel needs nsp <= 15, <= 64 reactions, "
                    "autoUpdateJacobian off, the constant-pressure reactor and no SRI, explicit "
                    "reverse (REV), PLOG, HIGH, LT, JAN, FIT1 or collision rate laws");
    // Per-cell costs in a flow step differ by orders of magnitude, and the
    // step lasts as long as its stiffest cell: the cooperative kernels (cell
    // group, warp per cell) share each Newton iteration of one cell among
    // lanes and finish a single cell several times sooner than one thread does.
    const bool use_t2 = t1_ok && m->t2_ok && m->kernel == 4;
    if (use_t2) {
        if (m->ylast_cells < (size_t)ncells) {
            // grows only: a first call with a new, larger size synchronises the
            // stream and must therefore come before any stream capture
            HC_CUDA(cudaStreamSynchronize(st));
            if (m->ylast) HC_CUDA(cudaFree(m->ylast));
            m->ylast = nullptr;
            m->ylast_cells = 0;
            HC_CUDA(cudaMalloc(&m->ylast, sizeof(double) * 2 * 16 * (size_t)ncells));
            m->ylast_cells = (size_t)ncells;
        }
        return variant_integrate_t2(N, m->t2, m->num_sms, P, io, m->ylast, m->block, st, g_err);
    }
    if (m->kernel == 7) {
        if (!m->w_ok || opts->reactor != 0)
            return fail(HC_E_UNSUPPORTED,
                        "segment-per-cell kernel needs nsp + 1 <= 16, the constant-pressure reactor and no "
                        "SRI, explicit reverse (REV), PLOG, HIGH, LT, JAN, FIT1 or collision rate laws");
        return launch_integrate_s(m->w, m->num_sms, P, io, st, g_err);
    }
    // automatic choice (kernel 0): the warp-per-cell kernel wherever it takes
    // the mechanism (the fastest on the batched workload: 1.14e8 Newton
    // iterations/s against 0.6e8 for the cell group), else the cell group
    const bool auto_w = m->kernel == 0 && m->w_ok && opts->reactor == 0;
    if (m->kernel == 6 || auto_w) {
        if (!m->w_ok || opts->reactor != 0)
            return fail(HC_E_UNSUPPORTED,
                        "warp-per-cell kernel needs nsp + 1 <= 16, the constant-pressure reactor and no "
                        "SRI, explicit reverse (REV), PLOG, HIGH, LT, JAN, FIT1 or collision rate laws");
        return launch_integrate_w(m->w, m->num_sms, P, io, st, g_err);
    }
    if (m->kernel == 5 && !t1_ok)
        return fail(HC_E_UNSUPPORTED,
                    "direct-assembly thread-per-cell kernel needs nsp <= 15, autoUpdateJacobian off, "
                    "the constant-pressure reactor and no SRI, explicit reverse (REV), PLOG, HIGH, "
                    "LT, JAN, FIT1 or collision rate laws");
    if (t1_ok && m->kernel == 5) {
        if (!m->jit5_tried) {
            // first use: generate, compile and load (host work, no stream operation)
            m->jit5_tried = true;
            std::string err;
            if (jit_build_t3(m->host, m->block, &m->jit5, err) != HC_OK) {
                m->jit5 = JitKernel();
                m->jit5_err = err;
            }
        }
        if (!m->jit5.func) return fail(HC_E_UNSUPPORTED, "generated kernel unavailable: " + m->jit5_err);
        if (m->ylast_cells < (size_t)ncells) {
            // grows only: a first call with a new, larger size synchronises the
            // stream and must therefore come before any stream capture
            HC_CUDA(cudaStreamSynchronize(st));
            if (m->ylast) HC_CUDA(cudaFree(m->ylast));
            m->ylast = nullptr;
            m->ylast_cells = 0;
            HC_CUDA(cudaMalloc(&m->ylast, sizeof(double) * 2 * 16 * (size_t)ncells));
            m->ylast_cells = (size_t)ncells;
        }
        return jit_launch_t1(m->jit5, m->num_sms, P, io, m->ylast, st, g_err);
    }
    if (m->kernel == 3 && !t1_ok)
        return fail(HC_E_UNSUPPORTED,
                    "generated thread-per-cell kernel needs nsp <= 15, autoUpdateJacobian off, the "
                    "constant-pressure reactor and no SRI, explicit reverse (REV), PLOG, HIGH, LT, "
                    "JAN, FIT1 or collision rate laws");
    bool use_jit = t1_ok && m->kernel == 3;
    if (use_jit && !m->jit_tried) {
        // first use: generate, compile and load (host work, no stream operation)
        m->jit_tried = true;
        std::string err;
        if (jit_build_t1(m->host, m->block, &m->jit, err) != HC_OK) {
            m->jit = JitKernel();
            m->jit_err = err;
        }
    }
    if (use_jit && !m->jit.func) {
        if (m->kernel == 3) return fail(HC_E_UNSUPPORTED, "generated kernel unavailable: " + m->jit_err);
        use_jit = false;   // automatic choice: the precompiled thread-per-cell kernel
    }
    const bool use_t1 = t1_ok && (m->kernel == 1 || use_jit);
    if (use_t1) {
        if (m->ylast_cells < (size_t)ncells) {
            // grows only: a first call with a new, larger size synchronises the
            // stream and must therefore come before any stream capture
            HC_CUDA(cudaStreamSynchronize(st));
            if (m->ylast) HC_CUDA(cudaFree(m->ylast));
            m->ylast = nullptr;
            m->ylast_cells = 0;
            HC_CUDA(cudaMalloc(&m->ylast, sizeof(double) * 2 * 16 * (size_t)ncells));
            m->ylast_cells = (size_t)ncells;
        }
        if (use_jit) return jit_launch_t1(m->jit, m->num_sms, P, io, m->ylast, st, g_err);
        return variant_integrate_t1(N, m->dm, m->num_sms, P, io, m->ylast, m->block, st, g_err);
    }
    HC_DISPATCH(m, integrate, m->dm, m->num_sms, P, io, st, g_err);
}

// grow the host-entry-point workspace (callers hold m->mu); growing
// synchronises the stream first
static int ensure_ws(hc_mech_t m, size_t bytes, cudaStream_t st) {
    if (m->ws_bytes >= bytes) return HC_OK;
    HC_CUDA(cudaStreamSynchronize(st));
    if (m->ws) cudaFree(m->ws);
    m->ws = nullptr;
    m->ws_bytes = 0;
    HC_CUDA(cudaMalloc(&m->ws, bytes));
    m->ws_bytes = bytes;
    return HC_OK;
}

static int read_counters(hc_mech_t m, hc_counters *c, cudaStream_t st) {
    if (!c) return HC_OK;
    unsigned long long h[7];
    HC_CUDA(cudaMemcpyAsync(h, m->queue, sizeof(h), cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    c->n_jac = (int64_t)h[1];
    c->n_rhs = (int64_t)h[2];
    c->n_lu = (int64_t)h[3];
    c->n_newton = (int64_t)h[4];
    c->n_steps = (int64_t)h[5];
    c->n_attempts = (int64_t)h[6];
    return HC_OK;
}

static int count_bad_status(const int32_t *status_host, int64_t n) {
    int bad = 0;
    for (int64_t i = 0; i < n; ++i)
        if (status_host[i] & (HC_CELL_UNDERFLOW | HC_CELL_ITER_LIMIT)) ++bad;
    return bad;
}

extern "C" {

int hc_integrate(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *T, const double *p,
                 double *rho, double *Y, const double *dt, double dt_factor, double *subdt,
                 double *Ri, int32_t *status, hc_counters *counters, void *stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = integrate_impl(m, opts, ncells, T, p, rho, Y, dt, dt_factor, subdt, Ri, status,
                            nullptr, nullptr, st);
    if (rc != HC_OK) return rc;
    return read_counters(m, counters, st);
}

int hc_integrate_ordered(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *T,
                         const double *p, double *rho, double *Y, const double *dt,
                         double dt_factor, double *subdt, double *Ri, int32_t *status,
                         const int32_t *order, int64_t *cost, hc_counters *counters,
                         void *stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = integrate_impl(m, opts, ncells, T, p, rho, Y, dt, dt_factor, subdt, Ri, status,
                            order, cost, st);
    if (rc != HC_OK) return rc;
    return read_counters(m, counters, st);
}

int hc_integrate_subset(hc_mech_t m, const hc_opts *opts, int64_t ncells, int64_t nsel,
                        const int32_t *sel, double *T, const double *p, double *rho, double *Y,
                        const double *dt, double dt_factor, double *subdt, double *Ri,
                        int32_t *status, int64_t *cost, hc_counters *counters, void *stream) {
    if (nsel < 0) return fail(HC_E_INVALID, "negative subset size");
    if (nsel > 0 && !sel) return fail(HC_E_INVALID, "null cell list");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = integrate_impl(m, opts, ncells, T, p, rho, Y, dt, dt_factor, subdt, Ri, status, sel,
                            cost, st, nsel);
    if (rc != HC_OK) return rc;
    return read_counters(m, counters, st);
}

int hc_integrate_host(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *T,
                      const double *p, double *rho, double *Y, const double *dt,
                      double dt_factor, double *subdt, double *Ri, int32_t *status,
                      hc_counters *counters, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (ncells <= 0)
        return integrate_impl(m, opts, ncells, T, p, rho, Y, dt, dt_factor, subdt, Ri, status,
                              nullptr, nullptr, st);
    std::lock_guard<std::mutex> lk(m->mu);
    const int nsp = m->dm.nsp;
    const size_t n = (size_t)ncells;
    const size_t bytes = sizeof(double) * (n * (5 + 2 * (size_t)nsp)) + sizeof(int32_t) * n + 256;
    int wrc = ensure_ws(m, bytes, st);
    if (wrc != HC_OK) return wrc;
    double *dT = static_cast<double *>(m->ws);
    double *dp = dT + n, *drho = dp + n, *ddt = drho + n, *dsub = ddt + n;
    double *dY = dsub + n, *dRi = dY + n * nsp;
    int32_t *dst = reinterpret_cast<int32_t *>(dRi + n * nsp);
    HC_CUDA(cudaMemcpyAsync(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dp, p, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(drho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(ddt, dt, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dsub, subdt, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dY, Y, sizeof(double) * n * nsp, cudaMemcpyHostToDevice, st));
    int rc = integrate_impl(m, opts, ncells, dT, dp, drho, dY, ddt, dt_factor, dsub,
                            Ri ? dRi : nullptr, dst, nullptr, nullptr, st);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaMemcpyAsync(T, dT, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaMemcpyAsync(rho, drho, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaMemcpyAsync(subdt, dsub, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaMemcpyAsync(Y, dY, sizeof(double) * n * nsp, cudaMemcpyDeviceToHost, st));
    if (Ri) HC_CUDA(cudaMemcpyAsync(Ri, dRi, sizeof(double) * n * nsp, cudaMemcpyDeviceToHost, st));
    std::vector<int32_t> stat_h;
    int32_t *stat_out = status;
    if (!stat_out) {
        stat_h.resize(n);
        stat_out = stat_h.data();
    }
    HC_CUDA(cudaMemcpyAsync(stat_out, dst, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    rc = read_counters(m, counters, st);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaStreamSynchronize(st));
    return count_bad_status(stat_out, ncells);
}

int hc_rhs_jacobian(hc_mech_t m, int64_t n, const double *c, const double *T, const double *p,
                    double *dydt, double *J, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!c || !T || !p) return fail(HC_E_INVALID, "null field");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    HC_DISPATCH(m, rhsjac, m->dm, n, c, T, p, dydt, J, st, g_err);
}

int hc_source_terms(hc_mech_t m, int64_t n, const double *T, const double *p, const double *rho,
                    const double *Y, double *Ri, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !rho || !Y || !Ri) return fail(HC_E_INVALID, "null field");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    HC_DISPATCH(m, source, m->dm, n, T, p, rho, Y, Ri, st, g_err);
}

int hc_source_terms_imp(hc_mech_t m, int64_t n, const double *T, const double *p,
                        const double *rho, const double *Y, double *Ri, double *diag,
                        void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !rho || !Y || !Ri || !diag) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp < 2) return fail(HC_E_INVALID, "point-implicit terms need at least 2 species");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    HC_DISPATCH(m, srcimp, m->dm, n, T, p, rho, Y, Ri, diag, st, g_err);
}

int hc_temperature_from_enthalpy(hc_mech_t m, int64_t n, const double *ha, const double *Y,
                                 const double *T0, double TLow, double THigh, double *T,
                                 int32_t *flag, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!ha || !Y || !T0 || !T) return fail(HC_E_INVALID, "null field");
    if (!(TLow > 0) || !(THigh > TLow)) return fail(HC_E_INVALID, "need 0 < TLow < THigh");
    return launch_t_from_ha(m->dm, n, ha, Y, T0, TLow, THigh, T, flag,
                            static_cast<cudaStream_t>(stream), g_err);
}

int hc_temperature_from_energy(hc_mech_t m, int64_t n, const double *ea, const double *Y,
                               const double *rho, const double *T0, double TLow, double THigh,
                               double *T, int32_t *flag, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!ea || !Y || !rho || !T0 || !T) return fail(HC_E_INVALID, "null field");
    if (!(TLow > 0) || !(THigh > TLow)) return fail(HC_E_INVALID, "need 0 < TLow < THigh");
    return launch_t_from_ea(m->dm, n, ea, Y, rho, T0, TLow, THigh, T, flag,
                            static_cast<cudaStream_t>(stream), g_err);
}

int hc_properties(hc_mech_t m, int64_t n, const double *T, const double *p, const double *Y,
                  double *ha, double *cp, double *mu, double *kappa, double *D, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !Y) return fail(HC_E_INVALID, "null field");
    if (!m->dm.geom || !m->dm.eps_k || !m->dm.sigma)
        return fail(HC_E_INVALID, "mechanism has no transport data");
    return launch_properties(m->dm, n, T, p, Y, ha, cp, mu, kappa, D,
                             static_cast<cudaStream_t>(stream), g_err);
}

int hc_source_terms_host(hc_mech_t m, int64_t n, const double *T, const double *p,
                         const double *rho, const double *Y, double *Ri, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !rho || !Y || !Ri) return fail(HC_E_INVALID, "null field");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    const size_t nn = (size_t)n, nsp = (size_t)m->dm.nsp;
    int rc = ensure_ws(m, sizeof(double) * nn * (3 + 2 * nsp), st);
    if (rc != HC_OK) return rc;
    double *dT = static_cast<double *>(m->ws), *dp = dT + nn, *dr = dp + nn, *dY = dr + nn;
    double *dR = dY + nn * nsp;
    HC_CUDA(cudaMemcpyAsync(dT, T, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dp, p, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dr, rho, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dY, Y, sizeof(double) * nn * nsp, cudaMemcpyHostToDevice, st));
    rc = hc_source_terms(m, n, dT, dp, dr, dY, dR, stream);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaMemcpyAsync(Ri, dR, sizeof(double) * nn * nsp, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    return HC_OK;
}

int hc_properties_host(hc_mech_t m, int64_t n, const double *T, const double *p, const double *Y,
                       double *ha, double *cp, double *mu, double *kappa, double *D,
                       void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !Y) return fail(HC_E_INVALID, "null field");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    const size_t nn = (size_t)n, nsp = (size_t)m->dm.nsp;
    int rc = ensure_ws(m, sizeof(double) * nn * (5 + 3 * nsp), st);
    if (rc != HC_OK) return rc;
    double *dT = static_cast<double *>(m->ws), *dp = dT + nn, *dY = dp + nn;
    double *dha = dY + nn * nsp, *dD = dha + nn * nsp, *dcp = dD + nn * nsp, *dmu = dcp + nn;
    double *dk = dmu + nn;
    HC_CUDA(cudaMemcpyAsync(dT, T, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dp, p, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(dY, Y, sizeof(double) * nn * nsp, cudaMemcpyHostToDevice, st));
    rc = hc_properties(m, n, dT, dp, dY, ha ? dha : nullptr, cp ? dcp : nullptr,
                       mu ? dmu : nullptr, kappa ? dk : nullptr, D ? dD : nullptr, stream);
    if (rc != HC_OK) return rc;
    if (ha) HC_CUDA(cudaMemcpyAsync(ha, dha, sizeof(double) * nn * nsp, cudaMemcpyDeviceToHost, st));
    if (D) HC_CUDA(cudaMemcpyAsync(D, dD, sizeof(double) * nn * nsp, cudaMemcpyDeviceToHost, st));
    if (cp) HC_CUDA(cudaMemcpyAsync(cp, dcp, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (mu) HC_CUDA(cudaMemcpyAsync(mu, dmu, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (kappa) HC_CUDA(cudaMemcpyAsync(kappa, dk, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    return HC_OK;
}

int hc_surrogate_features(hc_mech_t m, int64_t n, const double *T, const double *p,
                          const double *Y, const double *dt, double dt_factor, const double *mean,
                          const double *inv_std, float *X, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!T || !p || !Y || !dt || !mean || !inv_std || !X) return fail(HC_E_INVALID, "null field");
    return launch_features(m->dm, n, T, p, Y, dt, dt_factor, mean, inv_std, X,
                           static_cast<cudaStream_t>(stream));
}

int hc_surrogate_gate(hc_mech_t m, int64_t n, double *T, const double *p, double *rho, double *Y,
                      const float *pred, const float *X, const double *out_mean,
                      const double *out_std, const double *proj, const double *elem, int nel,
                      const float *spread, const hc_gate_opts *g, int32_t *accept,
                      int32_t *rejected, int64_t *n_rejected, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (!g || !n_rejected) return fail(HC_E_INVALID, "null argument");
    *n_rejected = 0;
    if (n <= 0) return HC_OK;
    if (!T || !p || !rho || !Y || !pred || !X || !out_mean || !out_std || !proj || !elem ||
        !accept || !rejected)
        return fail(HC_E_INVALID, "null field");
    if (nel < 1 || nel > 8) return fail(HC_E_INVALID, "the gate handles 1 to 8 elements");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long *cnt = m->queue + 7;
    HC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    GateArgs a;
    a.n = n;
    a.T = T;
    a.p = p;
    a.rho = rho;
    a.Y = Y;
    a.pred = pred;
    a.X = X;
    a.out_mean = out_mean;
    a.out_std = out_std;
    a.proj = proj;
    a.elem = elem;
    a.nel = nel;
    a.tol_T = g->tol_T;
    a.tol_proj = g->tol_proj;
    a.y_neg = g->y_neg;
    a.x_max = g->x_max;
    a.T_min = g->T_min;
    a.T_max = g->T_max;
    a.spread = spread;
    a.tol_spread = g->tol_spread;
    a.accept = accept;
    a.rejected = rejected;
    a.n_rejected = cnt;
    int rc = launch_gate(m->dm, a, st);
    if (rc != HC_OK) return rc;
    unsigned long long h = 0;
    HC_CUDA(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    *n_rejected = (int64_t)h;
    return HC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Record-per-cell entry points: the reference's CUDA-path buffers.
//
// Integration records are [T, Y_0..Y_{nsp-1}, rho] (calcChemODEsArray,
// CUDAChemistrySourceODEs.cu:823-858); source-term records are
// [Y_0..Y_{nsp-1}, rho, T] with RRi[cell * nsp + i] out
// (calcOnlyChemSourceTermsAsync via CUDAChemistrySource.cpp:189-198). The
// records are transposed into species-major rows in the mechanism's
// workspace (rows [T][Y][rho] or [Y][rho][T], so that a transpose of the
// whole record matrix is all it takes), the species-major kernels run on
// them, and the results are transposed back. p is taken from the caller when
// given, else from the ideal-gas law with the record's rho, T and Y.
// ---------------------------------------------------------------------------
namespace {

// workspace for the record-per-cell entry points (callers hold m->mu)
struct AosWs {
    double *recs;   // device copy of the caller's records (host entry points)
    double *rows;   // [rec][n]
    double *p;      // [n]
    double *dt, *subdt;
    double *out;    // source terms: Ri rows [nsp][n], then RRi records [n][nsp]
    int32_t *status;
};

int aos_ws(hc_mech_t m, int64_t ncells, bool host, bool source, cudaStream_t st, AosWs &w) {
    const size_t n = (size_t)ncells, rec = (size_t)m->dm.nsp + 2, nsp = (size_t)m->dm.nsp;
    size_t doubles = n * rec + n;                           // rows, p
    if (host) doubles += n * rec + (source ? 0 : 2 * n);    // records, dt, subdt
    if (source) doubles += 2 * n * nsp;                     // Ri rows, RRi records
    const size_t bytes = sizeof(double) * doubles + sizeof(int32_t) * n + 256;
    int rc = ensure_ws(m, bytes, st);
    if (rc != HC_OK) return rc;
    double *q = static_cast<double *>(m->ws);
    w = AosWs{};
    w.rows = q;
    q += n * rec;
    w.p = q;
    q += n;
    if (host) {
        w.recs = q;
        q += n * rec;
        if (!source) {
            w.dt = q;
            q += n;
            w.subdt = q;
            q += n;
        }
    }
    if (source) {
        w.out = q;
        q += 2 * n * nsp;
    }
    w.status = reinterpret_cast<int32_t *>(q);
    return HC_OK;
}

// device records in, device records out (stream-ordered)
int integrate_records(hc_mech_t m, const hc_opts *opts, int64_t n, double *recs, const double *p,
                      const double *dt, double *subdt, int return_ci, int32_t *status,
                      const AosWs &w, cudaStream_t st) {
    const int nsp = m->dm.nsp, rec = nsp + 2;
    double *T = w.rows, *Y = w.rows + n, *rho = w.rows + (size_t)n * (nsp + 1);
    int rc = launch_records_to_rows(n, rec, recs, w.rows, st, g_err);
    if (rc != HC_OK) return rc;
    if (!p) {
        rc = launch_ideal_gas_p(n, nsp, m->dm.W, T, rho, Y, w.p, st, g_err);
        if (rc != HC_OK) return rc;
        p = w.p;
    }
    rc = integrate_impl(m, opts, n, T, p, rho, Y, dt, 1.0, subdt, nullptr, status, nullptr,
                        nullptr, st);
    if (rc != HC_OK) return rc;
    // concentrations: T and c_i written, the record's rho kept (the
    // reference's returnCi form); else T, Y_i and the new rho
    return launch_rows_to_records(n, rec, return_ci ? nsp + 1 : rec, w.rows, recs,
                                  return_ci ? m->dm.W : nullptr, nsp, st, g_err);
}

int source_records(hc_mech_t m, int64_t n, const double *recs, const double *p, double *RRi,
                   const AosWs &w, cudaStream_t st) {
    const int nsp = m->dm.nsp, rec = nsp + 2;
    double *Y = w.rows, *rho = w.rows + (size_t)n * nsp, *T = w.rows + (size_t)n * (nsp + 1);
    int rc = launch_records_to_rows(n, rec, recs, w.rows, st, g_err);
    if (rc != HC_OK) return rc;
    if (!p) {
        rc = launch_ideal_gas_p(n, nsp, m->dm.W, T, rho, Y, w.p, st, g_err);
        if (rc != HC_OK) return rc;
        p = w.p;
    }
    rc = hc_source_terms(m, n, T, p, rho, Y, w.out, st);
    if (rc != HC_OK) return rc;
    return launch_rows_to_records(n, nsp, nsp, w.out, RRi, nullptr, nsp, st, g_err);
}

int aos_zero(hc_mech_t m, const hc_opts *opts, int64_t ncells, cudaStream_t st) {
    return integrate_impl(m, opts, ncells, nullptr, nullptr, nullptr, nullptr, nullptr, 1.0,
                          nullptr, nullptr, nullptr, nullptr, nullptr, st);
}

}  // namespace

extern "C" {

int hc_integrate_aos(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *TYiRho,
                     const double *p, const double *dt, double *subdt, int return_ci,
                     int32_t *status, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (ncells <= 0) return aos_zero(m, opts, ncells, st);
    int rc = check_opts(opts);
    if (rc != HC_OK) return rc;
    if (!TYiRho || !dt || !subdt) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    std::lock_guard<std::mutex> lk(m->mu);
    AosWs w;
    rc = aos_ws(m, ncells, false, false, st, w);
    if (rc != HC_OK) return rc;
    return integrate_records(m, opts, ncells, TYiRho, p, dt, subdt, return_ci, status, w, st);
}

int hc_integrate_aos_host(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *TYiRho,
                          const double *p, const double *dt, double *subdt, int return_ci,
                          int32_t *status, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (ncells <= 0) return aos_zero(m, opts, ncells, st);
    int rc = check_opts(opts);
    if (rc != HC_OK) return rc;
    if (!TYiRho || !dt || !subdt) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    std::lock_guard<std::mutex> lk(m->mu);
    AosWs w;
    rc = aos_ws(m, ncells, true, false, st, w);
    if (rc != HC_OK) return rc;
    const size_t n = (size_t)ncells, rec = (size_t)m->dm.nsp + 2;
    HC_CUDA(cudaMemcpyAsync(w.recs, TYiRho, sizeof(double) * n * rec, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(w.dt, dt, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HC_CUDA(cudaMemcpyAsync(w.subdt, subdt, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    const double *dp = nullptr;
    if (p) {
        HC_CUDA(cudaMemcpyAsync(w.p, p, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        dp = w.p;
    }
    rc = integrate_records(m, opts, ncells, w.recs, dp, w.dt, w.subdt, return_ci, w.status, w,
                           st);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaMemcpyAsync(TYiRho, w.recs, sizeof(double) * n * rec, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaMemcpyAsync(subdt, w.subdt, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    std::vector<int32_t> stat_h;
    int32_t *stat_out = status;
    if (!stat_out) {
        stat_h.resize(n);
        stat_out = stat_h.data();
    }
    HC_CUDA(cudaMemcpyAsync(stat_out, w.status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    return count_bad_status(stat_out, ncells);
}

int hc_source_terms_aos(hc_mech_t m, int64_t n, const double *YiRhoT, const double *p,
                        double *RRi, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!YiRhoT || !RRi) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    AosWs w;
    int rc = aos_ws(m, n, false, true, st, w);
    if (rc != HC_OK) return rc;
    return source_records(m, n, YiRhoT, p, RRi, w, st);
}

int hc_source_terms_aos_async(hc_mech_t m, int64_t n, const double *YiRhoT, const double *p,
                              double *RRi, void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n <= 0) return HC_OK;
    if (!YiRhoT || !RRi) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    AosWs w;
    int rc = aos_ws(m, n, true, true, st, w);
    if (rc != HC_OK) return rc;
    const size_t nn = (size_t)n, nsp = (size_t)m->dm.nsp, rec = nsp + 2;
    HC_CUDA(cudaMemcpyAsync(w.recs, YiRhoT, sizeof(double) * nn * rec, cudaMemcpyHostToDevice, st));
    const double *dp = nullptr;
    if (p) {
        HC_CUDA(cudaMemcpyAsync(w.p, p, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
        dp = w.p;
    }
    double *dR = w.out + nn * nsp;
    rc = source_records(m, n, w.recs, dp, dR, w, st);
    if (rc != HC_OK) return rc;
    // enqueued only: the caller overlaps its own host work and synchronises
    // the stream before reading RRi
    HC_CUDA(cudaMemcpyAsync(RRi, dR, sizeof(double) * nn * nsp, cudaMemcpyDeviceToHost, st));
    return HC_OK;
}

}  // extern "C"

// properties from records [Y..., T, p] (device pointers); rows is the
// workspace: [nsp+2][n] input rows, [nsp+1][n] ha / cp rows, [nsp+2][n]
// D / mu / kappa rows
static int properties_records(hc_mech_t m, int64_t n, const double *recs, double *haicp,
                              double *DMuKappa, double *rows, cudaStream_t st) {
    const int nsp = m->dm.nsp;
    const size_t nn = (size_t)n;
    double *in = rows, *hc = in + nn * (nsp + 2), *dmk = hc + nn * (nsp + 1);
    int rc = launch_records_to_rows(n, nsp + 2, recs, in, st, g_err);
    if (rc != HC_OK) return rc;
    const double *Y = in, *T = in + nn * nsp, *p = in + nn * (nsp + 1);
    rc = launch_properties(m->dm, n, T, p, Y, haicp ? hc : nullptr, haicp ? hc + nn * nsp : nullptr,
                           DMuKappa ? dmk + nn * nsp : nullptr,
                           DMuKappa ? dmk + nn * (nsp + 1) : nullptr, DMuKappa ? dmk : nullptr, st,
                           g_err);
    if (rc != HC_OK) return rc;
    if (haicp) {
        rc = launch_rows_to_records(n, nsp + 1, nsp + 1, hc, haicp, nullptr, nsp, st, g_err);
        if (rc != HC_OK) return rc;
    }
    if (DMuKappa)
        rc = launch_rows_to_records(n, nsp + 2, nsp + 2, dmk, DMuKappa, nullptr, nsp, st, g_err);
    return rc;
}

static int properties_records_check(hc_mech_t m, int64_t n, const void *recs, const void *a,
                                    const void *b) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (n < 0) return fail(HC_E_INVALID, "negative cell count");
    if (n > 0 && (!recs || (!a && !b))) return fail(HC_E_INVALID, "null field");
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    // the property kernel reads the transport tables (as hc_properties does)
    if (!m->dm.geom || !m->dm.eps_k || !m->dm.sigma)
        return fail(HC_E_INVALID, "mechanism has no transport data");
    return HC_OK;
}

extern "C" {

int hc_properties_aos(hc_mech_t m, int64_t n, const double *YiTP, double *haicp,
                      double *DMuKappa, void *stream) {
    int rc = properties_records_check(m, n, YiTP, haicp, DMuKappa);
    if (rc != HC_OK || n == 0) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    const size_t nn = (size_t)n, nsp = (size_t)m->dm.nsp;
    rc = ensure_ws(m, sizeof(double) * nn * (3 * nsp + 5), st);
    if (rc != HC_OK) return rc;
    return properties_records(m, n, YiTP, haicp, DMuKappa, static_cast<double *>(m->ws), st);
}

int hc_properties_aos_host(hc_mech_t m, int64_t n, const double *YiTP, double *haicp,
                           double *DMuKappa, void *stream) {
    int rc = properties_records_check(m, n, YiTP, haicp, DMuKappa);
    if (rc != HC_OK || n == 0) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(m->mu);
    const size_t nn = (size_t)n, nsp = (size_t)m->dm.nsp;
    // rows (3 nsp + 5) n, then the records in (nsp + 2) n, ha / cp out (nsp + 1) n,
    // D / mu / kappa out (nsp + 2) n
    rc = ensure_ws(m, sizeof(double) * nn * (6 * nsp + 10), st);
    if (rc != HC_OK) return rc;
    double *rows = static_cast<double *>(m->ws);
    double *rin = rows + nn * (3 * nsp + 5), *hout = rin + nn * (nsp + 2), *dout = hout + nn * (nsp + 1);
    HC_CUDA(cudaMemcpyAsync(rin, YiTP, sizeof(double) * nn * (nsp + 2), cudaMemcpyHostToDevice, st));
    rc = properties_records(m, n, rin, haicp ? hout : nullptr, DMuKappa ? dout : nullptr, rows, st);
    if (rc != HC_OK) return rc;
    if (haicp)
        HC_CUDA(cudaMemcpyAsync(haicp, hout, sizeof(double) * nn * (nsp + 1), cudaMemcpyDeviceToHost, st));
    if (DMuKappa)
        HC_CUDA(cudaMemcpyAsync(DMuKappa, dout, sizeof(double) * nn * (nsp + 2), cudaMemcpyDeviceToHost,
                                st));
    HC_CUDA(cudaStreamSynchronize(st));
    return HC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Device state: the fields of a flow's cells resident on the device between
// calls (T, p, rho, Y, the warm-start sub-steps, Ri, per-cell statuses), with
// uploads and downloads in species-major or record-per-cell layouts. One
// allocation laid out [T][Y][rho][p][subdt][Ri][status], so that integration
// records [T, Y..., rho] transpose straight into the first nsp + 2 rows.
// ---------------------------------------------------------------------------
struct hc_state_s {
    hc_mech_t m = nullptr;
    int64_t n = 0;
    void *block = nullptr;
    double *T = nullptr, *Y = nullptr, *rho = nullptr, *p = nullptr, *subdt = nullptr;
    double *Ri = nullptr;
    int32_t *status = nullptr;
    bool warm = false;   // subdt holds warm-start sub-steps
};

namespace {

int state_check(hc_state_t s) {
    if (!s || !s->m) return fail(HC_E_INVALID, "null state");
    return HC_OK;
}

// records (device) of one of the HC_RECORDS_* layouts -> the state's fields
int state_from_records(hc_state_t s, int layout, const double *recs, cudaStream_t st) {
    hc_mech_t m = s->m;
    const int nsp = m->dm.nsp;
    const size_t n = (size_t)s->n;
    if (layout == HC_RECORDS_T_Y_RHO) return launch_records_to_rows(s->n, nsp + 2, recs, s->T, st, g_err);
    int rc = ensure_ws(m, sizeof(double) * n * (nsp + 2), st);
    if (rc != HC_OK) return rc;
    double *rows = static_cast<double *>(m->ws);
    rc = launch_records_to_rows(s->n, nsp + 2, recs, rows, st, g_err);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaMemcpyAsync(s->Y, rows, sizeof(double) * n * nsp, cudaMemcpyDeviceToDevice, st));
    double *a = (layout == HC_RECORDS_Y_RHO_T) ? s->rho : s->T;
    double *b = (layout == HC_RECORDS_Y_RHO_T) ? s->T : s->p;
    HC_CUDA(cudaMemcpyAsync(a, rows + n * nsp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    HC_CUDA(cudaMemcpyAsync(b, rows + n * (nsp + 1), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    return HC_OK;
}

}  // namespace

extern "C" {

int hc_state_create(hc_mech_t m, int64_t ncells, hc_state_t *out) {
    if (!out) return fail(HC_E_INVALID, "null argument");
    *out = nullptr;
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    if (ncells < 1) return fail(HC_E_INVALID, "a state holds at least one cell");
    const size_t n = (size_t)ncells, nsp = (size_t)m->dm.nsp;
    const size_t doubles = n * (4 + 2 * nsp + 1);   // T, Y, rho, p, subdt, Ri
    void *b = nullptr;
    HC_CUDA(cudaMalloc(&b, sizeof(double) * doubles + sizeof(int32_t) * n));
    hc_state_s *s = new hc_state_s();
    s->m = m;
    s->n = ncells;
    s->block = b;
    double *q = static_cast<double *>(b);
    s->T = q;
    s->Y = q + n;
    s->rho = s->Y + n * nsp;
    s->p = s->rho + n;
    s->subdt = s->p + n;
    s->Ri = s->subdt + n;
    s->status = reinterpret_cast<int32_t *>(s->Ri + n * nsp);
    cudaError_t e = cudaMemset(b, 0, sizeof(double) * doubles + sizeof(int32_t) * n);
    if (e != cudaSuccess) {
        cudaFree(b);
        delete s;
        return fail(HC_E_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    }
    *out = s;
    return HC_OK;
}

int hc_state_destroy(hc_state_t s) {
    if (!s) return HC_OK;
    if (s->block) cudaFree(s->block);
    delete s;
    return HC_OK;
}

int hc_state_fields(hc_state_t s, double **T, double **p, double **rho, double **Y,
                    double **subdt, double **Ri, int32_t **status) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    if (T) *T = s->T;
    if (p) *p = s->p;
    if (rho) *rho = s->rho;
    if (Y) *Y = s->Y;
    if (subdt) *subdt = s->subdt;
    if (Ri) *Ri = s->Ri;
    if (status) *status = s->status;
    return HC_OK;
}

int hc_upload(hc_state_t s, const double *T, const double *p, const double *rho, const double *Y,
              const double *subdt, void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->n, nsp = (size_t)s->m->dm.nsp;
    if (T) HC_CUDA(cudaMemcpyAsync(s->T, T, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (p) HC_CUDA(cudaMemcpyAsync(s->p, p, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (rho) HC_CUDA(cudaMemcpyAsync(s->rho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (Y) HC_CUDA(cudaMemcpyAsync(s->Y, Y, sizeof(double) * n * nsp, cudaMemcpyHostToDevice, st));
    if (subdt) {
        HC_CUDA(cudaMemcpyAsync(s->subdt, subdt, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        s->warm = true;
    }
    return HC_OK;
}

int hc_upload_records(hc_state_t s, int layout, const double *recs, const double *p,
                      void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    if (layout < HC_RECORDS_T_Y_RHO || layout > HC_RECORDS_Y_T_P)
        return fail(HC_E_INVALID, "unknown record layout");
    if (!recs) return fail(HC_E_INVALID, "null records");
    hc_mech_t m = s->m;
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->n, rec = (size_t)m->dm.nsp + 2;
    std::lock_guard<std::mutex> lk(m->mu);
    // the host records are staged in the mechanism's workspace behind the rows
    // the transpose of layouts 1 and 2 uses
    rc = ensure_ws(m, sizeof(double) * n * 2 * rec, st);
    if (rc != HC_OK) return rc;
    double *stage = static_cast<double *>(m->ws) + n * rec;
    HC_CUDA(cudaMemcpyAsync(stage, recs, sizeof(double) * n * rec, cudaMemcpyHostToDevice, st));
    rc = state_from_records(s, layout, stage, st);
    if (rc != HC_OK) return rc;
    if (layout == HC_RECORDS_Y_T_P) return HC_OK;   // p came with the records
    if (p) {
        HC_CUDA(cudaMemcpyAsync(s->p, p, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        return HC_OK;
    }
    return launch_ideal_gas_p(s->n, m->dm.nsp, m->dm.W, s->T, s->rho, s->Y, s->p, st, g_err);
}

int hc_download(hc_state_t s, double *T, double *rho, double *Y, double *Ri, double *subdt,
                int32_t *status, void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->n, nsp = (size_t)s->m->dm.nsp;
    if (T) HC_CUDA(cudaMemcpyAsync(T, s->T, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (rho) HC_CUDA(cudaMemcpyAsync(rho, s->rho, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (Y) HC_CUDA(cudaMemcpyAsync(Y, s->Y, sizeof(double) * n * nsp, cudaMemcpyDeviceToHost, st));
    if (Ri) HC_CUDA(cudaMemcpyAsync(Ri, s->Ri, sizeof(double) * n * nsp, cudaMemcpyDeviceToHost, st));
    if (subdt) HC_CUDA(cudaMemcpyAsync(subdt, s->subdt, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (status)
        HC_CUDA(cudaMemcpyAsync(status, s->status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    return HC_OK;
}

int hc_download_records(hc_state_t s, int layout, double *recs, void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    if (layout != HC_RECORDS_T_Y_RHO && layout != HC_RECORDS_Y_RHO_T)
        return fail(HC_E_INVALID, "records of T, Y and rho are layouts 0 and 1");
    if (!recs) return fail(HC_E_INVALID, "null records");
    hc_mech_t m = s->m;
    if (m->dm.nsp + 2 > kAosMaxRec) return fail(HC_E_UNSUPPORTED, "too many species for records");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->n, nsp = (size_t)m->dm.nsp, rec = nsp + 2;
    std::lock_guard<std::mutex> lk(m->mu);
    rc = ensure_ws(m, sizeof(double) * n * 2 * rec, st);
    if (rc != HC_OK) return rc;
    double *rows = static_cast<double *>(m->ws), *out = rows + n * rec;
    const double *src = s->T;
    if (layout == HC_RECORDS_Y_RHO_T) {
        HC_CUDA(cudaMemcpyAsync(rows, s->Y, sizeof(double) * n * nsp, cudaMemcpyDeviceToDevice, st));
        HC_CUDA(cudaMemcpyAsync(rows + n * nsp, s->rho, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        HC_CUDA(cudaMemcpyAsync(rows + n * (nsp + 1), s->T, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                st));
        src = rows;
    }
    rc = launch_rows_to_records(s->n, (int)rec, (int)rec, src, out, nullptr, (int)nsp, st, g_err);
    if (rc != HC_OK) return rc;
    HC_CUDA(cudaMemcpyAsync(recs, out, sizeof(double) * n * rec, cudaMemcpyDeviceToHost, st));
    HC_CUDA(cudaStreamSynchronize(st));
    return HC_OK;
}

int hc_state_integrate(hc_state_t s, const hc_opts *opts, const double *dt, double dt_factor,
                       void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    if (!dt) return fail(HC_E_INVALID, "null dt");
    if (!(dt_factor > 0)) return fail(HC_E_INVALID, "dt_factor must be positive");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!s->warm) {
        // the first flow step starts from dtInit = dt dtFactor (chemistrySource.inl:86-95)
        rc = launch_scaled_copy(s->n, dt, dt_factor, s->subdt, st, g_err);
        if (rc != HC_OK) return rc;
        s->warm = true;
    }
    return integrate_impl(s->m, opts, s->n, s->T, s->p, s->rho, s->Y, dt, dt_factor, s->subdt,
                          s->Ri, s->status, nullptr, nullptr, st);
}

int hc_state_source_terms(hc_state_t s, void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    return hc_source_terms(s->m, s->n, s->T, s->p, s->rho, s->Y, s->Ri, stream);
}

int hc_state_properties(hc_state_t s, double *ha, double *cp, double *mu, double *kappa, double *D,
                        void *stream) {
    int rc = state_check(s);
    if (rc != HC_OK) return rc;
    return hc_properties(s->m, s->n, s->T, s->p, s->Y, ha, cp, mu, kappa, D, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free integration (hc_integrate_noalloc).
//
// For callers that must not allocate device memory during the call: a flow
// solver running under a fixed device-memory budget or a memory pool it
// manages itself, code that calls the chemistry from inside a region where
// the CUDA allocator must not be entered (a host callback, a section holding
// its own allocator's lock), or a real-time loop that cannot afford the
// synchronisation a growing allocation brings. hc_integrate keeps a per-cell
// scratch buffer in the mechanism handle and grows it with cudaMalloc (after
// a stream synchronisation) whenever a call brings more cells than before;
// this entry point never does: its scratch is the file-scope device array
// below, of a fixed size stated by HC_NOALLOC_MAX_CELLS.
//
// Scratch layout: the two previous step states of every cell (ImplicitEuler's
// yklast_, 2 x 16 doubles per cell) for HC_NOALLOC_MAX_CELLS cells, then the
// work-queue head and the six work counters (8 words reserved), which are
// zeroed with cudaMemsetAsync at every call (the per-cell states need no
// initialisation: each is written before it is read). Every call uses the
// same array, so calls that overlap in time (concurrent streams, or several
// host threads) race on it; callers serialise their calls.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocYlast = 2 * 16 * (size_t)HC_NOALLOC_MAX_CELLS;   // doubles
__device__ __align__(256) double g_noalloc_scratch[kNoAllocYlast + 8];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[256] = {};   // the array's device address at the last lookup, per device

}  // namespace

extern "C" int hc_integrate_noalloc(hc_mech_t m, const hc_opts *opts, int64_t ncells, double *T,
                                    const double *p, double *rho, double *Y, const double *dt,
                                    double dt_factor, double *subdt, double *Ri, int32_t *status,
                                    void *stream) {
    if (!m) return fail(HC_E_INVALID, "null mechanism");
    int rc = check_opts(opts);
    if (rc != HC_OK) return rc;
    if (ncells < 0) return fail(HC_E_INVALID, "negative cell count");
    if (ncells > HC_NOALLOC_MAX_CELLS)
        return fail(HC_E_INVALID, "hc_integrate_noalloc takes at most HC_NOALLOC_MAX_CELLS (" +
                                      std::to_string(HC_NOALLOC_MAX_CELLS) + ") cells per call, got " +
                                      std::to_string(ncells));
    if (ncells == 0) return HC_OK;
    if (!T || !p || !rho || !Y || !dt || !subdt) return fail(HC_E_INVALID, "null field");
    if (!(dt_factor > 0)) return fail(HC_E_INVALID, "dt_factor must be positive");
    const int N = m->dm.nsp + 1;
    if (N > 16 || opts->auto_update_jacobian || !m->t2_ok || opts->reactor != 0)
        return fail(HC_E_UNSUPPORTED,
                    "hc_integrate_noalloc needs nsp <= 15, <= 64 reactions, autoUpdateJacobian off, "
                    "the constant-pressure reactor and no SRI, explicit reverse (REV), PLOG, HIGH, "
                    "LT, JAN, FIT1 or collision rate laws");
    int dev = -1;
    HC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(HC_E_CUDA, "device ordinal out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void *base = nullptr;
    {
        // the array's address: looked up at every call outside a stream
        // capture (a new context after cudaDeviceReset places the array
        // anew), and taken from the last lookup on this device during a
        // capture (no context can be reset while one is open)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        HC_CUDA(cudaStreamIsCapturing(st, &cs));
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (cs == cudaStreamCaptureStatusNone || !g_noalloc_addr[dev]) {
            void *a = nullptr;
            HC_CUDA(cudaGetSymbolAddress(&a, g_noalloc_scratch));
            g_noalloc_addr[dev] = a;
        }
        base = g_noalloc_addr[dev];
    }
    double *ylast = static_cast<double *>(base);
    unsigned long long *queue = reinterpret_cast<unsigned long long *>(ylast + kNoAllocYlast);
    HC_CUDA(cudaMemsetAsync(queue, 0, 8 * sizeof(unsigned long long), st));
    CellIO io;
    io.ncells = ncells;
    io.nqueue = ncells;
    io.T = T;
    io.p = p;
    io.rho = rho;
    io.Y = Y;
    io.dt = dt;
    io.dt_factor = dt_factor;
    io.subdt = subdt;
    io.Ri = Ri;
    io.status = status;
    io.order = nullptr;
    io.cost = nullptr;
    io.queue_head = queue;
    io.counters = queue + 1;
    const IntegratorParams P = make_params(opts);
    return variant_integrate_t2(N, m->t2, m->num_sms, P, io, ylast, m->block, st, g_err);
}
