// Definitions shared by the precompiled kernels and the kernels generated
// and compiled at run time for one mechanism (NVRTC): physical constants,
// scalar helpers, rate-law formulas with their parameters passed by value,
// and the integrator's parameter / field structures. Nothing here reads the
// mechanism tables.
#pragma once

#ifndef __CUDACC_RTC__
#include <cstdint>
#include <cuda_runtime.h>
#else
typedef int int32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#endif

namespace hc {

constexpr double kTiny = 1.0e-15;          // doubleRealTiny (doubleReal.hpp:43)
constexpr double kVeryTiny = 1.0e-300;     // doubleRealVeryTiny
constexpr double kVeryLarge = 1.0e+300;    // doubleRealVeryLarge
constexpr double kRootVeryLarge = 1.0e+150;
constexpr double kPatm = 1.01325e5;        // physicalConstant.hpp:186
// Ru = (kB * NA) * 1e3 [J/kmol/K], evaluated like physicalConstant.hpp:158,183
constexpr double kRu = (1.380649e-23 * 6.02214076e23) * 1e3;
constexpr int kMaxSide = 4;

enum RateType : int32_t {
    kArrhenius = 0, kThirdBody = 1, kLindemann = 2, kTroe3 = 3, kTroe4 = 4, kSRI = 5, kPLOG = 6,
    kLandauTeller = 7, kJanev = 8, kPowerSeries = 9, kCollision = 10
};
// reversible flags: 1 kr = kf / Kc, 2 kr from explicit reverse Arrhenius parameters
constexpr int32_t kRevExplicit = 2;

__device__ __forceinline__ double hmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double hmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double notZeroD(double s) { return (s != 0) ? s : kVeryTiny; }
__device__ __forceinline__ bool finite(double x) { return !isnan(x) && !isinf(x); }

// x^y, with the exponents mechanisms use in practice done exactly as a
// correctly rounded pow returns them (y = 1: x; y = 2: one rounded multiply;
// y = 0: 1; y = -1: one rounded division); any other exponent calls pow().
// pow() out of line: one copy per kernel however many call sites use it
// (the inline expansion is a few KB of instructions per site)
#if defined(__CUDACC__) || defined(__CUDACC_RTC__)
#define HC_NOINLINE __noinline__
#else
#define HC_NOINLINE __attribute__((noinline))   // host builds of the device code
#endif
static __device__ HC_NOINLINE double pow_out(double x, double y) { return pow(x, y); }

__device__ __forceinline__ double pow_n(double x, double y) {
    if (y == 1.0) return x;
    if (y == 2.0) return x * x;
    if (y == 0.0) return 1.0;
    if (y == -1.0) return 1.0 / x;
    return pow_out(x, y);
}

// 1/b without a branch to a slow path: the hardware approximation (PTX
// rcp.approx.ftz.f64) refined by three Newton-Raphson steps r <- r + r (1 - b r),
// each of which doubles the number of correct bits (Markstein, IBM J. Res.
// Dev. 34 (1990) 111-119); the result is within a few ulp of the correctly
// rounded reciprocal. Zero, infinity and NaN keep the approximation's own
// result (+-inf, +-0, NaN), as do subnormal b (flushed: +-inf).
__device__ __forceinline__ double frcp(double b) {
#ifdef __CUDA_ARCH__
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double x = r;
    x = fma(x, fma(-b, x, 1.0), x);
    x = fma(x, fma(-b, x, 1.0), x);
    x = fma(x, fma(-b, x, 1.0), x);
    return (r != 0.0 && !isinf(r)) ? x : r;
#else
    return 1.0 / b;   // host builds of the device code (arithmetic checks on the CPU)
#endif
}

// a / b as a * frcp(b) (at most a few ulp from the correctly rounded quotient)
__device__ __forceinline__ double fdiv(double a, double b) { return a * frcp(b); }

// x^y for x > 0 as exp(y ln x), without pow's out-of-line accurate path
__device__ __forceinline__ double fpow_pos(double x, double y) { return exp(y * log(x)); }

__device__ __forceinline__ double conc_pow(double c, double ord) {
    return pow_n(hmax(c, 0.0), ord);
}

// ---------------------------------------------------------------- rate laws
// ArrheniusRR::k (ArrheniusRR.cpp:37-47), A T^b e^{-Ta/T}, evaluated as one
// exponential of b ln T - Ta/T with ln T shared by all reactions of a cell.
__device__ __forceinline__ double arrK_log(double A, double b, double Ta, double T, double logT) {
    double e = 0.0;
    if (fabs(b) > kVeryTiny) e = b * logT;
    if (fabs(Ta) > kVeryTiny) e -= Ta / T;
    return A * exp(e);
}

__device__ __forceinline__ double troe_logfcent_p(double alpha, double Tsss, double Ts, double Tss,
                                                  bool four, double T) {
    double s = (1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts);
    if (four) s += exp(-Tss / T);
    return log10(hmax(s, kTiny));
}

// fallOffFunctions.cpp:81-100 (Troe::F); Lindemann F = 1
__device__ __forceinline__ double fall_F(int type, double logFcent, double Pr) {
    if (type == kLindemann) return 1.0;
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPr = log10(hmax(Pr, kTiny));
    const double x = (logPr + c) / (n - d * (logPr + c));
    return pow(10.0, logFcent / (1.0 + x * x));
}

// The Pr-independent product of Troe::DFDci (fallOffFunctions.cpp:102-129):
// DFDci = [F * A * B * C] * (1/Pr * dPr/dci); returns F*A*B*C.
__device__ __forceinline__ double troe_dfdci_factor(int type, double logFcent, double Pr,
                                                    double F) {
    if (type == kLindemann) return 0.0;
    const double logPr = log10(hmax(Pr, kTiny));
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPrpc = logPr + c;
    const double nm = n - d * logPrpc;
    const double inv = logPrpc / nm;
    const double s1 = 1.0 + inv * inv;
    return F * ((-logFcent) / (s1 * s1)) * (2.0 * logPrpc / (nm * nm)) * (1.0 + d * inv);
}

// Troe::DFDT (fallOffFunctions.cpp:131-157)
__device__ __forceinline__ double troe_dfdt_p(int type, double alpha, double Tsss, double Ts,
                                              double Tss, double T, double Pr, double F,
                                              double DPrDT) {
    if (type == kLindemann) return 0.0;
    const double ln10 = log(10.0);
    const double logPr = log10(hmax(Pr, kTiny));
    double Fcent, DFcentDT;
    const double e1 = exp(-T / Tsss), e2 = exp(-T / Ts);
    if (type == kTroe3) {
        Fcent = hmax((1.0 - alpha) * e1 + alpha * e2, kTiny);
        DFcentDT = (1.0 - alpha) * e1 / (-Tsss) + alpha * e2 / (-Ts);
    } else {
        const double e3 = exp(-Tss / T);
        Fcent = hmax((1.0 - alpha) * e1 + alpha * e2 + e3, kTiny);
        DFcentDT = (1.0 - alpha) * e1 / (-Tsss) + alpha * e2 / (-Ts) + e3 * (Tss / (T * T));
    }
    const double logFcent = log10(Fcent);
    const double DlogFcentDT = 1.0 / (Fcent * ln10) * DFcentDT;
    const double c = -0.4 - 0.67 * logFcent;
    const double DcDT = -0.67 * DlogFcentDT;
    const double n = 0.75 - 1.27 * logFcent;
    const double DnDT = -1.27 * DlogFcentDT;
    const double d = 0.14;
    const double dlogPrDT = DPrDT / Pr / ln10;
    const double logPrpc = logPr + c;
    const double nm = n - d * logPrpc;
    const double inv = logPrpc / nm;
    const double dPPDT =
        2.0 * logPrpc / (nm * nm) * ((dlogPrDT + DcDT) - logPrpc / nm * (DnDT - d * (dlogPrDT + DcDT)));
    const double s1 = 1.0 + inv * inv;
    return (F * ln10 * (DlogFcentDT / s1 - logFcent / (s1 * s1) * dPPDT));
}

// SRI fall-off function (fallOffFunctions.cpp:54-61, parameters a, b, c, d, e):
//   F = d [a e^{-b/T} + e^{-T/c}]^X T^e,  X = 1 / (1 + log10(max(Pr, tiny))^2)
__device__ __forceinline__ double sri_base(const double *s, double T) {
    return s[0] * exp(-s[1] / T) + exp(-T / s[2]);
}

__device__ __forceinline__ double sri_F(const double *s, double T, double Pr) {
    const double logPr = log10(hmax(Pr, kTiny));
    const double X = 1.0 / (1.0 + logPr * logPr);
    return s[3] * pow(sri_base(s, T), X) * pow(T, s[4]);
}

// The factor f of SRI::DFDci (fallOffFunctions.cpp:63-69) written as
// DFDci = f * (1/Pr * dPr/dci):
// f = F * (-2 X^2 log10(Pr) / ln 10) * ln(a e^{-b/T} + e^{-T/c})
__device__ __forceinline__ double sri_dfdci_factor(const double *s, double T, double Pr,
                                                   double F) {
    const double lp = log10(hmax(Pr, kTiny));
    const double X = 1.0 / (1.0 + lp * lp);
    return F * (-X * X * 2.0 * log10(Pr) / log(10.0)) * log(sri_base(s, T));
}

// SRI::DFDT (fallOffFunctions.cpp:71-79)
__device__ __forceinline__ double sri_dfdt(const double *s, double T, double Pr, double F,
                                           double DPrDT) {
    const double lp = log10(hmax(Pr, kTiny));
    const double X = 1.0 / (1.0 + lp * lp);
    const double dXdPr = -X * X * 2.0 * log10(Pr) / Pr / log(10.0);
    const double eb = exp(-s[1] / T), ec = exp(-T / s[2]);
    const double base = s[0] * eb + ec;
    return F * (s[4] / T + dXdPr * DPrDT * log(base) +
                X * (s[0] * s[1] * eb / (T * T) - ec / s[2]) / base);
}

// PLOG (logInterpolationRR::k and ::DkDT, logInterpolationRR.cpp:78-147,
// 149-226) over one reaction's table: pressures pp[n] (Pa, sorted, the two
// highest distinct) and Arrhenius entries pa[3n]. Below the table the rates
// of the entries at the lowest pressure add, above it the highest entry is
// taken; inside, the reference's loop over intervals does not stop at the
// first that brackets p, so the interval it evaluates last -- the two
// highest pressures, with the entries sharing the lower of them added --
// is the one used, interpolated (or extrapolated) in ln p.
__device__ __forceinline__ double plog_entry_dkdt(const double *a, double kj, double T) {
    const double invT = 1.0 / hmax(T, kTiny);
    return kj * invT * (a[1] + a[2] * invT);
}

__device__ __forceinline__ double plog_k(const double *pp, const double *pa, int n, double p,
                                         double T, double logT) {
    if (p <= pp[0]) {
        double k = arrK_log(pa[0], pa[1], pa[2], T, logT);
        for (int i = 0; i < n - 1; ++i) {
            if (pp[i + 1] > pp[i]) break;
            k += arrK_log(pa[3 * (i + 1)], pa[3 * (i + 1) + 1], pa[3 * (i + 1) + 2], T, logT);
        }
        return k;
    }
    if (p >= pp[n - 1]) return arrK_log(pa[3 * (n - 1)], pa[3 * (n - 1) + 1], pa[3 * (n - 1) + 2], T, logT);
    const int i = n - 2;
    double k0 = arrK_log(pa[3 * i], pa[3 * i + 1], pa[3 * i + 2], T, logT);
    for (int j = i - 1; j >= 0; --j) {
        if (pp[j + 1] > pp[j]) break;
        k0 += arrK_log(pa[3 * j], pa[3 * j + 1], pa[3 * j + 2], T, logT);
    }
    const double k1 = arrK_log(pa[3 * (i + 1)], pa[3 * (i + 1) + 1], pa[3 * (i + 1) + 2], T, logT);
    const double lnk0 = log(k0), lnk1 = log(k1);
    const double lnp0 = log(pp[i]), lnp1 = log(pp[i + 1]), lnp = log(p);
    return exp(lnk0 + (lnk1 - lnk0) * (lnp - lnp0) / (lnp1 - lnp0));
}

__device__ __forceinline__ double plog_dkdt(const double *pp, const double *pa, int n, double kj,
                                            double p, double T, double logT) {
    if (p <= pp[0]) {
        double d = plog_entry_dkdt(&pa[0], arrK_log(pa[0], pa[1], pa[2], T, logT), T);
        for (int i = 0; i < n - 1; ++i) {
            if (pp[i + 1] > pp[i]) break;
            const double *a = &pa[3 * (i + 1)];
            d += plog_entry_dkdt(a, arrK_log(a[0], a[1], a[2], T, logT), T);
        }
        return d;
    }
    if (p >= pp[n - 1]) {
        const double *a = &pa[3 * (n - 1)];
        return plog_entry_dkdt(a, arrK_log(a[0], a[1], a[2], T, logT), T);
    }
    const int i = n - 2;
    double k0 = arrK_log(pa[3 * i], pa[3 * i + 1], pa[3 * i + 2], T, logT);
    double dk0 = plog_entry_dkdt(&pa[3 * i], k0, T);
    for (int j = i - 1; j >= 0; --j) {
        if (pp[j + 1] > pp[j]) break;
        const double kj0 = arrK_log(pa[3 * j], pa[3 * j + 1], pa[3 * j + 2], T, logT);
        k0 += kj0;
        dk0 += plog_entry_dkdt(&pa[3 * j], kj0, T);
    }
    const double *a1 = &pa[3 * (i + 1)];
    const double k1 = arrK_log(a1[0], a1[1], a1[2], T, logT);
    const double dk1 = plog_entry_dkdt(a1, k1, T);
    const double lnp0 = log(pp[i]), lnp1 = log(pp[i + 1]), lnp = log(p);
    const double dlnkdT = 1.0 / k0 * dk0 + (1.0 / k1 * dk1 - 1.0 / k0 * dk0) * (lnp - lnp0) / (lnp1 - lnp0);
    return kj * dlnkdT;
}

// Landau-Teller (LandauTellerRR::k, ::DkDT, LandauTellerRR.cpp:37-99):
// k = A T^b exp(-Ta/T + B T^(-1/3) + C T^(-2/3)),
// dk/dT = k (b + Ta/T - B T^(-1/3) / 3 - 2 C T^(-2/3) / 3) / T
__device__ __forceinline__ double lt_k(double A, double b, double Ta, double B, double C, double T,
                                       double logT) {
    double e = 0.0;
    if (fabs(b) > kVeryTiny) e = b * logT;
    if (fabs(Ta) > kVeryTiny) e -= Ta / T;
    if (fabs(B) > kVeryTiny) e += B / cbrt(T);
    if (fabs(C) > kVeryTiny) e += C / pow(T, 2.0 / 3.0);
    return A * exp(e);
}

__device__ __forceinline__ double lt_dkdt(double k, double b, double Ta, double B, double C,
                                          double T) {
    double d = 0.0;
    if (fabs(Ta) > kVeryTiny) d += Ta / T;
    if (fabs(B) > kVeryTiny) d -= (B / cbrt(T)) / 3.0;
    if (fabs(C) > kVeryTiny) d -= 2.0 * (C / pow(T, 2.0 / 3.0)) / 3.0;
    return k * (b + d) / T;
}

// Janev (JanevRR.cpp:37-88): k = A T^b exp(-Ta/T + sum_{n<9} b_n (ln T)^n),
// dk/dT = k (b + Ta/T + b_1 + sum_{n>=2} n b_n (ln T)^(n-1)) / T
__device__ __forceinline__ double janev_k(double A, double b, double Ta, const double *bn, double T,
                                          double logT) {
    double e = 0.0;
    if (fabs(b) > kVeryTiny) e = b * logT;
    if (fabs(Ta) > kVeryTiny) e -= Ta / T;
    double lp = 1.0;
    for (int n = 0; n < 9; ++n) {
        e += bn[n] * lp;
        lp *= logT;
    }
    return A * exp(e);
}

__device__ __forceinline__ double janev_dkdt(double k, double b, double Ta, const double *bn,
                                             double T, double logT) {
    double d = bn[1], lp = 1.0;
    for (int n = 2; n < 9; ++n) {
        lp *= logT;
        d += n * bn[n] * lp;
    }
    return k * (b + Ta / T + d) / T;
}

// collision efficiency (collisionRR.hpp:94-107, 146-169, collisionRR.cpp:36-46):
// k = min(1, A T^b exp(-Ta/T)) Z(T), Z = N_A d^2 sqrt(8 pi (Ru / W_AB) T), and
// dk/dT = (k > 1 ? k (b + Ta/T) / T : 0) N_A d^2 sqrt(2 pi (Ru / W_AB) / T), both as
// the reference states them; x = (N_A d^2, 8 pi Ru / W_AB, 2 pi Ru / W_AB)
__device__ __forceinline__ double collision_k(double A, double b, double Ta, const double *x,
                                              double T, double logT) {
    const double g = arrK_log(A, b, Ta, T, logT);   // std::min(1, g)
    return (g < 1.0 ? g : 1.0) * (x[0] * sqrt(x[1] * T));
}

__device__ __forceinline__ double collision_dkdt(double k, double b, double Ta, const double *x,
                                                 double T) {
    const double invT = 1.0 / hmax(T, kTiny);
    return (k > 1.0 ? k * invT * (b + Ta * invT) : 0.0) * (x[0] * sqrt(x[2] / T));
}

// power series (powerSeriesRateRR.cpp:37-74): k = A T^b exp(sum_{n<4} b_n / T^(n+1)),
// dk/dT = k (b - sum_{n<4} (n+1) b_n / T^(n+1)) / T
__device__ __forceinline__ double pseries_k(double A, double b, const double *bn, double T,
                                            double logT) {
    double e = 0.0;
    if (fabs(b) > kVeryTiny) e = b * logT;
    double ti = 1.0 / T, tp = ti;
    for (int n = 0; n < 4; ++n) {
        e += bn[n] * tp;
        tp *= ti;
    }
    return A * exp(e);
}

__device__ __forceinline__ double pseries_dkdt(double k, double b, const double *bn, double T) {
    double d = 0.0, ti = 1.0 / T, tp = ti;
    for (int n = 0; n < 4; ++n) {
        d -= (n + 1) * bn[n] * tp;
        tp *= ti;
    }
    return k * (b + d) / T;
}

struct IntegratorParams {
    int32_t maxstep;
    int32_t auto_update_jacobian;
    int32_t step_to_update_jac;
    double atol, rtol, safescale, minscale, maxscale, alphainc;
    double atol_inc, rtol_inc, T_threshold, T_alpha, T_beta, dt_max;
    double err_accept_limit;     // pow(maxscale/safescale, -1/alphainc)
    int64_t max_newton_total;
    int32_t reactor;             // 0 constant pressure, 1 constant volume (cell group only)
};

struct CellIO {
    int64_t ncells;         // field length (stride of species fields)
    int64_t nqueue;         // cells to integrate: queue entries 0..nqueue-1
    double *T;
    const double *p;
    double *rho;
    double *Y;              // [nsp][ncells]
    const double *dt;
    double dt_factor;
    double *subdt;
    double *Ri;             // optional [nsp][ncells]
    int32_t *status;        // optional
    const int32_t *order;   // optional queue order (cell indices)
    int64_t *cost;          // optional per-cell Newton iteration count out
    unsigned long long *queue_head;
    unsigned long long *counters;  // [6] n_jac, n_rhs, n_lu, n_newton, n_steps, n_attempts
};

}  // namespace hc
