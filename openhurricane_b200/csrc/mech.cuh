// Device-side mechanism tables and the per-species / per-reaction kinetics
// functions shared by the integrator, source-term and property kernels.
//
// Every function restates the reference's CPU formula (file:line cited at
// each) in FP64. Floating-point operations keep the reference's order where
// that is natural on the GPU; remaining differences are the CUDA libm
// (exp/log/pow within a few ulp of glibc), FMA contraction and the fused
// Arrhenius form noted at arrK_log.
#pragma once

#include "rtc_base.cuh"

namespace hc {

struct DevMech {
    int32_t nsp, nrc;
    const double *W;        // [nsp]
    const double *Trange;   // [nsp*3]
    const double *nasa;     // [nsp*14] low a0..a6, high a0..a6 (mass basis)
    const int32_t *rate_type, *reversible;
    const double *arr, *arr0, *troe;  // [nrc*3], [nrc*3], [nrc*4]
    const double *sri, *arr_rev;      // [nrc*5] SRI a..e, [nrc*3] explicit reverse Arrhenius
    int32_t ext;                      // any SRI, REV, PLOG, HIGH or LT reaction
    const int32_t *activated;         // [nrc] chemically activated bimolecular (HIGH)
    const double *lt;                 // [nrc*2] Landau-Teller B, C
    const double *xcoef;              // [nrc*9] Janev / power-series coefficients
    const int32_t *plog_ptr;          // [nrc+1] PLOG entries of each reaction
    const double *plog_p, *plog_arr;  // [n] Pa, [n*3] A, beta, Ta
    const double *eff;      // [nrc*nsp]
    const int32_t *nf, *nb; // [nrc]
    const int32_t *fidx, *bidx;       // [nrc*4]
    const double *ford, *bord;        // [nrc*4]
    const double *fnu, *bnu;          // [nrc*4]
    const double *sum_stoi;           // [nrc]
    // participation lists per species (sorted by reaction): coef = -fnu (reactant) / +bnu (product)
    const int32_t *sp_ptr;  // [nsp+1]
    const int32_t *sp_rxn;  // [npart]
    const double *sp_coef;  // [npart]
    // kinetic-theory transport
    const int32_t *geom;
    const double *eps_k, *sigma;
    // pair constants of the mixture-averaged transport, [nsp*nsp] (i*nsp + j)
    const double *pair_D;     // 1.858e-7 sqrt(1/Wi + 1/Wj) / sigma_ij^2 * Patm
    const double *pair_Dpow;  // (1/sqrt(eps_i eps_j))^-0.145
    const double *pair_r;     // 1/sqrt(eps_i eps_j)
    const double *pair_phi;   // (1/sqrt 8) / sqrt(1 + Wi/Wj)
    const double *pair_w;     // sqrt(Wi/Wj)
};

template <typename V>
__device__ __forceinline__ V ldg(const V *p) {
    return __ldg(p);
}

// ---------------------------------------------------------------- thermo
// JANAF (thermo/src/JANAF.cpp:142-219, thermo/include/JANAF.inl:33-86).
struct SpeciesThermo {
    double cp;     // molar Cp  (Cp0 = cp0 * W, thermo.inl:44)
    double h;      // molar H   (Ha0)
    double dcp;    // molar dCp/dT (JANAF::Dcp_pDT * W)
    double G0;     // molar Gibbs (JANAF::g0 * W)
    double DG0DT;  // molar dG/dT (thermo.inl:197-203)
};

__device__ __forceinline__ SpeciesThermo species_thermo(const DevMech &m, int i, double T,
                                                        double logT) {
    const double tl = ldg(&m.Trange[3 * i]), tc = ldg(&m.Trange[3 * i + 1]);
    const double th = ldg(&m.Trange[3 * i + 2]);
    const double *a = (T < tc) ? &m.nasa[14 * i] : &m.nasa[14 * i + 7];
    const double a0 = ldg(&a[0]), a1 = ldg(&a[1]), a2 = ldg(&a[2]), a3 = ldg(&a[3]);
    const double a4 = ldg(&a[4]), a5 = ldg(&a[5]), a6 = ldg(&a[6]);
    const double W = ldg(&m.W[i]);
    const bool out = (T < tl || T > th);
    const double T0 = out ? hmin(hmax(T, tl), th) : T;
    const double cp0 = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
    double h0 = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
    if (out) h0 += cp0 * (T - T0);
    // s0 and g0 use the unclamped T (JANAF.cpp:201-213); log(max(T, tiny))
    const double lT = (T > kTiny) ? logT : log(kTiny);
    const double s0 = ((((a4 / 4.0 * T + a3 / 3.0) * T + a2 / 2.0) * T + a1) * T + a0 * lT + a6);
    const double g0 = (((((-a4 / 20.0 * T - a3 / 12.0) * T - a2 / 6.0) * T - a1 / 2.0) * T +
                        a0 * (1 - lT) - a6) * T + a5);
    const double ds0 = (a0 / hmax(T, kTiny) + a1 + (a2 + (a3 + a4 * T) * T) * T);
    const double dcp = (a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T)));
    SpeciesThermo r;
    r.cp = cp0 * W;
    r.h = h0 * W;
    r.dcp = dcp * W;
    r.G0 = g0 * W;
    r.DG0DT = (cp0 - (s0 + T * ds0)) * W;
    return r;
}

// mass-basis cp0 and ha0 only (property kernels)
__device__ __forceinline__ void species_cp_h(const DevMech &m, int i, double T, double &cp,
                                             double &h) {
    const double tl = ldg(&m.Trange[3 * i]), tc = ldg(&m.Trange[3 * i + 1]);
    const double th = ldg(&m.Trange[3 * i + 2]);
    const double *a = (T < tc) ? &m.nasa[14 * i] : &m.nasa[14 * i + 7];
    const double a0 = ldg(&a[0]), a1 = ldg(&a[1]), a2 = ldg(&a[2]), a3 = ldg(&a[3]);
    const double a4 = ldg(&a[4]), a5 = ldg(&a[5]);
    const bool out = (T < tl || T > th);
    const double T0 = out ? hmin(hmax(T, tl), th) : T;
    cp = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
    h = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
    if (out) h += cp * (T - T0);
}

// Rate forms that only some mechanisms use (SRI fall-off, explicit reverse
// Arrhenius parameters), kept out of line so that the integrator's register
// allocation for the common forms does not carry them; parameters are read
// from the global tables.
static __device__ __noinline__ double sri_F_global(const double *s, double T, double Pr) {
    const double p[5] = {ldg(&s[0]), ldg(&s[1]), ldg(&s[2]), ldg(&s[3]), ldg(&s[4])};
    return sri_F(p, T, Pr);
}

static __device__ __noinline__ double sri_dfdt_global(const double *s, double T, double Pr, double F,
                                               double DPrDT) {
    const double p[5] = {ldg(&s[0]), ldg(&s[1]), ldg(&s[2]), ldg(&s[3]), ldg(&s[4])};
    return sri_dfdt(p, T, Pr, F, DPrDT);
}

static __device__ __noinline__ double sri_dfdci_factor_global(const double *s, double T, double Pr,
                                                       double F) {
    const double p[5] = {ldg(&s[0]), ldg(&s[1]), ldg(&s[2]), ldg(&s[3]), ldg(&s[4])};
    return sri_dfdci_factor(p, T, Pr, F);
}

static __device__ __noinline__ double plog_k_global(const int32_t *ptr, const double *pp,
                                                   const double *pa, int r, double p, double T,
                                                   double logT) {
    const int b = ldg(&ptr[r]), n = ldg(&ptr[r + 1]) - b;
    return plog_k(&pp[b], &pa[3 * b], n, p, T, logT);
}

static __device__ __noinline__ double plog_dkdt_global(const int32_t *ptr, const double *pp,
                                                      const double *pa, int r, double kj,
                                                      double p, double T, double logT) {
    const int b = ldg(&ptr[r]), n = ldg(&ptr[r + 1]) - b;
    return plog_dkdt(&pp[b], &pa[3 * b], n, kj, p, T, logT);
}

static __device__ __noinline__ double lt_k_global(const double *a, const double *bc, double T,
                                                 double logT) {
    return lt_k(ldg(&a[0]), ldg(&a[1]), ldg(&a[2]), ldg(&bc[0]), ldg(&bc[1]), T, logT);
}

static __device__ __noinline__ double lt_dkdt_global(const double *a, const double *bc, double k,
                                                    double T) {
    return lt_dkdt(k, ldg(&a[1]), ldg(&a[2]), ldg(&bc[0]), ldg(&bc[1]), T);
}

// Janev, power-series and collision rates: a = A, beta, Ta; x = the reaction's 9 coefficients
static __device__ __noinline__ double xrate_k_global(int type, const double *a, const double *x,
                                                    double T, double logT) {
    double bn[9];
    for (int n = 0; n < 9; ++n) bn[n] = ldg(&x[n]);
    if (type == kJanev) return janev_k(ldg(&a[0]), ldg(&a[1]), ldg(&a[2]), bn, T, logT);
    if (type == kCollision) return collision_k(ldg(&a[0]), ldg(&a[1]), ldg(&a[2]), bn, T, logT);
    return pseries_k(ldg(&a[0]), ldg(&a[1]), bn, T, logT);
}

static __device__ __noinline__ double xrate_dkdt_global(int type, const double *a, const double *x,
                                                       double k, double T, double logT) {
    double bn[9];
    for (int n = 0; n < 9; ++n) bn[n] = ldg(&x[n]);
    if (type == kJanev) return janev_dkdt(k, ldg(&a[1]), ldg(&a[2]), bn, T, logT);
    if (type == kCollision) return collision_dkdt(k, ldg(&a[1]), ldg(&a[2]), bn, T);
    return pseries_dkdt(k, ldg(&a[1]), bn, T);
}

static __device__ __noinline__ double arr_global(const double *a, double T, double logT) {
    return arrK_log(ldg(&a[0]), ldg(&a[1]), ldg(&a[2]), T, logT);
}

__device__ __forceinline__ double troe_logfcent(const double *tr, bool four, double T) {
    return troe_logfcent_p(ldg(&tr[0]), ldg(&tr[1]), ldg(&tr[2]), ldg(&tr[3]), four, T);
}

__device__ __forceinline__ double troe_dfdt(int type, const double *tr, double T, double Pr,
                                            double F, double DPrDT) {
    return troe_dfdt_p(type, ldg(&tr[0]), ldg(&tr[1]), ldg(&tr[2]), ldg(&tr[3]), T, Pr, F, DPrDT);
}

// Equilibrium constants (reactionTypes.cpp:178-241) from molar G0 / DG0DT
// read through accessors (shared memory layouts differ between kernels).
struct EquilK {
    double Kc, DKcDT;
};

template <typename GAt, typename DAt>
__device__ __forceinline__ EquilK equilibrium(const DevMech &m, int r, double T, GAt G0, DAt DG0) {
    double kp = 0.0, dk = 0.0;
    const double Tm = hmax(T, kTiny);
    const int nf = ldg(&m.nf[r]), nb = ldg(&m.nb[r]);
#pragma unroll
    for (int k = 0; k < kMaxSide; ++k) {
        if (k < nf) {
            const int i = ldg(&m.fidx[kMaxSide * r + k]);
            const double nu = ldg(&m.fnu[kMaxSide * r + k]);
            const double G = G0(i);
            kp -= G * nu;
            dk -= (DG0(i) - G / Tm) * nu;
        }
    }
#pragma unroll
    for (int k = 0; k < kMaxSide; ++k) {
        if (k < nb) {
            const int i = ldg(&m.bidx[kMaxSide * r + k]);
            const double nu = ldg(&m.bnu[kMaxSide * r + k]);
            const double G = G0(i);
            kp += G * nu;
            dk += (DG0(i) - G / Tm) * nu;
        }
    }
    kp /= (Tm * kRu);
    double Kp = exp(-kp);
    if (!finite(Kp)) Kp = kRootVeryLarge;
    dk /= (Tm * kRu);
    double DKp = Kp * dk;
    if (!finite(DKp)) DKp = kVeryLarge;
    const double s = ldg(&m.sum_stoi[r]);
    EquilK e;
    if (fabs(s) < kVeryTiny) {
        e.Kc = Kp;
        e.DKcDT = DKp;
    } else {
        const double f = pow_n(kPatm / (kRu * T), s);
        e.Kc = hmin(Kp * f, kVeryLarge);
        double v = (DKp + Kp * (-s) / T) * f;
        if (!finite(v)) v = kVeryLarge;
        e.DKcDT = v;
    }
    return e;
}

}  // namespace hc
