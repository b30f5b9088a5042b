// Warp-per-cell implicit-Euler integrator (kernel 6) for mechanisms of
// N = nsp + 1 <= 16 unknowns, FP64.
//
// One warp integrates one cell at a time and takes the next cell from the
// device work queue (the grid is persistent). The per-cell control flow is
// the reference's (chemistrySource.cpp:1511-1555, ImplicitEuler.cpp:101-342,
// ODEsSolver.cpp:148-225), uniform across the warp. Each Newton iteration:
//
//  * species: lane i evaluates species i (NASA-7, molar, from coefficients
//    pre-multiplied on the host) and publishes c_i, h_i, exp(+-G0_i/(Ru T))
//    to the warp's shared memory;
//  * reactions: lane r evaluates reaction r (r = lane + 32 k): kf, kr (1/Kc as a
//    product of the species' exp(+-G0/(Ru T))), q, dq/dT, the third-body /
//    fall-off factor and dq/dc of each participant, and writes them as a
//    record to shared memory;
//  * rows: lanes i, i + 11 and i + 22 (N <= 11; i and i + 16 above) walk
//    the list of reactions species i takes part in (mechanism order; every
//    third or second entry each) and sum its row of f and of the Jacobian
//    (rows in shared memory, the columns the reaction's participants), the
//    temperature column entry and its entry of the temperature row
//    (sum_r dH_r dq_r/dc_i, dH_r = sum nu h); the partial sums are then
//    added in lane order;
//  * LU: lane i holds row i of I - dt J in registers; partial pivoting picks
//    the first largest |a(k)| in the current row order (warp max reductions
//    of its bit pattern, then a min reduction of the logical position) and
//    broadcasts the pivot row by shuffles; rows are never moved, each lane
//    keeps its logical position;
//  * the triangular solves run along the logical order with shuffles.
//
// No division on the common path except one reciprocal per pivot, T and the
// mixture heat capacity (frcp). Tables are read through the read-only data
// cache in layouts where the 32 lanes of a warp read 32 consecutive values.
// Cells with a temperature outside some species' fitted range or with a
// |G0/(Ru T)| too large for the product form take the reference's own
// clamped forms for the thermo and the equilibrium constants (warp-uniform
// branch).
#pragma once

#include "integrator.cuh"
#include "t3_base.cuh"

namespace hc {

// reaction fields of WMech::rd (doubles) and ::ri (ints), field-major over reactions
enum WRD : int {
    kWA = 0, kWb, kWTa, kWA0, kWb0, kWTa0, kWalpha, kWiTsss, kWiTs, kWTss, kWTsss, kWTs, kWs,
    kWnu,                      // nu[8]: -fnu (reactants) then +bnu (products)
    kWord = kWnu + 8,          // ord[8]
    kWRDn = kWord + 8
};
// kWxj: the reaction's first extra exponential job (fall-off: k0, then the Troe
// centering terms exp(-T/T***), exp(-T/T*), exp(-T**/T))
enum WRI : int { kWtype = 0, kWrev, kWnf, kWnb, kWxj, kWidx, kWRIn = kWidx + 8 };
// species fields of WMech::th, field-major over 32 species slots
enum WTH : int {
    kWtl = 0, kWtc, kWth,
    kWrange = 3,               // then 2 ranges of 21: h[5], h5, s0, s[4], s6, cp[5], dcp[4]
    kWRangeN = 21,
    kWW = kWrange + 2 * kWRangeN,   // molecular weight
    kWTHn = kWW + 1
};

// Reactions come in rounds of 32 (reaction r = 32 * round + slot); the
// reaction tables and the records are round-major, [round][field][32], so
// that lane `slot` reads field f of its reaction at a fixed offset.
// Exponential jobs (round-major [round][3][32]: alpha, beta, gamma): job j
// is exp(alpha ln T + beta / T + gamma T); job r < nrc is reaction r's
// Arrhenius factor, the fall-off reactions' extra terms follow.
struct WMech {
    int32_t nsp, nrc, nrc32, ntb, nent, njob, njob32;
    const double *xj;     // [njob32 / 32][3][32]
    const double *th;     // [kWTHn][32]
    const double *rd;     // [nrc32 / 32][kWRDn][32]
    const int32_t *ri;    // [nrc32 / 32][kWRIn][32]
    const double *eff;    // [nrc][nsp] efficiencies (third-body / fall-off rows)
    const int32_t *lptr;  // [nsp + 1] participation lists of the species
    const int32_t *lent;  // [3 * nent] per entry: reaction | pos << 16 | np << 20 | third-body << 24,
                          // then the participants' columns packed 8 bits each (two words)
    const double *lnu;    // [nent] the species' signed coefficient in the entry's reaction
    const int32_t *tbl;   // [ntb] third-body / fall-off reactions
    const double *raw;    // [nsp][2][7] mass-basis NASA-7 (out-of-range forms)
    double glim;          // |G0/(Ru T)| bound of the product form of 1/Kc
};

constexpr int kWRec = 12;   // record: q, dq/dT, g, dH, d[8]

// per-warp shared memory (doubles)
template <int N>
struct WSmem {
    static constexpr int LD = (N % 2 == 0) ? N + 1 : N;
    static constexpr int kSV = 0;              // c, h, E, R, g, dgt: 6 x 32
    static constexpr int kJ = kSV + 6 * 32;    // rows of J, N x LD
    static constexpr int kW = (N <= 11) ? 3 : 2;   // lanes per species row
    static constexpr int kJ2 = kJ + N * LD;    // the other lanes' partial rows of J
    static constexpr int kRec = kJ2 + (kW - 1) * N * LD;  // records, kWRec x nrc32, then the exponentials (njob32)
    __host__ __device__ static size_t doubles(int nrc32, int njob32) { return (size_t)kRec + kWRec * (size_t)nrc32 + njob32; }
    static size_t bytes(int nrc32, int njob32) { return sizeof(double) * doubles(nrc32, njob32); }
};

// the mechanism tables as copied into the block's shared memory
struct WTabs {
    const double *th, *rd, *eff, *lnu, *xj;
    const int32_t *ri, *lptr, *lent, *tbl;
};

// shared memory of the block's table copy (bytes, 8-byte aligned parts)
__host__ __device__ inline size_t w_tables_bytes(int nsp, int nrc, int nrc32, int nent, int ntb, int njob32) {
    const size_t d = (size_t)kWTHn * 32 + (size_t)kWRDn * nrc32 + (size_t)(nrc > 0 ? nrc : 1) * nsp + nent +
                     3 * (size_t)njob32;
    const size_t i = (size_t)kWRIn * nrc32 + (nsp + 1) + 3 * (size_t)nent + (ntb > 0 ? ntb : 1);
    return sizeof(double) * d + ((sizeof(int32_t) * i + 7) & ~(size_t)7);
}


template <int N>
struct WCtx {
    static constexpr int TI = N - 1;
    using SM = WSmem<N>;
    const WMech &m;
    const WTabs &tb;
    const IntegratorParams &P;
    double *s;        // this warp's shared memory
    int lane;
    int nsp;
    double p;
    int n_jac, n_rhs, n_lu, n_newton, n_steps, n_attempts;
    int status;
    int lpos;         // LU: logical row of this lane's physical row
    double a[N];      // LU: this lane's row of I - dt J

    __device__ WCtx(const WMech &mm, const WTabs &t, const IntegratorParams &pp, double *sm, int l)
        : m(mm), tb(t), P(pp), s(sm), lane(l), nsp(mm.nsp), p(0), n_jac(0), n_rhs(0), n_lu(0), n_newton(0),
          n_steps(0), n_attempts(0), status(0), lpos(l) {}

    __device__ __forceinline__ double sum(double v) const {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }
    __device__ __forceinline__ double max(double v) const {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            v = (v < w) ? w : v;
        }
        return v;
    }
    // reaction r's fields in the round-major tables and its record
    __device__ __forceinline__ const double *rdp(int r) const { return tb.rd + (r >> 5) * (kWRDn * 32) + (r & 31); }
    __device__ __forceinline__ const int32_t *rip(int r) const { return tb.ri + (r >> 5) * (kWRIn * 32) + (r & 31); }
    __device__ __forceinline__ double *recp(int r) const { return s + SM::kRec + (r >> 5) * (kWRec * 32) + (r & 31); }

    // ---------------------------------------------------------------------
    // f(y) and, when jac, the Jacobian into shared memory (rows of J, the
    // temperature row and column). y is this lane's element (lane < N).
    __device__ __forceinline__ double evaluate(double y, bool jac) {
        if (jac) ++n_jac; else ++n_rhs;
        return eval_impl(y, jac);
    }

    __device__ __forceinline__ double eval_impl(double y, bool jac) {
        const unsigned full = 0xffffffffu;
        const double T = __shfl_sync(full, y, TI);
        const double Tm = hmax(T, kTiny);
        const double logT = log(T);
        const double invT = frcp(Tm);
        const double invRuT = invT * (1.0 / kRu);
        double *sv = s + SM::kSV;
        // ---- species
        double cp = 0.0, dcp = 0.0, h = 0.0;
        bool slow = false;
        if (lane < nsp) {
            const double *ts = tb.th + lane;
            auto th = [ts](int f) { return ts[f * 32]; };
            const double tl = th(kWtl), tc = th(kWtc), thh = th(kWth);
            double g, dgt;
            if (T >= tl && T <= thh) {
                const int b = kWrange + ((T < tc) ? 0 : kWRangeN);
                const double *tr = ts + b * 32;
                h = T * (tr[0] + T * (tr[32] + T * (tr[64] + T * (tr[96] + T * tr[128])))) + tr[160];
                const double sv0 = tr[192] * logT +
                                   (T * (tr[224] + T * (tr[256] + T * (tr[288] + T * tr[320]))) + tr[352]);
                g = (h - T * sv0) * invRuT;
                dgt = -h * invT;
                cp = tr[384] + T * (tr[416] + T * (tr[448] + T * (tr[480] + T * tr[512])));
                dcp = tr[544] + T * (tr[576] + T * (tr[608] + T * tr[640]));
            } else {
                t3_thermo_slow(&m.raw[14 * lane + ((T < tc) ? 0 : 7)], tl, thh, th(kWW),
                               T, logT, invRuT, cp, h, dcp, g, dgt);
                slow = true;
            }
            slow = slow || !(fabs(g) < m.glim);
            const double e = exp(hmin(hmax(g, -m.glim), m.glim));
            sv[0 * 32 + lane] = hmax(y, 0.0);
            sv[1 * 32 + lane] = h;
            sv[2 * 32 + lane] = e;
            sv[3 * 32 + lane] = frcp(e);
            sv[4 * 32 + lane] = g;
            sv[5 * 32 + lane] = dgt;
        }
        const bool wslow = __any_sync(full, slow);
        const double cCp = sum((lane < nsp) ? y * cp : 0.0);
        const double dcCpdT = jac ? sum((lane < nsp) ? y * dcp : 0.0) : 0.0;
        __syncwarp();
        // ---- reactions: one record each
        // every exponential of the reaction pass, one per lane
        double *X = s + SM::kRec + kWRec * m.nrc32;
        for (int j = lane; j < m.njob; j += 32) {
            const double *xj = tb.xj + (j >> 5) * 96 + (j & 31);
            X[j] = exp(xj[0] * logT + xj[32] * invT + xj[64] * T);
        }
        __syncwarp();
        for (int r = lane; r < m.nrc32; r += 32) {
            if (r < m.nrc) reaction(r, T, logT, invT, invRuT, wslow, jac, recp(r), X);
        }
        __syncwarp();
        // ---- rows of f and J
        double f = 0.0, jt = 0.0, S = 0.0;
        double *Jrow = s + SM::kJ + lane * SM::LD;
        // species i's entries are split between lanes i, i + WS (and i + 2 WS):
        // entry e goes to the (e - e0) mod kW-th of them, the others' partial
        // rows are added to lane i's
        constexpr int WS = (SM::kW == 3) ? 11 : 16;   // lane stride between a row's workers
        const int hi = lane / WS, sl = lane - WS * hi;
        double *Jp = hi ? s + SM::kJ2 + (hi - 1) * N * SM::LD + sl * SM::LD : Jrow;
        if (jac && sl < N - 1) {
#pragma unroll
            for (int j = 0; j < N; ++j) Jp[j] = 0.0;
        }
        if (sl < nsp) {
            const int e0 = tb.lptr[sl], e1 = tb.lptr[sl + 1];
            for (int e = e0 + hi; e < e1; e += SM::kW) {
                const int w0 = tb.lent[3 * e];
                const int r = w0 & 0xffff, pos = (w0 >> 16) & 7, np = (w0 >> 20) & 15;
                const double *R = recp(r);
                const double nu = tb.lnu[e];
                f += nu * R[0];
                if (!jac) continue;
                jt += nu * R[32];
                S += R[3 * 32] * R[(4 + pos) * 32];
                const unsigned c0 = (unsigned)tb.lent[3 * e + 1], c1 = (unsigned)tb.lent[3 * e + 2];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    if (k >= np) break;
                    const int col = ((k < 4 ? c0 : c1) >> (8 * (k & 3))) & 0xff;
                    Jp[col] += nu * R[(4 + k) * 32];
                }
                if (w0 & (1 << 24)) {
                    const double gn = nu * R[2 * 32];
                    const double *er = &tb.eff[(size_t)r * nsp];
                    for (int j = 0; j < nsp; ++j) Jp[j] += er[j] * gn;
                }
            }
            if (jac) {
                // the temperature row's third-body / fall-off columns
                for (int t = hi; t < m.ntb; t += SM::kW) {
                    const int r = tb.tbl[t];
                    const double *R = recp(r);
                    S += R[3 * 32] * (tb.eff[(size_t)r * nsp + sl] * R[2 * 32]);
                }
            }
        }
        if constexpr (SM::kW == 3) {
            const int s1 = (lane + 11) & 31, s2 = (lane + 22) & 31;
            f = (f + __shfl_sync(full, f, s1)) + __shfl_sync(full, f, s2);
            if (jac) {
                jt = (jt + __shfl_sync(full, jt, s1)) + __shfl_sync(full, jt, s2);
                S = (S + __shfl_sync(full, S, s1)) + __shfl_sync(full, S, s2);
                __syncwarp();
                if (lane < nsp) {
                    const double *J2 = s + SM::kJ2 + lane * SM::LD, *J3 = J2 + N * SM::LD;
#pragma unroll
                    for (int j = 0; j < N - 1; ++j) Jrow[j] = (Jrow[j] + J2[j]) + J3[j];
                }
            }
        } else {
            f += __shfl_xor_sync(full, f, 16);
            if (jac) {
                jt += __shfl_xor_sync(full, jt, 16);
                S += __shfl_xor_sync(full, S, 16);
                __syncwarp();
                if (lane < nsp) {
                    const double *J2 = s + SM::kJ2 + lane * SM::LD;
#pragma unroll
                    for (int j = 0; j < N - 1; ++j) Jrow[j] += J2[j];
                }
            }
        }
        // ---- temperature equation (constant pressure, chemistrySource.cpp:863-883, 991-1021)
        const double icCp = frcp(cCp);
        const double DTdt = sum((lane < nsp) ? f * h : 0.0) * icCp;
        if (lane == TI) f = -DTdt;
        if (jac) {
            const double cpf = sum((lane < nsp) ? cp * f + h * jt : 0.0);
            if (lane < N - 1) {
                Jrow[TI] = jt;
                s[SM::kJ + TI * SM::LD + lane] = (lane < nsp) ? (cp * DTdt - S) * icCp : 0.0;
            }
            if (lane == TI) Jrow[TI] = (dcCpdT * DTdt - cpf) * icCp;
            __syncwarp();
        }
        return f;
    }

    // one reaction's record (reactionTypes q / Kc / DqDci / DqDT,
    // reactionTypes.cpp:178-445, 843-876; ArrheniusRR, unimolecularFallOffRR,
    // fallOffFunctions Troe / Lindemann)
    __device__ __forceinline__ void reaction(int r, double T, double logT, double invT, double invRuT,
                                             bool slow, bool jac, double *R, const double *X) {
        const double *sv = s + SM::kSV;
        const double *x = rdp(r);
        const int32_t *xi = rip(r);
        const int type = xi[(kWtype) * 32], rev = xi[(kWrev) * 32], nf = xi[(kWnf) * 32], nb = xi[(kWnb) * 32];
        // concentration powers of the reactants (pf) and products (pb)
        double pf[kMaxSide], pb[kMaxSide];
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            pf[k] = (k < nf) ? conc_pow(sv[xi[(kWidx + k) * 32]], x[(kWord + k) * 32]) : 1.0;
            pb[k] = (k < nb) ? conc_pow(sv[xi[(kWidx + nf + k) * 32]], x[(kWord + nf + k) * 32]) : 1.0;
        }
        double M = 0.0;
        if (type != kArrhenius) {
            const double *er = &tb.eff[(size_t)r * nsp];
            for (int j = 0; j < nsp; ++j) M += er[j] * sv[j];
        }
        const double b = x[(kWb) * 32], Ta = x[(kWTa) * 32];
        const double kx = x[(kWA) * 32] * X[r];
        double kf, k0 = 0.0, Pr = 0.0, Ff = 1.0, logPr = 0.0;
        T3Cent cent{0.0, 0.0};
        if (type == kArrhenius) {
            kf = kx;
        } else if (type == kThirdBody) {
            kf = M * kx;
        } else {
            // unimolecularFallOffRR::k (unimolecularFallOffRR.cpp:37-53)
            const int xj = xi[(kWxj) * 32];
            k0 = x[(kWA0) * 32] * X[xj];
            Pr = fdiv(k0, notZeroD(kx)) * M;
            if (type != kLindemann) {
                const double iTsss = x[(kWiTsss) * 32], iTs = x[(kWiTs) * 32], Tss = x[(kWTss) * 32];
                cent = t3_troe_cent(type == kTroe4, x[(kWalpha) * 32], iTsss, iTs, Tss, X[xj + 1], X[xj + 2],
                                    (type == kTroe4) ? X[xj + 3] : 0.0, invT);
                logPr = log10(hmax(Pr, kTiny));
                Ff = t3_troe_F(cent.lf, logPr);
            }
            kf = kx * (Pr / (1.0 + Pr)) * Ff;
        }
        // reaction enthalpy (T row, T corner; DG0/DT - G0/T = -H0/T in the fitted range)
        double dH = 0.0;
        for (int k = 0; k < nf + nb; ++k) dH += x[(kWnu + k) * 32] * sv[32 + xi[(kWidx + k) * 32]];
        // kr = kf krf; dkr/dT = dkf/dT ra - kf rb
        double krf = 0.0, ra = 0.0, rb = 0.0;
        const double s_ = x[(kWs) * 32];
        if (rev) {
            if (!slow) {
                double ik = 1.0;
                for (int k = 0; k < nf; ++k) ik *= pow_small(sv[3 * 32 + xi[(kWidx + k) * 32]], -x[(kWnu + k) * 32]);
                for (int k = nf; k < nf + nb; ++k) ik *= pow_small(sv[2 * 32 + xi[(kWidx + k) * 32]], x[(kWnu + k) * 32]);
                if (s_ == -1.0) ik *= (kPatm / kRu) * invT;
                else if (s_ == 1.0) ik *= T * (kRu / kPatm);
                else if (s_ != 0.0) ik *= exp(-s_ * (log(kPatm / kRu) - logT));
                krf = ik;
                ra = ik;
                rb = ik * (-dH * invT * invRuT - s_ * invT);
            } else {
                double kp = 0.0, dk = 0.0;
                for (int k = 0; k < nf + nb; ++k) {
                    const int i = xi[(kWidx + k) * 32];
                    const double nu = x[(kWnu + k) * 32];
                    kp += nu * sv[4 * 32 + i];
                    dk += nu * sv[5 * 32 + i];
                }
                dk *= invRuT;
                const double lik = kp - s_ * (log(kPatm / kRu) - logT);
                if (fabs(lik) < 650.0) {
                    ra = exp(lik);
                    krf = ra;
                    rb = ra * (dk - s_ * invT);
                } else {
                    double Kc, DKcDT;
                    t3_kc_slow(kp, dk, s_, T, Kc, DKcDT);
                    krf = (fabs(Kc) > kVeryTiny) ? 1.0 / Kc : 0.0;
                    const double den = hmax(Kc, kVeryTiny);
                    ra = 1.0 / den;
                    rb = krf * DKcDT / den;
                }
            }
        }
        const double kr = kf * krf;
        double qf = kf, qr = kr;
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            qf *= pf[k];
            qr *= pb[k];
        }
        const double q = qf - (rev ? qr : 0.0);
        R[0] = q;
        if (!jac) return;
        // d q / d T (reactionTypes.cpp:843-876)
        double dkf = (type >= kLindemann) ? (Pr / (1.0 + Pr)) * Ff * (kx * invT * (b + Ta * invT))
                                          : kf * invT * (b + Ta * invT);
        double dkr = rev ? dkf * ra - kf * rb : 0.0;
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            dkf *= pf[k];
            dkr *= pb[k];
        }
        double dq = dkf - dkr;
        if (!finite(dq)) dq = 0.0;
        double g = 0.0;
        if (type == kThirdBody) {
            g = fdiv(q, hmax(M, kTiny));
        } else if (type >= kLindemann) {
            double dgdT;
            t3_falloff_jac_fast(type != kLindemann, cent, Ff, logPr, k0, kx, x[(kWb0) * 32], x[(kWTa0) * 32], b, Ta,
                                M, q, invT, g, dgdT);
            dq += dgdT;
        }
        R[1 * 32] = dq;
        R[2 * 32] = g;
        R[3 * 32] = dH;
        // d q / d c_k (reactionTypes::DqDci, reactionTypes.cpp:354-445): forward
        // products for the reactants, minus the reverse products for the products
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int n = side ? nb : nf, off = side ? nf : 0;
            const double K = side ? (rev ? -kr : 0.0) : kf;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k >= n) break;
                double d = K;
#pragma unroll
                for (int l = 0; l < kMaxSide; ++l) {
                    if (l >= n) break;
                    if (l == k) {
                        const double o = x[(kWord + off + k) * 32];
                        if (o == 1.0) continue;
                        const double cj = sv[xi[(kWidx + off + k) * 32]];
                        if (o < 1.0) d *= (cj > kTiny) ? o * pow_n(cj, o - 1.0) : 0.0;
                        else d *= o * pow_n(cj, o - 1.0);
                    } else {
                        d *= side ? pb[l] : pf[l];
                    }
                }
                R[(4 + off + k) * 32] = d;
            }
        }
    }

    // ---------------------------------------------------------------------
    // A = I - dt J from this lane's row of J, then the pivoted LU (lanes < N)
    __device__ __forceinline__ int factor(double dt) {
        const unsigned full = 0xffffffffu;
        const double *Jrow = s + SM::kJ + lane * SM::LD;
#pragma unroll
        for (int j = 0; j < N; ++j) a[j] = (lane < N) ? (((lane == j) ? 1.0 : 0.0) - dt * Jrow[j]) : 0.0;
        ++n_lu;
        lpos = lane;
        // keys of the argmax: |a(k)| over the rows not yet pivoted, the first
        // in the current logical order on ties (LUDecomposeDPivoting)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            // the largest |a(k)| by warp reductions of its bit pattern (a
            // non-negative double orders like its bits; NaN never wins), then
            // the first such row in the logical order
            const double av = fabs(a[k]);
            const bool cand = lane < N && lpos >= k;
            const unsigned long long bits = (cand && av == av) ? (unsigned long long)__double_as_longlong(av) : 0ull;
            const unsigned hi = (unsigned)(bits >> 32), lo = (unsigned)bits;
            const unsigned mhi = __reduce_max_sync(full, hi);
            const unsigned mlo = __reduce_max_sync(full, (hi == mhi) ? lo : 0u);
            const unsigned kb = (cand && hi == mhi && lo == mlo) ? (unsigned)((lpos << 5) | lane) : 0xffffffffu;
            const unsigned key = __reduce_min_sync(full, kb);
            const int pl = (int)(key & 31);          // pivot lane
            const int pos_p = (int)(key >> 5);       // its logical position
            // the rows swap logical positions k and pos_p
            if (lane == pl) lpos = k;
            else if (lpos == k) lpos = pos_p;
            double u[N];
#pragma unroll
            for (int j = k; j < N; ++j) u[j] = __shfl_sync(full, a[j], pl);
            const double inv = frcp(u[k]);
            if (lane == pl) {
                a[k] = inv;
            } else if (lane < N && lpos > k) {
                const double l = a[k] * inv;
                a[k] = l;
#pragma unroll
                for (int j = k + 1; j < N; ++j) a[j] -= l * u[j];
            }
        }
        return lpos;
    }

    // (L U) x = P b along the logical order; b and x are this lane's elements
    __device__ __forceinline__ double solve(int /*mystep*/, double b) {
        const unsigned full = 0xffffffffu;
        int lb[N];
#pragma unroll
        for (int t = 0; t < N; ++t) lb[t] = __ffs(__ballot_sync(full, lane < N && lpos == t)) - 1;
        double acc = 0.0, z = 0.0;
#pragma unroll
        for (int t = 0; t < N; ++t) {
            const double zt = __shfl_sync(full, b - acc, lb[t]);
            if (lpos == t) z = zt;
            if (lane < N && lpos > t) acc += a[t] * zt;
        }
        double x = 0.0;
        acc = 0.0;
#pragma unroll
        for (int t = N - 1; t >= 0; --t) {
            const double xt = __shfl_sync(full, (z - acc) * a[t], lb[t]);
            if (lane == t) x = xt;
            if (lane < N && lpos < t) acc += a[t] * xt;
        }
        return (lane < N) ? x : 0.0;
    }
};

// The reference's step control around WCtx (ImplicitEuler::solve /
// adaptiveSolve / NewtonIteration, ODEsSolver::maxError; the same control flow
// as CellIntegrator, warp-uniform).
template <int N>
struct WIntegrator : WCtx<N> {
    using Base = WCtx<N>;
    using Base::lane;
    using Base::P;
    using Base::nsp;
    int countStep;
    double lts0, lts1;    // lastTimeStep_[0], [1]
    double yk0, yk1;      // yklast_[0], [1] (this lane's element)

    __device__ WIntegrator(const WMech &mm, const WTabs &t, const IntegratorParams &pp, double *sm, int l)
        : Base(mm, t, pp, sm, l), countStep(0), lts0(0), lts1(0), yk0(0), yk1(0) {}

    // ODEsSolver::maxError (ODEsSolver.cpp:37-46); NaN terms do not raise the max
    __device__ double max_error(double y0, double y, double e) {
        double v = 0.0;
        if (lane < N) {
            const double tol = P.atol + P.rtol * hmax(fabs(y0), fabs(y));
            v = fabs(e) * frcp(tol);
            if (isnan(v)) v = 0.0;
        }
        return this->max(v);
    }

    // ImplicitEuler::maxIncrement (ImplicitEuler.cpp:40-52)
    __device__ double max_increment(double y0, double y, double e) {
        if (__any_sync(0xffffffffu, lane < N && isnan(y))) return 1.5;
        double v = 0.0;
        if (lane < N) {
            const double tol = P.atol_inc + P.rtol_inc * hmax(fabs(y0), fabs(y));
            v = fabs(e) * frcp(tol);
            if (isnan(v)) v = 0.0;
        }
        return this->max(v);
    }

    // ImplicitEuler::NewtonIteration (ImplicitEuler.cpp:161-251)
    __device__ double newton(double y0, double dt, double &yk, bool &conv, int &rc) {
        int count = 0;
        double maxErr = 0.0, lastErr = 0.0;
        const bool autoJ = P.auto_update_jacobian != 0;
        const int stepJ = P.step_to_update_jac;
        do {
            double f;
            if (!autoJ || count == 0 || count % stepJ == 0) {
                f = this->evaluate(yk, true);
                this->factor(dt);
            } else {
                f = this->evaluate(yk, false);
            }
            const double rhs = (lane < N) ? ((-yk + y0) + dt * f) : 0.0;
            const double x = this->solve(0, rhs);
            ++this->n_newton;
            const unsigned bad = __ballot_sync(0xffffffffu, lane < N && !finite(x));
            if (bad) {
                const int firstBad = __ffs(bad) - 1;
                if (lane < firstBad) yk += x;
                conv = false;
                return 1000.0;
            }
            if (lane < N) yk += x;
            maxErr = max_error(yk, yk, x);
            if (count > 0) {
                const double diver = maxErr * frcp(hmax(lastErr, kTiny));
                if (autoJ) {
                    const int lim = (30 * stepJ > 50) ? 30 * stepJ : 50;
                    if (diver > 2 && count > lim) {
                        conv = false;
                        return 1000.0;
                    }
                } else if (diver > 2 && count > 5) {
                    conv = false;
                    return 1000.0;
                }
            }
            lastErr = maxErr;
            count++;
            if (isnan(maxErr)) {
                conv = false;
                return 1000.0;
            }
            if (count > 1000) {
                conv = false;
                return maxErr;
            }
            if (P.max_newton_total > 0 && this->n_newton >= P.max_newton_total) {
                rc = kRcIterLimit;
                conv = false;
                return 1000.0;
            }
        } while (maxErr > 1.0);
        conv = true;
        return maxErr;
    }

    // ImplicitEuler::solve(t0, y0, dydt0, dt, y) (ImplicitEuler.cpp:101-142)
    __device__ double step(double y0, double dt, double &y, int &rc) {
        ++this->n_attempts;
        double yk = y0;
        bool conv = true;
        const double errN = newton(y0, dt, yk, conv, rc);
        y = yk;
        if (!conv) return errN;
        double e = 0.0;
        if (countStep == 0) {
            const double f = this->evaluate(yk, false);
            e = yk - y0 - dt * f;
        } else {
            const double dtn = lts0, dtn1 = lts1;
            const double f1 = 2.0 * frcp(dtn * (dtn + dtn1));
            const double f2 = 2.0 * frcp(dtn1 * (dtn + dtn1));
            const double LTEF = (dtn * dtn) * 0.5;
            e = f1 * (yk - y0) - f2 * (y0 - yk1);
            e *= LTEF;
        }
        return max_increment(y0, yk, e);
    }

    // ImplicitEuler::adaptiveSolve (ImplicitEuler.cpp:253-292) with checkNewY
    // (chemistrySource.cpp:1152-1164)
    __device__ int adaptive(double &t, double &dt0, double &y) {
        double dt = dt0;
        double error = 0.0;
        double yTemp = y;
        lts1 = lts0;
        int count = 0;
        const double Told = __shfl_sync(0xffffffffu, y, N - 1);
        do {
            lts0 = dt;
            int rc = kRcOk;
            error = step(y, dt, yTemp, rc);
            if (rc != kRcOk) return rc;
            const double Tnew = __shfl_sync(0xffffffffu, yTemp, N - 1);
            bool ok = true;
            if ((Tnew - Told) > P.T_alpha * Told) {
                dt *= P.T_beta;
                ok = false;
            }
            if (!ok && count < 100) {
                error = 2;
                count++;
                if (dt <= kVeryTiny) return kRcUnderflow;
                continue;
            }
            if (error > 1.0) {
                const double scale = hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale);
                dt *= scale;
                if (dt <= kVeryTiny) return kRcUnderflow;
            }
        } while (error > 1.0);
        t += dt;
        y = yTemp;
        ++this->n_steps;
        if (error > P.err_accept_limit)
            dt0 = hmin(hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale), P.maxscale) * dt;
        else
            dt0 = hmax(P.safescale * P.maxscale * dt, dt);
        return kRcOk;
    }

    // ImplicitEuler::solve(t0, tn, dt0, y) (ImplicitEuler.cpp:294-342), t0 = 0
    __device__ int interval(double &tn, double &dt0, double &y) {
        double t = 0.0;
        double dt = 0.2 * dt0;
        double dtReached = 0.0;
        bool last = false;
        for (int n = 0; n < P.maxstep; ++n) {
            countStep = n;
            if (n == 0) {
                yk0 = y;
            } else {
                yk1 = yk0;
                yk0 = y;
            }
            const double dtTry0 = dt;
            if ((t + dt - tn) * (t + dt - 0.0) > 0) {
                dt = tn - t;
                last = true;
            } else if (t + dt == tn) {
                last = true;
            }
            const int rc = adaptive(t, dt, y);
            if (rc != kRcOk) return rc;
            dtReached = t;
            if ((t - tn) * (tn - 0.0) >= 0) {
                if (n > 0 && last) dt0 = hmin(dtTry0, tn);
                return kRcOk;
            }
        }
        this->status |= 2;  // HC_CELL_MAXSTEP
        tn = dtReached;
        return kRcOk;
    }
};

#ifndef HC_W_MIN_BLOCKS
#define HC_W_MIN_BLOCKS 2   // blocks of kWWarps warps per SM the kernel is built for
#endif
constexpr int kWWarps = 8;  // warps (cells in flight) per block

template <int N>
__global__ void __launch_bounds__(32 * kWWarps, HC_W_MIN_BLOCKS)
integrate_w_kernel(const __grid_constant__ WMech m, const __grid_constant__ IntegratorParams P,
                   const __grid_constant__ CellIO io) {
    extern __shared__ double smem_w[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nsp = m.nsp;
    const unsigned full = 0xffffffffu;
    // the mechanism tables into the block's shared memory, once
    WTabs tb;
    {
        double *d = smem_w;
        const int nth = kWTHn * 32, nrd = kWRDn * m.nrc32, neff = (m.nrc > 0 ? m.nrc : 1) * nsp;
        for (int i = threadIdx.x; i < nth; i += blockDim.x) d[i] = m.th[i];
        for (int i = threadIdx.x; i < nrd; i += blockDim.x) d[nth + i] = m.rd[i];
        for (int i = threadIdx.x; i < neff; i += blockDim.x) d[nth + nrd + i] = m.eff[i];
        for (int i = threadIdx.x; i < m.nent; i += blockDim.x) d[nth + nrd + neff + i] = m.lnu[i];
        for (int i = threadIdx.x; i < 3 * m.njob32; i += blockDim.x) d[nth + nrd + neff + m.nent + i] = m.xj[i];
        tb.th = d;
        tb.rd = d + nth;
        tb.eff = d + nth + nrd;
        tb.lnu = d + nth + nrd + neff;
        tb.xj = d + nth + nrd + neff + m.nent;
        int32_t *q = reinterpret_cast<int32_t *>(d + nth + nrd + neff + m.nent + 3 * m.njob32);
        const int nri = kWRIn * m.nrc32, ntbl = m.ntb > 0 ? m.ntb : 1;
        for (int i = threadIdx.x; i < nri; i += blockDim.x) q[i] = m.ri[i];
        for (int i = threadIdx.x; i <= nsp; i += blockDim.x) q[nri + i] = m.lptr[i];
        for (int i = threadIdx.x; i < 3 * m.nent; i += blockDim.x) q[nri + nsp + 1 + i] = m.lent[i];
        for (int i = threadIdx.x; i < ntbl; i += blockDim.x) q[nri + nsp + 1 + 3 * m.nent + i] = m.tbl[i];
        tb.ri = q;
        tb.lptr = q + nri;
        tb.lent = q + nri + nsp + 1;
        tb.tbl = q + nri + nsp + 1 + 3 * m.nent;
        __syncthreads();
    }
    const size_t tab = w_tables_bytes(nsp, m.nrc, m.nrc32, m.nent, m.ntb, m.njob32) / sizeof(double);
    double *s = smem_w + tab + (size_t)warp * WSmem<N>::doubles(m.nrc32, m.njob32);
    while (true) {
        long long k = 0;
        if (lane == 0) k = (long long)atomicAdd(io.queue_head, 1ULL);
        k = __shfl_sync(full, k, 0);
        if (k >= io.nqueue) break;
        const int64_t cell = io.order ? (int64_t)io.order[k] : (int64_t)k;
        WIntegrator<N> ci(m, tb, P, s, lane);
        const double Ti = io.T[cell];
        const double tstep = io.dt[cell] * io.dt_factor;
        const double rho0 = io.rho[cell];
        const double W = (lane < nsp) ? tb.th[kWW * 32 + lane] : 1.0;
        double y = 0.0;
        if (lane < nsp) y = rho0 * io.Y[(int64_t)lane * io.ncells + cell] * frcp(W);
        const double c0 = y;
        if (Ti < P.T_threshold) {
            if (lane == 0) {
                io.subdt[cell] = tstep;
                if (io.status) io.status[cell] = 1;  // HC_CELL_SKIPPED
                if (io.cost) io.cost[cell] = 0;
            }
            if (io.Ri && lane < nsp) io.Ri[(int64_t)lane * io.ncells + cell] = 0.0;
            continue;
        }
        ci.p = io.p[cell];
        double leftTime = tstep;
        double sub = hmin(leftTime, hmin(io.subdt[cell], P.dt_max));
        if (lane == N - 1) y = Ti;
        int rc = kRcOk;
        while (leftTime > 0.0) {
            double d = leftTime;
            rc = ci.interval(d, sub, y);
            if (rc != kRcOk) break;
            leftTime -= d;
        }
        if (rc == kRcUnderflow) ci.status |= 4;
        if (rc == kRcIterLimit) ci.status |= 8;
        // ciToYi (chemistrySource.cpp:1225-1246) and rho = p / (Rm T)
        const double Tn = __shfl_sync(full, y, N - 1);
        double yi = (lane < nsp) ? hmax(0.0, y) : 0.0;
        const double rr = ci.sum(yi * ((lane < nsp) ? W : 0.0));
        yi = (lane < nsp) ? yi * W * frcp(hmax(rr, kTiny)) : 0.0;
        const double ys = ci.sum(yi);
        if (ys != 1.0) yi *= frcp(ys);
        const double wsum = ci.sum((lane < nsp) ? yi * frcp(W) : 0.0);
        const double Rm = kRu * hmax(wsum, kVeryTiny);
        if (lane < nsp) {
            io.Y[(int64_t)lane * io.ncells + cell] = yi;
            if (io.Ri) io.Ri[(int64_t)lane * io.ncells + cell] = (y - c0) * frcp(tstep) * W;
        }
        if (lane == 0) {
            io.T[cell] = Tn;
            io.rho[cell] = fdiv(ci.p, Rm * Tn);
            io.subdt[cell] = sub;
            if (io.status) io.status[cell] = ci.status;
            if (io.cost) io.cost[cell] = ci.n_newton;
            if (io.counters) {
                atomicAdd(&io.counters[0], (unsigned long long)ci.n_jac);
                atomicAdd(&io.counters[1], (unsigned long long)ci.n_rhs);
                atomicAdd(&io.counters[2], (unsigned long long)ci.n_lu);
                atomicAdd(&io.counters[3], (unsigned long long)ci.n_newton);
                atomicAdd(&io.counters[4], (unsigned long long)ci.n_steps);
                atomicAdd(&io.counters[5], (unsigned long long)ci.n_attempts);
            }
        }
    }
}

}  // namespace hc
