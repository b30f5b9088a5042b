// Segment-per-cell implicit-Euler integrator (kernel 7) for mechanisms of
// N = nsp + 1 <= 16 unknowns, FP64.
//
// A warp holds G = 32 / N cells at once, one per segment of N consecutive
// lanes (N = 10: three cells in lanes 0-9, 10-19, 20-29). Lane i of a
// segment owns element i of its cell's state (species i, the temperature in
// the last lane) and row i of the Newton matrix. Each segment takes its next
// cell from the device work queue (the grid is persistent).
//
// The reference's nested loops (chemistrySource.cpp:1511-1555,
// ImplicitEuler.cpp:101-342, ODEsSolver.cpp:148-225) are flattened into one
// state machine per segment, as in the thread-per-cell kernels: each trip of
// the main loop first lets every segment run its own bookkeeping up to its
// next heavy state (Newton iteration or first-step error evaluation; the
// segment's lanes shuffle among themselves only), then the whole warp runs
// the heavy block once for all of its cells:
//
//  * species: lane i of each segment evaluates species i (NASA-7 from
//    coefficients pre-multiplied on the host) and publishes c_i, h_i and
//    exp(+-G0_i/(Ru T)) to its segment's shared memory;
//  * exponentials exp(a ln T + b / T + c T) of the Arrhenius and fall-off
//    terms, and the reactions (r = lane + N k), one record each: q, dq/dT,
//    the third-body / fall-off factor, dH_r and dq/dc of each participant;
//  * rows: lane i walks the reactions species i takes part in and sums its
//    row of f and of the Jacobian, the temperature column entry and its
//    entry of the temperature row (sum_r dH_r dq_r/dc_i);
//  * LU with partial pivoting (LUDecomposeDPivoting: the first largest
//    |a(k)| in the current row order) on the rows held in the lanes'
//    registers: a segment argmax by rotation, the pivot row broadcast by
//    shuffles; rows keep their lanes and carry a logical position;
//  * the triangular solves along the logical order.
//
// The cell-level arithmetic (norms, step-size control, the temperature
// equation) is the reference's, with reductions over the segment.
#pragma once

#include "t1_body.cuh"
#include "wcell.cuh"

namespace hc {

// c^o for a reaction order o (reactionTypes.cpp:178-240: std::pow), and o
// c^(o-1) of DqDci (reactionTypes.cpp:354-445) for o != 1, zero at c <= 1e-15
// when o < 1: out of line, one copy for all call sites
static __device__ HC_NOINLINE double s_conc_pow(double c, double o) {
    c = hmax(c, 0.0);
    if (o == 0.0) return 1.0;
    if (o == -1.0) return 1.0 / c;
    return pow(c, o);
}
static __device__ HC_NOINLINE double s_dconc(double c, double o) {
    if (o < 1.0) return (c > kTiny) ? o * pow_n(c, o - 1.0) : 0.0;
    return o * pow_n(c, o - 1.0);
}
__device__ __forceinline__ double s_pow(double c, double o) {
    if (o == 1.0) return hmax(c, 0.0);
    if (o == 2.0) {
        c = hmax(c, 0.0);
        return c * c;
    }
    return s_conc_pow(c, o);
}

// per-segment shared memory (doubles)
template <int N>
struct SLayout {
    static constexpr int S = N;                      // lanes per cell
    static constexpr int G = 32 / N;                 // cells per warp
    static constexpr int LD = (N % 2 == 0) ? N + 1 : N;
    static constexpr int kSV = 0;                    // c, h, E, R, g, dgt: 6 x S
    static constexpr int kJ = 6 * S;                 // rows of J, N x LD
    static constexpr int kRec = kJ + N * LD;         // records [kWRec][nrc], then the exponentials [njob]
    __host__ __device__ static size_t doubles(int nrc, int njob) {
        return (size_t)kRec + kWRec * (size_t)(nrc > 0 ? nrc : 1) + (njob > 0 ? njob : 1);
    }
};

// a lane's place in its warp
template <int N>
struct SLane {
    static constexpr int S = N, G = 32 / N;
    static constexpr int kLevels = (S > 8) ? 4 : (S > 4) ? 3 : (S > 2) ? 2 : 1;  // ceil(log2 S)
    int lane, sl, base;
    bool act;              // the lane belongs to a cell segment (lanes above G * S idle)
    unsigned bits;         // the segment's lanes
    int rot[kLevels];      // lane base + (sl + 2^l) mod S

    __device__ void init(int l) {
        lane = l;
        const int seg = l / S;
        act = seg < G;
        base = act ? seg * S : G * S;
        sl = l - base;
        const unsigned m = (S >= 32) ? 0xffffffffu : ((1u << S) - 1u);
        bits = act ? (m << base) : ((G * S >= 32) ? 0u : (0xffffffffu << (G * S)));
#pragma unroll
        for (int i = 0; i < kLevels; ++i) {
            const int r = act ? base + (sl + (1 << i)) % S : l;
            rot[i] = r & 31;
        }
    }
    // sum over the segment, every lane of the segment gets it (a tree to the
    // segment's first lane, then a broadcast); `mask` names the lanes taking part
    __device__ __forceinline__ double sum(double v, unsigned mask) const {
#pragma unroll
        for (int o = (S > 16) ? 16 : (S > 8) ? 8 : (S > 4) ? 4 : (S > 2) ? 2 : 1; o > 0; o >>= 1) {
            const bool take = sl < o && sl + o < S;
            const double w = __shfl_sync(mask, v, take ? ((lane + o) & 31) : lane);
            if (take) v += w;
        }
        return __shfl_sync(mask, v, base & 31);
    }
    // max over the segment by rotation (windows of 2^levels >= S lanes)
    __device__ __forceinline__ double max(double v, unsigned mask) const {
#pragma unroll
        for (int i = 0; i < kLevels; ++i) {
            const double w = __shfl_sync(mask, v, rot[i]);
            v = (v < w) ? w : v;
        }
        return v;
    }
    __device__ __forceinline__ bool any(bool c, unsigned mask) const { return (__ballot_sync(mask, c) & bits) != 0u; }
};

// One cell segment's view of the chemistry (records, rows, LU, solve).
template <int N>
struct SCtx {
    static constexpr int TI = N - 1;
    using SL = SLayout<N>;
    const WMech &m;
    const WTabs &tb;
    const SLane<N> &L;
    double *s;        // this segment's shared memory
    int nsp, rs;      // species; record stride (= reactions)
    int lpos;         // LU: logical row of this lane's physical row
    double a[N];      // LU: this lane's row of I - dt J

    __device__ SCtx(const WMech &mm, const WTabs &t, const SLane<N> &ln, double *sm)
        : m(mm), tb(t), L(ln), s(sm), nsp(mm.nsp), rs(mm.nrc > 0 ? mm.nrc : 1), lpos(ln.sl) {
#pragma unroll
        for (int j = 0; j < N; ++j) a[j] = 0.0;
    }

    __device__ __forceinline__ const double *rdp(int r) const { return tb.rd + (r >> 5) * (kWRDn * 32) + (r & 31); }
    __device__ __forceinline__ const int32_t *rip(int r) const { return tb.ri + (r >> 5) * (kWRIn * 32) + (r & 31); }

    // f(y) and, when jac, the Jacobian rows into shared memory. Called by the
    // whole warp; y is this lane's element.
    __device__ __forceinline__ double evaluate(double y, bool jac) {
        const unsigned full = 0xffffffffu;
        const int sl = L.sl;
        const bool act = L.act;
        const double T = __shfl_sync(full, y, (L.base + TI) & 31);
        const double Tm = hmax(T, kTiny);
        const double logT = log(Tm);
        const double invT = frcp(Tm);
        const double invRuT = invT * (1.0 / kRu);
        double *sv = s + SL::kSV;
        constexpr int S = SL::S;
        const bool sp = act && sl < nsp;
        // ---- species
        double cp = 0.0, dcp = 0.0, h = 0.0;
        bool slow = false;
        if (sp) {
            const double *ts = tb.th + sl;
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
                t3_thermo_slow(&m.raw[14 * sl + ((T < tc) ? 0 : 7)], tl, thh, th(kWW), T, logT, invRuT, cp, h,
                               dcp, g, dgt);
                slow = true;
            }
            slow = slow || !(fabs(g) < m.glim);
            const double e = exp(hmin(hmax(g, -m.glim), m.glim));
            sv[0 * S + sl] = hmax(y, 0.0);
            sv[1 * S + sl] = h;
            sv[2 * S + sl] = e;
            sv[3 * S + sl] = frcp(e);
            sv[4 * S + sl] = g;
            sv[5 * S + sl] = dgt;
        }
        const bool cslow = L.any(slow, full);
        const double cCp = L.sum(sp ? y * cp : 0.0, full);
        const double dcCpdT = jac ? L.sum(sp ? y * dcp : 0.0, full) : 0.0;
        __syncwarp();
        // ---- exponentials, then the reactions' records
        double *X = s + SL::kRec + kWRec * rs;
        const int njob = act ? m.njob : 0, nrc = act ? m.nrc : 0;
#pragma unroll 1
        for (int j = sl; j < njob; j += S) {
            const double *xj = tb.xj + (j >> 5) * 96 + (j & 31);
            X[j] = exp(xj[0] * logT + xj[32] * invT + xj[64] * T);
        }
        __syncwarp();
#pragma unroll 1
        for (int r = sl; r < nrc; r += S) reaction(r, T, logT, invT, invRuT, cslow, jac, s + SL::kRec + r, X);
        __syncwarp();
        // ---- rows of f and J
        double f = 0.0, jt = 0.0, Sx = 0.0;
        double *Jrow = s + SL::kJ + sl * SL::LD;
        // rows of the species and of padding species between them and T
        // (zero rows: identity rows of I - dt J)
        if (jac && act && sl < N - 1) {
#pragma unroll
            for (int j = 0; j < N; ++j) Jrow[j] = 0.0;
        }
        if (sp) {
            const int e0 = tb.lptr[sl], e1 = tb.lptr[sl + 1];
#pragma unroll 1
            for (int e = e0; e < e1; ++e) {
                const int w0 = tb.lent[3 * e];
                const int r = w0 & 0xffff, pos = (w0 >> 16) & 7, np = (w0 >> 20) & 15;
                const double *R = s + SL::kRec + r;
                const double nu = tb.lnu[e];
                f += nu * R[0];
                if (!jac) continue;
                jt += nu * R[rs];
                Sx += R[3 * rs] * R[(4 + pos) * rs];
                const unsigned c0 = (unsigned)tb.lent[3 * e + 1], c1 = (unsigned)tb.lent[3 * e + 2];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    if (k >= np) break;
                    const int col = ((k < 4 ? c0 : c1) >> (8 * (k & 3))) & 0xff;
                    Jrow[col] += nu * R[(4 + k) * rs];
                }
                if (w0 & (1 << 24)) {
                    const double gn = nu * R[2 * rs];
                    const double *er = &tb.eff[(size_t)r * nsp];
#pragma unroll 1
                    for (int j = 0; j < nsp; ++j) Jrow[j] += er[j] * gn;
                }
            }
            if (jac) {
                // the temperature row's third-body / fall-off columns
#pragma unroll 1
                for (int t = 0; t < m.ntb; ++t) {
                    const int r = tb.tbl[t];
                    const double *R = s + SL::kRec + r;
                    Sx += R[3 * rs] * (tb.eff[(size_t)r * nsp + sl] * R[2 * rs]);
                }
            }
        }
        // ---- temperature equation (constant pressure, chemistrySource.cpp:863-883, 991-1021)
        const double icCp = frcp(cCp);
        const double DTdt = L.sum(sp ? f * h : 0.0, full) * icCp;
        if (act && sl == TI) f = -DTdt;
        if (jac) {
            const double cpf = L.sum(sp ? cp * f + h * jt : 0.0, full);
            if (act && sl < N - 1) {
                Jrow[TI] = jt;
                s[SL::kJ + TI * SL::LD + sl] = sp ? (cp * DTdt - Sx) * icCp : 0.0;
            }
            if (act && sl == TI) Jrow[TI] = (dcCpdT * DTdt - cpf) * icCp;
        }
        __syncwarp();
        return f;
    }

    // one reaction's record, fields R[k * rs] (reactionTypes q / Kc / DqDci /
    // DqDT, reactionTypes.cpp:178-445, 843-876; ArrheniusRR,
    // unimolecularFallOffRR, fallOffFunctions Troe / Lindemann)
    __device__ __forceinline__ void reaction(int r, double T, double logT, double invT, double invRuT, bool slow,
                                             bool jac, double *R, const double *X) {
        constexpr int S = SL::S;
        const double *sv = s + SL::kSV;
        const double *x = rdp(r);
        const int32_t *xi = rip(r);
        const int type = xi[kWtype * 32], rev = xi[kWrev * 32], nf = xi[kWnf * 32], nb = xi[kWnb * 32];
        // concentration powers of the reactants (pf) and products (pb)
        double pf[kMaxSide], pb[kMaxSide];
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            pf[k] = (k < nf) ? s_pow(sv[xi[(kWidx + k) * 32]], x[(kWord + k) * 32]) : 1.0;
            pb[k] = (k < nb) ? s_pow(sv[xi[(kWidx + nf + k) * 32]], x[(kWord + nf + k) * 32]) : 1.0;
        }
        double M = 0.0;
        if (type != kArrhenius) {
            const double *er = &tb.eff[(size_t)r * nsp];
#pragma unroll 1
            for (int j = 0; j < nsp; ++j) M += er[j] * sv[j];
        }
        const double b = x[kWb * 32], Ta = x[kWTa * 32];
        const double kx = x[kWA * 32] * X[r];
        double kf, k0 = 0.0, Pr = 0.0, Ff = 1.0, logPr = 0.0;
        T3Cent cent{0.0, 0.0};
        if (type == kArrhenius) {
            kf = kx;
        } else if (type == kThirdBody) {
            kf = M * kx;
        } else {
            // unimolecularFallOffRR::k (unimolecularFallOffRR.cpp:37-53)
            const int xj = xi[kWxj * 32];
            k0 = x[kWA0 * 32] * X[xj];
            Pr = fdiv(k0, notZeroD(kx)) * M;
            if (type != kLindemann) {
                cent = t3_troe_cent(type == kTroe4, x[kWalpha * 32], x[kWiTsss * 32], x[kWiTs * 32], x[kWTss * 32],
                                    X[xj + 1], X[xj + 2], (type == kTroe4) ? X[xj + 3] : 0.0, invT);
                logPr = log10(hmax(Pr, kTiny));
                Ff = t3_troe_F(cent.lf, logPr);
            }
            kf = kx * (Pr / (1.0 + Pr)) * Ff;
        }
        // reaction enthalpy (T row, T corner; DG0/DT - G0/T = -H0/T in the fitted range)
        double dH = 0.0;
        for (int k = 0; k < nf + nb; ++k) dH += x[(kWnu + k) * 32] * sv[S + xi[(kWidx + k) * 32]];
        // kr = kf krf; dkr/dT = dkf/dT ra - kf rb
        double krf = 0.0, ra = 0.0, rb = 0.0;
        const double s_ = x[kWs * 32];
        if (rev) {
            if (!slow) {
                double ik = 1.0;
                for (int k = 0; k < nf; ++k) ik *= pow_small(sv[3 * S + xi[(kWidx + k) * 32]], -x[(kWnu + k) * 32]);
                for (int k = nf; k < nf + nb; ++k) ik *= pow_small(sv[2 * S + xi[(kWidx + k) * 32]], x[(kWnu + k) * 32]);
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
                    kp += nu * sv[4 * S + i];
                    dk += nu * sv[5 * S + i];
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
            t3_falloff_jac_fast(type != kLindemann, cent, Ff, logPr, k0, kx, x[kWb0 * 32], x[kWTa0 * 32], b, Ta, M, q,
                                invT, g, dgdT);
            dq += dgdT;
        }
        R[1 * rs] = dq;
        R[2 * rs] = g;
        R[3 * rs] = dH;
        // d q / d c_k (reactionTypes::DqDci, reactionTypes.cpp:354-445): forward
        // products for the reactants, minus the reverse products for the products
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int n = side ? nb : nf, off = side ? nf : 0;
            const double K = side ? (rev ? -kr : 0.0) : kf;
            // d c^o / d c of each participant (1 for o = 1: the product skips it)
            double dp[kMaxSide];
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                dp[k] = 1.0;
                if (k < n) {
                    const double o = x[(kWord + off + k) * 32];
                    if (o != 1.0) dp[k] = s_dconc(sv[xi[(kWidx + off + k) * 32]], o);
                }
            }
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k >= n) break;
                double d = K;
#pragma unroll
                for (int l = 0; l < kMaxSide; ++l) {
                    if (l >= n) break;
                    d *= (l == k) ? dp[k] : (side ? pb[l] : pf[l]);
                }
                R[(4 + off + k) * rs] = d;
            }
        }
    }

    // A = I - dt J from this lane's row of J, then the pivoted LU. Called by
    // the whole warp; segments with fac false keep their previous factors.
    // The pivot steps are a loop (one copy of the step's code): column k of
    // the lane's row is picked from the registers by a select chain and the
    // broadcasts of the pivot row skip the columns left of k (a warp-uniform
    // test).
    __device__ __forceinline__ void factor(double dt, bool fac) {
        const unsigned full = 0xffffffffu;
        const int sl = L.sl;
        const bool act = L.act;
        if (fac) {
            const double *Jrow = s + SL::kJ + sl * SL::LD;
#pragma unroll
            for (int j = 0; j < N; ++j) a[j] = act ? (((sl == j) ? 1.0 : 0.0) - dt * Jrow[j]) : 0.0;
            lpos = sl;
        }
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
            double ak = a[0];
#pragma unroll
            for (int j = 1; j < N; ++j)
                if (j == k) ak = a[j];
            // argmax of |a(k)| over the rows not yet pivoted, the first in the
            // current logical order on ties
            double v = (act && lpos >= k) ? fabs(ak) : -1.0;
            int key = (lpos << 5) | sl;
#pragma unroll
            for (int i = 0; i < SLane<N>::kLevels; ++i) {
                const double w = __shfl_sync(full, v, L.rot[i]);
                const int kw = __shfl_sync(full, key, L.rot[i]);
                if (w > v || (w == v && kw < key)) {
                    v = w;
                    key = kw;
                }
            }
            const int pl = key & 31;          // pivot lane (in the segment)
            const int pos_p = key >> 5;       // its logical position
            const int src = (L.base + pl) & 31;
            const double inv = frcp(__shfl_sync(full, ak, src));
            const bool piv = sl == pl;
            if (fac) {
                // the rows swap logical positions k and pos_p
                if (piv) lpos = k;
                else if (lpos == k) lpos = pos_p;
            }
            const bool below = fac && act && !piv && lpos > k;
            const double l = ak * inv;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                if (j < k) continue;          // uniform: k is the same in all lanes
                if (j == k) {
                    if (fac && piv) a[j] = inv;
                    else if (below) a[j] = l;
                } else {
                    const double uj = __shfl_sync(full, a[j], src);
                    if (below) a[j] -= l * uj;
                }
            }
        }
    }

    // (L U) x = P b along the logical order; b and x are this lane's
    // elements. Called by the whole warp.
    __device__ __forceinline__ double solve(double b) {
        const unsigned full = 0xffffffffu;
        const int sl = L.sl;
        const bool act = L.act;
        int src[N];
#pragma unroll
        for (int t = 0; t < N; ++t) {
            const unsigned bt = (__ballot_sync(full, act && lpos == t) & L.bits) >> (L.base & 31);
            src[t] = (L.base + __ffs(bt) - 1) & 31;
        }
        double acc = 0.0, z = 0.0;
#pragma unroll
        for (int t = 0; t < N; ++t) {
            const double zt = __shfl_sync(full, b - acc, src[t]);
            if (lpos == t) z = zt;
            if (act && lpos > t) acc += a[t] * zt;
        }
        double x = 0.0;
        acc = 0.0;
#pragma unroll
        for (int t = N - 1; t >= 0; --t) {
            const double xt = __shfl_sync(full, (z - acc) * a[t], src[t]);
            if (sl == t) x = xt;
            if (act && lpos < t) acc += a[t] * xt;
        }
        return act ? x : 0.0;
    }
};

#ifndef HC_S_MIN_BLOCKS
#define HC_S_MIN_BLOCKS 2   // blocks of kSWarps warps per SM the kernel is built for
#endif
constexpr int kSWarps = 8;  // warps per block

template <int N>
__global__ void __launch_bounds__(32 * kSWarps, HC_S_MIN_BLOCKS)
integrate_s_kernel(const __grid_constant__ WMech m, const __grid_constant__ IntegratorParams P,
                   const __grid_constant__ CellIO io) {
    using SL = SLayout<N>;
    constexpr int TI = N - 1;
    extern __shared__ double smem_s[];
    const int nsp = m.nsp;
    const unsigned full = 0xffffffffu;
    // the mechanism tables into the block's shared memory, once
    WTabs tb;
    {
        double *d = smem_s;
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
    SLane<N> L;
    L.init(threadIdx.x & 31);
    const int warp = threadIdx.x >> 5;
    const size_t tab = w_tables_bytes(nsp, m.nrc, m.nrc32, m.nent, m.ntb, m.njob32) / sizeof(double);
    // idle lanes read (never write) the warp's first segment
    const int seg = L.act ? L.lane / N : 0;
    double *s = smem_s + tab + ((size_t)warp * SL::G + seg) * SL::doubles(m.nrc, m.njob);
    SCtx<N> cx(m, tb, L, s);
    const int sl = L.sl;
    const unsigned mask = L.bits;       // this segment's lanes (bookkeeping shuffles)
    const int src_T = (L.base + TI) & 31;
    const bool sp = L.act && sl < nsp;
    const double W = sp ? tb.th[kWW * 32 + sl] : 1.0;
    const double iW = frcp(W);
    const bool autoJ = P.auto_update_jacobian != 0;
    const int stepJ = P.step_to_update_jac > 0 ? P.step_to_update_jac : 1;

    // this lane's elements: y (accepted state), yk (Newton iterate), yk0 / yk1
    // (yklast_[0], [1]), c0 (initial concentration, for Ri)
    double y = 0.0, yk = 0.0, yk0 = 0.0, yk1 = 0.0, c0 = 0.0;
    int state = L.act ? kT1Fetch : kT1Done;
    int64_t cellid = -1;
    double leftTime = 0, sub = 0, tstep = 0, p = 0;
    double t = 0, tn = 0, dt = 0, dtReached = 0, dtTry0 = 0, adt = 0, lts0 = 0, lts1 = 0;
    double lastErr = 0, Told = 0, error = 0;
    int nstep = 0, tcount = 0, ncount = 0, cstatus = 0;
    bool last = false, jacNow = true;
    int n_jac = 0, n_rhs = 0, n_lu = 0, n_newton = 0, n_steps = 0, n_att = 0;

    while (true) {
        // ---------------- bookkeeping of each segment up to its next heavy state
        int guard = 0;
        while (state != kT1Newton && state != kT1Err0 && state != kT1Done && guard < 64) {
            ++guard;
            if (state == kT1Fetch) {
                if (cellid >= 0) {
                    // finish the previous cell: ciToYi (chemistrySource.cpp:1225-1246) and rho = p / (Rm T)
                    const double Tn = __shfl_sync(mask, y, src_T);
                    double yi = sp ? hmax(0.0, y) : 0.0;
                    const double rr = L.sum(yi * (sp ? W : 0.0), mask);
                    yi = sp ? yi * W * frcp(hmax(rr, kTiny)) : 0.0;
                    const double ys = L.sum(yi, mask);
                    if (ys != 1.0) yi *= frcp(ys);
                    const double wsum = L.sum(sp ? yi * iW : 0.0, mask);
                    const double Rm = kRu * hmax(wsum, kVeryTiny);
                    if (sp) {
                        const int64_t at = (int64_t)sl * io.ncells + cellid;
                        io.Y[at] = yi;
                        if (io.Ri) io.Ri[at] = (y - c0) * frcp(tstep) * W;
                    }
                    if (sl == 0) {
                        io.T[cellid] = Tn;
                        io.rho[cellid] = fdiv(p, Rm * Tn);
                        io.subdt[cellid] = sub;
                        if (io.status) io.status[cellid] = cstatus;
                        if (io.cost) io.cost[cellid] = n_newton;
                        if (io.counters) {
                            atomicAdd(&io.counters[0], (unsigned long long)n_jac);
                            atomicAdd(&io.counters[1], (unsigned long long)n_rhs);
                            atomicAdd(&io.counters[2], (unsigned long long)n_lu);
                            atomicAdd(&io.counters[3], (unsigned long long)n_newton);
                            atomicAdd(&io.counters[4], (unsigned long long)n_steps);
                            atomicAdd(&io.counters[5], (unsigned long long)n_att);
                        }
                    }
                    cellid = -1;
                }
                long long k = 0;
                if (sl == 0) k = (long long)atomicAdd(io.queue_head, 1ULL);
                k = __shfl_sync(mask, k, L.base & 31);
                if (k >= io.nqueue) {
                    state = kT1Done;
                    break;
                }
                cellid = io.order ? (int64_t)io.order[k] : (int64_t)k;
                n_jac = n_rhs = n_lu = n_newton = n_steps = n_att = 0;
                cstatus = 0;
                const double Ti = io.T[cellid];
                tstep = io.dt[cellid] * io.dt_factor;
                if (Ti < P.T_threshold) {
                    if (sl == 0) {
                        io.subdt[cellid] = tstep;
                        if (io.status) io.status[cellid] = 1;   // HC_CELL_SKIPPED
                        if (io.cost) io.cost[cellid] = 0;
                    }
                    if (io.Ri && sp) io.Ri[(int64_t)sl * io.ncells + cellid] = 0.0;
                    cellid = -1;
                    continue;
                }
                const double rho0 = io.rho[cellid];
                y = sp ? rho0 * io.Y[(int64_t)sl * io.ncells + cellid] * iW : 0.0;
                c0 = y;
                if (sl == TI) y = Ti;
                p = io.p[cellid];
                leftTime = tstep;
                sub = hmin(leftTime, hmin(io.subdt[cellid], P.dt_max));
                state = kT1Interval;
            } else if (state == kT1Interval) {
                // ImplicitEuler::solve(t0 = 0, tn = leftTime, dt0 = sub, y)
                tn = leftTime;
                t = 0.0;
                dt = 0.2 * sub;
                dtReached = 0.0;
                last = false;
                nstep = 0;
                state = kT1Step;
            } else if (state == kT1Step) {
                if (nstep >= P.maxstep) {
                    cstatus |= 2;       // HC_CELL_MAXSTEP
                    tn = dtReached;
                    leftTime -= tn;
                    state = (leftTime > 0.0) ? kT1Interval : kT1Fetch;
                    continue;
                }
                if (nstep == 0) {
                    yk0 = y;
                } else {
                    yk1 = yk0;
                    yk0 = y;
                }
                dtTry0 = dt;
                if ((t + dt - tn) * (t + dt - 0.0) > 0) {
                    dt = tn - t;
                    last = true;
                } else if (t + dt == tn) {
                    last = true;
                }
                // ImplicitEuler::adaptiveSolve start
                adt = dt;
                lts1 = lts0;
                tcount = 0;
                Told = __shfl_sync(mask, y, src_T);
                state = kT1Attempt;
            } else if (state == kT1Attempt) {
                lts0 = adt;
                ++n_att;
                yk = y;
                ncount = 0;
                lastErr = 0.0;
                jacNow = true;
                state = kT1Newton;
            } else {   // kT1AttemptEnd
                // adaptiveSolve after solve(): checkNewY, then the error test
                const double Tnew = __shfl_sync(mask, yk, src_T);
                bool ok = true;
                if ((Tnew - Told) > P.T_alpha * Told) {
                    adt *= P.T_beta;
                    ok = false;
                }
                if (!ok && tcount < 100) {
                    error = 2;
                    tcount++;
                    if (adt <= kVeryTiny) {
                        cstatus |= 4;
                        state = kT1Fetch;
                        continue;
                    }
                    state = kT1Attempt;
                    continue;
                }
                if (error > 1.0) {
                    const double scale = hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale);
                    adt *= scale;
                    if (adt <= kVeryTiny) {
                        cstatus |= 4;
                        state = kT1Fetch;
                        continue;
                    }
                    state = kT1Attempt;
                    continue;
                }
                // accepted
                t += adt;
                y = yk;
                ++n_steps;
                if (error > P.err_accept_limit)
                    dt = hmin(hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale), P.maxscale) * adt;
                else
                    dt = hmax(P.safescale * P.maxscale * adt, adt);
                dtReached = t;
                if ((t - tn) * (tn - 0.0) >= 0) {
                    if (nstep > 0 && last) sub = hmin(dtTry0, tn);
                    leftTime -= tn;
                    state = (leftTime > 0.0) ? kT1Interval : kT1Fetch;
                } else {
                    ++nstep;
                    state = kT1Step;
                }
            }
        }
        // ---------------- heavy block, the whole warp: f (J) at yk, LU, solve
        if (__ballot_sync(full, state != kT1Done) == 0u) break;    // no cell left in the warp
        const bool heavy = state == kT1Newton || state == kT1Err0;
        if (__ballot_sync(full, heavy) == 0u) continue;
        const bool newton = state == kT1Newton;
        const bool fac = newton && jacNow;
        const bool anyJ = __ballot_sync(full, fac) != 0u;
        const double f = cx.evaluate(yk, anyJ);
        if (anyJ) cx.factor(lts0, fac);
        double x = 0.0;
        if (__ballot_sync(full, newton) != 0u) x = cx.solve(L.act ? ((-yk + y) + lts0 * f) : 0.0);
        if (newton) {
            if (fac) {
                ++n_jac;
                ++n_lu;
            } else {
                ++n_rhs;
            }
            ++n_newton;
            // ImplicitEuler::NewtonIteration update and tests (ImplicitEuler.cpp:161-251)
            const unsigned bad = (__ballot_sync(mask, !finite(x)) & L.bits) >> (L.base & 31);
            if (bad) {
                const int firstBad = __ffs(bad) - 1;
                if (sl < firstBad) yk += x;
                error = 1000.0;
                state = kT1AttemptEnd;
            } else {
                yk += x;
                double v = fabs(x) * frcp(P.atol + P.rtol * hmax(fabs(yk), fabs(yk)));
                if (isnan(v)) v = 0.0;
                const double maxErr = L.max(v, mask);
                bool fail = false;
                if (ncount > 0) {
                    const double diver = maxErr * frcp(hmax(lastErr, kTiny));
                    if (autoJ) {
                        const int lim = (30 * stepJ > 50) ? 30 * stepJ : 50;
                        fail = diver > 2 && ncount > lim;
                    } else {
                        fail = diver > 2 && ncount > 5;
                    }
                }
                if (fail) {
                    error = 1000.0;
                    state = kT1AttemptEnd;
                } else {
                    lastErr = maxErr;
                    ncount++;
                    jacNow = !autoJ || ncount % stepJ == 0;
                    if (isnan(maxErr)) {
                        error = 1000.0;
                        state = kT1AttemptEnd;
                    } else if (ncount > 1000) {
                        error = maxErr;
                        state = kT1AttemptEnd;
                    } else if (P.max_newton_total > 0 && n_newton >= P.max_newton_total) {
                        cstatus |= 8;
                        state = kT1Fetch;
                    } else if (maxErr > 1.0) {
                        state = kT1Newton;
                    } else if (nstep == 0) {
                        state = kT1Err0;     // first step: error from f(y_k)
                    } else {
                        // 3-point error estimate (ImplicitEuler.cpp:121-140), maxIncrement
                        const double dtn = lts0, dtn1 = lts1;
                        const double f1 = 2.0 * frcp(dtn * (dtn + dtn1));
                        const double f2 = 2.0 * frcp(dtn1 * (dtn + dtn1));
                        const double LTEF = (dtn * dtn) * 0.5;
                        double e = f1 * (yk - y) - f2 * (y - yk1);
                        e *= LTEF;
                        const bool nan_y = L.any(isnan(yk), mask);
                        double w = fabs(e) * frcp(P.atol_inc + P.rtol_inc * hmax(fabs(y), fabs(yk)));
                        if (isnan(w)) w = 0.0;
                        const double me = L.max(w, mask);
                        error = nan_y ? 1.5 : me;
                        state = kT1AttemptEnd;
                    }
                }
            }
        } else if (state == kT1Err0) {
            // error = maxIncrement(y0, yk, yk - y0 - dt f(yk))
            ++n_rhs;
            const double e = yk - y - lts0 * f;
            const bool nan_y = L.any(isnan(yk), mask);
            double w = fabs(e) * frcp(P.atol_inc + P.rtol_inc * hmax(fabs(y), fabs(yk)));
            if (isnan(w)) w = 0.0;
            const double me = L.max(w, mask);
            error = nan_y ? 1.5 : me;
            state = kT1AttemptEnd;
        }
    }
}

}  // namespace hc
