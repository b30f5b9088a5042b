// Compact thread-per-cell integrator (kernel 5), generated per mechanism at
// run time and compiled with NVRTC for sm_100a.
//
// The generated source holds only the mechanism, as constant tables in the
// layout of t4_cell.cuh (NASA-7 coefficients pre-multiplied by W and by the
// polynomial factors for both ranges, reactions in the mechanism's own order
// with their stoichiometry, orders, rate and Troe parameters, the non-zero
// third-body efficiencies), and a kernel that runs the implicit-Euler state
// machine of t1_body.cuh over T4Cell. The Newton iteration itself is the
// short loops of t4_cell.cuh, so that it fits the SM's instruction cache.
#include <cmath>
#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hurchem_b200.h"
#include "jit.h"

namespace hc {

namespace {

std::string L(double v) {
    char buf[64];
    if (v == 0.0) return std::signbit(v) ? "(-0.0)" : "0.0";
    if (std::isinf(v)) return v > 0 ? "(__longlong_as_double(0x7ff0000000000000LL))" : "(-__longlong_as_double(0x7ff0000000000000LL))";
    std::snprintf(buf, sizeof(buf), "%a", v);
    return std::string("(") + buf + ")";
}

std::string I(int v) { return std::to_string(v); }

std::string list(const double *v, int n) {
    std::string s = "{";
    for (int k = 0; k < n; ++k) s += (k ? ", " : "") + L(v[k]);
    return s + "}";
}

// largest |G0/(Ru T)| for which every product of exp(+-g) that a reaction's
// 1/Kc needs stays far inside the double range
double g_limit(const HostMech &h) {
    double worst = 1.0;
    for (int r = 0; r < h.nrc; ++r) {
        if (!h.reversible[r]) continue;
        double sn = 0.0;
        for (int k = 0; k < h.nf[r]; ++k) sn += std::fabs(h.fnu[HC_MAX_SIDE * r + k]);
        for (int k = 0; k < h.nb[r]; ++k) sn += std::fabs(h.bnu[HC_MAX_SIDE * r + k]);
        worst = std::max(worst, sn);
    }
    return std::min(300.0, 580.0 / worst);
}

}  // namespace

// c^o with a literal order (conc_pow: 1 and 2 exactly, pow otherwise)
std::string cpow_lit(const std::string &c, double o) {
    if (o == 1.0) return c;
    if (o == 2.0) return "(" + c + " * " + c + ")";
    if (o == 0.0) return "1.0";
    return "pow(" + c + ", " + L(o) + ")";
}

// d(c^o)/dc as reactionTypes::DqDci forms it (o != 1)
std::string dcpow_lit(const std::string &c, double o) {
    if (o == 2.0) return "(2.0 * " + c + ")";
    if (o < 1.0) return "((" + c + " > kTiny) ? " + L(o) + " * pow(" + c + ", " + L(o - 1.0) + ") : 0.0)";
    return "(" + L(o) + " * pow(" + c + ", " + L(o - 1.0) + "))";
}

std::string pow_nu(const std::string &x, double nu) {
    if (nu == 1.0) return x;
    if (nu == 2.0) return "(" + x + " * " + x + ")";
    if (nu == 3.0) return "(" + x + " * " + x + " * " + x + ")";
    return "pow(" + x + ", " + L(nu) + ")";
}

// "a -= nu * w" / "a += nu * w" with unit coefficients folded
std::string acc(const std::string &a, bool minus, double nu, const std::string &w) {
    return a + (minus ? " -= " : " += ") + (nu == 1.0 ? w : L(nu) + " * " + w) + ";";
}

// The common path of the reaction pass: reactions grouped by shape (rate
// form, reversibility, side sizes, stoichiometric coefficients, orders); per
// shape one loop over its reactions whose body is written for that shape
// (no per-participant predicates), with the species indices and rate
// parameters of each reaction read from the constant table kR5.
void emit_shapes(std::ostringstream &o, const HostMech &h, const std::vector<int> &order) {
    const int nsp = h.nsp, nrc = h.nrc, S = HC_MAX_SIDE;
    // group reactions by shape, shapes in order of first appearance
    std::vector<std::vector<int>> groups;
    std::vector<std::string> keys;
    for (int rr = 0; rr < nrc; ++rr) {
        const int r = order[rr];
        std::ostringstream k;
        k << h.rate_type[r] << "|" << (h.reversible[r] ? 1 : 0) << "|" << h.nf[r] << "|" << h.nb[r];
        for (int j = 0; j < h.nf[r]; ++j) k << "|" << L(h.fnu[S * r + j]) << ":" << L(h.ford[S * r + j]);
        for (int j = 0; j < h.nb[r]; ++j) k << "|" << L(h.bnu[S * r + j]) << ":" << L(h.bord[S * r + j]);
        size_t g = 0;
        while (g < keys.size() && keys[g] != k.str()) ++g;
        if (g == keys.size()) {
            keys.push_back(k.str());
            groups.emplace_back();
        }
        groups[g].push_back(rr);
    }
    // efficiency ranges in kEff (the order kRx was emitted in)
    std::vector<int> e0(nrc, 0), e1(nrc, 0);
    {
        int ne = 0;
        for (int rr = 0; rr < nrc; ++rr) {
            const int r = order[rr];
            e0[rr] = ne;
            if (h.rate_type[r] != HC_RATE_ARRHENIUS)
                for (int i = 0; i < nsp; ++i)
                    if (h.eff[(size_t)r * nsp + i] != 0.0) ++ne;
            e1[rr] = ne;
        }
    }
    o << "struct T5R { int sp[" << 2 * S << "]; double A, b, Ta, A0, b0, Ta0, alpha, iTsss, iTs, Tss; "
         "int e0, e1; };\n"
      << "__constant__ T5R kR5[" << std::max(nrc, 1) << "] = {\n";
    int count = 0;
    for (const auto &g : groups) {
        for (int rr : g) {
            const int r = order[rr];
            const int nf = h.nf[r], nb = h.nb[r];
            const double *tr = &h.troe[4 * r];
            const bool troe = h.rate_type[r] == HC_RATE_TROE3 || h.rate_type[r] == HC_RATE_TROE4;
            o << "  {{";
            for (int k = 0; k < 2 * S; ++k) {
                int v = 0;
                if (k < nf) v = h.fidx[S * r + k];
                else if (k - nf < nb) v = h.bidx[S * r + k - nf];
                o << (k ? ", " : "") << v;
            }
            o << "}, " << L(h.arr[3 * r]) << ", " << L(h.arr[3 * r + 1]) << ", " << L(h.arr[3 * r + 2]) << ", "
              << L(h.arr0[3 * r]) << ", " << L(h.arr0[3 * r + 1]) << ", " << L(h.arr0[3 * r + 2]) << ", "
              << L(troe ? tr[0] : 0.0) << ", " << L(troe ? 1.0 / tr[1] : 0.0) << ", " << L(troe ? 1.0 / tr[2] : 0.0)
              << ", " << L(troe ? tr[3] : 0.0) << ", " << e0[rr] << ", " << e1[rr] << "}"
              << (++count < nrc ? "," : "") << "\n";
        }
    }
    if (nrc == 0) o << "  {}\n";
    o << "};\n}  // namespace hc\n#include \"t4_cell.cuh\"\nnamespace hc {\n"
      << "struct JitCell5 : T4Base<kN, kNSP, kB> {\n"
      << "  using Base = T4Base<kN, kNSP, kB>;\n"
      << "  __device__ JitCell5(double *smem, int tid) : Base(smem, tid) {}\n"
      << "  __device__ __forceinline__ void evaluate(const double (&y)[kN], bool jac, double dt) {\n"
      << "    const T4Ctx c = this->begin(y, jac, dt);\n"
      << "    const double htq = c.slow ? t4_reactions_table<kN, kNSP, kNRC, kB>(this->s, c, jac) : shapes(c, jac);\n"
      << "    this->finish(c, jac, htq);\n"
      << "  }\n"
      << "  __device__ __forceinline__ double shapes(const T4Ctx &c, bool jac) {\n"
      << "    constexpr int TI = kN - 1, kY = SL::kY, kH = SL::kH, kE = SL::kE, kR = SL::kR, kF = SL::kF, kA = SL::kA;\n"
      << "    double htq = 0.0;\n";
    int q0 = 0;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const int r = order[groups[gi][0]];
        const int type = h.rate_type[r];
        const bool rev = h.reversible[r] != 0;
        const int nf = h.nf[r], nb = h.nb[r];
        const double *fnu = &h.fnu[S * r], *bnu = &h.bnu[S * r];
        const double *fo = &h.ford[S * r], *bo = &h.bord[S * r];
        const int q1 = q0 + (int)groups[gi].size();
        const bool falloff = type >= HC_RATE_LINDEMANN;
        const bool troe = type == HC_RATE_TROE3 || type == HC_RATE_TROE4;
        auto F = [](int k) { return "f" + I(k); };
        auto Bk = [](int k) { return "b" + I(k); };
        o << "    // shape " << gi << ": " << keys[gi] << " (" << groups[gi].size() << " reactions)\n"
          << "#pragma unroll 1\n"
          << "    for (int n = " << q0 << "; n < " << q1 << "; ++n) {\n"
          << "      const T5R &x = kR5[n];\n";
        for (int k = 0; k < nf; ++k) o << "      const int f" << k << " = x.sp[" << k << "];\n";
        for (int k = 0; k < nb; ++k) o << "      const int b" << k << " = x.sp[" << nf + k << "];\n";
        for (int k = 0; k < nf; ++k) o << "      const double cf" << k << " = hmax(S(kY + f" << k << "), 0.0);\n";
        if (rev)
            for (int k = 0; k < nb; ++k) o << "      const double cb" << k << " = hmax(S(kY + b" << k << "), 0.0);\n";
        if (type != HC_RATE_ARRHENIUS)
            o << "      double M = 0.0;\n"
              << "#pragma unroll 1\n"
              << "      for (int k = x.e0; k < x.e1; ++k) M += kEff[k].e * hmax(S(kY + kEff[k].sp), 0.0);\n";
        o << "      const double kx = x.A * exp(x.b * c.logT - x.Ta * c.invT);\n";
        if (type == HC_RATE_ARRHENIUS) {
            o << "      const double kf = kx;\n";
        } else if (type == HC_RATE_THIRD_BODY) {
            o << "      const double kf = M * kx;\n";
        } else {
            // unimolecularFallOffRR::k (unimolecularFallOffRR.cpp:37-53)
            o << "      const double k0 = x.A0 * exp(x.b0 * c.logT - x.Ta0 * c.invT);\n"
              << "      const double Pr = fdiv(k0, notZeroD(kx)) * M;\n";
            if (troe) {
                o << "      const T3Cent cent = t3_troe_cent(" << (type == HC_RATE_TROE4 ? "true" : "false")
                  << ", x.alpha, x.iTsss, x.iTs, x.Tss, exp(-c.T * x.iTsss), exp(-c.T * x.iTs), "
                  << (type == HC_RATE_TROE4 ? "exp(-x.Tss * c.invT)" : "0.0") << ", c.invT);\n"
                  << "      const double logPr = log10(hmax(Pr, kTiny));\n"
                  << "      const double Ff = t3_troe_F(cent.lf, logPr);\n";
            } else {
                o << "      const T3Cent cent{0.0, 0.0};\n      const double logPr = 0.0, Ff = 1.0;\n";
            }
            o << "      const double kf = kx * (Pr / (1.0 + Pr)) * Ff;\n";
        }
        // reaction enthalpy (dH = sum nu h): the T row, the T corner and the
        // Kc derivative (DG0/DT - G0/T = -H0/T in the fitted range)
        o << "      const double dh = 0.0";
        for (int k = 0; k < nf; ++k) o << " - " << (fnu[k] == 1.0 ? "" : L(fnu[k]) + " * ") << "S(kH + f" << k << ")";
        for (int k = 0; k < nb; ++k) o << " + " << (bnu[k] == 1.0 ? "" : L(bnu[k]) + " * ") << "S(kH + b" << k << ")";
        o << ";\n";
        const double s = h.sum_stoi[r];
        if (rev) {
            // 1/Kc = prod exp(nu G0/(Ru T)) (Patm/(Ru T))^(-s)
            std::string prod;
            auto mul = [&](const std::string &v) { prod = prod.empty() ? v : prod + " * " + v; };
            for (int k = 0; k < nb; ++k) mul(pow_nu("S(kE + b" + I(k) + ")", bnu[k]));
            for (int k = 0; k < nf; ++k) mul(pow_nu("S(kR + f" + I(k) + ")", fnu[k]));
            if (s == -1.0) mul("c.PRT");
            else if (s == 1.0) mul("frcp(c.PRT)");
            else if (s != 0.0) mul("exp(" + L(-s) + " * c.lnPRT)");
            o << "      const double ik = " << (prod.empty() ? std::string("1.0") : prod) << ";\n"
              << "      const double kr = kf * ik;\n";
        }
        for (int k = 0; k < nf; ++k) o << "      const double pf" << k << " = " << cpow_lit("cf" + I(k), fo[k]) << ";\n";
        if (rev)
            for (int k = 0; k < nb; ++k) o << "      const double pb" << k << " = " << cpow_lit("cb" + I(k), bo[k]) << ";\n";
        o << "      const double q = kf";
        for (int k = 0; k < nf; ++k) o << " * pf" << k;
        if (rev) {
            o << " - kr";
            for (int k = 0; k < nb; ++k) o << " * pb" << k;
        }
        o << ";\n";
        for (int k = 0; k < nf; ++k) o << "      " << acc("S(kF + f" + I(k) + ")", true, fnu[k], "q") << "\n";
        for (int k = 0; k < nb; ++k) o << "      " << acc("S(kF + b" + I(k) + ")", false, bnu[k], "q") << "\n";
        o << "      if (jac) {\n";
        // d q / d T (reactionTypes.cpp:843-876)
        if (falloff)
            o << "        double dkf = (Pr / (1.0 + Pr)) * Ff * (kx * c.invT * (x.b + x.Ta * c.invT));\n";
        else
            o << "        double dkf = kf * c.invT * (x.b + x.Ta * c.invT);\n";
        if (rev)
            o << "        double dkr = dkf * ik - kf * (ik * (-dh * c.invT * c.invRuT"
              << (s != 0.0 ? " - " + L(s) + " * c.invT" : std::string()) << "));\n";
        for (int k = 0; k < S; ++k) {
            if (k < nf) o << "        dkf *= pf" << k << ";\n";
            if (rev && k < nb) o << "        dkr *= pb" << k << ";\n";
        }
        o << "        double dq = dkf" << (rev ? " - dkr" : "") << ";\n"
          << "        if (!finite(dq)) dq = 0.0;\n";
        if (type == HC_RATE_THIRD_BODY) {
            o << "        const double gr = fdiv(q, hmax(M, kTiny));\n";
        } else if (falloff) {
            o << "        double gr, dgdT;\n"
              << "        t3_falloff_jac_fast(" << (troe ? "true" : "false")
              << ", cent, Ff, logPr, k0, kx, x.b0, x.Ta0, x.b, x.Ta, M, q, c.invT, gr, dgdT);\n"
              << "        dq += dgdT;\n";
        }
        o << "        const double wq = c.mdt * dq;\n";
        for (int k = 0; k < nf; ++k) o << "        " << acc("S(kA + f" + I(k) + " * kN + TI)", true, fnu[k], "wq") << "\n";
        for (int k = 0; k < nb; ++k) o << "        " << acc("S(kA + b" + I(k) + " * kN + TI)", false, bnu[k], "wq") << "\n";
        o << "        htq += dh * dq;\n";
        // one Jacobian column: the participants' rows and the T row
        auto column = [&](const std::string &col, const std::string &v, bool neg) {
            o << "        { const double v = " << (neg ? "-(" + v + ")" : v) << ", w = c.mdt * v;\n";
            for (int l = 0; l < nf; ++l)
                o << "          " << acc("S(kA + f" + I(l) + " * kN + " + col + ")", true, fnu[l], "w") << "\n";
            for (int l = 0; l < nb; ++l)
                o << "          " << acc("S(kA + b" + I(l) + " * kN + " + col + ")", false, bnu[l], "w") << "\n";
            o << "          S(kA + TI * kN + " << col << ") += dh * v; }\n";
        };
        // d q / d c_j (reactionTypes::DqDci, reactionTypes.cpp:354-445): forward, then reverse
        for (int side = 0; side < 2; ++side) {
            if (side == 1 && !rev) break;
            const int n = side ? nb : nf;
            const double *ord = side ? bo : fo;
            for (int k = 0; k < n; ++k) {
                std::string d = side ? "kr" : "kf";
                for (int l = 0; l < n; ++l) {
                    if (l == k) {
                        if (ord[l] == 1.0) continue;
                        d += " * " + dcpow_lit((side ? "cb" : "cf") + I(l), ord[l]);
                    } else {
                        d += std::string(" * ") + (side ? "pb" : "pf") + I(l);
                    }
                }
                column(side ? Bk(k) : F(k), d, side == 1);
            }
        }
        if (type != HC_RATE_ARRHENIUS) {
            o << "#pragma unroll 1\n"
              << "        for (int k = x.e0; k < x.e1; ++k) {\n"
              << "          const int j = kEff[k].sp;\n";
            column("j", "kEff[k].e * gr", false);
            o << "        }\n";
        }
        o << "      }\n    }\n";
        q0 = q1;
    }
    o << "    return htq;\n  }\n};\n}  // namespace hc\n\n";
}

int t3_slots(int nsp) {
    const int N = nsp + 1;
    return N * N + N + 3 * nsp + N;
}

std::string jit_t3_source(const HostMech &h, int block) {
    const int nsp = h.nsp, N = nsp + 1, nrc = h.nrc, S = HC_MAX_SIDE;
    // reactions in the mechanism's own order (the device tables regroup them
    // by rate class; the reference sums f and J in file order)
    std::vector<int> order(nrc);
    for (int r = 0; r < nrc; ++r) order[r] = r;
    if ((int)h.perm.size() == nrc)
        for (int r = 0; r < nrc; ++r) order[h.perm[r]] = r;
    std::ostringstream o;
    o << "#include \"t1_body.cuh\"\n#include \"t3_base.cuh\"\n"
      << "namespace hc {\n"
      << "constexpr int kN = " << N << ", kNSP = " << nsp << ", kNRC = " << nrc << ", kB = " << block << ";\n"
      << "constexpr double kGLim = " << L(g_limit(h)) << ";\n";
    // species: molar NASA-7 for both ranges
    o << "__constant__ T4Species kSp[" << nsp << "] = {\n";
    for (int i = 0; i < nsp; ++i) {
        const double W = h.W[i];
        auto range = [&](int rg) {
            const double *a = &h.nasa[14 * i + 7 * rg];
            const double hc[5] = {W * a[0], W * a[1] / 2, W * a[2] / 3, W * a[3] / 4, W * a[4] / 5};
            const double sc[4] = {W * a[1], W * a[2] / 2, W * a[3] / 3, W * a[4] / 4};
            const double cp[5] = {W * a[0], W * a[1], W * a[2], W * a[3], W * a[4]};
            const double dc[4] = {W * a[1], 2 * W * a[2], 3 * W * a[3], 4 * W * a[4]};
            return "{" + list(hc, 5) + ", " + L(W * a[5]) + ", " + L(W * a[0]) + ", " + list(sc, 4) + ", " +
                   L(W * a[6]) + ", " + list(cp, 5) + ", " + list(dc, 4) + "}";
        };
        o << "  {" << L(h.Trange[3 * i]) << ", " << L(h.Trange[3 * i + 1]) << ", " << L(h.Trange[3 * i + 2])
          << ", " << L(W) << ",\n   " << range(0) << ",\n   " << range(1) << ",\n   {"
          << list(&h.nasa[14 * i], 7) << ", " << list(&h.nasa[14 * i + 7], 7) << "}}" << (i + 1 < nsp ? "," : "")
          << "\n";
    }
    o << "};\n";
    // efficiencies and reactions
    std::vector<std::pair<int, double>> effs;
    std::ostringstream rx;
    for (int rr = 0; rr < nrc; ++rr) {
        const int r = order[rr];
        const int type = h.rate_type[r];
        const int eb = (int)effs.size();
        if (type != HC_RATE_ARRHENIUS)
            for (int i = 0; i < nsp; ++i)
                if (h.eff[(size_t)r * nsp + i] != 0.0) effs.push_back({i, h.eff[(size_t)r * nsp + i]});
        const int ee = (int)effs.size();
        const double *tr = &h.troe[4 * r];
        const bool troe = type == HC_RATE_TROE3 || type == HC_RATE_TROE4;
        auto ilist = [&](const int *v, int n) {
            std::string s = "{";
            for (int k = 0; k < S; ++k) s += (k ? ", " : "") + I(k < n ? v[k] : 0);
            return s + "}";
        };
        auto dlist = [&](const double *v, int n) {
            double t[HC_MAX_SIDE];
            for (int k = 0; k < S; ++k) t[k] = k < n ? v[k] : 0.0;
            return list(t, S);
        };
        rx << "  {" << type << ", " << (h.reversible[r] ? 1 : 0) << ", " << h.nf[r] << ", " << h.nb[r] << ", "
           << ilist(&h.fidx[S * r], h.nf[r]) << ", " << ilist(&h.bidx[S * r], h.nb[r]) << ",\n   "
           << dlist(&h.fnu[S * r], h.nf[r]) << ", " << dlist(&h.bnu[S * r], h.nb[r]) << ", "
           << dlist(&h.ford[S * r], h.nf[r]) << ", " << dlist(&h.bord[S * r], h.nb[r]) << ",\n   "
           << L(h.arr[3 * r]) << ", " << L(h.arr[3 * r + 1]) << ", " << L(h.arr[3 * r + 2]) << ", "
           << L(h.arr0[3 * r]) << ", " << L(h.arr0[3 * r + 1]) << ", " << L(h.arr0[3 * r + 2]) << ",\n   "
           << L(troe ? tr[0] : 0.0) << ", " << L(troe ? 1.0 / tr[1] : 0.0) << ", " << L(troe ? 1.0 / tr[2] : 0.0)
           << ", " << L(troe ? tr[3] : 0.0) << ", " << L(troe ? tr[1] : 0.0) << ", " << L(troe ? tr[2] : 0.0)
           << ", " << L(h.sum_stoi[r]) << ", " << eb << ", " << ee << "}" << (rr + 1 < nrc ? "," : "") << "\n";
    }
    o << "__constant__ T4Rxn kRx[" << std::max(nrc, 1) << "] = {\n" << rx.str() << "};\n";
    o << "__constant__ T4Eff kEff[" << std::max<size_t>(effs.size(), 1) << "] = {";
    if (effs.empty()) o << "{0, 0.0}";
    for (size_t k = 0; k < effs.size(); ++k) o << (k ? ", " : "") << "{" << effs[k].first << ", " << L(effs[k].second) << "}";
    o << "};\n";
    emit_shapes(o, h, order);
    o << "extern \"C\" __global__ void __launch_bounds__(" << block << ")\n"
      << "hc_jit_t3(const __grid_constant__ hc::IntegratorParams P, const __grid_constant__ hc::CellIO io, "
         "double *ylast) {\n"
      << "  extern __shared__ double smem_jit[];\n"
      << "  hc::JitCell5 cell(smem_jit, threadIdx.x);\n"
      << "  hc::t1_run<hc::kN, true>(cell, P, io, ylast);\n"
      << "}\n";
    return o.str();
}

}  // namespace hc
