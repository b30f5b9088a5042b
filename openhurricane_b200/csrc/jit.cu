// Mechanism-specialised thread-per-cell integrator, generated at run time.
//
// For a mechanism with N = nsp + 1 <= 16 unknowns the library writes CUDA
// source in which every species index, stoichiometric coefficient, reaction
// order, rate parameter, efficiency and NASA-7 coefficient is a literal
// (hexadecimal floating point, so the values are exact), the reaction loop,
// the Jacobian scatter, the LU factorisation and the triangular solves are
// unrolled, and the Jacobian / LU lives in shared memory at constant offsets.
// NVRTC compiles it for sm_100a and the driver loads the cubin; the state
// machine around it (t1_body.cuh) is the one the precompiled kernel uses.
//
// The generated arithmetic is the precompiled thread-per-cell kernel's
// (integrator_t1.cuh, which restates chemistrySource::jacobian,
// chemistrySource.cpp:967-1021, and reactionTypes.cpp q / Kc / DqDci / DqDT),
// with two changes of evaluation order that stay far inside the integrator's
// tolerance: the LU factorisation is right-looking (the same pivots and
// factors as LUDecomposeDPivoting, SquareMatrix.hpp:185-237, summed in a
// different order) and multiplies by the pivot's reciprocal.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hurchem_b200.h"
#include "jit.h"
#include "jit_headers.inc"

namespace hc {

namespace {

// ------------------------------------------------------------------ literals
std::string lit(double v) {
    char buf[64];
    if (v == 0.0) return std::signbit(v) ? "(-0.0)" : "0.0";
    std::snprintf(buf, sizeof(buf), "%a", v);
    return std::string("(") + buf + ")";
}

std::string pow_lit(const std::string &x, double y) {
    if (y == 1.0) return x;
    if (y == 2.0) return "(" + x + " * " + x + ")";
    if (y == 0.0) return "1.0";
    if (y == -1.0) return "(1.0 / " + x + ")";
    return "pow(" + x + ", " + lit(y) + ")";
}

std::string Jx(int N, int i, int j) { return "J[" + std::to_string((i * N + j)) + " * B]"; }

}  // namespace

// ------------------------------------------------------------------ generator
std::string jit_t1_source(const HostMech &h, int block) {
    const int nsp = h.nsp, N = nsp + 1, TI = N - 1, S = HC_MAX_SIDE;
    std::ostringstream o;
    o << "#include \"t1_body.cuh\"\n"
      << "namespace hc {\n"
      << "struct JitCell {\n"
      << "  static constexpr int N = " << N << ", B = " << block << ";\n"
      << "  static constexpr bool kAssemblesA = false;\n"
      << "  int nsp = " << nsp << ";\n"
      << "  double *J;\n"
      << "  double f_[N];\n"
      << "  int piv_[N];\n"
      << "  __device__ JitCell(double *smem, int tid) : J(smem + tid) {}\n"
      << "  __device__ __forceinline__ double F(int i) const { return f_[i]; }\n"
      << "  __device__ __forceinline__ double W(int i) const {\n"
      << "    constexpr double w[" << nsp << "] = {";
    for (int i = 0; i < nsp; ++i) o << (i ? ", " : "") << lit(h.W[i]);
    o << "};\n    return w[i];\n  }\n";

    // species thermo: molar G0, dG0/dT (first pass) and cp, h, dcp (second pass)
    auto thermo = [&](int i, bool gibbs) {
        const double tl = h.Trange[3 * i], tc = h.Trange[3 * i + 1], th = h.Trange[3 * i + 2];
        const double *lo = &h.nasa[14 * i], *hi = &h.nasa[14 * i + 7];
        o << "    {\n      const bool lo = T < " << lit(tc) << ";\n";
        for (int k = 0; k < 7; ++k)
            o << "      const double a" << k << " = lo ? " << lit(lo[k]) << " : " << lit(hi[k]) << ";\n";
        o << "      const bool out = (T < " << lit(tl) << " || T > " << lit(th) << ");\n"
          << "      const double T0 = out ? hmin(hmax(T, " << lit(tl) << "), " << lit(th) << ") : T;\n"
          << "      const double cp0 = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);\n";
        if (gibbs) {
            o << "      const double lT = (T > kTiny) ? logT : log(kTiny);\n"
              << "      const double s0 = ((((a4 / 4.0 * T + a3 / 3.0) * T + a2 / 2.0) * T + a1) * T + a0 * lT + a6);\n"
              << "      const double g0 = (((((-a4 / 20.0 * T - a3 / 12.0) * T - a2 / 6.0) * T - a1 / 2.0) * T + a0 * (1 - lT) - a6) * T + a5);\n"
              << "      const double ds0 = (a0 / hmax(T, kTiny) + a1 + (a2 + (a3 + a4 * T) * T) * T);\n"
              << "      G0_" << i << " = g0 * " << lit(h.W[i]) << ";\n"
              << "      DG0_" << i << " = (cp0 - (s0 + T * ds0)) * " << lit(h.W[i]) << ";\n";
        } else {
            o << "      double h0 = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;\n"
              << "      if (out) h0 += cp0 * (T - T0);\n"
              << "      const double dcp = (a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T)));\n"
              << "      cp_" << i << " = cp0 * " << lit(h.W[i]) << ";\n"
              << "      h_" << i << " = h0 * " << lit(h.W[i]) << ";\n"
              << "      dcp_" << i << " = dcp * " << lit(h.W[i]) << ";\n";
        }
        o << "    }\n";
    };

    o << "  __device__ __forceinline__ void evaluate(const double (&y)[N], bool jac) {\n"
      << "    const double T = y[" << TI << "];\n"
      << "    const double logT = log(T);\n"
      << "    const double Tm = hmax(T, kTiny);\n"
      << "    const double invT = 1.0 / Tm;\n";
    for (int i = 0; i < nsp; ++i) o << "    const double c_" << i << " = hmax(y[" << i << "], 0.0);\n";
    for (int i = 0; i < N; ++i) o << "    double f" << i << " = 0.0;\n";
    o << "    if (jac) {\n#pragma unroll\n      for (int k = 0; k < N * N; ++k) J[k * B] = 0.0;\n    }\n";
    for (int i = 0; i < nsp; ++i) o << "    double G0_" << i << ", DG0_" << i << ";\n";
    for (int i = 0; i < nsp; ++i) thermo(i, true);

    for (int r = 0; r < h.nrc; ++r) {
        const int type = h.rate_type[r];
        const double A = h.arr[3 * r], b = h.arr[3 * r + 1], Ta = h.arr[3 * r + 2];
        const int nf = h.nf[r], nb = h.nb[r];
        const int *fi = &h.fidx[S * r], *bi = &h.bidx[S * r];
        const double *fo = &h.ford[S * r], *bo = &h.bord[S * r];
        const double *fnu = &h.fnu[S * r], *bnu = &h.bnu[S * r];
        const double *e = &h.eff[(size_t)r * nsp];
        auto arrk = [&](double AA, double bb, double TT) {
            std::string ex = "0.0";
            if (std::fabs(bb) > 1e-300) ex = lit(bb) + " * logT";
            if (std::fabs(TT) > 1e-300) ex = "(" + ex + ") - " + lit(TT) + " / T";
            return lit(AA) + " * exp(" + ex + ")";
        };
        o << "    { // reaction " << r << "\n";
        if (type != 0) {
            o << "      double M = 0.0;\n";
            for (int i = 0; i < nsp; ++i)
                if (e[i] != 0.0) o << "      M += " << lit(e[i]) << " * c_" << i << ";\n";
        }
        o << "      double kf, k0 = 0.0, kinf = 0.0, Pr = 0.0, F = 1.0, lf = 0.0;\n";
        const double A0 = h.arr0[3 * r], b0 = h.arr0[3 * r + 1], Ta0 = h.arr0[3 * r + 2];
        const double *tr = &h.troe[4 * r];
        if (type == 0) {
            o << "      kf = " << arrk(A, b, Ta) << ";\n";
        } else if (type == 1) {
            o << "      kf = M * (" << arrk(A, b, Ta) << ");\n";
        } else {
            o << "      k0 = " << arrk(A0, b0, Ta0) << ";\n"
              << "      kinf = " << arrk(A, b, Ta) << ";\n"
              << "      Pr = k0 / notZeroD(kinf) * M;\n";
            if (type != 2)
                o << "      lf = troe_logfcent_p(" << lit(tr[0]) << ", " << lit(tr[1]) << ", "
                  << lit(tr[2]) << ", " << lit(tr[3]) << ", " << (type == 4 ? "true" : "false")
                  << ", T);\n";
            o << "      F = fall_F(" << type << ", lf, Pr);\n"
              << "      kf = kinf * (Pr / (1.0 + Pr)) * F;\n";
        }
        o << "      double kr = 0.0, Kc = 0.0, DKcDT = 0.0;\n";
        if (h.reversible[r]) {
            // equilibrium constant (mech.cuh equilibrium(), reactionTypes.cpp:178-241)
            o << "      {\n        double kp = 0.0, dk = 0.0;\n";
            for (int k = 0; k < nf; ++k)
                o << "        kp -= G0_" << fi[k] << " * " << lit(fnu[k]) << ";\n"
                  << "        dk -= (DG0_" << fi[k] << " - G0_" << fi[k] << " / Tm) * " << lit(fnu[k]) << ";\n";
            for (int k = 0; k < nb; ++k)
                o << "        kp += G0_" << bi[k] << " * " << lit(bnu[k]) << ";\n"
                  << "        dk += (DG0_" << bi[k] << " - G0_" << bi[k] << " / Tm) * " << lit(bnu[k]) << ";\n";
            o << "        kp /= (Tm * kRu);\n"
              << "        double Kp = exp(-kp);\n"
              << "        if (!finite(Kp)) Kp = kRootVeryLarge;\n"
              << "        dk /= (Tm * kRu);\n"
              << "        double DKp = Kp * dk;\n"
              << "        if (!finite(DKp)) DKp = kVeryLarge;\n";
            const double s = h.sum_stoi[r];
            if (std::fabs(s) < 1e-300) {
                o << "        Kc = Kp;\n        DKcDT = DKp;\n";
            } else {
                o << "        const double fs = " << pow_lit("(kPatm / (kRu * T))", s) << ";\n"
                  << "        Kc = hmin(Kp * fs, kVeryLarge);\n"
                  << "        double v = (DKp + Kp * " << lit(-s) << " / T) * fs;\n"
                  << "        if (!finite(v)) v = kVeryLarge;\n"
                  << "        DKcDT = v;\n";
            }
            o << "      }\n      kr = (fabs(Kc) > kVeryTiny) ? kf / Kc : 0.0;\n";
        }
        o << "      double qf = kf, qr = kr;\n";
        for (int k = 0; k < S; ++k) {
            if (k < nf) o << "      const double pf" << k << " = " << pow_lit("c_" + std::to_string(fi[k]), fo[k]) << ";\n      qf *= pf" << k << ";\n";
            if (k < nb) o << "      const double pb" << k << " = " << pow_lit("c_" + std::to_string(bi[k]), bo[k]) << ";\n      qr *= pb" << k << ";\n";
        }
        o << "      const double q = qf - qr;\n";
        for (int k = 0; k < nf; ++k) o << "      f" << fi[k] << " -= " << lit(fnu[k]) << " * q;\n";
        for (int k = 0; k < nb; ++k) o << "      f" << bi[k] << " += " << lit(bnu[k]) << " * q;\n";
        o << "      if (jac) {\n";
        // DqDci, forward then reverse (reactionTypes.cpp:354-445)
        for (int side = 0; side < 2; ++side) {
            const int n = side ? nb : nf;
            const int *idx = side ? bi : fi;
            const double *ord = side ? bo : fo;
            for (int k = 0; k < n; ++k) {
                o << "        {\n          double d = " << (side ? "kr" : "kf") << ";\n";
                for (int j = 0; j < n; ++j) {
                    const std::string cj = "c_" + std::to_string(idx[j]);
                    if (j == k) {
                        if (ord[j] == 1.0) continue;
                        if (ord[j] < 1.0)
                            o << "          d *= (" << cj << " > kTiny) ? " << lit(ord[j]) << " * "
                              << pow_lit(cj, ord[j] - 1.0) << " : 0.0;\n";
                        else
                            o << "          d *= " << lit(ord[j]) << " * "
                              << pow_lit("hmax(" + cj + ", 0.0)", ord[j] - 1.0) << ";\n";
                    } else {
                        o << "          d *= " << (side ? "pb" : "pf") << j << ";\n";
                    }
                }
                const int col = idx[k];
                if (!side) {
                    for (int j = 0; j < nf; ++j) o << "          " << Jx(N, fi[j], col) << " -= " << lit(fnu[j]) << " * d;\n";
                    for (int j = 0; j < nb; ++j) o << "          " << Jx(N, bi[j], col) << " += " << lit(bnu[j]) << " * d;\n";
                } else {
                    for (int j = 0; j < nf; ++j) o << "          " << Jx(N, fi[j], col) << " += " << lit(fnu[j]) << " * d;\n";
                    for (int j = 0; j < nb; ++j) o << "          " << Jx(N, bi[j], col) << " -= " << lit(bnu[j]) << " * d;\n";
                }
                o << "        }\n";
            }
        }
        o << "        double dgdT = 0.0;\n";
        if (type == 1) {
            o << "        const double Mm = hmax(M, kTiny);\n";
            for (int i = 0; i < nsp; ++i) {
                o << "        { const double g = " << lit(e[i]) << " / Mm;\n          if (finite(g)) {\n";
                for (int j = 0; j < nf; ++j) o << "            " << Jx(N, fi[j], i) << " -= " << lit(fnu[j]) << " * g * q;\n";
                for (int j = 0; j < nb; ++j) o << "            " << Jx(N, bi[j], i) << " += " << lit(bnu[j]) << " * g * q;\n";
                o << "          }\n        }\n";
            }
        } else if (type >= 2) {
            o << "        if (M > kTiny) {\n"
              << "          const double Pr2 = k0 * M / notZeroD(kinf);\n"
              << "          const double F2 = fall_F(" << type << ", lf, Pr2);\n"
              << "          const double fabc = troe_dfdci_factor(" << type << ", lf, Pr2, F2);\n";
            for (int i = 0; i < nsp; ++i) {
                o << "          { const double dPrdci = " << lit(e[i]) << " * k0 / notZeroD(kinf);\n"
                  << "            const double dFdci = fabc * (1.0 / (Pr2)*dPrdci);\n"
                  << "            const double g = (dPrdci / (Pr2 * (1 + Pr2)) + dFdci / F2);\n"
                  << "            if (finite(g)) {\n";
                for (int j = 0; j < nf; ++j) o << "              " << Jx(N, fi[j], i) << " -= " << lit(fnu[j]) << " * g * q;\n";
                for (int j = 0; j < nb; ++j) o << "              " << Jx(N, bi[j], i) << " += " << lit(bnu[j]) << " * g * q;\n";
                o << "            }\n          }\n";
            }
            o << "          const double dPrdT = Pr2 * ((k0 * invT * (" << lit(b0) << " + " << lit(Ta0)
              << " * invT)) / notZeroD(k0) - (kinf * invT * (" << lit(b) << " + " << lit(Ta)
              << " * invT)) / notZeroD(kinf));\n"
              << "          const double dFdT = troe_dfdt_p(" << type << ", " << lit(tr[0]) << ", "
              << lit(tr[1]) << ", " << lit(tr[2]) << ", " << lit(tr[3]) << ", T, Pr2, F2, dPrdT);\n"
              << "          dgdT = q * (dPrdT / (Pr2 * (1 + Pr2)) + dFdT / F2);\n"
              << "        }\n";
        }
        // DqDT (reactionTypes.cpp:843-876)
        if (type <= 1)
            o << "        double dkfdT = kf * invT * (" << lit(b) << " + " << lit(Ta) << " * invT);\n";
        else
            o << "        double dkfdT = (Pr / (1.0 + Pr)) * F * (kinf * invT * (" << lit(b) << " + "
              << lit(Ta) << " * invT));\n";
        if (h.reversible[r])
            o << "        double dkrdT = (dkfdT - kr * DKcDT) / hmax(Kc, kVeryTiny);\n";
        else
            o << "        double dkrdT = 0.0;\n";
        for (int k = 0; k < S; ++k) {
            if (k < nf) o << "        dkfdT *= pf" << k << ";\n";
            if (k < nb) o << "        dkrdT *= pb" << k << ";\n";
        }
        o << "        double dqjdT = dkfdT - dkrdT;\n"
          << "        if (!finite(dqjdT)) dqjdT = 0;\n"
          << "        if (!finite(dgdT)) dgdT = 0;\n";
        for (int k = 0; k < nf; ++k) o << "        " << Jx(N, fi[k], TI) << " -= " << lit(fnu[k]) << " * (dqjdT + dgdT);\n";
        for (int k = 0; k < nb; ++k) o << "        " << Jx(N, bi[k], TI) << " += " << lit(bnu[k]) << " * (dqjdT + dgdT);\n";
        o << "      }\n    }\n";
    }

    // temperature equation of the constant-pressure reactor
    for (int i = 0; i < nsp; ++i) o << "    double cp_" << i << ", h_" << i << ", dcp_" << i << ";\n";
    for (int i = 0; i < nsp; ++i) thermo(i, false);
    o << "    double cCp = 0.0, DTdt = 0.0, dcCpdT = 0.0;\n";
    for (int i = 0; i < nsp; ++i)
        o << "    cCp += y[" << i << "] * cp_" << i << ";\n    dcCpdT += y[" << i << "] * dcp_" << i
          << ";\n    DTdt += f" << i << " * h_" << i << ";\n";
    o << "    DTdt /= cCp;\n    f" << TI << " = -DTdt;\n";
    for (int i = 0; i < N; ++i) o << "    f_[" << i << "] = f" << i << ";\n";
    o << "    if (!jac) return;\n";
    for (int i = 0; i < nsp; ++i) {
        o << "    { double d = " << Jx(N, TI, i) << ";\n";
        for (int j = 0; j < nsp; ++j) o << "      d -= " << Jx(N, j, i) << " * h_" << j << ";\n";
        o << "      d += cp_" << i << " * DTdt;\n      d /= cCp;\n      " << Jx(N, TI, i) << " = d; }\n";
    }
    o << "    { double dd = 0.0;\n";
    for (int i = 0; i < nsp; ++i) o << "      dd -= (cp_" << i << " * f" << i << " + h_" << i << " * " << Jx(N, i, TI) << ");\n";
    o << "      dd += dcCpdT * DTdt;\n      dd /= cCp;\n      " << Jx(N, TI, TI) << " = dd; }\n";
    o << "  }\n";

    // I - dt J and its LU factorisation with partial pivoting
    o << "  __device__ __forceinline__ void factor(double dt) {\n";
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            o << "    " << Jx(N, i, j) << " = -dt * " << Jx(N, i, j) << (i == j ? " + 1.0" : "") << ";\n";
    for (int k = 0; k < N; ++k) {
        o << "    { double amax = fabs(" << Jx(N, k, k) << "); int p = " << k << ";\n";
        for (int i = k + 1; i < N; ++i)
            o << "      { const double v = fabs(" << Jx(N, i, k) << "); if (v > amax) { amax = v; p = " << i << "; } }\n";
        o << "      piv_[" << k << "] = p;\n";
        if (k + 1 < N) {
            o << "      if (p != " << k << ") {\n        double *rp = J + p * (N * B);\n";
            for (int j = 0; j < N; ++j)
                o << "        { const double t = " << Jx(N, k, j) << "; " << Jx(N, k, j) << " = rp[" << j
                  << " * B]; rp[" << j << " * B] = t; }\n";
            o << "      }\n";
        }
        o << "      const double inv = 1.0 / " << Jx(N, k, k) << ";\n";
        for (int j = k + 1; j < N; ++j) o << "      const double u" << j << " = " << Jx(N, k, j) << ";\n";
        for (int i = k + 1; i < N; ++i) {
            o << "      { const double l = " << Jx(N, i, k) << " * inv; " << Jx(N, i, k) << " = l;\n";
            for (int j = k + 1; j < N; ++j) o << "        " << Jx(N, i, j) << " -= l * u" << j << ";\n";
            o << "      }\n";
        }
        o << "    }\n";
    }
    o << "  }\n";

    // LUBacksubstituteDPivoting (LUDecompose.hpp:68-100)
    o << "  __device__ __forceinline__ void solve(double (&b)[N]) {\n";
    for (int k = 0; k + 1 < N; ++k) {
        o << "    { const int p = piv_[" << k << "];\n";
        for (int i = k + 1; i < N; ++i)
            o << "      if (p == " << i << ") { const double t = b[" << k << "]; b[" << k << "] = b[" << i
              << "]; b[" << i << "] = t; }\n";
        o << "    }\n";
    }
    for (int i = 1; i < N; ++i) {
        o << "    { double s = 0.0;\n";
        for (int t = 0; t < i; ++t) o << "      s += " << Jx(N, i, t) << " * b[" << t << "];\n";
        o << "      b[" << i << "] -= s; }\n";
    }
    for (int i = N - 1; i >= 0; --i) {
        o << "    { double s = 0.0;\n";
        for (int t = i + 1; t < N; ++t) o << "      s += " << Jx(N, i, t) << " * b[" << t << "];\n";
        o << "      b[" << i << "] = (b[" << i << "] - s) / " << Jx(N, i, i) << "; }\n";
    }
    o << "  }\n};\n}  // namespace hc\n\n";

    o << "extern \"C\" __global__ void __launch_bounds__(" << block << ")\n"
      << "hc_jit_t1(const __grid_constant__ hc::IntegratorParams P, "
         "const __grid_constant__ hc::CellIO io, double *ylast) {\n"
      << "  extern __shared__ double smem_jit[];\n"
      << "  hc::JitCell cell(smem_jit, threadIdx.x);\n"
      << "  hc::t1_run<" << N << ">(cell, P, io, ylast);\n"
      << "}\n";
    return o.str();
}

}  // namespace hc

// ------------------------------------------------------------------ NVRTC + driver
namespace hc {

namespace {

typedef int nvrtcResult_t;
typedef struct _nvrtcProgram *nvrtcProgram_t;
struct Nvrtc {
    void *lib = nullptr;
    nvrtcResult_t (*create)(nvrtcProgram_t *, const char *, const char *, int, const char *const *,
                            const char *const *) = nullptr;
    nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char *const *) = nullptr;
    nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t *) = nullptr;
    nvrtcResult_t (*log)(nvrtcProgram_t, char *) = nullptr;
    nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t *) = nullptr;
    nvrtcResult_t (*cubin)(nvrtcProgram_t, char *) = nullptr;
    nvrtcResult_t (*destroy)(nvrtcProgram_t *) = nullptr;
    bool ok = false;
};

const Nvrtc &nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12",
                               "/usr/local/cuda/lib64/libnvrtc.so"};
        for (const char *nm : names) {
            n.lib = dlopen(nm, RTLD_NOW | RTLD_LOCAL);
            if (n.lib) break;
        }
        if (!n.lib) return;
        auto sym = [&](const char *s) { return dlsym(n.lib, s); };
        n.create = reinterpret_cast<decltype(n.create)>(sym("nvrtcCreateProgram"));
        n.compile = reinterpret_cast<decltype(n.compile)>(sym("nvrtcCompileProgram"));
        n.log_size = reinterpret_cast<decltype(n.log_size)>(sym("nvrtcGetProgramLogSize"));
        n.log = reinterpret_cast<decltype(n.log)>(sym("nvrtcGetProgramLog"));
        n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(sym("nvrtcGetCUBINSize"));
        n.cubin = reinterpret_cast<decltype(n.cubin)>(sym("nvrtcGetCUBIN"));
        n.destroy = reinterpret_cast<decltype(n.destroy)>(sym("nvrtcDestroyProgram"));
        n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    });
    return n;
}

struct Driver {
    PFN_cuModuleLoadData_v2000 load = nullptr;
    PFN_cuModuleGetFunction_v2000 get = nullptr;
    PFN_cuLaunchKernel_v4000 launch = nullptr;
    PFN_cuFuncSetAttribute_v9000 set_attr = nullptr;
    PFN_cuOccupancyMaxActiveBlocksPerMultiprocessor_v6050 occ = nullptr;
    bool ok = false;
};

const Driver &driver() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char *name, void **p) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPoint(name, p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess;
        };
        bool ok = get("cuModuleLoadData", reinterpret_cast<void **>(&d.load));
        ok = ok && get("cuModuleGetFunction", reinterpret_cast<void **>(&d.get));
        ok = ok && get("cuLaunchKernel", reinterpret_cast<void **>(&d.launch));
        ok = ok && get("cuFuncSetAttribute", reinterpret_cast<void **>(&d.set_attr));
        ok = ok && get("cuOccupancyMaxActiveBlocksPerMultiprocessor",
                       reinterpret_cast<void **>(&d.occ));
        d.ok = ok;
    });
    return d;
}

struct CacheEntry {
    void *module;
    void *func;
};
std::mutex g_cache_mu;
std::map<std::string, CacheEntry> g_cache;   // source text + device -> loaded module

}  // namespace

// NVRTC: generated source -> sm_100a cubin
int jit_compile(const std::string &src, std::vector<char> &cubin, std::string &err) {
    const Nvrtc &nv = nvrtc();
    if (!nv.ok) {
        err = "NVRTC (libnvrtc.so.12) not found";
        return HC_E_UNSUPPORTED;
    }
    nvrtcProgram_t prog = nullptr;
    if (nv.create(&prog, src.c_str(), "hc_jit.cu", kJitHeaderCount, kJitHeaders,
                  kJitHeaderNames) != 0) {
        err = "nvrtcCreateProgram failed";
        return HC_E_CUDA;
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device",
                          "-DHC_JIT=1"};
    const int crc = nv.compile(prog, 4, opts);
    if (crc != 0) {
        size_t ls = 0;
        nv.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) nv.log(prog, &log[0]);
        nv.destroy(&prog);
        err = "NVRTC compile failed: " + log.substr(0, 4000);
        return HC_E_CUDA;
    }
    size_t cs = 0;
    nv.cubin_size(prog, &cs);
    cubin.resize(cs);
    nv.cubin(prog, cubin.data());
    nv.destroy(&prog);
    return HC_OK;
}

namespace {

// compile (cached per device and source text) and load one generated kernel
int jit_build(const std::string &src, const char *fname, int N, int slots, int block, JitKernel *out,
              std::string &err) {
    const Driver &dr = driver();
    if (!dr.ok) {
        err = "CUDA driver entry points unavailable";
        return HC_E_CUDA;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const std::string key = std::to_string(dev) + "\n" + src;
    void *module = nullptr, *func = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            module = it->second.module;
            func = it->second.func;
        }
    }
    if (!func) {
        std::vector<char> cubin;
        const int crc = jit_compile(src, cubin, err);
        if (crc != HC_OK) return crc;
        CUmodule mod = nullptr;
        if (dr.load(&mod, cubin.data()) != CUDA_SUCCESS) {
            err = "cuModuleLoadData failed for the generated kernel";
            return HC_E_CUDA;
        }
        CUfunction f = nullptr;
        if (dr.get(&f, mod, fname) != CUDA_SUCCESS) {
            err = "cuModuleGetFunction failed for the generated kernel";
            return HC_E_CUDA;
        }
        module = mod;
        func = f;
        std::lock_guard<std::mutex> lk(g_cache_mu);
        g_cache[key] = CacheEntry{module, func};
    }
    const size_t smem = sizeof(double) * (size_t)slots * block;
    if (dr.set_attr(static_cast<CUfunction>(func), CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                    (int)smem) != CUDA_SUCCESS) {
        err = "cuFuncSetAttribute failed for the generated kernel";
        return HC_E_CUDA;
    }
    int per_sm = 0;
    if (dr.occ(&per_sm, static_cast<CUfunction>(func), block, smem) != CUDA_SUCCESS || per_sm < 1) {
        err = "generated kernel does not fit on an SM";
        return HC_E_UNSUPPORTED;
    }
    out->module = module;
    out->func = func;
    out->N = N;
    out->block = block;
    out->smem = smem;
    out->per_sm = per_sm;
    return HC_OK;
}

}  // namespace

int jit_build_t1(const HostMech &h, int block, JitKernel *out, std::string &err) {
    const int N = h.nsp + 1;
    if (N > 16) {
        err = "specialised thread-per-cell kernel is built for nsp + 1 <= 16";
        return HC_E_UNSUPPORTED;
    }
    return jit_build(jit_t1_source(h, block), "hc_jit_t1", N, N * N, block, out, err);
}

int jit_build_t3(const HostMech &h, int block, JitKernel *out, std::string &err) {
    const int N = h.nsp + 1;
    if (N > 16) {
        err = "direct-assembly thread-per-cell kernel is built for nsp + 1 <= 16";
        return HC_E_UNSUPPORTED;
    }
    return jit_build(jit_t3_source(h, block), "hc_jit_t3", N, t3_slots(h.nsp), block, out, err);
}

int jit_launch_t1(const JitKernel &k, int num_sms, const IntegratorParams &P, const CellIO &io,
                  double *ylast, cudaStream_t st, std::string &err) {
    const Driver &dr = driver();
    const int64_t blocks_needed = (io.nqueue + k.block - 1) / k.block;
    int64_t grid = (int64_t)k.per_sm * num_sms;
    if (blocks_needed < grid) grid = blocks_needed;
    if (grid <= 0) return HC_OK;
    IntegratorParams p = P;
    CellIO c = io;
    double *yl = ylast;
    void *args[] = {&p, &c, &yl};
    CUresult r = dr.launch(static_cast<CUfunction>(k.func), (unsigned)grid, 1, 1, (unsigned)k.block,
                           1, 1, (unsigned)k.smem, reinterpret_cast<CUstream>(st), args, nullptr);
    if (r != CUDA_SUCCESS) {
        err = "cuLaunchKernel failed for the generated kernel (" + std::to_string((int)r) + ")";
        return HC_E_CUDA;
    }
    return HC_OK;
}

}  // namespace hc
