// Host build of the device rate-law helpers (openhurricane_b200/csrc/rtc_base.cuh)
// for a CPU check of their arithmetic. Reads from stdin, printing 17
// significant digits:
//   "S a b c d e T Pr F DPrDT"  -> sri_F, sri_dfdt, sri_dfdci_factor
//   "P n p T  p_1 A_1 b_1 Ta_1 ... p_n A_n b_n Ta_n"  -> plog_k, plog_dkdt
//   "L A b Ta B C T"  -> lt_k, lt_dkdt
//   "J A b Ta b_0 .. b_8 T"  -> janev_k, janev_dkdt
//   "F A b b_0 .. b_3 T"  -> pseries_k, pseries_dkdt
//   "K A b Ta x_0 x_1 x_2 T"  -> collision_k, collision_dkdt
#include <cmath>
#include <cstdio>

using std::isinf;
using std::isnan;

#include "../../openhurricane_b200/csrc/rtc_base.cuh"

int main() {
    char kind[2];
    while (std::scanf("%1s", kind) == 1) {
        if (kind[0] == 'S') {
            double s[5], T, Pr, F, DPrDT;
            if (std::scanf("%lf %lf %lf %lf %lf %lf %lf %lf %lf", &s[0], &s[1], &s[2], &s[3], &s[4],
                           &T, &Pr, &F, &DPrDT) != 9)
                return 1;
            std::printf("%.17g %.17g %.17g\n", hc::sri_F(s, T, Pr),
                        hc::sri_dfdt(s, T, Pr, F, DPrDT), hc::sri_dfdci_factor(s, T, Pr, F));
        } else if (kind[0] == 'P') {
            int n = 0;
            double p, T, pp[16], pa[48];
            if (std::scanf("%d %lf %lf", &n, &p, &T) != 3 || n < 1 || n > 16) return 1;
            for (int i = 0; i < n; ++i)
                if (std::scanf("%lf %lf %lf %lf", &pp[i], &pa[3 * i], &pa[3 * i + 1],
                               &pa[3 * i + 2]) != 4)
                    return 1;
            const double k = hc::plog_k(pp, pa, n, p, T, std::log(T));
            std::printf("%.17g %.17g\n", k, hc::plog_dkdt(pp, pa, n, k, p, T, std::log(T)));
        } else if (kind[0] == 'L') {
            double A, b, Ta, B, C, T;
            if (std::scanf("%lf %lf %lf %lf %lf %lf", &A, &b, &Ta, &B, &C, &T) != 6) return 1;
            const double k = hc::lt_k(A, b, Ta, B, C, T, std::log(T));
            std::printf("%.17g %.17g\n", k, hc::lt_dkdt(k, b, Ta, B, C, T));
        } else if (kind[0] == 'K') {
            double A, b, Ta, x[3], T;
            if (std::scanf("%lf %lf %lf %lf %lf %lf %lf", &A, &b, &Ta, &x[0], &x[1], &x[2], &T) != 7)
                return 1;
            const double k = hc::collision_k(A, b, Ta, x, T, std::log(T));
            std::printf("%.17g %.17g\n", k, hc::collision_dkdt(k, b, Ta, x, T));
        } else if (kind[0] == 'J' || kind[0] == 'F') {
            const int nb = kind[0] == 'J' ? 9 : 4;
            double A, b, Ta = 0.0, bn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, T;
            if (std::scanf("%lf %lf", &A, &b) != 2) return 1;
            if (kind[0] == 'J' && std::scanf("%lf", &Ta) != 1) return 1;
            for (int i = 0; i < nb; ++i)
                if (std::scanf("%lf", &bn[i]) != 1) return 1;
            if (std::scanf("%lf", &T) != 1) return 1;
            const double lT = std::log(T);
            if (kind[0] == 'J') {
                const double k = hc::janev_k(A, b, Ta, bn, T, lT);
                std::printf("%.17g %.17g\n", k, hc::janev_dkdt(k, b, Ta, bn, T, lT));
            } else {
                const double k = hc::pseries_k(A, b, bn, T, lT);
                std::printf("%.17g %.17g\n", k, hc::pseries_dkdt(k, b, bn, T));
            }
        } else {
            return 1;
        }
    }
    return 0;
}
