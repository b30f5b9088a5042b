// C++ host program over include/hurchem_b200.hpp: reads a mechanism and a
// set of cells from a binary file, runs one flow step through
// hurchem::ChemistrySource::solveUpdate, the per-cell solve and
// calculateSourceTerms, and writes the results. Used by tests/test_cpp_host.py.
//
// input:  int32 nsp, nrc; int64 ncells; then float64/int32 arrays in the
//         order of hc_mech_desc (W, Trange, nasa, rate_type, reversible, arr,
//         arr0, troe, eff, nf, nb, fidx, bidx, fnu, bnu, ford, bord, geom,
//         eps_k, sigma), then T, p, rho, Y[nsp][n], dt, and float64 atol, rtol
// output: T, rho, Y (after solveUpdate), Ri (source terms at the new state),
//         T of cell 0 integrated again by the per-cell solve
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hurchem_b200.hpp"

template <typename T>
static std::vector<T> rd(FILE *f, size_t n) {
    std::vector<T> v(n);
    if (n && fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "short read\n");
        exit(2);
    }
    return v;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[2];
    int64_t n;
    if (fread(hdr, 4, 2, f) != 2 || fread(&n, 8, 1, f) != 1) return 2;
    const size_t nsp = hdr[0], nrc = hdr[1], S = HC_MAX_SIDE;
    auto W = rd<double>(f, nsp), Tr = rd<double>(f, 3 * nsp), nasa = rd<double>(f, 14 * nsp);
    auto rt = rd<int32_t>(f, nrc), rev = rd<int32_t>(f, nrc);
    auto arr = rd<double>(f, 3 * nrc), arr0 = rd<double>(f, 3 * nrc), troe = rd<double>(f, 4 * nrc);
    auto eff = rd<double>(f, nrc * nsp);
    auto nf = rd<int32_t>(f, nrc), nb = rd<int32_t>(f, nrc);
    auto fidx = rd<int32_t>(f, S * nrc), bidx = rd<int32_t>(f, S * nrc);
    auto fnu = rd<double>(f, S * nrc), bnu = rd<double>(f, S * nrc);
    auto ford = rd<double>(f, S * nrc), bord = rd<double>(f, S * nrc);
    auto geom = rd<int32_t>(f, nsp);
    auto epsk = rd<double>(f, nsp), sigma = rd<double>(f, nsp);
    auto T = rd<double>(f, n), p = rd<double>(f, n), rho = rd<double>(f, n);
    auto Y = rd<double>(f, nsp * n), dt = rd<double>(f, n);
    auto tol = rd<double>(f, 2);
    fclose(f);

    hc_mech_desc d{};
    d.nsp = (int32_t)nsp;
    d.nrc = (int32_t)nrc;
    d.W = W.data(); d.Trange = Tr.data(); d.nasa = nasa.data();
    d.rate_type = rt.data(); d.reversible = rev.data();
    d.arr = arr.data(); d.arr0 = arr0.data(); d.troe = troe.data(); d.eff = eff.data();
    d.nf = nf.data(); d.nb = nb.data(); d.fidx = fidx.data(); d.bidx = bidx.data();
    d.fnu = fnu.data(); d.bnu = bnu.data(); d.ford = ford.data(); d.bord = bord.data();
    d.geom = geom.data(); d.eps_k = epsk.data(); d.sigma = sigma.data();

    try {
        hurchem::Mechanism mech(d);
        hc_opts o = hurchem::defaultOptions();
        o.atol = tol[0];
        o.rtol = tol[1];
        // per-cell solve of cell 0 on copies, before the fields change
        double T0 = T[0], rho0 = rho[0];
        std::vector<double> y0(nsp);
        for (size_t i = 0; i < nsp; ++i) y0[i] = Y[i * n];
        std::vector<double> Tin(T), rin(rho), Yin(Y);
        hurchem::ChemistrySource cs(mech, n, T.data(), p.data(), rho.data(), Y.data(), o);
        {
            hurchem::ChemistrySource one(mech, 1, &T0, p.data(), &rho0, y0.data(), o);
            one.solve(dt[0], dt[0], p[0], T0, rho0, y0.data());
        }
        cs.solveUpdate(dt.data(), 1.0);
        cs.calculateSourceTerms();
        FILE *g = fopen(argv[2], "wb");
        if (!g) return 2;
        fwrite(T.data(), 8, n, g);
        fwrite(rho.data(), 8, n, g);
        fwrite(Y.data(), 8, nsp * n, g);
        for (size_t i = 0; i < nsp; ++i) fwrite(cs.Ri((int)i), 8, n, g);
        fwrite(&T0, 8, 1, g);
        fclose(g);
        printf("ok newton=%lld\n", (long long)cs.counters().n_newton);
    } catch (const hurchem::Error &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
