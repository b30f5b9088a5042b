"""Generate the golden fixtures of tests/golden/ with the REFERENCE itself.

Runs OpenHurricane's own CPU chemistry path (compiled from the reference
sources by oracle/Makefile.ref into oracle/_ref/hurchem_ref) on seeded inputs
and stores inputs and outputs:

  small_ref.npz : 9-species / 21-reaction mechanism, 48 cells drawn like the
                  small workload (T 1000-2500 K, p 1-5 atm, Y ~ Dirichlet(0.5)),
                  dt = 1e-6 s, reference default solver options; integrated
                  T, Y, rho, concentrations and warm-start sub-steps; plus KAT
                  states: DyDt, analytic Jacobian, species thermo, kf/Kc/kr;
                  plus mixture properties (h_i, cp, mu, kappa, D_i) of 32 cells.
  large_ref.npz : 53-species / 325-reaction mechanism, 2 cells drawn like the
                  large workload (T 800-2800 K, p 0.5-10 atm, Dirichlet(0.3)),
                  dt = 1e-7 s; plus KAT states and properties of 16 cells.
  cv_ref.npz    : the constant-volume reactor (chemSolvers type constVolume) on
                  48 cells of the small mechanism (dt = 1e-7 s) and 48 of the
                  extended one (dt = 3e-8 s; heat release at constant volume
                  makes longer steps of these cells far stiffer): integrated T,
                  Y, c, sub-steps and the reference's updated pressure; and
                  thermoList::TEa_rho (temperature from internal energy at
                  constant density) on 16 cells of each.
  ext_ref.npz   : 9-species / 21-reaction mechanism with the rate forms beyond
                  the small one (SRI, REV, FORD / RORD, REACTIONS-line and
                  per-reaction units, PLOG; synth.extended_mechanism), 48 cells
                  drawn like the small workload, dt = 1e-7 s (at 1e-6 s some
                  of its cells answer one-ulp input changes with 1e-6 changes
                  of T); plus KAT states,
                  point-implicit source terms and properties of 16 cells.
  batched_ref.npz: the benchmarked configuration: 256 cells strided from
                  the 1,048,576 cells of the batched workload (seed 2002; 20 %
                  ignition, 80 % near equilibrium), dt = 1e-5 s, the
                  benchmark's solver options (atol 1e-11, rtol 1e-4, maxstep
                  10000); integration outputs only.
  large32_ref.npz: 32 cells of the 53-species mechanism drawn like the large
                  workload, dt = 1e-6 s, atol 1e-15; integration outputs only.
  fitted_ref.npz: the small mechanism with Janev (JAN), power-series (FIT1),
                  reverse Landau-Teller (LT + REV + RLT) and collision-
                  efficiency (COLLEFF) reactions (synth.fitted_rates_mechanism),
                  96 cells, dt = 1e-7 s, run with a viscous flow model (the
                  reference reads collision diameters only then); plus KAT
                  states, point-implicit source terms and properties of 16 cells.

The mechanism files are regenerated from their seeds by
openhurricane_b200.synth at test time; a SHA-256 of the generated text files
is stored so that a change of the generator is detected.

    python tests/golden/make_golden.py [small] [large] [ext] [cv] [fitted] [batched] [large32]
    (default: all;
    needs oracle/_ref/hurchem_ref)
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from openhurricane_b200 import synth  # noqa: E402
from openhurricane_b200.mechanism import compile_mechanism  # noqa: E402
from oracle import props_oracle, refrun  # noqa: E402


def files_sha(paths):
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def kat_states(nsp, n, seed):
    rng = np.random.default_rng(seed)
    T = rng.uniform(800, 3000, n)
    p = rng.uniform(1, 5, n) * 101325.0
    c = rng.dirichlet(np.full(nsp, 0.5), n).T.copy() * rng.uniform(0.001, 0.1, n)
    c[0, 0] = 0.0                  # an absent species
    c[1, min(1, n - 1)] = -1e-12   # a slightly negative one (clamped by the reference)
    return T, p, np.ascontiguousarray(c)


def make(name, mech, cells, dt, nkat, prop_cells, out, flow="EulerFlow"):
    work = tempfile.mkdtemp(prefix="golden_")
    files = synth.write_chemkin(mech, work)
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *files, {"atol": 1e-15, "flowModel": flow})
    W = mech.weights()
    rho = synth.mixture_density(W, cells)
    res = refrun.integrate(case, cells.T, cells.p, rho, dt, dt, cells.Y,
                           procs=os.cpu_count() or 1, workdir=work)
    T, p, c = kat_states(len(mech.species), nkat, seed=4242)
    k = refrun.kat(case, p, T, c, workdir=work)
    pcase = os.path.join(work, "case_props.cont")
    refrun.write_case(pcase, *files, {"flowModel": "laminarFlow"})
    prho = synth.mixture_density(W, prop_cells)
    pr = refrun.props(pcase, prop_cells.T, prop_cells.p, prho, prop_cells.Y, workdir=work)
    si = refrun.srcimp(case, prop_cells.T, prop_cells.p, prho, prop_cells.Y, workdir=work)
    # temperature from enthalpy: the cells' own mass enthalpy, started 300 K
    # away (and once from far outside the table range)
    ha = (pr["ha"] * prop_cells.Y).sum(axis=0)     # the reference's per-species ha_i
    T0 = prop_cells.T + np.where(np.arange(prop_cells.T.shape[0]) % 2 == 0, 300.0, -300.0)
    T0[0] = 20.0
    th = refrun.tha(case, ha, prop_cells.p, T0, prop_cells.Y, workdir=work)
    np.savez_compressed(
        out, sha=files_sha(files), seed=mech.seed, dt=dt,
        in_T=cells.T, in_p=cells.p, in_rho=rho, in_Y=cells.Y,
        out_T=res["T"], out_Y=res["Y"], out_rho=res["rho"], out_c=res["c"],
        out_subdt=res["subdt"], out_status=res["status"],
        kat_T=T, kat_p=p, kat_c=c, kat_dydt=k["dydt"], kat_J=k["J"],
        kat_thermo=np.stack([k[n] for n in ("cp0", "ha0", "s0", "g0", "G0", "DG0DT", "Dcp_pDT")],
                            axis=-1),
        kat_rates=np.stack([k["kf"], k["Kc"], k["kr"]], axis=-1),
        prop_T=prop_cells.T, prop_p=prop_cells.p, prop_Y=prop_cells.Y,
        prop_ha=pr["ha"], prop_cp=pr["cp"], prop_mu=pr["mu"], prop_kappa=pr["kappa"],
        prop_D=pr["D"], prop_rho=prho, srcimp_Ri=si["Ri"], srcimp_diag=si["diag"],
        tha_ha=ha, tha_T0=T0, tha_T=th["T"], tha_flag=th["iflag"])
    print(name, "written", out, "reference seconds", res["seconds"])


def make_cv(out):
    """Constant-volume integrations of the small and extended mechanisms."""
    res = {}
    for name, mech, dt, seed in (("small", synth.small_mechanism(), 1e-7, 113),
                                 ("ext", synth.extended_mechanism(), 3e-8, 115)):
        work = tempfile.mkdtemp(prefix="golden_cv_")
        files = synth.write_chemkin(mech, work)
        case = os.path.join(work, "case.cont")
        refrun.write_case(case, *files, {"atol": 1e-15, "reactor": "constVolume"})
        cells = synth.dirichlet_cells(len(mech.species), 48, seed=seed)
        rho = synth.mixture_density(mech.weights(), cells)
        r = refrun.integrate(case, cells.T, cells.p, rho, dt, dt, cells.Y, procs=os.cpu_count() or 1,
                             workdir=work)
        res.update({f"{name}_sha": files_sha(files), f"{name}_dt": dt, f"{name}_in_T": cells.T,
                    f"{name}_in_p": cells.p, f"{name}_in_rho": rho, f"{name}_in_Y": cells.Y,
                    f"{name}_out_T": r["T"], f"{name}_out_Y": r["Y"], f"{name}_out_c": r["c"],
                    f"{name}_out_subdt": r["subdt"], f"{name}_out_p": r["p"],
                    f"{name}_out_rho": r["rho"]})
        # temperature from internal energy at constant density (thermoList::TEa_rho):
        # 16 cells' own energy, started 300 K away (and once from 20 K)
        tc = synth.dirichlet_cells(len(mech.species), 16, seed=seed + 1)
        trho = synth.mixture_density(mech.weights(), tc)
        tables = compile_mechanism(*files)
        ea = props_oracle.mixture_ea(tables, tc.T, trho, tc.Y)
        T0 = tc.T + np.where(np.arange(16) % 2 == 0, 300.0, -300.0)
        T0[0] = 20.0
        te = refrun.tea(case, ea, trho, T0, tc.Y, workdir=work)
        res.update({f"{name}_tea_ea": ea, f"{name}_tea_rho": trho, f"{name}_tea_Y": tc.Y,
                    f"{name}_tea_T0": T0, f"{name}_tea_T": te["T"], f"{name}_tea_flag": te["iflag"]})
    np.savez_compressed(out, **res)
    print("cv written", out)


def make_integration(out, mech, T, p, rho, Y, dt, opts):
    """Integration outputs only, at the given solver options."""
    work = tempfile.mkdtemp(prefix="golden_int_")
    files = synth.write_chemkin(mech, work)
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *files, dict(opts))
    res = refrun.integrate(case, T, p, rho, dt, dt, Y, procs=os.cpu_count() or 1, workdir=work)
    np.savez_compressed(out, sha=files_sha(files), seed=mech.seed, dt=dt,
                        opts=np.array(sorted(opts.items()), dtype=object).astype(str),
                        in_T=T, in_p=p, in_rho=rho, in_Y=Y,
                        out_T=res["T"], out_Y=res["Y"], out_rho=res["rho"], out_c=res["c"],
                        out_subdt=res["subdt"], out_status=res["status"])
    print(os.path.basename(out), "written, reference seconds", res["seconds"])


def main():
    if not refrun.available():
        raise SystemExit("oracle/_ref/hurchem_ref is missing: make -f oracle/Makefile.ref")
    which = set(sys.argv[1:]) or {"small", "large", "ext", "cv", "fitted", "batched", "large32"}
    if "batched" in which:
        # the benchmarked configuration: 256 cells strided from the 1,048,576
        # batched cells (seed 2002), dt = 1e-5 s, the benchmark's solver options
        from openhurricane_b200 import workloads
        wl = workloads.make_batched(1048576)
        idx = np.linspace(0, wl.n - 1, 256).astype(np.int64)
        make_integration(os.path.join(HERE, "batched_ref.npz"), synth.small_mechanism(),
                         wl.T[idx], wl.p[idx], wl.rho[idx], np.ascontiguousarray(wl.Y[:, idx]),
                         wl.dt, workloads.SOLVER_OPTS)
    if "large32" in which:
        # 32 cells of the 53-species mechanism drawn like the large workload, dt = 1e-6 s
        large = synth.large_mechanism()
        c = synth.dirichlet_cells(53, 32, seed=117, T_range=(800, 2800), p_atm_range=(0.5, 10),
                                  alpha=0.3)
        rho = synth.mixture_density(large.weights(), c)
        make_integration(os.path.join(HERE, "large32_ref.npz"), large, c.T, c.p, rho, c.Y, 1e-6,
                         {"atol": 1e-15})
    if "small" in which:
        small = synth.small_mechanism()
        make("small", small, synth.dirichlet_cells(9, 48, seed=101), 1e-6, 8,
             synth.dirichlet_cells(9, 32, seed=105), os.path.join(HERE, "small_ref.npz"))
    if "large" in which:
        large = synth.large_mechanism()
        make("large", large, synth.dirichlet_cells(53, 2, seed=103, T_range=(800, 2800),
                                                   p_atm_range=(0.5, 10), alpha=0.3),
             1e-7, 3, synth.dirichlet_cells(53, 16, seed=107, T_range=(800, 2800),
                                             p_atm_range=(0.5, 10), alpha=0.3),
             os.path.join(HERE, "large_ref.npz"))
    if "ext" in which:
        ext = synth.extended_mechanism()
        make("ext", ext, synth.dirichlet_cells(9, 48, seed=109), 1e-7, 8,
             synth.dirichlet_cells(9, 16, seed=111), os.path.join(HERE, "ext_ref.npz"))
    if "cv" in which:
        make_cv(os.path.join(HERE, "cv_ref.npz"))
    if "fitted" in which:
        # a viscous flow model: the reference reads the collision diameters of
        # the COLLEFF reaction from the transport table only then
        make("fitted", synth.fitted_rates_mechanism(), synth.dirichlet_cells(9, 96, seed=23), 1e-7,
             8, synth.dirichlet_cells(9, 16, seed=115), os.path.join(HERE, "fitted_ref.npz"),
             flow="laminarFlow")


if __name__ == "__main__":
    main()
