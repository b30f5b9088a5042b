"""Parity helpers shared by the GPU tests: tolerance check of integrated
cells and the explanation of a cell outside the tolerance by a one-ulp input
perturbation of the oracle (the oracle is the reference bit for bit)."""
import numpy as np

T_RTOL = 1e-6
Y_RTOL = 1e-5
Y_FLOOR = 1e-12
MAX_FLIP_FRACTION = 0.05


def oracle(tables, T, p, rho, Y, dt, **opts):
    from oracle import port
    return port.integrate(port.MechDesc(tables), T, p, rho, Y, dt, opts=port.default_opts(**opts))


def bad_cells(g, ref):
    dT = np.abs(g["T"] - ref["T"]) / np.abs(ref["T"])
    dr = np.abs(g["rho"] - ref["rho"]) / np.abs(ref["rho"])
    dY = (np.abs(g["Y"] - ref["Y"]) - Y_RTOL * np.abs(ref["Y"]) - Y_FLOOR).max(axis=0)
    return np.where((dT > T_RTOL) | (dr > T_RTOL) | (dY > 0.0))[0]


def perturbations(T, Y, k):
    """Inputs one unit in the last place away: T up / down, all Y up / down,
    then seeded +-1 ulp patterns over the species and T."""
    ulp = np.finfo(np.float64).eps
    if k == 0:
        return T * (1 + ulp), Y
    if k == 1:
        return T * (1 - ulp / 2), Y
    if k == 2:
        return T, Y * (1 + ulp)
    if k == 3:
        return T, Y * (1 - ulp / 2)
    rng = np.random.default_rng(k)
    sT = rng.choice([-0.5, 1.0], size=T.shape)
    sY = rng.choice([-0.5, 0.0, 1.0], size=Y.shape)
    return T * (1 + sT * ulp), Y * (1 + sY * ulp)


def explain(tables, inp, g, bad, dt, opts, tries=16):
    """The cells of `bad` that the oracle reproduces from a one-ulp
    perturbation of their inputs (within the parity tolerance of the GPU's
    answer); returns the unexplained ones."""
    T, p, rho, Y = (a[..., bad] for a in inp)
    gb = {k: g[k][..., bad] for k in ("T", "rho", "Y")}
    left = np.arange(bad.size)
    for k in range(tries):
        if left.size == 0:
            break
        Tk, Yk = perturbations(T[left], Y[:, left], k)
        o = oracle(tables, Tk, p[left], rho[left], Yk, dt, **opts)
        sub = {key: gb[key][..., left] for key in gb}
        still = bad_cells(sub, {"T": o["T"], "rho": o["rho"], "Y": o["Y"]})
        left = left[still]
    return bad[left]


def check(tables, inp, g, ref, dt, opts, what):
    bad = bad_cells(g, ref)
    n = inp[0].shape[0]
    assert bad.size <= MAX_FLIP_FRACTION * n, f"{what}: {bad.size} of {n} cells outside tolerance"
    unexplained = explain(tables, inp, g, bad, dt, opts) if bad.size else bad
    assert unexplained.size == 0, f"{what}: cells {unexplained.tolist()} outside tolerance, unexplained"
    # the statuses agree where the answers do
    return bad
